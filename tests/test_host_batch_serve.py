"""Host-side checks of the batch and serving APIs: argument validation and
status reporting, which return before any CUDA call, and a clean error (no
crash) where a call needs a device and none is present."""
import ctypes

import pytest


@pytest.fixture(scope="module")
def L():
    from sdtfe_b200 import lib

    return lib()


def _cuda_present():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def test_status_strings(L):
    L.dtfe_status_string.restype = ctypes.c_char_p
    L.dtfe_status_string.argtypes = [ctypes.c_int]
    assert L.dtfe_status_string(7) == b"admission refused"
    assert L.dtfe_status_string(8) == b"timed out"
    assert L.dtfe_status_string(99) == b"unknown"


def test_batch_argument_errors(L):
    from sdtfe_b200._lib import BatchJob

    out = ctypes.c_void_p()
    assert L.dtfe_batch_create(None, 0, 0, ctypes.byref(out)) == 1
    assert not out.value
    jobs = (BatchJob * 1)()  # NULL mesh and map
    assert L.dtfe_batch_create(jobs, 1, 0, ctypes.byref(out)) == 1
    assert b"NULL mesh" in L.dtfe_last_error()
    assert L.dtfe_batch_create(jobs, 1, 0, None) == 1
    assert L.dtfe_batch_launch(None, None) == 1
    assert L.dtfe_batch_sync(None) == 1
    assert L.dtfe_batch_stats(None, None) == 1
    assert L.dtfe_batch_destroy(None) == 0


def test_server_argument_errors(L):
    from sdtfe_b200._lib import MapParams, RequestInfo, ServerStats

    assert L.dtfe_server_create(None, None) == 1
    assert L.dtfe_server_add_mesh(None, None, None) == 1
    rid = ctypes.c_uint64()
    p = MapParams()
    assert L.dtfe_server_submit(None, 0, ctypes.byref(p), None, ctypes.byref(rid)) == 1
    assert L.dtfe_server_wait(None, 1, 0, ctypes.byref(RequestInfo())) == 1
    assert L.dtfe_server_stats(None, ctypes.byref(ServerStats())) == 1
    assert L.dtfe_server_destroy(None) == 0


@pytest.mark.skipif(_cuda_present(), reason="checks the no-device error path")
def test_server_without_device_fails_cleanly(L):
    from sdtfe_b200 import DTFEError, Server

    with pytest.raises(DTFEError) as e:
        Server()
    assert e.value.status in (2, 3)  # a CUDA error, reported, not a crash
