"""dtfe_density_noalloc: the density build for callers that cannot allocate
device memory mid-run (code inside a framework's memory pool, serving loops
that cannot afford cudaMalloc's device-wide synchronisation).  It keeps its
temporaries in one static device array, so it is checked here against the
allocating entry point on two calls in a row (the array keeps the previous
call's contents), on two different meshes, and for the size limit.

This file is collected last on purpose: if it fails, every other test has
already run.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden_set

pytestmark = pytest.mark.gpu


def _noalloc():
    import sdtfe_b200

    L = sdtfe_b200.lib()
    f = L.dtfe_density_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_float,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return L, f


def _device_density(f, pos4, tetra, p_mass):
    import torch

    d_pos = torch.from_numpy(np.ascontiguousarray(pos4)).cuda()
    d_tet = torch.from_numpy(np.ascontiguousarray(tetra)).cuda()
    d_rho = torch.full((len(pos4),), -7.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = f(d_pos.data_ptr(), len(pos4), d_tet.data_ptr(), len(tetra), p_mass, d_rho.data_ptr(), None)
    return st, d_rho.cpu().numpy()


def test_noalloc_density_matches_allocating_entry(golden):
    import sdtfe_b200 as sd

    L, f = _noalloc()
    a = golden_set(golden, "clustered")
    b = golden_set(golden, "uniform")
    with sd.Mesh(a["pos4"], a["tetra"], 1.0) as ma, sd.Mesh(b["pos4"], b["tetra"], 0.25) as mb:
        want_a, want_b = ma.density(), mb.density()
    assert np.array_equal(want_a, a["density"])  # the reference's own densities
    for pos4, tetra, p_mass, want in ((a["pos4"], a["tetra"], 1.0, want_a),
                                      (a["pos4"], a["tetra"], 1.0, want_a),
                                      (b["pos4"], b["tetra"], 0.25, want_b),
                                      (a["pos4"], a["tetra"], 1.0, want_a)):
        st, got = _device_density(f, pos4, tetra, p_mass)
        assert st == 0, L.dtfe_last_error()
        assert np.array_equal(got, want)


def test_noalloc_rejects_sizes_beyond_the_static_scratch():
    import torch

    L, f = _noalloc()
    # a tet count far beyond the scratch: rejected before anything runs
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = f(d.data_ptr(), 1, d.data_ptr(), 50_000_000, 1.0, d.data_ptr(), None)
    assert st == 5  # DTFE_ERR_UNSUPPORTED
    assert b"scratch" in L.dtfe_last_error()


def test_noalloc_orders_its_work_after_the_callers_stream(golden):
    """Inputs uploaded and the output filled on a caller's own stream, behind
    a slow kernel and with no host synchronisation: the call must run after
    that work, on that stream, and still return the allocating entry's
    densities."""
    import torch

    import sdtfe_b200 as sd

    L, f = _noalloc()
    a = golden_set(golden, "clustered")
    with sd.Mesh(a["pos4"], a["tetra"], 1.0) as ma:
        want = ma.density()
    assert f(None, 0, None, 0, 0.0, None, None) == 0  # the start-up (set-up only) call
    h_pos = torch.from_numpy(np.ascontiguousarray(a["pos4"])).pin_memory()
    h_tet = torch.from_numpy(np.ascontiguousarray(a["tetra"])).pin_memory()
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        d_pos = torch.empty(h_pos.shape, dtype=torch.float64, device="cuda")
        d_tet = torch.empty(h_tet.shape, dtype=torch.int32, device="cuda")
        d_rho = torch.empty(len(want), dtype=torch.float64, device="cuda")
        torch.cuda._sleep(50_000_000)  # the uploads below land well after the call is made
        d_pos.copy_(h_pos, non_blocking=True)
        d_tet.copy_(h_tet, non_blocking=True)
        d_rho.fill_(-7.0)
        st = f(d_pos.data_ptr(), len(want), d_tet.data_ptr(), len(a["tetra"]), 1.0,
               d_rho.data_ptr(), side.cuda_stream)
        assert st == 0, L.dtfe_last_error()
        got = d_rho.cpu().numpy()
    assert np.array_equal(got, want)
