"""Mesh lifetimes over the library's stream-ordered memory pool.

A mesh's arrays come from a pool that keeps freed memory for the next mesh
(dtfe_mesh_create / dtfe_mesh_destroy).  Meshes created, used on a caller's
stream and destroyed in turn, overlapping one another, must give the same
maps every time.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sd():
    import sdtfe_b200

    return sdtfe_b200


@pytest.fixture(scope="module")
def mesh_input(sd):
    from sdtfe_b200 import workloads

    pos4, _ = workloads.clustered_box(n=20000, seed=7, n_clusters=6, r_max=0.05)
    return pos4, sd.triangulate(pos4)


def test_meshes_created_and_destroyed_in_turn(sd, mesh_input):
    import torch

    pos4, tetra = mesh_input
    G = 96
    stream = torch.cuda.Stream()
    d_map = torch.zeros(G * G, dtype=torch.float64, device="cuda")
    want = {}
    with sd.Mesh(pos4, tetra, 1.0) as m:
        for prec in (sd.DTFE_FP64, sd.DTFE_MIXED):
            want[prec], _ = m.map(sd.map_params(G, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, 3,
                                                precision=prec))
    prev = None
    for k in range(6):
        m = sd.Mesh(pos4, tetra, 1.0)
        prec = sd.DTFE_MIXED if k % 2 else sd.DTFE_FP64
        with torch.cuda.stream(stream):
            d_map.zero_()
        m.map_device(sd.map_params(G, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, 3, precision=prec),
                     d_map.data_ptr(), stream.cuda_stream)
        stream.synchronize()
        assert np.array_equal(d_map.cpu().numpy().reshape(G, G), want[prec])
        if prev is not None:  # the older mesh goes while this one lives on
            prev.close()
        got, _ = m.map(sd.map_params(G, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, 3, precision=prec))
        assert np.array_equal(got, want[prec])
        prev = m
    prev.close()


def test_drop_in_calls_in_a_row(sd, mesh_input):
    """compute_density creates and destroys its own mesh per call; repeated
    calls give the same map and densities."""
    pos4, tetra = mesh_input
    L = sd.lib()
    L.dtfe_set_seed(11)
    try:
        outs = []
        for _ in range(3):
            pd = pos4.copy()
            rho = np.zeros(64 * 64)
            L.compute_density(pd, len(pd), tetra, len(tetra), 64, 1.0, 1.0, rho, 1.0, 0.5, 0.5,
                              0.5, 2, 0.0)
            outs.append((rho, pd[:, 3].copy()))
        for rho, dens in outs[1:]:
            assert np.array_equal(rho, outs[0][0])
            assert np.array_equal(dens, outs[0][1])
        assert (outs[0][1] > 0).all()
    finally:
        L.dtfe_set_seed(0)


def test_trim_returns_the_pools_memory(sd, mesh_input):
    import torch

    pos4, tetra = mesh_input
    meshes = [sd.Mesh(pos4, tetra, 1.0) for _ in range(4)]
    for m in meshes:
        m.map(sd.map_params(64, 1.0, 1.0, (0.5, 0.5, 0.5), 2, 0.0, 5, precision=sd.DTFE_MIXED))
    for m in meshes:
        m.close()
    free_before, _ = torch.cuda.mem_get_info()
    sd.trim_memory()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after >= free_before
    with sd.Mesh(pos4, tetra, 1.0) as m:  # the pool refills on the next mesh
        got, st = m.map(sd.map_params(64, 1.0, 1.0, (0.5, 0.5, 0.5), 2, 0.0, 5))
        assert st.rays == 64 * 64 * 2 and got.sum() > 0
