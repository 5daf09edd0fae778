"""Batched maps (dtfe_batch_*) and the serving loop (dtfe_server_*).

Every pixel of a map is formed by one block from the pixel's own samples, in
sample order, whatever else the launch holds.  So a map computed in a batch,
or by the serving loop in any mix of other requests, must be bit-identical
to the same map computed alone by dtfe_map, in both precisions; and the
per-map counters (rays, tets crossed, statuses) must agree exactly.
"""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sd():
    import sdtfe_b200

    return sdtfe_b200


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def cutouts(sd):
    """Five halo cutouts of uneven size (float32 positions)."""
    from sdtfe_b200 import workloads

    meshes = []
    for i, n in enumerate((3000, 9000, 20000, 5000, 14000)):
        pos4 = workloads.halo_cutout(n, 700 + i)
        meshes.append(sd.Mesh(pos4, sd.triangulate(pos4), 1.0))
    yield meshes
    for m in meshes:
        m.close()


def _params(sd, G, S, axis, precision, seed):
    return sd.map_params(G, 2.0, 2.0, (0.0, 0.0, 0.0), S, 0.0, seed, axis=axis,
                         precision=precision)


# (mesh, side, samples, axis): uneven sides and samples, every axis, one mesh twice
JOBS = [(0, 64, 8, 0), (1, 96, 4, 1), (2, 128, 16, 2), (3, 40, 5, 0), (4, 80, 8, 1),
        (2, 72, 3, 0)]


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("flags", [0, 1 | 2])
def test_batch_matches_single_maps(sd, torch_cuda, cutouts, precision, flags):
    torch = torch_cuda
    params = [_params(sd, G, S, ax, precision, 900 + k) for k, (_, G, S, ax) in enumerate(JOBS)]
    want, want_st = [], []
    for (mi, *_), p in zip(JOBS, params):
        m, st = cutouts[mi].map(p)
        want.append(m)
        want_st.append(st)
    d_maps = [torch.zeros(p.grid_dim * p.grid_dim, dtype=torch.float64, device="cuda")
              for p in params]
    b = sd.Batch([(cutouts[mi], p, d.data_ptr()) for (mi, *_), p, d in zip(JOBS, params, d_maps)],
                 flags)
    info = b.info()
    assert info["grid"] >= 148 and info["tiles"] > 0
    for rep in range(2):  # a second launch accumulates, unless the batch zeroes its maps
        b.launch()
        b.sync()
        for k, (d, w) in enumerate(zip(d_maps, want)):
            got = d.cpu().numpy().reshape(w.shape)
            expect = w if (flags & 2 or rep == 0) else 2 * w
            assert np.array_equal(got, expect), (k, rep)
        for st, ws in zip(b.stats(), want_st):
            assert st.rays == ws.rays and st.visits == ws.visits
            assert list(st.status) == list(ws.status)
            assert st.fp64_fallbacks == ws.fp64_fallbacks
    b.close()


def test_batch_larger_than_one_job_table(sd, torch_cuda, cutouts):
    """A mixed batch of 150 small maps: more jobs than one launch's parameter
    table holds (96), so it runs in chunks, each with its own tile numbering
    and queue; every map equal to dtfe_map, captured in a graph and not."""
    torch = torch_cuda
    rng = np.random.default_rng(31)
    jobs = [(int(rng.integers(len(cutouts))), int(rng.choice([16, 24, 40])),
             int(rng.integers(1, 9)), int(rng.integers(3))) for _ in range(150)]
    params = [_params(sd, G, S, ax, 1, 5000 + k) for k, (_, G, S, ax) in enumerate(jobs)]
    want = [cutouts[mi].map(p)[0] for (mi, *_), p in zip(jobs, params)]
    for flags in (sd.BATCH_ZERO_MAPS, sd.BATCH_GRAPH | sd.BATCH_ZERO_MAPS):
        d_maps = [torch.full((p.grid_dim * p.grid_dim,), 9.0, dtype=torch.float64, device="cuda")
                  for p in params]
        b = sd.Batch([(cutouts[mi], p, d.data_ptr()) for (mi, *_), p, d in
                      zip(jobs, params, d_maps)], flags)
        for _ in range(2):
            b.launch()
            b.sync()
            for k, (d, w) in enumerate(zip(d_maps, want)):
                assert np.array_equal(d.cpu().numpy().reshape(w.shape), w), (flags, k)
        b.close()


def test_batch_autotune_keeps_results(sd, torch_cuda, cutouts):
    torch = torch_cuda
    params = [_params(sd, G, S, ax, 1, 77 + k) for k, (_, G, S, ax) in enumerate(JOBS)]
    d_maps = [torch.zeros(p.grid_dim * p.grid_dim, dtype=torch.float64, device="cuda")
              for p in params]
    b = sd.Batch([(cutouts[mi], p, d.data_ptr()) for (mi, *_), p, d in zip(JOBS, params, d_maps)],
                 sd.BATCH_GRAPH | sd.BATCH_ZERO_MAPS)
    best, table = b.autotune()
    assert 0 <= best < len(table) and all(t["ms"] > 0 for t in table)
    b.launch()
    b.sync()
    for (mi, *_), p, d in zip(JOBS, params, d_maps):
        want, _ = cutouts[mi].map(p)
        assert np.array_equal(d.cpu().numpy().reshape(want.shape), want)
    b.close()


def test_batch_rejects_mixed_precisions(sd, torch_cuda, cutouts):
    torch = torch_cuda
    d = torch.zeros(64 * 64, dtype=torch.float64, device="cuda")
    jobs = [(cutouts[0], _params(sd, 64, 4, 0, 0, 1), d.data_ptr()),
            (cutouts[1], _params(sd, 64, 4, 0, 1, 1), d.data_ptr())]
    with pytest.raises(sd.DTFEError, match="same precision"):
        sd.Batch(jobs)


# --------------------------------------------------------------------------
# serving loop
# --------------------------------------------------------------------------
def _alone(cutouts, mi, p):
    m, st = cutouts[mi].map(p)
    return m, st


def test_server_results_alone_and_in_the_mix(sd, cutouts):
    """The same request served alone, then among many concurrent others of
    both precisions, every axis and uneven sizes: identical maps, and equal to
    dtfe_map."""
    rng = np.random.default_rng(5)
    probe = (2, _params(sd, 96, 8, 1, 1, 4242))
    with sd.Server(quantum_rays=1 << 16) as srv:
        ids = [srv.add_mesh(m) for m in cutouts]
        rid = srv.submit(ids[probe[0]], probe[1])
        alone, info_alone = srv.wait(rid)
        assert info_alone.status == 0 and info_alone.iterations >= 1
        # the mix: 40 other requests, the probe submitted in the middle
        others = []
        for k in range(40):
            mi = int(rng.integers(len(cutouts)))
            p = _params(sd, int(rng.choice([32, 48, 64, 128])), int(rng.integers(2, 9)),
                        int(rng.integers(3)), int(rng.integers(2)), 100 + k)
            others.append((mi, p, srv.submit(ids[mi], p)))
            if k == 20:
                rid_mix = srv.submit(ids[probe[0]], probe[1])
        mixed, info_mix = srv.wait(rid_mix)
        assert info_mix.iterations >= 1
        assert np.array_equal(mixed, alone)
        assert info_mix.stats.visits == info_alone.stats.visits
        want, st = _alone(cutouts, *probe)
        assert np.array_equal(alone, want)
        assert info_alone.stats.visits == st.visits
        for mi, p, r in others:
            got, info = srv.wait(r)
            want, st = _alone(cutouts, mi, p)
            assert np.array_equal(got, want)
            assert info.stats.rays == st.rays and info.stats.visits == st.visits
            assert info.latency_ms >= info.queue_ms >= 0
        s = srv.stats()
        assert s.completed == 42 and s.failed == 0 and s.active == 0 and s.queued == 0
        assert s.iterations >= 2


def test_server_concurrent_submitters(sd, cutouts):
    """Requests submitted from several host threads at once."""
    results = {}

    def worker(t, srv, ids):
        for k in range(6):
            mi = (t + k) % len(cutouts)
            p = _params(sd, 48, 4, k % 3, (t + k) % 2, 1000 * t + k)
            rid = srv.submit(ids[mi], p)
            results[(t, k)] = (mi, p, rid)

    with sd.Server(quantum_rays=1 << 15, policy=sd.SERVE_FIFO) as srv:
        ids = [srv.add_mesh(m) for m in cutouts]
        th = [threading.Thread(target=worker, args=(t, srv, ids)) for t in range(4)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        for (t, k), (mi, p, rid) in sorted(results.items()):
            got, _ = srv.wait(rid)
            want, _ = _alone(cutouts, mi, p)
            assert np.array_equal(got, want), (t, k)


def test_server_admission_and_eviction(sd, cutouts):
    """A small budget forces walk records out (least recently used first);
    results stay exact.  A request that cannot fit even alone is refused."""
    nt = max(m.info().n_tetra for m in cutouts)
    # room for one mesh's records on one axis (mixed: 4 x 80 B per tet, one
    # record per entry face; FP64: 160 B), plus a few maps
    budget = nt * (320 + 160) + 4 * 8 * 128 * 128
    with sd.Server(device_budget=budget, quantum_rays=1 << 15) as srv:
        ids = [srv.add_mesh(m) for m in cutouts]
        reqs = []
        for k in range(12):
            mi = k % len(cutouts)
            p = _params(sd, 64, 4, k % 3, 1, 50 + k)
            reqs.append((mi, p, srv.submit(ids[mi], p)))
        for mi, p, rid in reqs:
            got, _ = srv.wait(rid)
            want, _ = _alone(cutouts, mi, p)
            assert np.array_equal(got, want)
        s = srv.stats()
        assert s.evictions > 0 and s.peak <= budget
        big = _params(sd, 4096, 1, 0, 1, 1)  # a 128 MiB map alone exceeds the budget
        rid = srv.submit(ids[0], big)
        with pytest.raises(sd.DTFEError) as e:
            srv.wait(rid)
        assert e.value.status == sd.ERR_ADMISSION


def test_server_wait_timeout_and_invalid(sd, cutouts):
    with sd.Server() as srv:
        mid = srv.add_mesh(cutouts[2])
        rid = srv.submit(mid, _params(sd, 1024, 16, 0, 0, 3))
        try:
            srv.wait(rid, timeout_ms=0)
            finished_early = True
        except sd.DTFEError as e:
            assert e.status == sd.ERR_TIMEOUT
            finished_early = False
        if not finished_early:
            got, info = srv.wait(rid)
            assert info.status == 0
        with pytest.raises(sd.DTFEError):
            srv.wait(rid)  # already collected
        with pytest.raises(sd.DTFEError):
            srv.submit(99, _params(sd, 16, 1, 0, 0, 1))
        with pytest.raises(sd.DTFEError):
            srv.submit(mid, _params(sd, 0, 1, 0, 0, 1))
