"""Benchmark: Monte Carlo line-of-sight surface-density maps on B200.

Workload (default): the clustered single map - 1,048,576 float32 particles,
half uniform in the unit box and half in 100 r^-2 clusters (truncation 0.02),
Qhull Delaunay on the host, a 2048 x 2048 z-projection of the whole box with
16 Monte Carlo samples per pixel (67,108,864 rays per map).  Synthetic and
seeded (sdtfe_b200.workloads.clustered_box).

One step = one full map of that workload through the device-resident mesh
(tet records in HBM before the timed region; the map buffer is zeroed at the
start of the step, as callers of compute_density do).  Reported:

  value         rays/s of the product path (mixed precision unless --precision
                fp64), device-timed with CUDA events on the launching stream,
                L2 flushed between steps (inputs are also larger than L2)
  e2e           rays/s through the reference-facing drop-in compute_density()
                with pinned host buffers: every step uploads particle_data and
                tetra_data, builds densities/gradients/hull on the GPU, walks,
                and downloads the map and the densities
  fp64          rays/s of the plain FP64 path (the reference's arithmetic) on
                the same map, and the mixed map's max/RMS relative error
                against it
  roofline      the walk kernel's algorithmic bytes (tet visits x bytes per
                visit) over its event-timed duration, against the measured HBM
                copy bandwidth
  cpu_baseline  the reference's own compute_density (its C, built from its
                sources into oracle/_ref, OpenMP on all host cores) on a
                sub-window of the same map with the same pixel size

Sections (N=1; --sections none skips them), host Qhull for all of them in a
spawn process pool before CUDA starts:

  batch         64 halo cutouts (N log-uniform in [1e4, 5e5]), one map each
                (sides 256/512/1024, 8 samples/pixel) in one persistent launch
                captured in a CUDA graph, autotuned; against one launch per
                map and against the FP64 batch (speed-up, max/RMS error)
  serving       map requests (random cutout, axis, side 128..2048, 4-16
                samples/pixel) through the serving loop over --serve-handles
                resident cutouts: closed-loop capacity in rays/s, then Poisson
                arrivals at --serve-load of that capacity, p50/p99 latency,
                mixed vs FP64 and the mixed maps' error

--impl reference runs only the reference's CPU implementation (same metric).
Multi-GPU (torchrun, --gpus N): replicas; each rank maps its own copy of the
workload, value = all ranks' rays / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_VISIT = {"mixed": 96, "fp64": 160}  # tet record bytes read per walk step


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--workload", default="clustered",
                    choices=["clustered", "uniform", "clustered_262k"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--sections", default="plain_small,batch,serving,large_field",
                    help="extra sections on one GPU: batch (64 cutouts in one persistent launch), "
                         "serving (request stream with continuous batching); 'none' to skip")
    ap.add_argument("--large-side", type=int, default=192,
                    help="lattice side of the large field (192: the 9.2M-point configuration; "
                         "smaller sides make profiling cases of the same recipe)")
    ap.add_argument("--serve-handles", type=int, default=256)
    ap.add_argument("--serve-distinct", type=int, default=256,
                    help="distinct cutout triangulations behind the handles (default: one per handle)")
    ap.add_argument("--serve-requests", type=int, default=200)
    ap.add_argument("--serve-load", type=float, default=0.7,
                    help="Poisson arrival rate as a fraction of the measured mixed capacity")
    ap.add_argument("--serve-quantum", type=int, default=0,
                    help="rays per serving iteration (0: the library default)")
    return ap.parse_args()


def workloads_module():
    """sdtfe_b200/workloads.py (pure numpy), loaded by path so that the
    reference arm never imports the sdtfe_b200 package."""
    import importlib.util

    if "sdtfe_workloads" not in sys.modules:
        spec = importlib.util.spec_from_file_location(
            "sdtfe_workloads", os.path.join(ROOT, "sdtfe_b200", "workloads.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules["sdtfe_workloads"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["sdtfe_workloads"]


def workload(name):
    W = workloads_module()
    if name == "uniform":
        pos4, spec = W.uniform_box()
        desc = "uniform_32k_256x4"
    elif name == "clustered_262k":  # the profiling case: same recipe, a quarter of the points
        pos4, spec = W.clustered_box(n=1 << 18, grid_dim=1024)
        desc = "clustered_262k_1024x16"
    else:
        pos4, spec = W.clustered_box()
        desc = "clustered_1M_2048x16"
    return desc, pos4, spec


def _qhull_task(task):
    """One host triangulation (spawned worker): builds the particle set from
    its generator and seed, then Qhull + the library's layout step."""
    kind, key, n, seed = task
    import sdtfe_b200 as sd
    from sdtfe_b200 import workloads as W

    if kind == "main":
        pos4 = workload(key)[1]
    elif kind == "cutout":
        pos4 = W.halo_cutout(n, seed)
    elif kind == "large":  # seed slot: the lattice's side
        pos4 = W.perturbed_lattice(n_side=seed)
    else:  # "clustered": the clustered-box recipe at n particles
        pos4 = W.clustered_box(n=n, seed=seed)[0]
    t = time.perf_counter()
    tetra = sd.triangulate(pos4)
    return kind, key, pos4, tetra, time.perf_counter() - t


class QhullPool:
    """Host Qhull for every workload of the run in a spawn process pool, the
    main workload first, then the largest: sections that need a
    triangulation wait for it (get), so GPU work on the ones already done
    overlaps the rest."""

    def __init__(self, tasks):
        import multiprocessing as mp

        # one worker per core, as memory allows: Qhull takes about 3 GB per
        # million points, and the largest tasks (up to 9.2M points) run first
        try:
            import psutil

            avail_gb = psutil.virtual_memory().available / 2**30
        except ImportError:
            avail_gb = 256.0
        by_mem = max(1, int((avail_gb - 40.0) // 8.0))
        self.procs = max(1, min(len(tasks), len(os.sched_getaffinity(0)), 32, by_mem))
        order = tasks[:1] + sorted(tasks[1:], key=lambda t: -t[2])
        self.t0 = time.perf_counter()
        self.pool = mp.get_context("spawn").Pool(self.procs)
        self.pending = {(t[0], t[1]): self.pool.apply_async(_qhull_task, (t,)) for t in order}
        self.done, self.cpu_s, self.wall_s = {}, 0.0, None

    def get(self, kind, key):
        if (kind, key) not in self.done:
            _, _, pos4, tetra, dt = self.pending.pop((kind, key)).get()
            self.done[(kind, key)] = (pos4, tetra, dt)
            self.cpu_s += dt
        return self.done[(kind, key)]

    def drop(self, kind, key):
        self.done.pop((kind, key), None)

    def wait_all(self):
        """Every triangulation finished and the pool closed (host cores idle)."""
        for kind, key in list(self.pending):
            self.get(kind, key)
        if self.wall_s is None:
            self.wall_s = time.perf_counter() - self.t0
            self.pool.close()
            self.pool.join()

    def info(self):
        return {"procs": self.procs, "wall_s": round(self.wall_s or 0.0, 1),
                "cpu_s": round(self.cpu_s, 1)}


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # a short timed region may end before the first 200 ms sample:
            # start timing once nvidia-smi is reporting (at most 2 s)
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 2.0:
                time.sleep(0.01)
            self.first = len(self.lines)  # samples from here on fall in the timed region
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines[getattr(self, "first", 0):] or self.lines[-1:]
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


# ---------------------------------------------------------------------------
# the reference's CPU implementation
# ---------------------------------------------------------------------------
class RefCPU:
    """The reference's compute_density (its own C, oracle/_ref/libdtfe_ref.so),
    its OpenMP team set to every core this process may run on; `cores` is the
    team size the reference's OpenMP runtime reports."""

    def __init__(self):
        from oracle.oracle import Reference

        self.R = Reference(stock_only=True)
        self.cores = self.R.set_threads(len(os.sched_getaffinity(0)))

    def _quiet(self, fn):
        # the reference prints one stderr line per failed ray; send them to /dev/null
        sys.stderr.flush()
        saved = os.dup(2)
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 2)
        try:
            return fn()
        finally:
            os.dup2(saved, 2)
            os.close(devnull)
            os.close(saved)

    def window_run(self, pos4, tetra, spec, gw):
        """compute_density over a gw x gw window at the map's pixel size, centred
        on the map centre.  Returns seconds."""
        dxy = spec.box_len / spec.grid_dim
        rho = np.zeros(gw * gw)
        pd = pos4.copy()
        t = time.perf_counter()
        self._quiet(lambda: self.R.compute_density(pd, tetra, gw, gw * dxy, spec.box_len_z, rho,
                                                   1.0, spec.center, spec.n_samples, 0.0))
        return time.perf_counter() - t

    def calibrate(self, pos4, tetra, spec, seconds):
        """Precompute time (a 4 x 4 window: one tile, negligible walk) and a
        window side whose walk takes about `seconds`."""
        self.t_pre = min(self.window_run(pos4, tetra, spec, 4) for _ in range(2))
        gw = 64
        t = self.window_run(pos4, tetra, spec, gw)
        per_px = max(t - self.t_pre, 1e-6) / (gw * gw)
        gw = int(np.sqrt(seconds / per_px))
        self.gw = int(min(max(16, gw - gw % 16), spec.grid_dim))

    def step(self, pos4, tetra, spec):
        """Amortised full-map rays/s from one window: the measured precompute
        plus the window's walk time per ray times the map's rays.  Returns
        (rays_per_s, sample_description)."""
        t = self.window_run(pos4, tetra, spec, self.gw)
        rays_w = self.gw * self.gw * spec.n_samples
        walk = max(t - self.t_pre, 1e-9)
        full = self.t_pre + walk / rays_w * spec.rays
        sample = (f"compute_density on a {self.gw}x{self.gw}-pixel window at the map's pixel "
                  f"size ({rays_w} rays, {t:.2f} s incl. {self.t_pre:.2f} s single-threaded "
                  f"precompute); full-map time = precompute + walk/ray x {spec.rays} rays")
        return spec.rays / full, sample


def workload_config(desc, n_particles, n_tets, spec, world):
    """The `config` object of both arms' lines (identical for the same run)."""
    return {"workload": desc, "particles": int(n_particles), "tets": int(n_tets),
            "grid_dim": spec.grid_dim, "samples_per_pixel": spec.n_samples,
            "rays_per_map": spec.rays, "parallelism": f"replicas x{world}",
            "l2": f"tet records {n_tets * 320 / 1e6:.0f} MB (mixed walk, 320 B per tet) "
                  f"{'>' if n_tets * 320 > 126e6 else '<'} the 126 MB L2; the GPU arm flushes "
                  "L2 between steps (256 MiB write)"}


def run_reference(args):
    """The reference's own CPU code only: the sdtfe_b200 package is not
    imported in this process (Qhull through SciPy, the reference's tetra_data
    layout restated in numpy by oracle.oracle.delaunay_tetra)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.oracle import delaunay_tetra

    desc, pos4, spec = workload(args.workload)
    t = time.perf_counter()
    tetra = delaunay_tetra(pos4)
    t_qhull = time.perf_counter() - t
    ref = RefCPU()
    ref.calibrate(pos4, tetra, spec, args.cpu_seconds / 3)
    for _ in range(args.warmup):
        ref.step(pos4, tetra, spec)
    vals, samples = [], []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        v, sample = ref.step(pos4, tetra, spec)
        vals.append(v)
        samples.append(sample)
    wall = time.perf_counter() - t0
    value = float(np.median(vals))
    line = {
        "impl": "reference", "metric": "los_rays_per_s", "value": value, "unit": "rays/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": workload_config(desc, len(pos4), len(tetra), spec, args.gpus),
        "qhull_host_s": round(t_qhull, 2),
        "cpu_baseline": {"value": value, "unit": "rays/s", "cores": ref.cores,
                         "kind": "reference", "sample": samples[-1]},
        "e2e": {"value": value, "unit": "rays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def read_profile(kernel):
    """The committed ncu figures of `kernel` (profiles/roofline.json): the
    captured workload's tets and tet visits, and per launch its warp
    instructions, threads per warp instruction, DRAM bytes and cache hit
    rates."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "roofline.json")))[kernel]
    except (OSError, KeyError, ValueError):
        return None


def roofline(kernel, visits, n_tets, bytes_per_visit, kern_ms, sm_mhz, n_sm, hbm_peak, hbm_note):
    """The walk kernel against its bound, instruction issue: each SM issues at
    most one warp instruction per scheduler (4) per cycle, so the peak is
    SMs x 4 x the SM clock sampled during the timed region.  achieved = this
    launch's tet visits x the warp instructions per visit that ncu counted on
    the profiled workload, over the event-timed duration.  DRAM traffic is the
    profile's bytes per tet (each tet's records are read from DRAM about once
    per map), scaled to this mesh; the algorithmic bytes (96 B per mixed
    visit) are mostly served from L1/L2, and are reported beside it."""
    t = kern_ms / 1e3
    alg_gbs = visits * bytes_per_visit / t / 1e9
    prof = read_profile(kernel)
    if not prof:  # no committed profile: the algorithmic-bytes figure alone
        return {"bound": "hbm", "achieved": alg_gbs, "peak": hbm_peak, "unit": "GB/s",
                "frac": alg_gbs / hbm_peak, "traffic": None, "kernel": kernel,
                "note": f"peak {hbm_note}; no ncu profile committed for {kernel}"}
    wipv = prof["warp_inst"] / prof["visits"]
    achieved = visits * wipv / t
    peak = n_sm * 4 * sm_mhz * 1e6
    traffic = prof["dram_bytes"] / prof["tets"] * n_tets
    return {"bound": "issue", "achieved": achieved / 1e9, "peak": peak / 1e9,
            "unit": "G warp-instructions/s", "frac": achieved / peak, "traffic": traffic,
            "kernel": kernel, "warp_inst_per_visit": wipv,
            "threads_per_warp_inst": prof.get("threads_per_warp_inst"),
            "issue_active_pct_profiled": prof.get("issue_active_pct"),
            "dram_gbs": traffic / t / 1e9, "dram_frac": traffic / t / 1e9 / hbm_peak,
            "hbm_peak_gbs": hbm_peak, "hbm_peak_note": hbm_note,
            "l1_hit_pct": prof.get("l1_hit_pct"), "l2_hit_pct": prof.get("l2_hit_pct"),
            "algorithmic_gbs": alg_gbs, "bytes_per_visit": bytes_per_visit,
            "sm_mhz": sm_mhz, "sms": n_sm, "profile": prof.get("source"),
            "note": "peak = SMs x 4 schedulers x sampled SM clock; warp instructions per visit "
                    "and DRAM bytes per tet from the committed ncu capture"}


def slowest_rank_ms(total_ms, dist, device):
    """The job's device time over replicas: the slowest rank's (max over ranks;
    every rank calls this, in the same order)."""
    if dist is None:
        return total_ms
    import torch

    tt = torch.tensor([total_ms], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def replica_rays_per_s(rays_per_map, steps, world, total_ms):
    """Whole-job rays/s: every rank maps its own copy of the workload."""
    return rays_per_map * steps * world / (total_ms / 1e3)


def plan_sections(args):
    """Starts host Qhull for the main workload and the sections (N=1 only) in
    a spawn process pool; returns (pool, sections)."""
    from sdtfe_b200 import workloads as W

    world = int(os.environ.get("WORLD_SIZE", "1"))
    sections = [] if args.sections == "none" or world > 1 else args.sections.split(",")
    if not sections:
        return None
    n_main = {"uniform": 32768, "clustered_262k": 1 << 18}.get(args.workload, 1 << 20)
    tasks = [("main", args.workload, n_main, 0)]
    if "batch" in sections:
        tasks += [("cutout", i, n, seed) for i, (n, seed, _) in enumerate(W.cutout_specs())]
    if "serving" in sections:
        tasks += [("clustered", i, n, seed) for i, (n, seed) in enumerate(serving_cutouts(args))]
    if "large_field" in sections:
        side = args.large_side
        tasks += [("large", 0, side ** 3 + round(0.3 * side ** 3), side)]
    if "plain_small" in sections and args.workload != "uniform":
        tasks += [("main", "uniform", 32768, 0)]
    return QhullPool(tasks), sections


def serving_cutouts(args):
    """(particle count, seed) of the serving stream's resident cutouts: the
    stream's own counts (log-uniform in [1e4, 2e6]) and the clustered-box
    recipe, one distinct cutout per handle unless --serve-distinct is
    smaller (then handle h holds cutout h % distinct)."""
    from sdtfe_b200 import workloads as W

    ns, _ = W.serving_stream(n_cutouts=args.serve_handles, n_requests=args.serve_requests)
    k = min(args.serve_distinct, args.serve_handles)
    return [(int(ns[i]), 4 * 1000 + i) for i in range(k)]


def timed_launches(torch, stream, flush, fn, steps):
    """CUDA-event time (ms) of each of `steps` calls of fn on `stream`, the L2
    flushed before each."""
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    for a, b in ev:
        flush.zero_()
        a.record(stream)
        fn()
        b.record(stream)
    torch.cuda.synchronize()
    return np.array([a.elapsed_time(b) for a, b in ev])


def max_rel(got, want):
    ok = np.abs(want) > 0
    r = np.abs(got - want)[ok] / np.abs(want[ok])
    return float(r.max()) if r.size else 0.0, float(np.sqrt(np.mean(r ** 2))) if r.size else 0.0


def section_batch(args, sd, torch, dev, stream, flush, tri):
    """64 halo cutouts, one map each, in one persistent launch captured in a
    CUDA graph; against the same maps launched one by one, and the FP64
    batch.  Inputs resident; each step zeroes the maps (inside the graph)."""
    from sdtfe_b200 import workloads as W

    specs = W.cutout_specs()
    meshes, p32, p64, d32, d64 = [], [], [], [], []
    for i, (n, seed, sp) in enumerate(specs):
        pos4, tetra, _ = tri.get("cutout", i)
        meshes.append(sd.Mesh(pos4, tetra, 1.0))
        kw = dict(seed=5000 + i)
        p32.append(sd.map_params(sp.grid_dim, sp.box_len, sp.box_len_z, sp.center, sp.n_samples,
                                 precision=sd.DTFE_MIXED, **kw))
        p64.append(sd.map_params(sp.grid_dim, sp.box_len, sp.box_len_z, sp.center, sp.n_samples,
                                 precision=sd.DTFE_FP64, **kw))
        d32.append(torch.zeros(sp.grid_dim ** 2, dtype=torch.float64, device=dev))
        d64.append(torch.zeros(sp.grid_dim ** 2, dtype=torch.float64, device=dev))
    rays = sum(sp.rays for _, _, sp in specs)
    sptr = stream.cuda_stream
    flags = sd.BATCH_GRAPH | sd.BATCH_ZERO_MAPS
    b32 = sd.Batch(list(zip(meshes, p32, [d.data_ptr() for d in d32])), flags)
    best, table = b32.autotune()
    for _ in range(args.warmup):
        b32.launch(sptr)
    torch.cuda.synchronize()
    launches0 = sd.lib().dtfe_kernel_launches()
    ms = timed_launches(torch, stream, flush, lambda: b32.launch(sptr), args.steps)
    launches = sd.lib().dtfe_kernel_launches() - launches0
    st32 = b32.stats()
    info = b32.info()

    def one_by_one():  # the same 64 maps, one launch per map, default kernel variant
        for m, p, d in zip(meshes, p32, d32):
            d.zero_()
            m.map_device(p, d.data_ptr(), sptr)
    one_by_one()
    ms_seq = timed_launches(torch, stream, flush, one_by_one, 2)
    # FP64 batch and the mixed maps' error against it
    b64 = sd.Batch(list(zip(meshes, p64, [d.data_ptr() for d in d64])), flags)
    b64.launch(sptr)
    ms64 = timed_launches(torch, stream, flush, lambda: b64.launch(sptr), 2)
    st64 = b64.stats()
    b32.launch(sptr)
    torch.cuda.synchronize()
    errs = [max_rel(a.cpu().numpy(), b.cpu().numpy()) for a, b in zip(d32, d64)]
    # end to end: the graph launch plus every map to pinned host memory
    host = [torch.empty(d.numel(), dtype=torch.float64).pin_memory() for d in d32]

    def e2e():
        b32.launch(sptr)
        for h, d in zip(host, d32):
            h.copy_(d, non_blocking=True)
    e2e()
    ms_e2e = timed_launches(torch, stream, flush, e2e, 2)
    visits = sum(x.visits for x in st32)
    out = {
        "workload": "64 halo cutouts, N log-uniform [1e4, 5e5] (r^-2 cluster + 20% background), "
                    "sides {256,512,1024}, 8 samples/pixel, one persistent launch in a CUDA graph",
        "particles": int(sum(n for n, _, _ in specs)),
        "tets": int(sum(m.info().n_tetra for m in meshes)),
        "rays_per_step": int(rays),
        "rays_per_s": rays / (np.median(ms) / 1e3),
        "ms_per_step": float(np.median(ms)),
        "maps_per_s": len(specs) / (np.median(ms) / 1e3),
        "one_launch_per_map_rays_per_s": rays / (np.median(ms_seq) / 1e3),
        "fp64_batch_rays_per_s": rays / (np.median(ms64) / 1e3),
        "speedup_mixed_over_fp64": float(np.median(ms64) / np.median(ms)),
        "max_rel_err": max(e[0] for e in errs),
        "rms_rel_err": float(np.sqrt(np.mean([e[1] ** 2 for e in errs]))),
        "visits_equal_fp64": bool(visits == sum(x.visits for x in st64)),
        "visits_per_ray": visits / rays,
        "e2e_rays_per_s": rays / (np.median(ms_e2e) / 1e3),
        "e2e_d2h_bytes_per_step": int(sum(d.numel() * 8 for d in d32)),
        "grid": info["grid"], "block": info["block"], "tiles": info["tiles"],
        "autotune": {"chosen": best, "ms": [round(t["ms"], 3) for t in table]},
        "gpu_launches": int(launches),
    }
    b32.close()
    b64.close()
    for m in meshes:
        m.close()
    return out


def _run_stream(sd, srv, ids, reqs, precision, rate, keep=None, compare=None):
    """Replays `reqs` against the server: open loop at `rate` requests/s
    (inter-arrival times of the trace rescaled), or all at t=0 when rate is
    None.  Returns latency percentiles and the achieved rays/s."""
    t0 = time.perf_counter()
    scale = (len(reqs) / rate) / reqs[-1].t if rate is not None else None
    rids = []
    for k, r in enumerate(reqs):
        if scale is not None:
            due = t0 + r.t * scale
            while True:
                now = time.perf_counter()
                if now >= due:
                    break
                time.sleep(min(due - now, 0.002))
        sp = r.spec
        p = sd.map_params(sp.grid_dim, sp.box_len, sp.box_len_z, sp.center, sp.n_samples,
                          seed=7000 + k, axis=r.axis, precision=precision)
        rids.append(srv.submit(ids[r.cutout], p))
    lat, rays, errs, vis_eq, worst = [], 0, [], True, None
    for k, rid in enumerate(rids):
        m, info = srv.wait(rid)
        lat.append(info.latency_ms)
        rays += info.stats.rays
        if keep is not None:
            keep[k] = (m, info.stats.visits)
        if compare is not None:
            w, wv = compare[k]
            e = max_rel(w, m)  # the mixed map against this FP64 one
            errs.append(e)
            if worst is None or e[0] > worst[0]:
                r = reqs[k]
                worst = (e[0], {"request": k, "cutout": r.cutout, "axis": r.axis,
                                "side": r.spec.grid_dim, "samples": r.spec.n_samples})
            vis_eq = vis_eq and wv == info.stats.visits
    wall = time.perf_counter() - t0
    lat = np.array(lat)
    out = {"requests": len(reqs), "rays": int(rays), "wall_s": round(wall, 3),
           "rays_per_s": rays / wall,
           "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
           "max_ms": float(lat.max())}
    if rate is not None:
        out["rate_per_s"] = rate
    if errs:
        out["max_rel_err_mixed_vs_fp64"] = max(e[0] for e in errs)
        out["rms_rel_err_mixed_vs_fp64"] = float(np.sqrt(np.mean([e[1] ** 2 for e in errs])))
        out["worst_request"] = worst[1]
        out["visits_equal_fp64"] = bool(vis_eq)
    return out


def section_serving(args, sd, torch, tri):
    """Map requests over many resident cutouts through the serving loop:
    closed-loop capacity (all requests at once) and open-loop Poisson arrivals
    at a fraction of the mixed capacity, mixed vs FP64."""
    from sdtfe_b200 import workloads as W

    cut = serving_cutouts(args)
    meshes = []
    for h in range(args.serve_handles):
        pos4, tetra, _ = tri.get("clustered", h % len(cut))
        # no walk records at creation: the serving loop builds what requests need
        meshes.append(sd.Mesh(pos4, tetra, 1.0, sd.MESH_LAZY))
    for h in range(len(cut)):
        tri.drop("clustered", h)  # the meshes keep their own host copies
    _, reqs = W.serving_stream(n_cutouts=args.serve_handles, n_requests=args.serve_requests)
    out = {"workload": f"{args.serve_handles} resident cutouts ({len(cut)} distinct "
                       "clustered-box triangulations, N log-uniform [1e4, 2e6]); "
                       f"{len(reqs)} requests: random cutout, axis, side in "
                       "{128..2048}, 4-16 samples/pixel",
           "particles_resident": int(sum(cut[h % len(cut)][0] for h in range(args.serve_handles))),
           "tets_resident": int(sum(m.info().n_tetra for m in meshes))}
    with sd.Server(quantum_rays=args.serve_quantum) as srv:
        ids = [srv.add_mesh(m) for m in meshes]
        # warm-up: one small request per cutout touches every handle once
        warm = [srv.submit(i, sd.map_params(32, 1.0, 1.0, (0.5, 0.5, 0.5), 1, seed=1,
                                            precision=sd.DTFE_MIXED)) for i in ids]
        for w in warm:
            srv.wait(w)
        keep = {}
        out["capacity_mixed"] = _run_stream(sd, srv, ids, reqs, sd.DTFE_MIXED, None, keep=keep)
        out["capacity_fp64"] = _run_stream(sd, srv, ids, reqs, sd.DTFE_FP64, None, compare=keep)
        keep.clear()
        rate = args.serve_load * len(reqs) / out["capacity_mixed"]["wall_s"]
        out["poisson_mixed"] = _run_stream(sd, srv, ids, reqs, sd.DTFE_MIXED, rate)
        out["poisson_fp64"] = _run_stream(sd, srv, ids, reqs, sd.DTFE_FP64, rate)
        st = srv.stats()
        out["server"] = {"iterations": st.iterations, "evictions": st.evictions,
                         "budget_gb": st.budget / 1e9, "peak_gb": st.peak / 1e9,
                         "completed": st.completed, "failed": st.failed}
    out["speedup_mixed_over_fp64"] = (out["capacity_mixed"]["rays_per_s"] /
                                      out["capacity_fp64"]["rays_per_s"])
    for m in meshes:
        m.close()
    return out


def section_plain_small(args, sd, torch, dev, stream, flush, tri):
    """The plain method at its own, CPU-runnable size: 32,768 uniform float64
    points, a 256^2 map with 4 samples per pixel, FP64 throughout (and the
    mixed path beside it), against the reference's own compute_density over
    the whole map on every host core - no window, no extrapolation."""
    pos4, tetra, t_q = tri.get("main", "uniform")
    spec = workload("uniform")[2]
    mesh = sd.Mesh(pos4, tetra, 1.0)
    sptr = stream.cuda_stream
    d_map = torch.zeros(spec.grid_dim ** 2, dtype=torch.float64, device=dev)
    out = {"workload": "uniform_32k_256x4 (32,768 uniform float64 points, 256^2 x 4, FP64)",
           "particles": len(pos4), "tets": len(tetra), "rays": spec.rays}
    maps = {}
    for name, prec in (("fp64", sd.DTFE_FP64), ("mixed", sd.DTFE_MIXED)):
        p = sd.map_params(spec.grid_dim, spec.box_len, spec.box_len_z, spec.center,
                          spec.n_samples, 0.0, 4242, precision=prec)

        def one(p=p):
            d_map.zero_()
            mesh.map_device(p, d_map.data_ptr(), sptr)
        one()
        ms = float(np.median(timed_launches(torch, stream, flush, one, max(args.steps, 3))))
        st = mesh.last_stats()
        maps[name] = d_map.cpu().numpy().copy()
        out[name] = {"ms_per_map": ms, "rays_per_s": spec.rays / (ms / 1e3),
                     "visits_per_ray": st.visits / spec.rays}
    e_max, e_rms = max_rel(maps["mixed"], maps["fp64"])
    out["mixed"].update(max_rel_err=e_max, rms_rel_err=e_rms,
                        speedup_over_fp64=out["fp64"]["ms_per_map"] / out["mixed"]["ms_per_map"])
    out["fp64"]["mass_rel_diff"] = float(maps["fp64"].sum() / spec.grid_dim ** 2 / len(pos4) - 1)
    mesh.close()
    try:  # the reference's compute_density, whole map, all host cores
        ref = RefCPU()
        rho = np.zeros(spec.grid_dim ** 2)
        ts = []
        for _ in range(3):
            rho[:] = 0.0
            pd = pos4.copy()
            t = time.perf_counter()
            ref._quiet(lambda: ref.R.compute_density(pd, tetra, spec.grid_dim, spec.box_len,
                                                     spec.box_len_z, rho, 1.0, spec.center,
                                                     spec.n_samples, 0.0))
            ts.append(time.perf_counter() - t)
        t = float(np.median(ts))
        out["reference_cpu"] = {"s_per_map": t, "rays_per_s": spec.rays / t, "cores": ref.cores,
                                "mass_rel_diff": float(rho.sum() / spec.grid_dim ** 2 /
                                                       len(pos4) - 1)}
        out["fp64"]["speedup_over_reference_cpu"] = t / (out["fp64"]["ms_per_map"] / 1e3)
    except Exception as e:
        out["reference_cpu"] = {"unavailable": f"{type(e).__name__}: {e}"}
    return out


def section_large_field(args, sd, torch, dev, stream, flush, tri):
    """The large field: a 192^3 perturbed lattice (--large-side) plus 30% of its count in
    2,000 r^-2 clusters (float32), one 8192^2 x 4 z-projection and one 512^3
    grid (supersampling 1, the reference's column walk), mixed against FP64:
    device time, crossings, max/RMS relative error, projected mass."""
    pos4, tetra, t_q = tri.get("large", 0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mesh = sd.Mesh(pos4, tetra, 1.0, sd.MESH_LAZY)  # upload, densities (CSR), gradients
    t_build = time.perf_counter() - t0
    tri.drop("large", 0)
    info = mesh.info()
    sptr = stream.cuda_stream
    out = {"workload": f"{args.large_side}^3 lattice (sigma 0.3 spacing) + 30% in 2000 r^-2 "
                       "clusters (r 0.01), "
                       "float32; 8192^2 x 4 map and 512^3 grid (ss 1), mixed vs FP64",
           "particles": int(len(pos4)), "tets": int(info.n_tetra), "qhull_host_s": round(t_q, 1),
           "mesh_create_s": round(t_build, 3),
           "adjacency_max": int(mesh.adjacency().max())}
    G, S = 8192, 4
    kw = dict(grid_dim=G, box_len=1.0, box_len_z=1.0, center=(0.5, 0.5, 0.5), n_samples=S,
              seed=909)
    d_map = torch.zeros(G * G, dtype=torch.float64, device=dev)
    res = {}
    for name, prec, reps in (("mixed", sd.DTFE_MIXED, 2), ("fp64", sd.DTFE_FP64, 1)):
        p = sd.map_params(**kw, precision=prec)

        def one(p=p):
            d_map.zero_()
            mesh.map_device(p, d_map.data_ptr(), sptr)
        one()  # builds the records, warms up
        ms = timed_launches(torch, stream, flush, one, reps)
        st = mesh.last_stats()
        res[name] = (float(np.median(ms)), st, d_map.cpu().numpy())
    # FP64 again with one shared location walk per pixel tile: the large
    # projected hull is where the reference's per-ray walk from triangle 0
    # costs the most
    mesh.set_location(sd.LOCATE_TILE)
    p = sd.map_params(**kw, precision=sd.DTFE_FP64)

    def one_tile(p=p):
        d_map.zero_()
        mesh.map_device(p, d_map.data_ptr(), sptr)
    ms_tile = float(np.median(timed_launches(torch, stream, flush, one_tile, 1)))
    st_tile = mesh.last_stats()
    tile_equal = bool(np.array_equal(d_map.cpu().numpy(), res["fp64"][2]))
    mesh.set_location(sd.LOCATE_PER_RAY)
    rays = G * G * S
    (m32, s32, a32), (m64, s64, a64) = res["mixed"], res["fp64"]
    e_max, e_rms = max_rel(a32, a64)
    out["map"] = {"rays": rays, "mixed_ms": m32, "fp64_ms": m64,
                  "mixed_rays_per_s": rays / (m32 / 1e3), "fp64_rays_per_s": rays / (m64 / 1e3),
                  "speedup_mixed_over_fp64": m64 / m32, "visits_per_ray": s32.visits / rays,
                  "visits_equal_fp64": bool(s32.visits == s64.visits),
                  "status_equal_fp64": list(s32.status) == list(s64.status),
                  "fp64_fallbacks": s32.fp64_fallbacks,
                  "max_rel_err": e_max, "rms_rel_err": e_rms,
                  "mass_rel_diff": float(a32.sum() / G / G / len(pos4) - 1.0),
                  "hull_triangles": int(mesh.info().n_hull_tri[0]),
                  "fp64_tile_location": {
                      "ms": ms_tile, "rays_per_s": rays / (ms_tile / 1e3),
                      "speedup_mixed_over_it": ms_tile / m32, "map_equal": tile_equal,
                      "visits_equal": bool(st_tile.visits == s64.visits),
                      "status_equal": list(st_tile.status) == list(s64.status)}}
    del d_map, res
    torch.cuda.empty_cache()
    GG = 512
    d_grid = torch.zeros(GG ** 3, dtype=torch.float64, device=dev)
    gres = {}
    for name, prec in (("mixed", sd.DTFE_MIXED), ("fp64", sd.DTFE_FP64)):
        def one(prec=prec):
            d_grid.zero_()
            mesh.grid_device(GG, 1.0, (0.5, 0.5, 0.5), 1, 77, d_grid.data_ptr(), precision=prec,
                             stream_ptr=sptr)
        one()
        ms = timed_launches(torch, stream, flush, one, 2)
        gres[name] = (float(np.median(ms)), mesh.last_stats(), d_grid.cpu().numpy())
    (g32ms, gs32, g32), (g64ms, gs64, g64) = gres["mixed"], gres["fp64"]
    e_max, e_rms = max_rel(g32, g64)
    out["grid"] = {"grid_dim": GG, "columns": GG * GG, "mixed_ms": g32ms, "fp64_ms": g64ms,
                   "speedup_mixed_over_fp64": g64ms / g32ms,
                   "visits_equal_fp64": bool(gs32.visits == gs64.visits),
                   "status_equal_fp64": list(gs32.status) == list(gs64.status),
                   "zero_cells_equal": bool(np.array_equal(g32 == 0, g64 == 0)),
                   "max_rel_err": e_max, "rms_rel_err": e_rms,
                   "mass_rel_diff": float(g32.sum() / GG ** 3 / len(pos4) - 1.0)}
    del d_grid, gres
    mesh.close()
    torch.cuda.empty_cache()
    return out


def run_ours(args, pre=None):
    import torch

    import sdtfe_b200 as sd

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)

    desc, pos4, spec = workload(args.workload)
    tri = sections = None
    if pre is not None:  # host Qhull runs in the process pool
        tri, sections = pre
        _, tetra, t_qhull = tri.get("main", args.workload)
    else:
        t = time.perf_counter()
        tetra = sd.triangulate(pos4)
        t_qhull = time.perf_counter() - t
        sections = []
    prec = sd.DTFE_MIXED if args.precision == "mixed" else sd.DTFE_FP64
    mesh = sd.Mesh(pos4, tetra, 1.0)
    G, S = spec.grid_dim, spec.n_samples
    params = sd.map_params(G, spec.box_len, spec.box_len_z, spec.center, S, 0.0, 12345,
                           precision=prec)
    p64 = sd.map_params(G, spec.box_len, spec.box_len_z, spec.center, S, 0.0, 12345,
                        precision=sd.DTFE_FP64)
    # one dedicated stream for everything timed: the map launches, the map
    # zeroing and the L2 flush are ordered on it, and the events sit on it
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream
    assert sptr != 0
    d_map = torch.zeros((G, G), dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def step(p):
        d_map.zero_()
        mesh.map_device(p, d_map.data_ptr(), sptr)

    tuned = None
    if prec == sd.DTFE_MIXED:  # the project's autotuner picks the kernel variant
        best, table = mesh.autotune(params)
        tuned = {"chosen": best, "variants": table}

    for _ in range(args.warmup):
        step(params)
    torch.cuda.synchronize()
    st_w = mesh.last_stats()

    # timed region
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = sd.lib().dtfe_kernel_launches()
    for i in range(args.steps):
        flush.zero_()
        ev[i][0].record(stream)
        step(params)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    launches = sd.lib().dtfe_kernel_launches() - launches0
    if dist:
        dist.barrier()
    clk = clocks.stop()
    step_ms = np.array([a.elapsed_time(b) for a, b in ev])
    st = mesh.last_stats()
    total_ms = slowest_rank_ms(float(step_ms.sum()), dist, dev)
    value = replica_rays_per_s(spec.rays, args.steps, world, total_ms)
    mixed_map = d_map.cpu().numpy().copy()

    # the plain FP64 path on the same map, and the mixed map's error against it
    fp64 = None
    if prec == sd.DTFE_MIXED:
        step(p64)
        torch.cuda.synchronize()
        e64 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(3)]
        for a, b in e64:
            flush.zero_()
            a.record(stream)
            step(p64)
            b.record(stream)
        torch.cuda.synchronize()
        ms64 = float(np.median([a.elapsed_time(b) for a, b in e64]))
        st64 = mesh.last_stats()
        map64 = d_map.cpu().numpy()
        denom = np.abs(map64)
        ok = denom > 0
        rel = np.abs(mixed_map - map64)[ok] / denom[ok]
        fp64 = {"rays_per_s": spec.rays / (ms64 / 1e3), "ms_per_map": ms64,
                "speedup_mixed_over_fp64": (spec.rays / (np.median(step_ms) / 1e3)) /
                                           (spec.rays / (ms64 / 1e3)),
                "max_rel_err": float(rel.max()) if rel.size else 0.0,
                "rms_rel_err": float(np.sqrt(np.mean(rel ** 2))) if rel.size else 0.0,
                "zero_pixels_differ": int(((map64 == 0) != (mixed_map == 0)).sum()),
                "visits_equal": bool(st64.visits == st.visits)}
        # the same FP64 map with one shared location walk per pixel tile
        # instead of the reference's walk from hull triangle 0 for every ray
        mesh.set_location(sd.LOCATE_TILE)
        step(p64)
        torch.cuda.synchronize()
        for a, b in e64:
            flush.zero_()
            a.record(stream)
            step(p64)
            b.record(stream)
        torch.cuda.synchronize()
        mesh.set_location(sd.LOCATE_PER_RAY)
        ms64t = float(np.median([a.elapsed_time(b) for a, b in e64]))
        st64t = mesh.last_stats()
        fp64["tile_location"] = {
            "rays_per_s": spec.rays / (ms64t / 1e3), "ms_per_map": ms64t,
            "speedup_mixed_over_it": ms64t / float(np.median(step_ms)),
            "map_equal": bool(np.array_equal(d_map.cpu().numpy(), map64)),
            "visits_equal": bool(st64t.visits == st64.visits),
            "status_equal": list(st64t.status) == list(st64.status)}
    # device-timed sections run while host Qhull for the others continues;
    # everything host-timed (e2e, the CPU baseline, serving latency) runs
    # after the pool has finished, on idle host cores
    extra = {}

    def run_section(name, fn):
        if sections and name in sections:
            try:
                extra[name] = fn()
            except Exception as e:  # a section must not cost the headline line
                extra[name] = {"error": f"{type(e).__name__}: {e}"}
            torch.cuda.synchronize()

    run_section("batch", lambda: section_batch(args, sd, torch, dev, stream, flush, tri))
    if tri is not None:
        tri.wait_all()

    # projected mass inside the map footprint (unit box fully covered)
    dxy = spec.box_len / G
    mass_map = float(mixed_map.sum() * dxy * dxy)
    mass = float(len(pos4) * 1.0)

    # end to end through the reference-facing drop-in, pinned host buffers
    L = sd.lib()
    L.dtfe_set_default_precision(prec)
    L.dtfe_set_seed(12345)
    pin_pos = torch.from_numpy(pos4.copy()).pin_memory()
    pin_tet = torch.from_numpy(tetra.copy()).pin_memory()
    pin_map = torch.zeros(G * G, dtype=torch.float64).pin_memory()
    pos_np, tet_np, map_np = pin_pos.numpy(), pin_tet.numpy(), pin_map.numpy()
    e2e_ms = []
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        map_np[:] = 0.0
        pos_np[:, 3] = 0.0
        torch.cuda.synchronize()
        t = time.perf_counter()
        L.compute_density(pos_np, len(pos_np), tet_np, len(tet_np), G, spec.box_len,
                          spec.box_len_z, map_np, 1.0, *spec.center, S, 0.0)
        dt = time.perf_counter() - t
        if i:  # first call warms the allocator pools
            e2e_ms.append(dt * 1e3)
    L.dtfe_set_seed(0)
    e2e_val = spec.rays / (np.median(e2e_ms) / 1e3) * world if e2e_ms else None
    h2d = pos4.nbytes + tetra.nbytes + G * G * 8
    d2h = G * G * 8 + len(pos4) * 8

    # roofline of the walk kernel
    visits = st.visits  # one launch
    bpv = BYTES_PER_VISIT[args.precision]
    kern_ms = float(np.median(step_ms))
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = peaks.get("hbm_gbs")
    hbm_note = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    kname = "k_map32" if args.precision == "mixed" else "k_map64"
    roof = roofline(kname, visits, len(tetra), bpv, kern_ms, clk.get("sm_mhz") or 1965.0,
                    torch.cuda.get_device_properties(dev).multi_processor_count, hbm, hbm_note)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            ref = RefCPU()
            ref.calibrate(pos4, tetra, spec, args.cpu_seconds / 2)
            v, sample = ref.step(pos4, tetra, spec)
            cpu = {"value": v, "unit": "rays/s", "cores": ref.cores, "kind": "reference",
                   "sample": sample}
        except Exception as e:  # the oracle/_ref build is missing
            cpu = {"value": None, "unit": "rays/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    run_section("plain_small",
                lambda: section_plain_small(args, sd, torch, dev, stream, flush, tri))
    run_section("serving", lambda: section_serving(args, sd, torch, tri))
    run_section("large_field",
                lambda: section_large_field(args, sd, torch, dev, stream, flush, tri))
    if tri is not None:
        extra["qhull_pool"] = tri.info()

    if rank == 0:
        line = {
            "metric": "los_rays_per_s", "value": value, "unit": "rays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(step_ms.mean()),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+guarded-f64" if args.precision == "mixed" else "f64",
            "data": "synthetic (seeded)",
            "config": workload_config(desc, len(pos4), len(tetra), spec, world),
            "precision": args.precision,
            "qhull_host_s": round(t_qhull, 2),
            "latency_ms": {"p50": float(np.percentile(step_ms, 50)),
                           "p99": float(np.percentile(step_ms, 99)),
                           "max": float(step_ms.max())},
            "maps_per_s": args.steps * world / (total_ms / 1e3),
            "visits_per_ray": visits / spec.rays,
            "ray_status": list(st.status),
            "fp64_fallbacks": st.fp64_fallbacks,
            "fp64": fp64,
            "mass_check": {"projected": mass_map, "particles": mass,
                           "rel_diff": (mass_map - mass) / mass},
            "e2e": {"value": e2e_val, "unit": "rays/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h),
                    "ms_per_step": float(np.median(e2e_ms)) if e2e_ms else None,
                    "call": "compute_density (dtfe.h drop-in), pinned host buffers"},
            "roofline": roof,
            "cpu_baseline": cpu,
            "autotune": tuned,
            "clocks": clk,
            "gpu_launches": int(launches),
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    mesh.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args, plan_sections(args))


if __name__ == "__main__":
    main()
