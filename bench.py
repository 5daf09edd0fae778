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
    return ap.parse_args()


def workload(name):
    from sdtfe_b200 import workloads as W

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
        for ln in self.lines:
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
    """The reference's compute_density (its own C, oracle/_ref/libdtfe_ref.so)."""

    def __init__(self):
        from oracle.oracle import Reference

        self.R = Reference()
        self.cores = os.cpu_count()

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
        os.environ.setdefault("OMP_NUM_THREADS", str(self.cores))
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


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import sdtfe_b200 as sd

    desc, pos4, spec = workload(args.workload)
    tetra = sd.triangulate(pos4)
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
        "config": {"workload": desc, "particles": len(pos4), "tets": len(tetra),
                   "grid_dim": spec.grid_dim, "samples_per_pixel": spec.n_samples,
                   "rays_per_map": spec.rays},
        "cpu_baseline": {"value": value, "unit": "rays/s", "cores": ref.cores,
                         "kind": "reference", "sample": samples[-1]},
        "e2e": {"value": value, "unit": "rays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def read_ncu_traffic(kernel, n_tets):
    """DRAM bytes per launch of `kernel` from the committed ncu summary
    (profiles/traffic.json), scaled from the captured mesh to this one by the
    tet count: the walk reads each tet record from DRAM about once per map."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        d = json.load(open(path))[kernel]
        return d["dram_bytes"] / d["tets"] * n_tets
    except (OSError, KeyError, ValueError, ZeroDivisionError):
        return None


def run_ours(args):
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
    t = time.perf_counter()
    tetra = sd.triangulate(pos4)
    t_qhull = time.perf_counter() - t
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
    total_ms = float(step_ms.sum())
    if dist:
        tt = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
    rays_all = spec.rays * args.steps * world
    value = rays_all / (total_ms / 1e3)
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
    achieved = visits * bpv / (kern_ms / 1e3) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs")
    peak_note = "measured" if peak else "fallback"
    peak = peak or 6650.0
    kname = "k_map32" if args.precision == "mixed" else "k_map64"
    traffic = read_ncu_traffic(kname, len(tetra))

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

    if rank == 0:
        line = {
            "metric": "los_rays_per_s", "value": value, "unit": "rays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(step_ms.mean()),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+guarded-f64" if args.precision == "mixed" else "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": desc, "particles": len(pos4), "tets": len(tetra),
                       "grid_dim": G, "samples_per_pixel": S, "rays_per_map": spec.rays,
                       "precision": args.precision, "parallelism": f"replicas x{world}",
                       "l2": "flushed between steps (256 MiB write); tet records "
                             f"{len(tetra) * bpv / 1e6:.0f} MB > L2",
                       "qhull_host_s": round(t_qhull, 2)},
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
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": kname, "bytes_per_visit": bpv,
                         "note": f"peak {peak_note} (STREAM-style copy); achieved counts "
                                 "algorithmic tet-record bytes, much of it served by L1/L2"},
            "cpu_baseline": cpu,
            "autotune": tuned,
            "clocks": clk,
            "gpu_launches": int(launches),
        }
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
        run_ours(args)


if __name__ == "__main__":
    main()
