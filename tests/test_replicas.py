"""The multi-GPU mode of bench.py: independent replicas, one per rank, with
the job's time taken as the slowest rank's (no collective on the data path).
Exercised here with two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 10.0 * (rank + 1)  # rank 1 is the slow one
        t = bench.slowest_rank_ms(local_ms, dist, "cpu")
        v = bench.replica_rays_per_s(1000, 5, world, t)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{t} {v}")
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_slowest_rank_time_and_job_rate(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    for r in range(world):
        t, v = map(float, open(tmp_path / f"rank{r}.txt").read().split())
        assert t == 20.0                      # the max over ranks, on every rank
        assert v == 1000 * 5 * world / 0.020  # all ranks' rays over the slowest time


def test_single_process_time_is_its_own():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.slowest_rank_ms(12.5, None, "cpu") == 12.5
    assert bench.replica_rays_per_s(100, 2, 1, 1000.0) == 200.0


def test_reference_arm_runs_on_rank_0_only(monkeypatch):
    """Under torchrun the reference arm runs on rank 0; other ranks exit at
    once, without work and without output."""
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    args = bench.argparse.Namespace(workload="clustered", warmup=3, steps=10, cpu_seconds=15.0,
                                    gpus=2)
    assert bench.run_reference(args) is None  # returns before building anything


def test_reference_arm_stays_off_the_library_and_matches_the_config():
    """The reference arm on the 32k uniform workload, in a fresh interpreter:
    it prints the same config object the GPU arm would (same tets: the numpy
    restatement of the reference's layout equals the library's), and never
    loads the sdtfe_b200 package or its shared library."""
    import json
    import subprocess

    code = (
        "import sys, json, runpy\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'uniform',\n"
        "            '--steps', '1', '--warmup', '0', '--cpu-seconds', '1']\n"
        "runpy.run_path('bench.py', run_name='__main__')\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'pkg': 'sdtfe_b200' in sys.modules,\n"
        "                  'so': 'libsdtfe_b200' in maps}))\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    ref_line, probe = lines[0], lines[-1]
    assert probe == {"pkg": False, "so": False}
    assert ref_line["impl"] == "reference" and ref_line["value"] > 0

    sys.path.insert(0, ROOT)
    import bench
    import sdtfe_b200 as sd

    desc, pos4, spec = bench.workload("uniform")
    tetra = sd.triangulate(pos4)
    assert ref_line["config"] == bench.workload_config(desc, len(pos4), len(tetra), spec, 1)
