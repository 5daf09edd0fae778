"""bench.py's roofline line, recomputed from the committed profile.

The bench reports the walk kernel against instruction issue: warp
instructions per visit (from profiles/roofline.json) times the timed launch's
visits, over its time, against 148 SMs x 4 schedulers x the SM clock.  Fed
the profiled launch itself, the fraction must equal the issue activity ncu
measured on it, and the DRAM traffic must scale with the mesh's tets.
"""
import json
import os
import sys

from conftest import ROOT


def _bench():
    sys.path.insert(0, ROOT)
    import bench

    return bench


def test_profile_is_self_consistent():
    prof = json.load(open(os.path.join(ROOT, "profiles", "roofline.json")))["k_map32"]
    assert 100 < prof["visits"] / prof["rays"] < 1000
    assert 4.0 < prof["warp_inst"] / prof["visits"] < 8.0
    assert prof["dram_bytes"] > 0 and prof["tets"] > 0


def test_roofline_of_the_profiled_launch_is_its_issue_activity():
    bench = _bench()
    prof = json.load(open(os.path.join(ROOT, "profiles", "roofline.json")))["k_map32"]
    r = bench.roofline("k_map32", prof["visits"], prof["tets"], 96, prof["duration_ms_under_ncu"],
                       1960.0, 148, 6545.6, "measured")
    assert r["bound"] == "issue"
    # issue activity counts cycles with an issue; the two agree within a few
    # percent (the clock under ncu is sampled, not fixed)
    assert abs(r["frac"] - prof["issue_active_pct"] / 100.0) < 0.02
    assert r["traffic"] == prof["dram_bytes"]
    assert abs(r["achieved"] * 1e9 * prof["duration_ms_under_ncu"] / 1e3 - prof["warp_inst"]) \
        < 1e-6 * prof["warp_inst"]


def test_roofline_scales_with_the_timed_launch():
    bench = _bench()
    prof = json.load(open(os.path.join(ROOT, "profiles", "roofline.json")))["k_map32"]
    a = bench.roofline("k_map32", 2 * prof["visits"], 4 * prof["tets"], 96, 2.0, 1965.0, 148,
                       6545.6, "measured")
    b = bench.roofline("k_map32", prof["visits"], prof["tets"], 96, 1.0, 1965.0, 148, 6545.6,
                       "measured")
    assert abs(a["frac"] - b["frac"]) < 1e-12          # twice the visits in twice the time
    assert abs(a["traffic"] - 4 * b["traffic"]) < 1e-3  # DRAM bytes per tet
    assert abs(a["peak"] - 148 * 4 * 1.965) < 1e-9     # G warp instructions/s
