"""bench.py's host-side arithmetic on CPU: the roofline figures of a step profile."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def merged_profile(ms):
    """one RK4 step on the merged path: per stage y fwd (10), z (22), y inv (11), boundary (3)"""
    out = []
    for s in range(4):
        out += [(10, ms["y"]), (22, ms["z"]), (11, ms["y"]), (3, ms["b"][s])]
    return out


def test_roofline_of_a_merged_step():
    F = 256 ** 3 * 16
    r = {"profile": merged_profile({"y": 0.1, "z": 0.12, "b": [0.25, 0.3, 0.35, 0.3]}), "field_bytes": F}
    rf = bench.roofline(r, "c128")
    assert rf["kernel"] == "x_stage_boundary" and rf["launches_per_step"] == 4
    assert rf["algorithmic_bytes_per_launch"] == pytest.approx(5.75 * F)
    # achieved = algorithmic bytes of the kind / its total time
    assert rf["achieved"] == pytest.approx(23 * F / 1.2e-3 / 1e9, rel=1e-3)
    step = rf["step"]
    assert step["algorithmic_bytes"] == 47 * F and step["bytes_per_site"] == 752.0
    assert step["achieved"] == pytest.approx(47 * F / (4 * (0.1 + 0.12 + 0.1) + 1.2) / 1e6, rel=1e-3)
    peak, src = bench.measured_peaks()
    assert rf["peak"] == peak and rf["frac"] == pytest.approx(rf["achieved"] / peak, abs=1e-4)
    assert rf["share_of_step"] == pytest.approx(1.2 / (4 * 0.32 + 1.2), abs=1e-4)


def test_roofline_traffic_comes_from_the_matching_precision():
    F = 256 ** 3 * 16
    r = {"profile": merged_profile({"y": 0.1, "z": 0.12, "b": [0.3] * 4}), "field_bytes": F}
    t128 = bench.roofline(r, "c128")["traffic"]
    t64 = bench.roofline(dict(r, field_bytes=F // 2), "c64")["traffic"]
    # the committed ncu summaries: per launch of the boundary, 4F-7F of the precision's field
    assert t128 is not None and 4 * F < t128 < 7 * F
    assert t64 is not None and 4 * (F // 2) < t64 < 7 * (F // 2)


def test_unknown_profiles_give_no_roofline():
    assert bench.roofline({"profile": [(3, 1.0)] * 7, "field_bytes": 16}) is None


def test_roofline_of_a_step_with_l2_slabs():
    """With the y/z passes on x-slabs that stay in L2, only the slab's y forward read and its y
    inverse write reach HBM: per stage 2F for the y/z work, 31F per step."""
    F = 256 ** 3 * 16
    prof = []
    for s in range(4):
        for _ in range(4):
            prof += [(10, 0.02), (22, 0.03), (11, 0.02)]
        prof.append((3, 0.3))
    rf = bench.roofline({"profile": prof, "field_bytes": F}, "c128")
    assert rf["kernel"] == "x_stage_boundary"
    assert rf["step"]["algorithmic_bytes"] == pytest.approx(31 * F)
    assert rf["per_kind_ms"]["z_fwd_kinetic_inv"] == pytest.approx(16 * 0.03)


def test_cpu_baseline_of_the_preconditioned_leg(monkeypatch):
    """The oracle's preconditioned iteration is timed per iteration at each grid size of the
    leg and charged with the GPU's iteration count of every solve."""
    small = [dict(n=16, L=12.0, N=30.0, c3=-3.0, c4=2.5, omega=0.0, dt=0.0),
             dict(n=24, L=16.0, N=60.0, c3=-3.1, c4=2.5, omega=0.0, dt=0.0)]
    monkeypatch.setattr(bench, "batch_solves", lambda count, seed=2025, rank=0: small)
    gp = {"_steps": [40, 55], "_grids": [16, 24]}
    r = bench.cpu_precond_baseline(gp, iters=2)
    per = r["seconds_per_iteration"]
    assert set(per) == {"16", "24"} and all(t > 0 for t in per.values())
    assert r["value"] == pytest.approx(2 / (40 * per["16"] + 55 * per["24"]))
    assert r["unit"] == "ground states/s" and r["kind"] == "port" and r["cores"] >= 1
