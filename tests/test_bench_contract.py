"""Host-side pieces of bench.py that need no GPU: the clock record taken
during the timed region, the traffic figures read from the committed ncu
summaries, and the algorithmic flops per ray."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def smi(sm, mx, hw="Not Active", thermal="Not Active", sw_thermal="Not Active", power="Not Active"):
    return "0, %d, %d, 700.00, 0x0000000000000000, %s, %s, %s, %s" % (sm, mx, hw, thermal, sw_thermal, power)


def test_clock_record_keeps_the_timed_region_only():
    lines = [(0.0, smi(345, 1965)), (0.2, smi(345, 1965, thermal="Active")),  # idle lead-in
             (1.00, smi(1965, 1965)), (1.05, smi(1950, 1965)), (1.10, smi(1965, 1965, power="Active")),
             (3.0, smi(1200, 1965, hw="Active"))]  # after the region
    c = bench.ClockSampler.summarise(lines, (0.98, 1.12))
    assert c["samples"] == 3 and c["sm_mhz"] == 1965.0 and c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["sw_power_cap"] and c["scope"] == "timed region"


def test_clock_record_reports_throttling_and_falls_back_to_the_whole_run():
    lines = [(0.0, smi(1965, 1965)), (0.5, smi(1100, 1965, hw="Active", sw_thermal="Active")), (0.6, "garbage")]
    c = bench.ClockSampler.summarise(lines, (5.0, 6.0))  # nothing arrived inside
    assert c["scope"].startswith("whole run") and c["samples"] == 2
    assert c["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"] and c["sm_mhz"] == pytest.approx(1532.5)


@pytest.mark.parametrize("name,points", [("mid", 1 << 20), ("large", 1 << 23)])
def test_traffic_of_the_committed_summaries_covers_the_point_data(name, points):
    t = bench.read_traffic(name)
    assert t is not None
    # per point: heliostat id 4 B, mask record 16 B, world coordinates 32 B,
    # plus the per-sun geometry
    assert 52 * points <= t <= 1.25 * 52 * points


def test_flops_per_ray_of_the_reference_algorithm():
    # 1000 rays, 100 shadowed, 12 760 rectangle tests, 5 140 DDA cells
    assert bench.flops_per_ray([1000, 100, 0, 0, 0, 12760, 5140]) == pytest.approx(192 + 30 * 1.9 + 54 * 12.76 + 4 * 5.14)


def test_both_arms_quote_the_same_config():
    from onemirror_b200 import workloads as W
    for name in ("small", "mid", "large"):
        w = W.BUILDERS[name]()
        a, b = bench.bench_config(w, 1), bench.bench_config(W.BUILDERS[name](), 1)
        assert a == b and "Poisson sample points" in a["step"] and "smoothing" in a["step"]
        assert "flushed" in a["l2"]


@pytest.mark.parametrize("name", ["nine", "mid"])
def test_reference_cuda_scenes_pass_the_range_checks(name):
    # the CPU checks that gate every run of the reference's own CUDA pass
    sc = bench.ref_cuda_scene(name)
    assert bench.ref_cuda_checks(sc) is None
    assert np.allclose(np.linalg.norm(sc["normal"], axis=1), 1.0, atol=1e-5)


def test_reference_cuda_checks_catch_a_cube_outside_the_grid():
    sc = dict(bench.ref_cuda_scene("nine"))
    sc["pos"] = np.array(sc["pos"], np.float32)
    sc["pos"][0, 0] = sc["gpos"][0] + 0.2  # registration cube reaches below the grid origin
    assert bench.ref_cuda_checks(sc) is not None
