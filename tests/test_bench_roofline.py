"""The benchmark's issue roofline of the bound kernel: instructions scaled from
the captured case by the points, set against 4 warp instructions a cycle on
each of the 148 SMs at the sampled SM clock."""
import pytest

import bench


def test_issue_roofline_of_the_captured_case():
    # the captured 4096^2 launch: 404,377,736 warp instructions in 0.517 ms at 1914 MHz
    r = bench.issue_roofline("eb2d", 4096 ** 2, 0.517472, 1914.053)
    assert r["instructions"] == 404377736
    assert r["peak"] == pytest.approx(148 * 4 * 1.914053, rel=1e-4)
    assert r["achieved"] == pytest.approx(404377736 / 0.517472e-3 / 1e9, rel=1e-4)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"], abs=1e-4)
    assert 0.6 < r["frac"] < 0.8  # the capture's issue slots were about 70 % busy
    assert r["min_ms"] == pytest.approx(404377736 / (148 * 4 * 1.914053e9) * 1e3, rel=1e-3)
    assert r["unit"] == "G warp instructions/s"


def test_issue_roofline_scales_with_points_and_time():
    a = bench.issue_roofline("eb2d", 4096 ** 2, 0.5, 1965.0)
    b = bench.issue_roofline("eb2d", 8192 ** 2, 2.0, 1965.0)
    assert b["instructions"] == pytest.approx(4 * a["instructions"], rel=1e-9)
    assert b["achieved"] == pytest.approx(a["achieved"], rel=1e-3)
    assert b["min_ms"] == pytest.approx(4 * a["min_ms"], rel=1e-3)


@pytest.mark.parametrize("kernel,ms,mhz", [("wave2d_compress", 1.0, 1965.0), ("eb3d", 1.0, 1965.0),
                                           ("eb2d", 1.0, None), ("eb2d", 0.0, 1965.0), ("eb2d", None, 1965.0)])
def test_issue_roofline_absent_without_a_count_clock_or_time(kernel, ms, mhz):
    assert bench.issue_roofline(kernel, 1 << 20, ms, mhz) is None
