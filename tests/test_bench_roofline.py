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


# stage times (ms) of a measured 8192^2 step, eb 0.1
STAGES_2D = {"h2d+setup": 0.0822, "eb2d": 2.4675, "wave2d_compress": 0.5528, "blocks+hist+unpred": 0.4978,
             "host_trees": 0.3836, "huffman_encode": 0.4187, "blob_assembly": 0.0561}


def test_product_roofline_of_the_2d_step():
    """The line's roofline for the measured step: eb2d dominant, 10 B a vertex
    over its stage time against the measured copy bandwidth, the captured
    traffic scaled by points, and the issue roofline beside it."""
    n = 8192 ** 2
    r = bench.product_roofline("2d", n, STAGES_2D, 1965.0)
    peak, kind = bench.measured_peaks()
    assert r["kernel"] == "eb2d" and r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert r["algorithmic_bytes"] == 10 * n
    assert r["achieved"] == pytest.approx(10 * n / 2.4675e-3 / 1e9, rel=1e-4)
    assert r["peak"] == peak and r["peak_source"] == kind
    assert r["frac"] == pytest.approx(r["achieved"] / peak, abs=1e-4)
    assert r["traffic"] == round((134.725632e6 + 254.642176e6) * 4)
    assert r["issue"] == bench.issue_roofline("eb2d", n, 2.4675, 1965.0)
    assert r["issue"]["frac"] == pytest.approx(0.564, abs=2e-3)


def test_product_roofline_without_a_clock_or_an_issue_count():
    r = bench.product_roofline("2d", 8192 ** 2, STAGES_2D, None)
    assert r["kernel"] == "eb2d" and "issue" not in r
    r3 = bench.product_roofline("3d", 384 ** 3, {"eb3d": 15.7, "wave3d_compress": 3.0, "log3d": 1.5}, 1965.0)
    assert r3["kernel"] == "eb3d" and r3["algorithmic_bytes"] == 13 * 384 ** 3 and "issue" not in r3
    assert r3["traffic"] is None
    assert bench.product_roofline("2d", 100, {"host_trees": 1.0}, 1965.0) is None
    assert bench.product_roofline("2d", 100, {}, 1965.0) is None
