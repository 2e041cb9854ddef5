"""The compressor's filtered 2D bounds (float sign-keeping bounds with a
proven enclosure, exact recomputation of any vertex whose enclosure straddles
an id threshold) give exactly the ids of the fully exact evaluation, on large
fields and on fields built to sit on thresholds, at several bounds."""
import numpy as np
import pytest

import cpsz_b200
from cpsz_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _fields():
    rng = np.random.default_rng(7)
    yield "smooth_2048", W.cfg0_like(31, 2048, 2048)
    U, V = W.field_2d(32, 1500, 2600, 300, 25.0)
    yield "smooth_1500x2600", (U, V)
    yield "tiny_scale", (U * np.float32(1e-30), V * np.float32(1e-30))
    yield "huge_scale", (U * np.float32(1e25), V * np.float32(1e25))
    # noise: critical points in most cells
    yield "noise", (rng.standard_normal((700, 900)).astype(np.float32),
                    rng.standard_normal((700, 900)).astype(np.float32))
    # few distinct values: many equal products, zero sums and exact ties
    yield "plateaus", (rng.integers(-3, 4, (600, 800)).astype(np.float32),
                       rng.integers(-3, 4, (600, 800)).astype(np.float32))
    # V nearly proportional to U: the flag sums s_k and det nearly cancel
    # (undecided flags take the exact path)
    yield "near_degenerate", (U[:700, :800], U[:700, :800] * np.float32(1.5) +
                              np.float32(1e-6) * V[:700, :800])
    # magnitudes spread over 60 binades (sums near the float filter's range limits)
    mag = np.ldexp(1.0, rng.integers(-40, 21, (600, 700))).astype(np.float32)
    yield "spread", (mag * rng.standard_normal((600, 700)).astype(np.float32),
                     np.roll(mag, 3, axis=1) * rng.standard_normal((600, 700)).astype(np.float32))
    # products in the float subnormal range
    yield "subnormal_products", (U[:500, :600] * np.float32(1e-20), V[:500, :600] * np.float32(3e-21))
    # powers of two: bounds land on exact binary fractions near thresholds
    yield "pow2", (np.ldexp(1.0, rng.integers(-8, 8, (512, 512))).astype(np.float32) *
                   rng.choice([-1, 1], (512, 512)).astype(np.float32),
                   np.ldexp(1.0, rng.integers(-8, 8, (512, 512))).astype(np.float32))


@pytest.mark.parametrize("eb", [0.1, 0.01, 1e-5, 0.9])
def test_filtered_ids_equal_exact_ids(ctx, eb):
    for name, (U, V) in _fields():
        _, exact = cpsz_b200.debug_eb2d(U, V, eb, ctx=ctx, exact=True)
        _, fast = cpsz_b200.debug_eb2d(U, V, eb, ctx=ctx, exact=False)
        bad = np.flatnonzero(exact != fast)
        assert bad.size == 0, f"{name}: {bad.size} ids differ, first at {bad[:5]}"


def test_compressor_uses_the_filtered_path_consistently(ctx):
    U, V = W.cfg0_like(33, 1024, 1536)
    st = cpsz_b200.compress_2d_stages(U, V, 0.1, ctx=ctx)
    _, exact = cpsz_b200.debug_eb2d(U, V, 0.1, ctx=ctx, exact=True)
    assert np.array_equal(st["ids"], np.where(exact == 255, 0, exact).astype(np.int32))
