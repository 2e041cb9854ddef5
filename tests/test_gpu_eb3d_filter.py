"""The 3D bound kernel's filtered sign-keeping bounds (enclosures of all eight
keep_sign_3d values of a tet, exact evaluation of only those that can decide
the tet's bound) give the oracle's per-vertex bounds bit for bit, on fields
built to reach every branch of the filter: magnitudes far from 1 (sums of
triple products near 2^100, and at or above 2^126 where the approximation has
no enclosure), subnormal products, zeros beside tiny values, exact ties
between candidates, powers of two and noise."""
import math

import numpy as np
import pytest

import cpsz_b200
from cpsz_b200 import workloads as W
from tests._util import assert_bits_equal

pytestmark = pytest.mark.gpu

SHAPE = (20, 23, 27)


def _fields():
    rng = np.random.default_rng(11)
    n = lambda: rng.standard_normal(SHAPE).astype(np.float32)
    U, V, Wf = W.field_3d(91, *SHAPE, 3, 5.0)
    yield "smooth", (U, V, Wf)
    # triple products near 2^99: log2 of each magnitude sum is far from 0
    s = np.float32(2.0 ** 33)
    yield "large", (U * s, V * s, Wf * s)
    # products near 2^126 and above (no enclosure; some sums overflow to inf)
    s = np.float32(2.0 ** 42)
    yield "near_max", (n() * s, n() * s, n() * s)
    # products in the subnormal range
    s = np.float32(2.0 ** -45)
    yield "subnormal", (n() * s, n() * s, n() * s)
    # exact zeros beside magnitudes below 2^-60
    a, b, c = n(), n() * np.float32(2.0 ** -22), n() * np.float32(2.0 ** -22)
    a[rng.random(SHAPE) < 0.4] = 0
    b[rng.random(SHAPE) < 0.3] = 0
    yield "zeros_tiny", (a, b, c)
    # few distinct values: equal magnitudes, exact ties between minors
    yield "plateaus", tuple(rng.integers(-2, 3, SHAPE).astype(np.float32) for _ in range(3))
    # powers of two of both signs
    yield "pow2", tuple((np.ldexp(1.0, rng.integers(-6, 6, SHAPE)) * rng.choice([-1, 1], SHAPE)).astype(np.float32)
                        for _ in range(3))
    yield "noise", (n(), n(), n())
    # mixed scales inside one field
    e = rng.integers(-60, 60, SHAPE)
    yield "mixed_scales", (np.ldexp(n(), e).astype(np.float32), n(), np.ldexp(n(), -e).astype(np.float32))


KS3_DELTA = np.float32(1.5e-6)


def test_filter_premises_hold_on_this_device(ctx):
    """The enclosure proofs' premises, measured exhaustively on this GPU, and
    the 3D error budget recomputed from them term by term (the terms of the
    proof in eb_math.cuh) stays below KS3_DELTA less the rounding of k~ +-
    DELTA.  The 2D filter needs sqrt.approx below 2^-22 relative."""
    m = cpsz_b200.debug_filter_premises(ctx=ctx)
    u = 2.0 ** -24
    # acbrt1's deviation from the cube root, and the operations' maxima, as the proof states them
    assert m["acbrt1_hi"] <= 1.21e-6 and m["acbrt1_lo"] <= 7.14e-8
    assert m["rcp"] <= 9.9e-8 and m["ex2"] <= 1.44e-7 and m["sqrt"] < 2.0 ** -22
    term_roots = 0.5 * (math.log1p(m["acbrt1_hi"]) - math.log1p(-m["acbrt1_lo"]))
    ratio = math.log2(1 + m["rcp"] + u * (1 + m["rcp"]))  # |log2| of the ratio's relative error
    term_lg2 = 0.0
    for e, err in m["lg2"].items():
        # r in [2^e, 2^(e+1)): d >= -e - 1, and 1 - K^2 <= 4 s / (1 + s)^2 with s = 2^(-d/3)
        s = 2.0 ** (-max(0.0, -e - 1.0) / 3)
        term_lg2 = max(term_lg2, math.log(2) / 6 * 4 * s / (1 + s) ** 2 * (ratio + err))
    d = np.linspace(1e-3, 300, 300000)
    s = 2.0 ** (-d / 3)
    term_third = np.max(math.log(2) / 2 * 4 * s / (1 + s) ** 2 * (d / 3) * (abs(float(np.float32(1 / 3)) * 3 - 1) + u))
    total = term_roots + term_lg2 + term_third + m["ex2"] / 2 + (3 * u + m["rcp"]) + 3 * u
    assert total <= float(KS3_DELTA) - 6e-8, (term_roots, term_lg2, term_third, total)


@pytest.mark.parametrize("eb", [0.1, 0.01, 0.9])
def test_filtered_eb3d_equals_oracle(ctx, oracle, eb):
    for name, (U, V, Wf) in _fields():
        e, ids = cpsz_b200.debug_eb3d(U, V, Wf, eb, ctx=ctx)
        ref = oracle.eb_3d(U, V, Wf, eb)
        try:
            assert_bits_equal(e, ref, nan_equal=True)
        except AssertionError as err:
            raise AssertionError(f"{name}: {err}") from None
