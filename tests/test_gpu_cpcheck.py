"""The GPU exact critical-point checker against the exact-rational oracle, and
the compressor's guarantee measured with it (no CP lost, spurious or retyped)."""
import numpy as np
import pytest

import cpsz_b200
from cpsz_b200 import workloads as W
from oracle import cp_exact
from tests.test_cp_oracle import CASES_2D, CASES_3D, linear_2d, linear_3d

pytestmark = pytest.mark.gpu


def _fields_2d():
    rng = np.random.default_rng(21)
    yield "normal", tuple(rng.normal(size=(40, 50)).astype(np.float32) for _ in range(2))
    yield "integers", tuple(rng.integers(-2, 3, size=(30, 31)).astype(np.float32) for _ in range(2))
    base = [rng.integers(-3, 4, size=(30, 30)).astype(np.float32) for _ in range(2)]
    yield "near_degenerate", tuple((b + np.float32(2.0 ** -20) * rng.integers(-2, 3, size=b.shape)).astype(np.float32)
                                   for b in base)
    e = rng.integers(-60, 60, size=(25, 26))
    yield "wide_range", tuple((rng.normal(size=(25, 26)) * 2.0 ** e).astype(np.float32) for _ in range(2))
    yield "cfg0_like", W.cfg0_like(3, 60, 70)


@pytest.mark.parametrize("name,f", list(_fields_2d()), ids=lambda x: x if isinstance(x, str) else "")
def test_gpu_cp2d_equals_oracle(ctx, name, f):
    U, V = f
    got = cpsz_b200.cp_check_2d(U, V, cells=True, ctx=ctx)["cells"]
    assert np.array_equal(got, cp_exact.cells_2d(U, V))


@pytest.mark.parametrize("J,code", CASES_2D)
def test_gpu_cp2d_linear_fields(ctx, J, code):
    U, V = linear_2d(J, 3.25, 4.625)
    got = cpsz_b200.cp_check_2d(U, V, cells=True, ctx=ctx)["cells"]
    nz = np.flatnonzero(got)
    assert nz.size == 1 and got[nz[0]] == code


def _fields_3d():
    rng = np.random.default_rng(22)
    yield "normal", tuple(rng.normal(size=(9, 10, 11)).astype(np.float32) for _ in range(3))
    yield "integers", tuple(rng.integers(-2, 3, size=(8, 8, 9)).astype(np.float32) for _ in range(3))
    base = [rng.integers(-2, 3, size=(7, 8, 8)).astype(np.float32) for _ in range(3)]
    yield "near_degenerate", tuple((b + np.float32(2.0 ** -18) * rng.integers(-2, 3, size=b.shape)).astype(np.float32)
                                   for b in base)
    yield "field", W.field_3d(4, 10, 11, 12, 6, 3.0)


@pytest.mark.parametrize("name,f", list(_fields_3d()), ids=lambda x: x if isinstance(x, str) else "")
def test_gpu_cp3d_equals_oracle(ctx, name, f):
    U, V, Wf = f
    got = cpsz_b200.cp_check_3d(U, V, Wf, cells=True, ctx=ctx)["cells"]
    assert np.array_equal(got, cp_exact.cells_3d(U, V, Wf))


@pytest.mark.parametrize("J,code", CASES_3D)
def test_gpu_cp3d_linear_fields(ctx, J, code):
    U, V, Wf = linear_3d(J, (2.25, 2.625, 1.375))
    got = cpsz_b200.cp_check_3d(U, V, Wf, cells=True, ctx=ctx)["cells"]
    nz = np.flatnonzero(got)
    assert nz.size == 1 and got[nz[0]] == code


def test_gpu_cp_compare_counts(ctx):
    rng = np.random.default_rng(5)
    U, V = (rng.normal(size=(64, 65)).astype(np.float32) for _ in range(2))
    U2 = U.copy()
    U2[10:20, 10:20] += 0.5
    r = cpsz_b200.cp_check_2d(U, V, U2, V, ctx=ctx)
    a = cp_exact.cells_2d(U, V)
    b = cp_exact.cells_2d(U2, V)
    assert r == cp_exact.compare(a, b)


@pytest.mark.parametrize("eb", [0.1, 0.01])
def test_compressor_preserves_cps_2d(ctx, eb):
    U, V = W.cfg0_like(17, 600, 700)
    blob = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=eb, ctx=ctx)
    dU, dV = cpsz_b200.sz_decompress_cp_preserve_2d_offline(blob, *U.shape, ctx=ctx)
    r = cpsz_b200.cp_check_2d(U, V, dU, dV, ctx=ctx)
    assert r["cps_a"] > 0
    assert r["lost_or_spurious"] == 0 and r["type_changed"] == 0, r


def test_compressor_preserves_cps_3d(ctx):
    U, V, Wf = W.field_3d(7, 48, 50, 52, 30, 5.0)
    blob = cpsz_b200.sz_compress_cp_preserve_3d_offline_log(U, V, Wf, max_pwr_eb=0.05, ctx=ctx)
    d = cpsz_b200.sz_decompress_cp_preserve_3d_online_log(blob, *U.shape, ctx=ctx)
    r = cpsz_b200.cp_check_3d(U, V, Wf, *d, ctx=ctx)
    assert r["cps_a"] > 0
    assert r["lost_or_spurious"] == 0 and r["type_changed"] == 0, r
