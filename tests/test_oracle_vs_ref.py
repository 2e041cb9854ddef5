"""The restated oracle against the reference's own sources (oracle/_ref),
run live on seeded generator fields (skipped where the reference build is absent)."""
import numpy as np
import pytest

from cpsz_b200 import workloads as W
from oracle import ref_2d_in_bounds, ref_2d_log_in_bounds, ref_3d_in_bounds
from tests._util import assert_bits_equal, assert_blob_equal_2d, assert_blob_equal_2d_log


@pytest.mark.parametrize("r1,r2,eb,seed", [(200, 300, 0.1, 6), (517, 611, 0.1, 7), (300, 257, 0.01, 8),
                                           (64, 1000, 0.05, 9), (1000, 40, 0.1, 10)])
def test_2d_blob_and_decode_identical(oracle, reference, r1, r2, eb, seed):
    U, V = W.cfg0_like(seed, r1, r2)
    a = oracle.compress_2d(U, V, eb)
    if not ref_2d_in_bounds(a, r1, r2):
        pytest.skip("workload exceeds the reference's fixed scratch buffers")
    b = reference.compress_2d(U, V, eb)
    assert_blob_equal_2d(a, b)
    da = oracle.decompress_2d(a, r1, r2)
    db = reference.decompress_2d(b, r1, r2)
    for x, y in zip(da, db):
        assert_bits_equal(x, y)


def _edge_field(case):
    g = np.random.default_rng(31)
    if case == "zeros":
        return np.zeros((50, 70), np.float32), np.zeros((50, 70), np.float32), 0.1
    if case == "constant":
        return np.full((40, 40), 3.5, np.float32), np.full((40, 40), -2.0, np.float32), 0.1
    if case == "small_integers":  # many degenerate and tied triangles
        return (g.integers(-3, 4, (60, 50)).astype(np.float32), g.integers(-3, 4, (60, 50)).astype(np.float32), 0.1)
    if case == "tiny_magnitudes":
        U, V = W.cfg0_like(22, 80, 90)
        return U * np.float32(1e-30), V * np.float32(1e-30), 0.1
    if case == "bound_1":
        U, V = W.cfg0_like(23, 70, 60)
        return U, V, 1.0
    r1, r2 = (int(x) for x in case.split("x"))
    U, V = W.cfg0_like(25, r1, r2)
    return U, V, 0.1


# Fields whose products overflow float (|x| near 1e30) are left out: the
# reference's bounds are NaN there and its id histogram is indexed out of range.
@pytest.mark.parametrize("case", ["zeros", "constant", "small_integers", "tiny_magnitudes", "bound_1", "1x50", "50x1",
                                  "12x12", "13x25", "2x300"])
def test_2d_edge_cases_identical(oracle, reference, case):
    """Constant and all-zero fields, integer-valued fields, magnitudes near the
    float minimum, the largest relative bound, and shapes of one row, one
    column, exactly one block and one block plus a ragged edge."""
    U, V, eb = _edge_field(case)
    r1, r2 = U.shape
    a = oracle.compress_2d(U, V, eb)
    assert ref_2d_in_bounds(a, r1, r2)
    b = reference.compress_2d(U, V, eb)
    assert_blob_equal_2d(a, b)
    for x, y in zip(oracle.decompress_2d(a, r1, r2), reference.decompress_2d(b, r1, r2)):
        assert_bits_equal(x, y)


@pytest.mark.parametrize("r1,r2,eb,seed", [(200, 300, 0.1, 16), (317, 211, 0.01, 17), (64, 900, 0.05, 18)])
def test_2d_log_blob_and_decode_identical(oracle, reference, r1, r2, eb, seed):
    U, V = W.cfg0_like(seed, r1, r2)
    U.ravel()[::11] = 0  # logs of -100
    V.ravel()[::13] = -V.ravel()[::13]
    a = oracle.compress_2d_log(U, V, eb)
    if not ref_2d_log_in_bounds(a, r1, r2):
        pytest.skip("workload exceeds the reference's fixed scratch buffers")
    b = reference.compress_2d_log(U, V, eb)
    assert_blob_equal_2d_log(a, b, U.size)
    for x, y in zip(oracle.decompress_2d_log(a, r1, r2), reference.decompress_2d_log(b, r1, r2)):
        assert_bits_equal(x, y)


@pytest.mark.parametrize("shape,eb,seed", [((48, 48, 48), 0.05, 4), ((40, 33, 50), 0.01, 5), ((30, 60, 45), 0.1, 6)])
def test_3d_blob_and_decode_identical(oracle, reference, shape, eb, seed):
    U, V, Wf = W.field_3d(seed, *shape, max(1, int(np.prod(shape)) // 4000), 6.0)
    a = oracle.compress_3d(U, V, Wf, eb)
    if not ref_3d_in_bounds(a, *shape):
        pytest.skip("workload exceeds the reference's fixed scratch buffer")
    b = reference.compress_3d(U, V, Wf, eb)
    assert a == b
    for x, y in zip(oracle.decompress_3d(a, *shape), reference.decompress_3d(b, *shape)):
        assert_bits_equal(x, y)


@pytest.mark.parametrize("shape", [(1, 30, 40), (30, 1, 40), (30, 40, 1)])
def test_3d_single_plane_row_or_column_identical(oracle, reference, shape):
    """Fields one point thick along each axis (no tetrahedra: every bound is
    the relative one).  Constant, zero and integer-valued 3D fields are left
    out: in the log domain they exceed the reference's fixed scratch buffer."""
    U, V, Wf = W.field_3d(9, *shape, 2, 6.0)
    a = oracle.compress_3d(U, V, Wf, 0.05)
    assert ref_3d_in_bounds(a, *shape)
    b = reference.compress_3d(U, V, Wf, 0.05)
    assert a == b
    for x, y in zip(oracle.decompress_3d(a, *shape), reference.decompress_3d(b, *shape)):
        assert_bits_equal(x, y)


def test_zstd_stage_matches(reference):
    import cpsz_b200

    U, V = W.cfg0_like(3, 256, 256)
    data = U.tobytes() + V.tobytes()
    assert cpsz_b200.sz_lossless_compress(data, 3) == reference.zstd_compress(data)
