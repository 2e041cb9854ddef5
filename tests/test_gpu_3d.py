"""3D offline (log) path on the GPU vs the oracle: the host log2f / exp2f
reproduction, per-vertex bounds, blob bytes and decoded fields, bit-exact."""
import numpy as np
import pytest

import cpsz_b200
from cpsz_b200 import workloads as W
from tests._util import assert_bits_equal, golden_cases
from tests.test_libm_tables import _load

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["log2f", "exp2f"])
def test_gpu_libm_matches_host_library(ctx, oracle, name):
    _, fns = _load()
    band, hin, hout, mis = fns[name]
    rng = np.random.default_rng(11)
    if name == "log2f":
        rand = rng.integers(1, 0x7F800000, 4_000_000, dtype=np.uint32)
        near1 = (np.uint32(0x3E800000) + rng.integers(0, 1 << 25, 2_000_000, dtype=np.uint32)).astype(np.uint32)
        special = np.array([1, 2, 0x007FFFFF, 0x00800000, 0x3F800000, 0x3F800001, 0x3F7FFFFF, 0x7F7FFFFF, 0x7F800000],
                           np.uint32)
    else:
        rand = np.concatenate([rng.uniform(-99, 128, 4_000_000), rng.uniform(-2, 2, 1_000_000)]).astype(
            np.float32).view(np.uint32)
        near1 = np.array([], np.uint32)
        special = np.array([0, 0x80000000, 0x42FE0000, 0x43000000, 0x42FFFFFF, 0xC2C60000, 0x3F800000, 0xBF800000],
                           np.uint32)
    bits = np.concatenate([hin, mis, rand, near1, special]).astype(np.uint32)
    # neighbours of the listed inputs too
    bits = np.concatenate([bits, hin + 1, hin - 1, mis + 1, mis - 1]).astype(np.uint32)
    if name == "log2f":
        bits = bits[(bits >= 1) & (bits <= 0x7F800000)]
    x = bits.view(np.float32)
    if name == "exp2f":
        x = x[(x >= -99) & (x <= 128)]
    g = cpsz_b200.debug_libm(name, x, ctx=ctx)
    h = oracle.host_libm(name, x)
    bad = np.flatnonzero(g.view(np.uint32) != h.view(np.uint32))
    assert bad.size == 0, f"{bad.size} mismatches, first inputs {x[bad[:5]].view(np.uint32)}"


EB_SHAPES = [(2, 2, 2), (1, 5, 7), (5, 1, 7), (5, 7, 1), (33, 20, 17), (9, 40, 41), (40, 9, 70)]


@pytest.mark.parametrize("shape", EB_SHAPES)
@pytest.mark.parametrize("eb", [0.1, 0.01])
def test_gpu_eb3d_equals_oracle(ctx, oracle, shape, eb):
    U, V, Wf = W.field_3d(sum(shape) * 31 + 5, *shape, max(1, int(np.prod(shape)) // 3000), 5.0)
    e, ids = cpsz_b200.debug_eb3d(U, V, Wf, eb, ctx=ctx)
    assert_bits_equal(e, oracle.eb_3d(U, V, Wf, eb))


@pytest.mark.parametrize("path", golden_cases("3d_"), ids=lambda p: p.split("/")[-1])
def test_gpu_3d_matches_reference_fixture(ctx, path):
    g = np.load(path)
    U, V, Wf, eb = g["U"], g["V"], g["W"], float(g["eb"])
    blob = cpsz_b200.sz_compress_cp_preserve_3d_offline_log(U, V, Wf, max_pwr_eb=eb, ctx=ctx)
    assert blob == g["blob"].tobytes()
    out = cpsz_b200.sz_decompress_cp_preserve_3d_online_log(g["blob"].tobytes(), *U.shape, ctx=ctx)
    for a, k in zip(out, ("dU", "dV", "dW")):
        assert_bits_equal(a, g[k])


SHAPES = [(1, 1, 1), (2, 2, 2), (1, 1, 50), (1, 40, 3), (3, 4, 5), (16, 16, 16), (33, 20, 17), (20, 33, 17),
          (7, 100, 9), (64, 64, 64)]


def _check_roundtrip(ctx, oracle, U, V, Wf, eb):
    shape = U.shape
    a = cpsz_b200.sz_compress_cp_preserve_3d_offline_log(U, V, Wf, max_pwr_eb=eb, ctx=ctx)
    b = oracle.compress_3d(U, V, Wf, eb)
    assert len(a) == len(b)
    assert a == b
    assert cpsz_b200.blob_size_3d(a, *shape) == len(a)
    got = cpsz_b200.sz_decompress_cp_preserve_3d_online_log(a, *shape, ctx=ctx)
    exp = oracle.decompress_3d(b, *shape)
    for x, y in zip(got, exp):
        assert_bits_equal(x, y)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("eb", [0.1, 0.01])
def test_gpu_3d_blob_equals_oracle(ctx, oracle, shape, eb):
    U, V, Wf = W.field_3d(int(np.prod(shape)) + 17, *shape, max(1, int(np.prod(shape)) // 4000), 6.0)
    _check_roundtrip(ctx, oracle, U, V, Wf, eb)


def test_gpu_3d_all_unpredictable(ctx, oracle):
    U, V, Wf = W.field_3d(5, 12, 13, 14, 3, 4.0)
    _check_roundtrip(ctx, oracle, U, V, Wf, 0.0)


def test_gpu_3d_zeros_signs_and_repeats(ctx, oracle):
    rng = np.random.default_rng(3)
    shape = (18, 19, 21)
    # quantized values: exact zeros (log -100), repeated values, both signs
    U, V, Wf = (np.round(rng.normal(size=shape) * 4).astype(np.float32) / 4 for _ in range(3))
    U[::3] = 0
    V[:, ::2] = -V[:, ::2]
    _check_roundtrip(ctx, oracle, U, V, Wf, 0.1)


def test_gpu_3d_tiny_and_huge_magnitudes(ctx, oracle):
    rng = np.random.default_rng(4)
    shape = (10, 11, 12)
    e = rng.integers(-140, 120, size=shape)
    U = (rng.uniform(0.5, 1, shape) * 2.0 ** e).astype(np.float32)
    V = (rng.uniform(-1, 1, shape)).astype(np.float32)
    Wf = (rng.uniform(-1, 1, shape) * 1e-30).astype(np.float32)
    _check_roundtrip(ctx, oracle, U, V, Wf, 0.1)


def test_gpu_3d_128_cube(ctx, oracle):
    U, V, Wf = W.field_3d(9, 128, 128, 128, 40, 12.0)
    _check_roundtrip(ctx, oracle, U, V, Wf, 0.1)


def test_gpu_3d_device_arrays(ctx, oracle):
    torch = pytest.importorskip("torch")
    U, V, Wf = W.field_3d(21, 30, 31, 32, 8, 6.0)
    d = [torch.from_numpy(a).cuda() for a in (U, V, Wf)]
    a = cpsz_b200.sz_compress_cp_preserve_3d_offline_log(*d, max_pwr_eb=0.1, ctx=ctx)
    assert a == oracle.compress_3d(U, V, Wf, 0.1)
    out = [torch.empty(U.shape, dtype=torch.float32, device="cuda") for _ in range(3)]
    cpsz_b200.sz_decompress_cp_preserve_3d_online_log(a, *U.shape, *out, ctx=ctx)
    for x, y in zip(out, oracle.decompress_3d(a, *U.shape)):
        assert_bits_equal(x.cpu().numpy(), y)


def test_gpu_3d_repeatable(ctx, oracle):
    """The persistent wavefront's units run in whatever order the GPU
    schedules them; every run must give the oracle's blob and decode.  Many
    runs of one field (rows not a multiple of 32, a partial last plane group)
    would expose a read of a ring entry or input that has not landed, or of
    another unit's output before it was published."""
    torch = pytest.importorskip("torch")
    U, V, Wf = W.field_3d(23, 61, 97, 101, 10, 7.0)
    ref = oracle.compress_3d(U, V, Wf, 0.05)
    d = [torch.from_numpy(a).cuda() for a in (U, V, Wf)]
    out = torch.zeros(len(ref) + 65536, dtype=torch.uint8, device="cuda")
    for _ in range(16):
        n = cpsz_b200.compress_3d_into(*d, *U.shape, 0.05, out, ctx=ctx)
        assert n == len(ref) and out[:n].cpu().numpy().tobytes() == ref
    dec = oracle.decompress_3d(ref, *U.shape)
    outs = [torch.empty(U.shape, dtype=torch.float32, device="cuda") for _ in range(3)]
    for _ in range(8):
        cpsz_b200.sz_decompress_cp_preserve_3d_online_log(ref, *U.shape, *outs, ctx=ctx)
        for x, y in zip(outs, dec):
            assert_bits_equal(x.cpu().numpy(), y)


def test_gpu_3d_rejects_bad_input(ctx):
    U, V, Wf = W.field_3d(1, 6, 6, 6, 2, 3.0)
    blob = cpsz_b200.sz_compress_cp_preserve_3d_offline_log(U, V, Wf, max_pwr_eb=0.1, ctx=ctx)
    with pytest.raises(cpsz_b200.CpszError):
        cpsz_b200.sz_decompress_cp_preserve_3d_online_log(blob[: len(blob) // 2], 6, 6, 6, ctx=ctx)
    with pytest.raises(cpsz_b200.CpszError):
        cpsz_b200.sz_decompress_cp_preserve_3d_online_log(blob, 6, 6, 7, ctx=ctx)
    # A flat field has no tets, so every vertex keeps max_pwr_eb: at 5 the id
    # (log2(log2 6 / 2^-23) = 24.4) reaches the reference's unpredictable
    # marker 24, which its decoder would misread; the GPU path refuses it.
    F = [np.ones((1, 6, 6), np.float32) for _ in range(3)]
    with pytest.raises(cpsz_b200.CpszError):
        cpsz_b200.sz_compress_cp_preserve_3d_offline_log(*F, max_pwr_eb=5.0, ctx=ctx)


def test_gpu_eb3d_nonfinite_and_overflow(ctx, oracle):
    """Triple products that overflow float, and NaN / inf inputs: the bound
    kernel's division-free and pruned paths fall back exactly."""
    rng = np.random.default_rng(8)
    shape = (9, 10, 11)
    U, V, Wf = (rng.normal(size=shape).astype(np.float32) for _ in range(3))
    U[2:4] *= 3e13  # products beyond FLT_MAX
    V[:, 5] *= 1e30
    Wf[5, 5, 5] = np.nan
    U[7, 1, 2] = np.inf
    for eb in (0.1, 0.9):
        e, ids = cpsz_b200.debug_eb3d(U, V, Wf, eb, ctx=ctx)
        ref = oracle.eb_3d(U, V, Wf, eb)
        assert np.isnan(ref).any()
        assert_bits_equal(e, ref, nan_equal=True)
        assert np.array_equal(ids == 255, ~(ref > 0))
    _check_roundtrip(ctx, oracle, U, V, Wf, 0.1)
