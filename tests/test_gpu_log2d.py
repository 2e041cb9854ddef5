"""The 2D offline_log pair on the GPU against the reference's fixtures and the
oracle: blob bytes (meanInfo padding masked), decoded fields bit for bit, and
the decode's critical points and relative bound."""
import numpy as np
import pytest

import cpsz_b200
from cpsz_b200 import workloads as W
from tests._util import assert_bits_equal, assert_blob_equal_2d_log, golden_cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", golden_cases("2dlog_"), ids=lambda p: p.split("/")[-1])
def test_gpu_log_matches_reference_fixture(ctx, path):
    g = np.load(path)
    U, V, eb = g["U"], g["V"], float(g["eb"])
    blob = cpsz_b200.sz_compress_cp_preserve_2d_offline_log(U, V, max_pwr_eb=eb, ctx=ctx)
    assert_blob_equal_2d_log(blob, g["blob"].tobytes(), U.size)
    du, dv = cpsz_b200.sz_decompress_cp_preserve_2d_offline_log(g["blob"].tobytes(), *U.shape, ctx=ctx)
    assert_bits_equal(du, g["dU"])
    assert_bits_equal(dv, g["dV"])


SHAPES = [(1, 1), (1, 2), (2, 1), (2, 2), (1, 300), (300, 1), (3, 4097), (13, 17), (255, 257), (511, 33),
          (600, 700)]


def _field(r1, r2, seed):
    U, V = W.cfg0_like(seed, r1, r2)
    U.ravel()[::9] = 0          # log -100, sign bit 0
    V.ravel()[1::7] *= 1e-30    # tiny magnitudes
    V.ravel()[::17] = 0
    return U, V


@pytest.mark.parametrize("r1,r2", SHAPES)
@pytest.mark.parametrize("eb", [0.1, 0.01])
def test_gpu_log_equals_oracle(ctx, oracle, r1, r2, eb):
    U, V = _field(r1, r2, r1 * 31 + r2)
    a = cpsz_b200.sz_compress_cp_preserve_2d_offline_log(U, V, max_pwr_eb=eb, ctx=ctx)
    b = oracle.compress_2d_log(U, V, eb)
    assert_blob_equal_2d_log(a, b, U.size)
    du, dv = cpsz_b200.sz_decompress_cp_preserve_2d_offline_log(a, r1, r2, ctx=ctx)
    ou, ov = oracle.decompress_2d_log(b, r1, r2)
    assert_bits_equal(du, ou)
    assert_bits_equal(dv, ov)


def test_gpu_log_cfg0_full_size_and_io_kinds(ctx, oracle):
    torch = pytest.importorskip("torch")
    U, V = W.cfg0(0)
    eb = 0.1
    ref = oracle.compress_2d_log(U, V, eb)
    n = U.size
    a = cpsz_b200.sz_compress_cp_preserve_2d_offline_log(U, V, max_pwr_eb=eb, ctx=ctx)
    assert_blob_equal_2d_log(a, ref, n)
    dU, dV = torch.from_numpy(U).cuda(), torch.from_numpy(V).cuda()
    d_out = torch.zeros(len(ref) + 4096, dtype=torch.uint8, device="cuda")
    k = cpsz_b200.compress_2d_log_into(dU, dV, *U.shape, eb, d_out, ctx=ctx)
    assert_blob_equal_2d_log(d_out[:k].cpu().numpy().tobytes(), ref, n)
    h_out = torch.zeros(len(ref) + 4096, dtype=torch.uint8).pin_memory()
    k = cpsz_b200.compress_2d_log_into(U, V, *U.shape, eb, h_out.numpy(), ctx=ctx)
    assert_blob_equal_2d_log(h_out.numpy()[:k].tobytes(), ref, n)
    du, dv = cpsz_b200.sz_decompress_cp_preserve_2d_offline_log(a, *U.shape, ctx=ctx)
    ou, ov = oracle.decompress_2d_log(ref, *U.shape)
    assert_bits_equal(du, ou)
    assert_bits_equal(dv, ov)
    r = cpsz_b200.cp_check_2d(U, V, du, dv, ctx=ctx)
    assert r["cps_a"] > 0 and r["lost_or_spurious"] == 0 and r["type_changed"] == 0, r
    # relative bound in the log domain: |log2|d| - log2|x|| <= log2(1 + eb), signs and zeros kept
    for x, d in ((U, du), (V, dv)):
        x64, d64 = x.astype(np.float64), d.astype(np.float64)
        assert np.array_equal(np.sign(x64), np.sign(d64))
        nz = x64 != 0
        assert (np.abs(d64[nz] - x64[nz]) <= eb * np.abs(x64[nz]) * (1 + 2.0 ** -20)).all()


def test_gpu_log_rejects_an_offline_blob(ctx):
    U, V = W.cfg0_like(5, 40, 50)
    blob = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=ctx)
    with pytest.raises(cpsz_b200.CpszError):
        cpsz_b200.sz_decompress_cp_preserve_2d_offline_log(blob, 40, 50, ctx=ctx)
