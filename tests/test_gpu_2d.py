"""2D offline path on the GPU vs the oracle: blob bytes, decoded fields and the
intermediate streams, bit-exact (integer/byte data compared exactly, floats by bit pattern)."""
import numpy as np
import pytest

import cpsz_b200
from cpsz_b200 import workloads as W
from tests._util import assert_bits_equal, assert_blob_equal_2d, golden_cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", golden_cases("2d_"), ids=lambda p: p.split("/")[-1])
def test_gpu_matches_reference_fixture(ctx, path):
    g = np.load(path)
    U, V, eb = g["U"], g["V"], float(g["eb"])
    blob = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=eb, ctx=ctx)
    assert_blob_equal_2d(blob, g["blob"].tobytes())
    du, dv = cpsz_b200.sz_decompress_cp_preserve_2d_offline(g["blob"].tobytes(), *U.shape, ctx=ctx)
    assert_bits_equal(du, g["dU"])
    assert_bits_equal(dv, g["dV"])


SHAPES = [(1, 1), (1, 2), (2, 1), (2, 2), (1, 300), (300, 1), (3, 4097), (4097, 3), (13, 17), (255, 257),
          (256, 256), (257, 255), (511, 33), (600, 700)]


@pytest.mark.parametrize("r1,r2", SHAPES)
@pytest.mark.parametrize("eb", [0.1, 0.01])
def test_gpu_blob_equals_oracle(ctx, oracle, r1, r2, eb):
    U, V = W.cfg0_like(r1 * 7919 + r2, r1, r2)
    a = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=eb, ctx=ctx)
    b = oracle.compress_2d(U, V, eb)
    assert_blob_equal_2d(a, b)
    du, dv = cpsz_b200.sz_decompress_cp_preserve_2d_offline(a, r1, r2, ctx=ctx)
    ou, ov = oracle.decompress_2d(b, r1, r2)
    assert_bits_equal(du, ou)
    assert_bits_equal(dv, ov)


def test_gpu_stages_equal_oracle(ctx, oracle):
    r1, r2, eb = 345, 678, 0.1
    U, V = W.cfg0_like(42, r1, r2)
    st = cpsz_b200.compress_2d_stages(U, V, eb, ctx=ctx)
    e = oracle.eb_2d(U, V, eb)
    ids, eu, ev = oracle.quantize_eb_2d(U, V, e)
    assert np.array_equal(st["ids"], ids)
    for data, prec, key, rkey in ((U, eu, "codes_u", "recon_u"), (V, ev, "codes_v", "recon_v")):
        t, up, rec = oracle.lorenzo_2d(data, prec.reshape(data.shape))
        assert np.array_equal(st[key], t)
        assert_bits_equal(st[rkey], rec)


def test_gpu_cfg0_full_size(ctx, oracle):
    U, V = W.cfg0(0)
    a = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=ctx)
    b = oracle.compress_2d(U, V, 0.1)
    assert_blob_equal_2d(a, b)
    du, dv = cpsz_b200.sz_decompress_cp_preserve_2d_offline(a, *U.shape, ctx=ctx)
    ou, ov = oracle.decompress_2d(b, *U.shape)
    assert_bits_equal(du, ou)
    assert_bits_equal(dv, ov)


def test_gpu_device_resident_inputs(ctx, oracle):
    torch = pytest.importorskip("torch")
    U, V = W.cfg0_like(7, 500, 400)
    dU = torch.from_numpy(U).cuda()
    dV = torch.from_numpy(V).cuda()
    a = cpsz_b200.sz_compress_cp_preserve_2d_offline(dU, dV, max_pwr_eb=0.1, ctx=ctx)
    assert_blob_equal_2d(a, oracle.compress_2d(U, V, 0.1))
    oU = torch.empty_like(dU)
    oV = torch.empty_like(dV)
    cpsz_b200.sz_decompress_cp_preserve_2d_offline(a, 500, 400, oU, oV, ctx=ctx)
    torch.cuda.synchronize()
    ou, ov = oracle.decompress_2d(a, 500, 400)
    assert_bits_equal(oU.cpu().numpy(), ou)
    assert_bits_equal(oV.cpu().numpy(), ov)


def test_gpu_constant_and_zero_fields(ctx, oracle):
    for U in (np.zeros((40, 50), np.float32), np.full((40, 50), 0.5, np.float32)):
        V = U.copy()
        a = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=ctx)
        assert_blob_equal_2d(a, oracle.compress_2d(U, V, 0.1))
        du, dv = cpsz_b200.sz_decompress_cp_preserve_2d_offline(a, 40, 50, ctx=ctx)
        ou, ov = oracle.decompress_2d(a, 40, 50)
        assert_bits_equal(du, ou)


def test_gpu_rejects_corrupt_blobs(ctx):
    U, V = W.cfg0_like(9, 64, 64)
    blob = bytearray(cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=ctx))
    with pytest.raises(cpsz_b200.CpszError):
        cpsz_b200.sz_decompress_cp_preserve_2d_offline(bytes(blob[: len(blob) // 2]), 64, 64, ctx=ctx)
    bad = bytearray(blob)
    bad[12:20] = (10 ** 12).to_bytes(8, "little")  # absurd id-section size
    with pytest.raises(cpsz_b200.CpszError):
        cpsz_b200.sz_decompress_cp_preserve_2d_offline(bytes(bad), 64, 64, ctx=ctx)
    # the context is still usable afterwards
    du, dv = cpsz_b200.sz_decompress_cp_preserve_2d_offline(bytes(blob), 64, 64, ctx=ctx)
    assert np.isfinite(du).all()


def test_gpu_eb2d_nonfinite_signed_zero_and_overflow(ctx, oracle):
    """Products beyond FLT_MAX, NaN / inf inputs, signed zeros and exact ties:
    the bound kernel's division-free flags and pruned sign bounds fall back to
    the literal arithmetic exactly."""
    rng = np.random.default_rng(12)
    shape = (40, 45)
    U = rng.normal(size=shape).astype(np.float32)
    V = rng.normal(size=shape).astype(np.float32)
    U[5:8] *= 3e30
    V[:, 7] *= 2e25
    U[10, 10] = np.nan
    V[20, 3] = np.inf
    U[25:30, 25:30] = -0.0
    V[25:30, 27] = 0.0
    U[33:, :] = np.round(U[33:, :] * 2) / 2  # repeated values -> exact ties
    V[33:, :] = np.round(V[33:, :] * 2) / 2
    for eb in (0.1, 0.01):
        e, ids = cpsz_b200.debug_eb2d(U, V, eb, ctx=ctx)
        assert_bits_equal(e.ravel(), oracle.eb_2d(U, V, eb).ravel(), nan_equal=True)
    # A NaN bound (NaN / inf input, or products beyond FLT_MAX) has no
    # quantization id: the reference indexes out of range, the GPU path reports
    # unsupported input.  Whole blobs are compared for large but finite products.
    with pytest.raises(cpsz_b200.CpszError):
        cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=ctx)
    U[10, 10] = 1.5
    V[20, 3] = -2.5
    U[5:8] /= 1e12
    V[:, 7] /= 1e7
    blob = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=ctx)
    assert_blob_equal_2d(blob, oracle.compress_2d(U, V, 0.1))


def test_gpu_wavefront_wait_that_gives_up_reruns(oracle):
    """The wavefront beside the bound kernel waits (bounded) per row group for
    its bounds.  With every such wait made to run out (target one point more
    than a group holds, 1 ms limit), the pass runs its wavefront again after
    the bounds and still returns the oracle's blob."""
    torch = pytest.importorskip("torch")
    c = cpsz_b200.Context(0)  # own context: the setting stays off the shared one
    try:
        c.debug_band_wait(1_000_000, unreachable=True)
        # sizes at which the launch-shape table runs the wavefront beside the bounds
        for r1, r2, seed, dev in ((1000, 1100, 5, False), (1500, 1300, 6, False), (700, 900, 7, True)):
            U, V = W.cfg0_like(seed, r1, r2)
            n0 = c.wave_reruns
            if dev:
                a = cpsz_b200.sz_compress_cp_preserve_2d_offline(torch.from_numpy(U).cuda(),
                                                                 torch.from_numpy(V).cuda(), max_pwr_eb=0.1, ctx=c)
            else:
                a = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=c)
            assert c.wave_reruns == n0 + 1
            assert_blob_equal_2d(a, oracle.compress_2d(U, V, 0.1))
        c.debug_band_wait(0, unreachable=False)
        U, V = W.cfg0_like(8, 640, 480)
        n0 = c.wave_reruns
        a = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=c)
        assert c.wave_reruns == n0
        assert_blob_equal_2d(a, oracle.compress_2d(U, V, 0.1))
    finally:
        c.close()


def test_gpu_histogram_follower_that_gives_up_recounts(oracle):
    """A field compressed beside its bounds has its code histograms counted
    while the wavefront finishes its row groups.  With the wavefront held back
    past the follower's 100 ms wait (its own wait for the bounds made to run
    out after 300 ms), the follower gives up, the pass counts the histograms
    after the wavefront, runs the wavefront again and returns the oracle's blob."""
    import time

    c = cpsz_b200.Context(0)
    try:
        c.debug_band_wait(300_000_000, unreachable=True)
        U, V = W.cfg0_like(9, 1000, 1100)
        n0 = c.wave_reruns
        t0 = time.perf_counter()
        a = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=c)
        assert time.perf_counter() - t0 > 0.25
        assert c.wave_reruns == n0 + 1
        assert_blob_equal_2d(a, oracle.compress_2d(U, V, 0.1))
    finally:
        c.close()


def test_gpu_serialised_launches_still_compress(tmp_path):
    """With every launch serialised (CUDA_LAUNCH_BLOCKING=1, as under tools that
    run kernels one at a time) the wavefront waits for bounds that no kernel
    is computing: its wait gives up after 50 ms without progress, the pass
    runs the wavefront again after the bounds, and the blob equals the
    oracle's.  Runs in a child process so the setting applies from CUDA's start."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys; sys.path.insert(0, sys.argv[1]);"
        "import cpsz_b200; from cpsz_b200 import workloads as W; from oracle import Oracle;"
        "from tests._util import assert_blob_equal_2d;"
        "c = cpsz_b200.Context(0); U, V = W.cfg0_like(9, 1100, 900);"
        "import time; t = time.perf_counter();"
        "a = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=c);"
        "print('seconds', time.perf_counter() - t);"
        "assert_blob_equal_2d(a, Oracle().compress_2d(U, V, 0.1));"
        "print('reruns', c.wave_reruns)"
    )
    env = dict(os.environ, CUDA_LAUNCH_BLOCKING="1")
    r = subprocess.run([sys.executable, "-c", code, root], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "reruns 1" in r.stdout
    assert float(r.stdout.split("seconds")[1].split()[0]) < 3.0  # the wait, not a 4-second timeout
