"""Tensor-core (tcgen05) building blocks and the learned-bound MLP against
FP32 references of the same arithmetic."""
import numpy as np
import pytest

import cpsz_b200

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [0, 1])
def test_umma_tile_gemm_matches_fp32(ctx, seed):
    rng = np.random.default_rng(seed)
    A = cpsz_b200.to_bf16_bits(rng.normal(size=(128, 128)))
    B = cpsz_b200.to_bf16_bits(rng.normal(size=(128, 128)))
    D = cpsz_b200.debug_umma_gemm(A, B, ctx=ctx)
    ref = cpsz_b200.bf16_bits_to_f32(A).astype(np.float64) @ cpsz_b200.bf16_bits_to_f32(B).astype(np.float64).T
    np.testing.assert_allclose(D, ref, rtol=1e-5, atol=1e-4)


def test_umma_tile_gemm_structured(ctx):
    # identity times a matrix: exact, and shows the operand layouts are not transposed
    A = cpsz_b200.to_bf16_bits(np.eye(128))
    M = np.arange(128 * 128, dtype=np.float64).reshape(128, 128) % 251 - 125
    B = cpsz_b200.to_bf16_bits(M)
    D = cpsz_b200.debug_umma_gemm(A, B, ctx=ctx)
    np.testing.assert_array_equal(D, M.T)


from cpsz_b200 import workloads as W  # noqa: E402
from oracle import cp_exact, mlp_ref  # noqa: E402


def _mlp_and_data(ctx, n, seed=3):
    rng = np.random.default_rng(seed)
    mlp = cpsz_b200.Mlp(ctx, seed=seed)
    p = mlp.params()
    p[33152] = 0.5  # nonzero b3
    p[16384:16512] = rng.normal(size=128) * 0.1
    p[32896:33024] = rng.normal(size=128) * 0.1
    mlp.set_params(p)
    Xf = np.zeros((n, 128), np.float32)
    Xf[:, :99] = rng.normal(size=(n, 99))
    X = cpsz_b200.to_bf16_bits(Xf)
    return mlp, mlp.params(), X, cpsz_b200.bf16_bits_to_f32(X).reshape(n, 128)


@pytest.mark.parametrize("n", [1, 127, 1000, 70000])
def test_mlp_forward_matches_fp32_reference(ctx, n):
    mlp, p, X, Xf = _mlp_and_data(ctx, n)
    y = mlp.forward(X)
    ref, _, _ = mlp_ref.forward(p, Xf)
    np.testing.assert_allclose(y, ref, rtol=2e-3, atol=2e-3 * max(1.0, np.abs(ref).max()))


@pytest.mark.parametrize("n", [200, 5000])
def test_mlp_gradients_match_fp32_reference(ctx, n):
    mlp, p, X, Xf = _mlp_and_data(ctx, n, seed=7)
    t = np.random.default_rng(1).normal(size=n).astype(np.float32)
    loss, g = mlp.train_step(X, t, lr=0.0, grads=True)
    gref, lref = mlp_ref.gradients(p, Xf, t)
    assert abs(loss - lref) <= 1e-3 * max(1.0, lref)
    scale = np.abs(gref).max()
    for lo, hi in ((0, 16384), (16384, 16512), (16512, 32896), (32896, 33024), (33024, 33152), (33152, 33153)):
        np.testing.assert_allclose(g[lo:hi], gref[lo:hi], rtol=5e-3, atol=5e-3 * scale)


def test_mlp_training_reduces_loss(ctx):
    mlp, p, X, Xf = _mlp_and_data(ctx, 8192, seed=11)
    t = (np.tanh(Xf[:, 0] - 0.5 * Xf[:, 1]) * 3 + 4).astype(np.float32)
    first = None
    for _ in range(300):
        loss, _ = mlp.train_step(X, t, lr=3e-3)
        first = loss if first is None else first
    assert loss < 0.2 * first


def test_mlp_features_match_reference(ctx, oracle):
    U, V = W.cfg0_like(5, 60, 70)
    eb = oracle.eb_2d(U, V, 0.1).ravel()
    idx = np.array([0, 1, 69, 70, 71, 1000, 2099, 4199, 3000], np.int32)
    X = cpsz_b200.mlp_features_2d(U, V, eb, idx, ctx=ctx)
    ref = cpsz_b200.to_bf16_bits(mlp_ref.features(U, V, eb, idx))
    assert np.array_equal(X, ref)


@pytest.mark.parametrize("shape", [(300, 257), (61, 1030)])
def test_mlp_field_proposals_equal_feature_path(ctx, oracle, shape):
    """The proposer over a whole field (features built on the device, two
    128-row tiles in flight per CTA) gives bit for bit the floats of the
    feature rows of every vertex run through the plain forward pass."""
    U, V = W.cfg0_like(9, *shape)
    eb = oracle.eb_2d(U, V, 0.1).ravel()
    mlp = cpsz_b200.Mlp(ctx, seed=3)
    y = cpsz_b200.mlp_propose_2d(mlp, U, V, eb)
    X = cpsz_b200.mlp_features_2d(U, V, eb, np.arange(U.size, dtype=np.int32), ctx=ctx)
    ref = np.asarray(mlp.forward(X), np.float32).ravel()
    assert np.array_equal(y.ravel().view(np.uint32), ref.view(np.uint32))


def _label_ref(U, V, eb, v, steps=16, tmax=16.0):
    r1, r2 = U.shape
    i, j = divmod(v, r2)
    inc = [(0, 0, 0, 0), (0, 0, 1, 0), (-1, 0, 0, 1), (-1, -1, 0, 2), (-1, -1, 1, 2), (0, -1, 1, 1)]
    tris = []
    for di, dj, k, pos in inc:
        ci, cj = i + di, j + dj
        if ci < 0 or cj < 0 or ci > r1 - 2 or cj > r2 - 2:
            continue
        pts = [(ci, cj), (ci + (k == 0), cj + (k == 1)), (ci + 1, cj + 1)]
        vals = [(float(U[a, b]), float(V[a, b])) for a, b in pts]
        tris.append((vals, k, pos, cp_exact.tri_code(vals, k)))
    u0, v0, e0 = float(U[i, j]), float(V[i, j]), float(eb[v])
    lo, hi = np.float32(0), np.float32(tmax)
    for _ in range(steps):
        mid = np.float32(0.5) * (lo + hi)
        e = e0 * 2.0 ** float(mid)
        ok = True
        for c in range(4):
            cu = float(np.float32(u0 + (1 if c & 1 else -1) * abs(u0) * e))
            cv = float(np.float32(v0 + (1 if c & 2 else -1) * abs(v0) * e))
            for vals, k, pos, orig in tris:
                vv = list(vals)
                vv[pos] = (cu, cv)
                if cp_exact.tri_code(vv, k) != orig:
                    ok = False
        if ok:
            lo = mid
        else:
            hi = mid
    return float(lo)


def test_learned_labels_match_reference(ctx, oracle):
    U, V = W.cfg0_like(9, 40, 50)
    eb = oracle.eb_2d(U, V, 0.1).ravel()
    idx = np.array([0, 49, 51, 520, 1000, 1234, 1999], np.int32)
    t = cpsz_b200.learned_labels_2d(U, V, eb, idx, ctx=ctx)
    for s, v in enumerate(idx):
        assert t[s] == pytest.approx(_label_ref(U, V, eb, int(v)), abs=0), v


@pytest.mark.parametrize("mult", [1.0, 4.0])
def test_learned_compress_keeps_every_cp(ctx, oracle, mult):
    U, V = W.cfg0_like(31, 500, 600)
    plain = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=ctx)
    blob, st = cpsz_b200.compress_2d_learned(U, V, 0.1, log2_mult=np.full(U.shape, mult, np.float32), ctx=ctx)
    dU, dV = cpsz_b200.sz_decompress_cp_preserve_2d_offline(blob, *U.shape, ctx=ctx)
    r = cpsz_b200.cp_check_2d(U, V, dU, dV, ctx=ctx)
    assert r["lost_or_spurious"] == 0 and r["type_changed"] == 0, (r, st)
    assert st["fell_back"] == 0 and st["kept"] > 0
    assert len(blob) < len(plain)
    # the oracle decodes it too
    ou, ov = oracle.decompress_2d(blob, *U.shape)
    assert np.array_equal(ou.view(np.uint32), dU.view(np.uint32))


def test_learned_compress_with_mlp(ctx):
    U, V = W.cfg0_like(32, 300, 400)
    mlp = cpsz_b200.Mlp(ctx, seed=1)
    blob, st = cpsz_b200.compress_2d_learned(U, V, 0.1, mlp=mlp, ctx=ctx)
    dU, dV = cpsz_b200.sz_decompress_cp_preserve_2d_offline(blob, *U.shape, ctx=ctx)
    r = cpsz_b200.cp_check_2d(U, V, dU, dV, ctx=ctx)
    assert r["lost_or_spurious"] == 0 and r["type_changed"] == 0, (r, st)


def _within_relative_bound(x, d, eb):
    x64 = x.astype(np.float64)
    return int(np.count_nonzero(np.abs(d.astype(np.float64) - x64) > eb * np.abs(x64)))


def test_trained_proposer_gains_over_plain(ctx, oracle):
    """The committed proposer (trained on seeds 1000-1063, margin chosen on seed
    99991) on a held-out 2048^2 field of the same generator: a smaller ZSTD'd
    blob than the plain compressor's, no critical point lost, added or
    retyped, every point within max_pwr_eb of its value, and the blob decodes
    identically through the plain decoder of the oracle."""
    from cpsz_b200 import learned

    U, V = W.cfg0_like(123457, 2048, 2048)
    eb = 0.1
    mlp = learned.load(ctx)
    try:
        plain = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=eb, ctx=ctx)
        blob, st = cpsz_b200.compress_2d_learned(U, V, eb, mlp=mlp, ctx=ctx)
    finally:
        mlp.close()
    dU, dV = cpsz_b200.sz_decompress_cp_preserve_2d_offline(blob, *U.shape, ctx=ctx)
    r = cpsz_b200.cp_check_2d(U, V, dU, dV, ctx=ctx)
    assert r["cps_a"] > 0
    assert r["lost_or_spurious"] == 0 and r["type_changed"] == 0, (r, st)
    assert _within_relative_bound(U, dU, eb) == 0 and _within_relative_bound(V, dV, eb) == 0
    z_plain = len(cpsz_b200.sz_lossless_compress(plain, 3))
    z_learned = len(cpsz_b200.sz_lossless_compress(blob, 3))
    raw = U.nbytes + V.nbytes
    print(f"held-out 2048^2: ratio plain {raw / z_plain:.3f}, learned {raw / z_learned:.3f}; {st}")
    assert z_learned < z_plain
    ou, ov = oracle.decompress_2d(blob, *U.shape)
    assert np.array_equal(ou.view(np.uint32), dU.view(np.uint32))
    assert np.array_equal(ov.view(np.uint32), dV.view(np.uint32))


def test_learned_bounds_never_exceed_max_pwr_eb(ctx):
    """Multipliers far beyond any useful size are capped at max_pwr_eb: the
    decode keeps the plain compressor's point-wise relative bound."""
    U, V = W.cfg0_like(33, 400, 500)
    for eb in (0.1, 0.01):
        blob, st = cpsz_b200.compress_2d_learned(U, V, eb, log2_mult=np.full(U.shape, 16.0, np.float32), ctx=ctx)
        dU, dV = cpsz_b200.sz_decompress_cp_preserve_2d_offline(blob, *U.shape, ctx=ctx)
        assert _within_relative_bound(U, dU, eb) == 0 and _within_relative_bound(V, dV, eb) == 0
        r = cpsz_b200.cp_check_2d(U, V, dU, dV, ctx=ctx)
        assert r["lost_or_spurious"] == 0 and r["type_changed"] == 0, (r, st)
