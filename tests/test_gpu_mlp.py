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
