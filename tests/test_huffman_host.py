"""Host Huffman tree construction (CPU): serialized tree and code lengths of
the library's builder equal the oracle's restatement of the reference's
heap-based builder (src/sz_huffman.cpp:103-215) on assorted histograms."""
import numpy as np
import pytest

import cpsz_b200


def _streams():
    rng = np.random.default_rng(5)
    yield 131072, rng.integers(32768 - 40, 32768 + 40, 100_000)
    yield 131072, (32768 + np.round(rng.standard_cauchy(300_000) * 20)).clip(1, 65535)
    yield 131072, (32768 + np.round(rng.laplace(0, 5000, 1_000_000))).clip(1, 65535)
    yield 131072, np.full(5000, 32768)
    yield 131072, rng.integers(0, 65536, 70_000)
    yield 131072, np.repeat(np.arange(1, 65536, 7), 3)  # many equal frequencies
    yield 512, rng.integers(0, 25, 50_000)
    yield 512, np.array([0])
    yield 2048, rng.integers(0, 89, 200_000)


@pytest.mark.parametrize("k", range(9))
def test_tree_bytes_and_lengths_equal_oracle(oracle, k):
    state, sym = list(_streams())[k]
    sym = np.asarray(sym, np.int32)
    bins = 65536 if state == 131072 else 256
    hist = np.bincount(sym, minlength=bins).astype(np.uint64)
    code, ln, tree = cpsz_b200.huffman_codebook(hist, state)
    ref = oracle.huffman_encode(state, sym)
    assert ref[: len(tree)] == tree
    ref_len = oracle.huffman_code_lengths(state, sym)
    assert np.array_equal(ln, ref_len[:bins])
    nbytes = int.from_bytes(ref[len(tree): len(tree) + 8], "little")
    total = int((hist * ln.astype(np.uint64)).sum())
    assert (total + 7) // 8 == nbytes
