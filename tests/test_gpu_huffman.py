"""The Huffman stage alone: codebook (host) and GPU bit packing vs the oracle."""
import numpy as np
import pytest

import cpsz_b200

pytestmark = pytest.mark.gpu


def _streams():
    rng = np.random.default_rng(3)
    yield rng.integers(32768 - 40, 32768 + 40, 100_000).astype(np.int32)
    # a skewed stream with many distinct symbols and long codes
    yield (32768 + np.round(rng.standard_cauchy(300_000) * 20)).clip(1, 65535).astype(np.int32)
    yield np.full(5000, 32768, np.int32)  # single symbol: empty bit stream
    yield rng.integers(0, 65536, 70_000).astype(np.int32)


@pytest.mark.parametrize("k", range(4))
def test_gpu_huffman_matches_oracle(ctx, oracle, k):
    torch = pytest.importorskip("torch")
    sym = list(_streams())[k]
    hist = np.bincount(sym, minlength=65536).astype(np.uint64)
    code, ln, tree = cpsz_b200.huffman_codebook(hist, 131072)
    ref = oracle.huffman_encode(131072, sym)
    assert ref[: len(tree)] == tree
    nbytes = int.from_bytes(ref[len(tree): len(tree) + 8], "little")
    d_sym = torch.from_numpy(sym.astype(np.uint16)).cuda()
    d_code = torch.from_numpy(code.view(np.int64)).cuda()
    d_len = torch.from_numpy(ln).cuda()
    out = torch.zeros(nbytes + 64, dtype=torch.uint8, device="cuda")
    bits = cpsz_b200.huffman_encode_u16(d_sym, d_code, d_len, out, ctx=ctx)
    assert (bits + 7) // 8 == nbytes
    assert out[:nbytes].cpu().numpy().tobytes() == ref[len(tree) + 8:]


def _fib_stream(rng, n):
    """Symbols 32768 + i with Fibonacci counts, largest first: with 34 symbols
    (14.9 M in all) the reference's tree gives the two rarest 33-bit codes, so
    the few packing tiles that hold one take the long-code path."""
    f = [1, 1]
    while len(f) < n:
        f.append(f[-1] + f[-2])
    sym = np.repeat(32768 + np.arange(n, dtype=np.int32), f[::-1])
    rng.shuffle(sym)
    return sym


def _check_packing(ctx, oracle, sym, offset=0):
    torch = pytest.importorskip("torch")
    hist = np.bincount(sym, minlength=65536).astype(np.uint64)
    code, ln, tree = cpsz_b200.huffman_codebook(hist, 131072)
    ref = oracle.huffman_encode(131072, sym)
    assert ref[: len(tree)] == tree
    nbytes = int.from_bytes(ref[len(tree): len(tree) + 8], "little")
    # `offset` leading symbols shift the stream off the 16-byte grid
    d_all = torch.from_numpy(np.concatenate([np.zeros(offset, np.uint16), sym.astype(np.uint16)])).cuda()
    d_sym = d_all[offset:]
    out = torch.zeros(nbytes + 64, dtype=torch.uint8, device="cuda")
    bits = cpsz_b200.huffman_encode_u16(d_sym, torch.from_numpy(code.view(np.int64)).cuda(),
                                        torch.from_numpy(ln).cuda(), out, ctx=ctx)
    assert (bits + 7) // 8 == nbytes
    got = out[:nbytes].cpu().numpy().tobytes()
    want = ref[len(tree) + 8:]
    if got != want:
        a, b = np.frombuffer(got, np.uint8), np.frombuffer(want, np.uint8)
        raise AssertionError(f"bit streams differ from byte {int(np.flatnonzero(a != b)[0])} of {nbytes}")
    return int(ln.max())


def test_gpu_huffman_many_tiles(ctx, oracle):
    # 3.3 M symbols: ~400 packing tiles, so starting bits come from look-backs
    # over several windows of earlier tiles; the last tile is ragged
    rng = np.random.default_rng(11)
    sym = (32768 + np.round(rng.laplace(0, 2.5, 3_300_001))).clip(1, 65535).astype(np.int32)
    _check_packing(ctx, oracle, sym)


def test_gpu_huffman_long_codes(ctx, oracle):
    sym = _fib_stream(np.random.default_rng(12), 34)
    assert _check_packing(ctx, oracle, sym) > 32


@pytest.mark.parametrize("offset", [1, 3])
def test_gpu_huffman_unaligned_symbols(ctx, oracle, offset):
    rng = np.random.default_rng(13)
    sym = (32768 + np.round(rng.laplace(0, 30, 200_003))).clip(1, 65535).astype(np.int32)
    _check_packing(ctx, oracle, sym, offset)


def test_gpu_huffman_rejects_small_output(ctx):
    torch = pytest.importorskip("torch")
    sym = np.random.default_rng(1).integers(100, 5000, 50_000).astype(np.int32)
    hist = np.bincount(sym, minlength=65536).astype(np.uint64)
    code, ln, tree = cpsz_b200.huffman_codebook(hist, 131072)
    out = torch.zeros(64, dtype=torch.uint8, device="cuda")
    with pytest.raises(cpsz_b200.CpszError):
        cpsz_b200.huffman_encode_u16(torch.from_numpy(sym.astype(np.uint16)).cuda(),
                                     torch.from_numpy(code.view(np.int64)).cuda(), torch.from_numpy(ln).cuda(), out,
                                     ctx=ctx)
