"""The allocation-free Huffman packer (for callers that cannot allocate device
memory where they encode, e.g. an in-situ hook in a simulation that owns the
GPU's memory) must produce exactly the bytes of the context-based packer, on
repeated calls that reuse its fixed scratch array.  Kept in a file of its own
that pytest collects last."""
import ctypes

import numpy as np
import pytest

import cpsz_b200

pytestmark = pytest.mark.gpu


def _case(seed, n):
    rng = np.random.default_rng(seed)
    sym = (32768 + np.round(rng.standard_cauchy(n) * 30)).clip(1, 65535).astype(np.uint16)
    hist = np.bincount(sym, minlength=65536).astype(np.uint64)
    return sym, hist


def test_no_alloc_matches_context_encoder_twice():
    torch = pytest.importorskip("torch")
    ctx = cpsz_b200.Context(0)
    try:
        stream = torch.cuda.Stream()
        for seed, n in ((11, 1_000_003), (12, 250_000)):
            sym, hist = _case(seed, n)
            code, ln, _ = cpsz_b200.huffman_codebook(hist, 131072)
            d_sym = torch.from_numpy(sym.view(np.int16)).cuda()
            d_code = torch.from_numpy(code.view(np.int64)).cuda()
            d_len = torch.from_numpy(ln).cuda()
            cap = ((int((hist * ln.astype(np.uint64)).sum()) + 7) // 8 + 64) // 4 * 4
            ref = torch.zeros(cap, dtype=torch.uint8, device="cuda")
            ref_bits = cpsz_b200.huffman_encode_u16(d_sym, d_code, d_len, ref, ctx=ctx)
            for _ in range(2):  # two calls in a row share the scratch array
                out = torch.full((cap,), 0xAB, dtype=torch.uint8, device="cuda")
                bits = torch.zeros(1, dtype=torch.int64, device="cuda")
                with torch.cuda.stream(stream):
                    cpsz_b200.huffman_encode_u16_noalloc(d_sym, d_code, d_len, out, bits,
                                                         stream=stream.cuda_stream)
                stream.synchronize()
                assert int(bits.item()) == ref_bits
                assert torch.equal(out, ref)
    finally:
        ctx.close()


def test_no_alloc_rejects_oversized_stream():
    torch = pytest.importorskip("torch")
    buf = torch.zeros(64, dtype=torch.uint8, device="cuda")
    bits = torch.zeros(1, dtype=torch.int64, device="cuda")
    L = cpsz_b200.lib()
    # the size check runs before any device work, so the small buffers are never touched
    rc = L.cpsz_b200_huffman_encode_u16_noalloc(buf.data_ptr(), (1 << 26) + 1, buf.data_ptr(), buf.data_ptr(),
                                                buf.data_ptr(), 64, bits.data_ptr(), None)
    assert rc == 1
    assert b"exceed the no-alloc maximum" in L.cpsz_b200_last_error()


def test_no_alloc_capacity_rules():
    """out_cap must be a multiple of 4 (the packer stores whole words); a buffer
    short of the stream gets the stream's prefix and the full bit count, so the
    caller sees the overflow as (total_bits + 7) / 8 > out_cap."""
    torch = pytest.importorskip("torch")
    ctx = cpsz_b200.Context(0)
    try:
        sym, hist = _case(13, 300_001)
        code, ln, _ = cpsz_b200.huffman_codebook(hist, 131072)
        d_sym = torch.from_numpy(sym.view(np.int16)).cuda()
        d_code = torch.from_numpy(code.view(np.int64)).cuda()
        d_len = torch.from_numpy(ln).cuda()
        need = (int((hist * ln.astype(np.uint64)).sum()) + 7) // 8
        full = torch.zeros((need + 64) // 4 * 4, dtype=torch.uint8, device="cuda")
        ref_bits = cpsz_b200.huffman_encode_u16(d_sym, d_code, d_len, full, ctx=ctx)
        bits = torch.zeros(1, dtype=torch.int64, device="cuda")
        odd = torch.zeros(need + 3 - (need + 3) % 4 + 2, dtype=torch.uint8, device="cuda")
        with pytest.raises(cpsz_b200.CpszError) as ei:
            cpsz_b200.huffman_encode_u16_noalloc(d_sym, d_code, d_len, odd, bits)
        assert ei.value.code == 1 and "multiple of 4" in str(ei.value)
        short_cap = (need - 1) // 4 * 4  # one to four bytes short of the stream
        short = torch.full((short_cap,), 0xAB, dtype=torch.uint8, device="cuda")
        cpsz_b200.huffman_encode_u16_noalloc(d_sym, d_code, d_len, short, bits)
        torch.cuda.synchronize()
        assert int(bits.item()) == ref_bits
        assert (int(bits.item()) + 7) // 8 > short_cap
        assert torch.equal(short, full[:short_cap])
    finally:
        ctx.close()
