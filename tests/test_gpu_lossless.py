"""The GPU lossless stage writes standard Zstandard frames: the system libzstd
(the decoder behind the reference's sz_lossless_decompress) reads every frame
back to the input bytes, from host and device buffers, for empty, one-byte,
constant (RLE), incompressible and real compressor blobs."""
import numpy as np
import pytest

import cpsz_b200
from cpsz_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _roundtrip(data: bytes, ctx):
    frame = cpsz_b200.lossless_compress_gpu(data, ctx=ctx)
    assert cpsz_b200.sz_lossless_decompress(frame, len(data)) == data
    return frame


def test_small_and_degenerate_inputs(ctx):
    rng = np.random.default_rng(0)
    for data in (b"", b"\x07", bytes(100000), bytes(32768 * 3), rng.integers(0, 256, 200001, np.uint8).tobytes(),
                 (b"abcd" * 50000)[:199999]):
        frame = _roundtrip(data, ctx)
        assert len(frame) <= cpsz_b200.lib().cpsz_b200_lossless_bound(len(data))


def test_compressor_blobs_shrink(ctx, reference):
    U, V = W.cfg0_like(21, 1500, 1700)
    for eb in (0.1, 0.01):
        blob = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=eb, ctx=ctx)
        frame = _roundtrip(blob, ctx)
        assert len(frame) < 0.9 * len(blob)
        # the reference's own lossless decoder reads it
        assert reference.zstd_decompress(frame, len(blob)) == blob


def test_device_buffers(ctx):
    torch = pytest.importorskip("torch")
    U, V = W.cfg0_like(22, 900, 800)
    blob = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=ctx)
    d_in = torch.from_numpy(np.frombuffer(blob, np.uint8).copy()).cuda()
    d_out = torch.zeros(cpsz_b200.lib().cpsz_b200_lossless_bound(len(blob)), dtype=torch.uint8, device="cuda")
    n = cpsz_b200.lossless_compress_gpu(d_in, out=d_out, ctx=ctx)
    frame = d_out[:n].cpu().numpy().tobytes()
    assert frame == cpsz_b200.lossless_compress_gpu(blob, ctx=ctx)
    assert cpsz_b200.sz_lossless_decompress(frame, len(blob)) == blob
    small = torch.zeros(16, dtype=torch.uint8, device="cuda")
    with pytest.raises(cpsz_b200.CpszError):
        cpsz_b200.lossless_compress_gpu(d_in, out=small, ctx=ctx)
