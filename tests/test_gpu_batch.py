"""Batched 2D compression: every blob of a batch is byte-identical to the
single-field compressor's blob of that field (and to the oracle's)."""
import numpy as np
import pytest

import cpsz_b200
from cpsz_b200 import workloads as W
from tests._util import assert_blob_equal_2d

pytestmark = pytest.mark.gpu


def _batch(n, seed, lo, hi):
    rng = np.random.default_rng(seed)
    fields, ebs = [], []
    for k in range(n):
        r1, r2 = (int(x) for x in rng.integers(lo, hi + 1, 2))
        fields.append(W.cfg0_like(seed * 1000 + k, r1, r2))
        ebs.append(float(rng.choice([0.01, 0.05, 0.1])))
    return fields, ebs


def test_batch_blobs_equal_single_field_and_oracle(ctx, oracle):
    fields, ebs = _batch(12, 1, 1, 700)
    fields.append(W.cfg0_like(77, 1, 1))
    ebs.append(0.1)
    blobs = cpsz_b200.compress_2d_batch(fields, ebs, ctx=ctx)
    assert len(blobs) == len(fields)
    for (U, V), eb, b in zip(fields, ebs, blobs):
        single = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=eb, ctx=ctx)
        assert b == single
        assert_blob_equal_2d(b, oracle.compress_2d(U, V, eb))


def test_batch_several_passes_and_device_io(ctx):
    torch = pytest.importorskip("torch")
    fields, ebs = _batch(70, 2, 16, 200)  # more fields than one pass holds
    dev = [(torch.from_numpy(U).cuda(), torch.from_numpy(V).cuda()) for U, V in fields]
    out = torch.zeros(64 << 20, dtype=torch.uint8, device="cuda")
    offsets = cpsz_b200.compress_2d_batch(dev, ebs, out=out, ctx=ctx)
    host = out.cpu().numpy()
    for k, ((U, V), eb) in enumerate(zip(fields, ebs)):
        b = host[int(offsets[k]):int(offsets[k + 1])].tobytes()
        assert b == cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=eb, ctx=ctx)
        du, dv = cpsz_b200.sz_decompress_cp_preserve_2d_offline(b, *U.shape, ctx=ctx)
        assert np.all(np.isfinite(du)) and np.all(np.isfinite(dv))


def test_batch_rejects_small_output(ctx):
    fields, ebs = _batch(3, 3, 50, 60)
    with pytest.raises(cpsz_b200.CpszError):
        cpsz_b200.compress_2d_batch(fields, ebs, out=np.zeros(100, np.uint8), ctx=ctx)
