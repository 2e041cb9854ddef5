"""Bulk copies to and from pageable host memory go through the context's
pinned ring (chunked, several host threads); results must not depend on where
the data lives: pageable numpy, page-locked host memory or device memory, for
sizes that leave partial chunks and for fields below the staging threshold."""
import numpy as np
import pytest

import cpsz_b200
from cpsz_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(2049, 1031), (4100, 2051), (300, 257)])
def test_2d_pageable_pinned_and_device_give_equal_results(ctx, shape):
    torch = pytest.importorskip("torch")
    U, V = W.cfg0_like(61 + shape[0], *shape)
    ref = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.05, ctx=ctx)  # malloc'd blob
    pinned = [torch.from_numpy(a).pin_memory() for a in (U, V)]
    assert cpsz_b200.sz_compress_cp_preserve_2d_offline(*[p.numpy() for p in pinned], max_pwr_eb=0.05, ctx=ctx) == ref
    dev = [torch.from_numpy(a).cuda() for a in (U, V)]
    out = torch.zeros(len(ref) + 4096, dtype=torch.uint8, device="cuda")
    n = cpsz_b200.compress_2d_into(*dev, *shape, 0.05, out, ctx=ctx)
    assert out[:n].cpu().numpy().tobytes() == ref
    host_out = np.zeros(len(ref) + 4096, np.uint8)  # pageable destination
    n = cpsz_b200.compress_2d_into(U, V, *shape, 0.05, host_out, ctx=ctx)
    assert host_out[:n].tobytes() == ref
    a = cpsz_b200.sz_decompress_cp_preserve_2d_offline(ref, *shape, ctx=ctx)  # pageable outputs
    b = [torch.empty(shape, dtype=torch.float32, device="cuda") for _ in range(2)]
    cpsz_b200.sz_decompress_cp_preserve_2d_offline(ref, *shape, *b, ctx=ctx)
    for x, y in zip(a, b):
        assert x.tobytes() == y.cpu().numpy().tobytes()


@pytest.mark.parametrize("shape", [(1024, 1536), (8192, 8192)])
def test_2d_blob_written_straight_to_host_memory(ctx, shape):
    """A host output buffer gets the blob section by section (the bit streams
    and unpredictable floats copied from their device buffers as soon as they
    are produced when it is page-locked, after the whole pass otherwise): the
    bytes equal the device-assembled blob, repeatedly, and a buffer one byte
    short is refused."""
    torch = pytest.importorskip("torch")
    U, V = W.cfg0_like(71, *shape)
    dev = [torch.from_numpy(a).cuda() for a in (U, V)]
    d_out = torch.zeros(U.nbytes * 3, dtype=torch.uint8, device="cuda")
    n = cpsz_b200.compress_2d_into(*dev, *shape, 0.1, d_out, ctx=ctx)
    ref = d_out[:n].cpu().numpy().tobytes()
    pinned = [torch.from_numpy(a).pin_memory().numpy() for a in (U, V)]
    h_pin = torch.zeros(n + 64, dtype=torch.uint8).pin_memory().numpy()
    h_page = np.zeros(n + 64, np.uint8)
    for _ in range(3):
        h_pin[:] = 0x5A
        assert cpsz_b200.compress_2d_into(*pinned, *shape, 0.1, h_pin, ctx=ctx) == n
        assert h_pin[:n].tobytes() == ref
    assert cpsz_b200.compress_2d_into(U, V, *shape, 0.1, h_page, ctx=ctx) == n
    assert h_page[:n].tobytes() == ref
    for buf in (h_pin[:n - 1], h_page[:n - 1]):
        with pytest.raises(cpsz_b200.CpszError, match="output capacity"):
            cpsz_b200.compress_2d_into(*pinned, *shape, 0.1, buf, ctx=ctx)


def test_3d_pageable_and_device_give_equal_results(ctx):
    torch = pytest.importorskip("torch")
    U, V, Wf = W.field_3d(71, 130, 97, 101, n_flows=12, sigma=8.0)
    ref = cpsz_b200.sz_compress_cp_preserve_3d_offline_log(U, V, Wf, max_pwr_eb=0.05, ctx=ctx)
    dev = [torch.from_numpy(a).cuda() for a in (U, V, Wf)]
    out = torch.zeros(len(ref) + 4096, dtype=torch.uint8, device="cuda")
    n = cpsz_b200.compress_3d_into(*dev, *U.shape, 0.05, out, ctx=ctx)
    assert out[:n].cpu().numpy().tobytes() == ref
    a = cpsz_b200.sz_decompress_cp_preserve_3d_online_log(ref, *U.shape, ctx=ctx)
    b = [torch.empty(U.shape, dtype=torch.float32, device="cuda") for _ in range(3)]
    cpsz_b200.sz_decompress_cp_preserve_3d_online_log(ref, *U.shape, *b, ctx=ctx)
    for x, y in zip(a, b):
        assert x.tobytes() == y.cpu().numpy().tobytes()
