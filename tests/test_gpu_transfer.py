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
