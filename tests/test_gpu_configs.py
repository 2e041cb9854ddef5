"""Parity at the sizes the benchmark numbers are quoted on: the 2D 8192^2
field at both bounds (device, pageable-host and page-locked-host inputs: the
last two take the banded upload path), the 3D 384^3 field and the whole
256-field batch.  Each blob is compared byte for byte with the oracle's (the
meanInfo padding bytes masked), each decode bit for bit, and each decode is
checked for critical points (none lost, added or retyped, exact checker) and
for the point-wise relative bound.

The oracle work runs in a process pool started with `spawn` (the batch's 1.1 G
points take minutes on one core)."""
import multiprocessing as mp
import os

import numpy as np
import pytest

import cpsz_b200
from cpsz_b200 import workloads as W
from tests._util import assert_bits_equal, assert_blob_equal_2d

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bound_violations(x, d, eb):
    x64 = x.astype(np.float64)
    return int(np.count_nonzero(np.abs(d.astype(np.float64) - x64) > eb * np.abs(x64)))


def _cfg1_oracle(args):
    """Oracle blob and decode of the 8192^2 field (worker process)."""
    import sys

    sys.path.insert(0, ROOT)
    from oracle import Oracle

    eb, = args
    O = Oracle()
    U, V = O.field_2d(1, 8192, 8192, 2000, 60.0)
    blob = O.compress_2d(U, V, eb)
    du, dv = O.decompress_2d(blob, 8192, 8192)
    return blob, du, dv


def _batch_field_oracle(args):
    import sys

    sys.path.insert(0, ROOT)
    from oracle import Oracle

    r1, r2, seed, eb = args
    O = Oracle()
    U, V = O.field_2d(seed, r1, r2, max(1, (r1 * r2) // 1600), 40.0)
    return O.compress_2d(U, V, eb)


def _pool(n):
    return mp.get_context("spawn").Pool(n)


@pytest.fixture(scope="module")
def cfg1_oracle():
    with _pool(2) as p:
        res = p.map(_cfg1_oracle, [(0.1,), (0.01,)])
    return {0.1: res[0], 0.01: res[1]}


@pytest.mark.parametrize("eb", [0.1, 0.01])
def test_cfg1_8192_every_input_kind(ctx, cfg1_oracle, eb):
    torch = pytest.importorskip("torch")
    U, V = W.cfg1(1)
    ref_blob, ou, ov = cfg1_oracle[eb]
    # device-resident input (the benchmark's `value` path)
    dU, dV = torch.from_numpy(U).cuda(), torch.from_numpy(V).cuda()
    a = cpsz_b200.sz_compress_cp_preserve_2d_offline(dU, dV, max_pwr_eb=eb, ctx=ctx)
    assert_blob_equal_2d(a, ref_blob)
    del dU, dV
    # pageable host input (banded upload beside the bound kernel)
    b = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=eb, ctx=ctx)
    assert_blob_equal_2d(b, ref_blob)
    # page-locked host input into a page-locked host output (the benchmark's e2e path)
    pU, pV = torch.from_numpy(U).pin_memory(), torch.from_numpy(V).pin_memory()
    out = torch.empty(len(ref_blob) + (1 << 20), dtype=torch.uint8).pin_memory()
    n = cpsz_b200.compress_2d_into(pU.numpy(), pV.numpy(), 8192, 8192, eb, out.numpy(), ctx=ctx)
    assert_blob_equal_2d(out.numpy()[:n].tobytes(), ref_blob)
    du, dv = cpsz_b200.sz_decompress_cp_preserve_2d_offline(a, 8192, 8192, ctx=ctx)
    assert_bits_equal(du, ou)
    assert_bits_equal(dv, ov)
    r = cpsz_b200.cp_check_2d(U, V, du, dv, ctx=ctx)
    assert r["cps_a"] > 0
    assert r["lost_or_spurious"] == 0 and r["type_changed"] == 0, r
    assert _bound_violations(U, du, eb) == 0 and _bound_violations(V, dv, eb) == 0
    assert ctx.wave_reruns == 0


def test_cfg2_384_cubed(ctx, oracle):
    U, V, Wf = W.cfg2(2)
    eb = 0.05
    a = cpsz_b200.sz_compress_cp_preserve_3d_offline_log(U, V, Wf, max_pwr_eb=eb, ctx=ctx)
    b = oracle.compress_3d(U, V, Wf, eb)
    assert a == b
    d = cpsz_b200.sz_decompress_cp_preserve_3d_online_log(a, *U.shape, ctx=ctx)
    o = oracle.decompress_3d(b, *U.shape)
    for x, y in zip(d, o):
        assert_bits_equal(x, y)
    r = cpsz_b200.cp_check_3d(U, V, Wf, *d, ctx=ctx)
    assert r["cps_a"] > 0
    assert r["lost_or_spurious"] == 0 and r["type_changed"] == 0, r


def test_cfg3_whole_batch(ctx):
    lay = W.batch_layout(3, 256, 128, 4096)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    # the oracle's blobs first (spawned workers, longest fields first)
    order = sorted(range(len(lay)), key=lambda k: -lay[k][0] * lay[k][1])
    with _pool(max(1, min(cores, 32))) as p:
        blobs = dict(zip(order, p.map(_batch_field_oracle, [lay[k] for k in order], chunksize=1)))
    fields = [W.cfg3_field(r1, r2, seed) for r1, r2, seed, _ in lay]
    ebs = [eb for *_, eb in lay]
    raw = sum(U.nbytes + V.nbytes for U, V in fields)
    out = np.empty(raw + (256 << 20), np.uint8)
    offs = cpsz_b200.compress_2d_batch(fields, ebs, out=out, ctx=ctx)
    assert len(offs) == 257
    for k in range(len(lay)):
        assert_blob_equal_2d(out[int(offs[k]):int(offs[k + 1])].tobytes(), blobs[k])
    # decode and check a spread of them (smallest, largest, every bound)
    picks = {order[0], order[-1]} | {next(k for k in order if ebs[k] == e) for e in (0.01, 0.05, 0.1)}
    for k in sorted(picks):
        U, V = fields[k]
        du, dv = cpsz_b200.sz_decompress_cp_preserve_2d_offline(blobs[k], *U.shape, ctx=ctx)
        r = cpsz_b200.cp_check_2d(U, V, du, dv, ctx=ctx)
        assert r["lost_or_spurious"] == 0 and r["type_changed"] == 0, (k, r)
        assert _bound_violations(U, du, ebs[k]) == 0 and _bound_violations(V, dv, ebs[k]) == 0
