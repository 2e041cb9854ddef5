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


@pytest.mark.parametrize("shape", range(6))
def test_batch_one_bound_launch_every_tile_shape(ctx, shape):
    """A batch of device fields derives all its fields' bounds in one launch
    (each CTA finds its field in a per-pass table, largest field first): for
    every launch shape, with ragged fields (single rows, single columns, a
    single point, sizes that are no multiple of a tile), every blob equals
    the single-field compressor's."""
    torch = pytest.importorskip("torch")
    fields, ebs = _batch(9, 10 + shape, 1, 300)
    for k, (r1, r2) in enumerate([(1, 1), (1, 97), (83, 1), (33, 65), (17, 129)]):
        fields.append(W.cfg0_like(500 + 10 * shape + k, r1, r2))
        ebs.append(0.1 if k % 2 else 0.01)
    dev = [(torch.from_numpy(U).cuda(), torch.from_numpy(V).cuda()) for U, V in fields]
    out = torch.zeros(32 << 20, dtype=torch.uint8, device="cuda")
    try:
        cpsz_b200.tuning_set("eb2d.tile", shape, min_points=0)
        offs = cpsz_b200.compress_2d_batch(dev, ebs, out=out, ctx=ctx)
        host = out[:int(offs[-1])].cpu().numpy().tobytes()
        for k, ((U, V), eb) in enumerate(zip(fields, ebs)):
            assert host[int(offs[k]):int(offs[k + 1])] == cpsz_b200.sz_compress_cp_preserve_2d_offline(
                U, V, max_pwr_eb=eb, ctx=ctx), k
    finally:
        cpsz_b200.tuning_clear()
        cpsz_b200.tuning_load()


def test_batch_rejects_small_output(ctx):
    fields, ebs = _batch(3, 3, 50, 60)
    with pytest.raises(cpsz_b200.CpszError):
        cpsz_b200.compress_2d_batch(fields, ebs, out=np.zeros(100, np.uint8), ctx=ctx)


def test_batch_graph_capture_and_replay(ctx):
    """A batch of device fields runs its pre-tree device work from a CUDA graph:
    the first call captures it, a repeated identical call replays it, and a
    change of a bound or of the tuning table captures again.  Every result
    equals the single-field compressor's blobs, and a replay counts the same
    kernels as the call that captured."""
    torch = pytest.importorskip("torch")
    fields, ebs = _batch(24, 3, 40, 400)
    dev = [(torch.from_numpy(U).cuda(), torch.from_numpy(V).cuda()) for U, V in fields]
    out = torch.zeros(64 << 20, dtype=torch.uint8, device="cuda")

    def run(e):
        before = ctx.kernel_launches
        offs = cpsz_b200.compress_2d_batch(dev, e, out=out, ctx=ctx)
        host = out[:int(offs[-1])].cpu().numpy().tobytes()
        return [host[int(offs[k]):int(offs[k + 1])] for k in range(len(dev))], ctx.kernel_launches - before

    def singles(e):
        return [cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=b, ctx=ctx) for (U, V), b in zip(fields, e)]

    ref = singles(ebs)
    c0, r0 = ctx.graph_stats
    first, n_first = run(ebs)
    assert first == ref
    c1, r1 = ctx.graph_stats
    assert c1 == c0 + 1 and r1 == r0  # one pass, captured
    for k in range(3):
        again, n_again = run(ebs)
        assert again == ref
        assert n_again == n_first
        assert ctx.graph_stats == (c1, r1 + k + 1)  # replayed
    ebs2 = list(ebs)
    ebs2[5] = 0.02 if ebs2[5] != 0.02 else 0.03
    changed, _ = run(ebs2)
    assert changed == singles(ebs2)
    assert ctx.graph_stats[0] == c1 + 1  # a new bound: captured again
    try:
        cpsz_b200.tuning_set("eb2d.tile", 1, min_points=0)
        retuned, _ = run(ebs)
        assert retuned == ref
        assert ctx.graph_stats[0] == c1 + 2  # a new launch shape: captured again
    finally:
        cpsz_b200.tuning_clear()
        cpsz_b200.tuning_load()
    assert run(ebs)[0] == ref


def test_sharded_batch_with_the_gpu_compressor(ctx, oracle, tmp_path):
    """The field-sharded batch (cpsz_b200.shard) driving the GPU batch
    compressor, on one rank: every blob equals the oracle's and the written
    file is the blobs' concatenation in field order."""
    from cpsz_b200 import shard

    fields, ebs = _batch(9, 5, 1, 500)
    shapes = [U.shape for U, _ in fields]
    out = str(tmp_path / "batch.bin")
    r = shard.compress_2d_batch_sharded(shapes, ebs, lambda k: fields[k], ctx=ctx, out_path=out)
    assert r.own == list(range(len(fields)))
    data = open(out, "rb").read()
    assert len(data) == int(r.offsets[-1])
    for k, ((U, V), eb) in enumerate(zip(fields, ebs)):
        assert_blob_equal_2d(r.blobs[k], oracle.compress_2d(U, V, eb))
        assert data[int(r.offsets[k]):int(r.offsets[k + 1])] == r.blobs[k]


def _nccl_rank(rank, port, out_path, res_path):
    import os

    import torch
    import torch.distributed as dist

    from cpsz_b200 import shard

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=rank, world_size=1)
    try:
        c = cpsz_b200.Context(0)
        fields, ebs = _batch(6, 6, 8, 300)
        r = shard.compress_2d_batch_sharded([U.shape for U, _ in fields], ebs, lambda k: fields[k], ctx=c,
                                            out_path=out_path)
        np.save(res_path, r.offsets)
        c.close()
    finally:
        dist.destroy_process_group()


def test_sharded_batch_over_nccl_one_rank(oracle, tmp_path):
    """The same through an initialised NCCL process group (one rank, so the
    size all-reduce runs on the device)."""
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out, res = str(tmp_path / "b.bin"), str(tmp_path / "offs.npy")
    mp.spawn(_nccl_rank, args=(port, out, res), nprocs=1, join=True)
    offs = np.load(res)
    data = open(out, "rb").read()
    fields, ebs = _batch(6, 6, 8, 300)
    for k, ((U, V), eb) in enumerate(zip(fields, ebs)):
        assert_blob_equal_2d(data[int(offs[k]):int(offs[k + 1])], oracle.compress_2d(U, V, eb))


def test_batch_graphs_dropped_when_workspace_grows():
    """Cached pass graphs hold workspace and staging addresses: a call that
    grows either (a larger batch) drops them, so the first batch is captured
    again afterwards instead of replayed from a graph whose copy nodes refer
    to freed memory (a same-address reallocation once crashed the replay)."""
    torch = pytest.importorskip("torch")
    c = cpsz_b200.Context(0)
    try:
        small, ebs_s = _batch(6, 7, 40, 120)
        big, ebs_b = _batch(30, 8, 200, 500)
        dev_s = [(torch.from_numpy(U).cuda(), torch.from_numpy(V).cuda()) for U, V in small]
        dev_b = [(torch.from_numpy(U).cuda(), torch.from_numpy(V).cuda()) for U, V in big]
        out = torch.zeros(128 << 20, dtype=torch.uint8, device="cuda")

        def run(dev, e):
            offs = cpsz_b200.compress_2d_batch(dev, e, out=out, ctx=c)
            host = out[:int(offs[-1])].cpu().numpy().tobytes()
            return [host[int(offs[k]):int(offs[k + 1])] for k in range(len(dev))]

        first = run(dev_s, ebs_s)
        c0, _ = c.graph_stats
        assert run(dev_s, ebs_s) == first
        assert c.graph_stats[0] == c0  # replayed
        run(dev_b, ebs_b)  # grows the workspace and the staging
        c1, _ = c.graph_stats
        assert run(dev_s, ebs_s) == first
        assert c.graph_stats[0] == c1 + 1  # captured again, not replayed
    finally:
        c.close()
