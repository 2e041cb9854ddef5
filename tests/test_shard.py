"""Batch sharding across ranks: the partition, and a world-size-2 gloo run on
CPU whose concatenated output equals the single-rank batch byte for byte.
The per-field compressor here is the oracle (the GPU compressor's blobs
equal the oracle's, which the GPU tests check); the sharding, the size
all-reduce and the offset arithmetic are what this file tests."""
import os
import socket

import numpy as np
import pytest

from cpsz_b200 import shard
from cpsz_b200 import workloads as W


def test_partition_covers_every_field_once_and_balances():
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 8):
        sizes = [int(a) * int(b) for a, b in rng.integers(1, 4096, (256, 2))]
        own = shard.partition(sizes, world)
        flat = sorted(k for o in own for k in o)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[k] for k in o) for o in own]
        assert max(loads) - min(loads) <= max(sizes)  # greedy LPT bound
        assert own == shard.partition(sizes, world)  # a pure function of the sizes
    assert shard.partition([5, 5, 5], 4) == [[0], [1], [2], []]
    assert shard.partition([], 2) == [[], []]
    with pytest.raises(ValueError):
        shard.partition([1], 0)


SHAPES = [(40, 33), (1, 90), (71, 17), (2, 2), (64, 64), (9, 130), (33, 47)]
EBS = [0.1, 0.05, 0.01, 0.1, 0.05, 0.1, 0.01]


def _field(k):
    return W.cfg0_like(500 + k, *SHAPES[k])


def _oracle_compress():
    from oracle import Oracle

    o = Oracle()
    return lambda fields, ebs: [o.compress_2d(U, V, eb) for (U, V), eb in zip(fields, ebs)]


def _worker(rank, world, port, out_path, res_dir):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r = shard.compress_2d_batch_sharded(SHAPES, EBS, _field, compress=_oracle_compress(), out_path=out_path)
        np.savez(os.path.join(res_dir, f"r{rank}.npz"), own=np.array(r.own, np.int64), sizes=r.sizes,
                 offsets=r.offsets)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_on_gloo_equal_the_single_rank_batch(tmp_path):
    import torch.multiprocessing as mp

    out = str(tmp_path / "batch.bin")
    mp.spawn(_worker, args=(2, _free_port(), out, str(tmp_path)), nprocs=2, join=True)
    single = shard.compress_2d_batch_sharded(SHAPES, EBS, _field, compress=_oracle_compress(),
                                             out_path=str(tmp_path / "single.bin"))
    assert single.own == list(range(len(SHAPES)))
    data = open(out, "rb").read()
    assert data == open(tmp_path / "single.bin", "rb").read()
    r = [np.load(tmp_path / f"r{k}.npz") for k in range(2)]
    assert sorted(list(r[0]["own"]) + list(r[1]["own"])) == list(range(len(SHAPES)))
    assert set(r[0]["own"]).isdisjoint(r[1]["own"]) and len(r[0]["own"]) and len(r[1]["own"])
    for k in range(2):
        np.testing.assert_array_equal(r[k]["sizes"], single.sizes)
        np.testing.assert_array_equal(r[k]["offsets"], single.offsets)
    for k in range(len(SHAPES)):
        assert data[single.offsets[k]:single.offsets[k + 1]] == single.blobs[k]
