"""Every launch-shape parameter value leaves the output unchanged: blobs are
byte-identical to the default shape's (and, for 2D, to the oracle's), for
ragged sizes that leave partial tiles, bands and i-chunks."""
import numpy as np
import pytest

import cpsz_b200
from cpsz_b200 import autotune
from cpsz_b200 import workloads as W
from tests._util import assert_blob_equal_2d

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _restore_table():
    cpsz_b200.tuning_clear()
    yield
    cpsz_b200.tuning_clear()


@pytest.mark.parametrize("shape", [(333, 517), (1, 700), (2, 65), (129, 31), (17, 1)])
def test_eb2d_tiles_and_wave_shapes_give_equal_blobs(ctx, oracle, shape):
    U, V = W.cfg0_like(11 + shape[0], *shape)
    ref = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=ctx)
    assert_blob_equal_2d(ref, oracle.compress_2d(U, V, 0.1))
    lo, hi = cpsz_b200.tuning_params()["eb2d.tile"][1:]
    for v in range(lo, hi + 1):
        cpsz_b200.tuning_set("eb2d.tile", v)
        assert cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=ctx) == ref, v
    cpsz_b200.tuning_clear()
    cpsz_b200.tuning_set("wave2d.overlap", 0)
    assert cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=ctx) == ref
    cpsz_b200.tuning_clear()
    for v in (1, 2, 3):
        cpsz_b200.tuning_set("wave2d.ctas_per_sm", v)
        b = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.1, ctx=ctx)
        assert b == ref, v
        du, dv = cpsz_b200.sz_decompress_cp_preserve_2d_offline(b, *shape, ctx=ctx)
        cpsz_b200.tuning_clear()
        eu, ev = cpsz_b200.sz_decompress_cp_preserve_2d_offline(b, *shape, ctx=ctx)
        assert du.tobytes() == eu.tobytes() and dv.tobytes() == ev.tobytes()


def test_upload_chunks_give_equal_blobs(ctx):
    U, V = W.cfg0_like(5, 2053, 2049)  # above the chunked-upload threshold, ragged bands
    dev_ref = cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.05, ctx=ctx)
    for k in (1, 2, 3, 5, 8):
        cpsz_b200.tuning_set("h2d.chunks", k)
        for tile in (0, 3):
            cpsz_b200.tuning_set("eb2d.tile", tile)
            assert cpsz_b200.sz_compress_cp_preserve_2d_offline(U, V, max_pwr_eb=0.05, ctx=ctx) == dev_ref, (k, tile)


@pytest.mark.parametrize("shape", [(37, 41, 29), (9, 70, 33), (70, 5, 66)])
def test_eb3d_splits_give_equal_blobs(ctx, shape):
    U, V, Wf = W.field_3d(21 + shape[0], *shape, n_flows=6, sigma=6.0)
    ref = cpsz_b200.sz_compress_cp_preserve_3d_offline_log(U, V, Wf, max_pwr_eb=0.05, ctx=ctx)
    for fill in (1, 2, 8, 32):
        for mc in (1, 3, 8, 64):
            cpsz_b200.tuning_set("eb3d.fill", fill)
            cpsz_b200.tuning_set("eb3d.min_chunk", mc)
            assert cpsz_b200.sz_compress_cp_preserve_3d_offline_log(U, V, Wf, max_pwr_eb=0.05, ctx=ctx) == ref


def test_quick_sweep_writes_a_loadable_table(tmp_path):
    table = autotune.sweep(quick=True, reps=2, log=lambda s: None)
    assert table["format"] == autotune.FORMAT and table["entries"]
    p = tmp_path / "t.json"
    import json

    p.write_text(json.dumps(table))
    cpsz_b200.tuning_load(str(p))
    for e in table["entries"]:
        assert cpsz_b200.tuning_get(e["param"], e["min_points"]) == e["value"]
