"""Launch-shape tuning table: parameter list, lookup by field size, the JSON
reader (valid tables load, malformed ones are rejected whole) and the
automatic load at context creation.  Host-only: no kernel runs here."""
import json
import os
import subprocess
import sys

import pytest

import cpsz_b200
from cpsz_b200 import autotune

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(autouse=True)
def _restore_table():
    yield
    cpsz_b200.tuning_clear()


def test_parameters_and_defaults():
    p = cpsz_b200.tuning_params()
    assert set(p) == {"eb2d.tile", "wave2d.ctas_per_sm", "eb3d.fill", "eb3d.min_chunk", "h2d.chunks",
                      "wave2d.overlap", "eb2d.skew"}
    for name, (d, lo, hi) in p.items():
        assert lo <= d <= hi
    cpsz_b200.tuning_clear()
    for name, (d, _, _) in p.items():
        assert cpsz_b200.tuning_get(name, 12345) == d
    # every parameter the sweep names exists, with candidates inside its range
    for name, (_, _, cands, _) in autotune.SWEEP.items():
        assert name in p
        assert all(p[name][1] <= v <= p[name][2] for v in cands)


def test_lookup_by_field_size():
    cpsz_b200.tuning_clear()
    cpsz_b200.tuning_set("eb2d.tile", 3, min_points=1 << 20)
    cpsz_b200.tuning_set("eb2d.tile", 1, min_points=0)
    cpsz_b200.tuning_set("eb2d.tile", 4, min_points=1 << 24)
    assert cpsz_b200.tuning_get("eb2d.tile", 0) == 1
    assert cpsz_b200.tuning_get("eb2d.tile", (1 << 20) - 1) == 1
    assert cpsz_b200.tuning_get("eb2d.tile", 1 << 20) == 3
    assert cpsz_b200.tuning_get("eb2d.tile", 1 << 30) == 4
    cpsz_b200.tuning_set("eb2d.tile", 2, min_points=1 << 20)  # replaces the entry at that threshold
    assert cpsz_b200.tuning_get("eb2d.tile", 1 << 21) == 2
    # below the smallest threshold the built-in default applies
    cpsz_b200.tuning_clear()
    cpsz_b200.tuning_set("h2d.chunks", 2, min_points=1000)
    assert cpsz_b200.tuning_get("h2d.chunks", 999) == cpsz_b200.tuning_params()["h2d.chunks"][0]


@pytest.mark.parametrize("name,value", [("eb2d.tile", 6), ("eb2d.tile", -1), ("h2d.chunks", 0),
                                        ("h2d.chunks", 33), ("nope", 1)])
def test_set_rejects_bad_values(name, value):
    with pytest.raises(cpsz_b200.CpszError):
        cpsz_b200.tuning_set(name, value)


def _write(tmp_path, obj, name="t.json"):
    p = tmp_path / name
    p.write_text(obj if isinstance(obj, str) else json.dumps(obj))
    return str(p)


def test_load_valid_table(tmp_path):
    t = {"format": "cpsz_b200-tuning-1", "device": "x", "entries": [
        {"param": "wave2d.ctas_per_sm", "min_points": 0, "value": 2, "ms": {"0": 1.0, "2": 0.9}},
        {"param": "wave2d.ctas_per_sm", "min_points": 4000000, "value": 3},
        {"param": "eb3d.fill", "min_points": 100, "value": 8, "note": [1, 2, {"a": None, "b": True}]}]}
    p = _write(tmp_path, t)
    cpsz_b200.tuning_load(p)
    assert cpsz_b200.tuning_source() == p
    assert cpsz_b200.tuning_get("wave2d.ctas_per_sm", 10) == 2
    assert cpsz_b200.tuning_get("wave2d.ctas_per_sm", 5000000) == 3
    assert cpsz_b200.tuning_get("eb3d.fill", 99) == 4
    assert cpsz_b200.tuning_get("eb3d.fill", 100) == 8


@pytest.mark.parametrize("text", [
    '{"format": "cpsz_b200-tuning-1", "entries": [{"param": "eb2d.tile", "min_points": 0, "value": 9}]}',
    '{"format": "cpsz_b200-tuning-1", "entries": [{"param": "eb2d.tyle", "min_points": 0, "value": 1}]}',
    '{"format": "cpsz_b200-tuning-1", "entries": [{"param": "eb2d.tile", "min_points": -5, "value": 1}]}',
    '{"format": "cpsz_b200-tuning-1", "entries": [{"param": "eb2d.tile", "min_points": 0, "value": 1.5}]}',
    '{"format": "cpsz_b200-tuning-1", "entries": [{"param": "eb2d.tile", "value": 1}]}',
    '{"format": "other", "entries": []}',
    '{"format": "cpsz_b200-tuning-1", "entries": [}',
    '{"format": "cpsz_b200-tuning-1", "entries": []} trailing',
    '[1, 2]',
    '',
])
def test_malformed_tables_are_rejected_whole(tmp_path, text):
    cpsz_b200.tuning_clear()
    cpsz_b200.tuning_set("eb2d.tile", 5)
    with pytest.raises(cpsz_b200.CpszError):
        cpsz_b200.tuning_load(_write(tmp_path, text))
    assert cpsz_b200.tuning_get("eb2d.tile", 1 << 20) == 5  # the previous table stays


def test_missing_table_file(tmp_path):
    with pytest.raises(cpsz_b200.CpszError):
        cpsz_b200.tuning_load(str(tmp_path / "absent.json"))


def _ctx_create_in_child(env_value):
    code = ("import ctypes as C, cpsz_b200 as c; h = C.c_void_p(); "
            "rc = c.lib().cpsz_b200_ctx_create(0, C.byref(h)); "
            "print(rc, c.lib().cpsz_b200_last_error().decode())")
    env = dict(os.environ, CPSZ_B200_TUNING=env_value)
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    rc, _, msg = r.stdout.strip().partition(" ")
    return int(rc), msg


def test_malformed_table_fails_context_creation(tmp_path):
    p = _write(tmp_path, '{"format": "cpsz_b200-tuning-1", "entries": [{"param": "x", "min_points": 0, "value": 1}]}')
    rc, msg = _ctx_create_in_child(p)
    assert rc == 1 and "unknown parameter" in msg  # CPSZ_ERR_INVALID, before any device is touched
    rc, msg = _ctx_create_in_child("none")
    assert rc != 1  # no table: ctx creation proceeds (CPSZ_OK on a GPU, NO_DEVICE without one)


def test_committed_table_is_valid():
    p = autotune.DEFAULT_OUT
    if not os.path.exists(p):
        pytest.skip("no committed table")
    cpsz_b200.tuning_load(p)
    t = json.load(open(p))
    assert t["format"] == autotune.FORMAT
    for e in t["entries"]:
        assert cpsz_b200.tuning_get(e["param"], e["min_points"]) == e["value"]


def test_bucket_edges():
    assert autotune.bucket_edges([100, 400, 1600]) == [0, 200, 800]
