"""The reference's own 2D test driver (test/sz_compress_cp_preserve_2d_test.cpp,
unchanged), built once against the reference's library and once against
libcpsz_b200.so through the drop-in's mangled template symbols
(`make -C oracle ref`, binaries in oracle/_ref/): on the same input files the
two report the same ZSTD'd size and write bit-identical decoded fields.  This
exercises the drop-in's ownership contract as the reference's callers use it:
a malloc'd blob the driver frees, and decoded arrays allocated by the call."""
import os
import re
import subprocess

import numpy as np
import pytest

from cpsz_b200 import workloads as W

pytestmark = pytest.mark.gpu
REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


def _run(exe, d, r1, r2, eb):
    r = subprocess.run([exe, "U.dat", "V.dat", str(r1), str(r2), str(eb)], cwd=d, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    m = re.search(r"Compressed size = (\d+)", r.stdout)
    assert m, r.stdout[-2000:]
    return int(m.group(1)), [np.fromfile(os.path.join(d, f + ".out"), np.float32) for f in ("U.dat", "V.dat")]


@pytest.mark.parametrize("r1,r2,eb,seed", [(600, 700, 0.1, 41), (1024, 1536, 0.01, 42)])
def test_reference_driver_on_the_drop_in(tmp_path, r1, r2, eb, seed):
    exe = {k: os.path.join(REF, f"drv_2d_{k}") for k in ("ref", "b200")}
    if not all(os.path.exists(p) for p in exe.values()):
        pytest.skip("drivers not built (make -C oracle ref where the reference sources are present)")
    U, V = W.cfg0_like(seed, r1, r2)
    out = {}
    for k in exe:
        d = tmp_path / k
        d.mkdir()
        U.tofile(d / "U.dat")
        V.tofile(d / "V.dat")
        out[k] = _run(exe[k], str(d), r1, r2, eb)
    assert out["b200"][0] == out["ref"][0]
    for a, b in zip(out["b200"][1], out["ref"][1]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
