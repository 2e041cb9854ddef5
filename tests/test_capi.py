"""The C ABI library loads and exports what include/*.h declares (no GPU needed)."""
import ctypes
import os
import subprocess

import cpsz_b200
from tests._util import header_symbols

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROP_IN = [
    "_Z34sz_compress_cp_preserve_2d_offlineIfEPhPKT_S3_mmRmbd",
    "_Z36sz_decompress_cp_preserve_2d_offlineIfEvPKhmmRPT_S4_",
    "_Z38sz_compress_cp_preserve_3d_offline_logIfEPhPKT_S3_S3_mmmRmbd",
    "_Z39sz_decompress_cp_preserve_3d_online_logIfEvPKhmmmRPT_S4_S4_",
    "_Z38sz_compress_cp_preserve_2d_offline_logIfEPhPKT_S3_mmRmbd",
    "_Z40sz_decompress_cp_preserve_2d_offline_logIfEvPKhmmRPT_S4_",
]


def test_every_declared_symbol_is_exported():
    L = cpsz_b200.lib()
    names = header_symbols(os.path.join(ROOT, "include", "cpsz_b200.h"))
    assert len(names) > 10
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_reference_mangled_drop_ins_are_exported():
    L = cpsz_b200.lib()
    missing = [n for n in DROP_IN if not hasattr(L, n)]
    assert not missing, missing


def test_errors_are_reported_without_a_device():
    L = cpsz_b200.lib()
    # null output pointers are rejected before any device work
    rc = L.cpsz_b200_compress_2d_offline_f32(None, None, None, 4, 4, ctypes.c_double(0.1), None, None)
    assert rc == 1
    assert b"null" in L.cpsz_b200_last_error()


def test_generator_is_seeded_and_scaled():
    a = cpsz_b200.workloads.cfg0_like(5, 120, 90)
    b = cpsz_b200.workloads.cfg0_like(5, 120, 90)
    c = cpsz_b200.workloads.cfg0_like(6, 120, 90)
    assert all((x == y).all() for x, y in zip(a, b))
    assert not (a[0] == c[0]).all()
    m = max(abs(a[0]).max(), abs(a[1]).max())
    assert abs(m - 1.0) < 1e-6
