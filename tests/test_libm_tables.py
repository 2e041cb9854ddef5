"""The host log2f / exp2f tables the 3D kernels use (CPU): every listed
input is checked against the host C library itself and against long-double
results, and a random sample of unlisted inputs is checked to be correctly
rounded by the host library (so the GPU's correctly rounded float is right)."""
import ctypes
import os
import struct

import numpy as np
import pytest

import cpsz_b200

TABLE = os.path.join(os.path.dirname(cpsz_b200.LIB_PATH), "libm_f32_tables.bin")


def _load():
    if not os.path.exists(TABLE):
        cpsz_b200.libm_tables_prepare()
    b = open(TABLE, "rb").read()
    assert b[:8] == b"CPSZLM02"
    (vlen,) = struct.unpack_from("<I", b, 8)
    ver = b[12:12 + vlen].decode()
    o = 12 + vlen
    fns = {}
    for name in ("log2f", "exp2f"):
        nh, nm = struct.unpack_from("<II", b, o)
        o += 8
        band = np.frombuffer(b, np.float64, 512, o)
        o += 512 * 8
        hin = np.frombuffer(b, np.uint32, nh, o)
        o += 4 * nh
        hout = np.frombuffer(b, np.uint32, nh, o)
        o += 4 * nh
        mis = np.frombuffer(b, np.uint32, nm, o)
        o += 4 * nm
        fns[name] = (band, hin, hout, mis)
    assert o == len(b)
    return ver, fns


@pytest.fixture(scope="module")
def tables():
    return _load()


def _exact(name, x):
    xl = x.astype(np.longdouble)
    return (np.log2(xl) if name == "log2f" else np.exp2(xl)).astype(np.float32)


def test_table_version_is_this_c_library(tables):
    libc = ctypes.CDLL(None)
    libc.gnu_get_libc_version.restype = ctypes.c_char_p
    assert tables[0] == libc.gnu_get_libc_version().decode()


@pytest.mark.parametrize("name", ["log2f", "exp2f"])
def test_listed_inputs_match_the_host_library(oracle, tables, name):
    band, hin, hout, mis = tables[1][name]
    assert np.all(np.diff(hin.astype(np.int64)) > 0) and np.all(np.diff(mis.astype(np.int64)) > 0)
    # hard cases: stored output is the host library's output
    x = hin.view(np.float32)
    assert np.array_equal(oracle.host_libm(name, x).view(np.uint32), hout)
    # misrounded: the host output is the neighbour of the correctly rounded float
    x = mis.view(np.float32)
    h = oracle.host_libm(name, x).view(np.uint32).astype(np.int64)
    c = _exact(name, x).view(np.uint32).astype(np.int64)
    assert np.all(np.abs(h - c) == 1)
    # every misrounded input's binade has a band
    keys = mis >> 23
    assert np.all(band[keys] > 0) and np.all(band < 0.5)


@pytest.mark.parametrize("name", ["log2f", "exp2f"])
def test_unlisted_inputs_are_correctly_rounded(oracle, tables, name):
    band, hin, hout, mis = tables[1][name]
    rng = np.random.default_rng(7)
    if name == "log2f":
        bits = rng.integers(1, 0x7F800000, 2_000_000, dtype=np.uint32)
        # inputs near 1, where the host library misrounds most
        near1 = (np.uint32(0x3F000000) + rng.integers(0, 1 << 24, 1_000_000, dtype=np.uint32)).astype(np.uint32)
        bits = np.concatenate([bits, near1])
    else:
        x = np.concatenate([rng.uniform(-99, 128, 2_000_000), rng.uniform(-1, 1, 500_000)]).astype(np.float32)
        bits = x.view(np.uint32)
    listed = np.isin(bits, hin) | np.isin(bits, mis)
    x = bits[~listed].view(np.float32)
    h = oracle.host_libm(name, x)
    assert np.array_equal(h.view(np.uint32), _exact(name, x).view(np.uint32))
