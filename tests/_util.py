"""Shared helpers of the test suite."""
import glob
import os
import re
import struct

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_cases(prefix):
    return sorted(glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def padding_mask_2d(blob: bytes) -> np.ndarray:
    """Mask of the bytes of a 2D offline blob that carry meaning.

    The reference writes meanInfo<float> (bool + 3 padding bytes + float) raw
    (src/sz_compress_3d.cpp:222), so those 3 padding bytes of each field header
    are indeterminate in its output; every other byte is compared."""
    m = np.ones(len(blob), bool)
    eb_size, u_size, v_size = struct.unpack_from("<QQQ", blob, 12)
    for off in (36 + eb_size, 36 + eb_size + u_size):
        m[off + 10: off + 13] = False
    return m


def padding_mask_2d_log(blob: bytes, n: int) -> np.ndarray:
    """The same for a 2D offline_log blob of n points (its field blobs follow
    the id section and the two sign maps)."""
    m = np.ones(len(blob), bool)
    eb_size, u_size, v_size = struct.unpack_from("<QQQ", blob, 12)
    at = 36 + eb_size + 2 * ((n - 1) // 8 + 1)
    for off in (at, at + u_size):
        m[off + 10: off + 13] = False
    return m


def assert_blob_equal_2d_log(a: bytes, b: bytes, n: int):
    assert len(a) == len(b), f"blob sizes differ: {len(a)} vs {len(b)}"
    x = np.frombuffer(a, np.uint8)
    y = np.frombuffer(b, np.uint8)
    bad = np.nonzero((x != y) & padding_mask_2d_log(a, n))[0]
    assert bad.size == 0, f"{bad.size} bytes differ, first at {bad[:8].tolist()}"


def assert_blob_equal_2d(a: bytes, b: bytes):
    assert len(a) == len(b), f"blob sizes differ: {len(a)} vs {len(b)}"
    x = np.frombuffer(a, np.uint8)
    y = np.frombuffer(b, np.uint8)
    m = padding_mask_2d(a)
    bad = np.nonzero((x != y) & m)[0]
    assert bad.size == 0, f"{bad.size} bytes differ, first at {bad[:8].tolist()}"


def assert_bits_equal(a, b, nan_equal: bool = False):
    """Bit-pattern equality of two arrays.  nan_equal: any NaN matches any NaN
    (for intermediate bounds, where only NaN-ness reaches the output: x86 and
    the GPU encode the NaN of an invalid operation differently)."""
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert a.shape == b.shape and a.dtype == b.dtype
    views = {np.dtype(np.float32): np.uint32, np.dtype(np.float64): np.uint64}
    va = a.view(views[a.dtype]) if a.dtype in views else a
    vb = b.view(views[b.dtype]) if b.dtype in views else b
    diff = va.ravel() != vb.ravel()
    if nan_equal and a.dtype in views:
        diff &= ~(np.isnan(a.ravel()) & np.isnan(b.ravel()))
    bad = np.nonzero(diff)[0]
    assert bad.size == 0, f"{bad.size} of {a.size} values differ, first at {bad[:8].tolist()}"


def header_symbols(path):
    """Function names declared in a C header."""
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cpsz_b200_\w+)\s*\(", src)))
