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


def assert_blob_equal_2d(a: bytes, b: bytes):
    assert len(a) == len(b), f"blob sizes differ: {len(a)} vs {len(b)}"
    x = np.frombuffer(a, np.uint8)
    y = np.frombuffer(b, np.uint8)
    m = padding_mask_2d(a)
    bad = np.nonzero((x != y) & m)[0]
    assert bad.size == 0, f"{bad.size} bytes differ, first at {bad[:8].tolist()}"


def assert_bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert a.shape == b.shape and a.dtype == b.dtype
    va = a.view(np.uint32) if a.dtype == np.float32 else a
    vb = b.view(np.uint32) if b.dtype == np.float32 else b
    bad = np.nonzero(va.ravel() != vb.ravel())[0]
    assert bad.size == 0, f"{bad.size} of {a.size} values differ, first at {bad[:8].tolist()}"


def header_symbols(path):
    """Function names declared in a C header."""
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cpsz_b200_\w+)\s*\(", src)))
