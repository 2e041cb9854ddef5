"""Host-computed quantization thresholds reproduce the reference's log2-based
quantizer (include/sz_cp_preserve_utils.hpp:14-22) exactly around every threshold."""
import ctypes as C
import math

import numpy as np

import cpsz_b200


def _table(which):
    t = np.zeros(256)
    n = C.c_int()
    assert cpsz_b200.lib().cpsz_b200_debug_quant_table(which, t.ctypes.data_as(C.c_void_p), C.byref(n)) == 0
    return t, n.value


def _walk(x, d):
    for _ in range(abs(d)):
        x = np.nextafter(x, np.inf if d > 0 else -np.inf)
    return x


def test_2d_table_matches_log2_quantizer():
    t, n = _table(2)
    assert n == 256
    thr = 2.0 ** -52

    def ref(e):
        return 0 if e <= thr else int(math.log2(e / thr) / math.log2(4))

    for k in range(1, 60):
        for d in range(-40, 41):
            x = _walk(t[k], d)
            assert int(np.searchsorted(t[1:n], x, side="right")) == ref(x), (k, d)
    rng = np.random.default_rng(0)
    for x in 10.0 ** rng.uniform(-15, 3, 20000):
        assert int(np.searchsorted(t[1:n], x, side="right")) == ref(x)


def test_3d_table_matches_log2_quantizer():
    t, n = _table(3)
    thr = float(np.finfo(np.float32).eps)

    def ref(r):
        a = math.log2(1 + r)
        return 0 if a <= thr else int(math.log2(a / thr) / math.log2(2))

    for k in range(1, n):
        for d in range(-40, 41):
            x = _walk(t[k], d)
            if x > 0:
                assert int(np.searchsorted(t[1:n], x, side="right")) == ref(x), (k, d)


def test_2d_log_table_matches_log2_quantizer():
    """offline_log: id of log2(1 + eb) with base 2 and threshold DBL_EPSILON
    (src/sz_compress_cp_preserve_2d.cpp:345-350); t[0] is the largest bound
    that quantizes to precision 0."""
    t, n = _table(1)
    thr = 2.0 ** -52

    def prec0(r):
        return math.log2(1 + r) <= thr

    def ref(r):
        a = math.log2(1 + r)
        return 0 if a <= thr else int(math.log2(a / thr) / math.log2(2))

    assert prec0(t[0]) and not prec0(np.nextafter(t[0], np.inf))
    for k in range(1, n):
        for d in range(-40, 41):
            x = _walk(t[k], d)
            if x > t[0]:
                assert int(np.searchsorted(t[1:n], x, side="right")) == ref(x), (k, d)
    rng = np.random.default_rng(1)
    for x in 10.0 ** rng.uniform(-15.4, 0, 20000):
        if x > t[0]:
            assert int(np.searchsorted(t[1:n], x, side="right")) == ref(x)
