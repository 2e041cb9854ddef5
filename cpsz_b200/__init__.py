"""cpsz_b200 -- B200-native (sm_100a) cpSZ critical-point-preserving compressor.

Python mirror of the reference's public operator interface for the offline path
(bzhan166/cpSZ):

=============================================  =====================================================
reference (C++)                                here
=============================================  =====================================================
``sz_compress_cp_preserve_2d_offline<float>``  :func:`sz_compress_cp_preserve_2d_offline`
``sz_decompress_cp_preserve_2d_offline``       :func:`sz_decompress_cp_preserve_2d_offline`
``sz_compress_cp_preserve_2d_offline_log``     :func:`sz_compress_cp_preserve_2d_offline_log`
``sz_decompress_cp_preserve_2d_offline_log``   :func:`sz_decompress_cp_preserve_2d_offline_log`
``sz_compress_cp_preserve_3d_offline_log``     :func:`sz_compress_cp_preserve_3d_offline_log`
``sz_decompress_cp_preserve_3d_online_log``    :func:`sz_decompress_cp_preserve_3d_online_log`
``sz_lossless_compress/decompress`` (ZSTD)     :func:`sz_lossless_compress` / :func:`sz_lossless_decompress`
=============================================  =====================================================

Everything runs through ``libcpsz_b200.so`` (C ABI, ``include/cpsz_b200.h``):
hand-written CUDA kernels for sm_100a driven by C++ host code.  There is no CPU
fallback; without the library or a GPU every call raises :class:`CpszError`.
Fields are numpy arrays (host) or CUDA tensors/arrays exposing
``__cuda_array_interface__`` (device, used in place).
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "_lib", "libcpsz_b200.so")

CPSZ_OK = 0
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "out of memory", 4: "malformed blob", 5: "device wait timed out",
          6: "unsupported input", 7: "no CUDA device"}


class CpszError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{ERRORS.get(code, code)}] {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()
_sz = C.c_size_t
_vp = C.c_void_p


def _declare(L):
    L.cpsz_b200_last_error.restype = C.c_char_p
    L.cpsz_b200_version.restype = C.c_int
    L.cpsz_b200_ctx_create.argtypes = [C.c_int, C.POINTER(_vp)]
    L.cpsz_b200_ctx_destroy.argtypes = [_vp]
    L.cpsz_b200_ctx_kernel_launches.argtypes = [_vp, C.POINTER(C.c_uint64)]
    L.cpsz_b200_ctx_graph_stats.argtypes = [_vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.cpsz_b200_ctx_stream.argtypes = [_vp, C.POINTER(_vp)]
    L.cpsz_b200_ctx_wave_reruns.argtypes = [_vp, C.POINTER(C.c_uint64)]
    L.cpsz_b200_debug_band_wait.argtypes = [_vp, C.c_longlong, C.c_int]
    L.cpsz_b200_compress_2d_offline_f32.argtypes = [_vp, _vp, _vp, _sz, _sz, C.c_double, C.POINTER(_vp), C.POINTER(_sz)]
    L.cpsz_b200_compress_2d_offline_f32_into.argtypes = [_vp, _vp, _vp, _sz, _sz, C.c_double, _vp, _sz, C.POINTER(_sz)]
    L.cpsz_b200_decompress_2d_offline_f32.argtypes = [_vp, C.c_char_p, _sz, _sz, _sz, _vp, _vp]
    L.cpsz_b200_compress_2d_offline_log_f32.argtypes = [_vp, _vp, _vp, _sz, _sz, C.c_double, C.POINTER(_vp),
                                                        C.POINTER(_sz)]
    L.cpsz_b200_compress_2d_offline_log_f32_into.argtypes = [_vp, _vp, _vp, _sz, _sz, C.c_double, _vp, _sz,
                                                             C.POINTER(_sz)]
    L.cpsz_b200_decompress_2d_offline_log_f32.argtypes = [_vp, C.c_char_p, _sz, _sz, _sz, _vp, _vp]
    L.cpsz_b200_blob_size_2d_log.argtypes = [C.c_char_p, _sz, _sz]
    L.cpsz_b200_blob_size_2d_log.restype = _sz
    L.cpsz_b200_compress_2d_stages.argtypes = [_vp, _vp, _vp, _sz, _sz, C.c_double, _vp, _vp, _vp, _vp, _vp, _vp]
    L.cpsz_b200_blob_size_2d.argtypes = [C.c_char_p]
    L.cpsz_b200_blob_size_2d.restype = _sz
    L.cpsz_b200_generate_field_2d.argtypes = [C.c_uint64, _sz, _sz, C.c_int, C.c_double, C.c_double, _vp, _vp]
    L.cpsz_b200_generate_field_3d.argtypes = [C.c_uint64, _sz, _sz, _sz, C.c_int, C.c_double, C.c_double, _vp, _vp, _vp]
    L.cpsz_b200_batch_layout.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp]
    L.cpsz_b200_huffman_codebook.argtypes = [_vp, _sz, _sz, _vp, _vp, _vp, C.POINTER(_sz)]
    L.cpsz_b200_huffman_encode_u16.argtypes = [_vp, _vp, _sz, _vp, _vp, _vp, _sz, C.POINTER(C.c_uint64)]
    L.cpsz_b200_huffman_encode_u16_noalloc.argtypes = [_vp, _sz, _vp, _vp, _vp, _sz, _vp, _vp]
    L.cpsz_b200_lossless_bound.argtypes = [_sz]
    L.cpsz_b200_lossless_bound.restype = _sz
    L.cpsz_b200_lossless_compress.argtypes = [_vp, _vp, _sz, _vp, _sz, C.POINTER(_sz)]
    L.cpsz_b200_zstd_compress.argtypes = [C.c_char_p, _sz, C.c_int, C.POINTER(_vp), C.POINTER(_sz)]
    L.cpsz_b200_zstd_decompress.argtypes = [C.c_char_p, _sz, _vp, _sz]
    for name in ("cpsz_b200_compress_3d_offline_log_f32", "cpsz_b200_decompress_3d_online_log_f32",
                 "cpsz_b200_cp_check_2d", "cpsz_b200_cp_check_3d"):
        if hasattr(L, name):
            getattr(L, name).restype = C.c_int
    L.cpsz_b200_compress_2d_batch_f32.argtypes = [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp]
    L.cpsz_b200_compress_3d_offline_log_f32.argtypes = [_vp, _vp, _vp, _vp, _sz, _sz, _sz, C.c_double,
                                                        C.POINTER(_vp), C.POINTER(_sz)]
    L.cpsz_b200_compress_3d_offline_log_f32_into.argtypes = [_vp, _vp, _vp, _vp, _sz, _sz, _sz, C.c_double, _vp, _sz,
                                                             C.POINTER(_sz)]
    L.cpsz_b200_decompress_3d_online_log_f32.argtypes = [_vp, C.c_char_p, _sz, _sz, _sz, _sz, _vp, _vp, _vp]
    L.cpsz_b200_blob_size_3d.argtypes = [C.c_char_p, _sz, _sz, _sz]
    L.cpsz_b200_blob_size_3d.restype = _sz
    L.cpsz_b200_libm_tables_prepare.argtypes = [C.c_char_p]
    L.cpsz_b200_debug_eb3d.argtypes = [_vp, _vp, _vp, _vp, _sz, _sz, _sz, C.c_double, _vp, _vp]
    L.cpsz_b200_debug_eb2d.argtypes = [_vp, _vp, _vp, _sz, _sz, C.c_double, _vp, _vp]
    L.cpsz_b200_debug_libm.argtypes = [_vp, C.c_int, _vp, _sz, _vp]
    L.cpsz_b200_debug_filter_premises.argtypes = [_vp, _vp, _sz]
    L.cpsz_b200_mlp_propose_2d.argtypes = [_vp, _vp, _vp, _sz, _sz, _vp, _vp]
    L.cpsz_b200_debug_mlp_forward_ms.argtypes = [_vp, _vp, _vp, _sz, _sz, _vp, C.c_int, C.POINTER(C.c_float)]
    L.cpsz_b200_debug_umma_gemm.argtypes = [_vp, _vp, _vp, _vp]
    L.cpsz_b200_mlp_param_count.restype = _sz
    L.cpsz_b200_mlp_create.argtypes = [_vp, C.c_uint64, C.POINTER(_vp)]
    L.cpsz_b200_mlp_destroy.argtypes = [_vp]
    L.cpsz_b200_mlp_get_params.argtypes = [_vp, _vp]
    L.cpsz_b200_mlp_set_params.argtypes = [_vp, _vp]
    L.cpsz_b200_mlp_forward.argtypes = [_vp, _vp, _sz, _vp]
    L.cpsz_b200_mlp_train_step.argtypes = [_vp, _vp, _vp, _sz, C.c_float, _vp, _vp]
    L.cpsz_b200_mlp_features_2d.argtypes = [_vp, _vp, _vp, _sz, _sz, _vp, _vp, _sz, _vp]
    L.cpsz_b200_learned_labels_2d.argtypes = [_vp, _vp, _vp, _sz, _sz, _vp, _vp, _sz, C.c_int, _vp]
    L.cpsz_b200_compress_2d_learned_f32.argtypes = [_vp, _vp, _vp, _vp, _sz, _sz, C.c_double, _vp, _vp, _sz,
                                                    C.POINTER(_sz), _vp]
    L.cpsz_b200_ctx_set_timing.argtypes = [_vp, C.c_int]
    L.cpsz_b200_ctx_stage_times.argtypes = [_vp, C.c_int, _vp, _vp, C.POINTER(C.c_int)]
    L.cpsz_b200_tuning_param_count.restype = C.c_int
    L.cpsz_b200_tuning_param_info.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_int),
                                              C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.cpsz_b200_tuning_set.argtypes = [C.c_char_p, _sz, C.c_int]
    L.cpsz_b200_tuning_get.argtypes = [C.c_char_p, _sz, C.POINTER(C.c_int)]
    L.cpsz_b200_tuning_load.argtypes = [C.c_char_p]
    L.cpsz_b200_tuning_source.restype = C.c_char_p
    if hasattr(L, "cpsz_b200_cp_check_2d"):
        L.cpsz_b200_cp_check_2d.argtypes = [_vp, _vp, _vp, _vp, _vp, _sz, _sz, _vp, C.POINTER(C.c_uint64)]
        L.cpsz_b200_cp_check_3d.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _sz, _sz, _vp,
                                            C.POINTER(C.c_uint64)]


def lib():
    """The loaded native library (built in-tree on first use if absent)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                from . import build as _b
                _b.build()
            L = C.CDLL(LIB_PATH)
            _declare(L)
            _lib = L
    return _lib


def _check(rc: int):
    if rc != CPSZ_OK:
        raise CpszError(rc, lib().cpsz_b200_last_error().decode(errors="replace"))


class Context:
    """A device workspace + stream (``cpsz_b200_ctx``)."""

    def __init__(self, device: int = 0):
        h = _vp()
        _check(lib().cpsz_b200_ctx_create(device, C.byref(h)))
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            lib().cpsz_b200_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def kernel_launches(self) -> int:
        v = C.c_uint64()
        _check(lib().cpsz_b200_ctx_kernel_launches(self.handle, C.byref(v)))
        return v.value

    @property
    def graph_stats(self) -> tuple:
        """(graphs captured, batch passes replayed from a captured graph)."""
        c, r = C.c_uint64(), C.c_uint64()
        _check(lib().cpsz_b200_ctx_graph_stats(self.handle, C.byref(c), C.byref(r)))
        return c.value, r.value

    @property
    def wave_reruns(self) -> int:
        """Passes whose wavefront ran again after the bounds because a wait
        beside the bound kernel gave up (``cpsz_b200_ctx_wave_reruns``)."""
        v = C.c_uint64()
        _check(lib().cpsz_b200_ctx_wave_reruns(self.handle, C.byref(v)))
        return v.value

    def debug_band_wait(self, wait_ns: int = 0, unreachable: bool = False) -> None:
        """Limit of the wavefront's per-group wait for the bounds (0 = default);
        ``unreachable`` makes every such wait run out (``cpsz_b200_debug_band_wait``)."""
        _check(lib().cpsz_b200_debug_band_wait(self.handle, int(wait_ns), int(bool(unreachable))))

    @property
    def stream(self) -> int:
        v = _vp()
        _check(lib().cpsz_b200_ctx_stream(self.handle, C.byref(v)))
        return v.value or 0

    def set_timing(self, on: bool = True) -> None:
        """Per-stage CUDA-event timing of the following calls (``cpsz_b200_ctx_set_timing``)."""
        _check(lib().cpsz_b200_ctx_set_timing(self.handle, int(bool(on))))

    def stage_times(self) -> dict:
        """{stage name: ms} of the last call made with timing on; repeated names are summed."""
        names = (C.c_char_p * 24)()
        ms = (C.c_float * 24)()
        n = C.c_int()
        _check(lib().cpsz_b200_ctx_stage_times(self.handle, 24, names, ms, C.byref(n)))
        out: dict = {}
        for k in range(n.value):
            nm = names[k].decode()
            out[nm] = out.get(nm, 0.0) + float(ms[k])
        return out


# ---- launch-shape tuning table (output-invariant parameters) ----------------

def tuning_params() -> dict:
    """{name: (default, lo, hi)} of every launch-shape parameter."""
    L = lib()
    out = {}
    for k in range(L.cpsz_b200_tuning_param_count()):
        nm, d, lo, hi = C.c_char_p(), C.c_int(), C.c_int(), C.c_int()
        _check(L.cpsz_b200_tuning_param_info(k, C.byref(nm), C.byref(d), C.byref(lo), C.byref(hi)))
        out[nm.value.decode()] = (d.value, lo.value, hi.value)
    return out


def tuning_set(param: str, value: int, min_points: int = 0) -> None:
    _check(lib().cpsz_b200_tuning_set(param.encode(), int(min_points), int(value)))


def tuning_get(param: str, points: int) -> int:
    v = C.c_int()
    _check(lib().cpsz_b200_tuning_get(param.encode(), int(points), C.byref(v)))
    return v.value


def tuning_clear() -> None:
    _check(lib().cpsz_b200_tuning_clear())


def tuning_load(path: str | None = None) -> None:
    _check(lib().cpsz_b200_tuning_load(path.encode() if path else None))


def tuning_source() -> str:
    return (lib().cpsz_b200_tuning_source() or b"").decode()


def _h(ctx):
    return ctx.handle if ctx is not None else None


def _ptr(a, dtype=np.float32):
    """(pointer, keepalive, shape) of a host numpy array or a device array."""
    if hasattr(a, "__cuda_array_interface__"):
        cai = a.__cuda_array_interface__
        got, want = np.dtype(cai["typestr"]), np.dtype(dtype)
        same_int = got.kind in "iu" and want.kind in "iu" and got.itemsize == want.itemsize
        if got != want and not same_int:
            raise TypeError(f"expected {want} device array, got {got}")
        if cai.get("strides") not in (None,):
            exp = []
            s = np.dtype(dtype).itemsize
            for d in reversed(cai["shape"]):
                exp.insert(0, s)
                s *= d
            if tuple(cai["strides"]) != tuple(exp):
                raise TypeError("device array must be C-contiguous")
        return cai["data"][0], a, tuple(cai["shape"])
    arr = np.ascontiguousarray(a, dtype=dtype)
    return arr.ctypes.data, arr, arr.shape


# ---- 2D ---------------------------------------------------------------------------

def sz_compress_cp_preserve_2d_offline(U, V, r1: int | None = None, r2: int | None = None, max_pwr_eb: float = 0.1,
                                       ctx: Context | None = None) -> bytes:
    """GPU ``sz_compress_cp_preserve_2d_offline<float>``: returns the blob (bytes)."""
    pu, ku, su = _ptr(U)
    pv, kv, sv = _ptr(V)
    if r1 is None:
        r1, r2 = su
    if su != sv or int(np.prod(su)) != r1 * r2:
        raise ValueError("U and V must both hold r1*r2 floats")
    out = _vp()
    n = _sz()
    _check(lib().cpsz_b200_compress_2d_offline_f32(_h(ctx), pu, pv, r1, r2, float(max_pwr_eb), C.byref(out),
                                                   C.byref(n)))
    try:
        return C.string_at(out, n.value)
    finally:
        C.CDLL(None).free(out)


def compress_2d_into(U, V, r1, r2, max_pwr_eb, out, ctx: Context | None = None) -> int:
    """Compress into caller memory ``out`` (host numpy uint8 or device uint8 array); returns the blob size."""
    pu, ku, _ = _ptr(U)
    pv, kv, _ = _ptr(V)
    po, ko, so = _ptr(out, np.uint8)
    n = _sz()
    _check(lib().cpsz_b200_compress_2d_offline_f32_into(_h(ctx), pu, pv, r1, r2, float(max_pwr_eb), po,
                                                        int(np.prod(so)), C.byref(n)))
    return n.value


def compress_2d_batch(fields, ebs, out=None, ctx: Context | None = None):
    """Batched 2D compression of [(U, V), ...] with per-field bounds.

    With out=None returns the list of blobs (bytes); with `out` (host numpy
    uint8 or device uint8 array) writes them back to back and returns the
    offsets array (n + 1 entries)."""
    n = len(fields)
    ptrs_u = (_vp * max(n, 1))()
    ptrs_v = (_vp * max(n, 1))()
    r1 = np.zeros(max(n, 1), np.uint64)
    r2 = np.zeros(max(n, 1), np.uint64)
    keep = []
    for k, (U, V) in enumerate(fields):
        pu, _, su = _ptr(U)
        pv, _, sv = _ptr(V)
        if su != sv or len(su) != 2:
            raise ValueError("each field is a pair of equal 2D arrays")
        ptrs_u[k], ptrs_v[k] = pu, pv
        r1[k], r2[k] = su
        keep.append((U, V))
    ebs = np.ascontiguousarray(np.broadcast_to(np.asarray(ebs, np.float64), (n,)))
    ret_bytes = out is None
    if out is None:
        cap = sum(int(a.size) * 8 for a, _ in fields) * 2 + n * (4 << 20) + (1 << 20)
        out = np.empty(cap, np.uint8)
    po, _, so = _ptr(out, np.uint8)
    offsets = np.zeros(n + 1, np.uint64)
    _check(lib().cpsz_b200_compress_2d_batch_f32(_h(ctx), n, ptrs_u, ptrs_v, r1.ctypes.data, r2.ctypes.data,
                                                 ebs.ctypes.data, po, int(np.prod(so)), offsets.ctypes.data))
    if ret_bytes:
        return [out[int(offsets[k]):int(offsets[k + 1])].tobytes() for k in range(n)]
    return offsets


def sz_decompress_cp_preserve_2d_offline(blob: bytes, r1: int, r2: int, U=None, V=None,
                                         ctx: Context | None = None):
    """GPU ``sz_decompress_cp_preserve_2d_offline<float>``: returns (U, V).

    U, V may be given as preallocated host or device float32 arrays of r1*r2."""
    if U is None:
        U = np.empty((r1, r2), np.float32)
    if V is None:
        V = np.empty((r1, r2), np.float32)
    pu, ku, _ = _ptr(U)
    pv, kv, _ = _ptr(V)
    if ku is not U or kv is not V:
        raise TypeError("output arrays must be C-contiguous float32")
    _check(lib().cpsz_b200_decompress_2d_offline_f32(_h(ctx), blob, len(blob), r1, r2, pu, pv))
    return U, V


def sz_compress_cp_preserve_2d_offline_log(U, V, r1: int | None = None, r2: int | None = None,
                                           max_pwr_eb: float = 0.1, ctx: Context | None = None) -> bytes:
    """GPU ``sz_compress_cp_preserve_2d_offline_log<float>``: returns the blob (bytes)."""
    pu, ku, su = _ptr(U)
    pv, kv, sv = _ptr(V)
    if r1 is None:
        r1, r2 = su
    if su != sv or int(np.prod(su)) != r1 * r2:
        raise ValueError("U and V must both hold r1*r2 floats")
    out = _vp()
    n = _sz()
    _check(lib().cpsz_b200_compress_2d_offline_log_f32(_h(ctx), pu, pv, r1, r2, float(max_pwr_eb), C.byref(out),
                                                       C.byref(n)))
    try:
        return C.string_at(out, n.value)
    finally:
        C.CDLL(None).free(out)


def compress_2d_log_into(U, V, r1, r2, max_pwr_eb, out, ctx: Context | None = None) -> int:
    """The offline_log compressor into caller memory ``out`` (host or device uint8); returns the blob size."""
    pu, ku, _ = _ptr(U)
    pv, kv, _ = _ptr(V)
    po, ko, so = _ptr(out, np.uint8)
    n = _sz()
    _check(lib().cpsz_b200_compress_2d_offline_log_f32_into(_h(ctx), pu, pv, r1, r2, float(max_pwr_eb), po,
                                                            int(np.prod(so)), C.byref(n)))
    return n.value


def sz_decompress_cp_preserve_2d_offline_log(blob: bytes, r1: int, r2: int, U=None, V=None,
                                             ctx: Context | None = None):
    """GPU ``sz_decompress_cp_preserve_2d_offline_log<float>``: returns (U, V)."""
    if U is None:
        U = np.empty((r1, r2), np.float32)
    if V is None:
        V = np.empty((r1, r2), np.float32)
    pu, ku, _ = _ptr(U)
    pv, kv, _ = _ptr(V)
    if ku is not U or kv is not V:
        raise TypeError("output arrays must be C-contiguous float32")
    _check(lib().cpsz_b200_decompress_2d_offline_log_f32(_h(ctx), blob, len(blob), r1, r2, pu, pv))
    return U, V


def compress_2d_stages(U, V, max_pwr_eb: float, ctx: Context | None = None) -> dict:
    """Intermediate streams of the 2D compressor (ids, block-order codes, reconstruction)."""
    U = np.ascontiguousarray(U, np.float32)
    V = np.ascontiguousarray(V, np.float32)
    r1, r2 = U.shape
    n = r1 * r2
    ids = np.empty(2 * n, np.int32)
    cu = np.empty(n, np.int32)
    cv = np.empty(n, np.int32)
    ru = np.empty((r1, r2), np.float32)
    rv = np.empty((r1, r2), np.float32)
    nu = (C.c_size_t * 2)()
    _check(lib().cpsz_b200_compress_2d_stages(_h(ctx), U.ctypes.data, V.ctypes.data, r1, r2, float(max_pwr_eb),
                                              ids.ctypes.data, cu.ctypes.data, cv.ctypes.data, ru.ctypes.data,
                                              rv.ctypes.data, C.addressof(nu)))
    return {"ids": ids, "codes_u": cu, "codes_v": cv, "recon_u": ru, "recon_v": rv, "n_unpred": (nu[0], nu[1])}


def blob_size_2d(blob: bytes) -> int:
    return lib().cpsz_b200_blob_size_2d(blob)


# ---- 3D ---------------------------------------------------------------------------

def sz_compress_cp_preserve_3d_offline_log(U, V, W, r1=None, r2=None, r3=None, max_pwr_eb: float = 0.1,
                                           ctx: Context | None = None) -> bytes:
    """GPU ``sz_compress_cp_preserve_3d_offline_log<float>``: returns the blob (bytes)."""
    pu, ku, su = _ptr(U)
    pv, kv, sv = _ptr(V)
    pw, kw, sw = _ptr(W)
    if r1 is None:
        r1, r2, r3 = su
    if not (su == sv == sw) or int(np.prod(su)) != r1 * r2 * r3:
        raise ValueError("U, V, W must each hold r1*r2*r3 floats")
    out = _vp()
    n = _sz()
    _check(lib().cpsz_b200_compress_3d_offline_log_f32(_h(ctx), pu, pv, pw, r1, r2, r3, float(max_pwr_eb),
                                                       C.byref(out), C.byref(n)))
    try:
        return C.string_at(out, n.value)
    finally:
        C.CDLL(None).free(out)


def sz_decompress_cp_preserve_3d_online_log(blob: bytes, r1: int, r2: int, r3: int, U=None, V=None, W=None,
                                            ctx: Context | None = None):
    """GPU ``sz_decompress_cp_preserve_3d_online_log<float>``: returns (U, V, W)."""
    outs = []
    for a in (U, V, W):
        outs.append(np.empty((r1, r2, r3), np.float32) if a is None else a)
    ptrs = [_ptr(a)[0] for a in outs]
    _check(lib().cpsz_b200_decompress_3d_online_log_f32(_h(ctx), blob, len(blob), r1, r2, r3, *ptrs))
    return tuple(outs)


def compress_3d_into(U, V, W, r1, r2, r3, max_pwr_eb, out, ctx: Context | None = None) -> int:
    """3D compression into a caller buffer (numpy uint8 or device array); returns the blob size."""
    pu, _, _ = _ptr(U)
    pv, _, _ = _ptr(V)
    pw, _, _ = _ptr(W)
    po, _, so = _ptr(out, np.uint8)
    n = _sz()
    _check(lib().cpsz_b200_compress_3d_offline_log_f32_into(_h(ctx), pu, pv, pw, r1, r2, r3, float(max_pwr_eb), po,
                                                            int(np.prod(so)), C.byref(n)))
    return n.value


def blob_size_3d(blob: bytes, r1: int, r2: int, r3: int) -> int:
    return lib().cpsz_b200_blob_size_3d(blob, r1, r2, r3)


def libm_tables_prepare(path: str | None = None) -> None:
    """Builds (or loads) the host log2f / exp2f tables the 3D kernels use."""
    _check(lib().cpsz_b200_libm_tables_prepare(path.encode() if path else None))


def debug_eb2d(U, V, max_pwr_eb: float, ctx: Context | None = None, exact: bool = True):
    """Per-vertex 2D analytic bound (float64) and id bytes (2N; 255 = precision 0) from the GPU kernel.

    exact=False runs the compressor's filtered path and returns (None, ids)."""
    U = np.ascontiguousarray(U, np.float32)
    V = np.ascontiguousarray(V, np.float32)
    r1, r2 = U.shape
    eb = np.empty(U.shape, np.float64) if exact else None
    ids = np.empty(2 * U.size, np.uint8)
    _check(lib().cpsz_b200_debug_eb2d(_h(ctx), U.ctypes.data, V.ctypes.data, r1, r2, float(max_pwr_eb),
                                      eb.ctypes.data if exact else None, ids.ctypes.data))
    return eb, ids


def debug_eb3d(U, V, W, max_pwr_eb: float, ctx: Context | None = None):
    """Per-vertex 3D bound (float64) and id bytes (255 = bound not positive) from the GPU kernel."""
    U, V, W = (np.ascontiguousarray(a, np.float32) for a in (U, V, W))
    r1, r2, r3 = U.shape
    eb = np.empty(U.shape, np.float64)
    ids = np.empty(U.shape, np.uint8)
    _check(lib().cpsz_b200_debug_eb3d(_h(ctx), U.ctypes.data, V.ctypes.data, W.ctypes.data, r1, r2, r3,
                                      float(max_pwr_eb), eb.ctypes.data, ids.ctypes.data))
    return eb, ids


# ---- learned error bounds ----------------------------------------------------------------

class Mlp:
    """The learned bound proposer (99 -> 128 -> 128 -> 1 MLP on the tensor cores)."""

    def __init__(self, ctx: Context, seed: int = 0, params=None):
        self.ctx = ctx
        h = _vp()
        _check(lib().cpsz_b200_mlp_create(ctx.handle, seed, C.byref(h)))
        self.handle = h
        if params is not None:
            self.set_params(params)

    @staticmethod
    def param_count() -> int:
        return int(lib().cpsz_b200_mlp_param_count())

    def params(self) -> np.ndarray:
        out = np.empty(self.param_count(), np.float32)
        _check(lib().cpsz_b200_mlp_get_params(self.handle, out.ctypes.data))
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.param_count()
        _check(lib().cpsz_b200_mlp_set_params(self.handle, p.ctypes.data))

    def forward(self, X_bits) -> np.ndarray:
        X = np.ascontiguousarray(X_bits, np.uint16)
        y = np.empty(X.shape[0], np.float32)
        _check(lib().cpsz_b200_mlp_forward(self.handle, X.ctypes.data, X.shape[0], y.ctypes.data))
        return y

    def forward_ms(self, U, V, eb_analytic, reps: int = 5) -> float:
        """Mean time (ms, CUDA events) of the fused forward pass over every vertex
        of field (U, V) with analytic bounds eb_analytic (device arrays)."""
        pu, _, su = _ptr(U)
        pv, _, _ = _ptr(V)
        pe, _, _ = _ptr(eb_analytic, np.float64)
        ms = C.c_float()
        _check(lib().cpsz_b200_debug_mlp_forward_ms(self.handle, pu, pv, su[0], su[1], pe, int(reps), C.byref(ms)))
        return ms.value

    def train_step(self, X_bits, t, lr: float, grads: bool = False):
        """(mean squared error, gradients or None); Adam step when lr > 0."""
        X = np.ascontiguousarray(X_bits, np.uint16)
        t = np.ascontiguousarray(t, np.float32)
        g = np.empty(self.param_count(), np.float32) if grads else None
        loss = C.c_float()
        _check(lib().cpsz_b200_mlp_train_step(self.handle, X.ctypes.data, t.ctypes.data, X.shape[0], float(lr),
                                               g.ctypes.data if grads else None, C.byref(loss)))
        return loss.value, g

    def close(self):
        # the MLP lives on its context's stream: once the context is closed
        # there is nothing left to release through it (its device memory goes
        # with the process)
        if getattr(self, "handle", None):
            if getattr(self.ctx, "handle", None):
                lib().cpsz_b200_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mlp_features_2d(U, V, eb_analytic, idx, ctx: Context | None = None) -> np.ndarray:
    U = np.ascontiguousarray(U, np.float32)
    V = np.ascontiguousarray(V, np.float32)
    eb = np.ascontiguousarray(eb_analytic, np.float64)
    idx = np.ascontiguousarray(idx, np.int32)
    X = np.empty((idx.size, 128), np.uint16)
    _check(lib().cpsz_b200_mlp_features_2d(_h(ctx), U.ctypes.data, V.ctypes.data, U.shape[0], U.shape[1],
                                           eb.ctypes.data, idx.ctypes.data, idx.size, X.ctypes.data))
    return X


def mlp_propose_2d(mlp, U, V, eb_analytic) -> np.ndarray:
    """The proposer's raw outputs (log2 multipliers) for every vertex of (U, V)."""
    U = np.ascontiguousarray(U, np.float32)
    V = np.ascontiguousarray(V, np.float32)
    eb = np.ascontiguousarray(eb_analytic, np.float64)
    y = np.empty(U.shape, np.float32)
    _check(lib().cpsz_b200_mlp_propose_2d(mlp.handle, U.ctypes.data, V.ctypes.data, U.shape[0], U.shape[1],
                                          eb.ctypes.data, y.ctypes.data))
    return y


def learned_labels_2d(U, V, eb_analytic, idx, steps: int = 16, ctx: Context | None = None) -> np.ndarray:
    U = np.ascontiguousarray(U, np.float32)
    V = np.ascontiguousarray(V, np.float32)
    eb = np.ascontiguousarray(eb_analytic, np.float64)
    idx = np.ascontiguousarray(idx, np.int32)
    t = np.empty(idx.size, np.float32)
    _check(lib().cpsz_b200_learned_labels_2d(_h(ctx), U.ctypes.data, V.ctypes.data, U.shape[0], U.shape[1],
                                             eb.ctypes.data, idx.ctypes.data, idx.size, steps, t.ctypes.data))
    return t


def compress_2d_learned(U, V, max_pwr_eb: float = 0.1, mlp: Mlp | None = None, log2_mult=None, out=None,
                        ctx: Context | None = None):
    """2D offline blob with learned bounds; returns (blob bytes or size, stats dict)."""
    pu, _, su = _ptr(U)
    pv, _, sv = _ptr(V)
    r1, r2 = su
    pm = None
    keep = None
    if log2_mult is not None:
        pm, keep, _ = _ptr(log2_mult)
    ret_bytes = out is None
    if out is None:
        out = np.empty(int(np.prod(su)) * 8 + (8 << 20), np.uint8)
    po, _, so = _ptr(out, np.uint8)
    n = _sz()
    stats = np.zeros(4, np.uint64)
    _check(lib().cpsz_b200_compress_2d_learned_f32(_h(ctx), mlp.handle if mlp else None, pu, pv, r1, r2,
                                                   float(max_pwr_eb), pm, po, int(np.prod(so)), C.byref(n),
                                                   stats.ctypes.data))
    st = {"passes": int(stats[0]), "reverted": int(stats[1]), "fell_back": int(stats[2]), "kept": int(stats[3])}
    del keep
    if ret_bytes:
        return out[:n.value].tobytes(), st
    return n.value, st


def debug_filter_premises(ctx: Context | None = None) -> dict:
    """Exhaustive maxima, on this device, of the operations whose error bounds
    the filtered 2D / 3D bounds rely on: acbrt1 relative error above / below a
    double cube root ("acbrt1_hi", "acbrt1_lo"), the relative errors of
    rcp.approx, ex2.approx and sqrt.approx, and lg2.approx's absolute error
    per binade ("lg2": {e: max over [2^e, 2^(e+1))}, e = -126..0)."""
    out = np.zeros(132, np.float64)
    _check(lib().cpsz_b200_debug_filter_premises(_h(ctx), out.ctypes.data, out.size))
    return {"acbrt1_hi": out[0], "acbrt1_lo": out[1], "rcp": out[2], "ex2": out[3], "sqrt": out[4],
            "lg2": {e: out[5 + e + 126] for e in range(-126, 1)}}


def debug_libm(which: str, x, ctx: Context | None = None):
    """The GPU's reproduction of the host library's log2f ('log2f') or exp2f ('exp2f')."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    _check(lib().cpsz_b200_debug_libm(_h(ctx), {"log2f": 0, "exp2f": 1}[which], x.ctypes.data, x.size,
                                      out.ctypes.data))
    return out


def to_bf16_bits(x) -> np.ndarray:
    """float32 -> bfloat16 bit patterns (round to nearest even)."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint16)


def bf16_bits_to_f32(b) -> np.ndarray:
    return (np.asarray(b, np.uint32) << 16).view(np.float32)


def debug_umma_gemm(A_bits, B_bits, ctx: Context | None = None):
    """128x128 fp32 D = A B^T from bf16 bit arrays, on the tensor cores (tcgen05)."""
    A = np.ascontiguousarray(A_bits, np.uint16)
    B = np.ascontiguousarray(B_bits, np.uint16)
    assert A.shape == (128, 128) and B.shape == (128, 128)
    D = np.zeros((128, 128), np.float32)
    _check(lib().cpsz_b200_debug_umma_gemm(_h(ctx), A.ctypes.data, B.ctypes.data, D.ctypes.data))
    return D


# ---- exact critical-point check ------------------------------------------------------

CP_TYPES_2D = ("NONE", "SINGULAR", "ATTRACTING", "REPELLING", "SADDLE", "ATTRACTING_FOCUS", "REPELLING_FOCUS",
               "CENTER")


def cp_check_2d(Ua, Va, Ub=None, Vb=None, cells: bool = False, ctx: Context | None = None):
    """Exact per-cell CP classification of (Ua, Va), compared with (Ub, Vb) if given.

    Returns dict(cps_a, cps_b, lost_or_spurious, type_changed[, cells])."""
    pa = [_ptr(a) for a in (Ua, Va)]
    r1, r2 = pa[0][2]
    pb = [_ptr(b) for b in (Ub, Vb)] if Ub is not None else None
    ncell = 2 * (r1 - 1) * (r2 - 1) if r1 > 1 and r2 > 1 else 0
    out = np.zeros(max(ncell, 1), np.uint8) if cells else None
    counts = (C.c_uint64 * 4)()
    _check(lib().cpsz_b200_cp_check_2d(_h(ctx), pa[0][0], pa[1][0], pb[0][0] if pb else None,
                                       pb[1][0] if pb else None, r1, r2, out.ctypes.data if cells else None, counts))
    res = {"cps_a": counts[0], "cps_b": counts[1], "lost_or_spurious": counts[2], "type_changed": counts[3]}
    if cells:
        res["cells"] = out[:ncell]
    return res


def cp_check_3d(Ua, Va, Wa, Ub=None, Vb=None, Wb=None, cells: bool = False, ctx: Context | None = None):
    pa = [_ptr(a) for a in (Ua, Va, Wa)]
    r1, r2, r3 = pa[0][2]
    pb = [_ptr(b) for b in (Ub, Vb, Wb)] if Ub is not None else None
    ncell = 6 * (r1 - 1) * (r2 - 1) * (r3 - 1) if min(r1, r2, r3) > 1 else 0
    out = np.zeros(max(ncell, 1), np.uint8) if cells else None
    counts = (C.c_uint64 * 4)()
    _check(lib().cpsz_b200_cp_check_3d(_h(ctx), pa[0][0], pa[1][0], pa[2][0], pb[0][0] if pb else None,
                                       pb[1][0] if pb else None, pb[2][0] if pb else None, r1, r2, r3,
                                       out.ctypes.data if cells else None, counts))
    res = {"cps_a": counts[0], "cps_b": counts[1], "lost_or_spurious": counts[2], "type_changed": counts[3]}
    if cells:
        res["cells"] = out[:ncell]
    return res


# ---- Huffman stage ----------------------------------------------------------------------

def huffman_codebook(hist, state_num: int):
    """(code[u64], len[u8], tree_section bytes) of the reference's tree for a histogram."""
    hist = np.ascontiguousarray(hist, np.uint64)
    bins = hist.size
    code = np.zeros(bins, np.uint64)
    ln = np.zeros(bins, np.uint8)
    size = _sz(0)
    _check(lib().cpsz_b200_huffman_codebook(hist.ctypes.data, bins, state_num, None, None, None, C.byref(size)))
    tree = np.zeros(size.value, np.uint8)
    _check(lib().cpsz_b200_huffman_codebook(hist.ctypes.data, bins, state_num, code.ctypes.data, ln.ctypes.data,
                                            tree.ctypes.data, C.byref(size)))
    return code, ln, tree.tobytes()


def huffman_encode_u16(sym, code, ln, out, ctx: Context | None = None) -> int:
    """GPU bit packing of device uint16 symbols with a device codebook into device `out`; returns the bit count."""
    ps, ks, ss = _ptr(sym, np.uint16)
    pc, kc, _ = _ptr(code, np.uint64)
    pl, kl, _ = _ptr(ln, np.uint8)
    po, ko, so = _ptr(out, np.uint8)
    bits = C.c_uint64()
    _check(lib().cpsz_b200_huffman_encode_u16(_h(ctx), ps, int(np.prod(ss)), pc, pl, po, int(np.prod(so)),
                                              C.byref(bits)))
    return bits.value


def huffman_encode_u16_noalloc(sym, code, ln, out, total_bits, stream: int = 0) -> None:
    """The allocation-free variant: all arguments are device arrays (total_bits: one uint64);
    enqueued on `stream` (a cudaStream_t value) without waiting."""
    ps, ks, ss = _ptr(sym, np.uint16)
    pc, kc, _ = _ptr(code, np.uint64)
    pl, kl, _ = _ptr(ln, np.uint8)
    po, ko, so = _ptr(out, np.uint8)
    pt, kt, _ = _ptr(total_bits, np.uint64)
    _check(lib().cpsz_b200_huffman_encode_u16_noalloc(ps, int(np.prod(ss)), pc, pl, po, int(np.prod(so)), pt,
                                                      stream or None))


# ---- lossless stage (host ZSTD, as the reference) -------------------------------------

def lossless_compress_gpu(data, out=None, ctx: Context | None = None):
    """GPU Zstandard frame of `data` (bytes / host uint8 array, or a device
    uint8 array).  Returns bytes, or with `out` (host or device uint8 array)
    the frame size written there."""
    if isinstance(data, (bytes, bytearray, memoryview)):
        data = np.frombuffer(bytes(data), np.uint8)
    pi, ki, si = _ptr(data, np.uint8)
    n = int(np.prod(si))
    size = _sz()
    if out is None:
        buf = np.empty(lib().cpsz_b200_lossless_bound(n), np.uint8)
        _check(lib().cpsz_b200_lossless_compress(_h(ctx), pi, n, buf.ctypes.data, buf.size, C.byref(size)))
        return buf[:size.value].tobytes()
    po, ko, so = _ptr(out, np.uint8)
    _check(lib().cpsz_b200_lossless_compress(_h(ctx), pi, n, po, int(np.prod(so)), C.byref(size)))
    return size.value


def sz_lossless_compress(data: bytes, level: int = 3) -> bytes:
    out = _vp()
    n = _sz()
    _check(lib().cpsz_b200_zstd_compress(data, len(data), level, C.byref(out), C.byref(n)))
    try:
        return C.string_at(out, n.value)
    finally:
        C.CDLL(None).free(out)


def sz_lossless_decompress(data: bytes, target_size: int) -> bytes:
    buf = C.create_string_buffer(target_size)
    _check(lib().cpsz_b200_zstd_decompress(data, len(data), C.addressof(buf), target_size))
    return buf.raw


from . import workloads  # noqa: E402  (synthetic generators; needs lib())

__all__ = [
    "Context", "CpszError", "lib", "sz_compress_cp_preserve_2d_offline", "sz_decompress_cp_preserve_2d_offline",
    "sz_compress_cp_preserve_3d_offline_log", "sz_decompress_cp_preserve_3d_online_log", "compress_2d_into",
    "compress_2d_stages", "cp_check_2d", "cp_check_3d", "sz_lossless_compress", "sz_lossless_decompress",
    "workloads",
]
