"""CPU oracle for the cpSZ offline path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import this package; the product (``cpsz_b200``) never does.  It exposes

* :class:`Oracle` -- ctypes bindings of ``oracle/_build/libcpsz_oracle.so``, the
  plain-C restatement of the reference (``cpsz_oracle*.c``), built by
  ``make -C oracle`` (gcc only, so it can be rebuilt on any box), and
* :class:`Reference` -- bindings of ``oracle/_ref/libcpsz_ref.so``, the
  reference's own sources compiled by ``make -C oracle ref`` (only where the
  reference sources are present; the built .so then travels with the tree).
* :mod:`oracle.cp_exact` -- exact-rational critical-point classification used
  to check the CUDA checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libcpsz_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libcpsz_ref.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_sz = C.c_size_t


def build_oracle(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("cpsz_oracle.c", "cpsz_oracle_huffman.c", "cpsz_oracle_3d.c",
                                            "cpsz_oracle_gen.c", "cpsz_oracle.h")]
    if force or not os.path.exists(ORACLE_SO) or any(os.path.getmtime(s) > os.path.getmtime(ORACLE_SO) for s in srcs):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return ORACLE_SO


def build_reference(ref_dir: str | None = None) -> str | None:
    """Compile the reference sources into oracle/_ref when they are present
    (``ref_dir``, else the environment variable ``CPSZ_REF_DIR``); returns the
    library path, or None when it is neither built nor buildable here."""
    ref_dir = ref_dir or os.environ.get("CPSZ_REF_DIR")
    if ref_dir and os.path.isdir(os.path.join(ref_dir, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_DIR={ref_dir}"], check=True)
    return REF_SO if os.path.exists(REF_SO) else None


def _take_blob(lib, ptr, size) -> bytes:
    if not ptr:
        raise ValueError("input outside the compressor's domain (bound ids out of range)")
    out = C.string_at(ptr, size)
    lib.cpo_free(ptr) if hasattr(lib, "cpo_free") else lib.cpsz_ref_free(ptr)
    return out


class Oracle:
    """Bindings of the plain-C restatement."""

    def __init__(self, path: str | None = None):
        self.lib = C.CDLL(path or build_oracle())
        L = self.lib
        L.cpo_eb_2d.argtypes = [_f32p, _f32p, _sz, _sz, C.c_double, _f64p]
        L.cpo_quantize_eb_2d.argtypes = [_f32p, _f32p, _f64p, _sz, _i32p, _f64p, _f64p]
        L.cpo_lorenzo_2d.argtypes = [_f32p, _f64p, _sz, _sz, _i32p, _f32p, _f32p]
        L.cpo_lorenzo_2d.restype = _sz
        L.cpo_compress_2d_offline.argtypes = [_f32p, _f32p, _sz, _sz, C.c_double, C.POINTER(_sz)]
        L.cpo_compress_2d_offline.restype = C.c_void_p
        L.cpo_decompress_2d_offline.argtypes = [C.c_char_p, _sz, _sz, _sz, _f32p, _f32p]
        L.cpo_compress_2d_offline_log.argtypes = [_f32p, _f32p, _sz, _sz, C.c_double, C.POINTER(_sz)]
        L.cpo_compress_2d_offline_log.restype = C.c_void_p
        L.cpo_decompress_2d_offline_log.argtypes = [C.c_char_p, _sz, _sz, _sz, _f32p, _f32p]
        L.cpo_huffman_encode.argtypes = [_sz, _i32p, _sz, C.c_void_p]
        L.cpo_huffman_encode.restype = _sz
        L.cpo_huffman_encode_bound.argtypes = [_sz, _sz]
        L.cpo_huffman_encode_bound.restype = _sz
        L.cpo_huffman_decode.argtypes = [_sz, _sz, C.c_char_p, _sz, _i32p]
        L.cpo_huffman_decode.restype = _sz
        L.cpo_huffman_code_lengths.argtypes = [_sz, _i32p, _sz, _u8p]
        L.cpo_huffman_code_lengths.restype = _sz
        L.cpo_eb_3d.argtypes = [_f32p, _f32p, _f32p, _sz, _sz, _sz, C.c_double, _f64p]
        L.cpo_compress_3d_offline_log.argtypes = [_f32p, _f32p, _f32p, _sz, _sz, _sz, C.c_double, C.POINTER(_sz)]
        L.cpo_compress_3d_offline_log.restype = C.c_void_p
        L.cpo_decompress_3d_online_log.argtypes = [C.c_char_p, _sz, _sz, _sz, _sz, _f32p, _f32p, _f32p]
        L.cpo_free.argtypes = [C.c_void_p]
        L.cpo_log2f_array.argtypes = [_f32p, _sz, _f32p]
        L.cpo_exp2f_array.argtypes = [_f32p, _sz, _f32p]
        L.cpo_generate_field_2d.argtypes = [C.c_uint64, _sz, _sz, C.c_int, C.c_double, C.c_double, _f32p, _f32p]
        L.cpo_generate_field_3d.argtypes = [C.c_uint64, _sz, _sz, _sz, C.c_int, C.c_double, C.c_double, _f32p,
                                            _f32p, _f32p]
        L.cpo_batch_layout.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p]

    # -- seeded workloads (the same fields as cpsz_b200.workloads, built without the product) --
    def field_2d(self, seed, r1, r2, n_flows, sigma, noise=0.01):
        U = np.empty((r1, r2), np.float32)
        V = np.empty((r1, r2), np.float32)
        if self.lib.cpo_generate_field_2d(seed, r1, r2, n_flows, sigma, noise, U, V):
            raise ValueError("oracle generator: bad arguments or out of memory")
        return U, V

    def field_3d(self, seed, r1, r2, r3, n_flows, sigma, noise=0.01):
        out = [np.empty((r1, r2, r3), np.float32) for _ in range(3)]
        if self.lib.cpo_generate_field_3d(seed, r1, r2, r3, n_flows, sigma, noise, *out):
            raise ValueError("oracle generator: bad arguments or out of memory")
        return tuple(out)

    def batch_layout(self, base_seed=3, n_fields=256, lo=128, hi=4096):
        r1 = np.empty(n_fields, np.uint64)
        r2 = np.empty(n_fields, np.uint64)
        seeds = np.empty(n_fields, np.uint64)
        ebs = np.empty(n_fields, np.float64)
        if self.lib.cpo_batch_layout(base_seed, n_fields, lo, hi, r1.ctypes.data, r2.ctypes.data,
                                     seeds.ctypes.data, ebs.ctypes.data):
            raise ValueError("oracle batch layout: bad arguments")
        return [(int(a), int(b), int(s), float(e)) for a, b, s, e in zip(r1, r2, seeds, ebs)]

    # -- 2D --
    def eb_2d(self, U, V, eb):
        r1, r2 = U.shape
        out = np.empty(r1 * r2, np.float64)
        self.lib.cpo_eb_2d(_c(U), _c(V), r1, r2, eb, out)
        return out.reshape(r1, r2)

    def quantize_eb_2d(self, U, V, ebv):
        n = U.size
        ids = np.empty(2 * n, np.int32)
        eu = np.empty(n, np.float64)
        ev = np.empty(n, np.float64)
        self.lib.cpo_quantize_eb_2d(_c(U).ravel(), _c(V).ravel(), np.ascontiguousarray(ebv, np.float64).ravel(), n, ids, eu, ev)
        return ids, eu, ev

    def lorenzo_2d(self, data, prec):
        r1, r2 = data.shape
        n = r1 * r2
        types = np.empty(n, np.int32)
        unpred = np.empty(n, np.float32)
        recon = np.empty(n, np.float32)
        k = self.lib.cpo_lorenzo_2d(_c(data).ravel(), np.ascontiguousarray(prec, np.float64).ravel(), r1, r2, types, unpred, recon)
        return types, unpred[:k].copy(), recon.reshape(r1, r2)

    def compress_2d(self, U, V, eb) -> bytes:
        r1, r2 = U.shape
        sz = _sz()
        p = self.lib.cpo_compress_2d_offline(_c(U), _c(V), r1, r2, eb, C.byref(sz))
        return _take_blob(self.lib, p, sz.value)

    def decompress_2d(self, blob: bytes, r1, r2):
        U = np.empty((r1, r2), np.float32)
        V = np.empty((r1, r2), np.float32)
        rc = self.lib.cpo_decompress_2d_offline(blob, len(blob), r1, r2, U, V)
        if rc:
            raise ValueError(f"oracle: malformed 2D blob (code {rc})")
        return U, V

    def compress_2d_log(self, U, V, eb) -> bytes:
        r1, r2 = U.shape
        sz = _sz()
        p = self.lib.cpo_compress_2d_offline_log(_c(U), _c(V), r1, r2, eb, C.byref(sz))
        return _take_blob(self.lib, p, sz.value)

    def decompress_2d_log(self, blob: bytes, r1, r2):
        U = np.empty((r1, r2), np.float32)
        V = np.empty((r1, r2), np.float32)
        rc = self.lib.cpo_decompress_2d_offline_log(blob, len(blob), r1, r2, U, V)
        if rc:
            raise ValueError(f"oracle: malformed 2D log blob (code {rc})")
        return U, V

    def huffman_encode(self, state_num, sym) -> bytes:
        sym = np.ascontiguousarray(sym, np.int32)
        cap = self.lib.cpo_huffman_encode_bound(state_num, sym.size)
        buf = C.create_string_buffer(cap)
        k = self.lib.cpo_huffman_encode(state_num, sym, sym.size, buf)
        return buf.raw[:k]

    def huffman_decode(self, state_num, n, data: bytes):
        out = np.empty(max(n, 1), np.int32)
        k = self.lib.cpo_huffman_decode(state_num, n, data, len(data), out)
        if not k:
            raise ValueError("oracle: malformed Huffman section")
        return out[:n], k

    def huffman_code_lengths(self, state_num, sym):
        sym = np.ascontiguousarray(sym, np.int32)
        lens = np.empty(2 * state_num, np.uint8)
        self.lib.cpo_huffman_code_lengths(state_num, sym, sym.size, lens)
        return lens

    # -- 3D --
    def eb_3d(self, U, V, W, eb):
        r1, r2, r3 = U.shape
        out = np.empty(U.size, np.float64)
        self.lib.cpo_eb_3d(_c(U), _c(V), _c(W), r1, r2, r3, eb, out)
        return out.reshape(U.shape)

    def compress_3d(self, U, V, W, eb) -> bytes:
        r1, r2, r3 = U.shape
        sz = _sz()
        p = self.lib.cpo_compress_3d_offline_log(_c(U), _c(V), _c(W), r1, r2, r3, eb, C.byref(sz))
        return _take_blob(self.lib, p, sz.value)

    def decompress_3d(self, blob: bytes, r1, r2, r3):
        out = [np.empty((r1, r2, r3), np.float32) for _ in range(3)]
        rc = self.lib.cpo_decompress_3d_online_log(blob, len(blob), r1, r2, r3, *out)
        if rc:
            raise ValueError(f"oracle: malformed 3D blob (code {rc})")
        return tuple(out)

    def host_libm(self, which: str, x):
        """The host C library's log2f ('log2f') or exp2f ('exp2f') of a float array."""
        x = np.ascontiguousarray(x, np.float32).ravel()
        out = np.empty_like(x)
        fn = self.lib.cpo_log2f_array if which == "log2f" else self.lib.cpo_exp2f_array
        fn(x, x.size, out)
        return out


class Reference:
    """Bindings of the reference's own implementation (oracle/_ref)."""

    def __init__(self, path: str | None = None):
        path = path or REF_SO
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        L.cpsz_ref_compress_2d_offline_f32.argtypes = [_f32p, _f32p, _sz, _sz, C.c_double, C.POINTER(_sz)]
        L.cpsz_ref_compress_2d_offline_f32.restype = C.c_void_p
        L.cpsz_ref_decompress_2d_offline_f32.argtypes = [C.c_char_p, _sz, _sz, _f32p, _f32p]
        L.cpsz_ref_compress_2d_offline_log_f32.argtypes = [_f32p, _f32p, _sz, _sz, C.c_double, C.POINTER(_sz)]
        L.cpsz_ref_compress_2d_offline_log_f32.restype = C.c_void_p
        L.cpsz_ref_decompress_2d_offline_log_f32.argtypes = [C.c_char_p, _sz, _sz, _f32p, _f32p]
        L.cpsz_ref_compress_3d_offline_log_f32.argtypes = [_f32p, _f32p, _f32p, _sz, _sz, _sz, C.c_double, C.POINTER(_sz)]
        L.cpsz_ref_compress_3d_offline_log_f32.restype = C.c_void_p
        L.cpsz_ref_decompress_3d_online_log_f32.argtypes = [C.c_char_p, _sz, _sz, _sz, _f32p, _f32p, _f32p]
        L.cpsz_ref_zstd_compress.argtypes = [C.c_char_p, _sz, C.POINTER(C.c_void_p)]
        L.cpsz_ref_zstd_compress.restype = _sz
        L.cpsz_ref_zstd_decompress.argtypes = [C.c_char_p, _sz, C.POINTER(C.c_void_p), _sz]
        L.cpsz_ref_zstd_decompress.restype = _sz
        L.cpsz_ref_free.argtypes = [C.c_void_p]

    def compress_2d(self, U, V, eb) -> bytes:
        r1, r2 = U.shape
        sz = _sz()
        p = self.lib.cpsz_ref_compress_2d_offline_f32(_c(U), _c(V), r1, r2, eb, C.byref(sz))
        return _take_blob(self.lib, p, sz.value)

    def decompress_2d(self, blob: bytes, r1, r2):
        U = np.empty((r1, r2), np.float32)
        V = np.empty((r1, r2), np.float32)
        self.lib.cpsz_ref_decompress_2d_offline_f32(blob, r1, r2, U, V)
        return U, V

    def compress_2d_log(self, U, V, eb) -> bytes:
        r1, r2 = U.shape
        sz = _sz()
        p = self.lib.cpsz_ref_compress_2d_offline_log_f32(_c(U), _c(V), r1, r2, eb, C.byref(sz))
        return _take_blob(self.lib, p, sz.value)

    def decompress_2d_log(self, blob: bytes, r1, r2):
        U = np.empty((r1, r2), np.float32)
        V = np.empty((r1, r2), np.float32)
        self.lib.cpsz_ref_decompress_2d_offline_log_f32(blob, r1, r2, U, V)
        return U, V

    def compress_3d(self, U, V, W, eb) -> bytes:
        r1, r2, r3 = U.shape
        sz = _sz()
        p = self.lib.cpsz_ref_compress_3d_offline_log_f32(_c(U), _c(V), _c(W), r1, r2, r3, eb, C.byref(sz))
        return _take_blob(self.lib, p, sz.value)

    def decompress_3d(self, blob: bytes, r1, r2, r3):
        out = [np.empty((r1, r2, r3), np.float32) for _ in range(3)]
        self.lib.cpsz_ref_decompress_3d_online_log_f32(blob, r1, r2, r3, *out)
        return tuple(out)

    def zstd_compress(self, data: bytes) -> bytes:
        p = C.c_void_p()
        n = self.lib.cpsz_ref_zstd_compress(data, len(data), C.byref(p))
        out = C.string_at(p, n)
        self.lib.cpsz_ref_free(p)
        return out

    def zstd_decompress(self, data: bytes, target: int) -> bytes:
        p = C.c_void_p()
        n = self.lib.cpsz_ref_zstd_decompress(data, len(data), C.byref(p), target)
        out = C.string_at(p, n)
        self.lib.cpsz_ref_free(p)
        return out


def _c(a):
    return np.ascontiguousarray(a, np.float32)


def ref_2d_in_bounds(oracle_blob: bytes, r1: int, r2: int) -> bool:
    """True if the reference's fixed-size scratch buffers hold this workload.

    The reference sizes its per-field output as (size_t)(N*sizeof(float)*1.2)
    (src/sz_compress_3d.cpp:214-216) and its id output as 2N*sizeof(int)
    (src/sz_compress_cp_preserve_2d.cpp:246), and its Huffman packer writes up
    to 8 bytes past the stream (src/sz_huffman.cpp:236-246).  Small, rough
    fields with many distinct codes exceed that and corrupt the reference's
    heap, so parity against the compiled reference is only run where the
    restated oracle's section sizes (identical by construction) fit."""
    import struct
    n = r1 * r2
    eb_size, u_size, v_size = struct.unpack_from("<QQQ", oracle_blob, 12)
    est = int(n * 4 * 1.2)
    return u_size + 16 <= est and v_size + 16 <= est and eb_size + 16 <= 2 * n * 4


def ref_2d_log_in_bounds(oracle_blob: bytes, r1: int, r2: int) -> bool:
    """The offline_log form: the id section goes into N*sizeof(int) bytes
    (src/sz_compress_cp_preserve_2d.cpp:352) and each field blob into
    (size_t)(N*sizeof(float)*1.2) bytes, each plus the packer's write-ahead."""
    import struct
    n = r1 * r2
    eb_size, u_size, v_size = struct.unpack_from("<QQQ", oracle_blob, 12)
    est = int(n * 4 * 1.2)
    return u_size + 16 <= est and v_size + 16 <= est and eb_size + 16 <= n * 4


def ref_3d_in_bounds(oracle_blob: bytes, r1: int, r2: int, r3: int) -> bool:
    """The reference writes the whole 3D blob into 3*N*sizeof(float) bytes
    (src/sz_compress_cp_preserve_3d.cpp:555) plus the packer's 8-byte write-ahead."""
    return len(oracle_blob) + 16 <= 3 * r1 * r2 * r3 * 4
