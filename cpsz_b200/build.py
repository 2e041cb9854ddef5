"""Build libcpsz_b200.so in-tree (cpsz_b200/_lib/) with nvcc for sm_100a.

Every CUDA source is compiled with ``-gencode arch=compute_100a,code=sm_100a``.
The kernels that must reproduce the reference's CPU arithmetic bit for bit
(error-bound derivation, quantization, Lorenzo, checker) are compiled with
``-fmad=false`` so no multiply-add is contracted; files listed in
``FMA_OK`` (tensor-core MLP) keep contraction.  Host C++ is compiled by nvcc's
host compiler.  The shared library links the CUDA runtime statically and the
system ``libzstd.so.1`` for the host lossless stage.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libcpsz_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FMA_OK = {"mlp.cu"}


def _nvcc() -> str:
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _zstd_so() -> str | None:
    for c in ("/usr/lib/x86_64-linux-gnu/libzstd.so.1", "/usr/lib64/libzstd.so.1", "/lib/x86_64-linux-gnu/libzstd.so.1"):
        if os.path.exists(c):
            return c
    return None


def _compile(src: str, extra: list[str]) -> str:
    nvcc = _nvcc()
    base = os.path.basename(src)
    obj = os.path.join(OBJ, base + ".o")
    deps = [src] + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + [
        os.path.join(ROOT, "include", "cpsz_b200.h")]
    if os.path.exists(obj) and all(os.path.getmtime(d) <= os.path.getmtime(obj) for d in deps if os.path.exists(d)):
        return obj
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    if src.endswith(".cu"):
        cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
               "-Xptxas", "-warn-spills", *inc, *extra, "-c", src, "-o", obj]
        if base not in FMA_OK:
            cmd.insert(1, "-fmad=false")
    else:
        cmd = [nvcc, "-O2", "-std=c++17", "-Wno-deprecated-gpu-targets", "-Xcompiler", "-fPIC,-Wall,-Wno-unused-function", *inc, *extra, "-c", src,
               "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra or []), srcs))
    if os.path.exists(LIB) and all(os.path.getmtime(o) <= os.path.getmtime(LIB) for o in objs):
        return LIB
    link = [_nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lpthread", "-ldl"]
    z = _zstd_so()
    if z:
        link += ["-Xlinker", z]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(link)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print("built", LIB)
    return LIB


def prepare_tables(verbose: bool = False) -> str:
    """Generates the host log2f / exp2f tables beside the library (skipped when
    a cache for this C library version exists); runs in a child process so the
    build process does not keep the library loaded."""
    code = ("import ctypes,sys; L=ctypes.CDLL(sys.argv[1]); L.cpsz_b200_libm_tables_prepare.argtypes=[ctypes.c_char_p];"
            "sys.exit(L.cpsz_b200_libm_tables_prepare(None))")
    r = subprocess.run([sys.executable, "-c", code, LIB], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"libm table generation failed ({r.returncode}): {r.stderr}")
    path = os.path.join(LIBDIR, "libm_f32_tables.bin")
    if verbose:
        print("tables", path)
    return path


if __name__ == "__main__":
    build(verbose=True)
    prepare_tables(verbose=True)
