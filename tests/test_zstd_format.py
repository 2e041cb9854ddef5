"""The Zstandard frame writer shared by the GPU lossless stage
(cpsz_b200/csrc/zstd_format.h) on the CPU: tests/zstd_format_check.cpp drives
it with a plain greedy matcher and decodes every frame with the system
libzstd (empty input, one byte, RLE blocks, incompressible data, long and
short matches over every length and offset code range, 16 KB and 128 KB
blocks)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ZSTD_SO = next((p for p in ("/usr/lib/x86_64-linux-gnu/libzstd.so.1", "/usr/lib64/libzstd.so.1",
                            "/lib/x86_64-linux-gnu/libzstd.so.1") if os.path.exists(p)), None)


@pytest.mark.skipif(shutil.which("g++") is None or ZSTD_SO is None, reason="needs g++ and libzstd")
def test_frames_decode_with_libzstd(tmp_path):
    exe = str(tmp_path / "zfc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "cpsz_b200", "csrc"), "-o", exe,
                    os.path.join(ROOT, "tests", "zstd_format_check.cpp"), ZSTD_SO], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ALL OK" in r.stdout, r.stdout + r.stderr
