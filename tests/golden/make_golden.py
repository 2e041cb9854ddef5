"""Generates tests/golden/*.npz from the reference's own implementation.

Run where the reference sources are present (they are compiled into
oracle/_ref by `make -C oracle ref`), naming their directory:

    CPSZ_REF_DIR=<reference source tree> python tests/golden/make_golden.py

Each fixture holds the input field(s), the reference's compressed blob and the
reference's decompressed field(s).  Inputs come from the seeded generators in
cpsz_b200.workloads; the arrays themselves are stored, so the fixtures do not
depend on the generator staying unchanged.  Only workloads that fit the
reference's fixed scratch buffers are used (see oracle.ref_2d_in_bounds).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cpsz_b200 import workloads as W  # noqa: E402
from oracle import (Oracle, Reference, build_reference, ref_2d_in_bounds, ref_2d_log_in_bounds,  # noqa: E402
                    ref_3d_in_bounds)

CASES_2D = [  # (name, r1, r2, eb, seed)
    ("2d_33x47_eb0.1", 33, 47, 0.1, 11),
    ("2d_64x64_eb0.01", 64, 64, 0.01, 12),
    ("2d_1x50_eb0.1", 1, 50, 0.1, 13),
    ("2d_13x17_eb0.05", 13, 17, 0.05, 14),
    ("2d_100x120_eb0.1", 100, 120, 0.1, 15),
    ("2d_37x300_eb0.05", 37, 300, 0.05, 16),
]
CASES_2D_LOG = [  # (name, r1, r2, eb, seed, zeros): the offline_log pair; `zeros` plants exact zeros
    ("2dlog_33x47_eb0.1", 33, 47, 0.1, 31, False),
    ("2dlog_64x64_eb0.01", 64, 64, 0.01, 32, False),
    ("2dlog_100x120_eb0.05", 100, 120, 0.05, 33, False),
    ("2dlog_40x50_zeros_eb0.1", 40, 50, 0.1, 34, True),
]
CASES_3D = [  # (name, r1, r2, r3, eb, seed)
    ("3d_16x16x16_eb0.05", 16, 16, 16, 0.05, 21),
    ("3d_33x20x17_eb0.1", 33, 20, 17, 0.1, 22),
    ("3d_24x30x28_eb0.01", 24, 30, 28, 0.01, 23),
]


def log_case(seed, r1, r2, zeros):
    """A cfg0-like field; with `zeros`, every 7th point of U and every 5th of V
    set to exactly 0 (logs of -100 and sign bits 0 in the offline_log blob)."""
    U, V = W.cfg0_like(seed, r1, r2)
    if zeros:
        U.ravel()[::7] = 0
        V.ravel()[::5] = 0
    return U, V


def main():
    if not build_reference():
        raise SystemExit("reference sources not available")
    R = Reference()
    O = Oracle()
    for name, r1, r2, eb, seed in CASES_2D:
        U, V = W.cfg0_like(seed, r1, r2)
        if not ref_2d_in_bounds(O.compress_2d(U, V, eb), r1, r2):
            print("skip (reference scratch too small):", name)
            continue
        blob = R.compress_2d(U, V, eb)
        du, dv = R.decompress_2d(blob, r1, r2)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), U=U, V=V, eb=eb,
                            blob=np.frombuffer(blob, np.uint8), dU=du, dV=dv)
        print("wrote", name, len(blob))
    for name, r1, r2, eb, seed, zeros in CASES_2D_LOG:
        U, V = log_case(seed, r1, r2, zeros)
        if not ref_2d_log_in_bounds(O.compress_2d_log(U, V, eb), r1, r2):
            print("skip (reference scratch too small):", name)
            continue
        blob = R.compress_2d_log(U, V, eb)
        du, dv = R.decompress_2d_log(blob, r1, r2)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), U=U, V=V, eb=eb,
                            blob=np.frombuffer(blob, np.uint8), dU=du, dV=dv)
        print("wrote", name, len(blob))
    for name, r1, r2, r3, eb, seed in CASES_3D:
        U, V, Wf = W.field_3d(seed, r1, r2, r3, max(1, (r1 * r2 * r3) // 4000), 6.0)
        if not ref_3d_in_bounds(O.compress_3d(U, V, Wf, eb), r1, r2, r3):
            print("skip (reference scratch too small):", name)
            continue
        blob = R.compress_3d(U, V, Wf, eb)
        du, dv, dw = R.decompress_3d(blob, r1, r2, r3)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), U=U, V=V, W=Wf, eb=eb,
                            blob=np.frombuffer(blob, np.uint8), dU=du, dV=dv, dW=dw)
        print("wrote", name, len(blob))


if __name__ == "__main__":
    main()
