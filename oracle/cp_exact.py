"""Exact-rational restatement of the critical-point checker (test
infrastructure only).

Pure Python with fractions.Fraction: every float is converted exactly, so
each sign below is the sign of the exact value.  It states the checker's
definitions once more, independently of the GPU code, for small fields:

* a cell (triangle / tetrahedron) holds a critical point (CP) when the origin
  lies strictly inside the convex hull of the cell's vertex values, with ties
  broken by moving the origin to (e, e^2[, e^3]) for an infinitesimal e
  (Simulation of Simplicity, Edelsbrunner & Muecke 1990);
* a cell with a vertex whose value is exactly zero, or a non-finite value,
  holds no CP (the zero rule of the reference's tools,
  test/cp_extraction_2d.cpp:63-68, test/cp_extraction_3d.cpp:124-126);
* CP types from the Jacobian of the linear interpolant
  (test/cp_extraction_2d.cpp:32-38, test/cp_extraction_3d.cpp:30-38), with
  degenerate cases (zero determinant, a complex pair on the imaginary axis,
  repeated roots) classified SINGULAR.

Cells and codes are numbered as the library's checker numbers them: code 0 =
no CP, else 1 + type.
"""
from __future__ import annotations

import math
from fractions import Fraction as F

import numpy as np

# 3D tets: corners as (dk, dj, di), corner 0 = (0,0,0), corner 3 = (1,1,1)
# (test/cp_extraction_3d.cpp:39-77)
TETS = [
    [(0, 0, 0), (0, 0, 1), (0, 1, 1), (1, 1, 1)],
    [(0, 0, 0), (0, 1, 0), (0, 1, 1), (1, 1, 1)],
    [(0, 0, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1)],
    [(0, 0, 0), (1, 0, 0), (1, 0, 1), (1, 1, 1)],
    [(0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 1, 1)],
    [(0, 0, 0), (1, 0, 0), (1, 1, 0), (1, 1, 1)],
]


def _sgn(x) -> int:
    return (x > 0) - (x < 0)


def _bad(vals) -> bool:
    return any(not math.isfinite(x) for x in vals)


# ---- 2D --------------------------------------------------------------------------------

def _orient2(pa, pb) -> int:
    ua, va = pa
    ub, vb = pb
    s = _sgn(ua * vb - ub * va)
    if s:
        return s
    s = _sgn(va - vb)
    if s:
        return s
    return _sgn(ub - ua)


def _tri_type(P, kind) -> int:
    if kind == 0:  # unit coordinates {(0,0),(0,1),(1,1)}
        a, b = P[2][0] - P[1][0], P[1][0] - P[0][0]
        c, d = P[2][1] - P[1][1], P[1][1] - P[0][1]
    else:  # {(0,0),(1,0),(1,1)}
        a, b = P[1][0] - P[0][0], P[2][0] - P[1][0]
        c, d = P[1][1] - P[0][1], P[2][1] - P[1][1]
    tr = _sgn(a + d)
    det = _sgn(a * d - b * c)
    delta = _sgn((a - d) ** 2 + 4 * b * c)
    if det == 0:
        t = 0
    elif delta >= 0:
        t = 3 if det < 0 else (1 if tr < 0 else 2)
    else:
        t = 4 if tr < 0 else (5 if tr > 0 else 6)
    return t + 1


def tri_code(vals, kind) -> int:
    """vals: three (u, v) float pairs in the reference's vertex order."""
    flat = [x for p in vals for x in p]
    if _bad(flat) or any(u == 0 and v == 0 for u, v in vals):
        return 0
    P = [(F(u), F(v)) for u, v in vals]
    s0 = _orient2(P[1], P[2])
    s1 = _orient2(P[2], P[0])
    s2 = _orient2(P[0], P[1])
    if s0 == 0 or s0 != s1 or s0 != s2:
        return 0
    return _tri_type(P, kind)


def cells_2d(U, V) -> np.ndarray:
    U = np.asarray(U, np.float32)
    V = np.asarray(V, np.float32)
    r1, r2 = U.shape
    out = np.zeros(max(2 * (r1 - 1) * (r2 - 1), 0), np.uint8)
    for i in range(r1 - 1):
        for j in range(r2 - 1):
            q = i * (r2 - 1) + j
            p00 = (float(U[i, j]), float(V[i, j]))
            p10 = (float(U[i + 1, j]), float(V[i + 1, j]))
            p11 = (float(U[i + 1, j + 1]), float(V[i + 1, j + 1]))
            p01 = (float(U[i, j + 1]), float(V[i, j + 1]))
            out[2 * q] = tri_code([p00, p10, p11], 0)
            out[2 * q + 1] = tri_code([p00, p01, p11], 1)
    return out


# ---- 3D --------------------------------------------------------------------------------

def _det3(a, b, c):
    return (a[0] * (b[1] * c[2] - b[2] * c[1]) - b[0] * (a[1] * c[2] - a[2] * c[1])
            + c[0] * (a[1] * b[2] - a[2] * b[1]))


def _cross(p, q):
    return (p[1] * q[2] - p[2] * q[1], p[2] * q[0] - p[0] * q[2], p[0] * q[1] - p[1] * q[0])


def _orient3(a, b, c) -> int:
    s = _sgn(_det3(a, b, c))
    if s:
        return s
    n = [x + y + z for x, y, z in zip(_cross(b, c), _cross(c, a), _cross(a, b))]
    for comp in n:
        if comp:
            return -_sgn(comp)
    return 0


def _xinv(t):
    X = TETS[t]
    M = [[F(X[c][r] - X[3][r]) for c in range(3)] for r in range(3)]
    # inverse of an integer 3x3 matrix with determinant +-1
    det = _det3([M[0][0], M[1][0], M[2][0]], [M[0][1], M[1][1], M[2][1]], [M[0][2], M[1][2], M[2][2]])
    cof = [[(M[(r + 1) % 3][(c + 1) % 3] * M[(r + 2) % 3][(c + 2) % 3]
             - M[(r + 1) % 3][(c + 2) % 3] * M[(r + 2) % 3][(c + 1) % 3]) for c in range(3)] for r in range(3)]
    return [[cof[c][r] / det for c in range(3)] for r in range(3)]


_XINV = [_xinv(t) for t in range(6)]


def _tet_type(P, t) -> int:
    Xi = _XINV[t]
    Ud = [[P[c][k] - P[3][k] for c in range(3)] for k in range(3)]
    J = [[sum(Xi[r][k] * Ud[k][c] for k in range(3)) for c in range(3)] for r in range(3)]
    tr = J[0][0] + J[1][1] + J[2][2]
    c2 = (J[0][0] * J[1][1] - J[0][1] * J[1][0] + J[0][0] * J[2][2] - J[0][2] * J[2][0]
          + J[1][1] * J[2][2] - J[1][2] * J[2][1])
    det = _det3([J[0][0], J[1][0], J[2][0]], [J[0][1], J[1][1], J[2][1]], [J[0][2], J[1][2], J[2][2]])
    a2, a1, a0 = -tr, c2, -det
    h = a2 * a1 - a0
    disc = 18 * a2 * a1 * a0 - 4 * a2 ** 3 * a0 + a2 ** 2 * a1 ** 2 - 4 * a1 ** 3 - 27 * a0 ** 2
    return _cubic_type(_sgn(a2), _sgn(a1), _sgn(a0), _sgn(h), _sgn(disc))


def _cubic_type(s_a2, s_a1, s_a0, s_h, s_d) -> int:
    """1 + type of l^3 + a2 l^2 + a1 l + a0 from exact signs.  Complex pair
    (d < 0) with real root r and real part al: r < 0 iff a0 > 0 (product of
    the roots), al < 0 iff h = a2 a1 - a0 > 0 (h = -2 al ((r + al)^2 + b^2)).
    Three distinct real roots (d > 0): Descartes' rule of signs is exact."""
    if s_a0 == 0 or s_d == 0:
        return 0 + 1
    if s_d < 0:
        if s_h == 0:
            return 0 + 1
        neg = (s_a0 > 0) + 2 * (s_h > 0)
        return 1 + 2 * neg + 1 + 1
    seq = [x for x in (1, s_a2, s_a1, s_a0) if x != 0]
    changes = sum(seq[q] != seq[q + 1] for q in range(len(seq) - 1))
    return 1 + 2 * (3 - changes) + 1


def tet_code(vals, t) -> int:
    """vals: four (u, v, w) float triples in the tet's corner order."""
    flat = [x for p in vals for x in p]
    if _bad(flat) or any(p[0] == 0 and p[1] == 0 and p[2] == 0 for p in vals):
        return 0
    P = [tuple(F(x) for x in p) for p in vals]
    s0 = _orient3(P[1], P[2], P[3])
    if s0 == 0:
        return 0
    if -_orient3(P[0], P[2], P[3]) != s0 or _orient3(P[0], P[1], P[3]) != s0 or -_orient3(P[0], P[1], P[2]) != s0:
        return 0
    return _tet_type(P, t)


def cells_3d(U, V, W) -> np.ndarray:
    U, V, W = (np.asarray(a, np.float32) for a in (U, V, W))
    r1, r2, r3 = U.shape
    out = np.zeros(max(6 * (r1 - 1) * (r2 - 1) * (r3 - 1), 0), np.uint8)
    q = 0
    for i in range(r1 - 1):
        for j in range(r2 - 1):
            for k in range(r3 - 1):
                for t in range(6):
                    vals = []
                    for dk, dj, di in TETS[t]:
                        ii, jj, kk = i + di, j + dj, k + dk
                        vals.append((float(U[ii, jj, kk]), float(V[ii, jj, kk]), float(W[ii, jj, kk])))
                    out[6 * q + t] = tet_code(vals, t)
                q += 1
    return out


def compare(a: np.ndarray, b: np.ndarray):
    """{cps_a, cps_b, lost_or_spurious, type_changed} of two cell-code arrays."""
    a = np.asarray(a)
    b = np.asarray(b)
    return {"cps_a": int((a != 0).sum()), "cps_b": int((b != 0).sum()),
            "lost_or_spurious": int(((a != 0) != (b != 0)).sum()),
            "type_changed": int(((a != 0) & (b != 0) & (a != b)).sum())}
