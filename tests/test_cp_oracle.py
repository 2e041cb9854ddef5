"""The exact-rational CP oracle on fields with known critical points (CPU)."""
import numpy as np
import pytest

from oracle import cp_exact

# (J, expected code = 1 + type) for a linear 2D field u,v = J (x - x0, y - y0)
CASES_2D = [
    ([[1, 0], [0, 1]], 3),         # REPELLING
    ([[-1, 0], [0, -1]], 2),       # ATTRACTING
    ([[1, 0], [0, -1]], 4),        # SADDLE
    ([[0, -1], [1, 0]], 7),        # CENTER
    ([[0.5, -1], [1, 0.5]], 6),    # REPELLING_FOCUS
    ([[-0.5, -1], [1, -0.5]], 5),  # ATTRACTING_FOCUS
    ([[2, 1], [0, 1]], 3),         # REPELLING, distinct eigenvalues
]


def linear_2d(J, x0, y0, r1=9, r2=11):
    y, x = np.mgrid[0:r1, 0:r2].astype(np.float64)
    dx, dy = x - x0, y - y0
    U = (J[0][0] * dx + J[0][1] * dy).astype(np.float32)
    V = (J[1][0] * dx + J[1][1] * dy).astype(np.float32)
    return U, V


@pytest.mark.parametrize("J,code", CASES_2D)
def test_2d_single_cp_and_type(J, code):
    U, V = linear_2d(J, 3.25, 4.625)
    cells = cp_exact.cells_2d(U, V)
    nz = np.flatnonzero(cells)
    assert nz.size == 1 and cells[nz[0]] == code
    # the CP sits in cube (4, 3): x in [3,4), y in [4,5)
    assert nz[0] // 2 == 4 * (11 - 1) + 3


def test_2d_zero_on_edge_counted_once():
    for x0, y0 in ((3.5, 4.0), (3.0, 4.5), (3.5, 4.5)):
        U, V = linear_2d([[1, 0.25], [0.5, 1]], x0, y0)
        assert (cp_exact.cells_2d(U, V) != 0).sum() == 1, (x0, y0)


def test_2d_zero_vertex_rule():
    U, V = linear_2d([[1, 0], [0, 1]], 3.0, 4.0)
    assert (cp_exact.cells_2d(U, V) != 0).sum() == 0


CASES_3D = [
    (np.diag([1.0, 2.0, 3.0]), 2),        # 3 positive real roots: STABLE_SOURCE
    (np.diag([-1.0, -2.0, -3.0]), 8),     # 3 negative: STABLE_SINK
    (np.diag([1.0, -2.0, 3.0]), 4),       # 1 negative: STABLE_REPELLING_SADDLE
    (np.diag([-1.0, -2.0, 3.0]), 6),      # 2 negative: STABLE_ATTRACTING_SADDLE
    (np.array([[0.5, -1, 0], [1, 0.5, 0], [0, 0, -1.0]]), 5),  # 0.5 +- i, -1: UNSTABLE_REPELLING_SADDLE
    (np.array([[-0.5, -1, 0], [1, -0.5, 0], [0, 0, 2.0]]), 7),  # -0.5 +- i, 2: UNSTABLE_ATTRACTING_SADDLE
    (np.eye(3), 1),                       # triple root: SINGULAR
]


def linear_3d(J, c, n=6):
    z, y, x = np.mgrid[0:n, 0:n, 0:n].astype(np.float64)
    d = [x - c[0], y - c[1], z - c[2]]
    return tuple((J[r][0] * d[0] + J[r][1] * d[1] + J[r][2] * d[2]).astype(np.float32) for r in range(3))


@pytest.mark.parametrize("J,code", CASES_3D)
def test_3d_single_cp_and_type(J, code):
    U, V, W = linear_3d(J, (2.25, 2.625, 1.375))
    cells = cp_exact.cells_3d(U, V, W)
    nz = np.flatnonzero(cells)
    assert nz.size == 1 and cells[nz[0]] == code


def test_3d_zero_on_face_counted_once():
    for c in ((2.5, 2.5, 2.0), (2.0, 2.5, 1.5), (2.5, 2.0, 2.0)):
        U, V, W = linear_3d(np.array([[1, 0.25, 0], [0, 2, 0.5], [0.25, 0, 3.0]]), c)
        assert (cp_exact.cells_3d(U, V, W) != 0).sum() == 1, c
