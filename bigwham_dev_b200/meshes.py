"""Synthetic crack meshes used by the tests and the benchmark.

All meshes are generated from their definition (no data files):

* ``straight_crack_2d``: n equal segments on x in [a, b], y = 0, kernel 2DS0-H.
* ``square_crack_3d``: nx x ny rectangles on [-L, L]^2 in z = 0, kernel 3DR0-H.
  Vertex order per element (0: bottom-left, 1: bottom-right, 2: top-right,
  3: top-left) is the one of the reference's 3DR0 example
  (interfaces/python/examples/example_3DR0_kernel.py:108-131).
* ``penny_crack_3d``: points of a hexagonal lattice of spacing h clipped to the
  unit disk, jittered by U(-0.1h, 0.1h), Delaunay-triangulated; kernel 3DT0-H.
"""
from __future__ import annotations

import numpy as np


def straight_crack_2d(n: int, a: float = -1.0, b: float = 1.0):
    x = np.linspace(a, b, n + 1)
    coor = np.stack([x, np.zeros_like(x)], axis=1)
    conn = np.stack([np.arange(n), np.arange(1, n + 1)], axis=1).astype(np.int32)
    return coor, conn


def square_crack_3d(nx: int, ny: int | None = None, half: float = 1.0):
    ny = nx if ny is None else ny
    xs = np.linspace(-half, half, nx + 1)
    ys = np.linspace(-half, half, ny + 1)
    X, Y = np.meshgrid(xs, ys)  # node index i + j*(nx+1)
    coor = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1)
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    i, j = i.ravel(), j.ravel()
    conn = np.stack([i + j * (nx + 1), i + 1 + j * (nx + 1), i + 1 + (j + 1) * (nx + 1), i + (j + 1) * (nx + 1)],
                    axis=1).astype(np.int32)
    return coor, conn


def penny_crack_3d(h: float, seed: int = 2, radius: float = 1.0):
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    ny = int(np.ceil(radius / (h * np.sqrt(3) / 2))) + 1
    nx = int(np.ceil(radius / h)) + 1
    pts = []
    for j in range(-ny, ny + 1):
        y = j * h * np.sqrt(3) / 2
        off = 0.5 * h if (j % 2) else 0.0
        xs = np.arange(-nx, nx + 1) * h + off
        pts.append(np.stack([xs, np.full_like(xs, y)], axis=1))
    P = np.concatenate(pts)
    P = P[np.hypot(P[:, 0], P[:, 1]) <= radius]
    P = P + rng.uniform(-0.1 * h, 0.1 * h, size=P.shape)
    tri = Delaunay(P)
    conn = tri.simplices.astype(np.int32)
    # orient counter-clockwise (normal +z)
    a, b, c = P[conn[:, 0]], P[conn[:, 1]], P[conn[:, 2]]
    cross = (b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0])
    flip = cross < 0
    conn[flip, 1], conn[flip, 2] = conn[flip, 2].copy(), conn[flip, 1].copy()
    # drop slivers of zero area (collinear boundary points)
    keep = np.abs(cross) > 1e-12 * h * h
    conn = conn[keep]
    coor = np.concatenate([P, np.zeros((P.shape[0], 1))], axis=1)
    return coor, conn
