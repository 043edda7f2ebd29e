"""Generate the golden fixtures of the H-matrix matvec from the reference itself.

Run in a tree where the reference library has been compiled by
``make -C oracle ref`` (it needs the reference sources only at compile time):

    python tests/golden/make_golden.py           # square cases (tests/golden/*.npz)
    python tests/golden/make_golden.py --rect    # rectangular cases (tests/golden/rect/)

For every case the reference's own code (BigWhamIO + BuildHierarchicalMatrix,
src/io/bigwham_io.cc:635-704) builds the H-matrix; the fixture stores the flat
blocks, pattern and permutations, a seeded input x, and the reference's own
outputs:

* ``y_ref``       BigWhamIO::MatVec(x), original ordering (bigwham_io.cc:927-933)
* ``y_perm_ref``  BigWhamIO::MatVecPerm(x), permuted ordering (bigwham_io.cc:965-980)
* ``diag_ref``    BigWhamIO::GetDiagonal (bigwham_io.cc:909-916)
* ``y_dense``     MatVec of the same kernel built with eta = 0: every block is
                  full rank (cluster.h:148-159), i.e. the dense FP64 product
* ``yt_dense``    the dense transpose product D^T x, with D assembled from the
                  eta = 0 blocks
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from bigwham_dev_b200.meshes import penny_crack_3d, square_crack_3d, straight_crack_2d  # noqa: E402
from oracle import RefHmat  # noqa: E402

CASES = {
    # name: (kernel, mesh fn, properties, leaf, eta, eps, seed)
    "2ds0_n256": ("2DS0-H", lambda: straight_crack_2d(256), [1.0, 0.25], 16, 3.0, 1e-5, 0),
    "3dr0_10x10": ("3DR0-H", lambda: square_crack_3d(10), [1.0, 0.25], 8, 3.0, 1e-4, 1),
    "3dt0_penny": ("3DT0-H", lambda: penny_crack_3d(0.3, seed=2), [1.0, 0.2], 8, 3.0, 1e-3, 2),
}


# rectangular cases (source mesh x receiver mesh), stored under rect/ so the
# square-only fixture set (every *.npz here) is unchanged
RECT_CASES = {
    # name: (kernel, source mesh fn, receiver mesh fn, properties, leaf, eta, eps, seed)
    "3dr0_rect": ("3DR0-3DR0-H", lambda: square_crack_3d(10),
                  lambda: (square_crack_3d(7, 9, half=1.3)[0] + np.array([0.05, -0.1, 0.4]),
                           square_crack_3d(7, 9, half=1.3)[1]),
                  [1.0, 0.25], 16, 3.0, 1e-6, 6),
}


def dense_from(arr):
    D = np.zeros((arr.n_rows, arr.n_cols))
    for i0, j0, a in arr.fr_blocks():
        D[i0:i0 + a.shape[0], j0:j0 + a.shape[1]] = a
    for i0, j0, A, B in arr.lr_blocks():
        D[i0:i0 + A.shape[0], j0:j0 + B.shape[1]] = A @ B
    # to original ordering
    dof = arr.dof
    rp = (dof * arr.perm0[:, None] + np.arange(dof)[None, :]).ravel()
    cp = (dof * arr.perm1[:, None] + np.arange(dof)[None, :]).ravel()
    Do = np.zeros_like(D)
    Do[np.ix_(rp, cp)] = D
    return Do


def main():
    for name, (kernel, mesh, props, leaf, eta, eps, seed) in CASES.items():
        coor, conn = mesh()
        R = RefHmat(kernel, coor, conn, props, leaf, eta, eps, n_threads=4)
        arr = R.arrays()
        x = np.random.default_rng(seed).uniform(-1.0, 1.0, R.shape[1])
        Rd = RefHmat(kernel, coor, conn, props, leaf, 0.0, eps, n_threads=4)
        D = dense_from(Rd.arrays())
        y_dense = Rd.matvec(x)
        out = os.path.join(HERE, f"{name}.npz")
        arr.save(out, kernel=kernel, coor=coor, conn=conn, properties=np.asarray(props), leaf=leaf, eta=eta,
                 eps=eps, seed=seed, x=x, y_ref=R.matvec(x), y_perm_ref=R.matvec_perm(x), diag_ref=R.diagonal(),
                 y_dense=y_dense, yt_dense=D.T @ x, y_dense_assembled=D @ x)
        print(f"{name}: N={R.shape[0]} n_fr={arr.fr.shape[0]} n_lr={arr.lr.shape[0]} "
              f"entries={arr.fr_data.size + arr.lr_data.size} size={os.path.getsize(out) / 1e3:.0f} kB")


def main_rect():
    os.makedirs(os.path.join(HERE, "rect"), exist_ok=True)
    for name, (kernel, src, rec, props, leaf, eta, eps, seed) in RECT_CASES.items():
        (cs, es), (cr, er) = src(), rec()
        R = RefHmat.rectangular(kernel, cs, es, cr, er, props, leaf, eta, eps, n_threads=4)
        arr = R.arrays()
        x = np.random.default_rng(seed).uniform(-1.0, 1.0, R.shape[1])
        Rd = RefHmat.rectangular(kernel, cs, es, cr, er, props, leaf, 0.0, eps, n_threads=4)
        D = dense_from(Rd.arrays())
        out = os.path.join(HERE, "rect", f"{name}.npz")
        arr.save(out, kernel=kernel, properties=np.asarray(props), leaf=leaf, eta=eta, eps=eps, seed=seed, x=x,
                 y_ref=R.matvec(x), y_perm_ref=R.matvec_perm(x), y_dense=Rd.matvec(x), y_dense_assembled=D @ x)
        print(f"{name}: {R.shape[0]} x {R.shape[1]} n_fr={arr.fr.shape[0]} n_lr={arr.lr.shape[0]} "
              f"size={os.path.getsize(out) / 1e3:.0f} kB")


if __name__ == "__main__":
    if "--rect" in sys.argv:
        main_rect()
    else:
        main()
