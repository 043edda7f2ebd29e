"""GMRES and mixed-precision refinement on the GPU (-m gpu).

Targets: Jacobi-preconditioned GMRES(50) on the FP64 H-matrix to
a relative residual of 1e-8; refinement with FP32 / BF16 inner solves reaches
the same residual with <= 1e-6 relative error against the FP64 solution; the
solution of the small golden systems matches a dense FP64 solve of the same
H-matrix.  Each GMRES restart cycle runs as one replayed CUDA graph.
"""
import numpy as np
import pytest
from conftest import rel

from bigwham_dev_b200 import HmatGpu
from bigwham_dev_b200.meshes import square_crack_3d
from bigwham_dev_b200.solve import Gmres, refine
from oracle import RefHmat

pytestmark = pytest.mark.gpu


def _dense(arr):
    D = np.zeros((arr.n_rows, arr.n_cols))
    for i0, j0, a in arr.fr_blocks():
        D[i0:i0 + a.shape[0], j0:j0 + a.shape[1]] = a
    for i0, j0, A, B in arr.lr_blocks():
        D[i0:i0 + A.shape[0], j0:j0 + B.shape[1]] = A @ B
    d = arr.dof
    rp = (d * arr.perm0[:, None] + np.arange(d)[None, :]).ravel()
    cp = (d * arr.perm1[:, None] + np.arange(d)[None, :]).ravel()
    Do = np.zeros_like(D)
    Do[np.ix_(rp, cp)] = D
    return Do


def _ops(h):
    return {p: (lambda x, y, p=p: h.matvec(x, p, out=y)) for p in h.precisions}


def _upload(arr, precs=("fp64", "fp32", "bf16")):
    return HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                             arr.perm1, device=0, precisions=precs)


def test_gmres_matches_dense_solve(golden):
    import torch

    arr, ex = golden
    h = _upload(arr)
    D = _dense(arr)
    b_np = np.random.default_rng(3).uniform(-1, 1, arr.n_rows)
    x_ref = np.linalg.solve(D, b_np)
    b = torch.from_numpy(b_np).cuda()
    minv = torch.from_numpy(1.0 / h.diagonal()).cuda()
    ops = _ops(h)
    g = Gmres(ops["fp64"], arr.n_rows, restart=30, minv=minv)
    x, info = g.solve(b, tol=1e-12, maxiter=3000)
    assert info.converged
    cond = np.linalg.cond(D)
    assert rel(x.cpu().numpy(), x_ref) < max(1e-9, 1e-14 * cond)
    for p in ("fp32", "bf16"):
        xr, inf = refine(ops["fp64"], ops[p], b, arr.n_rows, minv=minv, tol=1e-12, inner_tol=1e-3, restart=30)
        assert inf.converged, (p, inf.residuals)
        assert rel(xr.cpu().numpy(), x_ref) < max(1e-9, 1e-14 * cond)
    h.sync()


@pytest.mark.parametrize("n", [64, 128])
def test_refined_gmres_3dr0_unit_traction(n):
    """3DR0-H n x n square crack, uniform unit normal traction: Jacobi GMRES(50)
    to 1e-8 in FP64; FP32 / BF16 refinement to the same residual within 1e-6
    of the FP64 solution."""
    import torch

    coor, conn = square_crack_3d(n)
    R = RefHmat("3DR0-H", coor, conn, [1.0, 0.25], 32, 3.0, 1e-5, n_threads=16)
    arr = R.arrays()
    h = _upload(arr)
    b_np = np.zeros(arr.n_rows)
    b_np[2::3] = 1.0  # local normal component of every element
    b = torch.from_numpy(b_np).cuda()
    minv = torch.from_numpy(1.0 / h.diagonal()).cuda()
    ops = _ops(h)
    g = Gmres(ops["fp64"], arr.n_rows, restart=50, minv=minv)
    x64, info = g.solve(b, tol=1e-8, maxiter=5000)
    assert info.converged, info.residuals[-3:]
    r = torch.empty_like(b)
    ops["fp64"](x64, r)
    assert float(torch.linalg.vector_norm(b - r) / torch.linalg.vector_norm(b)) <= 1e-8
    for p in ("fp32", "bf16"):
        xr, inf = refine(ops["fp64"], ops[p], b, arr.n_rows, minv=minv, tol=1e-8, inner_tol=1e-3, restart=50)
        assert inf.converged, (p, inf.residuals)
        assert rel(xr.cpu().numpy(), x64.cpu().numpy()) <= 1e-6, p
    h.sync()
