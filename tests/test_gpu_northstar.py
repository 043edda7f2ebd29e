"""The target configuration on one B200 (-m gpu, slow): 3DR0-H planar square
crack, 256 x 256 rectangles on [-1,1]^2 in z = 0 (196,608 DoF), E = 1,
nu = 0.25, leaf 32, eta 3, ACA eps 1e-5, built by the reference's own code.

* FP64 parity: the GPU matvec against the reference's OpenMP matvec
  (BigWhamIO::MatVec, src/io/bigwham_io.cc:927-933) on the same H-matrix,
  x ~ U(-1,1) seed 1: relative error <= 1e-12.
* The FP64 dense oracle of the same kernel on a sampled row subset: the
  reference's influence() for 683 collocation points (2,049 rows, numpy
  default_rng(7)) over all 196,608 columns (BieMatrixGenerator::set's entry
  rule, src/hmat/bie_matrix_generator.h:94-142).  Matvec errors on those rows
  are printed for every storage precision and bounded by the H-matrix error
  plus the storage rounding (FP64 / FP32 <= 1e-6, BF16 <= 2e-3).
* Refined GMRES: uniform unit normal traction, FP64 Jacobi GMRES(50) to a
  relative residual of 1e-8, then iterative refinement with FP32 and with
  BF16 inner solves (FP64 residual and update) to 1e-8.  The refined
  solutions lie within 1e-6 of the FP64 GMRES solution.  Against the dense
  rows, the FP64 solution's residual is the H-matrix's own approximation
  error at ACA eps 1e-5 (measured 5.0e-6; bound 1e-5), and mixed precision
  adds at most 1e-6 to it.
* The 64-right-hand-side tensor-core matmat (BF16 blocks and X, FP32
  accumulation) against the FP64 restatement of the reference's block loop
  (oracle_matvec) on columns 0 and 63: <= 8e-3, the BF16 bound of the suite.
* 64 right-hand sides ~ U(-1,1) (seed 5) solved together: inner GMRES(50)
  Arnoldi steps on that matmat (one launch sequence for all 64, each restart
  cycle a replayed CUDA graph), FP64 residual and update, to 1e-8 per
  right-hand side; columns 0 and 63 within 1e-6 of their own FP64 GMRES
  solutions.
"""
import os

import numpy as np
import pytest
from conftest import rel

from bigwham_dev_b200 import HmatGpu
from bigwham_dev_b200.meshes import square_crack_3d
from bigwham_dev_b200.solve import Gmres, refine, refine_multi
from oracle import RefHmat, oracle_matvec

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

PROPS = [1.0, 0.25]
N_SIDE = int(os.environ.get("BW_NORTHSTAR_N", "256"))


@pytest.fixture(scope="module")
def c4b():
    import torch

    coor, conn = square_crack_3d(N_SIDE)
    R = RefHmat("3DR0-H", coor, conn, PROPS, 32, 3.0, 1e-5, n_threads=os.cpu_count() or 16)
    arr = R.arrays()
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=0, precisions=("fp64", "fp32", "bf16"), matmat=True)
    npts = arr.n_rows // 3
    sample = np.sort(np.random.default_rng(7).choice(npts, size=683, replace=False))
    D = R.dense_rows("3DR0-H", PROPS, sample)
    rows = (3 * sample[:, None] + np.arange(3)[None, :]).ravel()
    b = np.zeros(arr.n_rows)
    b[2::3] = 1.0
    minv = torch.from_numpy(1.0 / h.diagonal()).cuda()
    yield {"R": R, "arr": arr, "h": h, "D": D, "rows": rows, "b": b, "minv": minv}
    h.close()


def test_fp64_parity_and_dense_rows(c4b):
    R, h, D, rows = c4b["R"], c4b["h"], c4b["D"], c4b["rows"]
    x = np.random.default_rng(1).uniform(-1, 1, h.n_cols)
    y64 = h.matvec(x, "fp64")
    par = rel(y64, R.matvec(x))
    print(f"C4b {h.n_rows} DoF: FP64 GPU vs reference OpenMP matvec {par:.2e}")
    assert par <= 1e-12
    yd = D @ x
    for p, tol in (("fp64", 1e-6), ("fp32", 1e-6), ("bf16", 2e-3)):
        e = rel((y64 if p == "fp64" else h.matvec(x, p))[rows], yd)
        print(f"C4b {p} matvec vs dense rows: {e:.3e}")
        assert e <= tol, p


def test_refined_gmres_against_the_dense_rows(c4b):
    import torch

    h, D, rows, minv = c4b["h"], c4b["D"], c4b["rows"], c4b["minv"]
    b = torch.from_numpy(c4b["b"]).cuda()
    ops = {p: (lambda x, y, p=p: h.matvec(x, p, out=y)) for p in ("fp64", "fp32", "bf16")}
    x64, info = Gmres(ops["fp64"], h.n_rows, restart=50, minv=minv).solve(b, tol=1e-8, maxiter=5000)
    assert info.converged, info.residuals[-3:]
    r = torch.empty_like(b)
    ops["fp64"](x64, r)
    assert float(torch.linalg.vector_norm(b - r) / torch.linalg.vector_norm(b)) <= 1e-8
    X = x64.cpu().numpy()
    b_rows = c4b["b"][rows]
    dres = rel(D @ X, b_rows)
    print(f"C4b FP64 GMRES(50): {info.iterations} Arnoldi steps; dense-row residual {dres:.2e}")
    assert dres <= 1e-5  # the H-matrix itself (ACA eps 1e-5)
    for p in ("fp32", "bf16"):
        xr, inf = refine(ops["fp64"], ops[p], b, h.n_rows, minv=minv, tol=1e-8, inner_tol=1e-3, restart=50)
        assert inf.converged, (p, inf.residuals)
        ops["fp64"](xr, r)
        res = float(torch.linalg.vector_norm(b - r) / torch.linalg.vector_norm(b))
        Xr = xr.cpu().numpy()
        e64, ed = rel(Xr, X), rel(D @ Xr, b_rows)
        print(f"C4b refine {p}: {inf.outer} outer steps, {inf.iterations} inner; residual {res:.2e}, "
              f"vs FP64 solution {e64:.2e}, dense-row residual {ed:.2e}")
        assert res <= 1e-8 and e64 <= 1e-6 and ed <= dres + 1e-6, p


def test_matmat_64_rhs_against_the_oracle(c4b):
    import torch

    arr, h = c4b["arr"], c4b["h"]
    X = np.random.default_rng(5).uniform(-1, 1, (h.n_cols, 64))
    Y = h.matmat(torch.from_numpy(X).cuda(), "bf16")
    torch.cuda.synchronize()
    Yh = Y.cpu().numpy()
    for j in (0, 63):
        e = rel(Yh[:, j], oracle_matvec(arr, np.ascontiguousarray(X[:, j]), os.cpu_count() or 16))
        print(f"C4b matmat column {j} vs FP64 oracle: {e:.2e}")
        assert e <= 8e-3


def test_64_rhs_refined_gmres_on_the_tensor_cores(c4b):
    import torch

    h, minv = c4b["h"], c4b["minv"]
    n, k = h.n_rows, 64
    B = torch.from_numpy(np.random.default_rng(5).uniform(-1, 1, (k, n))).cuda()

    def op_hi(Z, W):
        h.matmat(Z.t(), "fp64", out=W.t())

    def op_tc(Z, W):
        h.matmat(Z.t(), "bf16", out=W.t())

    X, info = refine_multi(op_hi, op_tc, B, minv=minv, tol=1e-8, inner_tol=1e-3, restart=50)
    assert info.converged, info.residuals
    W = torch.empty_like(B)
    op_hi(X, W)
    res = torch.linalg.vector_norm(B - W, dim=1) / torch.linalg.vector_norm(B, dim=1)
    print(f"C4b 64 right-hand sides: {info.outer} outer steps, {info.iterations} inner Arnoldi steps, "
          f"max residual {float(res.max()):.2e}")
    assert float(res.max()) <= 1e-8
    for j in (0, 63):
        xj, inf = Gmres(lambda x, y: h.matvec(x, "fp64", out=y), n, restart=50, minv=minv).solve(
            B[j].contiguous(), tol=1e-10, maxiter=5000)
        assert inf.converged
        assert rel(X[j].cpu().numpy(), xj.cpu().numpy()) <= 1e-6, j
