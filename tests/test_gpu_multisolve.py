"""Many systems per GMRES on the GPU (-m gpu), each restart cycle one replayed
CUDA graph (solve.MultiGmres / refine_multi).

* C4a: 48 independent 2DS0-H straight cracks on [-1,1] (segment counts
  log-uniform in [256, 16,384], numpy default_rng(3); E = 1, nu = 0.25, leaf
  32, eta 3, eps 1e-5, built by the reference), one batched handle
  (bw_create_batch), unit normal traction on every member.  Every Arnoldi
  step applies all 48 H-matrices in one matvec (BatchOperator); every member
  keeps its own Krylov space and stopping test.  FP64 Jacobi GMRES(50) to a
  relative residual of 1e-10 per member, checked member by member with that
  member's own handle; FP32 refinement (FP64 residual and update) to 1e-8
  per member, within 1e-6 of the FP64 solution.  BF16 refinement contracts
  only where cond(A) x 5e-4 < 1: the short cracks converge to 1e-8; the long
  ones (cond grows with the segment count) either stop at their best iterate,
  reported as diverged, or stall; every iterate stays finite.
* C4b at a test size: 3DR0-H 64 x 64 (12,288 DoF), 64 right-hand sides
  ~ U(-1,1) (seed 5): inner Arnoldi steps on the tensor-core matmat (BF16
  blocks and right-hand sides, FP32 accumulation, one launch sequence for all
  64), FP64 residual and update, to 1e-8 per right-hand side, each within
  1e-6 of that right-hand side's own FP64 GMRES solution.
"""
import numpy as np
import pytest
from conftest import rel
from test_gpu_batch import c4a_members

from bigwham_dev_b200 import HmatGpu
from bigwham_dev_b200.meshes import square_crack_3d
from bigwham_dev_b200.solve import BatchOperator, Gmres, MultiGmres, refine_multi
from oracle import RefHmat

pytestmark = pytest.mark.gpu


def test_c4a_batched_gmres_per_member():
    import torch

    ms = c4a_members()
    hb = HmatGpu.batch(ms, device=0, precisions=("fp64", "fp32", "bf16"))
    op64, op32, op16 = BatchOperator(hb, "fp64"), BatchOperator(hb, "fp32"), BatchOperator(hb, "bf16")
    b_cat = np.zeros(hb.n_rows)
    b_cat[1::2] = 1.0  # normal component of every segment
    B = op64.pad(torch.from_numpy(b_cat).cuda())
    diag = torch.from_numpy(hb.diagonal()).cuda()
    minv = op64.pad(1.0 / diag)  # zero on the padding
    X, info = MultiGmres(op64, op64.count, op64.L, restart=50, minv=minv).solve(B, tol=1e-10, maxiter=6000)
    assert info.converged, [s.residuals[-1] for s in info.per_system if not s.converged]
    x_cat = op64.unpad(X).cpu().numpy()
    for k in (0, 17, 47) + tuple(int(i) for i in np.argsort([m.n_rows for m in ms])[-2:]):
        m = ms[k]
        r0, r1 = int(hb.row_offsets[k]), int(hb.row_offsets[k + 1])
        s = HmatGpu.from_flat(m.dof, m.n_rows, m.n_cols, m.fr, m.lr, m.fr_data, m.lr_data, m.perm0, m.perm1,
                              device=0, precisions=("fp64",))
        y = s.matvec(x_cat[r0:r1])
        assert rel(y, b_cat[r0:r1]) <= 2e-10, k  # the member's own handle
        s.close()
    R = torch.empty_like(B)
    Xr, inf = refine_multi(op64, op32, B, minv=minv, tol=1e-8, inner_tol=1e-3, restart=50)
    assert inf.converged, inf.residuals
    op64(Xr, R)
    res = torch.linalg.vector_norm(B - R, dim=1) / torch.linalg.vector_norm(B, dim=1)
    assert float(res.max()) <= 1e-8
    err = torch.linalg.vector_norm(Xr - X, dim=1) / torch.linalg.vector_norm(X, dim=1)
    assert float(err.max()) <= 1e-6
    # BF16 inner solves: the short cracks converge; no iterate overflows
    Xb, inf = refine_multi(op64, op16, B, minv=minv, tol=1e-8, inner_tol=1e-3, restart=50)
    assert bool(torch.isfinite(Xb).all())
    op64(Xb, R)
    res = (torch.linalg.vector_norm(B - R, dim=1) / torch.linalg.vector_norm(B, dim=1)).cpu().numpy()
    conv = [i for i, p in enumerate(inf.per_system) if p.converged]
    div = [i for i, p in enumerate(inf.per_system) if p.diverged]
    sizes = [int(m.n_rows) for m in ms]
    print(f"C4a BF16 refinement: {len(conv)} members converged (largest {max(sizes[i] for i in conv)} DoF), "
          f"{len(div)} stopped as diverged, {len(ms) - len(conv) - len(div)} stalled")
    assert len(conv) > 0 and min(sizes[i] for i in conv) == min(sizes)
    assert float(res[conv].max()) <= 1e-8
    assert all(res[i] <= 1.0 for i in div)
    hb.close()


def test_c4b_64_rhs_on_the_tensor_cores():
    import torch

    coor, conn = square_crack_3d(64)
    R = RefHmat("3DR0-H", coor, conn, [1.0, 0.25], 32, 3.0, 1e-5, n_threads=16)
    arr = R.arrays()
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=0, precisions=("fp64", "bf16"), matmat=True)
    n, k = h.n_rows, 64
    B = torch.from_numpy(np.random.default_rng(5).uniform(-1, 1, (k, n))).cuda()
    minv = torch.from_numpy(1.0 / h.diagonal()).cuda()

    def op_hi(Z, W):  # FP64: one matvec per right-hand side
        h.matmat(Z.t(), "fp64", out=W.t())

    def op_tc(Z, W):  # tensor cores: all 64 right-hand sides per launch sequence
        h.matmat(Z.t(), "bf16", out=W.t())

    X, info = refine_multi(op_hi, op_tc, B, minv=minv, tol=1e-8, inner_tol=1e-3, restart=50)
    assert info.converged, info.residuals
    W = torch.empty_like(B)
    op_hi(X, W)
    res = torch.linalg.vector_norm(B - W, dim=1) / torch.linalg.vector_norm(B, dim=1)
    assert float(res.max()) <= 1e-8
    for j in (0, 31, 63):
        xj, inf = Gmres(lambda x, y: h.matvec(x, "fp64", out=y), n, restart=50, minv=minv).solve(
            B[j].contiguous(), tol=1e-10, maxiter=5000)
        assert inf.converged
        assert rel(X[j].cpu().numpy(), xj.cpu().numpy()) <= 1e-6, j
    h.close()
