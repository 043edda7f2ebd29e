"""Block-Jacobi preconditioner on CPU (precond.BlockJacobi, host plan).

* The diagonal full-rank blocks of a built 3DR0-H H-matrix tile the diagonal
  in the clustered ordering; a pattern whose diagonal has a hole is rejected.
* The batched handle of the inverses, replayed as the kernels would run it,
  undoes the diagonal blocks: M_perm^-1 (blockdiag(D) v) = v to 1e-12.
* In the original ordering the preconditioner is P1^T M_perm^-1 P0 (dense
  check with the permutation matrices).
* GMRES(10) on the oracle's matvec converges to 1e-8 with fewer Arnoldi steps
  than with the reference's point Jacobi (BEMatrix.H_jacobi_prec).
"""
import os

import numpy as np
import pytest
import torch

from planreplay import replay

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST_LIB = os.path.join(ROOT, "bigwham_dev_b200", "_lib", "libbigwham_host.so")
pytestmark = pytest.mark.skipif(not os.path.exists(HOST_LIB), reason="host adapter not built")


def _crack(n):
    from bigwham_dev_b200.bigwham4py import BigWhamIOGpu
    from bigwham_dev_b200.meshes import square_crack_3d

    coor, conn = square_crack_3d(n)
    io = BigWhamIOGpu(coor, conn, "3DR0-H", [1.0, 0.25], 4, useCuda=False)
    io.build_hierarchical_matrix(32, 3.0, 1e-5)
    ex = io.export_blocks()
    io.close()
    return ex


@pytest.fixture(scope="module")
def crack16():
    return _crack(16)


def _host_bj(ex):
    """BlockJacobi with a host plan whose products are the kernel replay."""
    from bigwham_dev_b200.precond import BlockJacobi

    bj = BlockJacobi(ex, device=-1, plan_only=True)
    bj.h.matvec = lambda x, precision="fp64": replay(bj.h, np.asarray(x, dtype=np.float64), precision)
    return bj


def test_diagonal_blocks_tile_and_holes_are_rejected(crack16):
    from bigwham_dev_b200.precond import diagonal_blocks

    diag = diagonal_blocks(crack16)
    fr = crack16["fr"]
    assert fr[diag[0], 0] == 0 and fr[diag[-1], 2] * crack16["dof"] == crack16["n_rows"]
    assert all(fr[a, 2] == fr[b, 0] for a, b in zip(diag[:-1], diag[1:]))
    holed = dict(crack16, fr=np.delete(fr, diag[len(diag) // 2], axis=0))
    with pytest.raises(ValueError, match="tile the diagonal"):
        diagonal_blocks(holed)
    with pytest.raises(ValueError, match="square"):
        diagonal_blocks(dict(crack16, n_cols=crack16["n_cols"] + 3))


def test_batched_inverses_undo_the_diagonal_blocks(crack16):
    from bigwham_dev_b200.precond import diagonal_blocks, inverted_blocks

    ex = crack16
    bj = _host_bj(ex)
    blocks = inverted_blocks(ex, diagonal_blocks(ex))
    assert bj.blocks == len(blocks) and bj.entries == sum(D.size for _, D in blocks)
    v = np.random.default_rng(4).uniform(-1, 1, ex["n_rows"])
    dv = np.empty_like(v)
    for s, Dinv in blocks:
        m = Dinv.shape[0]
        dv[s:s + m] = np.linalg.solve(Dinv, v[s:s + m])  # D_k v_k
    back = bj.h.matvec(dv)
    assert np.linalg.norm(back - v) / np.linalg.norm(v) < 1e-12


def test_original_ordering_is_p1t_minv_p0(crack16):
    from bigwham_dev_b200.precond import diagonal_blocks, inverted_blocks

    ex = crack16
    n, d = ex["n_rows"], ex["dof"]
    bj = _host_bj(ex)
    Mp = np.zeros((n, n))
    for s, Dinv in inverted_blocks(ex, diagonal_blocks(ex)):
        Mp[s:s + Dinv.shape[0], s:s + Dinv.shape[0]] = Dinv

    def pmat(perm):  # (P x)[d i + j] = x[d perm[i] + j]
        P = np.zeros((n, n))
        P[np.arange(n), (d * np.asarray(perm)[:, None] + np.arange(d)).ravel()] = 1.0
        return P

    x = np.random.default_rng(5).uniform(-1, 1, n)
    want = pmat(ex["perm1"]).T @ (Mp @ (pmat(ex["perm0"]) @ x))
    got = bj(x, np.empty(n))
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-12


def test_gmres_needs_fewer_steps_than_point_jacobi():
    from bigwham_dev_b200.precond import diagonal_blocks, inverted_blocks
    from bigwham_dev_b200.solve import Gmres
    from oracle import HmatArrays, oracle_matvec

    ex = _crack(48)
    n = ex["n_rows"]
    arr = HmatArrays(ex["dof"], n, ex["n_cols"], ex["fr"], ex["lr"], ex["fr_data"], ex["lr_data"], ex["perm0"],
                     ex["perm1"])
    bj = _host_bj(ex)

    def op(x, y):
        y.copy_(torch.from_numpy(oracle_matvec(arr, x.numpy(), 4)))

    def block(x, out):
        out.copy_(torch.from_numpy(bj(x.numpy(), np.empty(n))))

    diag = np.empty(n)
    for s, Dinv in inverted_blocks(ex, diagonal_blocks(ex)):
        diag[s:s + Dinv.shape[0]] = np.diag(np.linalg.inv(Dinv))  # diagonal of H, clustered ordering
    d = ex["dof"]
    p0 = (d * np.asarray(ex["perm0"])[:, None] + np.arange(d)).ravel()
    diag_orig = np.empty(n)
    diag_orig[p0] = diag  # H_diag in the original ordering
    b = torch.zeros(n, dtype=torch.float64)
    b[2::3] = 1.0  # unit normal traction on every element
    steps = {}
    for name, minv in (("jacobi", torch.from_numpy(1.0 / diag_orig)), ("block", block)):
        x, info = Gmres(op, n, restart=10, minv=minv, device="cpu", use_graph=False).solve(b, tol=1e-8, maxiter=400)
        r = b - torch.from_numpy(oracle_matvec(arr, x.numpy(), 4))
        assert info.converged and float(torch.linalg.vector_norm(r) / torch.linalg.vector_norm(b)) < 2e-8
        steps[name] = info.iterations
    assert steps["block"] < steps["jacobi"], steps
