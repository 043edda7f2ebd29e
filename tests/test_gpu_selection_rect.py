"""Sub-matrix selection and rectangular H-matrices on the GPU (-m gpu).

Selection (selection.HmatSelection, BEMatrix.__getitem__; the reference's
HmatSelection, src/hmat/hmatrix/hmat_selection.cc:141-200, reached through
BigWhamIO::hmatSelection, src/io/bigwham_io.cc:1365): the selected
sub-blocks uploaded as a handle of their own and applied by the streaming
kernels, host-array and device-tensor paths, against the reference's own
selection MatVec on 2DS0-H and 3DR0-H meshes: FP64 1e-13, FP32 2e-6 of the
largest value.

Rectangular matrices (BigWhamIO's source x receiver constructor,
src/io/bigwham_io.cc:293; the reference's CUDA path aborts on them,
hmat_cuda.cc:1358-1362): the reference-built 3DR0-3DR0-H golden case with
the reference's own MatVec / MatVecPerm outputs (1e-12), H^T against the
restatement; synthetic partitions with n_rows != n_cols against the
restatement in all precisions; and BEMatrixRectangular built by the
reference's host code through libbigwham_host.so against the reference's
own rectangular matvec.
"""
import os

import numpy as np
import pytest
from conftest import rel
from synth import synthetic_hmat
from test_selection_cpu import _cases, built  # noqa: F401

from bigwham_dev_b200 import HmatGpu
from bigwham_dev_b200.meshes import square_crack_3d
from bigwham_dev_b200.selection import HmatSelection
from oracle import HmatArrays, RefHmat, oracle_matvec, oracle_rmatvec

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 2e-6, "bf16": 1e-2}


def test_selection_matvec_on_the_gpu_equals_the_reference(built):
    import torch

    ref, ex, n = built
    rng = np.random.default_rng(3)
    for name, rows, cols in _cases(n, rng):
        sel = HmatSelection(ex, rows, cols, device=0, precisions=("fp64", "fp32"))
        x = rng.uniform(-1, 1, cols.size * ex["dof"])
        want = ref.selection_matvec(rows, cols, x)
        scale = max(1.0, np.abs(want).max())
        got = sel.matvec(x)  # host arrays
        assert got.shape == want.shape, name
        assert np.abs(got - want).max() <= 1e-13 * scale, name
        y = torch.empty(want.size, dtype=torch.float64, device="cuda")
        sel.matvec(torch.from_numpy(x).cuda(), out=y)  # device tensors
        torch.cuda.synchronize()
        assert np.array_equal(y.cpu().numpy(), got), name
        xf = x.astype(np.float32).astype(np.float64)
        assert np.abs(sel.matvec(xf, "fp32") - ref.selection_matvec(rows, cols, xf)).max() <= 2e-6 * scale, name
        sel.close()


def test_bematrix_getitem_runs_the_selection_on_the_gpu():
    """BEMatrix(...)[np.ix_(rows, cols)] (reference bigwham4py.py:462-484,
    which raises when CUDA is on) against the reference's selection MatVec."""
    from bigwham_dev_b200.bigwham4py import BEMatrix

    coor, conn = square_crack_3d(16)
    props = [1.0, 0.25]
    A = BEMatrix("3DR0-H", coor, conn, props, max_leaf_size=16, eta=3.0, eps_aca=1e-5, n_openMP_threads=8,
                 keep_host=True)
    ref = RefHmat("3DR0-H", coor, conn, props, 16, 3.0, 1e-5, n_threads=8)
    rng = np.random.default_rng(9)
    n = len(conn)
    rows, cols = rng.choice(n, 70, replace=False), rng.choice(n, 90, replace=False)
    S = A[np.ix_(rows, cols)]
    assert S.shape == (3 * rows.size, 3 * cols.size)
    x = rng.uniform(-1, 1, S.shape[1])
    want = ref.selection_matvec(rows, cols, x)
    assert np.abs(S @ x - want).max() <= 1e-13 * max(1.0, np.abs(want).max())
    S.close()


def test_rectangular_golden_on_the_gpu():
    import torch

    arr, ex = HmatArrays.load(os.path.join(os.path.dirname(__file__), "golden", "rect", "3dr0_rect.npz"))
    assert arr.n_rows != arr.n_cols
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=0, precisions=("fp64", "fp32", "bf16"), transpose=True)
    x = ex["x"]
    assert rel(h.matvec(x), ex["y_ref"]) < 1e-12
    assert rel(h.matvec(x, permuted=True), ex["y_perm_ref"]) < 1e-12
    g = np.random.default_rng(4).uniform(-1, 1, arr.n_rows)
    assert rel(h.rmatvec(g), oracle_rmatvec(arr, g, 1)) < 1e-12
    for p in ("fp32", "bf16"):
        assert rel(h.matvec(x, p), ex["y_ref"]) < TOL[p]
        assert rel(h.rmatvec(g, p), oracle_rmatvec(arr, g, 1)) < TOL[p]
    # device tensors, same bits as the host path
    yd = h.matvec(torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    assert np.array_equal(yd.cpu().numpy(), h.matvec(x))
    h.sync()


@pytest.mark.parametrize("npr,npc,dof", [(40, 25, 2), (17, 60, 3), (1, 9, 3), (33, 1, 2), (300, 170, 3)])
def test_synthetic_rectangular_partitions_on_the_gpu(npr, npc, dof):
    arr = synthetic_hmat(npr, npc, dof, seed=npr * 100 + npc, rank0_share=0.2)
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=0, precisions=("fp64", "fp32", "bf16"), transpose=True)
    x = np.random.default_rng(2).uniform(-1, 1, arr.n_cols)
    g = np.random.default_rng(3).uniform(-1, 1, arr.n_rows)
    y_or, yt_or = oracle_matvec(arr, x, 1), oracle_rmatvec(arr, g, 1)
    for p in ("fp64", "fp32", "bf16"):
        assert rel(h.matvec(x, p), y_or) < TOL[p], p
        assert rel(h.rmatvec(g, p), yt_or) < TOL[p], p
    h.sync()


def test_bematrix_rectangular_against_the_reference():
    """A 3DR0-3DR0-H matrix (a 24 x 24 crack acting on a 17 x 21 receiver grid
    on a parallel plane) built by the reference's host code in
    libbigwham_host.so with the GPU backend installed, against the
    reference's own build and matvec (FP64, 1e-12)."""
    from bigwham_dev_b200.bigwham4py import BEMatrixRectangular

    cs, es = square_crack_3d(24)
    cr, er = square_crack_3d(17, 21, half=1.3)
    cr = cr + np.array([0.05, -0.1, 0.4])
    props = [1.0, 0.25]
    A = BEMatrixRectangular("3DR0-3DR0-H", cs, es, cr, er, props, max_leaf_size=16, eta=3.0, eps_aca=1e-6,
                            n_openMP_threads=8, precisions=("fp64",), transpose=True)
    R = RefHmat.rectangular("3DR0-3DR0-H", cs, es, cr, er, props, 16, 3.0, 1e-6, n_threads=8)
    assert A.shape == R.shape and A.shape[0] != A.shape[1]
    x = np.random.default_rng(8).uniform(-1, 1, A.shape[1])
    assert rel(A @ x, R.matvec(x)) < 1e-12
    # H^T against the reference's dense columns: <A x, g> = <x, A^T g>
    g = np.random.default_rng(9).uniform(-1, 1, A.shape[0])
    assert abs(np.dot(A @ x, g) - np.dot(x, A.rmatvec(g))) <= 1e-12 * np.linalg.norm(A @ x) * np.linalg.norm(g)
