"""Rectangular and irregular H-matrices through the layout (host plan).

Hmat::matvec (src/hmat/hmatrix/hmat.cc:472-537) does not assume a square
matrix: BigWhamIO's rectangular constructor (src/io/bigwham_io.h:85-96) pairs
a source mesh with a different receiver mesh.  The reference's own CUDA path
aborts on non-square matrices (hmat_cuda.cc:1358-1362); this backend lays
them out like square ones.  Synthetic quadtree partitions (tests/synth.py)
with n_rows != n_cols, dof 1-3, odd block shapes and ragged ranks; the
replayed plan must match the oracle in FP64 (1e-14) for H and H^T, and the
reduced precisions within their rounding bounds.
"""
import numpy as np
import pytest

from oracle import oracle_matvec_perm, oracle_rmatvec_perm
from planreplay import replay
from synth import synthetic_hmat

from bigwham_dev_b200 import HmatGpu

SHAPES = [(40, 25, 2), (17, 60, 3), (64, 64, 1), (1, 9, 3), (33, 1, 2)]
TOL = {"fp64": 1e-14, "fp32": 2e-6, "bf16": 1e-2}


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("npr,npc,dof", SHAPES)
@pytest.mark.parametrize("precision", ["fp64", "fp32", "bf16"])
def test_rectangular_plan_matches_the_oracle(npr, npc, dof, precision):
    arr = synthetic_hmat(npr, npc, dof, seed=npr * 100 + npc)
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=-1, plan_only=True, precisions=(precision,), transpose=True)
    x = np.random.default_rng(2).uniform(-1, 1, arr.n_cols)
    xr = np.random.default_rng(3).uniform(-1, 1, arr.n_rows)
    assert _rel(replay(h, x, precision), oracle_matvec_perm(arr, x, 1)) < TOL[precision]
    assert _rel(replay(h, xr, precision, True), oracle_rmatvec_perm(arr, xr, 1)) < TOL[precision]


def test_dense_single_block_and_all_low_rank():
    """Degenerate partitions: one full-rank block; only low-rank blocks."""
    one = synthetic_hmat(5, 7, 3, seed=9, leaf=100)
    assert len(one.fr) + len(one.lr) == 1
    lr_only = synthetic_hmat(32, 24, 2, seed=4, leaf=4, stop=0.0, lr_share=1.0)
    assert len(lr_only.fr) == 0 and len(lr_only.lr) > 10
    for arr in (one, lr_only):
        h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                              arr.perm1, device=-1, plan_only=True, precisions=("fp64",))
        x = np.random.default_rng(5).uniform(-1, 1, arr.n_cols)
        assert _rel(replay(h, x, "fp64"), oracle_matvec_perm(arr, x, 1)) < 1e-14


def test_reference_built_rectangular_hmatrix():
    """A real rectangular H-matrix (BigWhamIO's source x receiver constructor,
    kernel 3DR0-3DR0-H: a 10 x 10 crack acting on a 7 x 9 grid of receivers on
    a parallel plane): export, lay out, replay against the oracle, H and H^T."""
    import os

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if not os.path.exists(os.path.join(root, "bigwham_dev_b200", "_lib", "libbigwham_host.so")):
        pytest.skip("host adapter not built")
    from bigwham_dev_b200.bigwham4py import BigWhamIOGpu
    from bigwham_dev_b200.meshes import square_crack_3d
    from oracle import HmatArrays

    cs, es = square_crack_3d(10)
    cr, er = square_crack_3d(7, 9, half=1.3)
    cr = cr + np.array([0.05, -0.1, 0.4])
    io = BigWhamIOGpu.rectangular(cs, es, cr, er, "3DR0-3DR0-H", [1.0, 0.25], 2, useCuda=False)
    io.build_hierarchical_matrix(16, 3.0, 1e-6)
    ex = io.export_blocks()
    assert (ex["n_rows"], ex["n_cols"]) == (3 * len(er), 3 * len(es))
    assert sorted(ex["perm0"]) == list(range(len(er))) and sorted(ex["perm1"]) == list(range(len(es)))
    assert np.array_equal(io.get_permutation(), ex["perm1"])
    io.close()
    arr = HmatArrays(ex["dof"], ex["n_rows"], ex["n_cols"], ex["fr"], ex["lr"], ex["fr_data"], ex["lr_data"],
                     ex["perm0"], ex["perm1"])
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=-1, plan_only=True, precisions=("fp64", "bf16"), transpose=True)
    x = np.random.default_rng(4).uniform(-1, 1, arr.n_cols)
    xr = np.random.default_rng(5).uniform(-1, 1, arr.n_rows)
    assert _rel(replay(h, x, "fp64"), oracle_matvec_perm(arr, x, 1)) < 1e-14
    assert _rel(replay(h, xr, "fp64", True), oracle_rmatvec_perm(arr, xr, 1)) < 1e-14
    assert _rel(replay(h, x, "bf16"), oracle_matvec_perm(arr, x, 1)) < 1e-2


def test_rectangular_golden_against_the_reference_matvec():
    """tests/golden/rect/3dr0_rect.npz (make_golden.py --rect): a 3DR0-3DR0-H
    matrix built by the reference, with the reference's own MatVec and
    MatVecPerm outputs.  The oracle restatement and our replayed plan must
    match them to 1e-12; both are within the ACA tolerance of the dense
    (eta = 0) product."""
    import os

    from oracle import HmatArrays, oracle_matvec

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rect", "3dr0_rect.npz")
    arr, ex = HmatArrays.load(path)
    assert arr.n_rows != arr.n_cols
    x = ex["x"]
    assert _rel(oracle_matvec(arr, x, 1), ex["y_ref"]) < 1e-12
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=-1, plan_only=True, precisions=("fp64",))
    # MatVecPerm takes x in the clustered ordering, as the replay does
    assert _rel(replay(h, x, "fp64"), ex["y_perm_ref"]) < 1e-12
    assert _rel(ex["y_ref"], ex["y_dense"]) < 1e-4
