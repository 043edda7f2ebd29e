"""The BigWhamIO pass-throughs behind bigwham4py.BEMatrix's reference-named
methods (convert_to_local / _global, get_element_normals, get_rotation_matrix,
get_max_error_ACA, _getFullBlocks, compute_displacements / _stresses,
getStorageRequirement, get_omp_threads), on CPU through the host library.

Each calls the reference's own BigWhamIO method (compiled unmodified into the
host library), so the checks are consistency checks against other views of the
same build: the oracle's element frames, the exported blocks, the block file's
ACA estimates, and linearity of the field computations.
"""
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST_LIB = os.path.join(ROOT, "bigwham_dev_b200", "_lib", "libbigwham_host.so")
pytestmark = pytest.mark.skipif(not os.path.exists(HOST_LIB), reason="host adapter not built")


@pytest.fixture(scope="module")
def built3d():
    from bigwham_dev_b200.bigwham4py import BigWhamIOGpu
    from bigwham_dev_b200.meshes import square_crack_3d

    coor, conn = square_crack_3d(14)
    io = BigWhamIOGpu(coor, conn, "3DR0-H", [1.0, 0.25], 3, useCuda=False)
    io.build_hierarchical_matrix(32, 3.0, 1e-5)
    yield io, coor, conn
    io.close()


def test_frames_normals_and_conversions(built3d):
    from oracle import RefHmat, ref_available

    io, coor, conn = built3d
    n = len(conn)
    nrm, rot = io.get_element_normals(), io.get_rotation_matrix()
    assert nrm.shape == (3 * n,) and rot.shape == (9 * n,)
    # the reference clamps the request to the process's current OpenMP team
    # size, which an earlier BigWhamIO in this process may have lowered
    assert io.get_spatial_dimension() == 3 and 1 <= io.get_omp_threads() <= 3
    if ref_available():
        fr = RefHmat("3DR0-H", coor, conn, [1.0, 0.25], 32, 3.0, 1e-5, n_threads=2).element_frames()
        assert np.array_equal(rot.reshape(n, 9), fr[:, 3:12]) and np.array_equal(nrm.reshape(n, 3), fr[:, 12:15])
    # local = R global per element (dof-interleaved), and back
    x = np.random.default_rng(1).uniform(-1, 1, 3 * n)
    loc = io.convert_to_local(x)
    R = rot.reshape(n, 3, 3)
    assert np.allclose(loc.reshape(n, 3), np.einsum("eij,ej->ei", R, x.reshape(n, 3)), atol=1e-15)
    assert np.allclose(io.convert_to_global(loc), x, atol=1e-14)


def test_aca_error_full_blocks_and_storage(built3d, tmp_path):
    from bigwham_dev_b200 import blockfile

    io, coor, conn = built3d
    ex = io.export_blocks()
    io.write_to_file(tmp_path / "h.bwb")
    assert io.get_max_error_ACA() == blockfile.read(tmp_path / "h.bwb")["lr_error"].max() > 0
    assert io.get_storage_requirement() == 8 * (ex["fr_data"].size + ex["lr_data"].size)
    val, row, col = io.get_full_blocks(original_order=False)
    assert val.size == ex["fr_data"].size
    # permuted-order entries are the exported FR blocks, column-major per block
    d, k, o = ex["dof"], 0, 0
    i0, j0, i1, j1 = ex["fr"][0]
    m, nn = (i1 - i0) * d, (j1 - j0) * d
    blk = ex["fr_data"][:m * nn].reshape(m, nn, order="F")
    sel = (row >= i0 * d) & (row < i1 * d) & (col >= j0 * d) & (col < j1 * d)
    assert sel.sum() == m * nn
    assert np.array_equal(np.sort(val[sel]), np.sort(blk.ravel()))
    vo, ro, co = io.get_full_blocks(original_order=True)
    assert np.array_equal(np.sort(vo), np.sort(val))


def test_field_computations_are_linear():
    """ComputeStresses / ComputeDisplacements on a 2DS0 crack (below the size
    where the reference's parallel accumulation races): shape, zero for a zero
    solution, linear in the solution."""
    from bigwham_dev_b200.bigwham4py import BigWhamIOGpu
    from bigwham_dev_b200.meshes import straight_crack_2d

    coor, conn = straight_crack_2d(40)
    io = BigWhamIOGpu(coor, conn, "2DS0-H", [1.0, 0.25], 1, useCuda=False)
    io.build_hierarchical_matrix(16, 2.0, 1e-4)
    pts = np.array([[0.1, 0.3], [-0.5, 1.2], [2.0, -0.7]])
    sol = np.random.default_rng(2).uniform(-1, 1, 2 * len(conn))
    s1, s2 = io.compute_stresses(pts, sol), io.compute_stresses(pts, 2 * sol)
    u1 = io.compute_displacements(pts, sol)
    assert s1.shape == (9,) and u1.shape == (6,)
    assert np.all(np.isfinite(s1)) and np.abs(s1).max() > 0
    assert np.allclose(s2, 2 * s1, rtol=1e-13, atol=0)
    assert np.array_equal(io.compute_stresses(pts, 0 * sol), np.zeros(9))
    io.close()


def test_bematrix_reference_methods_without_gpu():
    """BEMatrix built with useCuda=False (host build, no GPU H-matrix): the
    reference-named methods that do not apply the operator, and the selection's
    full-block entries."""
    from scipy.sparse.linalg import LinearOperator

    from bigwham_dev_b200.bigwham4py import BEMatrix
    from bigwham_dev_b200.meshes import straight_crack_2d

    coor, conn = straight_crack_2d(64)
    A = BEMatrix("2DS0-H", coor, conn, np.array([1.0, 0.25]), 16, 2.0, 1e-4, n_openMP_threads=2, useCuda=False)
    n = 2 * len(conn)
    assert A.shape == (n, n) and A.getSpatialDimension() == 2
    # the reference clamps the request to the process's current OpenMP team
    # size, which every earlier BigWhamIO constructor set globally
    assert 1 <= A.get_omp_threads() <= 2
    assert A.getCollocationPoints().shape == (len(conn), 2)
    assert A.getStorageRequirement() > 0 and A.getGPUStorageRequirement() == 0
    fb = A._getFullBlocks()
    assert fb.shape == (n, n) and fb.nnz > 0
    assert np.allclose(fb.diagonal(), A.H_diag())
    half = A._getFullBlocks(keep_ratio=0.5)
    assert 0 < half.nnz < fb.nnz
    assert isinstance(A.H_ILU_prec(), LinearOperator)
    # no dropping and room for all fill-in: the ILU is the LU of the full blocks
    P = A.H_ILU_prec(fill_factor=100, drop_tol=0.0)
    v = np.random.default_rng(3).uniform(-1, 1, n)
    assert np.linalg.norm(fb @ (P @ v) - v) / np.linalg.norm(v) < 1e-10
    pat = A._getPattern()
    assert pat.shape[1] == 6
    # plotPattern(plot_index=True) labels: each block's index among its kind, in pattern order
    from bigwham_dev_b200.bigwham4py import pattern_kind_index

    idx = pattern_kind_index(pat)
    for kind in (0, 1):
        assert np.array_equal(idx[pat[:, 4] == kind], np.arange(int((pat[:, 4] == kind).sum())))
    x = np.random.default_rng(4).uniform(-1, 1, n)
    assert np.allclose(A.convert_to_global(A.convert_to_local(x)), x)
    pts = np.array([[0.0, 0.5], [3.0, -1.0]])
    assert A.compute_stresses(pts, x).shape == (2, 3) and A.compute_displacements(pts, x).shape == (2, 2)
    assert A.get_max_error_ACA() >= 0
    assert A.get_element_normals().size == 2 * len(conn) and A.get_rotation_matrix().size == 4 * len(conn)
    # selection (the reference raises here with CUDA): the selected full-rank
    # entries are the full matrix's, at the selected rows and columns
    rows, cols = np.array([0, 1, 5, 40]), np.array([3, 1, 60])
    S = A[np.ix_(rows, cols)]
    assert S.shape == (2 * rows.size, 2 * cols.size)
    rd = (2 * rows[:, None] + np.arange(2)).ravel()
    cd = (2 * cols[:, None] + np.arange(2)).ravel()
    assert np.array_equal(S._getFullBlocks().toarray(), fb.toarray()[np.ix_(rd, cd)])
    with pytest.raises(IndexError):
        A[np.ix_([0, len(conn)], [0])]
