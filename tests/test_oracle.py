"""The oracle is pinned before it is trusted.

* the C restatement (oracle/hmatvec_oracle.c) against the golden vectors made
  by the reference itself (tests/golden/make_golden.py);
* the reference build (oracle/_ref) against the known-answer tests of the
  reference's own suite (src/io/_test/bigwham_io_gen_test_2d.cc:141-187,
  src/elasticity/_test/elastic_square_matrix_generator_test.cc:134-182);
* the restatement against the live reference on meshes not in the fixtures.
"""
import numpy as np
import pytest
from conftest import rel

from oracle import (RefHmat, oracle_diagonal, oracle_entries, oracle_matmat, oracle_matvec, oracle_matvec_perm,
                    oracle_rmatvec, ref_available)
from bigwham_dev_b200.meshes import square_crack_3d, straight_crack_2d

needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")


def test_restatement_matches_golden(golden):
    arr, ex = golden
    x = ex["x"]
    # summation order differs from the BLAS; 1e-13 is far below any real difference
    assert rel(oracle_matvec(arr, x, 1), ex["y_ref"]) < 1e-13
    assert rel(oracle_matvec(arr, x, 3), ex["y_ref"]) < 1e-13
    assert rel(oracle_matvec_perm(arr, x, 2), ex["y_perm_ref"]) < 1e-13
    assert np.array_equal(oracle_diagonal(arr), ex["diag_ref"])
    assert oracle_entries(arr) == arr.fr_data.size + arr.lr_data.size


def test_golden_hmatrix_close_to_dense(golden):
    arr, ex = golden
    eps = float(ex["eps"])
    # the eta = 0 build is the dense product of the same kernel
    assert rel(ex["y_dense"], ex["y_dense_assembled"]) < 1e-13
    assert rel(ex["y_ref"], ex["y_dense"]) < 30 * eps
    assert rel(oracle_rmatvec(arr, ex["x"], 2), ex["yt_dense"]) < 30 * eps


def test_restatement_matmat_is_columnwise(golden):
    arr, ex = golden
    X = np.random.default_rng(5).standard_normal((arr.n_cols, 3))
    Y = oracle_matmat(arr, X, 2)
    for k in range(3):
        assert rel(Y[:, k], oracle_matvec(arr, X[:, k], 1)) < 1e-14


@needs_ref
def test_reference_known_answer_griffith():
    # 2DS0-H Griffith crack: diag ~ 190.985 and traction ~ 1 for the elliptical opening
    coor, conn = straight_crack_2d(1200)
    R = RefHmat("2DS0-H", coor, conn, [1.0, 0.0], 32, 2.0, 1e-3, n_threads=4)
    d = R.diagonal()
    assert np.mean(np.abs(d[1::2] - 190.985)) < 0.05
    xc = 0.5 * (coor[conn[:, 0], 0] + coor[conn[:, 1], 0])
    x = np.zeros(R.shape[1])
    x[1::2] = 4.0 * np.sqrt(1.0 - xc ** 2)
    y = R.matvec(x)
    assert np.mean(np.abs(y[1::2] - 1.0)) < 0.05
    arr = R.arrays()
    assert rel(oracle_matvec(arr, x, 2), y) < 1e-13


@needs_ref
@pytest.mark.parametrize("kind", ["2ds0", "3dr0"])
def test_restatement_matches_live_reference(kind):
    if kind == "2ds0":
        coor, conn = straight_crack_2d(700)
        R = RefHmat("2DS0-H", coor, conn, [1.0, 0.25], 32, 3.0, 1e-5, n_threads=4)
    else:
        coor, conn = square_crack_3d(14)
        R = RefHmat("3DR0-H", coor, conn, [1.0, 0.25], 16, 3.0, 1e-4, n_threads=4)
    arr = R.arrays()
    x = np.random.default_rng(11).uniform(-1, 1, R.shape[1])
    assert rel(oracle_matvec(arr, x, 4), R.matvec(x)) < 1e-13
    assert rel(oracle_matvec_perm(arr, x, 4), R.matvec_perm(x)) < 1e-13
    assert np.array_equal(oracle_diagonal(arr), R.diagonal())


@needs_ref
@pytest.mark.parametrize("kind", ["2ds0", "3dr0", "3dt0"])
def test_dense_rows_equal_eta0_build(kind):
    """ref_dense_rows (the exact kernel, evaluated as the reference's matrix
    generator does) against an eta = 0 build of the reference, whose blocks are
    all full rank: the same entries, bitwise."""
    from bigwham_dev_b200.meshes import penny_crack_3d

    if kind == "2ds0":
        coor, conn = straight_crack_2d(300)
        kern, props = "2DS0-H", [1.0, 0.25]
    elif kind == "3dr0":
        coor, conn = square_crack_3d(9)
        kern, props = "3DR0-H", [1.0, 0.25]
    else:
        coor, conn = penny_crack_3d(0.2, seed=2)
        kern, props = "3DT0-H", [1.0, 0.2]
    R = RefHmat(kern, coor, conn, props, 16, 0.0, 1e-4, n_threads=4)
    arr = R.arrays()
    assert arr.lr.shape[0] == 0
    D = np.zeros((arr.n_rows, arr.n_cols))
    for i0, j0, a in arr.fr_blocks():
        D[i0:i0 + a.shape[0], j0:j0 + a.shape[1]] = a
    d = arr.dof
    rp = (d * arr.perm0[:, None] + np.arange(d)[None, :]).ravel()
    cp = (d * arr.perm1[:, None] + np.arange(d)[None, :]).ravel()
    Do = np.zeros_like(D)
    Do[np.ix_(rp, cp)] = D
    pts = np.random.default_rng(0).choice(arr.n_rows // d, size=7, replace=False)
    rows = R.dense_rows(kern, props, pts)
    want = Do[(d * pts[:, None] + np.arange(d)[None, :]).ravel()]
    assert np.array_equal(rows, want)
