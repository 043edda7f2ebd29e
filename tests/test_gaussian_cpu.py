"""The reference's own H-matrix test over a synthetic kernel
(src/hmat/hmatrix/_test/Hmat_test_gaussian_mat.cpp:44-71): a Gaussian-matrix
H-matrix on n points of a line, built by the reference's cluster tree,
pattern, GaussianMatrix generator and Hmat (dof 1, ACA with 1 x 1 pivots).
Its assertion, the diagonal sums to n exactly, holds for this backend's
diagonal; the backend's plan for those blocks, replayed as the kernels walk
it, equals the reference's own Hmat::matvec."""
import numpy as np
import pytest
from conftest import rel
from planreplay import replay

from bigwham_dev_b200 import HmatGpu
from oracle import RefGaussian, oracle_matvec_perm, ref_available

pytestmark = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")


@pytest.fixture(scope="module", params=[(150, 10.0), (1000, 0.01)])
def gauss(request):
    n, alpha = request.param
    ref = RefGaussian(n, alpha, leaf=32, eta=3.0, eps=1e-3)
    arr = ref.arrays()
    h = HmatGpu(1, n, n, arr.perm0, arr.perm1, device=-1)
    h.add_flat(arr.fr, arr.lr, arr.fr_data, arr.lr_data)
    h.finalize(plan_only=True, precisions=("fp64", "fp32", "bf16"), transpose=True)
    return ref, arr, h


def test_diagonal_sums_to_n(gauss):
    ref, arr, h = gauss
    d_ref = ref.diagonal()
    assert d_ref.sum() == 1.0 * arr.n_rows  # the reference's own assertion
    d = h.diagonal(permuted=True)
    assert np.array_equal(d, d_ref) and d.sum() == 1.0 * arr.n_rows


def test_plan_replay_equals_the_reference_matvec(gauss):
    ref, arr, h = gauss
    x = np.random.default_rng(1).uniform(-1, 1, arr.n_cols)
    want = ref.matvec_perm(x)
    assert rel(oracle_matvec_perm(arr, x, 1), want) < 1e-14
    assert rel(replay(h, x, "fp64"), want) < 1e-14
    xf = x.astype(np.float32).astype(np.float64)
    assert rel(replay(h, xf, "fp32"), ref.matvec_perm(xf)) < 2e-6
    assert rel(replay(h, xf, "bf16"), ref.matvec_perm(xf)) < 8e-3
    # the Gaussian kernel is symmetric and so is its H-matrix pattern: H^T x = H x
    # up to the ACA error of the low-rank blocks
    assert rel(replay(h, x, "fp64", transposed=True), want) < 1e-2
    assert arr.lr.shape[0] > 0 and (arr.lr[:, 4] >= 1).all()
