"""Adjoint (transposed) H-matvec as a torch autograd backward (-m gpu).

Workload: 3DR0-H square crack n x n on [-1,1]^2 (n = 64: 12,288 DoF, n = 128:
49,152 DoF), E = 1, nu = 0.25, leaf 32, eta = 3, eps = 1e-5.  The field to
recover is x* = sqrt(max(0, 1 - r^2)) in the normal component of every element
(r: distance of the collocation point from the centre) plus N(0, 0.01^2)
noise (numpy default_rng(4)); the target tractions are t* = H x*.

Checks:
* the autograd gradient of <w, H x> (that is, H^T w) against the oracle's transposed
  product on the same blocks (FP64 1e-12, FP32 2e-6, BF16 8e-3);
* <H x, g> = <x, H^T g> at FP64 rounding;
* H^T g against the reference's dense FP64 matrix (an eta = 0 build: every block
  full rank) to 1e-6 on 64^2;
* the gradient of the misfit 1/2 ||H x - t*||^2 / ||t*||^2 against central finite
  differences (step 1e-6) along 32 random directions, to 1e-6;
* L-BFGS on that misfit recovers x* (misfit <= 1e-8, ||x - x*|| / ||x*|| <= 1e-3).
"""
import numpy as np
import pytest
from conftest import rel

from bigwham_dev_b200 import HmatGpu
from bigwham_dev_b200.autograd import TractionMisfit, hmatvec
from bigwham_dev_b200.meshes import square_crack_3d
from oracle import RefHmat, oracle_rmatvec

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 2e-6, "bf16": 8e-3}
PROPS, LEAF, ETA, EPS = [1.0, 0.25], 32, 3.0, 1e-5


class Crack:
    def __init__(self, n):
        self.coor, self.conn = square_crack_3d(n)
        R = RefHmat("3DR0-H", self.coor, self.conn, PROPS, LEAF, ETA, EPS, n_threads=16)
        self.arr = a = R.arrays()
        self.h = HmatGpu.from_flat(a.dof, a.n_rows, a.n_cols, a.fr, a.lr, a.fr_data, a.lr_data, a.perm0, a.perm1,
                                   device=0, precisions=("fp64", "fp32", "bf16"), transpose=True)
        cp = R.collocation_points().reshape(-1, 3)
        r = np.hypot(cp[:, 0], cp[:, 1])
        xs = np.zeros(a.n_rows)
        xs[2::3] = np.sqrt(np.maximum(0.0, 1.0 - r ** 2))
        xs += np.random.default_rng(4).normal(0.0, 0.01, a.n_rows)
        self.x_star = xs


_cracks = {}


@pytest.fixture(params=[64, 128], scope="module")
def crack(request):
    if request.param not in _cracks:
        _cracks[request.param] = Crack(request.param)
    return _cracks[request.param]


def _cuda(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("prec", ["fp64", "fp32", "bf16"])
def test_autograd_gradient_is_transposed_product(crack, prec):
    import torch

    rng = np.random.default_rng(7)
    w = rng.uniform(-1, 1, crack.arr.n_rows)
    x = _cuda(rng.uniform(-1, 1, crack.arr.n_cols)).requires_grad_()
    y = hmatvec(x, crack.h, prec)
    torch.dot(y, _cuda(w)).backward()
    assert rel(x.grad.cpu().numpy(), oracle_rmatvec(crack.arr, w, 16)) < TOL[prec]


def test_dot_product_identity(crack):
    import torch

    rng = np.random.default_rng(8)
    x = _cuda(rng.uniform(-1, 1, crack.arr.n_cols))
    g = _cuda(rng.uniform(-1, 1, crack.arr.n_rows))
    lhs = float(torch.dot(crack.h.matvec(x), g))
    rhs = float(torch.dot(x, crack.h.rmatvec(g)))
    scale = float(torch.linalg.vector_norm(crack.h.matvec(x)) * torch.linalg.vector_norm(g))
    assert abs(lhs - rhs) <= 1e-13 * scale


def test_adjoint_against_dense_reference():
    """H^T g against the reference's dense FP64 matrix: an eta = 0 build makes
    every block full rank, so its transposed product is the dense A^T g."""
    import torch

    c = _cracks.get(64) or Crack(64)
    _cracks[64] = c
    dense = RefHmat("3DR0-H", c.coor, c.conn, PROPS, LEAF, 0.0, EPS, n_threads=16).arrays()
    assert dense.lr.shape[0] == 0
    g = np.random.default_rng(5).uniform(-1, 1, c.arr.n_rows)
    x = _cuda(np.zeros(c.arr.n_cols)).requires_grad_()
    torch.dot(hmatvec(x, c.h), _cuda(g)).backward()
    assert rel(x.grad.cpu().numpy(), oracle_rmatvec(dense, g, 16)) <= 1e-6


def test_misfit_gradient_against_finite_differences(crack):
    import torch

    loss_fn = TractionMisfit(crack.h, crack.h.matvec(_cuda(crack.x_star)))
    rng = np.random.default_rng(9)
    x0 = _cuda(crack.x_star + rng.normal(0.0, 0.1, crack.arr.n_cols))
    x = x0.clone().requires_grad_()
    loss_fn(x).backward()
    grad = x.grad.detach()
    step = 1e-6
    fd, ad = [], []
    with torch.no_grad():
        for _ in range(32):
            d = _cuda(rng.normal(0.0, 1.0, crack.arr.n_cols))
            d /= torch.linalg.vector_norm(d)
            fd.append((float(loss_fn(x0 + step * d)) - float(loss_fn(x0 - step * d))) / (2 * step))
            ad.append(float(torch.dot(grad, d)))
    assert rel(fd, ad) <= 1e-6


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_lbfgs_recovers_opening(prec):
    import torch

    c = _cracks.get(64) or Crack(64)
    _cracks[64] = c
    xs = _cuda(c.x_star)
    loss_fn = TractionMisfit(c.h, c.h.matvec(xs), precision=prec)
    x = torch.zeros_like(xs, requires_grad=True)
    opt = torch.optim.LBFGS([x], lr=1, max_iter=400, tolerance_grad=1e-20, tolerance_change=0, history_size=20,
                            line_search_fn="strong_wolfe")

    def closure():
        opt.zero_grad()
        loss = loss_fn(x)
        loss.backward()
        return loss

    opt.step(closure)
    with torch.no_grad():
        assert float(loss_fn(x)) <= 1e-8
        assert float(torch.linalg.vector_norm(x - xs) / torch.linalg.vector_norm(xs)) <= 1e-3
