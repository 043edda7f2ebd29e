"""HmatApply host logic on CPU with a dense stand-in operator (no GPU).

The stand-in has the same matvec signature as HmatGpu.  These tests check the
autograd wiring: the forward and backward directions, double backward,
several right-hand sides, dtype round trips, and that backward refuses a
handle without the transposed layout.
"""
import numpy as np
import pytest
import torch

from bigwham_dev_b200.autograd import HmatApply, TractionMisfit, hmatvec


class DenseOp:
    def __init__(self, M, has_transpose=True):
        self.M = M
        self.n_rows, self.n_cols = M.shape
        self.has_transpose = has_transpose
        self.calls = []

    def matvec(self, x, precision="fp64", transpose=False, permuted=False, out=None):
        self.calls.append((precision, transpose, permuted))
        y = (self.M.t() if transpose else self.M) @ x
        out.copy_(y)
        return out


def _op(m=7, n=5, seed=0, **kw):
    g = torch.Generator().manual_seed(seed)
    return DenseOp(torch.randn(m, n, generator=g, dtype=torch.float64), **kw)


def test_forward_and_transpose():
    op = _op()
    x = torch.randn(5, dtype=torch.float64)
    assert torch.allclose(hmatvec(x, op), op.M @ x)
    g = torch.randn(7, dtype=torch.float64)
    assert torch.allclose(hmatvec(g, op, transpose=True), op.M.t() @ g)


def test_gradcheck_and_gradgradcheck():
    op = _op()
    x = torch.randn(5, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda v: HmatApply.apply(v, op, "fp64", False, False), (x,))
    assert torch.autograd.gradgradcheck(lambda v: HmatApply.apply(v, op, "fp64", False, False), (x,))
    X = torch.randn(5, 3, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda v: HmatApply.apply(v, op, "fp64", False, False), (X,))


def test_backward_uses_transposed_kernel_and_precision():
    op = _op()
    x = torch.randn(5, dtype=torch.float64, requires_grad=True)
    y = hmatvec(x, op, precision="fp32", permuted=True)
    y.sum().backward()
    assert op.calls == [("fp32", False, True), ("fp32", True, True)]
    assert torch.allclose(x.grad, op.M.t() @ torch.ones(7, dtype=torch.float64))


def test_float32_input_keeps_dtype():
    op = _op()
    x = torch.randn(5, dtype=torch.float32, requires_grad=True)
    y = hmatvec(x, op)
    assert y.dtype == torch.float32
    y.sum().backward()
    assert x.grad.dtype == torch.float32


def test_backward_needs_transposed_layout():
    op = _op(has_transpose=False)
    x = torch.randn(5, dtype=torch.float64, requires_grad=True)
    y = hmatvec(x, op)
    with pytest.raises(RuntimeError, match="transposed layout"):
        y.sum().backward()


def test_shape_checked():
    with pytest.raises(ValueError):
        hmatvec(torch.zeros(6, dtype=torch.float64), _op())


def test_lbfgs_inverts_tractions():
    rng = np.random.default_rng(4)
    n = 40
    M = torch.from_numpy(np.eye(n) * 4 + rng.uniform(-1, 1, (n, n)) / np.sqrt(n))
    op = DenseOp(M)
    x_true = torch.from_numpy(rng.uniform(0, 1, n))
    loss_fn = TractionMisfit(op, M @ x_true)
    x = torch.zeros(n, dtype=torch.float64, requires_grad=True)
    opt = torch.optim.LBFGS([x], lr=1, max_iter=200, tolerance_grad=1e-14, tolerance_change=0,
                            history_size=20, line_search_fn="strong_wolfe")

    def closure():
        opt.zero_grad()
        loss = loss_fn(x)
        loss.backward()
        return loss

    opt.step(closure)
    assert float(torch.linalg.vector_norm(x.detach() - x_true) / torch.linalg.vector_norm(x_true)) < 1e-8
