"""GMRES / iterative refinement logic on CPU tensors (no graph capture)."""
import numpy as np
import pytest
import torch

from bigwham_dev_b200.solve import Gmres, refine


def _system(n=300, seed=0):
    rng = np.random.default_rng(seed)
    A = np.eye(n) * 4 + rng.standard_normal((n, n)) / np.sqrt(n)
    return torch.from_numpy(A), torch.from_numpy(rng.standard_normal(n))


def test_gmres_converges_with_restarts_and_jacobi():
    A, b = _system()
    op = lambda x, y: y.copy_(A @ x)  # noqa: E731
    minv = 1.0 / torch.diagonal(A)
    g = Gmres(op, A.shape[0], restart=10, minv=minv, device="cpu", use_graph=False)
    x, info = g.solve(b, tol=1e-10, maxiter=500)
    assert info.converged and info.cycles >= 1
    assert float(torch.linalg.vector_norm(b - A @ x) / torch.linalg.vector_norm(b)) < 1e-9


def test_refine_recovers_high_precision_from_perturbed_operator():
    A, b = _system(seed=1)
    E = torch.from_numpy(np.random.default_rng(2).standard_normal(A.shape)) * 1e-3 / np.sqrt(A.shape[0])
    op_hi = lambda x, y: y.copy_(A @ x)  # noqa: E731
    op_lo = lambda x, y: y.copy_((A + E) @ x)  # noqa: E731  (a 1e-3 "low-precision" operator)
    x, info = refine(op_hi, op_lo, b, A.shape[0], tol=1e-12, inner_tol=1e-3, restart=20, use_graph=False)
    assert info.converged and info.outer >= 2
    x_true = torch.linalg.solve(A, b)
    assert float(torch.linalg.vector_norm(x - x_true) / torch.linalg.vector_norm(x_true)) < 1e-10


def test_zero_rhs():
    A, _ = _system(50)
    g = Gmres(lambda x, y: y.copy_(A @ x), 50, restart=5, device="cpu", use_graph=False)
    x, info = g.solve(torch.zeros(50, dtype=torch.float64))
    assert info.converged and float(x.abs().max()) == 0.0
