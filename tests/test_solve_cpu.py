"""GMRES / iterative refinement logic on CPU tensors (no graph capture)."""
import numpy as np
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


def _systems(k=5, n=120, seed=3):
    rng = np.random.default_rng(seed)
    As = [np.eye(n) * (3 + i) + rng.standard_normal((n, n)) / np.sqrt(n) for i in range(k)]
    return torch.from_numpy(np.stack(As)), torch.from_numpy(rng.standard_normal((k, n)))


def test_multi_gmres_solves_each_system_with_its_own_krylov_space():
    from bigwham_dev_b200.solve import MultiGmres

    A, B = _systems()
    B[2] = 0.0  # a zero right-hand side: converged from the start, stays zero
    op = lambda Z, W: W.copy_(torch.bmm(A, Z.unsqueeze(2)).squeeze(2))  # noqa: E731
    minv = 1.0 / torch.diagonal(A, dim1=1, dim2=2)
    X, info = MultiGmres(op, A.shape[0], A.shape[1], restart=8, minv=minv, device="cpu",
                         use_graph=False).solve(B, tol=1e-11, maxiter=800)
    assert info.converged and all(s.converged for s in info.per_system)
    for i in range(A.shape[0]):
        xt = torch.linalg.solve(A[i], B[i])
        assert float(torch.linalg.vector_norm(X[i] - xt)) <= 1e-9 * max(1.0, float(torch.linalg.vector_norm(xt)))
    assert float(X[2].abs().max()) == 0.0
    # the same systems one at a time: the same Krylov spaces, the same answer
    for i in (0, 4):
        g = Gmres(lambda x, y, i=i: y.copy_(A[i] @ x), A.shape[1], restart=8, minv=minv[i], device="cpu",
                  use_graph=False)
        x1, _ = g.solve(B[i], tol=1e-11, maxiter=800)
        assert float(torch.linalg.vector_norm(x1 - X[i])) <= 1e-9 * float(torch.linalg.vector_norm(x1))


def test_refine_multi_recovers_high_precision():
    from bigwham_dev_b200.solve import refine_multi

    A, B = _systems(k=4, seed=5)
    E = torch.from_numpy(np.random.default_rng(6).standard_normal(A.shape)) * 1e-3 / np.sqrt(A.shape[1])
    op_hi = lambda Z, W: W.copy_(torch.bmm(A, Z.unsqueeze(2)).squeeze(2))  # noqa: E731
    op_lo = lambda Z, W: W.copy_(torch.bmm(A + E, Z.unsqueeze(2)).squeeze(2))  # noqa: E731
    X, info = refine_multi(op_hi, op_lo, B, tol=1e-12, inner_tol=1e-3, restart=15, use_graph=False)
    assert info.converged and info.outer >= 2
    for i in range(A.shape[0]):
        xt = torch.linalg.solve(A[i], B[i])
        assert float(torch.linalg.vector_norm(X[i] - xt) / torch.linalg.vector_norm(xt)) < 1e-10


def test_batch_operator_pads_members_and_keeps_padding_zero():
    """BatchOperator on a stand-in batched handle (block-diagonal dense
    members of uneven size, concatenated vectors)."""
    from types import SimpleNamespace

    from bigwham_dev_b200.solve import BatchOperator, MultiGmres

    rng = np.random.default_rng(7)
    sizes = [7, 30, 1, 18]
    mats = [np.eye(s) * 5 + rng.standard_normal((s, s)) / np.sqrt(s) for s in sizes]
    off = np.concatenate([[0], np.cumsum(sizes)])
    D = np.zeros((off[-1], off[-1]))
    for k, M in enumerate(mats):
        D[off[k]:off[k + 1], off[k]:off[k + 1]] = M
    Dt = torch.from_numpy(D)
    hb = SimpleNamespace(row_offsets=off, col_offsets=off,
                         matvec=lambda x, p, out: out.copy_(Dt @ x))
    op = BatchOperator(hb, "fp64", device="cpu")
    assert (op.count, op.L) == (4, 30)
    b = torch.from_numpy(rng.standard_normal(off[-1]))
    Bp = op.pad(b)
    assert torch.equal(op.unpad(Bp), b)
    W = torch.zeros_like(Bp)
    op(Bp, W)
    assert torch.allclose(op.unpad(W), Dt @ b)
    mask = torch.ones_like(Bp, dtype=torch.bool)
    mask.view(-1)[op.idx] = False
    assert float(W[mask].abs().max()) == 0.0
    X, info = MultiGmres(op, op.count, op.L, restart=10, device="cpu", use_graph=False).solve(Bp, tol=1e-12)
    assert info.converged
    assert float(torch.linalg.vector_norm(Dt @ op.unpad(X) - b) / torch.linalg.vector_norm(b)) < 1e-11
    assert float(X[mask].abs().max()) == 0.0


def test_refine_multi_over_a_batch_with_tiny_members():
    """Members of 1 and 3 unknowns exhaust their Krylov spaces within a
    50-step cycle (breakdown: they continue with zero vectors), and output
    buffers whose padding holds garbage (torch.empty) are zeroed by the batch
    operator: every member converges, repeatably."""
    from types import SimpleNamespace

    from bigwham_dev_b200.solve import BatchOperator, refine_multi

    rng = np.random.default_rng(7)
    sizes = [8, 30, 1, 18, 60, 100, 3]
    mats = [np.eye(s) * 5 + rng.standard_normal((s, s)) / np.sqrt(s) for s in sizes]
    off = np.concatenate([[0], np.cumsum(sizes)])
    D = np.zeros((off[-1], off[-1]))
    for k, M in enumerate(mats):
        D[off[k]:off[k + 1], off[k]:off[k + 1]] = M
    Dt = torch.from_numpy(D)
    E = torch.from_numpy(rng.standard_normal(D.shape) * 1e-3) * (Dt != 0)
    hb = SimpleNamespace(row_offsets=off, col_offsets=off,
                         matvec=lambda x, p, out: out.copy_((Dt if p == "fp64" else Dt + E) @ x))
    op64, op_lo = BatchOperator(hb, "fp64", device="cpu"), BatchOperator(hb, "lo", device="cpu")
    b = torch.ones(off[-1], dtype=torch.float64)
    B = op64.pad(b)
    minv = op64.pad(1.0 / torch.diagonal(Dt))
    for _ in range(3):
        X, info = refine_multi(op64, op_lo, B, minv=minv, tol=1e-10, inner_tol=1e-3, restart=50, use_graph=False)
        assert info.converged and info.residuals[0] == 1.0, info.residuals[:4]
        x = op64.unpad(X)
        assert float(torch.linalg.vector_norm(Dt @ x - b) / torch.linalg.vector_norm(b)) <= 1e-10


def test_refinement_stops_when_the_low_precision_operator_is_too_coarse():
    """Refinement contracts by ~cond(A) x (low-precision error) per step; with
    cond 1e5 and a 1e-3 perturbation the residual grows.  The solver stops at
    its best iterate and reports the divergence (no overflow); in the batched
    form only that system stops, the well-conditioned one converges."""
    from bigwham_dev_b200.solve import refine, refine_multi

    rng = np.random.default_rng(11)
    n = 60
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A_bad = torch.from_numpy(Q @ np.diag(np.logspace(0, -5, n)) @ Q.T)
    A_good = torch.from_numpy(np.eye(n) * 3 + rng.standard_normal((n, n)) / np.sqrt(n))
    E = torch.from_numpy(rng.standard_normal((n, n))) * 1e-3 / np.sqrt(n)
    b = torch.from_numpy(rng.standard_normal(n))
    x, info = refine(lambda v, w: w.copy_(A_bad @ v), lambda v, w: w.copy_((A_bad + E) @ v), b, n, tol=1e-12,
                     inner_tol=1e-6, restart=n, use_graph=False)
    assert info.diverged and not info.converged and bool(torch.isfinite(x).all())
    assert float(torch.linalg.vector_norm(b - A_bad @ x) / torch.linalg.vector_norm(b)) <= 1.0
    A2, B = torch.stack([A_good, A_bad]), torch.stack([b, b])
    E2 = torch.stack([E, E])
    X, info = refine_multi(lambda Z, W: W.copy_(torch.bmm(A2, Z.unsqueeze(2)).squeeze(2)),
                           lambda Z, W: W.copy_(torch.bmm(A2 + E2, Z.unsqueeze(2)).squeeze(2)), B, tol=1e-12,
                           inner_tol=1e-6, restart=n, use_graph=False)
    assert info.per_system[0].converged and info.per_system[1].diverged and not info.converged
    assert bool(torch.isfinite(X).all())
    assert float(torch.linalg.vector_norm(b - A_good @ X[0]) / torch.linalg.vector_norm(b)) <= 1e-12
