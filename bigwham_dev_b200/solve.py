"""GMRES and mixed-precision iterative refinement on the GPU.

The reference has no solver of its own: users hand its scipy LinearOperator
(interfaces/python/bigwham4py/bigwham4py.py:49) to scipy's GMRES with the
Jacobi preconditioner of ``BEMatrix.H_jacobi_prec`` (bigwham4py.py:373-380).
Here the whole loop stays on the device:

* ``gmres``: right-preconditioned restarted GMRES.  The Arnoldi basis, the
  Hessenberg matrix and the classical Gram-Schmidt with re-orthogonalisation
  (two passes) are FP64; the operator can be any precision of the H-matvec.
  Each restart cycle (``restart`` Arnoldi steps) is captured once in a CUDA
  graph and replayed; only the small (restart+1) x restart least-squares
  problem goes to the host between cycles.
* ``refine``: iterative refinement.  The residual b - A x and the solution
  update use the FP64 H-matrix; the correction equation A d = r is solved by
  ``gmres`` with the FP32 or BF16 H-matrix (mixed precision), to a loose
  inner tolerance.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class SolveInfo:
    converged: bool = False
    iterations: int = 0          # Arnoldi steps (inner matvecs)
    cycles: int = 0              # restart cycles
    outer: int = 0               # refinement steps (refine only)
    residuals: list = field(default_factory=list)  # relative residual estimates per cycle / outer step


def _lstsq_prefix(Hh: np.ndarray, beta: float, tol_abs: float):
    """Smallest k with ||beta e1 - H[:k+1,:k] y|| <= tol_abs (or k = m) and its y."""
    m = Hh.shape[1]
    best = None
    for k in range(1, m + 1):
        Hk = Hh[:k + 1, :k]
        rhs = np.zeros(k + 1)
        rhs[0] = beta
        y, *_ = np.linalg.lstsq(Hk, rhs, rcond=None)
        res = float(np.linalg.norm(rhs - Hk @ y))
        best = (k, y, res)
        if res <= tol_abs or not np.isfinite(Hh[k, k - 1]) or Hh[k, k - 1] == 0.0:
            break
    return best


class Gmres:
    """Restarted GMRES(m) for y = op(x) on CUDA float64 vectors of length n.

    op(x, y): writes op applied to x into y (both CUDA float64, length n),
    stream-ordered on the current torch stream; called at capture time.
    minv: optional right preconditioner M^-1: a CUDA float64 vector (Jacobi,
    diag^-1, applied elementwise) or a callable minv(x, out) with op's
    conventions (e.g. precond.BlockJacobi).
    """

    def __init__(self, op, n: int, restart: int = 50, minv=None, device="cuda", use_graph: bool = True):
        import torch

        self.torch = torch
        self.op, self.n, self.m = op, int(n), int(restart)
        self.minv = minv
        dt = torch.float64
        self.V = torch.zeros(self.m + 1, self.n, dtype=dt, device=device)
        self.H = torch.zeros(self.m + 1, self.m, dtype=dt, device=device)
        self.z = torch.zeros(self.n, dtype=dt, device=device)
        self.w = torch.zeros(self.n, dtype=dt, device=device)
        self.use_graph = use_graph
        self.graph = None

    def _cycle(self):
        """m Arnoldi steps from V[0]; fills V and H (FP64)."""
        V, H, z, w = self.V, self.H, self.z, self.w
        for j in range(self.m):
            self._precondition(V[j], z)
            self.op(z, w)
            Vj = V[:j + 1]
            h = Vj @ w
            w.sub_(Vj.t() @ h)
            h2 = Vj @ w
            w.sub_(Vj.t() @ h2)
            H[:j + 1, j] = h + h2
            nrm = self.torch.linalg.vector_norm(w)
            H[j + 1, j] = nrm
            self.torch.div(w, nrm, out=V[j + 1])

    def _precondition(self, v, out):
        if self.minv is None:
            out.copy_(v)
        elif callable(self.minv):
            self.minv(v, out)
        else:
            self.torch.mul(v, self.minv, out=out)

    def _run_cycle(self):
        torch = self.torch
        if not self.use_graph:
            self._cycle()
            return
        if self.graph is None:
            # warm the operator (kernel attributes, lazy set-up) outside capture
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                self._cycle()
            torch.cuda.current_stream().wait_stream(s)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._cycle()
            self.graph = g
        self.graph.replay()

    def solve(self, b, x0=None, tol: float = 1e-8, maxiter: int = 2000, residual_op=None):
        """Solve op(x) = b to ||b - op(x)|| <= tol ||b||.  residual_op (default
        op) computes the true residual at each restart."""
        torch = self.torch
        info = SolveInfo()
        x = torch.zeros_like(b) if x0 is None else x0.clone()
        rop = residual_op or self.op
        bnorm = float(torch.linalg.vector_norm(b))
        if bnorm == 0.0:
            info.converged = True
            return x, info
        r = torch.empty_like(b)
        while info.iterations < maxiter:
            if info.iterations == 0 and x0 is None:
                r.copy_(b)
            else:
                rop(x, r)
                torch.sub(b, r, out=r)
            beta = float(torch.linalg.vector_norm(r))
            info.residuals.append(beta / bnorm)
            if beta <= tol * bnorm:
                info.converged = True
                break
            torch.div(r, beta, out=self.V[0])
            self._run_cycle()
            info.cycles += 1
            Hh = self.H.cpu().numpy()
            k, y, res = _lstsq_prefix(Hh, beta, tol * bnorm)
            info.iterations += self.m
            yt = torch.from_numpy(y).to(b.device)
            upd = self.V[:k].t() @ yt
            self._precondition(upd, self.z)
            x.add_(self.z)
            if res <= tol * bnorm and residual_op is None:
                info.residuals.append(res / bnorm)
                info.converged = True
                break
        return x, info


def refine(op_hi, op_lo, b, n: int, minv=None, tol: float = 1e-8, inner_tol: float = 1e-3, restart: int = 50,
           max_outer: int = 50, use_graph: bool = True):
    """Mixed-precision iterative refinement: x += GMRES_lo(A d = b - A_hi x)."""
    import torch

    info = SolveInfo()
    inner = Gmres(op_lo, n, restart, minv, device=b.device, use_graph=use_graph)
    x = torch.zeros_like(b)
    r = torch.empty_like(b)
    bnorm = float(torch.linalg.vector_norm(b))
    for it in range(max_outer):
        op_hi(x, r)
        torch.sub(b, r, out=r)
        rel = float(torch.linalg.vector_norm(r)) / bnorm
        info.residuals.append(rel)
        info.outer = it
        if rel <= tol:
            info.converged = True
            break
        d, inf = inner.solve(r, tol=inner_tol, maxiter=20 * restart)
        info.iterations += inf.iterations
        info.cycles += inf.cycles
        x.add_(d)
    return x, info
