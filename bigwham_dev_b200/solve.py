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
* ``MultiGmres`` / ``refine_multi``: k systems at once, each with its own
  Krylov space and stopping test, sharing one operator call per Arnoldi step:
  the 64-right-hand-side tensor-core matmat (one H-matrix, k right-hand
  sides), or one batched H-matrix (k independent H-matrices of uneven size,
  vectors padded to a common length; ``BatchOperator``).  Each restart cycle
  is one replayed CUDA graph, as in ``Gmres``.
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
    diverged: bool = False       # refinement stopped: the residual grew (see refine)


# Relative size of an Arnoldi residual, against the operator output it was
# taken from, below which the Krylov space counts as exhausted (breakdown).
_BREAKDOWN = 1e-12


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
            w0 = self.torch.linalg.vector_norm(w)
            Vj = V[:j + 1]
            h = Vj @ w
            w.sub_(Vj.t() @ h)
            h2 = Vj @ w
            w.sub_(Vj.t() @ h2)
            H[:j + 1, j] = h + h2
            nrm = self.torch.linalg.vector_norm(w)
            # breakdown (see MultiGmres._cycle): zero vectors from here on
            live = nrm > _BREAKDOWN * w0
            nrm = self.torch.where(live, nrm, self.torch.zeros_like(nrm))
            H[j + 1, j] = nrm
            self.torch.div(w, self.torch.where(live, nrm, self.torch.ones_like(nrm)), out=V[j + 1])
            V[j + 1].mul_(live.to(V.dtype))

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


# Refinement contracts the residual by about cond(A) x (the low precision's
# relative error) per step.  Where that product exceeds one (an ill-conditioned
# system with BF16 blocks) the residual grows instead; a system whose residual
# exceeds _DIVERGED x its best so far is stopped at its best iterate and
# reported as diverged (SolveInfo.diverged) rather than iterated to overflow.
_DIVERGED = 10.0


def refine(op_hi, op_lo, b, n: int, minv=None, tol: float = 1e-8, inner_tol: float = 1e-3, restart: int = 50,
           max_outer: int = 50, use_graph: bool = True):
    """Mixed-precision iterative refinement: x += GMRES_lo(A d = b - A_hi x).
    Stops at the best iterate, with info.diverged set, when the residual
    grows (see _DIVERGED)."""
    import torch

    info = SolveInfo()
    inner = Gmres(op_lo, n, restart, minv, device=b.device, use_graph=use_graph)
    x = torch.zeros_like(b)
    r = torch.empty_like(b)
    best, x_best = np.inf, x.clone()
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
        if not np.isfinite(rel) or rel > _DIVERGED * best:
            info.diverged = True
            x.copy_(x_best)
            break
        if rel < best:
            best = rel
            x_best.copy_(x)
        d, inf = inner.solve(r, tol=inner_tol, maxiter=20 * restart)
        info.iterations += inf.iterations
        info.cycles += inf.cycles
        x.add_(d)
    return x, info


class MultiGmres:
    """Restarted GMRES(m) for k systems op(X) = B at once.

    Vectors are (k, n) CUDA float64 tensors, one system per row (row-major,
    i.e. the column-major n x k layout of a matmat).  op(Z, W) writes the k
    operator applications of Z's rows into W's rows, stream-ordered on the
    current torch stream.  Every system keeps its own Arnoldi basis, FP64
    Hessenberg matrix (classical Gram-Schmidt, two passes) and stopping test;
    a system whose residual is zero contributes zero vectors.  minv: optional
    right preconditioner, a (k, n) or (n,) tensor applied elementwise.
    """

    def __init__(self, op, k: int, n: int, restart: int = 50, minv=None, device="cuda", use_graph: bool = True):
        import torch

        self.torch = torch
        self.op, self.k, self.n, self.m = op, int(k), int(n), int(restart)
        self.minv = minv
        dt = torch.float64
        self.V = torch.zeros(self.m + 1, self.k, self.n, dtype=dt, device=device)
        self.H = torch.zeros(self.k, self.m + 1, self.m, dtype=dt, device=device)
        self.Z = torch.zeros(self.k, self.n, dtype=dt, device=device)
        self.W = torch.zeros(self.k, self.n, dtype=dt, device=device)
        self.use_graph = use_graph
        self.graph = None

    def _precondition(self, v, out):
        if self.minv is None:
            out.copy_(v)
        else:
            self.torch.mul(v, self.minv, out=out)

    def _cycle(self):
        torch = self.torch
        V, H, Z, W = self.V, self.H, self.Z, self.W
        for j in range(self.m):
            self._precondition(V[j], Z)
            self.op(Z, W)
            w0 = torch.linalg.vector_norm(W, dim=1)         # (k,)
            Vj = V[:j + 1].transpose(0, 1)                  # (k, j+1, n)
            h = torch.bmm(Vj, W.unsqueeze(2))               # (k, j+1, 1)
            W.sub_(torch.bmm(Vj.transpose(1, 2), h).squeeze(2))
            h2 = torch.bmm(Vj, W.unsqueeze(2))
            W.sub_(torch.bmm(Vj.transpose(1, 2), h2).squeeze(2))
            H[:, :j + 1, j] = (h + h2).squeeze(2)
            nrm = torch.linalg.vector_norm(W, dim=1)        # (k,)
            # Breakdown: the system's Krylov space is exhausted (what is left
            # of W is rounding).  It continues with zero vectors and a zero
            # subdiagonal, where its least-squares problem stops.
            live = nrm > _BREAKDOWN * w0
            nrm = torch.where(live, nrm, torch.zeros_like(nrm))
            H[:, j + 1, j] = nrm
            safe = torch.where(live, nrm, torch.ones_like(nrm))
            torch.div(W, safe.unsqueeze(1), out=V[j + 1])
            V[j + 1].mul_(live.unsqueeze(1).to(V.dtype))

    def _run_cycle(self):
        torch = self.torch
        if not self.use_graph:
            self._cycle()
            return
        if self.graph is None:
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

    def solve(self, B, tol: float = 1e-8, maxiter: int = 2000):
        """Solve op(X) = B row by row to ||b_i - op(x_i)|| <= tol ||b_i||.
        Returns (X, info) with info.converged true when every system met the
        tolerance, and info.per_system the SolveInfo of each system."""
        torch = self.torch
        k = self.k
        X = torch.zeros_like(B)
        R = torch.empty_like(B)
        bn = torch.linalg.vector_norm(B, dim=1).cpu().numpy()
        infos = [SolveInfo() for _ in range(k)]
        done = bn == 0.0
        for i in np.nonzero(done)[0]:
            infos[i].converged = True
        total = SolveInfo()
        while not done.all() and total.iterations < maxiter:
            if total.iterations == 0:
                R.copy_(B)
            else:
                self.op(X, R)
                torch.sub(B, R, out=R)
            beta = torch.linalg.vector_norm(R, dim=1).cpu().numpy()
            for i in range(k):
                if not done[i]:
                    infos[i].residuals.append(beta[i] / bn[i])
                    if beta[i] <= tol * bn[i]:
                        done[i], infos[i].converged = True, True
            if done.all():
                break
            scale = torch.from_numpy(np.where(done | (beta == 0.0), 0.0, 1.0 / np.where(beta == 0.0, 1.0, beta)))
            torch.mul(R, scale.to(R.device).unsqueeze(1), out=self.V[0])
            self._run_cycle()
            total.cycles += 1
            total.iterations += self.m
            Hh = self.H.cpu().numpy()
            Y = np.zeros((k, self.m))
            for i in range(k):
                if done[i]:
                    continue
                kk, y, res = _lstsq_prefix(Hh[i], float(beta[i]), tol * bn[i])
                Y[i, :kk] = y
                infos[i].iterations += self.m
                infos[i].cycles += 1
            upd = torch.einsum("jkn,kj->kn", self.V[:self.m], torch.from_numpy(Y).to(B.device))
            self._precondition(upd, self.Z)
            X.add_(self.Z)
        total.converged = bool(done.all())
        total.per_system = infos
        return X, total


class BatchOperator:
    """The block-diagonal operator of a batched handle (HmatGpu.batch) on the
    padded (count, L) layout of MultiGmres: member k's vector is row k, and
    the entries beyond its length are ignored on input and zero on output."""

    def __init__(self, hb, precision: str = "fp64", device="cuda"):
        import torch

        self.hb, self.precision = hb, precision
        ro, co = np.asarray(hb.row_offsets), np.asarray(hb.col_offsets)
        if not np.array_equal(ro, co):
            raise ValueError("BatchOperator needs square members")
        self.count = len(ro) - 1
        sizes = np.diff(ro)
        self.L = int(sizes.max()) if self.count else 0
        idx = np.concatenate([k * self.L + np.arange(sizes[k]) for k in range(self.count)]).astype(np.int64)
        self.idx = torch.from_numpy(idx).to(device)
        self.x = torch.zeros(int(ro[-1]), dtype=torch.float64, device=device)
        self.y = torch.zeros(int(ro[-1]), dtype=torch.float64, device=device)

    def pad(self, v):
        """(count, L) padded form of a concatenated vector."""
        import torch

        out = torch.zeros(self.count, self.L, dtype=torch.float64, device=v.device)
        out.view(-1).index_copy_(0, self.idx, v)
        return out

    def unpad(self, V):
        return V.reshape(-1).index_select(0, self.idx)

    def __call__(self, Z, W):
        import torch

        torch.index_select(Z.reshape(-1), 0, self.idx, out=self.x)
        self.hb.matvec(self.x, self.precision, out=self.y)
        W.zero_()  # the padding of an output buffer may hold anything
        W.view(-1).index_copy_(0, self.idx, self.y)


def refine_multi(op_hi, op_lo, B, minv=None, tol: float = 1e-8, inner_tol: float = 1e-3, restart: int = 50,
                 max_outer: int = 50, use_graph: bool = True):
    """Mixed-precision iterative refinement of k systems (rows of B):
    X += MultiGmres_lo(A D = B - A_hi X), until every row's relative residual
    is <= tol.  op_hi, op_lo: (Z, W) operators on (k, n) tensors.  A row whose
    residual grows (see _DIVERGED) is stopped at its best iterate;
    info.per_system[i] tells converged / diverged, info.converged is true when
    every row converged."""
    import torch

    k, n = B.shape
    info = SolveInfo()
    per = [SolveInfo() for _ in range(k)]
    inner = MultiGmres(op_lo, k, n, restart, minv, device=B.device, use_graph=use_graph)
    X = torch.zeros_like(B)
    R = torch.empty_like(B)
    X_best = torch.zeros_like(B)
    best = np.full(k, np.inf)
    active = np.ones(k, dtype=bool)
    bn = torch.linalg.vector_norm(B, dim=1)
    bn = torch.where(bn > 0, bn, torch.ones_like(bn))
    for it in range(max_outer):
        op_hi(X, R)
        torch.sub(B, R, out=R)
        rel = (torch.linalg.vector_norm(R, dim=1) / bn).cpu().numpy()
        info.outer = it
        for i in np.nonzero(active)[0]:
            per[i].residuals.append(float(rel[i]))
            per[i].outer = it
            if rel[i] <= tol:
                per[i].converged, active[i] = True, False
            elif not np.isfinite(rel[i]) or rel[i] > _DIVERGED * best[i]:
                per[i].diverged, active[i] = True, False
                X[i].copy_(X_best[i])
            elif rel[i] < best[i]:
                best[i] = rel[i]
                X_best[i].copy_(X[i])
        info.residuals.append(float(max((per[i].residuals[-1] for i in range(k) if per[i].residuals), default=0.0)))
        if not active.any():
            break
        # finished rows get a zero right-hand side: the inner solve leaves them alone
        R.mul_(torch.from_numpy(active.astype(np.float64)).to(R.device).unsqueeze(1))
        D, inf = inner.solve(R, tol=inner_tol, maxiter=20 * restart)
        info.iterations += inf.iterations
        info.cycles += inf.cycles
        X.add_(D)
    info.converged = all(p.converged for p in per)
    info.diverged = any(p.diverged for p in per)
    info.per_system = per
    return X, info
