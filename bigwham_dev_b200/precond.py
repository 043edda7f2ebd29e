"""Preconditioners built from the H-matrix's full-rank blocks, applied on the GPU.

The reference's Python API has two, both applied on the host by scipy:
* point Jacobi, ``BEMatrix.H_jacobi_prec``
  (interfaces/python/bigwham4py/bigwham4py.py:373-380), the inverse of
  ``H_diag`` (:362-371);
* an incomplete LU of all full-rank blocks, ``H_ILU_prec`` (:345-360, scipy
  ``spilu`` over ``_getFullBlocks`` :252-276), which it cannot build once the
  blocks live on the GPU.

``BlockJacobi`` is the GPU preconditioner here.  It is
M^-1 = blockdiag(D_1^-1, ..., D_K^-1), D_k the diagonal full-rank blocks.
* D_k is a leaf cluster's self-interaction.  It is always inadmissible, hence
  full rank, and in the clustered ordering these blocks tile the diagonal.
* The inverses come from an FP64 LU on the host, once.
* They are the members of one batched handle (bw_create_batch, one member per
  block).  Applying M^-1 is one batched product: the launches of a
  matvec, over sum_k m_k^2 entries.  For 3DR0-H 256 x 256 (196,608 DoF) that
  is 151 MB in FP64, 1.3% of the H-matrix.
* It is stream-ordered and allocation-free after the first call, so
  ``solve.Gmres`` captures it in its CUDA graph like the operator.

Orderings: H_orig = P0^T H_perm P1, where P1 gathers x through permutation_1_
and P0^T scatters y through permutation_0_ (hmat.cc:572-635).  So
M_orig^-1 = P1^T M_perm^-1 P0: the input is gathered through permutation_0_
and the output scattered through permutation_1_.
"""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from .hmat import HmatGpu


def diagonal_blocks(ex) -> list:
    """Indices of the diagonal full-rank blocks of the flat form `ex`, in
    clustered order.  ValueError unless they tile the diagonal."""
    d = int(ex["dof"])
    if int(ex["n_rows"]) != int(ex["n_cols"]):
        raise ValueError("block Jacobi needs a square H-matrix")
    fr = np.asarray(ex["fr"], dtype=np.int64).reshape(-1, 4)
    diag = np.flatnonzero((fr[:, 0] == fr[:, 1]) & (fr[:, 2] == fr[:, 3]))
    diag = diag[np.argsort(fr[diag, 0], kind="stable")]
    if (len(diag) == 0 or fr[diag[0], 0] != 0 or fr[diag[-1], 2] * d != int(ex["n_rows"])
            or np.any(fr[diag[1:], 0] != fr[diag[:-1], 2])):
        raise ValueError("the diagonal full-rank blocks do not tile the diagonal")
    return [int(k) for k in diag]


def inverted_blocks(ex, diag) -> list:
    """(start row, D_k^-1) per diagonal block, in the clustered ordering (FP64,
    LU with partial pivoting).  numpy.linalg.LinAlgError if a D_k is singular."""
    d = int(ex["dof"])
    fr = np.asarray(ex["fr"], dtype=np.int64).reshape(-1, 4)
    sizes = (fr[:, 2] - fr[:, 0]) * (fr[:, 3] - fr[:, 1]) * d * d
    off = np.concatenate([[0], np.cumsum(sizes)])
    fd = np.asarray(ex["fr_data"], dtype=np.float64)
    out = []
    for k in diag:
        m = int(fr[k, 2] - fr[k, 0]) * d
        D = fd[off[k]:off[k] + m * m].reshape(m, m, order="F")
        out.append((int(fr[k, 0]) * d, np.linalg.inv(D)))
    return out


class BlockJacobi:
    """M^-1 from the diagonal full-rank blocks, on one GPU.

    ex: the flat form of the H-matrix (BigWhamIOGpu.export_blocks,
    blockfile.read).  precision: storage of the inverses ("fp64", "fp32",
    "bf16").  ordering: "original" (vectors in the mesh's dof ordering, as
    HmatGpu.matvec) or "permuted" (clustered, as matvec(permuted=True)).
    device -1 with plan_only=True builds the host plan only.

    Call as ``M(x, out)``.  x and out are CUDA float64 tensors, or numpy
    arrays for the host path.
    """

    def __init__(self, ex, device: int = 0, precision: str = "fp64", ordering: str = "original",
                 plan_only: bool = False):
        if ordering not in ("original", "permuted"):
            raise ValueError("ordering is 'original' or 'permuted'")
        d = int(ex["dof"])
        self.n, self.dof, self.precision, self.ordering = int(ex["n_rows"]), d, precision, ordering
        diag = diagonal_blocks(ex)
        blocks = inverted_blocks(ex, diag)
        members = []
        for _, Dinv in blocks:
            m = Dinv.shape[0]
            members.append(SimpleNamespace(dof=d, n_rows=m, n_cols=m, fr=np.array([[0, 0, m // d, m // d]]),
                                           lr=np.zeros((0, 5), np.int64), fr_data=Dinv.ravel(order="F"),
                                           lr_data=np.zeros(0), perm0=np.arange(m // d), perm1=np.arange(m // d)))
        self.blocks = len(blocks)
        self.entries = int(sum(D.size for _, D in blocks))
        self.h = HmatGpu.batch(members, device=device, precisions=(precision,), plan_only=plan_only)
        p0 = np.asarray(ex["perm0"], dtype=np.int64)
        p1 = np.asarray(ex["perm1"], dtype=np.int64)
        # M_orig^-1 = P1^T M_perm^-1 P0
        self.gather = (d * p0[:, None] + np.arange(d)).ravel()   # x_perm = x[gather]
        self.scatter = (d * p1[:, None] + np.arange(d)).ravel()  # out[scatter] = y_perm
        self._dev = None

    def _buffers(self, x):
        import torch

        if self._dev is None or self._dev[0] != x.device:
            self._dev = (x.device, torch.from_numpy(self.gather).to(x.device), torch.from_numpy(self.scatter).to(x.device),
                         torch.empty(self.n, dtype=torch.float64, device=x.device),
                         torch.empty(self.n, dtype=torch.float64, device=x.device))
        return self._dev[1:]

    def __call__(self, x, out):
        if isinstance(x, np.ndarray):
            if self.ordering == "permuted":
                out[:] = self.h.matvec(x, self.precision)
            else:
                out[self.scatter] = self.h.matvec(x[self.gather], self.precision)
            return out
        if self.ordering == "permuted":
            return self.h.matvec(x, self.precision, out=out)
        import torch

        gi, si, xp, yp = self._buffers(x)
        torch.index_select(x, 0, gi, out=xp)
        self.h.matvec(xp, self.precision, out=yp)
        out.index_copy_(0, si, yp)
        return out

    def close(self) -> None:
        self.h.close()
