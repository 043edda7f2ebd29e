"""Sub-matrix selection of a built H-matrix, on the GPU.

The reference's HmatSelection (src/hmat/hmatrix/hmat_selection.{h,cc}, made by
BigWhamIO::hmatSelection, src/io/bigwham_io.cc:1365-1375, and by
BEMatrix.__getitem__, interfaces/python/bigwham4py/bigwham4py.py:462-484) is
H[rows, cols] for element index lists `rows` / `cols` (original ordering).
Its matvec (hmat_selection.cc:230-258) scatters x into a full-length vector,
runs every block that touches a selected row and a selected column
(blockSelection, :43-140) over whole blocks, and gathers the selected rows.

Here the selection is its own H-matrix.  In the clustered ordering a block
covers a contiguous range of points, so once the selected points are sorted by
clustered position, the selected rows of any block are again a contiguous
range.  The blocks the reference keeps, cut down to their selected rows and
columns, therefore tile a complete rectangular H-matrix of size
(len(rows) dof) x (len(cols) dof):
* a full-rank block becomes its selected sub-block;
* a low-rank block A B stays low rank: the selected rows of A and the
  selected columns of B, same rank.
That matrix is uploaded as an ordinary handle, so a selection matvec streams
only the selected entries (the reference multiplies whole blocks), and it is
stream-ordered and allocation-free like any other product.

Index semantics follow the reference's matvecOriginal:
* y[i] = (H x_full)[rows[i]], so a repeated row is computed once and
  repeated;
* x_full[cols[i]] = x[i] in list order, so for a repeated column the last
  occurrence counts and the earlier ones are ignored;
* indices outside [0, points) raise IndexError, as validateIndices
  (:10-40) throws std::out_of_range.
The reference maps both lists through permutation_1_ and sizes both by the
row count (:43-81), which is right only for square matrices; here rows go
through permutation_0_ and columns through permutation_1_.
"""
from __future__ import annotations

import numpy as np


def _dof_index(points, d):
    return (d * np.asarray(points, dtype=np.int64)[:, None] + np.arange(d)).ravel()


def _check(idx, n, what):
    idx = np.asarray(idx)
    if idx.ndim != 1:
        idx = idx.ravel()
    if idx.size and (idx.min() < 0 or idx.max() >= n):
        raise IndexError(f"{what} index out of bounds")
    return idx.astype(np.int64)


class _Side:
    """One side (rows or columns) of a selection, as compact clustered
    positions.  `pos[c]` is the base clustered position of compact point c,
    `orig[c]` its index in the unique selection list."""

    def __init__(self, sel, perm):
        inv = np.empty(perm.size, dtype=np.int64)
        inv[perm] = np.arange(perm.size)
        uniq, self.inverse = np.unique(sel, return_inverse=True)  # rows: y_sel = y_u[inverse]
        _, first_in_rev = np.unique(sel[::-1], return_index=True)
        self.take = (sel.size - 1 - first_in_rev).astype(np.int64)  # columns: x_u = x_sel[take], last occurrence
        cpos = inv[uniq]
        order = np.argsort(cpos, kind="stable")
        self.unique = uniq
        self.pos = cpos[order]
        self.orig = order  # compact clustered position c -> index into `unique`

    def cut(self, b0, b1):
        """Compact range [c0, c1) of the base points [b0, b1), and the offsets
        of its points inside the block."""
        c0, c1 = np.searchsorted(self.pos, b0), np.searchsorted(self.pos, b1)
        return int(c0), int(c1), self.pos[c0:c1] - b0


def select_blocks(ex, rows, cols) -> dict:
    """The selection of the flat H-matrix `ex` (BigWhamIOGpu.export_blocks,
    blockfile.read) as a flat form of its own, plus the index maps of
    HmatSelection.  Blocks are kept by the reference's rule and cut to their
    selected rows and columns."""
    d = int(ex["dof"])
    p0 = np.asarray(ex["perm0"], dtype=np.int64)
    p1 = np.asarray(ex["perm1"], dtype=np.int64)
    rows = _check(rows, p0.size, "Row")
    cols = _check(cols, p1.size, "Column")
    R, Cs = _Side(rows, p0), _Side(cols, p1)
    fr = np.asarray(ex["fr"], dtype=np.int64).reshape(-1, 4)
    lr = np.asarray(ex["lr"], dtype=np.int64).reshape(-1, 5)
    fd = np.asarray(ex["fr_data"], dtype=np.float64)
    ld = np.asarray(ex["lr_data"], dtype=np.float64)
    fr_out, fd_out, lr_out, ld_out = [], [], [], []
    o = 0
    for (i0, j0, i1, j1) in fr:
        m, n = (i1 - i0) * d, (j1 - j0) * d
        r0, r1, ri = R.cut(i0, i1)
        c0, c1, ci = Cs.cut(j0, j1)
        if r1 > r0 and c1 > c0:
            a = fd[o:o + m * n].reshape(n, m).T
            fd_out.append(a[np.ix_(_dof_index(ri, d), _dof_index(ci, d))].ravel(order="F"))
            fr_out.append((r0, c0, r1, c1))
        o += m * n
    o = 0
    for (i0, j0, i1, j1, r) in lr:
        m, n = (i1 - i0) * d, (j1 - j0) * d
        r0, r1, ri = R.cut(i0, i1)
        c0, c1, ci = Cs.cut(j0, j1)
        if r1 > r0 and c1 > c0:
            A = ld[o:o + m * r].reshape(r, m).T
            B = ld[o + m * r:o + m * r + r * n].reshape(n, r).T
            ld_out += [A[_dof_index(ri, d), :].ravel(order="F"), B[:, _dof_index(ci, d)].ravel(order="F")]
            lr_out.append((r0, c0, r1, c1, r))
        o += m * r + r * n
    cat = lambda a: np.concatenate(a) if a else np.zeros(0)  # noqa: E731
    return {"dof": d, "n_rows": d * R.unique.size, "n_cols": d * Cs.unique.size,
            "fr": np.array(fr_out, np.int64).reshape(-1, 4), "lr": np.array(lr_out, np.int64).reshape(-1, 5),
            "fr_data": cat(fd_out), "lr_data": cat(ld_out), "perm0": R.orig, "perm1": Cs.orig,
            "_rows": R, "_cols": Cs, "_n_sel": (rows.size, cols.size), "_sel": (rows, cols)}


def full_blocks_original(ex, rows, cols):
    """(val, pos) of the selection's full-rank entries in the reference's
    order (HmatSelection::fullBlocksOriginal, hmat_selection.cc:265-375):
    selected FR blocks in pattern order, then block rows, block columns and
    the dof pairs; val[i] = H_sel(pos[i, 0], pos[i, 1]), positions in the
    selection's dof ordering (for a repeated index, its last occurrence)."""
    d = int(ex["dof"])
    p0 = np.asarray(ex["perm0"], dtype=np.int64)
    p1 = np.asarray(ex["perm1"], dtype=np.int64)
    rows = _check(rows, p0.size, "Row")
    cols = _check(cols, p1.size, "Column")

    def last_slot(sel, perm):  # base clustered point -> last selection index, -1 elsewhere
        inv = np.empty(perm.size, dtype=np.int64)
        inv[perm] = np.arange(perm.size)
        slot = np.full(perm.size, -1, dtype=np.int64)
        slot[inv[sel]] = np.arange(sel.size)  # later assignments win, as in the reference's loop
        return slot

    rs, cs = last_slot(rows, p0), last_slot(cols, p1)
    fr = np.asarray(ex["fr"], dtype=np.int64).reshape(-1, 4)
    fd = np.asarray(ex["fr_data"], dtype=np.float64)
    vals, poss = [], []
    o = 0
    for (i0, j0, i1, j1) in fr:
        m, n = (i1 - i0) * d, (j1 - j0) * d
        ii = np.flatnonzero(rs[i0:i1] >= 0)
        jj = np.flatnonzero(cs[j0:j1] >= 0)
        if ii.size and jj.size:
            a = fd[o:o + m * n].reshape(n, m).T
            # order: ii, jj, iii, jjj (hmat_selection.cc:350-370)
            I = (d * ii[:, None, None, None] + np.arange(d)[None, None, :, None])
            J = (d * jj[None, :, None, None] + np.arange(d)[None, None, None, :])
            I, J = np.broadcast_arrays(I, J)
            vals.append(a[I.ravel(), J.ravel()])
            pr = d * rs[i0 + ii][:, None, None, None] + np.arange(d)[None, None, :, None]
            pc = d * cs[j0 + jj][None, :, None, None] + np.arange(d)[None, None, None, :]
            pr, pc = np.broadcast_arrays(pr, pc)
            poss.append(np.stack([pr.ravel(), pc.ravel()], axis=1))
        o += m * n
    if not vals:
        return np.zeros(0), np.zeros((0, 2), np.int64)
    return np.concatenate(vals), np.concatenate(poss)


class HmatSelection:
    """H[rows, cols] of a built H-matrix on the GPU (the reference's
    HmatSelection).  ex: the base's flat form; rows / cols: element indices
    (original ordering); further keywords go to HmatGpu.finalize
    (precisions, transpose, ...).  device -1 with plan_only=True builds the
    host plan only.

    matvec(x): x of length len(cols) * dof in the selection's order, numpy or
    a CUDA float64 tensor; y of length len(rows) * dof.
    """

    def __init__(self, ex, rows, cols, device: int = 0, precisions=("fp64",), **finalize):
        from .hmat import HmatGpu

        s = select_blocks(ex, rows, cols)
        # full_blocks reads the base's full-rank blocks only: keep those
        self._base = {k: ex[k] for k in ("dof", "fr", "fr_data", "perm0", "perm1")}
        self._sel = s["_sel"]
        self.dof = d = s["dof"]
        self._R, self._C = s["_rows"], s["_cols"]
        self.shape = (d * s["_n_sel"][0], d * s["_n_sel"][1])
        self.blocks = (s["fr"].shape[0], s["lr"].shape[0])
        self.entries = int(s["fr_data"].size + s["lr_data"].size)
        self.perm0, self.perm1 = s["perm0"], s["perm1"]  # the compact handle's permutations
        self.precisions = tuple(precisions)
        self.h = HmatGpu.from_flat(d, s["n_rows"], s["n_cols"], s["fr"], s["lr"], s["fr_data"], s["lr_data"],
                                   s["perm0"], s["perm1"], device=device, precisions=precisions, **finalize)
        # x_u = x[x_take] (last occurrence of each column), y = y_u[y_take]
        self.x_take = _dof_index(self._C.take, d)
        self.y_take = _dof_index(self._R.inverse, d)
        self._dev = None

    def _buffers(self, x):
        """Index maps and the unique-index vectors on x's device, made once."""
        import torch

        if self._dev is None or self._dev[0] != x.device:
            self._dev = (x.device, torch.from_numpy(self.x_take).to(x.device),
                         torch.from_numpy(self.y_take).to(x.device),
                         torch.empty(self.h.n_cols, dtype=torch.float64, device=x.device),
                         torch.empty(self.h.n_rows, dtype=torch.float64, device=x.device))
        return self._dev[1:]

    def matvec(self, x, precision=None, out=None):
        precision = precision or self.precisions[0]
        if not hasattr(x, "data_ptr"):  # numpy arrays, lists: the host path
            x = np.asarray(x, dtype=np.float64).ravel()
            if x.size != self.shape[1]:
                raise ValueError(f"x has {x.size} entries, the selection {self.shape[1]} columns")
            y_u = self.h.matvec(np.ascontiguousarray(x[self.x_take]), precision)
            y = y_u[self.y_take]
            if out is not None:
                out[:] = y
                return out
            return y
        import torch

        if x.numel() != self.shape[1]:
            raise ValueError(f"x has {x.numel()} entries, the selection {self.shape[1]} columns")
        xt, yt, x_u, y_u = self._buffers(x)
        torch.index_select(x, 0, xt, out=x_u)
        self.h.matvec(x_u, precision, out=y_u)
        if out is None:
            return torch.index_select(y_u, 0, yt)
        return torch.index_select(y_u, 0, yt, out=out)

    def full_blocks(self):
        """(val, pos) as the reference's GetFullBlocks on the selection."""
        return full_blocks_original(self._base, *self._sel)

    def close(self) -> None:
        self.h.close()
