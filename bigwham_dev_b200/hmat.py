"""Device-resident H-matrix: the Python face of the C ABI (include/bigwham_b200.h).

``HmatGpu`` plays the role of the reference's ``Hmat<double>`` on the GPU
(src/hmat/hmatrix/hmat.h:31-122): it receives the blocks the reference built,
lays them out once in device memory, and applies the operator.

* ``matvec(x)`` with a host (numpy) array follows ``Hmat::matvecOriginal`` /
  ``BigWhamIO::MatVec`` (hmat.cc:572-635, bigwham_io.cc:927-933): original dof
  ordering, FP64 in and out.
* ``matvec(x)`` with a CUDA torch tensor is stream-ordered on the current torch
  stream and returns a CUDA tensor.
* ``matvec_raw_ptr(x_ptr, y_ptr)`` is the device-pointer entry the reference
  exposes to CuPy/JAX users (py_bigwham.cc:213-222, bigwham4py.py:152-181):
  FP64, original ordering, synchronized before returning.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A


def _ptr(a) -> int:
    return a.ctypes.data if isinstance(a, np.ndarray) else int(a)


def _prec_flag(precision) -> int:
    if isinstance(precision, int):
        return precision
    try:
        return A.PRECISIONS[precision]
    except KeyError:
        raise ValueError(f"precision must be one of {sorted(A.PRECISIONS)}") from None


class HmatGpu:
    """An H-matrix stored on one GPU.

    dof, n_rows, n_cols: dofs per collocation point and scalar sizes.
    perm0, perm1: row / column permutations of the collocation points.
    device: CUDA ordinal, or -1 for a host-only plan (``finalize(plan_only=True)``).
    """

    has_matmat = False
    _plan_only = False

    def __init__(self, dof: int, n_rows: int, n_cols: int, perm0, perm1, device: int = 0):
        self._lib = A.lib()
        self.dof, self.n_rows, self.n_cols, self.device = int(dof), int(n_rows), int(n_cols), int(device)
        p0 = np.ascontiguousarray(perm0, dtype=np.int64)
        p1 = np.ascontiguousarray(perm1, dtype=np.int64)
        h = C.c_void_p()
        st = self._lib.bw_create(self.dof, self.n_rows, self.n_cols, p0.ctypes.data, p1.ctypes.data, self.device,
                                 C.byref(h))
        A.check(st, None)
        self._h = h
        self._keep = []  # block arrays borrowed until finalize
        self._finalized = False
        self.precisions = ()
        self.has_transpose = False

    # ------------------------------------------------------------------ construction
    def add_full(self, i0: int, j0: int, a) -> None:
        a = np.asfortranarray(a, dtype=np.float64)
        self._keep.append(a)
        A.check(self._lib.bw_add_full(self._h, int(i0), int(j0), a.shape[0], a.shape[1], a.ctypes.data,
                                      max(1, a.shape[0])), self._h)

    def add_lowrank(self, i0: int, j0: int, Amat, Bmat) -> None:
        Amat = np.asfortranarray(Amat, dtype=np.float64)
        Bmat = np.asfortranarray(Bmat, dtype=np.float64)
        if Amat.shape[1] != Bmat.shape[0]:
            raise ValueError("A is m x r and B is r x n")
        self._keep += [Amat, Bmat]
        A.check(self._lib.bw_add_lowrank(self._h, int(i0), int(j0), Amat.shape[0], Bmat.shape[1], Amat.shape[1],
                                         Amat.ctypes.data, max(1, Amat.shape[0]), Bmat.ctypes.data,
                                         max(1, Bmat.shape[0])), self._h)

    def add_flat(self, fr, lr, fr_data, lr_data, row0: int = 0, col0: int = 0) -> None:
        """Register all blocks from flat arrays laid out like the reference's
        block containers: FR blocks back to back (column-major), and per LR
        block A (m x r) then B (r x n).  fr rows: (i0, j0, iend, jend) and lr
        rows (i0, j0, iend, jend, r) in collocation-point units (HPattern,
        h_pattern.h:21-33), shifted by the scalar offsets row0 / col0 (a batch
        member's place).  Zero-copy: the arrays are borrowed until finalize."""
        d = self.dof
        fr = np.asarray(fr, dtype=np.int64).reshape(-1, 4)
        lr = np.asarray(lr, dtype=np.int64).reshape(-1, 5)
        fr_data = np.ascontiguousarray(fr_data, dtype=np.float64)
        lr_data = np.ascontiguousarray(lr_data, dtype=np.float64)
        self._keep += [fr_data, lr_data]
        base = fr_data.ctypes.data
        o = 0
        for i0, j0, i1, j1 in fr:
            m, n = int(i1 - i0) * d, int(j1 - j0) * d
            if (o + m * n) > fr_data.size:
                raise ValueError("fr_data shorter than the pattern says")
            A.check(self._lib.bw_add_full(self._h, row0 + int(i0) * d, col0 + int(j0) * d, m, n, base + 8 * o, m),
                    self._h)
            o += m * n
        base = lr_data.ctypes.data
        o = 0
        for i0, j0, i1, j1, r in lr:
            m, n, r = int(i1 - i0) * d, int(j1 - j0) * d, int(r)
            if (o + r * (m + n)) > lr_data.size:
                raise ValueError("lr_data shorter than the pattern says")
            A.check(self._lib.bw_add_lowrank(self._h, row0 + int(i0) * d, col0 + int(j0) * d, m, n, r, base + 8 * o,
                                             max(1, m),
                                             base + 8 * (o + m * r), max(1, r)), self._h)
            o += r * (m + n)

    def set_wait_limit(self, ns: int) -> None:
        """Bound of every in-kernel wait (bw_set_wait_limit); default 2 s."""
        A.check(self._lib.bw_set_wait_limit(self._h, int(ns)), self._h)

    def set_tuning(self, **kw) -> "HmatGpu":
        """Plan parameters (bw_set_tuning), before finalize: items_per_cta_phase1,
        items_per_cta_phase2, chunk_bytes, mm_items_per_cta, unit_bytes, narrow_rows, narrow_cols,
        narrow_coop."""
        for k, v in kw.items():
            A.check(self._lib.bw_set_tuning(self._h, k.encode(), int(v)), self._h)
        return self

    def finalize(self, precisions=("fp64",), transpose: bool = False, check_finite: bool = True,
                 plan_only: bool = False, device_limit: int | None = None, matmat: bool = False,
                 tuning: dict | None = None) -> "HmatGpu":
        """Lay the blocks out on the device.  precisions: storage copies for
        matvec ("fp64", "fp32", "bf16"); transpose: also H^T; matmat: also the
        BF16 layout of the tensor-core multi-right-hand-side product; tuning:
        plan parameters (set_tuning)."""
        if tuning:
            self.set_tuning(**tuning)
        flags = 0
        for p in precisions:
            flags |= _prec_flag(p)
        if transpose:
            flags |= A.BW_STORE_TRANSPOSE
        if not check_finite:
            flags |= A.BW_NO_FINITE_CHECK
        if plan_only:
            flags |= A.BW_PLAN_ONLY
        if matmat:
            flags |= A.BW_STORE_MATMAT
        if device_limit is not None:
            A.check(self._lib.bw_set_device_limit(self._h, int(device_limit)), self._h)
        st = self._lib.bw_finalize(self._h, flags)
        self._keep = []
        A.check(st, self._h)
        self._finalized = True
        self.precisions = tuple(precisions)
        self.has_transpose = bool(transpose)
        self.has_matmat = bool(matmat)
        self._plan_only = bool(plan_only)
        return self

    @classmethod
    def from_flat(cls, dof, n_rows, n_cols, fr, lr, fr_data, lr_data, perm0, perm1, device=0, **kw) -> "HmatGpu":
        h = cls(dof, n_rows, n_cols, perm0, perm1, device)
        h.add_flat(fr, lr, fr_data, lr_data)
        return h.finalize(**kw)

    @classmethod
    def from_device_flat(cls, dof, n_rows, n_cols, fr, lr, fr_data, lr_data, perm0, perm1, device=0,
                         **kw) -> "HmatGpu":
        """Handle from the flat form with the block data in device memory
        (CUDA float64 tensors on `device`, e.g. from devbuild.build_r0(...,
        on_device=True)), laid out on the device by finalize(**kw)
        (bw_add_flat_device): the host never reads the blocks."""
        fr = np.ascontiguousarray(fr, dtype=np.int64).reshape(-1, 4)
        lr = np.ascontiguousarray(lr, dtype=np.int64).reshape(-1, 5)
        for t in (fr_data, lr_data):
            if not (getattr(t, "is_cuda", False) and str(t.dtype) == "torch.float64" and t.is_contiguous()):
                raise TypeError("fr_data and lr_data must be contiguous CUDA float64 tensors")
        self = cls(dof, n_rows, n_cols, perm0, perm1, device)
        A.check(self._lib.bw_add_flat_device(self._h, fr.shape[0], fr.ctypes.data, lr.shape[0], lr.ctypes.data,
                                             fr_data.data_ptr(), fr_data.numel(), lr_data.data_ptr(),
                                             lr_data.numel()), self._h)
        self._keep = [fr, lr, fr_data, lr_data]
        return self.finalize(**kw)

    @classmethod
    def from_file(cls, path, device: int = 0, verify: bool = True, **kw) -> "HmatGpu":
        """Handle from a block file (bw_create_from_file; written by
        ``blockfile.write`` or ``BigWhamIOGpu.write_to_file``): the blocks are
        registered straight from the mapped file and laid out by
        ``finalize(**kw)``, with no H-matrix rebuild.  verify: check the block
        data checksums first.  The counterpart of the reference's
        ``Hmat(filename)`` constructor (src/hmat/hmatrix/hmat.cc:64-74)."""
        from . import blockfile

        head = blockfile.info(path)
        self = cls.__new__(cls)
        self._lib = A.lib()
        self.dof, self.n_rows, self.n_cols, self.device = head["dof"], head["n_rows"], head["n_cols"], int(device)
        h = C.c_void_p()
        A.check(self._lib.bw_create_from_file(blockfile._path(path), self.device, int(bool(verify)), C.byref(h)),
                None)
        self._h = h
        self._keep = []
        self._finalized = False
        self.precisions = ()
        self.has_transpose = False
        return self.finalize(**kw)

    @classmethod
    def batch(cls, members, device: int = 0, **kw) -> "HmatGpu":
        """One handle for several independent H-matrices of the same dof
        (bw_create_batch): the block-diagonal H-matrix of the members, applied
        by one matvec.  members: objects with the fields of a flat block list
        (dof, n_rows, n_cols, fr, lr, fr_data, lr_data, perm0, perm1).  x and y
        hold the members' vectors back to back; ``row_offsets`` /
        ``col_offsets`` (count + 1 entries) give where each starts."""
        members = list(members)
        if not members:
            raise ValueError("empty batch")
        dof = int(members[0].dof)
        if any(int(m.dof) != dof for m in members):
            raise ValueError("all members of a batch must have the same dof")
        p0 = [np.ascontiguousarray(m.perm0, dtype=np.int64) for m in members]
        p1 = [np.ascontiguousarray(m.perm1, dtype=np.int64) for m in members]
        nr = np.array([int(m.n_rows) for m in members], dtype=np.int64)
        nc = np.array([int(m.n_cols) for m in members], dtype=np.int64)
        pp0 = (C.c_void_p * len(members))(*[a.ctypes.data for a in p0])
        pp1 = (C.c_void_p * len(members))(*[a.ctypes.data for a in p1])
        self = cls.__new__(cls)
        self._lib = A.lib()
        self.dof, self.n_rows, self.n_cols, self.device = dof, int(nr.sum()), int(nc.sum()), int(device)
        h = C.c_void_p()
        A.check(self._lib.bw_create_batch(dof, len(members), nr.ctypes.data, nc.ctypes.data, pp0, pp1, self.device,
                                          C.byref(h)), None)
        self._h = h
        self._keep = []
        self._finalized = False
        self.precisions = ()
        self.has_transpose = False
        self.row_offsets = np.concatenate([[0], np.cumsum(nr)])
        self.col_offsets = np.concatenate([[0], np.cumsum(nc)])
        for k, m in enumerate(members):
            self.add_flat(m.fr, m.lr, m.fr_data, m.lr_data, row0=int(self.row_offsets[k]),
                          col0=int(self.col_offsets[k]))
        return self.finalize(**kw)

    # ------------------------------------------------------------------ application
    @property
    def shape(self):
        return (self.n_rows, self.n_cols)

    def _flags(self, precision, permuted, transpose):
        f = _prec_flag(precision)
        if permuted:
            f |= A.BW_PERMUTED
        if transpose:
            f |= A.BW_TRANSPOSE
        return f

    def matvec(self, x, precision="fp64", permuted: bool = False, transpose: bool = False, out=None,
               stream=None):
        """y = H x (H^T x with transpose=True).

        numpy input: host path (copies in, synchronizes, returns numpy).
        torch CUDA input: device path on `stream` (default: current torch
        stream), returns a CUDA float64 tensor; no synchronization."""
        flags = self._flags(precision, permuted, transpose)
        nin, nout = (self.n_rows, self.n_cols) if transpose else (self.n_cols, self.n_rows)
        if isinstance(x, np.ndarray):
            x = np.ascontiguousarray(x, dtype=np.float64)
            if x.shape != (nin,):
                raise ValueError(f"x must have shape ({nin},)")
            y = out if out is not None else np.empty(nout)
            A.check(self._lib.bw_matvec_host(self._h, x.ctypes.data, y.ctypes.data, flags), self._h)
            return y
        import torch

        if not (isinstance(x, torch.Tensor) and x.is_cuda):
            raise TypeError("x must be a numpy array or a CUDA torch tensor")
        if x.dtype != torch.float64 or x.numel() != nin or not x.is_contiguous():
            raise ValueError(f"x must be a contiguous float64 CUDA tensor of {nin} values")
        y = out if out is not None else torch.empty(nout, dtype=torch.float64, device=x.device)
        if stream is None:
            stream = torch.cuda.current_stream(x.device)
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        A.check(self._lib.bw_matvec(self._h, x.data_ptr(), y.data_ptr(), flags, sp), self._h)
        return y

    def rmatvec(self, x, precision="fp64", **kw):
        return self.matvec(x, precision=precision, transpose=True, **kw)

    def matvec_ptr(self, x_ptr: int, y_ptr: int, precision="fp64", permuted=False, transpose=False,
                   stream: int = 0) -> None:
        """Stream-ordered product on raw device pointers (no synchronization)."""
        A.check(self._lib.bw_matvec(self._h, int(x_ptr), int(y_ptr), self._flags(precision, permuted, transpose),
                                    int(stream)), self._h)

    def matvec_raw_ptr(self, x_ptr: int, y_ptr: int) -> None:
        """Reference semantics of matvec_raw_ptr: FP64, original ordering,
        device pointers, returns once y is complete."""
        self.matvec_ptr(x_ptr, y_ptr, "fp64", stream=0)
        self.sync(0)

    def matmat_ptr(self, X_ptr: int, ldx: int, Y_ptr: int, ldy: int, nrhs: int, precision="fp64",
                   stream: int = 0, permuted: bool = False, transpose: bool = False) -> None:
        A.check(self._lib.bw_matmat(self._h, int(X_ptr), int(ldx), int(Y_ptr), int(ldy), int(nrhs),
                                    self._flags(precision, permuted, transpose), int(stream)), self._h)

    def matmat(self, X, precision="fp64", permuted: bool = False, transpose: bool = False, out=None, stream=None):
        """Y = H X (H^T X) for a CUDA float64 tensor X of shape (n, k),
        stream-ordered on `stream` (default: the current torch stream).
        X and Y are column-major (each right-hand side contiguous); X is copied
        to that layout when it is not.  "bf16" on a handle finalized with
        matmat=True runs on the tensor cores, 64 right-hand sides per pass;
        everything else applies one matvec per column."""
        import torch

        nin, nout = (self.n_rows, self.n_cols) if transpose else (self.n_cols, self.n_rows)
        if not (isinstance(X, torch.Tensor) and X.is_cuda and X.dtype == torch.float64 and X.dim() == 2):
            raise TypeError("X must be a 2-D float64 CUDA tensor")
        if X.shape[0] != nin:
            raise ValueError(f"X must have {nin} rows")
        k = X.shape[1]
        if X.stride(0) != 1 or (k > 1 and X.stride(1) < nin):
            X = X.t().contiguous().t()
        if out is None:
            out = torch.empty(k, nout, dtype=torch.float64, device=X.device).t()
        elif out.shape != (nout, k) or out.stride(0) != 1 or (k > 1 and out.stride(1) < nout):
            raise ValueError(f"out must be a column-major ({nout}, {k}) tensor")
        if stream is None:
            stream = torch.cuda.current_stream(X.device)
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        ldx = X.stride(1) if k > 1 else nin
        ldy = out.stride(1) if k > 1 else nout
        self.matmat_ptr(X.data_ptr(), ldx, out.data_ptr(), ldy, k, precision, sp, permuted, transpose)
        return out

    def mm_plan_export(self, phase: int, transposed: bool = False) -> dict:
        """Host view of the matmat plan of one phase (finalize(matmat=True)):
        chunk words (n, 16), cta offsets, T8 rows, and (plan-only handles) the
        raw BF16 data words."""
        nch, nel, ncta, t8 = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        A.check(self._lib.bw_mm_plan_export(self._h, phase, int(transposed), C.byref(nch), None, C.byref(nel), None,
                                            C.byref(ncta), None, C.byref(t8)), self._h)
        chunks = np.zeros((nch.value, 16), np.int32)
        cta = np.zeros(ncta.value, np.int32)
        data = np.zeros(nel.value, np.uint16) if self._plan_only else None
        A.check(self._lib.bw_mm_plan_export(self._h, phase, int(transposed), None, chunks.ctypes.data, None,
                                            data.ctypes.data if data is not None else None, None, cta.ctypes.data,
                                            None), self._h)
        return {"chunks": chunks, "item_ptr": cta, "data": data, "t8_len": t8.value}

    def sync(self, stream=0) -> None:
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        A.check(self._lib.bw_sync(self._h, sp), self._h)

    def diagonal(self, permuted: bool = False):
        d = np.empty(max(self.n_rows, self.n_cols))
        A.check(self._lib.bw_diagonal(self._h, d.ctypes.data, A.BW_PERMUTED if permuted else 0), self._h)
        return d

    # ------------------------------------------------------------------ introspection
    def info(self) -> dict:
        keys = ["n_rows", "n_cols", "dof", "n_full", "n_lowrank", "entries", "sum_rank", "n_panels", "device_bytes",
                "grid", "phase1_chunks", "phase2_chunks", "stored"]
        out = (C.c_int64 * len(keys))()
        A.check(self._lib.bw_info(self._h, out, len(keys)), self._h)
        return dict(zip(keys, list(out)))

    def algorithmic_bytes(self, precision="fp64") -> int:
        b = C.c_int64()
        A.check(self._lib.bw_algorithmic_bytes(self._h, _prec_flag(precision), C.byref(b)), self._h)
        return int(b.value)

    def plan_export(self, precision="fp64", phase=2, transposed=False, with_data=True) -> dict:
        nc, ne, nt = C.c_int64(), C.c_int64(), C.c_int64()
        f = _prec_flag(precision)
        A.check(self._lib.bw_plan_export(self._h, f, phase, int(transposed), C.byref(nc), None, C.byref(ne), None,
                                         C.byref(nt), None), self._h)
        chunks = np.zeros((nc.value, 8), np.int32)
        items = np.zeros(nt.value, np.int32)
        data = np.zeros(ne.value) if with_data else None
        A.check(self._lib.bw_plan_export(self._h, f, phase, int(transposed), C.byref(nc), chunks.ctypes.data,
                                         C.byref(ne), data.ctypes.data if with_data else None, C.byref(nt),
                                         items.ctypes.data), self._h)
        n_wide, n_coop = C.c_int64(), C.c_int64()
        A.check(self._lib.bw_plan_split(self._h, f, phase, int(transposed), C.byref(n_wide), C.byref(n_coop)),
                self._h)
        return {"chunks": chunks, "item_ptr": items, "data": data, "n_wide": int(n_wide.value),
                "n_coop": int(n_coop.value)}

    def launches(self, precision="fp64", transposed=False) -> int:
        """Kernel launches of one matvec (bw_matvec_launches)."""
        n = C.c_int64()
        A.check(self._lib.bw_matvec_launches(self._h, _prec_flag(precision), int(transposed), C.byref(n)), self._h)
        return int(n.value)

    def set_timing(self, enable: bool = True) -> None:
        """Record CUDA events around each launch of every following matvec."""
        A.check(self._lib.bw_set_timing(self._h, int(enable)), self._h)

    def timing_read_launches(self):
        """Summed durations (ms) of the (x gather, phase 1 CTA-wide, phase 1
        unstaged, G2 gather, phase 2 CTA-wide, phase 2 unstaged) launches
        recorded since the last read, and the number of matvecs."""
        ms = (C.c_double * 6)()
        n = C.c_int64()
        A.check(self._lib.bw_timing_read_launches(self._h, ms, C.byref(n)), self._h)
        return list(ms), int(n.value)

    def timing_read(self):
        """Summed durations (ms) of the (x gather, phase 1, G2 gather, phase 2)
        launches recorded since the last read, and the number of matvecs."""
        ms = (C.c_double * 4)()
        n = C.c_int64()
        A.check(self._lib.bw_timing_read(self._h, ms, C.byref(n)), self._h)
        return list(ms), int(n.value)

    def phase_bytes(self, precision="fp64", transposed=False):
        b1, b2 = C.c_int64(), C.c_int64()
        A.check(self._lib.bw_phase_bytes(self._h, _prec_flag(precision), int(transposed), C.byref(b1),
                                         C.byref(b2)), self._h)
        return int(b1.value), int(b2.value)

    @classmethod
    def _borrow(cls, handle: int, dof: int, n_rows: int, n_cols: int, precisions, transpose: bool, owner):
        """Non-owning view of a handle created elsewhere (e.g. by the host
        adapter); `owner` is kept alive while the view exists."""
        self = cls.__new__(cls)
        self._lib = A.lib()
        self._h = C.c_void_p(handle)
        self.dof, self.n_rows, self.n_cols, self.device = int(dof), int(n_rows), int(n_cols), 0
        self._keep, self._finalized = [], True
        self.precisions, self.has_transpose = tuple(precisions), bool(transpose)
        self._owner = owner
        return self

    def close(self) -> None:
        if getattr(self, "_owner", None) is not None:
            self._h = None
            self._owner = None
            return
        if getattr(self, "_h", None):
            self._lib.bw_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
