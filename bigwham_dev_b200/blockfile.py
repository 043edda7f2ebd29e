"""Block files: a built H-matrix on disk (the C ABI's bw_file_* entries).

The reference saves a built Hmat with ``Hmat<T>::writeToFile`` and loads it
with ``readFromFile`` / the ``Hmat(filename)`` constructor
(src/hmat/hmatrix/hmat.cc:64-74, :749-935); both need HDF5.  A block file holds
the same content in a flat, page-aligned binary with checksums:

* dof and sizes, both permutations;
* the HPattern columns of every block;
* the full-rank blocks, each low-rank block's A and B;
* optionally the ACA error estimates.

``HmatGpu.from_file`` maps it and uploads without rebuilding the H-matrix.

    ex = io.export_blocks()                 # BigWhamIOGpu, before attach_gpu
    blockfile.write("crack.bwb", ex)        # or io.write_to_file("crack.bwb")
    h = HmatGpu.from_file("crack.bwb", precisions=("fp64", "bf16"))
    ex2 = blockfile.read("crack.bwb")       # the flat arrays back, bitwise equal

Flat form (as ``BigWhamIOGpu.export_blocks`` returns it): ``fr`` (n_FR x 4:
i0, j0, i_end, j_end in points), ``lr`` (n_LR x 5: the same + rank in scalar
columns), ``fr_data`` (FR blocks back to back, column-major), ``lr_data`` (per
LR block A then B), ``perm0`` and ``perm1``.
"""
from __future__ import annotations

import os

import numpy as np

from . import _capi as A

INFO_KEYS = ("dof", "n_rows", "n_cols", "n_fr", "n_lr", "fr_entries", "lr_entries", "has_lr_error", "file_bytes")


def _path(path) -> bytes:
    return os.fsencode(os.fspath(path))


def _arr(a, dtype, shape=None):
    a = np.ascontiguousarray(a, dtype=dtype)
    return a.reshape(shape) if shape is not None else a


def write(path, ex: dict, lr_error=None) -> None:
    """Write the flat form `ex` (keys dof, n_rows, n_cols, fr, lr, fr_data,
    lr_data, perm0, perm1) to `path`; lr_error: the n_LR ACA error estimates
    (optional).  The file appears complete or not at all."""
    fr = _arr(ex["fr"], np.int64, (-1, 4))
    lr = _arr(ex["lr"], np.int64, (-1, 5))
    fd = _arr(ex["fr_data"], np.float64)
    ld = _arr(ex["lr_data"], np.float64)
    p0 = _arr(ex["perm0"], np.int64)
    p1 = _arr(ex["perm1"], np.int64)
    d = int(ex["dof"])
    need_fr = int(((fr[:, 2] - fr[:, 0]) * (fr[:, 3] - fr[:, 1])).sum()) * d * d
    need_lr = int((lr[:, 4] * ((lr[:, 2] - lr[:, 0]) + (lr[:, 3] - lr[:, 1])) * d).sum())
    if fd.size < need_fr or ld.size < need_lr:
        raise ValueError("block data shorter than the pattern says")
    if p0.size * d != int(ex["n_rows"]) or p1.size * d != int(ex["n_cols"]):
        raise ValueError("permutation lengths do not match the sizes")
    err = None
    if lr_error is not None:
        err = _arr(lr_error, np.float64)
        if err.size != lr.shape[0]:
            raise ValueError("lr_error needs one value per low-rank block")
    L = A.lib()
    A.check(L.bw_file_write(_path(path), d, int(ex["n_rows"]), int(ex["n_cols"]), p0.ctypes.data, p1.ctypes.data,
                            fr.shape[0], fr.ctypes.data, fd.ctypes.data, lr.shape[0], lr.ctypes.data, ld.ctypes.data,
                            None if err is None else err.ctypes.data), None)


def info(path) -> dict:
    """Header of a block file (checked: header checksum, section bounds,
    pattern and permutations)."""
    out = np.zeros(9, dtype=np.int64)
    A.check(A.lib().bw_file_info(_path(path), out.ctypes.data), None)
    return dict(zip(INFO_KEYS, (int(v) for v in out)))


def read(path, verify: bool = True, alloc=np.empty, patterns: bool = False) -> dict:
    """The flat form stored in `path`, plus ``lr_error`` (zeros when the file
    has none) and, with patterns=True, the HPattern columns ``fr_pattern`` /
    ``lr_pattern`` (n x 6).  verify: also check the block data checksums.
    `alloc` (shape, dtype) -> array places the arrays (e.g. in shared
    memory)."""
    h = info(path)
    d = h["dof"]
    out = {"dof": d, "n_rows": h["n_rows"], "n_cols": h["n_cols"],
           "fr": alloc((h["n_fr"], 4), np.int64), "lr": alloc((h["n_lr"], 5), np.int64),
           "fr_data": alloc((h["fr_entries"],), np.float64), "lr_data": alloc((h["lr_entries"],), np.float64),
           "perm0": alloc((h["n_rows"] // d,), np.int64), "perm1": alloc((h["n_cols"] // d,), np.int64),
           "lr_error": alloc((h["n_lr"],), np.float64)}
    if patterns:
        out["fr_pattern"] = alloc((h["n_fr"], 6), np.int64)
        out["lr_pattern"] = alloc((h["n_lr"], 6), np.int64)
    ptr = {k: out[k].ctypes.data for k in out if isinstance(out[k], np.ndarray)}
    A.check(A.lib().bw_file_read(_path(path), int(bool(verify)), ptr["fr"], ptr["lr"], ptr["fr_data"],
                                 ptr["lr_data"], ptr["perm0"], ptr["perm1"], ptr["lr_error"],
                                 ptr.get("fr_pattern"), ptr.get("lr_pattern")), None)
    return out
