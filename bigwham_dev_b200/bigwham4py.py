"""BigWham's Python interface with the B200 backend behind it.

Mirrors the reference's ``bigwham4py`` (interfaces/python/bigwham4py/bigwham4py.py)
for the matvec path:

* ``BigWhamIOGpu`` stands for the pybind11 ``BigWhamIOSelf``
  (interfaces/python/py_bigwham.cc:141-260): same constructor arguments, same
  method names (build_hierarchical_matrix, matvec, matvec_permute,
  matvec_raw_ptr, get_diagonal, get_permutation, ...).  The H-matrix is
  built by the reference's own host code (compiled into libbigwham_host.so) and
  then uploaded once; every matvec afterwards runs on the GPU.
* ``BEMatrix`` is the scipy ``LinearOperator`` of the reference
  (bigwham4py.py:49-485) with ``useCuda=True`` meaning this backend.

Driven through the C ABI of include/bigwham_host.h.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _capi as A
from .hmat import HmatGpu, _prec_flag

_HERE = os.path.dirname(os.path.abspath(__file__))
HOST_LIB_PATH = os.path.join(_HERE, "_lib", "libbigwham_host.so")

kernels_id = ["2DS0-H", "2DS1-H", "S3DS0-H", "Axi3DS0-H", "3DT0-H", "3DT6-H", "3DR0-H", "3DR0-H-mode1"]
# kernels of the rectangular (source mesh x receiver mesh) BigWhamIO, bigwham_io.cc:300-470
kernels_rect_id = ["2DS0-2DS0-H", "2DS1-2DS1-H", "2DS0-2DP-T", "3DT0-3DT0-H", "3DR0-3DR0-H", "3DR0-3DR0-H-mode1"]

_P, _I64 = C.c_void_p, C.c_int64
_HSIGS = {
    "bwh_create": (C.c_int, [_P, _I64, _P, _I64, C.c_char_p, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_P)]),
    "bwh_create_rect": (C.c_int, [_P, _I64, _P, _I64, _P, _I64, _P, _I64, C.c_char_p, _P, C.c_int, C.c_int, C.c_int,
                                  C.c_int, C.POINTER(_P)]),
    "bwh_build": (C.c_int, [_P, C.c_int, C.c_double, C.c_double]),
    "bwh_build_pattern": (C.c_int, [_P, C.c_int, C.c_double]),
    "bwh_attach_gpu": (C.c_int, [_P, C.c_int, C.c_int, C.c_int]),
    "bwh_set_precision": (C.c_int, [_P, C.c_int]),
    "bwh_set_tuning": (C.c_int, [_P, C.c_char_p, C.c_int64]),
    "bwh_matvec": (C.c_int, [_P, _P, _P]),
    "bwh_matvec_perm": (C.c_int, [_P, _P, _P]),
    "bwh_matvec_raw_ptr": (C.c_int, [_P, _P, _P]),
    "bwh_diagonal": (C.c_int, [_P, _P]),
    "bwh_size": (_I64, [_P, C.c_int]),
    "bwh_dof": (C.c_int, [_P]),
    "bwh_compression": (C.c_double, [_P]),
    "bwh_hmat_time": (C.c_double, [_P]),
    "bwh_permutation": (C.c_int, [_P, _P]),
    "bwh_collocation_points": (_I64, [_P, _P]),
    "bwh_hpattern": (_I64, [_P, _P]),
    "bwh_n_blocks": (_I64, [_P, C.c_int]),
    "bwh_entries": (_I64, [_P, C.c_int]),
    "bwh_export": (C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "bwh_write_to_file": (C.c_int, [_P, C.c_char_p]),
    "bwh_element_frames": (_I64, [_P, _P]),
    "bwh_convert": (C.c_int, [_P, C.c_int, _P, _I64, _P]),
    "bwh_element_normals": (_I64, [_P, _P]),
    "bwh_rotation_matrix": (_I64, [_P, _P]),
    "bwh_max_error_aca": (C.c_double, [_P]),
    "bwh_full_blocks": (_I64, [_P, C.c_int, _P, _P, _P]),
    "bwh_compute_fields": (_I64, [_P, C.c_int, _P, _I64, _P, _I64, _P, _I64]),
    "bwh_storage_requirement": (_I64, [_P]),
    "bwh_omp_threads": (C.c_int, [_P]),
    "bwh_spatial_dimension": (C.c_int, [_P]),
    "bwh_gpu_handle": (_P, [_P]),
    "bwh_destroy": (C.c_int, [_P]),
    "bwh_last_error": (C.c_char_p, []),
}
_hlib = None


def host_lib():
    global _hlib
    if _hlib is None:
        if not os.path.exists(HOST_LIB_PATH):
            raise RuntimeError(f"host adapter not built: {HOST_LIB_PATH} is missing "
                               f"(python -m bigwham_dev_b200.build --host, needs the BigWham sources)")
        A.lib()  # the CUDA backend first (libbigwham_host.so links against it)
        L = C.CDLL(HOST_LIB_PATH)
        for name, (res, args) in _HSIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _hlib = L
    return _hlib


def _check(st):
    if st != 0:
        raise RuntimeError("bigwham_host: " + (host_lib().bwh_last_error() or b"").decode(errors="replace"))


class BigWhamIOGpu:
    """BigWhamIO (square self-interaction) with the GPU matvec installed."""

    def __init__(self, coor, conn, kernel: str, properties, n_openMP_threads: int = 8, n_GPUs: int = 1,
                 verbose: bool = False, homogeneous_size_pattern: bool = False, useCuda: bool = True,
                 fixed_rank: int = -1, device: int = 0):
        if kernel not in kernels_id:
            raise ValueError(f"invalid kernel {kernel}; available: {', '.join(kernels_id)}")
        L = host_lib()
        coor = np.ascontiguousarray(coor, dtype=np.float64).ravel()
        conn = np.ascontiguousarray(conn, dtype=np.int32).ravel()
        props = np.ascontiguousarray(properties, dtype=np.float64).ravel()
        h = C.c_void_p()
        _check(L.bwh_create(coor.ctypes.data, coor.size, conn.ctypes.data, conn.size, kernel.encode(),
                            props.ctypes.data, props.size, int(n_openMP_threads), int(verbose), int(fixed_rank),
                            C.byref(h)))
        self._h = h
        self._L = L
        self._coor, self._conn = coor, conn  # mesh, for element_records
        self.kernel = kernel
        self.use_cuda = bool(useCuda)
        self.device = int(device)
        self.gpu: HmatGpu | None = None
        self._precisions = ("fp64",)
        self._transpose = False

    @classmethod
    def rectangular(cls, coor_src, conn_src, coor_rec, conn_rec, kernel: str, properties, n_openMP_threads: int = 8,
                    n_GPUs: int = 1, verbose: bool = False, homogeneous_size_pattern: bool = False,
                    useCuda: bool = True, fixed_rank: int = -1, device: int = 0) -> "BigWhamIOGpu":
        """The rectangular BigWhamIO (pybind11 BigWhamIORect): receiver rows,
        source columns."""
        if kernel not in kernels_rect_id:
            raise ValueError(f"invalid kernel {kernel}; available: {', '.join(kernels_rect_id)}")
        L = host_lib()
        arrs = [np.ascontiguousarray(a, dtype=t).ravel() for a, t in
                ((coor_src, np.float64), (conn_src, np.int32), (coor_rec, np.float64), (conn_rec, np.int32))]
        props = np.ascontiguousarray(properties, dtype=np.float64).ravel()
        h = C.c_void_p()
        _check(L.bwh_create_rect(*[v for a in arrs for v in (a.ctypes.data, a.size)], kernel.encode(),
                                 props.ctypes.data, props.size, int(n_openMP_threads), int(verbose), int(fixed_rank),
                                 C.byref(h)))
        self = cls.__new__(cls)
        self._h, self._L = h, L
        self._coor, self._conn = arrs[0], arrs[1]  # source mesh
        self._keep = arrs
        self.kernel = kernel
        self.use_cuda = bool(useCuda)
        self.device = int(device)
        self.gpu = None
        self._precisions = ("fp64",)
        self._transpose = False
        return self

    # ---------------------------------------------------------------- build
    def set_gpu_storage(self, precisions=("fp64",), transpose: bool = False, keep_host: bool = False) -> None:
        """Precisions (and H^T) to lay out on the device at the next build;
        keep_host: keep the host blocks after the upload (write_hmatrix needs
        them)."""
        self._precisions = tuple(precisions)
        self._transpose = bool(transpose)
        self._keep_host = bool(keep_host)

    def build_hierarchical_matrix(self, max_leaf_size: int, eta: float, eps_aca: float) -> None:
        _check(self._L.bwh_build(self._h, int(max_leaf_size), float(eta), float(eps_aca)))
        if self.use_cuda:
            self.attach_gpu(self._precisions, self._transpose, release_host=not getattr(self, "_keep_host", False))

    def build_pattern(self, max_leaf_size: int, eta: float) -> None:
        """Cluster tree and block pattern only (BigWhamIO::BuildPattern); see
        devbuild.build_r0 for building the blocks on the device."""
        _check(self._L.bwh_build_pattern(self._h, int(max_leaf_size), float(eta)))

    def attach_gpu(self, precisions=("fp64",), transpose: bool = False, release_host: bool = True,
                   matmat: bool = False, tuning: dict | None = None) -> HmatGpu:
        for k, v in (tuning or {}).items():
            _check(self._L.bwh_set_tuning(self._h, k.encode(), int(v)))
        flags = 0
        for p in precisions:
            flags |= _prec_flag(p)
        if transpose:
            flags |= A.BW_STORE_TRANSPOSE
        if matmat:
            flags |= A.BW_STORE_MATMAT
        _check(self._L.bwh_attach_gpu(self._h, self.device, flags, int(release_host)))
        h = self._L.bwh_gpu_handle(self._h)
        self.gpu = HmatGpu._borrow(h, self.get_dof(), self.matrix_size(0), self.matrix_size(1), precisions,
                                   transpose, owner=self)
        self.gpu.has_matmat = bool(matmat)
        self.set_precision(precisions[0] if "fp64" not in precisions else "fp64")
        return self.gpu

    def set_precision(self, precision) -> None:
        """Precision of the reference-facing calls (matvec, matvec_raw_ptr)."""
        _check(self._L.bwh_set_precision(self._h, _prec_flag(precision)))

    # ---------------------------------------------------------------- products (reference names)
    def matvec(self, x):
        """BigWhamIO::MatVec: host arrays, original ordering."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.matrix_size(0))
        _check(self._L.bwh_matvec(self._h, x.ctypes.data, y.ctypes.data))
        return y

    def matvec_permute(self, x):
        """BigWhamIO::MatVecPerm: host arrays, permuted ordering."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.matrix_size(0))
        _check(self._L.bwh_matvec_perm(self._h, x.ctypes.data, y.ctypes.data))
        return y

    def matvec_raw_ptr(self, x: int, y: int) -> None:
        """BigWhamIO::MatVec(double*, double*): device pointers (CuPy / torch / JAX)."""
        _check(self._L.bwh_matvec_raw_ptr(self._h, C.c_void_p(int(x)), C.c_void_p(int(y))))

    # ---------------------------------------------------------------- queries (reference names)
    def matrix_size(self, k: int) -> int:
        return int(self._L.bwh_size(self._h, int(k)))

    def get_dof(self) -> int:
        return int(self._L.bwh_dof(self._h))

    def get_compression_ratio(self) -> float:
        return float(self._L.bwh_compression(self._h))

    def get_hmat_time(self) -> float:
        return float(self._L.bwh_hmat_time(self._h))

    def get_diagonal(self):
        d = np.empty(max(self.matrix_size(0), self.matrix_size(1)))
        _check(self._L.bwh_diagonal(self._h, d.ctypes.data))
        return d

    def get_permutation(self):
        p = np.empty(self.matrix_size(1) // self.get_dof(), np.int64)
        _check(self._L.bwh_permutation(self._h, p.ctypes.data))
        return p

    def get_collocation_points(self):
        n = self._L.bwh_collocation_points(self._h, None)
        out = np.empty(n)
        self._L.bwh_collocation_points(self._h, out.ctypes.data)
        return out

    def get_hpattern(self):
        n = self._L.bwh_hpattern(self._h, None)
        out = np.empty(n)
        self._L.bwh_hpattern(self._h, out.ctypes.data)
        return out.reshape(-1, 6)

    def n_blocks(self):
        return int(self._L.bwh_n_blocks(self._h, 0)), int(self._L.bwh_n_blocks(self._h, 1))

    def export_blocks(self, alloc=np.empty) -> dict:
        """Flat copy of the built H-matrix (before attach_gpu, or after it with
        the host blocks kept, set_gpu_storage(keep_host=True)): pattern,
        permutations and block data, as HmatGpu.add_flat takes them.  `alloc`
        (shape, dtype) -> array lets the caller place the arrays (e.g. in
        shared memory)."""
        nfr, nlr = self.n_blocks()
        dof = self.get_dof()
        out = {"dof": dof, "n_rows": self.matrix_size(0), "n_cols": self.matrix_size(1),
               "fr": alloc((nfr, 4), np.int64), "lr": alloc((nlr, 5), np.int64),
               "fr_data": alloc((int(self._L.bwh_entries(self._h, 0)),), np.float64),
               "lr_data": alloc((int(self._L.bwh_entries(self._h, 1)),), np.float64),
               "perm0": alloc((self.matrix_size(0) // dof,), np.int64),
               "perm1": alloc((self.matrix_size(1) // dof,), np.int64)}
        _check(self._L.bwh_export(self._h, *(out[k].ctypes.data for k in
                                             ("fr", "lr", "fr_data", "lr_data", "perm0", "perm1"))))
        return out

    def element_records(self):
        """(n_elements, 17) records of the device assembly (bw_r0_assemble_fr):
        collocation point, rotation matrix (row-major, local = R global) and
        unit normal from the reference's element objects, then the half sides
        |v1 - v0| / 2 and |v3 - v0| / 2 of each quadrilateral (the reference's
        get_a_and_b, elastic_3dR0_common.cc:443-468)."""
        n = int(self._L.bwh_element_frames(self._h, None))
        if n < 0:
            _check(1)
        fr = np.empty((n, 15))
        self._L.bwh_element_frames(self._h, fr.ctypes.data)
        v = np.asarray(self._coor, dtype=np.float64).reshape(-1, 3)[np.asarray(self._conn).reshape(n, -1)]
        if v.shape[1] != 4:
            raise ValueError("element records need quadrilateral (3DR0) elements")
        ab = np.stack([np.linalg.norm(v[:, 1] - v[:, 0], axis=1), np.linalg.norm(v[:, 3] - v[:, 0], axis=1)], 1) / 2
        return np.ascontiguousarray(np.hstack([fr, ab]))

    # -- pass-throughs to the reference's BigWhamIO (py_bigwham.cc:141-260) --
    def _vec(self, fn, *args):
        n = int(fn(self._h, *args, None))
        if n < 0:
            _check(1)
        out = np.empty(n)
        fn(self._h, *args, out.ctypes.data)
        return out

    def get_spatial_dimension(self) -> int:
        return int(self._L.bwh_spatial_dimension(self._h))

    def convert_to_local(self, x_global):
        x = np.ascontiguousarray(x_global, dtype=np.float64).ravel()
        out = np.empty_like(x)
        _check(self._L.bwh_convert(self._h, 0, x.ctypes.data, x.size, out.ctypes.data))
        return out

    def convert_to_global(self, x_local):
        x = np.ascontiguousarray(x_local, dtype=np.float64).ravel()
        out = np.empty_like(x)
        _check(self._L.bwh_convert(self._h, 1, x.ctypes.data, x.size, out.ctypes.data))
        return out

    def get_element_normals(self):
        return self._vec(self._L.bwh_element_normals)

    def get_rotation_matrix(self):
        return self._vec(self._L.bwh_rotation_matrix)

    def get_max_error_ACA(self) -> float:
        e = float(self._L.bwh_max_error_aca(self._h))
        if e < 0:
            _check(1)
        return e

    def get_full_blocks(self, original_order: bool = True):
        """(values, rows, cols) of the full-rank blocks' entries (GetFullBlocks /
        GetFullBlocksPerm)."""
        n = int(self._L.bwh_full_blocks(self._h, int(original_order), None, None, None))
        if n < 0:
            _check(1)
        val, row, col = np.empty(n), np.empty(n, np.int32), np.empty(n, np.int32)
        self._L.bwh_full_blocks(self._h, int(original_order), val.ctypes.data, row.ctypes.data, col.ctypes.data)
        return val, row, col

    def _fields(self, kind, coor, x):
        c = np.ascontiguousarray(coor, dtype=np.float64).ravel()
        v = np.ascontiguousarray(x, dtype=np.float64).ravel()
        n = int(self._L.bwh_compute_fields(self._h, kind, c.ctypes.data, c.size, v.ctypes.data, v.size, None, 0))
        if n < 0:
            _check(1)
        out = np.empty(n)
        if self._L.bwh_compute_fields(self._h, kind, c.ctypes.data, c.size, v.ctypes.data, v.size, out.ctypes.data,
                                      n) < 0:
            _check(1)
        return out

    def compute_displacements(self, coor, x):
        """ComputeDisplacements: the reference's host code (flat output)."""
        return self._fields(0, coor, x)

    def compute_stresses(self, coor, x):
        """ComputeStresses: the reference's host code (flat output)."""
        return self._fields(1, coor, x)

    def get_storage_requirement(self) -> int:
        return int(self._L.bwh_storage_requirement(self._h))

    def get_gpu_storage_requirement(self) -> int:
        """Device bytes held by the GPU H-matrix (0 before attach_gpu)."""
        return int(self.gpu.info()["device_bytes"]) if self.gpu is not None else 0

    def get_omp_threads(self) -> int:
        return int(self._L.bwh_omp_threads(self._h))

    def get_cuda_available(self) -> bool:
        try:
            import torch

            return bool(torch.cuda.is_available()) and os.path.exists(A.LIB_PATH)
        except Exception:
            return False

    def write_hmatrix(self, filename) -> None:
        """Hmat::writeToFile's counterpart: a block file (see write_to_file)."""
        self.write_to_file(filename)

    def write_to_file(self, path) -> None:
        """Save the built H-matrix as a block file (before attach_gpu): the
        reference's Hmat::writeToFile (src/hmat/hmatrix/hmat.cc:749-835) without
        HDF5.  Load it with HmatGpu.from_file or blockfile.read."""
        _check(self._L.bwh_write_to_file(self._h, os.fsencode(os.fspath(path))))

    def close(self) -> None:
        if getattr(self, "_h", None):
            if self.gpu is not None:
                self.gpu.close()
                self.gpu = None
            self._L.bwh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


try:
    from scipy.sparse.linalg import LinearOperator as _LinOp
except Exception:  # pragma: no cover - scipy is part of the image
    _LinOp = object


def pattern_kind_index(pat):
    """Index of every block of a pattern (rows as _getPattern returns them,
    column 4 the kind: 0 full rank, 1 low rank) among the blocks of its kind,
    in pattern order: the labels of plotPattern(plot_index=True)."""
    low = np.asarray(pat)[:, 4] == 1
    return np.where(low, np.cumsum(low) - 1, np.cumsum(~low) - 1).astype(np.int64)


def _csc_entries(val, row, col, shape, keep_ratio: float):
    """CSC matrix of the entries; keep_ratio < 1 keeps the largest |entries|
    (that share of them, ties kept), as the reference's _getFullBlocks."""
    from scipy.sparse import csc_matrix

    if keep_ratio < 1.0:
        k = int(np.ceil(keep_ratio * val.size))
        if k == 0:
            return csc_matrix(shape)
        thr = np.partition(np.abs(val), -k)[-k]
        keep = np.abs(val) >= thr
        val, row, col = val[keep], row[keep], col[keep]
    return csc_matrix((val, (row, col)), shape=shape)


class BEMatrix(_LinOp):
    """scipy LinearOperator over the GPU H-matrix (reference: bigwham4py.BEMatrix)."""

    def __init__(self, kernel: str, coor, conn, properties, max_leaf_size: int = 32, eta: float = 3.0,
                 eps_aca: float = 1.0e-3, n_openMP_threads: int = 8, n_GPUs: int = 1, directly_build: bool = True,
                 verbose: bool = False, homogeneous_size_pattern: bool = False, fixed_rank=-1, useCuda=True,
                 precisions=("fp64",), transpose: bool = False, device: int = 0, keep_host: bool = False):
        self.kernel_ = kernel
        self.properties_ = properties
        self.useCuda = True  # the matvec always runs on the GPU here
        self.max_leaf_size_, self.eta_, self.eps_aca_ = int(max_leaf_size), float(eta), float(eps_aca)
        self.n_openMP_threads_ = n_openMP_threads
        self.H_ = BigWhamIOGpu(coor, conn, kernel, properties, n_openMP_threads, n_GPUs, verbose,
                               homogeneous_size_pattern, useCuda, fixed_rank, device)
        self.H_.set_gpu_storage(precisions, transpose, keep_host)
        self.built_ = False
        shape = (0, 0)
        if directly_build:
            self._build()
            shape = (self.H_.matrix_size(0), self.H_.matrix_size(1))
        self.dtype_ = np.dtype(float)
        super().__init__(self.dtype_, shape)

    def _build(self):
        if not self.built_:
            self.H_.build_hierarchical_matrix(self.max_leaf_size_, self.eta_, self.eps_aca_)
            self.built_ = True
            super().__init__(np.dtype(float), (self.H_.matrix_size(0), self.H_.matrix_size(1)))

    def _matvec(self, v):
        return self.H_.matvec(np.asarray(v, dtype=np.float64).ravel())

    def _rmatvec(self, v):
        if self.H_.gpu is None or not self.H_.gpu.has_transpose:
            raise RuntimeError("H^T not stored: build with transpose=True")
        return self.H_.gpu.rmatvec(np.asarray(v, dtype=np.float64).ravel())

    def _matvec_torch(self, x, y):
        """y = H x on CUDA float64 torch tensors (device pointers, as _matvec_cupy)."""
        assert x.is_cuda and y.is_cuda and x.dtype == y.dtype and str(x.dtype) == "torch.float64"
        self.H_.matvec_raw_ptr(x.data_ptr(), y.data_ptr())

    def _matvec_cupy(self, x, y):
        self.H_.matvec_raw_ptr(x.data.ptr, y.data.ptr)

    def getCompression(self) -> float:
        return self.H_.get_compression_ratio()

    def getPermutation(self):
        return self.H_.get_permutation()

    def getCollocationPoints(self):
        """(n_points, dim) collocation points of the mesh."""
        n = self.getSpatialDimension()
        return self.H_.get_collocation_points().reshape(-1, n)

    def getMeshCollocationPoints(self):
        return self.getCollocationPoints()

    def getSpatialDimension(self):
        return self.H_.get_spatial_dimension()

    def get_omp_threads(self) -> int:
        return self.H_.get_omp_threads()

    def getStorageRequirement(self) -> int:
        """Bytes of the H-matrix entries (entries x 8)."""
        self._build()
        return self.H_.get_storage_requirement()

    def getGPUStorageRequirement(self) -> int:
        """Device bytes of the laid-out H-matrix (all stored precisions)."""
        self._build()
        return self.H_.get_gpu_storage_requirement()

    def convert_to_global(self, x_local):
        return self.H_.convert_to_global(x_local)

    def convert_to_local(self, x_global):
        return self.H_.convert_to_local(x_global)

    def get_element_normals(self):
        return self.H_.get_element_normals()

    def get_rotation_matrix(self):
        return self.H_.get_rotation_matrix()

    def get_diagonal(self):
        return self.H_.get_diagonal()

    def get_max_error_ACA(self) -> float:
        return self.H_.get_max_error_ACA()

    def isCudaAvailable(self) -> bool:
        return self.H_.get_cuda_available()

    def write_hmatrix(self, filename) -> None:
        """The reference writes HDF5 (Hmat::writeToFile); this writes a block
        file with the same content (HmatGpu.from_file / blockfile.read read it).
        Needs keep_host=True (the host blocks are otherwise released once the
        H-matrix is on the GPU)."""
        self._build()
        self.H_.write_hmatrix(filename)

    def _getFullBlocks(self, original_order=True, keep_ratio: float = 1.0):
        """Full-rank blocks as a scipy CSC matrix (bigwham4py.py:252-276)."""
        if not (0 < keep_ratio <= 1):
            raise ValueError("ratio must be a float between 0 and 1.")
        self._build()
        val, row, col = self.H_.get_full_blocks(original_order)
        return _csc_entries(val, row, col, self.shape, keep_ratio)

    def _getPattern(self):
        return self.H_.get_hpattern()

    def H_ILU_prec(self, fill_factor=1, drop_tol=1e-3, keep_ratio=1.0):
        """ILU of the full-rank blocks (scipy spilu, host), as the reference's
        H_ILU_prec (bigwham4py.py:345-360); the full-rank blocks stay on the host
        beside the GPU H-matrix, so this works with the GPU matvec."""
        from scipy.sparse.linalg import LinearOperator, spilu

        ilu = spilu(self._getFullBlocks(keep_ratio=keep_ratio), fill_factor=fill_factor, drop_tol=drop_tol)
        return LinearOperator(self.shape, ilu.solve)

    def _device_fields(self):
        """The GPU evaluator of observation fields for this mesh (fields.py;
        kernels 2DS0-H and 3DR0-H), made once."""
        if getattr(self, "_dev_fields", None) is None:
            from .fields import R0Fields, S0Fields

            E, nu = float(self.properties_[0]), float(self.properties_[1])
            if self.kernel_ == "2DS0-H":
                self._dev_fields = S0Fields(self.H_._coor.reshape(-1, 2), self.H_._conn.reshape(-1, 2), E, nu,
                                            self.H_.device)
            elif self.kernel_ == "3DR0-H":
                self._dev_fields = R0Fields(self.H_.element_records(), E, nu, self.H_.device)
            else:
                raise NotImplementedError(f"device fields for {self.kernel_}: 2DS0-H and 3DR0-H only")
        return self._dev_fields

    def compute_displacements(self, list_coor, local_solu, device: bool = False):
        """Displacements at points; (n_points, dim).  device=False: the
        reference's host code; device=True: the GPU kernels of fields.py
        (2DS0-H, 3DR0-H; for 3DR0-H the reference returns zeros)."""
        self._build()
        n = self.getSpatialDimension()
        list_coor = np.asarray(list_coor, dtype=np.float64)
        assert n == list_coor.shape[1], "Coordinates dimension of the given points is not matching the problem spatial dimension !"
        if device:
            return self._device_fields().fields(list_coor, np.asarray(local_solu, dtype=np.float64),
                                                want_stress=False)[1]
        return self.H_.compute_displacements(list_coor, local_solu).reshape(-1, n)

    def compute_stresses(self, list_coor, local_solu, device: bool = False):
        """Stresses at points; (n_points, 3 or 6).  device as for
        compute_displacements."""
        self._build()
        n = self.getSpatialDimension()
        list_coor = np.asarray(list_coor, dtype=np.float64)
        assert n == list_coor.shape[1], "Coordinates dimension of the given points is not matching the problem spatial dimension !"
        if device:
            return self._device_fields().fields(list_coor, np.asarray(local_solu, dtype=np.float64),
                                                want_disp=False)[0]
        return self.H_.compute_stresses(list_coor, local_solu).reshape(-1, 3 if n == 2 else 6)

    def getMatvecTime(self, N_matvec=100):
        """Seconds per matvec (host arrays, as the reference times it)."""
        import time

        x = np.ones(self.shape[0])
        self._matvec(x)
        t0 = time.time()
        for _ in range(N_matvec):
            self._matvec(x)
        return (time.time() - t0) / N_matvec

    def plotPattern(self, plot_index=False):
        """The block pattern as a matplotlib figure (needs matplotlib).
        plot_index: write each block's index among the blocks of its kind
        (full-rank or low-rank, in pattern order) at its centre."""
        import matplotlib.pyplot as plt
        from matplotlib.collections import PatchCollection
        from matplotlib.patches import Rectangle

        pat = self._getPattern()
        max_y = pat[:, 3].max()
        fig, ax = plt.subplots()
        patches = [Rectangle((r[1], max_y - r[0] - abs(r[0] - r[2])), abs(r[1] - r[3]), abs(r[0] - r[2])) for r in pat]
        if plot_index:
            for r, k in zip(patches, pattern_kind_index(pat)):
                ax.text(r.get_x() + r.get_width() / 2, r.get_y() + r.get_height() / 2, str(int(k)), ha="center",
                        va="center", fontsize=8, fontweight="bold", color="black")
        pc = PatchCollection(patches, edgecolors="black", alpha=0.4)
        pc.set_array(pat[:, 4])
        ax.add_collection(pc)
        ax.set_ylim([pat[:, 0].min(), pat[:, 3].max()])
        ax.set_xlim([pat[:, 1].min(), pat[:, 2].max()])
        ax.set_aspect("equal")
        return fig

    def __getitem__(self, indices):
        """Sub-matrix selection ``A[np.ix_(rows, cols)]`` (reference:
        bigwham4py.py:462-484 over BigWhamIO::hmatSelection, which raises with
        CUDA): a LinearOperator over H[rows, cols] whose matvec runs on the GPU
        (selection.HmatSelection, the selected sub-blocks as a handle of their
        own).  rows / cols: element indices, original ordering, any shape (both
        are flattened; the reference's binding reads only the first dimension,
        py_bigwham.cc:262-268, so np.ix_'s 1 x m column array gives it one
        column).  Needs the host blocks: build with keep_host=True."""
        if not isinstance(indices, tuple) or len(indices) != 2:
            raise IndexError("Subsetting requires indices of the form (np.ix_(row_indices, col_indices))")
        self._build()
        rows, cols = (np.asarray(i).ravel() for i in indices)
        return BEMatrixSelection(self, rows, cols)

    def H_diag(self):
        return self.H_.get_diagonal()

    def H_jacobi_prec(self):
        """Jacobi preconditioner (bigwham4py.py:373-380)."""
        from scipy.sparse.linalg import LinearOperator

        inv = 1.0 / self.H_diag()
        return LinearOperator(self.shape, lambda v: inv * np.asarray(v).ravel(), dtype=float)


class BEMatrixSelection(_LinOp):
    """H[rows, cols] of a BEMatrix on the GPU (BEMatrix.__getitem__).  Made
    from a host copy of the base's blocks (export_blocks: as large as the
    H-matrix); once the selection's own handle is laid out only the
    full-rank part is kept (for _getFullBlocks)."""

    def __init__(self, parent: "BEMatrix", rows, cols):
        from .selection import HmatSelection

        io = parent.H_
        ex = io.export_blocks()
        precisions = tuple(io._precisions)
        self.parent = parent
        self.rows, self.cols = rows, cols
        if io.use_cuda:
            self.S_ = HmatSelection(ex, rows, cols, device=io.device, precisions=precisions)
        else:  # a host build: the selection's plan only (no GPU H-matrix to apply)
            self.S_ = HmatSelection(ex, rows, cols, device=-1, precisions=precisions, plan_only=True)
        super().__init__(np.dtype(float), self.S_.shape)

    def _matvec(self, v):
        return self.S_.matvec(np.asarray(v, dtype=np.float64).ravel())

    def _matvec_torch(self, x, y):
        """y = H[rows, cols] x on CUDA float64 torch tensors."""
        self.S_.matvec(x, out=y)

    def _getFullBlocks(self, keep_ratio: float = 1.0):
        """The selection's full-rank entries as a scipy CSC matrix (the
        reference's GetFullBlocks on the selection, hmat_selection.cc:265-375)."""
        if not (0 < keep_ratio <= 1):
            raise ValueError("ratio must be a float between 0 and 1.")
        val, pos = self.S_.full_blocks()
        return _csc_entries(val, pos[:, 0], pos[:, 1], self.shape, keep_ratio)

    def H_ILU_prec(self, fill_factor=1, drop_tol=1e-3, keep_ratio=1.0):
        from scipy.sparse.linalg import LinearOperator, spilu

        ilu = spilu(self._getFullBlocks(keep_ratio=keep_ratio), fill_factor=fill_factor, drop_tol=drop_tol)
        return LinearOperator(self.shape, ilu.solve)

    def close(self) -> None:
        self.S_.close()


class BEMatrixRectangular(_LinOp):
    """scipy LinearOperator over the GPU H-matrix of a source mesh and a
    receiver mesh (reference: bigwham4py.BEMatrixRectangular)."""

    def __init__(self, kernel: str, coor_src, conn_src, coor_rec, conn_rec, properties, max_leaf_size: int = 100,
                 eta: float = 3.0, eps_aca: float = 1.0e-3, n_openMP_threads: int = 8, n_GPUs: int = 1,
                 directly_build: bool = True, verbose: bool = False, homogeneous_size_pattern: bool = False,
                 useCuda=True, fixed_rank=-1, precisions=("fp64",), transpose: bool = False, device: int = 0):
        self.kernel_ = kernel
        self.properties_ = properties
        self.max_leaf_size_, self.eta_, self.eps_aca_ = int(max_leaf_size), float(eta), float(eps_aca)
        self.n_openMP_threads_ = n_openMP_threads
        self.H_ = BigWhamIOGpu.rectangular(coor_src, conn_src, coor_rec, conn_rec, kernel, properties,
                                           n_openMP_threads, n_GPUs, verbose, homogeneous_size_pattern, useCuda,
                                           fixed_rank, device)
        self.H_.set_gpu_storage(precisions, transpose)
        self.built_ = False
        shape = (0, 0)
        if directly_build:
            self._build()
            shape = (self.H_.matrix_size(0), self.H_.matrix_size(1))
        else:
            self.H_.build_pattern(self.max_leaf_size_, self.eta_)
        self.dtype_ = np.dtype(float)
        super().__init__(self.dtype_, shape)

    def _build(self):
        if not self.built_:
            self.H_.build_hierarchical_matrix(self.max_leaf_size_, self.eta_, self.eps_aca_)
            self.built_ = True
            self.matvec_size_ = self.H_.matrix_size(0)
            super().__init__(np.dtype(float), (self.H_.matrix_size(0), self.H_.matrix_size(1)))

    def _matvec(self, v):
        return self.H_.matvec(np.asarray(v, dtype=np.float64).ravel())

    def _rmatvec(self, v):
        if self.H_.gpu is None or not self.H_.gpu.has_transpose:
            raise RuntimeError("H^T not stored: build with transpose=True")
        return self.H_.gpu.rmatvec(np.asarray(v, dtype=np.float64).ravel())

    def getCompression(self) -> float:
        return self.H_.get_compression_ratio()

    def getPermutation(self):
        return self.H_.get_permutation()

    def getSpatialDimension(self):
        return self.H_.get_spatial_dimension()
