"""ctypes drivers for the two oracle libraries (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_REF_SO = os.path.join(_HERE, "_ref", "libbigwham_ref.so")
_ORACLE_SO = os.path.join(_HERE, "_lib", "libhmat_oracle.so")

_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def ref_available() -> bool:
    return os.path.exists(_REF_SO)


def oracle_available() -> bool:
    return os.path.exists(_ORACLE_SO)


@dataclass
class HmatArrays:
    """Flat copy of a built reference H-matrix.

    fr: (n_fr, 4) int64 rows (i0, j0, iend, jend) in collocation points.
    lr: (n_lr, 5) int64 rows (i0, j0, iend, jend, r), r = columns of A.
    fr_data: FR blocks back to back, each column-major m x n.
    lr_data: per LR block A (m x r) then B (r x n), column-major.
    perm0 / perm1: row / column permutations (HRepresentation, hierarchical_representation.h:28-29).
    """

    dof: int
    n_rows: int
    n_cols: int
    fr: np.ndarray
    lr: np.ndarray
    fr_data: np.ndarray
    lr_data: np.ndarray
    perm0: np.ndarray
    perm1: np.ndarray

    def save(self, path: str, **extra) -> None:
        np.savez_compressed(
            path, dof=self.dof, n_rows=self.n_rows, n_cols=self.n_cols, fr=self.fr, lr=self.lr,
            fr_data=self.fr_data, lr_data=self.lr_data, perm0=self.perm0, perm1=self.perm1, **extra)

    @staticmethod
    def load(path: str):
        z = np.load(path)
        h = HmatArrays(int(z["dof"]), int(z["n_rows"]), int(z["n_cols"]), z["fr"], z["lr"], z["fr_data"],
                       z["lr_data"], z["perm0"], z["perm1"])
        extra = {k: z[k] for k in z.files if k not in
                 ("dof", "n_rows", "n_cols", "fr", "lr", "fr_data", "lr_data", "perm0", "perm1")}
        return h, extra

    # iteration helpers used by tests
    def fr_blocks(self):
        o = 0
        for k in range(self.fr.shape[0]):
            i0, j0, i1, j1 = (int(v) for v in self.fr[k])
            m, n = (i1 - i0) * self.dof, (j1 - j0) * self.dof
            yield i0 * self.dof, j0 * self.dof, self.fr_data[o:o + m * n].reshape(n, m).T
            o += m * n

    def lr_blocks(self):
        o = 0
        for k in range(self.lr.shape[0]):
            i0, j0, i1, j1, r = (int(v) for v in self.lr[k])
            m, n = (i1 - i0) * self.dof, (j1 - j0) * self.dof
            A = self.lr_data[o:o + m * r].reshape(r, m).T
            o += m * r
            B = self.lr_data[o:o + r * n].reshape(n, r).T
            o += r * n
            yield i0 * self.dof, j0 * self.dof, A, B


# --------------------------------------------------------------------------- reference library
_ref_lib = None


def _ref():
    global _ref_lib
    if _ref_lib is None:
        if not ref_available():
            raise RuntimeError(f"reference library not built: {_REF_SO} (run make -C oracle ref)")
        lib = C.CDLL(_REF_SO)
        lib.ref_set_threads.argtypes = [C.c_int]
        lib.ref_set_threads.restype = C.c_int
        lib.ref_create.argtypes = [_f64p, C.c_int64, _i32p, C.c_int64, C.c_char_p, _f64p, C.c_int, C.c_int,
                                   C.c_int]
        lib.ref_create.restype = C.c_void_p
        lib.ref_create_rect.argtypes = [_f64p, C.c_int64, _i32p, C.c_int64, _f64p, C.c_int64, _i32p, C.c_int64,
                                        C.c_char_p, _f64p, C.c_int, C.c_int, C.c_int]
        lib.ref_create_rect.restype = C.c_void_p
        lib.ref_build.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
        lib.ref_size.argtypes = [C.c_void_p, C.c_int]
        lib.ref_size.restype = C.c_int64
        lib.ref_dof.argtypes = [C.c_void_p]
        lib.ref_compression.argtypes = [C.c_void_p]
        lib.ref_compression.restype = C.c_double
        lib.ref_n_blocks.argtypes = [C.c_void_p, C.c_int]
        lib.ref_n_blocks.restype = C.c_int64
        lib.ref_pattern.argtypes = [C.c_void_p, _i64p, _i64p]
        lib.ref_permutation.argtypes = [C.c_void_p, _i64p, _i64p]
        lib.ref_fr_block.argtypes = [C.c_void_p, C.c_int64, _f64p]
        lib.ref_lr_block.argtypes = [C.c_void_p, C.c_int64, _f64p, _f64p]
        lib.ref_matvec.argtypes = [C.c_void_p, _f64p, _f64p]
        lib.ref_matvec_perm.argtypes = [C.c_void_p, _f64p, _f64p]
        lib.ref_diagonal.argtypes = [C.c_void_p, _f64p]
        lib.ref_gaussian_create.argtypes = [C.c_int64, C.c_double, C.c_int, C.c_double, C.c_double, C.c_int]
        lib.ref_gaussian_create.restype = C.c_void_p
        lib.ref_gaussian_sizes.argtypes = [C.c_void_p, _i64p]
        lib.ref_gaussian_export.argtypes = [C.c_void_p, _i64p, _i64p, _f64p, _f64p, _i64p]
        lib.ref_gaussian_matvec_perm.argtypes = [C.c_void_p, _f64p, _f64p]
        lib.ref_gaussian_diagonal.argtypes = [C.c_void_p, _f64p]
        lib.ref_gaussian_destroy.argtypes = [C.c_void_p]
        lib.ref_selection_matvec.argtypes = [C.c_void_p, _i32p, C.c_int64, _i32p, C.c_int64, _f64p, _f64p]
        lib.ref_selection_full_blocks.argtypes = [C.c_void_p, _i32p, C.c_int64, _i32p, C.c_int64, C.c_void_p,
                                                  C.c_void_p, C.c_int64]
        lib.ref_selection_full_blocks.restype = C.c_int64
        lib.ref_collocation_points.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_dense_rows.argtypes = [C.c_void_p, C.c_char_p, _f64p, _i64p, C.c_int64, _f64p]
        lib.ref_collocation_points.restype = C.c_int64
        lib.ref_destroy.argtypes = [C.c_void_p]
        lib.ref_element_frames.argtypes = [C.c_void_p, _f64p]
        lib.ref_r0_stress.argtypes = [C.c_double] * 7 + [_f64p]
        lib.ref_r0_displacement.argtypes = [C.c_double] * 6 + [_f64p]
        _ref_lib = lib
    return _ref_lib


def ref_r0_stress(x, y, z, a, b, G, nu):
    """The reference's StressesKernelR0: (3, 6) stresses (rows DD x, y, z;
    columns xx, yy, zz, xy, xz, yz) at (x, y, z) in a rectangle's local frame."""
    out = np.zeros(18)
    if _ref().ref_r0_stress(x, y, z, a, b, G, nu, out) != 0:
        raise RuntimeError("ref_r0_stress failed")
    return out.reshape(3, 6)


def ref_r0_displacement(x, y, z, a, b, nu):
    """The reference's DisplacementKernelR0 as its 3 x 3 array."""
    out = np.zeros(9)
    if _ref().ref_r0_displacement(x, y, z, a, b, nu, out) != 0:
        raise RuntimeError("ref_r0_displacement failed")
    return out.reshape(3, 3)


class RefGaussian:
    """The reference's Gaussian-matrix H-matrix (its own cluster tree,
    pattern, GaussianMatrix generator and Hmat build, as
    src/hmat/hmatrix/_test/Hmat_test_gaussian_mat.cpp makes it): n points on
    a line, dof 1."""

    def __init__(self, n: int, alpha: float, leaf: int = 32, eta: float = 3.0, eps: float = 1e-3, n_threads: int = 4):
        lib = _ref()
        self._h = lib.ref_gaussian_create(int(n), float(alpha), int(leaf), float(eta), float(eps), int(n_threads))
        if not self._h:
            raise RuntimeError("reference Gaussian H-matrix construction failed")
        self.n = int(n)

    def __del__(self):
        if getattr(self, "_h", None) and _ref_lib is not None:
            _ref_lib.ref_gaussian_destroy(self._h)
            self._h = None

    def arrays(self) -> "HmatArrays":
        sz = np.zeros(4, np.int64)
        _ref().ref_gaussian_sizes(self._h, sz)
        fr, lr = np.zeros((sz[0], 4), np.int64), np.zeros((sz[1], 5), np.int64)
        fd, ld = np.zeros(max(1, sz[2])), np.zeros(max(1, sz[3]))
        perm = np.zeros(self.n, np.int64)
        _ref().ref_gaussian_export(self._h, fr, lr, fd, ld, perm)
        return HmatArrays(1, self.n, self.n, fr, lr, fd[:sz[2]], ld[:sz[3]], perm, perm.copy())

    def matvec_perm(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.n)
        _ref().ref_gaussian_matvec_perm(self._h, x, y)
        return y

    def diagonal(self):
        d = np.empty(self.n)
        _ref().ref_gaussian_diagonal(self._h, d)
        return d


class RefHmat:
    """The reference's BigWhamIO, built and applied by the reference's own code."""

    def __init__(self, kernel: str, coor, conn, properties, max_leaf_size=32, eta=3.0, eps_aca=1e-3,
                 n_threads=8, verbose=False):
        lib = _ref()
        self.n_threads = lib.ref_set_threads(int(n_threads))
        coor = np.ascontiguousarray(coor, dtype=np.float64).ravel()
        conn = np.ascontiguousarray(conn, dtype=np.int32).ravel()
        props = np.ascontiguousarray(properties, dtype=np.float64).ravel()
        self._h = lib.ref_create(coor, coor.size, conn, conn.size, kernel.encode(), props, props.size,
                                 int(n_threads), int(verbose))
        if not self._h:
            raise RuntimeError("reference BigWhamIO construction failed")
        rc = lib.ref_build(self._h, int(max_leaf_size), float(eta), float(eps_aca))
        if rc != 0:
            raise RuntimeError(f"reference BuildHierarchicalMatrix failed ({rc})")
        self.shape = (lib.ref_size(self._h, 0), lib.ref_size(self._h, 1))
        self.dof = lib.ref_dof(self._h)

    @classmethod
    def rectangular(cls, kernel: str, coor_src, conn_src, coor_rec, conn_rec, properties, max_leaf_size=32,
                    eta=3.0, eps_aca=1e-3, n_threads=8, verbose=False) -> "RefHmat":
        """The reference's rectangular BigWhamIO (receiver rows, source columns)."""
        lib = _ref()
        self = cls.__new__(cls)
        self.n_threads = lib.ref_set_threads(int(n_threads))
        a = [np.ascontiguousarray(v, dtype=t).ravel() for v, t in
             ((coor_src, np.float64), (conn_src, np.int32), (coor_rec, np.float64), (conn_rec, np.int32))]
        props = np.ascontiguousarray(properties, dtype=np.float64).ravel()
        self._h = lib.ref_create_rect(a[0], a[0].size, a[1], a[1].size, a[2], a[2].size, a[3], a[3].size,
                                      kernel.encode(), props, props.size, int(n_threads), int(verbose))
        if not self._h:
            raise RuntimeError("reference rectangular BigWhamIO construction failed")
        rc = lib.ref_build(self._h, int(max_leaf_size), float(eta), float(eps_aca))
        if rc != 0:
            raise RuntimeError(f"reference BuildHierarchicalMatrix failed ({rc})")
        self.shape = (lib.ref_size(self._h, 0), lib.ref_size(self._h, 1))
        self.dof = lib.ref_dof(self._h)
        return self

    def __del__(self):
        if getattr(self, "_h", None) and _ref_lib is not None:
            _ref_lib.ref_destroy(self._h)
            self._h = None

    def matvec(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.shape[0])
        _ref().ref_matvec(self._h, x, y)
        return y

    def matvec_perm(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.shape[0])
        _ref().ref_matvec_perm(self._h, x, y)
        return y

    def selection_matvec(self, rows, cols, x):
        """The reference's BigWhamIO::hmatSelection(rows, cols).MatVec(x)."""
        r = np.ascontiguousarray(rows, dtype=np.int32)
        c = np.ascontiguousarray(cols, dtype=np.int32)
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(r.size * self.dof)
        if _ref().ref_selection_matvec(self._h, r, r.size, c, c.size, x, y) != 0:
            raise IndexError("the reference rejected the selection")
        return y

    def selection_full_blocks(self, rows, cols):
        """(val, pos) of the selection's GetFullBlocks: val[i] = H_sel(pos[i, 0], pos[i, 1])."""
        r = np.ascontiguousarray(rows, dtype=np.int32)
        c = np.ascontiguousarray(cols, dtype=np.int32)
        n = _ref().ref_selection_full_blocks(self._h, r, r.size, c, c.size, None, None, 0)
        if n < 0:
            raise IndexError("the reference rejected the selection")
        val, pos = np.empty(n), np.empty(2 * n, dtype=np.int32)
        _ref().ref_selection_full_blocks(self._h, r, r.size, c, c.size, val.ctypes.data, pos.ctypes.data, n)
        return val, pos.reshape(n, 2)

    def diagonal(self):
        d = np.empty(max(self.shape))
        _ref().ref_diagonal(self._h, d)
        return d

    def compression(self) -> float:
        return _ref().ref_compression(self._h)

    def dense_rows(self, kernel: str, properties, points):
        """Rows of the dense FP64 operator (exact kernel, no H-matrix
        approximation) for the given collocation points, original ordering:
        (len(points) * dof, n_cols)."""
        lib = _ref()
        pts = np.ascontiguousarray(points, dtype=np.int64)
        props = np.ascontiguousarray(properties, dtype=np.float64)
        out = np.empty((pts.size * self.dof, self.shape[1]))
        rc = lib.ref_dense_rows(self._h, kernel.encode(), props, pts, pts.size, out)
        if rc != 0:
            raise RuntimeError(f"ref_dense_rows failed ({rc})")
        return out

    def element_frames(self):
        """(n_elements, 15): collocation point, row-major rotation matrix
        (local = R global) and unit normal of each element, from the
        reference's element objects (3D meshes, one collocation point per
        element)."""
        n = self.shape[1] // self.dof
        out = np.empty((n, 15))
        if _ref().ref_element_frames(self._h, out) != 0:
            raise RuntimeError("ref_element_frames failed")
        return out

    def collocation_points(self):
        lib = _ref()
        n = lib.ref_collocation_points(self._h, None)
        out = np.empty(n)
        lib.ref_collocation_points(self._h, out.ctypes.data)
        return out

    def arrays(self) -> HmatArrays:
        lib = _ref()
        nfr, nlr = lib.ref_n_blocks(self._h, 0), lib.ref_n_blocks(self._h, 1)
        fr = np.zeros((nfr, 4), np.int64)
        lr = np.zeros((nlr, 5), np.int64)
        lib.ref_pattern(self._h, fr, lr)
        p0 = np.zeros(self.shape[0] // self.dof, np.int64)
        p1 = np.zeros(self.shape[1] // self.dof, np.int64)
        lib.ref_permutation(self._h, p0, p1)
        d = self.dof
        fr_sizes = (fr[:, 2] - fr[:, 0]) * (fr[:, 3] - fr[:, 1]) * d * d
        lr_sizes = lr[:, 4] * ((lr[:, 2] - lr[:, 0]) + (lr[:, 3] - lr[:, 1])) * d
        fr_data = np.empty(int(fr_sizes.sum()))
        lr_data = np.empty(int(lr_sizes.sum()))
        o = 0
        for k in range(nfr):
            buf = np.empty(int(fr_sizes[k]))
            lib.ref_fr_block(self._h, k, buf)
            fr_data[o:o + buf.size] = buf
            o += buf.size
        o = 0
        for k in range(nlr):
            m = int((lr[k, 2] - lr[k, 0]) * d)
            n = int((lr[k, 3] - lr[k, 1]) * d)
            r = int(lr[k, 4])
            A = np.empty(m * r)
            B = np.empty(r * n)
            lib.ref_lr_block(self._h, k, A, B)
            lr_data[o:o + A.size] = A
            o += A.size
            lr_data[o:o + B.size] = B
            o += B.size
        return HmatArrays(d, self.shape[0], self.shape[1], fr, lr, fr_data, lr_data, p0, p1)


# --------------------------------------------------------------------------- C restatement
class _OHmat(C.Structure):
    _fields_ = [("dof", C.c_int32), ("pad_", C.c_int32), ("n_rows", C.c_int64), ("n_cols", C.c_int64),
                ("n_fr", C.c_int64), ("n_lr", C.c_int64), ("fr", C.c_void_p), ("lr", C.c_void_p),
                ("fr_data", C.c_void_p), ("lr_data", C.c_void_p), ("perm0", C.c_void_p), ("perm1", C.c_void_p)]


_or_lib = None


def _or():
    global _or_lib
    if _or_lib is None:
        if not oracle_available():
            raise RuntimeError(f"oracle restatement not built: {_ORACLE_SO} (run make -C oracle restatement)")
        lib = C.CDLL(_ORACLE_SO)
        for name in ("oracle_matvec_perm", "oracle_matvec", "oracle_rmatvec_perm", "oracle_rmatvec"):
            getattr(lib, name).argtypes = [C.POINTER(_OHmat), _f64p, _f64p, C.c_int]
        lib.oracle_matmat.argtypes = [C.POINTER(_OHmat), _f64p, _f64p, C.c_int64, C.c_int]
        lib.oracle_diagonal.argtypes = [C.POINTER(_OHmat), _f64p]
        lib.oracle_entries.argtypes = [C.POINTER(_OHmat)]
        lib.oracle_entries.restype = C.c_int64
        _or_lib = lib
    return _or_lib


def _struct(h: HmatArrays):
    keep = [np.ascontiguousarray(a) for a in (h.fr.astype(np.int64), h.lr.astype(np.int64), h.fr_data,
                                               h.lr_data, h.perm0.astype(np.int64), h.perm1.astype(np.int64))]
    s = _OHmat(h.dof, 0, h.n_rows, h.n_cols, h.fr.shape[0], h.lr.shape[0], *(a.ctypes.data for a in keep))
    return s, keep


def _call(name, h, x, nout, threads):
    s, keep = _struct(h)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty(nout)
    rc = getattr(_or(), name)(C.byref(s), x, y, int(threads))
    if rc:
        raise RuntimeError(f"{name} failed")
    return y


def oracle_matvec_perm(h: HmatArrays, x, threads=1):
    return _call("oracle_matvec_perm", h, x, h.n_rows, threads)


def oracle_matvec(h: HmatArrays, x, threads=1):
    return _call("oracle_matvec", h, x, h.n_rows, threads)


def oracle_rmatvec_perm(h: HmatArrays, x, threads=1):
    return _call("oracle_rmatvec_perm", h, x, h.n_cols, threads)


def oracle_rmatvec(h: HmatArrays, x, threads=1):
    return _call("oracle_rmatvec", h, x, h.n_cols, threads)


def oracle_matmat(h: HmatArrays, X, threads=1):
    """X: (n_cols, k) array; returns (n_rows, k)."""
    s, keep = _struct(h)
    X = np.asfortranarray(X, dtype=np.float64)
    k = X.shape[1]
    Xc = np.ascontiguousarray(X.T).ravel()
    Y = np.empty(h.n_rows * k)
    _or().oracle_matmat(C.byref(s), Xc, Y, k, int(threads))
    return Y.reshape(k, h.n_rows).T


def oracle_diagonal(h: HmatArrays):
    s, keep = _struct(h)
    d = np.empty(max(h.n_rows, h.n_cols))
    _or().oracle_diagonal(C.byref(s), d)
    return d


def oracle_entries(h: HmatArrays) -> int:
    s, keep = _struct(h)
    return int(_or().oracle_entries(C.byref(s)))
