"""Observation-point fields of a 2DS0 or 3DR0 solution on the GPU.

The reference computes stresses and displacements at arbitrary points from a
displacement-discontinuity solution on the host (BigWhamIO::ComputeStresses /
ComputeDisplacements, src/io/bigwham_io.cc:1166-1324): a dense loop over
(source element, observation point) pairs, OpenMP over the source points.
Here the same dense sum runs in ``bw_s0_fields`` (one thread per observation
point, elements in mesh order; bw_s0.h holds the element's closed forms).

2DS0 (``S0Fields``, bw_s0_fields): per point (s11, s22, s12) and (u1, u2),
global frame, from the local DD per element (shear, normal), mesh order.
Stresses agree with the reference.  Displacements agree except for u2 due to
a shear DD: the reference's point kernel returns u1 there
(bie_elastostatic_segment_0_influence.h:280-283); the values here are the
displacement field whose strains give the stresses (Hooke's law, plane
strain).

3DR0 (``R0Fields``, bw_r0_fields): per point (s11, s22, s33, s12, s13, s23)
and (u1, u2, u3), from the local DD per element (d1, d2 in the plane, d3
normal).  The reference's BigWhamIO returns zeros here (its 3DR0 observation
kernels are stubs, bie_elastostatic_rectangle_0_influence.h:222-245); these
are the sums of its element kernels StressesKernelR0 / DisplacementKernelR0,
in the layout of its 3D observation kernels.
"""
from __future__ import annotations

import numpy as np

from . import _capi as A


def s0_records(coor, conn) -> np.ndarray:
    """(n_elems, 5) element records: centre, half length, unit tangent from
    the first vertex to the second (src/elements/segment.h:70-90)."""
    coor = np.asarray(coor, dtype=np.float64).reshape(-1, 2)
    conn = np.asarray(conn, dtype=np.int64).reshape(-1, 2)
    v0, v1 = coor[conn[:, 0]], coor[conn[:, 1]]
    t = v1 - v0
    h = np.sqrt(np.einsum("ij,ij->i", t, t))
    if np.any(h <= 0):
        raise ValueError("zero-length element")
    return np.ascontiguousarray(np.column_stack([0.5 * (v0 + v1), 0.5 * h, t / h[:, None]]))


class _Fields:
    """Device plumbing shared by the element families: records on the device,
    points and DDs moved there, one launch, outputs back in the input's kind."""

    entry = ""
    dim = 0        # coordinates per point
    dof = 0        # DD components per element
    n_stress = 0   # stress components per point

    def _setup(self, records, E: float, nu: float, device: int):
        import torch

        self.torch = torch
        self.device = int(device)
        self.G, self.nu = E / (2.0 * (1.0 + nu)), float(nu)
        self.n_elems = records.shape[0]
        self.records = torch.from_numpy(np.ascontiguousarray(records, dtype=np.float64)).to(f"cuda:{self.device}")

    def fields(self, points, dd, want_stress: bool = True, want_disp: bool = True):
        torch = self.torch
        host = not torch.is_tensor(points)  # numpy arrays, lists: numpy results
        dev = f"cuda:{self.device}"
        p = torch.as_tensor(np.ascontiguousarray(points, dtype=np.float64) if host else points,
                            dtype=torch.float64, device=dev).reshape(-1, self.dim).contiguous()
        d = torch.as_tensor(dd if torch.is_tensor(dd) else np.ascontiguousarray(dd, dtype=np.float64),
                            dtype=torch.float64, device=dev).reshape(-1).contiguous()
        if d.numel() != self.dof * self.n_elems:
            raise ValueError(f"dd has {d.numel()} values, the mesh {self.dof * self.n_elems} DDs")
        n = p.shape[0]
        s = torch.empty((n, self.n_stress), dtype=torch.float64, device=dev) if want_stress else None
        u = torch.empty((n, self.dim), dtype=torch.float64, device=dev) if want_disp else None
        A.check(getattr(A.lib(), self.entry)(self.device, self.n_elems, self.records.data_ptr(), d.data_ptr(),
                                             self.G, self.nu, n, p.data_ptr(), 0 if s is None else s.data_ptr(),
                                             0 if u is None else u.data_ptr(),
                                             torch.cuda.current_stream(self.device).cuda_stream), None)
        if host:
            return (None if s is None else s.cpu().numpy()), (None if u is None else u.cpu().numpy())
        return s, u


class S0Fields(_Fields):
    """Stresses / displacements at points from a 2DS0 DD solution, on one GPU.

    coor, conn: the segment mesh; E, nu: Young's modulus and Poisson ratio
    (the reference's properties).  ``fields(points, dd)``: points (n, 2), dd
    (n_elems * 2, local shear / normal per element), numpy or CUDA float64
    tensors; returns (stress (n, 3), disp (n, 2)) of the same kind.
    """

    entry, dim, dof, n_stress = "bw_s0_fields", 2, 2, 3

    def __init__(self, coor, conn, E: float, nu: float, device: int = 0):
        self._setup(s0_records(coor, conn), E, nu, device)


class R0Fields(_Fields):
    """Stresses / displacements at points from a 3DR0 DD solution, on one GPU.

    records: (n_elems, 17) element records (BigWhamIOGpu.element_records);
    ``fields(points, dd)``: points (n, 3), dd (n_elems * 3, local DDs);
    returns (stress (n, 6), disp (n, 3)).
    """

    entry, dim, dof, n_stress = "bw_r0_fields", 3, 3, 6

    def __init__(self, records, E: float, nu: float, device: int = 0):
        records = np.asarray(records, dtype=np.float64)
        if records.ndim != 2 or records.shape[1] != 17:
            raise ValueError("records: (n_elems, 17)")
        self._setup(records, E, nu, device)
