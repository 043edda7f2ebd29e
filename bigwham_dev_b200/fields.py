"""Observation-point fields of a 2DS0 solution on the GPU.

The reference computes stresses and displacements at arbitrary points from a
displacement-discontinuity solution on the host (BigWhamIO::ComputeStresses /
ComputeDisplacements, src/io/bigwham_io.cc:1166-1324): a dense loop over
(source element, observation point) pairs, OpenMP over the source points.
Here the same dense sum runs in ``bw_s0_fields`` (one thread per observation
point, elements in mesh order; bw_s0.h holds the element's closed forms).

Outputs follow the reference's layout: per point (s11, s22, s12) and
(u1, u2), global frame; the solution is the local DD per element (shear,
normal), mesh order.  Stresses agree with the reference.  Displacements agree
except for u2 due to a shear DD: the reference's point kernel returns u1
there (bie_elastostatic_segment_0_influence.h:280-283); the values here are
the displacement field whose strains give the stresses (Hooke's law, plane
strain).
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


class S0Fields:
    """Stresses / displacements at points from a 2DS0 DD solution, on one GPU.

    coor, conn: the segment mesh; E, nu: Young's modulus and Poisson ratio
    (the reference's properties).  ``fields(points, dd)``: points (n, 2), dd
    (n_elems * 2, local shear / normal per element), numpy or CUDA float64
    tensors; returns (stress (n, 3), disp (n, 2)) of the same kind.
    """

    def __init__(self, coor, conn, E: float, nu: float, device: int = 0):
        import torch

        self.torch = torch
        self.device = int(device)
        self.G, self.nu = E / (2.0 * (1.0 + nu)), float(nu)
        rec = s0_records(coor, conn)
        self.n_elems = rec.shape[0]
        self.records = torch.from_numpy(rec).to(f"cuda:{self.device}")

    def fields(self, points, dd, want_stress: bool = True, want_disp: bool = True):
        torch = self.torch
        host = isinstance(points, np.ndarray)
        dev = f"cuda:{self.device}"
        p = torch.as_tensor(np.ascontiguousarray(points, dtype=np.float64) if host else points,
                            dtype=torch.float64, device=dev).reshape(-1, 2).contiguous()
        d = torch.as_tensor(np.ascontiguousarray(dd, dtype=np.float64) if isinstance(dd, np.ndarray) else dd,
                            dtype=torch.float64, device=dev).reshape(-1).contiguous()
        if d.numel() != 2 * self.n_elems:
            raise ValueError(f"dd has {d.numel()} values, the mesh {2 * self.n_elems} DDs")
        n = p.shape[0]
        s = torch.empty((n, 3), dtype=torch.float64, device=dev) if want_stress else None
        u = torch.empty((n, 2), dtype=torch.float64, device=dev) if want_disp else None
        A.check(A.lib().bw_s0_fields(self.device, self.n_elems, self.records.data_ptr(), d.data_ptr(), self.G,
                                     self.nu, n, p.data_ptr(), 0 if s is None else s.data_ptr(),
                                     0 if u is None else u.data_ptr(),
                                     torch.cuda.current_stream(self.device).cuda_stream), None)
        if host:
            return (None if s is None else s.cpu().numpy()), (None if u is None else u.cpu().numpy())
        return s, u
