"""Building a 3DR0-H H-matrix's blocks on the device.

The reference builds every block on the host (Hmat::build,
src/hmat/hmatrix/hmat.cc:290-416): full-rank blocks entry by entry (buildFR)
and low-rank blocks by block ACA (buildLR, adaptiveCrossApproximation<3>).
Here the host keeps only what is sequential and cheap, the cluster tree and
the block pattern (BigWhamIO::BuildPattern, src/io/bigwham_io.cc:487-511),
and the device computes the blocks:
* full-rank blocks with bw_r0_assemble_fr;
* low-rank blocks with bw_r0_aca: each block gets room for `cap_blocks` rank
  blocks (3 scalar columns each); blocks that need more are redone with twice
  the room until they fit (a block's rank never exceeds its side).
The result is the flat form of BigWhamIOGpu.export_blocks (plus the ACA error
estimates), ready for HmatGpu.from_flat or blockfile.write.

    io = BigWhamIOGpu(coor, conn, "3DR0-H", [E, nu], useCuda=False)
    ex = build_r0(io, 32, 3.0, 1e-5, E, nu)
    h = HmatGpu.from_flat(**ex_args(ex), precisions=("fp64", "bf16"))
"""
from __future__ import annotations

import numpy as np

from . import _capi as A


def factor_layout(lr4, cap_blocks: int):
    """Capacity (rank blocks) and storage offsets of each low-rank block, as
    bw_r0_aca lays them out: A_k (rows 3 x cap 3) then B_k (cap 3 x cols 3)."""
    lr4 = np.asarray(lr4, dtype=np.int64).reshape(-1, 4)
    n0, n1 = lr4[:, 2] - lr4[:, 0], lr4[:, 3] - lr4[:, 1]
    cap = np.minimum(cap_blocks, np.minimum(n0, n1))
    a_size, b_size = 9 * n0 * cap, 9 * n1 * cap
    a_off = np.concatenate([[0], np.cumsum(a_size)])
    b_off = np.concatenate([[0], np.cumsum(b_size)])
    return n0, n1, cap, a_off, b_off


class DeviceKernels:
    """The device entries, on CUDA float64 tensors of one device."""

    def __init__(self, device: int = 0):
        import torch

        self.torch, self.device = torch, int(device)
        self.lib = A.lib()

    def _stream(self):
        return self.torch.cuda.current_stream(self.device).cuda_stream

    def assemble_fr(self, records, G, nu, fr, perm):
        torch = self.torch
        fr = np.ascontiguousarray(fr, dtype=np.int64).reshape(-1, 4)
        total = int((9 * (fr[:, 2] - fr[:, 0]) * (fr[:, 3] - fr[:, 1])).sum())
        out = torch.empty(max(1, total), dtype=torch.float64, device=f"cuda:{self.device}")
        A.check(self.lib.bw_r0_assemble_fr(self.device, records.shape[0], records.ctypes.data, G, nu, fr.shape[0],
                                           fr.ctypes.data, perm.ctypes.data, perm.size, out.data_ptr(), out.numel(),
                                           self._stream()), None)
        return out[:total]

    def aca(self, records, G, nu, lr4, perm, eps, cap_blocks):
        torch = self.torch
        lr4 = np.ascontiguousarray(lr4, dtype=np.int64).reshape(-1, 4)
        _, _, _, a_off, b_off = factor_layout(lr4, cap_blocks)
        fa = torch.empty(max(1, int(a_off[-1])), dtype=torch.float64, device=f"cuda:{self.device}")
        fb = torch.empty(max(1, int(b_off[-1])), dtype=torch.float64, device=f"cuda:{self.device}")
        ranks = np.zeros(lr4.shape[0], dtype=np.int32)
        errs = np.zeros(lr4.shape[0])
        A.check(self.lib.bw_r0_aca(self.device, records.shape[0], records.ctypes.data, G, nu, lr4.shape[0],
                                   lr4.ctypes.data, perm.ctypes.data, perm.size, eps, int(cap_blocks), fa.data_ptr(),
                                   fa.numel(), fb.data_ptr(), fb.numel(), ranks.ctypes.data, errs.ctypes.data,
                                   self._stream()), None)
        return fa, fb, ranks, errs


def _cat(parts):
    if parts and not isinstance(parts[0], np.ndarray):
        import torch

        return torch.cat(parts)
    return np.concatenate(parts) if parts else np.zeros(0)


def _host(a):
    return a if isinstance(a, np.ndarray) else a.cpu().numpy()


def build_r0(io, max_leaf_size: int, eta: float, eps_aca: float, E: float, nu: float, device: int = 0,
             cap_blocks: int = 48, kernels=None, on_device: bool = False) -> dict:
    """Blocks of the 3DR0-H H-matrix of `io` (a BigWhamIOGpu of a rectangle
    mesh) built on the device; returns the flat form with "lr_error".  The
    block data are numpy arrays, or (on_device) CUDA tensors for
    HmatGpu.from_device_flat.  kernels: an object with the methods of
    DeviceKernels (default: the CUDA entries on `device`)."""
    kernels = kernels or DeviceKernels(device)
    io.build_pattern(max_leaf_size, eta)
    pat = io.get_hpattern()
    fr = np.ascontiguousarray(pat[pat[:, 4] == 0, :4], dtype=np.int64)
    lr4 = np.ascontiguousarray(pat[pat[:, 4] == 1, :4], dtype=np.int64)
    n_pts = int(io._L.bwh_collocation_points(io._h, None)) // 3
    perm = np.empty(n_pts, dtype=np.int64)
    if io._L.bwh_permutation(io._h, perm.ctypes.data) != 0:
        raise RuntimeError("bwh_permutation failed")
    records = io.element_records()
    G = E / (2.0 * (1.0 + nu))
    fr_data = kernels.assemble_fr(records, G, nu, fr, perm)
    # low-rank blocks, redoing the ones that outgrow their room
    n_lr = lr4.shape[0]
    ranks = np.full(n_lr, -1, dtype=np.int64)
    errs = np.zeros(n_lr)
    parts = [None] * n_lr
    todo = np.arange(n_lr)
    cap = int(cap_blocks)
    while todo.size:
        sub = lr4[todo]
        fa, fb, r_sub, e_sub = kernels.aca(records, G, nu, sub, perm, eps_aca, cap)
        n0, n1, capk, a_off, b_off = factor_layout(sub, cap)
        for q, k in enumerate(todo):
            r = int(r_sub[q])
            if r < 0:
                continue
            lda, c3 = 3 * int(n0[q]), 3 * int(capk[q])
            a_part = fa[int(a_off[q]):int(a_off[q]) + r * lda]
            b_part = fb[int(b_off[q]):int(b_off[q + 1])].reshape(3 * int(n1[q]), c3)[:, :r].reshape(-1)
            parts[k] = (a_part, b_part)
            ranks[k], errs[k] = r, e_sub[q]
        todo = todo[np.asarray(r_sub) < 0]
        cap *= 2
    lr_data = _cat([p for ab in parts for p in ab])
    d = 3
    if on_device:
        fr_out, lr_out = fr_data.contiguous(), lr_data.contiguous()
    else:
        fr_out, lr_out = np.ascontiguousarray(_host(fr_data)), np.ascontiguousarray(_host(lr_data))
    return {"dof": d, "n_rows": d * n_pts, "n_cols": d * n_pts, "fr": fr,
            "lr": np.column_stack([lr4, ranks]).astype(np.int64).reshape(-1, 5),
            "fr_data": fr_out, "lr_data": lr_out, "perm0": perm, "perm1": perm.copy(), "lr_error": errs}


def ex_args(ex: dict) -> dict:
    """The arguments of HmatGpu.from_flat from a flat form."""
    return {k: ex[k] for k in ("dof", "n_rows", "n_cols", "fr", "lr", "fr_data", "lr_data", "perm0", "perm1")}


def main(argv=None) -> int:
    """python -m bigwham_dev_b200.devbuild --mesh 64: build the 3DR0-H square
    crack's blocks on the device and with the reference's host code, print
    both build times and the relative difference of their FP64 matvecs."""
    import argparse
    import json
    import time

    import torch

    from .bigwham4py import BigWhamIOGpu
    from .hmat import HmatGpu
    from .meshes import square_crack_3d

    ap = argparse.ArgumentParser()
    ap.add_argument("--mesh", type=int, default=64)
    ap.add_argument("--eps", type=float, default=1e-5)
    ap.add_argument("--cap", type=int, default=48)
    a = ap.parse_args(argv)
    E, nu = 1.0, 0.25
    coor, conn = square_crack_3d(a.mesh)
    io = BigWhamIOGpu(coor, conn, "3DR0-H", [E, nu], useCuda=False)
    torch.cuda.synchronize()
    t0 = time.time()
    exd = build_r0(io, 32, 3.0, a.eps, E, nu, cap_blocks=a.cap, on_device=True)
    torch.cuda.synchronize()
    t_dev = time.time() - t0
    t0 = time.time()
    h0 = HmatGpu.from_device_flat(**ex_args(exd), precisions=("fp64",))
    torch.cuda.synchronize()
    t_dev_layout = time.time() - t0
    ex = dict(exd, fr_data=exd["fr_data"].cpu().numpy(), lr_data=exd["lr_data"].cpu().numpy())
    io.close()
    io = BigWhamIOGpu(coor, conn, "3DR0-H", [E, nu], useCuda=False)
    t0 = time.time()
    io.build_hierarchical_matrix(32, 3.0, a.eps)
    t_host = time.time() - t0
    ref = io.export_blocks()
    io.close()
    x = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, ex["n_cols"])).cuda()
    h1 = HmatGpu.from_flat(**ex_args(ex), precisions=("fp64",))
    h2 = HmatGpu.from_flat(**ex_args(ref), precisions=("fp64",))
    y1, y2, y0 = h1.matvec(x), h2.matvec(x), h0.matvec(x)
    torch.cuda.synchronize()
    print(json.dumps({"mesh": a.mesh, "dof": ex["n_rows"], "device_build_s": round(t_dev, 3),
                      "device_layout_s": round(t_dev_layout, 3),
                      "device_layout_vs_host_layout_max_diff": float(torch.max(torch.abs(y0 - y1))),
                      "host_build_s": round(t_host, 3), "lr_entries": [int(ex["lr_data"].size), int(ref["lr_data"].size)],
                      "matvec_rel_diff": float(torch.linalg.vector_norm(y1 - y2) / torch.linalg.vector_norm(y2))}))
    return 0


if __name__ == "__main__":
    import sys

    sys.exit(main())
