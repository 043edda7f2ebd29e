"""Building a 3DR0-H H-matrix's blocks on the GPU (-m gpu): r0_fr_assemble_kernel
(bw_r0_assemble_fr), r0_aca_kernel (bw_r0_aca), and the device layout of
device-resident blocks (bw_add_flat_device: block_maxabs_kernel,
pack_runs_kernel, diag_kernel).

Against the reference's own build of the same mesh (BuildHierarchicalMatrix:
Hmat::buildFR / buildLR, src/hmat/hmatrix/hmat.cc:315-416, block ACA
src/hmat/compression/adaptiveCrossApproximation.h:24-226):
* full-rank blocks from the reference's pattern: 1e-13 of the largest entry;
* low-rank blocks: the device ACA against the host build of the same ACA
  (tests/cpp/r0_probe.cc): the same ranks on >= 95% of the blocks, and where
  the ranks agree the products A B within 1e-9 of the block's norm;
* the whole device build (devbuild.build_r0): the reference's pattern and
  permutations, full-rank data to 1e-13, >= 90% of its ranks, and a matvec as
  close to the exact operator (every entry evaluated by the reference's
  kernel) as the reference's H-matrix, within 1.5x;
* the device layout of the device-resident blocks equals the host layout of
  the same blocks: bitwise-equal matvecs in FP64, FP32 and BF16, and the same
  diagonal.
"""
import numpy as np
import pytest
from test_devbuild_cpu import HostKernels

from bigwham_dev_b200 import HmatGpu
from bigwham_dev_b200.bigwham4py import BigWhamIOGpu
from bigwham_dev_b200.devbuild import DeviceKernels, build_r0, ex_args, factor_layout
from bigwham_dev_b200.meshes import square_crack_3d
from oracle import HmatArrays, RefHmat, oracle_matvec_perm

pytestmark = pytest.mark.gpu

E, NU, EPS = 1.0, 0.25, 1e-5
G = E / (2.0 * (1.0 + NU))


def _reference_build(n):
    coor, conn = square_crack_3d(n)
    io = BigWhamIOGpu(coor, conn, "3DR0-H", [E, NU], 8, useCuda=False)
    io.build_hierarchical_matrix(32, 3.0, EPS)
    ref = io.export_blocks()
    rec = io.element_records()
    io.close()
    return coor, conn, ref, rec


def test_fr_assembly_equals_the_reference_blocks():
    coor, conn, ref, rec = _reference_build(16)
    out = DeviceKernels(0).assemble_fr(rec, G, NU, ref["fr"], ref["perm1"]).cpu().numpy()
    assert out.shape == ref["fr_data"].shape
    assert np.abs(out - ref["fr_data"]).max() <= 1e-13 * np.abs(ref["fr_data"]).max()


def test_device_aca_equals_the_host_build_of_the_same_aca():
    coor, conn, ref, rec = _reference_build(24)
    lr4 = np.ascontiguousarray(ref["lr"][:, :4])
    perm = ref["perm1"]
    cap = 64
    fa, fb, rk, er = DeviceKernels(0).aca(rec, G, NU, lr4, perm, EPS, cap)
    ha, hb, hrk, her = HostKernels().aca(rec, G, NU, lr4, perm, EPS, cap)
    fa, fb = fa.cpu().numpy(), fb.cpu().numpy()
    assert np.all(rk > 0)
    same = rk == hrk
    assert np.mean(same) >= 0.95, np.mean(same)
    n0, n1, capk, a_off, b_off = factor_layout(lr4, cap)
    for q in np.nonzero(same)[0]:
        r, m, n, c = int(rk[q]), 3 * int(n0[q]), 3 * int(n1[q]), 3 * int(capk[q])
        Ad = fa[a_off[q]:a_off[q] + m * r].reshape(r, m).T
        Bd = fb[b_off[q]:b_off[q + 1]].reshape(n, c)[:, :r].T
        Ah = ha[a_off[q]:a_off[q] + m * r].reshape(r, m).T
        Bh = hb[b_off[q]:b_off[q + 1]].reshape(n, c)[:, :r].T
        P = Ah @ Bh
        assert np.linalg.norm(Ad @ Bd - P) <= 1e-9 * np.linalg.norm(P), q
    # the reference's own ranks (its ACA on the host): most blocks agree
    assert np.mean(rk == ref["lr"][:, 4]) >= 0.9


def test_device_build_matches_the_reference_build():
    import torch

    coor, conn, ref, _ = _reference_build(24)
    io = BigWhamIOGpu(coor, conn, "3DR0-H", [E, NU], 8, useCuda=False)
    ex = build_r0(io, 32, 3.0, EPS, E, NU, cap_blocks=2)  # capacity 2: retries with 4, 8, ...
    io.close()
    assert np.array_equal(ex["fr"], ref["fr"]) and np.array_equal(ex["lr"][:, :4], ref["lr"][:, :4])
    assert np.array_equal(ex["perm0"], ref["perm0"]) and np.array_equal(ex["perm1"], ref["perm1"])
    assert np.abs(ex["fr_data"] - ref["fr_data"]).max() <= 1e-13 * np.abs(ref["fr_data"]).max()
    assert np.mean(ex["lr"][:, 4] == ref["lr"][:, 4]) >= 0.9
    # operator accuracy against the exact operator, beside the reference's
    R = RefHmat("3DR0-H", coor, conn, [E, NU], 32, 3.0, EPS, n_threads=8)
    n = ex["n_rows"]
    dense = R.dense_rows("3DR0-H", [E, NU], np.arange(n // 3))  # original ordering
    x = np.random.default_rng(3).uniform(-1, 1, n)
    y_exact = dense @ x
    h = HmatGpu.from_flat(**ex_args(ex), device=0, precisions=("fp64",))
    mine = np.linalg.norm(h.matvec(x) - y_exact) / np.linalg.norm(y_exact)
    d = 3
    xp = x[(d * np.asarray(ref["perm1"])[:, None] + np.arange(d)).ravel()]
    arr = HmatArrays(ref["dof"], ref["n_rows"], ref["n_cols"], ref["fr"], ref["lr"], ref["fr_data"], ref["lr_data"],
                     ref["perm0"], ref["perm1"])
    yp = oracle_matvec_perm(arr, xp, 8)
    y_ref = np.empty_like(yp)
    y_ref[(d * np.asarray(ref["perm0"])[:, None] + np.arange(d)).ravel()] = yp
    theirs = np.linalg.norm(y_ref - y_exact) / np.linalg.norm(y_exact)
    print(f"devbuild 24x24: operator error {mine:.3e} (reference {theirs:.3e})")
    assert mine <= 1.5 * theirs + 1e-12, (mine, theirs)
    assert mine < 1e-4
    h.close()
    torch.cuda.synchronize()


def test_device_layout_equals_the_host_layout():
    """64 x 64 crack (12,288 DoF) built on the device and laid out on the
    device (the host never reads the blocks) against the host layout of the
    same blocks: the same bits in every precision, forward and transposed."""
    import torch

    coor, conn = square_crack_3d(64)
    io = BigWhamIOGpu(coor, conn, "3DR0-H", [E, NU], 8, useCuda=False)
    exd = build_r0(io, 32, 3.0, EPS, E, NU, on_device=True)
    io.close()
    precs = ("fp64", "fp32", "bf16")
    h_dev = HmatGpu.from_device_flat(**ex_args(exd), device=0, precisions=precs, transpose=True)
    exh = dict(exd, fr_data=exd["fr_data"].cpu().numpy(), lr_data=exd["lr_data"].cpu().numpy())
    h_host = HmatGpu.from_flat(**ex_args(exh), device=0, precisions=precs, transpose=True)
    assert np.array_equal(h_dev.diagonal(), h_host.diagonal())
    x = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, exd["n_cols"])).cuda()
    for p in precs:
        assert torch.equal(h_dev.matvec(x, p), h_host.matvec(x, p)), p
        assert torch.equal(h_dev.rmatvec(x, p), h_host.rmatvec(x, p)), p
    torch.cuda.synchronize()
    h_dev.close()
    h_host.close()
