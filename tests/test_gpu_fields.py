"""Observation-point fields on the GPU (-m gpu): s0_fields_kernel (2DS0) and
r0_fields_kernel (3DR0) through bw_s0_fields / bw_r0_fields.

Oracles, as on CPU (tests/test_fields_cpu.py):
* 2DS0 stresses: the reference's own BigWhamIO::ComputeStresses on a bent,
  unevenly meshed crack (src/io/bigwham_io.cc:1166-1324; cases below its
  OpenMP threshold, where its shared accumulation does not race), 1e-12 of
  the largest stress; displacements for normal DDs against
  ComputeDisplacements, 1e-12;
* 3DR0: the sums of the reference's element kernels StressesKernelR0 /
  DisplacementKernelR0 rotated to global (its BigWhamIO returns zeros for
  this family), 1e-12;
* at larger sizes (thousands of elements and points), the host build of the
  same device code (tests/cpp/fields_probe.cc) on a sample of the points,
  1e-12 of the largest value (the device's libm and FMA contraction differ
  from the host's in the last bits).
Also BEMatrix.compute_stresses / compute_displacements(device=True).
"""
import numpy as np
import pytest
from test_fields_cpu import (E, NU, bent_crack, host_fields, off_mesh_points, probe, r0_fields_host,  # noqa: F401
                             r0_reference_fields, ref_io, tilted_r0)

pytestmark = pytest.mark.gpu


def _close(a, b, tol=1e-12):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)) <= tol


def test_s0_fields_equal_the_reference(ref_io):
    from bigwham_dev_b200.fields import S0Fields

    io, coor, conn = ref_io
    f = S0Fields(coor, conn, E, NU, device=0)
    rng = np.random.default_rng(1)
    pts = off_mesh_points(rng, 200)
    dd = rng.uniform(-1, 1, 2 * len(conn))
    s, _ = f.fields(pts, dd)
    assert _close(s, io.compute_stresses(pts, dd).reshape(-1, 3))
    n = len(conn)
    ddn = np.zeros(2 * n)
    ddn[1::2] = rng.uniform(-1, 1, n)
    _, u = f.fields(pts, ddn)
    assert _close(u, io.compute_displacements(pts, ddn).reshape(-1, 2))


def test_s0_fields_at_scale_against_the_host_build(probe):
    """4,000 segments, 50,000 points (16 M element-point pairs per component)
    on the device; a 500-point sample against the host build."""
    import torch

    from bigwham_dev_b200.fields import S0Fields
    from bigwham_dev_b200.meshes import straight_crack_2d

    coor, conn = straight_crack_2d(4000)
    coor = np.asarray(coor, dtype=np.float64).reshape(-1, 2).copy()
    coor[:, 1] = 0.2 * np.sin(3.0 * coor[:, 0])  # bent: every element frame differs
    rng = np.random.default_rng(5)
    pts = off_mesh_points(rng, 50_000)
    dd = rng.uniform(-1, 1, 2 * len(conn))
    f = S0Fields(coor, conn, E, NU, device=0)
    s, u = f.fields(torch.from_numpy(pts).cuda(), torch.from_numpy(dd).cuda())
    torch.cuda.synchronize()
    pick = rng.choice(len(pts), 500, replace=False)
    hs, hu = host_fields(probe, coor, conn, dd, pts[pick])
    assert _close(s.cpu().numpy()[pick], hs) and _close(u.cpu().numpy()[pick], hu)
    # repeated launches give the same bits (each point sums the elements in mesh order)
    s2, _ = f.fields(torch.from_numpy(pts).cuda(), torch.from_numpy(dd).cuda())
    assert torch.equal(s, s2)


def test_r0_fields_equal_the_reference_element_kernels(tilted_r0):
    from oracle import ref_available

    from bigwham_dev_b200.fields import R0Fields

    if not ref_available():
        pytest.skip("oracle/_ref not built")
    rec = tilted_r0
    rng = np.random.default_rng(11)
    dd = rng.uniform(-1, 1, 3 * rec.shape[0])
    pts = rng.uniform(-1.5, 1.5, (25, 3))
    s, u = R0Fields(rec, E, NU, device=0).fields(pts, dd)
    ws, wu = r0_reference_fields(rec, dd, pts)
    assert _close(s, ws) and _close(u, wu)


def test_r0_fields_at_scale_against_the_host_build(probe):
    """3DR0 64 x 64 crack (4,096 elements), 20,000 points; a 200-point sample
    against the host build."""
    from bigwham_dev_b200.bigwham4py import BigWhamIOGpu
    from bigwham_dev_b200.fields import R0Fields
    from bigwham_dev_b200.meshes import square_crack_3d

    coor, conn = square_crack_3d(64)
    io = BigWhamIOGpu(coor, conn, "3DR0-H", [E, NU], 8, useCuda=False)
    rec = io.element_records()
    io.close()
    rng = np.random.default_rng(13)
    pts = rng.uniform(-1.5, 1.5, (20_000, 3))
    # at least 0.05 off the crack plane: the closed forms cancel near it, and
    # the last-bit differences of the two builds' libm would be amplified
    pts[:, 2] = np.where(pts[:, 2] < 0, np.minimum(pts[:, 2], -0.05), np.maximum(pts[:, 2], 0.05))
    dd = rng.uniform(-1, 1, 3 * rec.shape[0])
    s, u = R0Fields(rec, E, NU, device=0).fields(pts, dd)
    pick = rng.choice(len(pts), 200, replace=False)
    hs, hu = r0_fields_host(probe, rec, dd, pts[pick])
    assert _close(s[pick], hs) and _close(u[pick], hu)


def test_bematrix_device_fields_equal_the_host_path():
    """BEMatrix(...).compute_stresses(device=True) against the reference's
    host ComputeStresses of the same object (2DS0-H)."""
    from bigwham_dev_b200.bigwham4py import BEMatrix

    coor, conn = bent_crack(80, seed=4)
    A = BEMatrix("2DS0-H", coor, conn, [E, NU], max_leaf_size=16, eta=2.0, eps_aca=1e-4, n_openMP_threads=1)
    rng = np.random.default_rng(6)
    pts = off_mesh_points(rng, 150)
    dd = rng.uniform(-1, 1, 2 * len(conn))
    assert _close(A.compute_stresses(pts, dd, device=True), A.compute_stresses(pts, dd))
    ddn = np.zeros_like(dd)
    ddn[1::2] = dd[1::2]
    assert _close(A.compute_displacements(pts, ddn, device=True), A.compute_displacements(pts, ddn))
