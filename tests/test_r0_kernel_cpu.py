"""The rectangular-element kernel restated in bigwham_dev_b200/csrc/bw_r0.h
(host build of the header) against the reference's own StressesKernelR0 and
DisplacementKernelR0 (compiled from its sources into the oracle library).

Points: off the element plane at random; in the plane (z = 0, the case of
every entry of a planar crack) at random, at the offsets of a uniform mesh
(self-effect included), and on the lines of the element's edges beyond the
element, where the reference uses limit forms.

Bars, relative to the largest entry of each 3 x 6 / 3 x 3 block:
* against a 40-digit evaluation of the same closed forms (mpmath): 1e-11;
* against the reference: 1e-11 in the element plane, 2e-9 off it.  The
  reference itself is off by up to 9e-10 there (terms such as
  2 I_xz - z I_xxx cancel at small z), while this header stays within
  4e-12 of the 40-digit values.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from oracle import ref_available
from oracle.pyoracle import ref_r0_displacement, ref_r0_stress

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.skipif(not ref_available(), reason="reference library not built")
TOL = 1e-11
TOL_REF_OFFPLANE = 2e-9


@pytest.fixture(scope="module")
def probe():
    out = os.path.join(ROOT, "_build", "libr0_probe.so")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    subprocess.run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-I", os.path.join(ROOT, "bigwham_dev_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "r0_probe.cc"), "-o", out], check=True)
    lib = C.CDLL(out)
    p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    lib.probe_r0_stress.argtypes = [C.c_double] * 7 + [p]
    lib.probe_r0_displacement.argtypes = [C.c_double] * 6 + [p]
    lib.probe_r0_influence.argtypes = [p, C.c_double, C.c_double, p, C.c_double, C.c_double, p]

    def stress(*a):
        o = np.zeros(18)
        lib.probe_r0_stress(*a, o)
        return o.reshape(3, 6)

    def disp(*a):
        o = np.zeros(9)
        lib.probe_r0_displacement(*a, o)
        return o.reshape(3, 3)

    lib.probe_r0_fr_blocks.argtypes = [p, C.c_double, C.c_double, C.c_longlong,
                                       np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS"),
                                       np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS"), p]

    class Probe(tuple):
        influence = staticmethod(lib.probe_r0_influence)
        fr_blocks = staticmethod(lib.probe_r0_fr_blocks)

    return Probe((stress, disp))


def _err(mine, ref):
    return float(np.max(np.abs(mine - ref)) / np.max(np.abs(ref)))


def _check(probe, pts, G=1.3, nu=0.27, disp=True, tol=TOL):
    stress, displacement = probe
    for x, y, z, a, b in pts:
        sr = ref_r0_stress(x, y, z, a, b, G, nu)
        assert np.all(np.isfinite(sr)), (x, y, z, a, b)
        assert _err(stress(x, y, z, a, b, G, nu), sr) < tol, (x, y, z, a, b)
        if disp:
            ur = ref_r0_displacement(x, y, z, a, b, nu)
            assert _err(displacement(x, y, z, a, b, nu), ur) < tol, (x, y, z, a, b)


def _truth_stress(x, y, z, a, b, G, nu):
    """The closed forms of bw_r0.h evaluated with 40 significant digits."""
    import mpmath as mp

    mp.mp.dps = 40
    x, y, z, a, b, G, nu = (mp.mpf(v) for v in (x, y, z, a, b, G, nu))
    D = dict.fromkeys(["xx", "yy", "zz", "xy", "xz", "yz", "xxx", "yyy", "xxy", "xyy", "xxz", "yyz", "xzz", "yzz",
                       "xyz"], mp.mpf(0))
    for sx in (1, -1):
        for sy in (1, -1):
            s, X, Y = sx * sy, x + sx * a, y + sy * b
            R = mp.sqrt(X * X + Y * Y + z * z)
            R3 = R ** 3
            D["xx"] += s * X / (R * (R + Y))
            D["yy"] += s * Y / (R * (R + X))
            D["xy"] += s / R
            D["xz"] += s * z / (R * (R + Y))
            D["yz"] += s * z / (R * (R + X))
            D["zz"] += s * X * Y * (X * X + Y * Y + 2 * z * z) / (R * (X * X + z * z) * (Y * Y + z * z))
            D["xxy"] -= s * X / R3
            D["xyy"] -= s * Y / R3
            D["xyz"] -= s * z / R3
            D["xxx"] += s * (R * (R + Y) - X * X * (2 * R + Y) / R) / (R * R * (R + Y) ** 2)
            D["yyy"] += s * (R * (R + X) - Y * Y * (2 * R + X) / R) / (R * R * (R + X) ** 2)
            D["xxz"] -= s * X * z * (2 * R + Y) / (R3 * (R + Y) ** 2)
            D["yyz"] -= s * Y * z * (2 * R + X) / (R3 * (R + X) ** 2)
            D["xzz"] += s * (R * (R + Y) - z * z * (2 * R + Y) / R) / (R * R * (R + Y) ** 2)
            D["yzz"] += s * (R * (R + X) - z * z * (2 * R + X) / R) / (R * R * (R + X) ** 2)
    zzz = -(D["xxz"] + D["yyz"])
    c = G / (4 * mp.pi * (1 - nu))
    S = [[2 * D["xz"] - z * D["xxx"], 2 * nu * D["xz"] - z * D["xyy"], -z * D["xzz"],
          (1 - nu) * D["yz"] - z * D["xxy"], D["zz"] + nu * D["yy"] - z * D["xxz"], -(nu * D["xy"] + z * D["xyz"])],
         [2 * nu * D["yz"] - z * D["xxy"], 2 * D["yz"] - z * D["yyy"], -z * D["yzz"],
          (1 - nu) * D["xz"] - z * D["xyy"], -(nu * D["xy"] + z * D["xyz"]), D["zz"] + nu * D["xx"] - z * D["yyz"]],
         [D["zz"] + (1 - 2 * nu) * D["yy"] - z * D["xxz"], D["zz"] + (1 - 2 * nu) * D["xx"] - z * D["yyz"],
          D["zz"] - z * zzz, -((1 - 2 * nu) * D["xy"] + z * D["xyz"]), -z * D["xzz"], -z * D["yzz"]]]
    return np.array([[float(c * v) for v in row] for row in S])


def test_off_plane_against_high_precision(probe):
    stress, _ = probe
    rng = np.random.default_rng(11)
    for _ in range(80):
        a, b = rng.uniform(0.1, 2.0, 2)
        z = rng.choice([-1, 1]) * 10 ** rng.uniform(-2.5, 0.7)
        x, y = rng.uniform(-6, 6, 2)
        assert _err(stress(x, y, z, a, b, 1.3, 0.27), _truth_stress(x, y, z, a, b, 1.3, 0.27)) < TOL, (x, y, z)


def test_off_plane_points(probe):
    rng = np.random.default_rng(1)
    pts = []
    for _ in range(400):
        a, b = rng.uniform(0.1, 2.0, 2)
        z = rng.choice([-1, 1]) * 10 ** rng.uniform(-2.5, 0.7)
        pts.append((rng.uniform(-6, 6), rng.uniform(-6, 6), z, a, b))
    _check(probe, pts, tol=TOL_REF_OFFPLANE)


def test_in_plane_points(probe):
    rng = np.random.default_rng(2)
    pts = []
    for _ in range(400):
        a, b = rng.uniform(0.1, 2.0, 2)
        x, y = rng.uniform(-6, 6, 2)
        if min(abs(abs(x) - a), abs(abs(y) - b)) > 1e-3:  # not on an edge's line
            pts.append((x, y, 0.0, a, b))
    _check(probe, pts)


def test_uniform_mesh_offsets_and_self_effect(probe):
    a, b = 1.0 / 256, 1.0 / 256
    pts = [(2 * a * i, 2 * b * j, 0.0, a, b) for i in range(-6, 7) for j in range(-6, 7)]
    pts += [(2 * 0.3 * i, 2 * 0.7 * j, 0.0, 0.3, 0.7) for i in (0, 1, 5, 40) for j in (0, -1, 3)]
    _check(probe, pts)


def test_on_edge_lines_beyond_the_element(probe):
    """x = +-a with |y| > b, and y = +-b with |x| > a, in the plane: finite
    here (paired corner sums), equal to the reference where its limit forms
    give a finite value, and continuous with the reference 1e-7 off the line
    (it returns NaN on part of these lines)."""
    stress, _ = probe
    a, b, G, nu = 0.5, 0.35, 1.3, 0.27
    pts = [(sx * a, y) for sx in (1, -1) for y in (0.36, 0.9, 2.0, -0.4, -3.0)]
    pts += [(x, sy * b) for sy in (1, -1) for x in (0.51, 1.2, 4.0, -0.6, -2.5)]
    compared = 0
    for x, y in pts:
        mine = stress(x, y, 0.0, a, b, G, nu)
        assert np.all(np.isfinite(mine)), (x, y)
        ref = ref_r0_stress(x, y, 0.0, a, b, G, nu)
        if np.all(np.isfinite(ref)):
            assert _err(mine, ref) < TOL, (x, y)
            compared += 1
        dx, dy = (1e-7, 0.0) if abs(abs(x) - a) < 1e-15 else (0.0, 1e-7)
        near = ref_r0_stress(x + dx, y + dy, 0.0, a, b, G, nu)
        assert _err(mine, near) < 1e-5, (x, y)
    assert compared >= 4


def _cylinder_strip(n_theta=10, n_h=5, radius=1.0, height=1.2):
    """Planar rectangles on a cylinder (chords): neighbours lie off each
    other's plane, so the entries use the off-plane forms."""
    th = np.linspace(0.0, 0.9 * np.pi, n_theta + 1)
    hs = np.linspace(0.0, height, n_h + 1)
    coor = np.array([[radius * np.cos(t), radius * np.sin(t), h] for h in hs for t in th])
    conn = []
    for j in range(n_h):
        for i in range(n_theta):
            v = i + j * (n_theta + 1)
            conn.append([v, v + 1, v + 1 + (n_theta + 1), v + (n_theta + 1)])
    return coor, np.array(conn, dtype=np.int32)


@pytest.mark.parametrize("mesh", ["planar", "cylinder"])
def test_h_kernel_entries_match_the_reference_operator(probe, mesh):
    """Every 3 x 3 entry of the dense operator of a mesh (the reference's
    BieElastostatic<Rectangle<0>, Rectangle<0>, H>::influence, through the
    oracle's dense rows) from bw::r0::influence_h with the reference's own
    element frames."""
    from bigwham_dev_b200.meshes import square_crack_3d
    from oracle import RefHmat

    E, nu = 1.7, 0.23
    G = E / (2 * (1 + nu))
    coor, conn = square_crack_3d(7) if mesh == "planar" else _cylinder_strip()
    R = RefHmat("3DR0-H", coor, conn, [E, nu], 32, 3.0, 1e-5, n_threads=2)
    fr = np.ascontiguousarray(R.element_frames())
    n = fr.shape[0]
    dense = R.dense_rows("3DR0-H", [E, nu], np.arange(n))
    v = coor[conn]
    a = np.linalg.norm(v[:, 1] - v[:, 0], axis=1) / 2
    b = np.linalg.norm(v[:, 3] - v[:, 0], axis=1) / 2
    mine = np.empty_like(dense)
    out = np.zeros(9)
    for r in range(n):
        for s_ in range(n):
            probe.influence(fr[s_], a[s_], b[s_], fr[r], G, nu, out)
            mine[3 * r:3 * r + 3, 3 * s_:3 * s_ + 3] = out.reshape(3, 3)
    scale = np.max(np.abs(dense))
    err = np.max(np.abs(mine - dense)) / scale
    assert err < (1e-13 if mesh == "planar" else 1e-12), err  # measured: 4e-16 and 2e-15


def element_records(R, coor, conn):
    """(n_elements, 17) records of the assembly: the reference's frames plus
    the half sides |v1 - v0| / 2, |v3 - v0| / 2."""
    v = coor[conn]
    ab = np.stack([np.linalg.norm(v[:, 1] - v[:, 0], axis=1) / 2, np.linalg.norm(v[:, 3] - v[:, 0], axis=1) / 2], 1)
    return np.ascontiguousarray(np.hstack([R.element_frames(), ab]))


@pytest.mark.parametrize("mesh", ["planar", "cylinder"])
def test_fr_blocks_assembled_like_the_reference(probe, mesh):
    """The full-rank blocks of a built 3DR0-H H-matrix, assembled from its
    pattern and permutation with the device kernel's entry function, equal
    the reference's blocks (Hmat::buildFR, hmat.cc:315-353)."""
    from bigwham_dev_b200.meshes import square_crack_3d
    from oracle import RefHmat

    E, nu = 1.0, 0.25
    coor, conn = square_crack_3d(24) if mesh == "planar" else _cylinder_strip(24, 12)
    R = RefHmat("3DR0-H", coor, conn, [E, nu], 32, 3.0, 1e-5, n_threads=4)
    arr = R.arrays()
    assert np.array_equal(arr.perm0, arr.perm1)
    out = np.full(arr.fr_data.size, np.nan)
    probe.fr_blocks(element_records(R, coor, conn), E / (2 * (1 + nu)), nu, len(arr.fr),
                    np.ascontiguousarray(arr.fr, dtype=np.int64), np.ascontiguousarray(arr.perm0, dtype=np.int64), out)
    err = np.max(np.abs(out - arr.fr_data)) / np.max(np.abs(arr.fr_data))
    assert err < 1e-13, err


def test_assembly_entry_rejects_bad_input_before_the_device():
    """bw_r0_assemble_fr checks every index the kernel would use on the host;
    these calls fail there, before any CUDA call."""
    import ctypes as C

    from bigwham_dev_b200 import _capi as A

    L = A.lib()
    rec = np.zeros((4, 17))
    rec[:, 15:] = 0.5
    fr = np.array([[0, 0, 2, 2], [2, 2, 4, 4]], dtype=np.int64)
    perm = np.arange(4, dtype=np.int64)
    out = C.c_void_p(8)  # never dereferenced: every call below fails its checks

    def call(rec=rec, G=1.0, nu=0.25, fr=fr, perm=perm, n_points=4, out_len=72):
        return L.bw_r0_assemble_fr(0, rec.shape[0], rec.ctypes.data, G, nu, fr.shape[0], fr.ctypes.data,
                                   perm.ctypes.data, n_points, out, out_len, None)

    assert call(perm=np.array([0, 1, 2, 4], dtype=np.int64)) == A.BW_ERR_ARG
    assert "perm" in A.last_error(None)
    assert call(fr=np.array([[0, 0, 2, 2], [2, 2, 5, 4]], dtype=np.int64)) == A.BW_ERR_ARG
    assert "outside" in A.last_error(None)
    assert call(out_len=71) == A.BW_ERR_ARG
    assert call(G=0.0) == A.BW_ERR_ARG and call(nu=0.5) == A.BW_ERR_ARG


def test_host_library_records_equal_the_oracles():
    """BigWhamIOGpu.element_records (the host library's reference objects)
    gives the same records as the oracle's build of the same mesh."""
    if not os.path.exists(os.path.join(ROOT, "bigwham_dev_b200", "_lib", "libbigwham_host.so")):
        pytest.skip("host adapter not built")
    from bigwham_dev_b200.bigwham4py import BigWhamIOGpu
    from oracle import RefHmat

    coor, conn = _cylinder_strip(9, 4)
    io = BigWhamIOGpu(coor, conn, "3DR0-H", [1.0, 0.25], 2, useCuda=False)
    mine = io.element_records()
    io.close()
    R = RefHmat("3DR0-H", coor, conn, [1.0, 0.25], 32, 3.0, 1e-5, n_threads=2)
    assert mine.shape == (36, 17)
    assert np.array_equal(mine, element_records(R, coor, conn))


def test_continuity_between_the_in_plane_and_off_plane_forms(probe):
    """z = +-1e-13 (rounding of a frame rotation on a nearly planar mesh) goes
    through the off-plane forms; it must agree with the z = 0 forms, and with
    the reference at the same z, on points inside, outside and at the centre
    of the element."""
    stress, _ = probe
    a, b, G, nu = 0.5, 0.35, 1.3, 0.27
    for x, y in ((0.0, 0.0), (0.2, -0.1), (1.7, 0.3), (-2.5, -1.9), (0.3, 2.2)):
        s0 = stress(x, y, 0.0, a, b, G, nu)
        for z in (1e-13, -1e-13):
            sz = stress(x, y, z, a, b, G, nu)
            assert _err(sz, s0) < 1e-9, (x, y, z)
            assert _err(sz, ref_r0_stress(x, y, z, a, b, G, nu)) < 1e-9, (x, y, z)
