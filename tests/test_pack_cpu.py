"""Run-based packing (bw_pack.h, the element copy a device packer runs) against
the host layout fill (bw::fill_items), byte for byte, for H and H^T, both
phases and all three storage precisions, on a built 3DR0-H crack and on an
irregular rectangular synthetic H-matrix.  The probe links the layout
library's own plan builder (tests/cpp/pack_probe.cc)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "bigwham_dev_b200", "_lib")


@pytest.fixture(scope="module")
def probe():
    if not os.path.exists(os.path.join(LIBDIR, "libbigwham_b200.so")):
        pytest.skip("backend not built")
    out = os.path.join(ROOT, "_build", "libpack_probe.so")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    subprocess.run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-I", os.path.join(ROOT, "bigwham_dev_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "pack_probe.cc"), "-o", out, "-L", LIBDIR, "-lbigwham_b200",
                    f"-Wl,-rpath,{LIBDIR}"], check=True)
    L = C.CDLL(out)
    p, pi = np.ctypeslib.ndpointer(np.float64, flags="C"), np.ctypeslib.ndpointer(np.int64, flags="C")
    L.probe_pack_compare.argtypes = [C.c_int, C.c_longlong, C.c_longlong, C.c_longlong, pi, p, C.c_longlong,
                                     C.c_longlong, pi, p, C.c_longlong, pi, pi]
    return L


def _compare(L, arr):
    diff, runs = np.zeros(12, np.int64), np.zeros(12, np.int64)
    fr = np.ascontiguousarray(arr.fr, dtype=np.int64)
    lr = np.ascontiguousarray(arr.lr, dtype=np.int64)
    fd = np.ascontiguousarray(arr.fr_data) if arr.fr_data.size else np.zeros(1)
    ld = np.ascontiguousarray(arr.lr_data) if arr.lr_data.size else np.zeros(1)
    assert L.probe_pack_compare(arr.dof, arr.n_rows, arr.n_cols, fr.shape[0], fr, fd, arr.fr_data.size, lr.shape[0],
                                lr, ld, arr.lr_data.size, diff, runs) == 0
    assert np.all(diff == 0), diff
    assert np.all(runs > 0), runs


def test_pack_runs_equal_the_host_fill_on_a_crack(probe, golden):
    arr, _ = golden
    _compare(probe, arr)


def test_pack_runs_equal_the_host_fill_on_a_rectangular_synthetic(probe):
    from synth import synthetic_hmat

    _compare(probe, synthetic_hmat(70, 45, 3, seed=5))


def test_device_blocks_need_a_device_handle():
    """bw_add_flat_device is refused on a host-only handle (before any device
    call); the device path itself runs on a GPU."""
    from bigwham_dev_b200 import HmatGpu
    from bigwham_dev_b200 import _capi as A

    h = HmatGpu(3, 12, 12, np.arange(4), np.arange(4), device=-1)
    assert h._lib.bw_add_flat_device(h._h, 0, None, 0, None, None, 0, None, 0) == A.BW_ERR_STATE
    assert "device" in A.last_error(h._h)


def test_pack_runs_with_rank_zero_leaves(probe):
    """Rank-0 low-rank leaves (no factors) between ordinary ones."""
    from synth import synthetic_hmat

    arr = synthetic_hmat(40, 25, 3, seed=21, lr_share=0.7, rank0_share=0.5)
    assert (arr.lr[:, 4] == 0).any()
    _compare(probe, arr)
