"""Parity of the CUDA backend against the oracle (run on a B200: -m gpu).

Tolerances: FP64 storage and accumulation must match the reference's OpenMP
matvec to 1e-12 relative (L2); FP32 storage with FP32 accumulation to 2e-6;
BF16 storage (per-block FP32 scale, FP32 accumulation) to 8e-3.
"""
import numpy as np
import pytest
from conftest import rel

from bigwham_dev_b200 import BigWhamError, HmatGpu
from bigwham_dev_b200 import _capi as A
from bigwham_dev_b200.meshes import square_crack_3d, straight_crack_2d
from oracle import RefHmat, oracle_matvec, oracle_rmatvec

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 2e-6, "bf16": 8e-3}


def upload(arr, precisions=("fp64", "fp32", "bf16"), transpose=True, **kw):
    return HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                             arr.perm1, device=0, precisions=precisions, transpose=transpose, **kw)


def test_golden_fp64(golden):
    import torch

    arr, ex = golden
    h = upload(arr)
    x = ex["x"]
    y = h.matvec(x)
    assert rel(y, ex["y_ref"]) < TOL["fp64"]
    assert rel(h.matvec(x, permuted=True), ex["y_perm_ref"]) < TOL["fp64"]
    assert np.array_equal(h.diagonal(), ex["diag_ref"])
    # device path on the torch stream gives the same bits as the host path
    yd = h.matvec(torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    assert np.array_equal(yd.cpu().numpy(), y)
    # transposed product against the oracle on the same blocks
    xr = np.random.default_rng(7).uniform(-1, 1, arr.n_rows)
    assert rel(h.rmatvec(xr), oracle_rmatvec(arr, xr, 2)) < TOL["fp64"]
    h.sync()


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_golden_reduced_precision(golden, prec):
    arr, ex = golden
    h = upload(arr, precisions=(prec,), transpose=True)
    assert rel(h.matvec(ex["x"], prec), ex["y_ref"]) < TOL[prec]
    xr = np.random.default_rng(8).uniform(-1, 1, arr.n_rows)
    assert rel(h.rmatvec(xr, prec), oracle_rmatvec(arr, xr, 2)) < TOL[prec]


def test_repeatable_bits(golden):
    arr, ex = golden
    h = upload(arr, precisions=("fp64", "bf16"), transpose=False)
    for p in ("fp64", "bf16"):
        a, b = h.matvec(ex["x"], p), h.matvec(ex["x"], p)
        assert np.array_equal(a, b)


def _ref_case(kind):
    if kind == "C1":
        coor, conn = straight_crack_2d(4000)
        return RefHmat("2DS0-H", coor, conn, [1.0, 0.25], 32, 3.0, 1e-5, n_threads=8), 0
    coor, conn = square_crack_3d(128)
    return RefHmat("3DR0-H", coor, conn, [1.0, 0.25], 32, 3.0, 1e-5, n_threads=8), 1


@pytest.mark.parametrize("kind", ["C1", "C2"])
def test_config_parity_against_reference(kind):
    """C1: 2DS0-H 4,000 segments (8,000 DoF); C2: 3DR0-H 128 x 128 (49,152 DoF).
    The reference builds the H-matrix and runs its own OpenMP matvec; the GPU
    runs the same blocks."""
    R, seed = _ref_case(kind)
    arr = R.arrays()
    x = np.random.default_rng(seed).uniform(-1, 1, R.shape[1])
    y_ref = R.matvec(x)
    h = upload(arr, transpose=False)
    assert rel(h.matvec(x), y_ref) < TOL["fp64"]
    assert rel(h.matvec(x, permuted=True), R.matvec_perm(x)) < TOL["fp64"]
    for p in ("fp32", "bf16"):
        assert rel(h.matvec(x, p), y_ref) < TOL[p]
    assert np.array_equal(h.diagonal(), R.diagonal())


def test_known_answer_griffith_gpu():
    coor, conn = straight_crack_2d(1200)
    R = RefHmat("2DS0-H", coor, conn, [1.0, 0.0], 32, 2.0, 1e-3, n_threads=4)
    h = upload(R.arrays(), transpose=False)
    xc = 0.5 * (coor[conn[:, 0], 0] + coor[conn[:, 1], 0])
    x = np.zeros(R.shape[1])
    x[1::2] = 4.0 * np.sqrt(1.0 - xc ** 2)
    # The hypersingular operator cancels ~1000x on this smooth opening (diag ~190
    # times openings ~4 sum to a traction of 1), so the traction needs FP32 or
    # FP64 blocks; BF16 storage (2^-9) cannot resolve it and is checked on its
    # normwise error elsewhere.
    for p in ("fp64", "fp32"):
        y = h.matvec(x, p)
        assert np.mean(np.abs(y[1::2] - 1.0)) < 0.05
    assert np.mean(np.abs(h.diagonal()[1::2] - 190.985)) < 0.05


def test_matmat_matches_columns(golden):
    import torch

    arr, ex = golden
    h = upload(arr, precisions=("fp64",), transpose=False)
    X = torch.randn(arr.n_cols, 3, dtype=torch.float64, device="cuda").t().contiguous()  # 3 columns, ld = n_cols
    Y = torch.empty(3, arr.n_rows, dtype=torch.float64, device="cuda")
    h.matmat_ptr(X.data_ptr(), arr.n_cols, Y.data_ptr(), arr.n_rows, 3, stream=torch.cuda.current_stream().cuda_stream)
    for k in range(3):
        assert torch.equal(Y[k], h.matvec(X[k].contiguous()))


def test_errors_are_status_codes(golden):
    import torch

    arr, ex = golden
    h = upload(arr, precisions=("fp64",), transpose=False)
    with pytest.raises(BigWhamError) as e:
        h.matvec(ex["x"], "bf16")
    assert e.value.status == A.BW_ERR_UNSUPPORTED
    with pytest.raises(BigWhamError) as e:
        h.rmatvec(np.zeros(arr.n_rows))
    assert e.value.status == A.BW_ERR_UNSUPPORTED
    buf = torch.zeros(arr.n_rows + arr.n_cols, dtype=torch.float64, device="cuda")
    with pytest.raises(BigWhamError) as e:
        h.matvec_ptr(buf.data_ptr(), buf.data_ptr() + 8, "fp64")
    assert e.value.status == A.BW_ERR_ARG
    # allocation cap simulating an out-of-memory device
    h2 = HmatGpu(arr.dof, arr.n_rows, arr.n_cols, arr.perm0, arr.perm1, device=0)
    h2.add_flat(arr.fr, arr.lr, arr.fr_data, arr.lr_data)
    with pytest.raises(BigWhamError) as e:
        h2.finalize(device_limit=1024)
    assert e.value.status == A.BW_ERR_OOM
    # matvec before finalize
    h3 = HmatGpu(arr.dof, arr.n_rows, arr.n_cols, arr.perm0, arr.perm1, device=0)
    with pytest.raises(BigWhamError) as e:
        h3.matvec(ex["x"])
    assert e.value.status == A.BW_ERR_STATE
    h.sync()


def test_raw_ptr_reference_semantics(golden):
    import torch

    arr, ex = golden
    h = upload(arr, precisions=("fp64",), transpose=False)
    x = torch.from_numpy(ex["x"]).cuda()
    y = torch.empty(arr.n_rows, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    h.matvec_raw_ptr(x.data_ptr(), y.data_ptr())
    assert rel(y.cpu().numpy(), ex["y_ref"]) < TOL["fp64"]
