"""Tensor-core H-matmat (BW_STORE_MATMAT + BW_BF16) on the GPU (-m gpu).

The result is checked two ways:
* against the same plan replayed in numpy with the kernel's roundings (BF16
  blocks, X and T8 rounded to BF16) in FP64, which isolates the kernel:
  relative 1e-5 per column, the FP32 accumulation's error;
* against the oracle's FP64 product, which bounds the BF16 accuracy.
Right-hand-side counts cover one partial pass (1, 5), a full pass (64) and
two passes (70); the original and the permuted orderings and H^T are covered.
"""
import numpy as np
import pytest
from conftest import rel
from planreplay import mm_replay

from bigwham_dev_b200 import HmatGpu
from bigwham_dev_b200.meshes import square_crack_3d
from oracle import RefHmat, oracle_matvec, oracle_rmatvec

pytestmark = pytest.mark.gpu


def _handles(arr):
    kw = dict(precisions=("fp64", "bf16"), transpose=True, matmat=True)
    dev = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                            arr.perm1, device=0, **kw)
    host = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                             arr.perm1, device=-1, plan_only=True, **kw)
    return dev, host


def _colerr(A, B):
    return max(rel(A[:, j], B[:, j]) for j in range(A.shape[1]))


def _run(arr, k, transpose, seed):
    import torch

    dev, host = _handles(arr)
    nin = arr.n_rows if transpose else arr.n_cols
    X = np.random.default_rng(seed).uniform(-1, 1, (nin, k))
    Y = dev.matmat(torch.from_numpy(X).cuda(), "bf16", permuted=True, transpose=transpose).cpu().numpy()
    Yr = mm_replay(host, X, transposed=transpose, round_operands=True)
    assert _colerr(Y, Yr) < 1e-5
    # original ordering through the permutations, against the FP64 oracle
    Yo = dev.matmat(torch.from_numpy(X).cuda(), "bf16", transpose=transpose).cpu().numpy()
    f = oracle_rmatvec if transpose else oracle_matvec
    ref = np.stack([f(arr, X[:, j], 8) for j in range(k)], axis=1)
    dev.close()
    return _colerr(Yo, ref)


@pytest.mark.parametrize("k", [1, 5, 64, 70])
def test_matmat_golden(golden, k):
    arr, ex = golden
    err = _run(arr, k, False, k)
    assert err < (3e-2 if ex["name"].startswith("2ds0") else 8e-3), err


@pytest.mark.parametrize("transpose", [False, True])
def test_matmat_3dr0_64(transpose):
    coor, conn = square_crack_3d(64)
    arr = RefHmat("3DR0-H", coor, conn, [1.0, 0.25], 32, 3.0, 1e-5, n_threads=16).arrays()
    assert _run(arr, 64, transpose, 3) < 8e-3
