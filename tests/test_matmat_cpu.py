"""Matmat layout (BW_STORE_MATMAT) on CPU.

The plan built by bw_finalize(BW_PLAN_ONLY | BW_STORE_MATMAT) is replayed in
numpy as the tensor-core kernel walks it.  The replay uses the BF16 block data
but keeps X and the low-rank products exact, so the layout itself is under
test, not its rounding:
  * the widened 8-aligned operand windows;
  * the zero padding of columns and ranks;
  * the operand runs;
  * the T8 numbering.
The replay must reproduce the oracle applied to the same BF16-rounded blocks to
FP64 rounding (1e-13), forward and transposed.  Every chunk is checked against
the kernel's limits:
  * kc a multiple of 16 and at most 512;
  * at most 4 runs, each 8-aligned and 8-row multiple, covering exactly kc rows;
  * block data + operand rows within one 48 KB stage;
  * hpad a multiple of 8 and at most 256;
  * every item at least 32 columns (a K-step for each MMA issuer).
"""
import numpy as np
import pytest
from conftest import rel
from planreplay import mm_replay

from bigwham_dev_b200 import HmatGpu
from bigwham_dev_b200.meshes import square_crack_3d, straight_crack_2d
from oracle import HmatArrays, RefHmat, oracle_matvec_perm, oracle_rmatvec_perm, ref_available

needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")


def bf16(a):
    """Round to BF16 (through FP32, nearest-even), as the layout stores blocks."""
    u = np.ascontiguousarray(a, dtype=np.float64).astype(np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def rounded(arr):
    return HmatArrays(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, bf16(arr.fr_data), bf16(arr.lr_data),
                      arr.perm0, arr.perm1)


def check_chunk(w):
    kc, hpad = int(w[2]), int(w[3])
    nr = (int(np.uint32(w[6])) >> 8) & 0xFF
    assert 0 < kc <= 512 and kc % 16 == 0
    assert 0 < hpad <= 256 and hpad % 8 == 0
    if (int(np.uint32(w[6])) & 3) == 3:  # an item of one chunk still has a K-step for each of the two MMA issuers
        assert kc >= 32
    assert 1 <= nr <= 4
    rows = [int(w[9 + 2 * r]) for r in range(nr)]
    srcs = [int(np.uint32(w[8 + 2 * r])) & 0x7FFFFFFF for r in range(nr)]
    assert sum(rows) == kc
    assert all(r % 8 == 0 for r in rows) and all(s % 8 == 0 for s in srcs)
    assert kc * hpad * 2 + kc * 128 <= 49152


def plan(arr, transpose=True):
    h = HmatGpu(arr.dof, arr.n_rows, arr.n_cols, arr.perm0, arr.perm1, device=-1)
    h.add_flat(arr.fr, arr.lr, arr.fr_data, arr.lr_data)
    return h.finalize(plan_only=True, precisions=("bf16",), transpose=transpose, matmat=True)


def _check(arr, k=5, seed=0):
    h = plan(arr)
    r = rounded(arr)
    rng = np.random.default_rng(seed)
    X = rng.uniform(-1, 1, (arr.n_cols, k))
    Y = mm_replay(h, X, check=check_chunk)
    for j in range(k):
        assert rel(Y[:, j], oracle_matvec_perm(r, X[:, j], 1)) < 1e-13, j
    G = rng.uniform(-1, 1, (arr.n_rows, k))
    Yt = mm_replay(h, G, transposed=True, check=check_chunk)
    for j in range(k):
        assert rel(Yt[:, j], oracle_rmatvec_perm(r, G[:, j], 1)) < 1e-13, j


def test_matmat_plan_replay_golden(golden):
    arr, ex = golden
    _check(arr)


@needs_ref
@pytest.mark.parametrize("kind", ["2ds0", "3dr0"])
def test_matmat_plan_replay_reference_builds(kind):
    if kind == "2ds0":
        coor, conn = straight_crack_2d(1500)
        R = RefHmat("2DS0-H", coor, conn, [1.0, 0.25], 32, 3.0, 1e-5, n_threads=4)
    else:
        coor, conn = square_crack_3d(24)
        R = RefHmat("3DR0-H", coor, conn, [1.0, 0.25], 32, 3.0, 1e-5, n_threads=4)
    _check(R.arrays(), k=3, seed=1)


def test_matmat_plan_t8_is_padded_ranks(golden):
    arr, ex = golden
    h = plan(arr, transpose=False)
    ranks = arr.lr[:, 4] * 1
    assert h.mm_plan_export(1)["t8_len"] == int(sum((r + 7) // 8 * 8 for r in ranks if r > 0))
