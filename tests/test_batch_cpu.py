"""Batched H-matrices (bw_create_batch) on CPU: several independent 2DS0-H
members in one handle are the block-diagonal H-matrix of the members.  Its
plan (BW_PLAN_ONLY) is replayed in numpy as the kernel walks it, and each
member's slice of the result must equal that member's own oracle product.
Malformed batches are rejected."""
import numpy as np
import pytest
from conftest import rel
from planreplay import replay

from bigwham_dev_b200 import BigWhamError, HmatGpu
from bigwham_dev_b200 import _capi as A
from bigwham_dev_b200.meshes import straight_crack_2d
from oracle import RefHmat, oracle_matvec_perm, oracle_rmatvec_perm, ref_available

needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")


def members(sizes=(256, 301, 64, 777), seed=0):
    out = []
    for k, n in enumerate(sizes):
        coor, conn = straight_crack_2d(n, -1.0 - k, 1.0 + k)
        out.append(RefHmat("2DS0-H", coor, conn, [1.0, 0.25], 32, 3.0, 1e-5, n_threads=4).arrays())
    return out


@needs_ref
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-14), ("fp32", 2e-6)])
def test_batch_plan_replay_matches_each_member(prec, tol):
    ms = members()
    h = HmatGpu.batch(ms, device=-1, plan_only=True, precisions=(prec,), transpose=True)
    assert list(h.row_offsets) == list(np.cumsum([0] + [m.n_rows for m in ms]))
    x = np.random.default_rng(1).uniform(-1, 1, h.n_cols)
    if prec == "fp32":
        x = x.astype(np.float32).astype(np.float64)
    y = replay(h, x, prec)
    yt = replay(h, x, prec, transposed=True)
    for k, m in enumerate(ms):
        r0, r1 = h.row_offsets[k], h.row_offsets[k + 1]
        c0, c1 = h.col_offsets[k], h.col_offsets[k + 1]
        assert rel(y[r0:r1], oracle_matvec_perm(m, x[c0:c1], 1)) < tol
        assert rel(yt[c0:c1], oracle_rmatvec_perm(m, x[r0:r1], 1)) < tol


@needs_ref
def test_batch_offsets_and_count():
    ms = members((100, 40))
    h = HmatGpu.batch(ms, device=-1, plan_only=True)
    lib = A.lib()
    assert lib.bw_batch_count(h._h) == 2
    r0, c0 = A.C.c_int64(), A.C.c_int64()
    assert lib.bw_batch_offsets(h._h, 1, A.C.byref(r0), A.C.byref(c0)) == A.BW_OK
    assert (r0.value, c0.value) == (200, 200)
    assert lib.bw_batch_offsets(h._h, 2, None, None) == A.BW_ERR_ARG
    # a single handle is a batch of one at (0, 0)
    s = HmatGpu(1, 4, 4, np.arange(4), np.arange(4), device=-1)
    assert lib.bw_batch_count(s._h) == 1


def _two(n=4):
    class M:
        pass

    out = []
    for _ in range(2):
        m = M()
        m.dof, m.n_rows, m.n_cols = 1, n, n
        m.perm0 = m.perm1 = np.arange(n)
        m.fr = np.array([[0, 0, n, n]])
        m.lr = np.zeros((0, 5), np.int64)
        m.fr_data = np.arange(n * n, dtype=np.float64)
        m.lr_data = np.zeros(0)
        out.append(m)
    return out


def test_block_across_members_is_rejected():
    # member 0's rows get one block that spans both members' columns
    p0 = [np.arange(4), np.arange(4)]
    lib = A.lib()
    handle = A.C.c_void_p()
    nr = np.array([4, 4], np.int64)
    pp = (A.C.c_void_p * 2)(*[a.ctypes.data for a in p0])
    assert lib.bw_create_batch(1, 2, nr.ctypes.data, nr.ctypes.data, pp, pp, -1, A.C.byref(handle)) == A.BW_OK
    a = np.ones((4, 8), order="F")
    b = np.ones((4, 4), order="F")
    assert lib.bw_add_full(handle, 0, 0, 4, 8, a.ctypes.data, 4) == A.BW_OK
    assert lib.bw_add_full(handle, 4, 4, 4, 4, b.ctypes.data, 4) == A.BW_OK
    assert lib.bw_finalize(handle, A.BW_FP64 | A.BW_PLAN_ONLY) == A.BW_ERR_ARG
    msg = A.C.create_string_buffer(256)
    lib.bw_last_error(handle, msg, 256)
    assert b"outside its batch member" in msg.value
    lib.bw_destroy(handle)


def test_batch_member_dof_and_permutation_checked():
    ms = _two()
    ms[1].dof = 2
    with pytest.raises(ValueError, match="same dof"):
        HmatGpu.batch(ms, device=-1, plan_only=True)
    ms = _two()
    ms[1].perm0 = np.array([0, 1, 2, 4])
    with pytest.raises(BigWhamError, match="permutation"):
        HmatGpu.batch(ms, device=-1, plan_only=True)


def test_small_batch_equals_block_diagonal_dense():
    ms = _two()
    h = HmatGpu.batch(ms, device=-1, plan_only=True, precisions=("fp64",))
    x = np.random.default_rng(2).uniform(-1, 1, 8)
    D = np.zeros((8, 8))
    blk = np.arange(16, dtype=np.float64).reshape(4, 4).T
    D[:4, :4] = blk
    D[4:, 4:] = blk
    assert rel(replay(h, x), D @ x) < 1e-14
