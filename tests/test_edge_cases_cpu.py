"""Edge cases of the block layout, on CPU: the host plan (BW_PLAN_ONLY) is
replayed in numpy as the kernels walk it (per-precision matvec, H^T, and the
tensor-core matmat), against the dense matrix assembled from the same blocks.

Cases: low-rank blocks of rank 0 (A m x 0, B 0 x n; the reference's LowRank
container allows them, LowRank.h:18-24), row panels whose only blocks have
rank 0, matrices with no low-rank or no full-rank blocks, a single collocation
point, one-point blocks, all-zero blocks under BF16 scaling, a zero input, and
rectangular matrices narrower or shorter than one panel.  The replay starts y
as NaN, so a row the plan never writes fails the comparison.
"""
import numpy as np
import pytest
from planreplay import mm_replay, replay

from bigwham_dev_b200 import HmatGpu

# componentwise bars: |y - D x| <= TOL * (|D| |x|), |A| |B| for low-rank blocks
TOL = {"fp64": 1e-14, "fp32": 1e-6, "bf16": 8e-3}


def build(dof, n_rows, n_cols, blocks, matmat=False):
    """Host plan of the blocks ("F", i0, j0, a) / ("L", i0, j0, A, B), scalar
    units, the dense matrix they make and its absolute-value bound."""
    h = HmatGpu(dof, n_rows, n_cols, np.arange(n_rows // dof), np.arange(n_cols // dof), device=-1)
    D = np.zeros((n_rows, n_cols))
    Dabs = np.zeros((n_rows, n_cols))
    for b in blocks:
        if b[0] == "F":
            _, i0, j0, a = b
            h.add_full(i0, j0, a)
            D[i0:i0 + a.shape[0], j0:j0 + a.shape[1]] = a
            Dabs[i0:i0 + a.shape[0], j0:j0 + a.shape[1]] = np.abs(a)
        else:
            _, i0, j0, Am, Bm = b
            h.add_lowrank(i0, j0, Am, Bm)
            D[i0:i0 + Am.shape[0], j0:j0 + Bm.shape[1]] = Am @ Bm
            Dabs[i0:i0 + Am.shape[0], j0:j0 + Bm.shape[1]] = np.abs(Am) @ np.abs(Bm)
    h.finalize(plan_only=True, precisions=("fp64", "fp32", "bf16"), transpose=True, matmat=matmat)
    return h, (D, Dabs)


def check_all(h, DD, seed=0, exact_zero_rows=()):
    D, Dabs = DD
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, D.shape[1]).astype(np.float32).astype(np.float64)
    g = rng.uniform(-1, 1, D.shape[0]).astype(np.float32).astype(np.float64)
    for prec, tol in TOL.items():
        y = replay(h, x, prec)
        yt = replay(h, g, prec, transposed=True)
        assert np.all(np.isfinite(y)) and np.all(np.isfinite(yt)), prec
        assert np.all(np.abs(y - D @ x) <= tol * (Dabs @ np.abs(x))), prec
        assert np.all(np.abs(yt - D.T @ g) <= tol * (Dabs.T @ np.abs(g))), prec
        for r in exact_zero_rows:
            assert y[r] == 0.0, (prec, r)
    return x


def check_mm(h, DD, X, transposed=False):
    """The matmat plan (block data in BF16) against the BF16 bar."""
    D, Dabs = (DD[0].T, DD[1].T) if transposed else DD
    Y = mm_replay(h, X, transposed)
    assert np.all(np.abs(Y - D @ X) <= TOL["bf16"] * (Dabs @ np.abs(X)))
    return Y


def _lr(rng, m, n, r):
    return rng.standard_normal((m, r)), rng.standard_normal((r, n))


def test_rank_zero_blocks_and_panels_of_rank_zero_only():
    """Rows 48..95 are covered by one rank-0 block and nothing else: the plan
    still writes them, as zeros."""
    rng = np.random.default_rng(1)
    n = 96
    blocks = [("F", 0, 0, rng.standard_normal((48, 48))),
              ("L", 0, 48, *_lr(rng, 48, 48, 0)),
              ("L", 48, 0, np.zeros((48, 0)), np.zeros((0, 96)))]
    h, DD = build(1, n, n, blocks, matmat=True)
    check_all(h, DD, exact_zero_rows=range(48, 96))
    X = rng.uniform(-1, 1, (n, 5))
    check_mm(h, DD, X)
    check_mm(h, DD, X, transposed=True)


def test_only_full_rank_blocks():
    rng = np.random.default_rng(2)
    sizes = [3, 30, 1, 62]
    edges = np.concatenate([[0], np.cumsum(sizes)])
    n = int(edges[-1])
    blocks = [("F", int(edges[i]), int(edges[j]), rng.standard_normal((sizes[i], sizes[j])))
              for i in range(4) for j in range(4)]
    h, DD = build(1, n, n, blocks, matmat=True)
    check_all(h, DD)
    X = rng.uniform(-1, 1, (n, 3))
    check_mm(h, DD, X)


def test_only_low_rank_blocks():
    rng = np.random.default_rng(3)
    blocks = [("L", i, j, *_lr(rng, 40, 40, 1 + (i + 2 * j) % 7)) for i in (0, 40) for j in (0, 40)]
    h, DD = build(2, 80, 80, blocks, matmat=True)
    check_all(h, DD)
    X = rng.uniform(-1, 1, (80, 9))
    check_mm(h, DD, X)


@pytest.mark.parametrize("dof", [1, 2, 3])
def test_single_collocation_point(dof):
    rng = np.random.default_rng(4)
    h, DD = build(dof, dof, dof, [("F", 0, 0, rng.standard_normal((dof, dof)))], matmat=True)
    check_all(h, DD)
    X = rng.uniform(-1, 1, (dof, 2))
    check_mm(h, DD, X)


def test_one_point_blocks_everywhere():
    """A 5-point dof-3 matrix cut into 25 one-point (3 x 3) blocks, alternating
    full rank and low rank."""
    rng = np.random.default_rng(5)
    blocks = []
    for i in range(5):
        for j in range(5):
            if (i + j) % 2 == 0:
                blocks.append(("F", 3 * i, 3 * j, rng.standard_normal((3, 3))))
            else:
                blocks.append(("L", 3 * i, 3 * j, *_lr(rng, 3, 3, 1 + (i * j) % 3)))
    h, DD = build(3, 15, 15, blocks, matmat=True)
    check_all(h, DD)
    X = rng.uniform(-1, 1, (15, 4))
    check_mm(h, DD, X)


def test_all_zero_blocks_under_bf16_scaling():
    """Blocks whose maximum is 0 (a zero full block, zero low-rank factors)
    keep a unit scale: no 0/0 in the BF16 layout, exact zeros out."""
    rng = np.random.default_rng(6)
    blocks = [("F", 0, 0, np.zeros((32, 32))), ("L", 0, 32, np.zeros((32, 4)), rng.standard_normal((4, 32))),
              ("L", 32, 0, rng.standard_normal((32, 2)), np.zeros((2, 32))), ("F", 32, 32, np.eye(32))]
    h, DD = build(1, 64, 64, blocks)
    x = check_all(h, DD, exact_zero_rows=range(32))
    assert np.array_equal(replay(h, x, "bf16")[32:], x[32:].astype(np.float32).astype(np.float64))


def test_zero_input_gives_zero_output(golden):
    arr, _ = golden
    h = HmatGpu(arr.dof, arr.n_rows, arr.n_cols, arr.perm0, arr.perm1, device=-1)
    h.add_flat(arr.fr, arr.lr, arr.fr_data, arr.lr_data)
    h.finalize(plan_only=True, precisions=("fp64", "fp32", "bf16"), transpose=True)
    for prec in TOL:
        assert np.array_equal(replay(h, np.zeros(arr.n_cols), prec), np.zeros(arr.n_rows))
        assert np.array_equal(replay(h, np.zeros(arr.n_rows), prec, transposed=True), np.zeros(arr.n_cols))


@pytest.mark.parametrize("shape", [(6, 600), (600, 6), (2, 2000)])
def test_rectangular_thin_matrices(shape):
    """Fewer rows than one 16-row panel alignment, or fewer columns than one
    8-column chunk, with both block kinds."""
    rng = np.random.default_rng(7)
    m, n = shape
    blocks = []
    cuts = [0, n // 3, n]
    for c in range(2):
        w = cuts[c + 1] - cuts[c]
        if c == 0:
            blocks.append(("F", 0, cuts[c], rng.standard_normal((m, w))))
        else:
            blocks.append(("L", 0, cuts[c], *_lr(rng, m, w, min(m, w, 2))))
    h, DD = build(1, m, n, blocks, matmat=True)
    check_all(h, DD)
    X = rng.uniform(-1, 1, (n, 3))
    check_mm(h, DD, X)
    G = rng.uniform(-1, 1, (m, 3))
    check_mm(h, DD, G, transposed=True)


def test_rank_zero_leaves_of_a_synthetic_partition():
    """Irregular rectangular partitions where every leaf is low rank and half
    of them have rank 0 (so whole row and column panels do), against the
    restatement, H and H^T, every precision."""
    from oracle import oracle_matvec_perm, oracle_rmatvec_perm
    from synth import synthetic_hmat

    for seed, (nr, nc) in enumerate([(40, 25), (25, 40), (33, 33)]):
        arr = synthetic_hmat(nr, nc, 3, seed=20 + seed, lr_share=1.0, rank0_share=0.5)
        assert (arr.lr[:, 4] == 0).any() and (arr.lr[:, 4] > 0).any()
        h = HmatGpu(arr.dof, arr.n_rows, arr.n_cols, arr.perm0, arr.perm1, device=-1)
        h.add_flat(arr.fr, arr.lr, arr.fr_data, arr.lr_data)
        h.finalize(plan_only=True, precisions=("fp64", "fp32", "bf16"), transpose=True, matmat=True)
        rng = np.random.default_rng(seed)
        x = rng.uniform(-1, 1, arr.n_cols)
        g = rng.uniform(-1, 1, arr.n_rows)
        want, want_t = oracle_matvec_perm(arr, x, 1), oracle_rmatvec_perm(arr, g, 1)
        assert np.abs(replay(h, x) - want).max() <= 1e-13 * max(1.0, np.abs(want).max())
        assert np.abs(replay(h, g, transposed=True) - want_t).max() <= 1e-13 * max(1.0, np.abs(want_t).max())
        for prec in ("fp32", "bf16"):
            assert np.all(np.isfinite(replay(h, x, prec))) and np.all(np.isfinite(replay(h, g, prec, transposed=True)))
        X = rng.uniform(-1, 1, (arr.n_cols, 4))
        Y = mm_replay(h, X)
        W = np.stack([oracle_matvec_perm(arr, X[:, c], 1) for c in range(4)], axis=1)
        assert np.abs(Y - W).max() <= 2e-2 * max(1.0, np.abs(W).max())


def test_batch_with_rank_zero_leaves_and_a_one_point_member():
    """A batch of irregular members (rank-0 leaves among them) and a member of
    one collocation point: each member's slice is its own product."""
    from types import SimpleNamespace

    from oracle import oracle_matvec_perm, oracle_rmatvec_perm
    from synth import synthetic_hmat

    rng = np.random.default_rng(9)
    one = SimpleNamespace(dof=3, n_rows=3, n_cols=3, fr=np.array([[0, 0, 1, 1]]), lr=np.zeros((0, 5), np.int64),
                          fr_data=rng.standard_normal(9), lr_data=np.zeros(0), perm0=np.zeros(1, np.int64),
                          perm1=np.zeros(1, np.int64))
    ms = [synthetic_hmat(20, 20, 3, seed=40, lr_share=0.8, rank0_share=0.5), one,
          synthetic_hmat(17, 26, 3, seed=41, lr_share=1.0, rank0_share=0.5)]
    h = HmatGpu.batch(ms, device=-1, plan_only=True, precisions=("fp64", "bf16"), transpose=True)
    x = rng.uniform(-1, 1, h.n_cols)
    g = rng.uniform(-1, 1, h.n_rows)
    y, yt = replay(h, x), replay(h, g, transposed=True)
    assert np.all(np.isfinite(replay(h, x, "bf16")))
    for k, m in enumerate(ms):
        r0, r1 = h.row_offsets[k], h.row_offsets[k + 1]
        c0, c1 = h.col_offsets[k], h.col_offsets[k + 1]
        w, wt = oracle_matvec_perm(m, x[c0:c1], 1), oracle_rmatvec_perm(m, g[r0:r1], 1)
        assert np.abs(y[r0:r1] - w).max() <= 1e-13 * max(1.0, np.abs(w).max()), k
        assert np.abs(yt[c0:c1] - wt).max() <= 1e-13 * max(1.0, np.abs(wt).max()), k


def test_two_element_meshes_built_by_the_reference():
    """The reference's two-element 3D meshes (the square [0,1]^2 as two
    triangles, src/io/_test/bigwham_io_gen_test_3d.cc:22-48; and as two
    rectangles): 6 x 6 H-matrices through the plan, against its own MatVec
    (original ordering, both permutations applied)."""
    from oracle import RefHmat, ref_available

    if not ref_available():
        pytest.skip("oracle/_ref not built")
    tri = (np.array([0, 0, 0, 1, 0, 0, 0, 1, 0, 1, 1, 0], float), np.array([0, 1, 2, 1, 2, 3]), "3DT0-H")
    rect = (np.array([0, 0, 0, 0.5, 0, 0, 1, 0, 0, 0, 1, 0, 0.5, 1, 0, 1, 1, 0], float),
            np.array([0, 1, 4, 3, 1, 2, 5, 4]), "3DR0-H")
    for coor, conn, kernel in (tri, rect):
        ref = RefHmat(kernel, coor.reshape(-1, 3), conn.reshape(2, -1), [1.0, 0.0 if kernel == "3DT0-H" else 0.25],
                      32, 0.0, 1e-3, n_threads=2)
        arr = ref.arrays()
        assert (arr.n_rows, arr.n_cols) == (6, 6)
        h = HmatGpu(3, 6, 6, arr.perm0, arr.perm1, device=-1)
        h.add_flat(arr.fr, arr.lr, arr.fr_data, arr.lr_data)
        h.finalize(plan_only=True, precisions=("fp64",), transpose=True)
        x = np.random.default_rng(3).uniform(-1, 1, 6)
        d = 3
        xp = x[(d * np.asarray(arr.perm1)[:, None] + np.arange(d)).ravel()]
        y = np.empty(6)
        y[(d * np.asarray(arr.perm0)[:, None] + np.arange(d)).ravel()] = replay(h, xp)
        want = ref.matvec(x)
        assert np.abs(y - want).max() <= 1e-14 * np.abs(want).max(), kernel
