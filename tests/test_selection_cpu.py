"""Sub-matrix selection (bigwham_dev_b200.selection, the reference's
HmatSelection) on CPU against the reference's own BigWhamIO::hmatSelection:
the selection handle's host plan is replayed as the kernels walk it, in the
selection's original ordering, and must equal the reference's selection MatVec
(FP64, 1e-13); its full-block entries must equal the reference's
GetFullBlocks on the selection, values and positions in the same order."""
import numpy as np
import pytest
from planreplay import replay

from bigwham_dev_b200.meshes import square_crack_3d, straight_crack_2d
from bigwham_dev_b200.selection import HmatSelection, select_blocks
from oracle import RefHmat, ref_available

pytestmark = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")


@pytest.fixture(scope="module", params=["2DS0-H", "3DR0-H"])
def built(request):
    if request.param == "2DS0-H":
        coor, conn = straight_crack_2d(300)
        ref = RefHmat("2DS0-H", coor, conn, [1.0, 0.25], 16, 3.0, 1e-5, n_threads=2)
    else:
        coor, conn = square_crack_3d(12)
        ref = RefHmat("3DR0-H", coor, conn, [1.0, 0.25], 16, 3.0, 1e-5, n_threads=2)
    arr = ref.arrays()
    ex = {"dof": arr.dof, "n_rows": arr.n_rows, "n_cols": arr.n_cols, "fr": arr.fr, "lr": arr.lr,
          "fr_data": arr.fr_data, "lr_data": arr.lr_data, "perm0": arr.perm0, "perm1": arr.perm1}
    return ref, ex, len(conn)


def sel_matvec(sel, x, precision="fp64"):
    """The selection's matvec with its handle's plan replayed on the host."""
    d = sel.dof
    x_u = x[sel.x_take]
    x_perm = x_u[(d * sel.perm1[:, None] + np.arange(d)).ravel()]
    y_perm = replay(sel.h, x_perm, precision)
    y_u = np.empty_like(y_perm)
    y_u[(d * sel.perm0[:, None] + np.arange(d)).ravel()] = y_perm
    return y_u[sel.y_take]


def _cases(n, rng):
    yield "contiguous", np.arange(n // 4, n // 2), np.arange(n // 3, n - 5)
    yield "scattered", rng.choice(n, n // 3, replace=False), rng.choice(n, n // 5, replace=False)
    yield "sorted", np.sort(rng.choice(n, 40, replace=False)), np.sort(rng.choice(n, 50, replace=False))
    yield "one each", np.array([n // 2]), np.array([7])
    yield "all", rng.permutation(n), np.arange(n)
    yield "repeats", rng.integers(0, n, 60), rng.integers(0, n, 45)


def test_selection_matvec_equals_the_reference(built):
    ref, ex, n = built
    rng = np.random.default_rng(3)
    for name, rows, cols in _cases(n, rng):
        sel = HmatSelection(ex, rows, cols, device=-1, plan_only=True, precisions=("fp64", "fp32"))
        x = rng.uniform(-1, 1, cols.size * ex["dof"])
        want = ref.selection_matvec(rows, cols, x)
        got = sel_matvec(sel, x)
        assert got.shape == want.shape, name
        assert np.abs(got - want).max() <= 1e-13 * max(1.0, np.abs(want).max()), name
        xf = x.astype(np.float32).astype(np.float64)
        assert np.abs(sel_matvec(sel, xf, "fp32") - ref.selection_matvec(rows, cols, xf)).max() <= \
            2e-6 * max(1.0, np.abs(want).max()), name


def test_selection_streams_only_selected_entries(built):
    """The selection handle holds the selected sub-blocks only: for a quarter
    of the rows and columns, a small share of the base's entries."""
    ref, ex, n = built
    rng = np.random.default_rng(4)
    rows, cols = rng.choice(n, n // 4, replace=False), rng.choice(n, n // 4, replace=False)
    s = select_blocks(ex, rows, cols)
    base = ex["fr_data"].size + ex["lr_data"].size
    assert s["fr_data"].size + s["lr_data"].size < 0.35 * base
    # every selected scalar pair is covered exactly once
    d = ex["dof"]
    cover = np.zeros((s["n_rows"], s["n_cols"]), np.int32)
    for blk in list(s["fr"]) + [b[:4] for b in s["lr"]]:
        i0, j0, i1, j1 = blk
        cover[i0 * d:i1 * d, j0 * d:j1 * d] += 1
    assert np.all(cover == 1)


def test_full_blocks_equal_the_reference(built):
    ref, ex, n = built
    rng = np.random.default_rng(5)
    for name, rows, cols in _cases(n, rng):
        sel = HmatSelection(ex, rows, cols, device=-1, plan_only=True)
        val, pos = sel.full_blocks()
        rval, rpos = ref.selection_full_blocks(rows, cols)
        assert np.array_equal(val, rval), name
        assert np.array_equal(pos, rpos), name


def test_out_of_range_indices_are_rejected_like_the_reference(built):
    ref, ex, n = built
    for rows, cols in (([0, n], [1]), ([0], [-1]), ([n + 5], [0])):
        with pytest.raises(IndexError):
            HmatSelection(ex, rows, cols, device=-1, plan_only=True)
        with pytest.raises(IndexError):
            ref.selection_matvec(rows, cols, np.zeros(len(cols) * ex["dof"]))


def test_selection_of_a_rectangular_base():
    """A reference-built rectangular H-matrix (3DR0-3DR0-H, 63 receiver and
    100 source elements: permutation_0_ and permutation_1_ differ in length):
    rows go through permutation_0_, columns through permutation_1_; the
    selection's product equals the H-matrix operator's own, restricted."""
    import os

    from oracle import HmatArrays, oracle_matvec

    arr, _ = HmatArrays.load(os.path.join(os.path.dirname(__file__), "golden", "rect", "3dr0_rect.npz"))
    ex = {"dof": arr.dof, "n_rows": arr.n_rows, "n_cols": arr.n_cols, "fr": arr.fr, "lr": arr.lr,
          "fr_data": arr.fr_data, "lr_data": arr.lr_data, "perm0": arr.perm0, "perm1": arr.perm1}
    d = arr.dof
    D = np.column_stack([oracle_matvec(arr, np.eye(arr.n_cols)[:, j], 1) for j in range(arr.n_cols)])
    rng = np.random.default_rng(6)
    for rows, cols in ((rng.choice(63, 20, replace=False), rng.choice(100, 37, replace=False)),
                       (np.arange(63), np.arange(100)), (np.array([62, 0, 62]), np.array([99, 5, 5]))):
        sel = HmatSelection(ex, rows, cols, device=-1, plan_only=True)
        x = rng.uniform(-1, 1, d * cols.size)
        xf = np.zeros(arr.n_cols)
        for i, c in enumerate(cols):  # in list order: the last of a repeated column counts
            xf[d * c:d * c + d] = x[d * i:d * i + d]
        want = (D @ xf)[(d * rows[:, None] + np.arange(d)).ravel()]
        got = sel_matvec(sel, x)
        assert np.abs(got - want).max() <= 1e-13 * max(1.0, np.abs(want).max())


def test_empty_selections_match_the_reference(built):
    """No columns: the selected rows are zero (the reference's x_full is all
    zero); no rows: an empty product."""
    ref, ex, n = built
    d = ex["dof"]
    for rows, cols in (([1, 2, 7], []), ([], [3, 4]), ([], [])):
        rows, cols = np.array(rows, np.int64), np.array(cols, np.int64)
        sel = HmatSelection(ex, rows, cols, device=-1, plan_only=True)
        assert sel.shape == (d * rows.size, d * cols.size)
        x = np.ones(d * cols.size)
        got, want = sel_matvec(sel, x), ref.selection_matvec(rows, cols, x)
        assert got.shape == want.shape and np.array_equal(got, want)
