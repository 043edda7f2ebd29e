"""Host logic of the CUDA backend, on CPU: the plan (row panels, chunks, LPT
schedule) built by bw_finalize(BW_PLAN_ONLY) is replayed in numpy exactly as
the kernel walks it, and must reproduce the oracle; malformed inputs are
rejected with the documented status codes."""
import numpy as np
import pytest
from conftest import rel
from planreplay import decode, gather_runs, replay

from bigwham_dev_b200 import BigWhamError, HmatGpu
from bigwham_dev_b200 import _capi as A
from oracle import oracle_matvec_perm, oracle_rmatvec_perm


def plan(arr, **kw):
    h = HmatGpu(arr.dof, arr.n_rows, arr.n_cols, arr.perm0, arr.perm1, device=-1)
    h.add_flat(arr.fr, arr.lr, arr.fr_data, arr.lr_data)
    return h.finalize(plan_only=True, **kw)


def test_plan_replay_fp64_forward_and_transpose(golden):
    arr, ex = golden
    h = plan(arr, precisions=("fp64",), transpose=True)
    xp = np.random.default_rng(3).uniform(-1, 1, arr.n_cols)
    assert rel(replay(h, xp, "fp64"), oracle_matvec_perm(arr, xp, 1)) < 1e-14
    xr = np.random.default_rng(4).uniform(-1, 1, arr.n_rows)
    assert rel(replay(h, xr, "fp64", transposed=True), oracle_rmatvec_perm(arr, xr, 1)) < 1e-14


@pytest.mark.parametrize("prec,tol", [("fp32", 2e-6), ("bf16", 8e-3)])
def test_plan_replay_reduced_precision(golden, prec, tol):
    arr, ex = golden
    h = plan(arr, precisions=(prec,))
    xp = np.random.default_rng(3).uniform(-1, 1, arr.n_cols)
    y = replay(h, xp.astype(np.float32).astype(np.float64), prec)
    assert rel(y, oracle_matvec_perm(arr, xp, 1)) < tol


def test_plan_structure(golden):
    arr, ex = golden
    h = plan(arr, precisions=("fp64", "fp32", "bf16"))
    info = h.info()
    assert info["entries"] == arr.fr_data.size + arr.lr_data.size
    assert info["sum_rank"] == int(arr.lr[:, 4].sum())
    for prec, es in (("fp64", 8), ("fp32", 4), ("bf16", 2)):
        for phase in (1, 2):
            p = h.plan_export(prec, phase, with_data=False)
            items = p["item_ptr"]
            assert items[0] == 0 and np.all(np.diff(items) > 0) and items[-1] == len(p["chunks"])
            # each item range opens with its first chunk and closes with its last
            for b in range(len(items) - 1):
                assert decode(p["chunks"][items[b]])["flags"] & 1
                assert decode(p["chunks"][items[b + 1] - 1])["flags"] & 2
            open_item = False
            for w in p["chunks"]:
                d = decode(w)
                assert d["hpad"] % 8 == 0 and d["rows"] <= d["hpad"] <= 512
                cols = (d["ncols"] + 7) // 8 * 8 if prec == "bf16" else d["ncols"]
                assert cols * d["hpad"] * es <= 32768 and d["ncols"] <= 512
                assert (d["data_off"] * es) % 16 == 0  # every chunk starts 16-byte aligned
                if phase == 2:
                    assert d["g_off"] % 4 == 0  # 16-byte aligned slice of the gather array
                # chunks of one item are consecutive: FIRST opens, LAST closes
                assert bool(d["flags"] & 1) != open_item
                open_item = not (d["flags"] & 2)
            assert not open_item
        # the gather runs tile the phase-2 slices exactly
        runs = gather_runs(h, prec, False)
        cols = (runs[:, 2].view(np.uint32) & 0x7FFFFFFF)
        if prec != "bf16":
            assert np.all(runs[:, 3].view(np.float32) == 1.0)
        p2 = h.plan_export(prec, 2, with_data=False)
        assert int(cols.sum()) == sum(decode(w)["ncols"] for w in p2["chunks"])


def test_items_longest_first():
    # 400 equal full blocks on a 20 x 20 block grid, plus a wider last block
    # column: the items come out in non-increasing cost order
    dof, nb, bs = 1, 20, 24
    n = nb * bs
    rng = np.random.default_rng(0)
    h = HmatGpu(dof, n, n, np.arange(n), np.arange(n), device=-1)
    blocks = {}
    for i in range(nb):
        for j in range(nb):
            blocks[i, j] = rng.standard_normal((bs, bs))
            h.add_full(i * bs, j * bs, blocks[i, j])
    h.finalize(plan_only=True)
    p = h.plan_export("fp64", 2)
    # items (FIRST .. LAST chunk runs) come in non-increasing cost order
    cost, cur = [], 0
    for w in p["chunks"]:
        d = decode(w)
        cur += d["ncols"] * d["hpad"] * 8 + 1024
        if d["flags"] & 2:
            cost.append(cur)
            cur = 0
    assert len(cost) == nb and all(a >= b for a, b in zip(cost, cost[1:]))
    # by default the queue hands out one item at a time
    assert len(p["item_ptr"]) == len(cost) + 1
    D = np.block([[blocks[i, j] for j in range(nb)] for i in range(nb)])
    x = rng.standard_normal(n)
    assert rel(replay(h, x), D @ x) < 1e-14


def test_queue_units_group_small_items():
    """The queue hands out runs of whole items, each costing at least
    unit_bytes (but the last); the plan's product does not change."""
    dof, nb, bs = 1, 20, 24
    n = nb * bs
    rng = np.random.default_rng(1)
    blocks = {(i, j): rng.standard_normal((bs, bs)) for i in range(nb) for j in range(nb)}
    x = rng.standard_normal(n)
    outs = []
    for unit in (0, 65536, 300000):
        h = HmatGpu(dof, n, n, np.arange(n), np.arange(n), device=-1).set_tuning(unit_bytes=unit)
        for (i, j), b in blocks.items():
            h.add_full(i * bs, j * bs, b)
        h.finalize(plan_only=True)
        p = h.plan_export("fp64", 2)
        units = p["item_ptr"]
        ucost = [sum(decode(w)["ncols"] * decode(w)["hpad"] * 8 + 1024 for w in p["chunks"][units[b]:units[b + 1]])
                 for b in range(len(units) - 1)]
        assert all(c >= unit for c in ucost[:-1])
        assert decode(p["chunks"][units[0]])["flags"] & 1 and all(
            decode(p["chunks"][u - 1])["flags"] & 2 for u in units[1:])
        n_items = sum(1 for w in p["chunks"] if decode(w)["flags"] & 2)
        if unit == 0:
            assert len(units) - 1 == n_items
        if unit == 300000:
            assert len(units) - 1 < n_items / 2
        outs.append(replay(h, x))
    assert all(np.array_equal(outs[0], o) for o in outs[1:])


def _simple(n=8):
    return HmatGpu(1, n, n, np.arange(n), np.arange(n), device=-1)


def test_rejects_overlap():
    h = _simple()
    h.add_full(0, 0, np.ones((8, 8)))
    h.add_full(0, 4, np.ones((4, 4)))
    with pytest.raises(BigWhamError, match="overlap"):
        h.finalize(plan_only=True)


def test_rejects_gap():
    h = _simple()
    h.add_full(0, 0, np.ones((8, 4)))
    with pytest.raises(BigWhamError, match="not covered"):
        h.finalize(plan_only=True)


def test_rejects_out_of_range():
    h = _simple()
    with pytest.raises(BigWhamError):
        h.add_full(4, 4, np.ones((8, 8)))
        h.finalize(plan_only=True)


def test_rejects_nonfinite_and_allows_opt_out():
    a = np.ones((8, 8))
    a[3, 5] = np.nan
    h = _simple()
    h.add_full(0, 0, a)
    with pytest.raises(BigWhamError, match="non-finite") as e:
        h.finalize(plan_only=True)
    assert e.value.status == A.BW_ERR_ARG
    h = _simple()
    h.add_full(0, 0, a)
    h.finalize(plan_only=True, check_finite=False)


def test_rejects_bad_permutation_and_sizes():
    with pytest.raises(BigWhamError):
        HmatGpu(1, 4, 4, [0, 1, 1, 3], [0, 1, 2, 3], device=-1)
    with pytest.raises(BigWhamError):
        HmatGpu(3, 10, 9, np.arange(3), np.arange(3), device=-1)


def test_lowrank_shapes_checked():
    h = _simple()
    with pytest.raises(ValueError):
        h.add_lowrank(0, 0, np.ones((8, 2)), np.ones((3, 8)))


def test_matvec_on_plan_only_handle_is_a_state_error(golden):
    arr, ex = golden
    h = plan(arr)
    with pytest.raises(BigWhamError) as e:
        h.matvec(np.zeros(arr.n_cols))
    assert e.value.status == A.BW_ERR_STATE


def test_tall_panels_and_high_rank_are_split():
    # a 1-block-row matrix taller than 512 rows and a rank-600 low-rank block
    rng = np.random.default_rng(1)
    n = 1300
    h = HmatGpu(1, n, n, np.arange(n), np.arange(n), device=-1)
    F = rng.standard_normal((n, 700))
    Al, Bl = rng.standard_normal((n, 600)), rng.standard_normal((600, 600))
    h.add_full(0, 0, F)
    h.add_lowrank(0, 700, Al, Bl)
    h.finalize(plan_only=True, precisions=("fp64",), transpose=True)
    x = rng.standard_normal(n)
    D = np.concatenate([F, Al @ Bl], axis=1)
    assert rel(replay(h, x), D @ x) < 1e-13
    assert rel(replay(h, x, transposed=True), D.T @ x) < 1e-13


def test_tuning_changes_the_plan_not_the_result(golden):
    arr, ex = golden
    x = np.random.default_rng(3).uniform(-1, 1, arr.n_cols)
    ref = oracle_matvec_perm(arr, x, 1)
    sizes = set()
    for tuning in ({}, {"items_per_cta_phase1": 32, "items_per_cta_phase2": 2, "chunk_bytes": 4096},
                   {"items_per_cta_phase1": 1, "chunk_bytes": 16384}):
        h = HmatGpu(arr.dof, arr.n_rows, arr.n_cols, arr.perm0, arr.perm1, device=-1)
        h.add_flat(arr.fr, arr.lr, arr.fr_data, arr.lr_data)
        h.finalize(plan_only=True, precisions=("fp64", "bf16"), tuning=tuning)
        assert rel(replay(h, x, "fp64"), ref) < 1e-14
        p = h.plan_export("fp64", 2, with_data=False)
        sizes.add(len(p["chunks"]))
        if tuning.get("chunk_bytes"):
            assert max(decode(w)["ncols"] * decode(w)["hpad"] * 8 for w in p["chunks"]) <= max(
                tuning["chunk_bytes"], 8 * max(decode(w)["hpad"] for w in p["chunks"]))
    assert len(sizes) > 1


def test_tuning_rejects_bad_values():
    h = _simple()
    for k, v in (("chunk_bytes", 1000), ("chunk_bytes", 65536), ("items_per_cta_phase1", 0), ("nope", 1),
                 ("narrow_rows", -1), ("narrow_rows", 65), ("narrow_cols", 0), ("narrow_coop", 2),
                 ("unit_bytes", -1)):
        with pytest.raises(BigWhamError) as e:
            h.set_tuning(**{k: v})
        assert e.value.status == A.BW_ERR_ARG
    h.set_tuning(narrow_rows=0, narrow_cols=1, narrow_coop=1, unit_bytes=0)  # in range
    h.add_full(0, 0, np.ones((8, 8)))
    h.finalize(plan_only=True)
    with pytest.raises(BigWhamError) as e:
        h.set_tuning(chunk_bytes=8192)
    assert e.value.status == A.BW_ERR_STATE
