"""The warp-per-item kernel (narrow_items_kernel), restated lane by lane in
numpy over an exported host plan: the same descriptor words, the same element
indices (column slots of 16-byte row runs for FP64 / FP32, (column,
row-group) lanes over 8x8 tiles for BF16), the same reductions over column
slots and the same output rows.

Each phase's items divide at bw_plan_split: the items before it run in the
CTA-wide kernel (restated by planreplay.run_phase), the small items after it
(at most 64 padded rows and 512 columns, in the queue's cost order) warp per
item.  The split is checked against that rule, and the replay of both
launches against the oracle on the golden cases (2DS0-H: every item narrow;
3DR0-H: mixed) and on synthetic partitions, H and H^T, every precision within
its rounding bound.
"""
import numpy as np
import pytest
from planreplay import build_g2, decode, gather_runs, run_phase

from bigwham_dev_b200 import HmatGpu
from oracle import oracle_matvec_perm, oracle_rmatvec_perm

NARROW_ROWS, NARROW_COLS = 64, 512
TOL = {"fp64": 1e-13, "fp32": 2e-6, "bf16": 1e-2}


def narrow_phase(plan, gsrc, out, precision, u0=0):
    """Lane-level restatement of narrow_items_kernel over units [u0, end)."""
    data, chunks, units = plan["data"], plan["chunks"], plan["item_ptr"]
    R = {"fp64": 2, "fp32": 4, "bf16": 1}[precision]
    for u in range(u0, len(units) - 1):
        acc = None
        for i in range(units[u], units[u + 1]):
            d = decode(chunks[i])
            hpad, ncols, off, g = d["hpad"], d["ncols"], d["data_off"], d["g_off"]
            assert 0 < hpad <= NARROW_ROWS and hpad % 8 == 0
            if d["flags"] & 1:
                acc = np.zeros((32, hpad))  # per lane, per item row
            if precision == "bf16":
                nrg = hpad // 8
                for lane in range(32):
                    c8, slot = lane & 7, lane >> 3
                    for cg in range((ncols + 7) // 8):
                        c = 8 * cg + c8
                        if c >= ncols:
                            continue
                        for j in (0, 1):
                            rg = slot + 4 * j
                            if rg < nrg:
                                e = off + cg * 8 * hpad + rg * 64 + c8 * 8
                                acc[lane, rg * 8:rg * 8 + 8] += data[e:e + 8] * gsrc[g + c]
            else:
                lpc = 1
                while lpc * R < hpad:
                    lpc *= 2
                cpp = 32 // lpc
                for lane in range(32):
                    slot, r0 = lane // lpc, (lane % lpc) * R
                    if r0 >= hpad:
                        continue
                    for c in range(slot, ncols, cpp):
                        e = off + c * hpad + r0
                        acc[lane, r0:r0 + R] += data[e:e + R] * gsrc[g + c]
            if d["flags"] & 2:
                rows = acc.sum(axis=0)[:d["rows"]]  # the shuffles sum the column slots
                out[d["out_off"]:d["out_off"] + d["rows"]] = rows
    return out


def split_rule(plan):
    """First unit after which every unit is small (<= 64 padded rows and <= 512
    columns per item)."""
    chunks, units = plan["chunks"], plan["item_ptr"]
    split = 0
    for u in range(len(units) - 1):
        cols, small = 0, True
        for i in range(units[u], units[u + 1]):
            d = decode(chunks[i])
            cols = (0 if d["flags"] & 1 else cols) + d["ncols"]
            small &= d["hpad"] <= NARROW_ROWS and cols <= NARROW_COLS
        if not small:
            split = u + 1
    return split


def split_phase(plan, gsrc, out, precision):
    n_wide = plan["n_wide"]
    assert n_wide == split_rule(plan)
    wide = dict(plan, item_ptr=plan["item_ptr"][:n_wide + 1])
    run_phase(wide, gsrc, out, precision == "bf16")
    narrow_phase(plan, gsrc, out, precision, n_wide)
    return n_wide, len(plan["item_ptr"]) - 1


def narrow_replay(h, x_perm, precision, transposed=False):
    p1 = h.plan_export(precision, 1, transposed)
    p2 = h.plan_export(precision, 2, transposed)
    t = np.zeros(max(1, h.info()["sum_rank"]))
    s1 = split_phase(p1, x_perm, t, precision)
    g2 = build_g2(gather_runs(h, precision, transposed), x_perm, t)
    y = np.full(h.n_cols if transposed else h.n_rows, np.nan)
    s2 = split_phase(p2, g2, y, precision)
    return y, (s1, s2)


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "bf16"])
def test_split_restatement_on_the_golden_cases(golden, precision):
    arr, ex = golden
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=-1, plan_only=True, precisions=(precision,), transpose=True)
    x = np.random.default_rng(1).uniform(-1, 1, arr.n_cols)
    y, splits = narrow_replay(h, x, precision)
    if ex["name"] == "2ds0_n256":  # row panels of 62-64 rows, short stacks: every item narrow
        assert all(w == 0 for w, _ in splits), splits
    assert _rel(y, oracle_matvec_perm(arr, x, 1)) < TOL[precision]
    g = np.random.default_rng(2).uniform(-1, 1, arr.n_rows)
    yt, _ = narrow_replay(h, g, precision, transposed=True)
    assert _rel(yt, oracle_rmatvec_perm(arr, g, 1)) < TOL[precision]


def test_split_phases_are_mixed_on_larger_partitions():
    """Partitions with row panels and stacks of more than 512 columns split:
    both launches of a phase run, so the replays below cover both."""
    from synth import synthetic_hmat

    for npr, npc, dof, leaf in MIXED:
        arr = synthetic_hmat(npr, npc, dof, seed=npr + npc + leaf, leaf=leaf, rank0_share=0.2)
        h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                              arr.perm1, device=-1, plan_only=True, precisions=("fp32",))
        p = h.plan_export("fp32", 2, with_data=False)
        assert 0 < p["n_wide"] < len(p["item_ptr"]) - 1


MIXED = [(300, 300, 2, 20), (600, 600, 1, 64)]


@pytest.mark.parametrize("npr,npc,dof,leaf", [(40, 25, 2, 4), (96, 96, 2, 16), (17, 60, 3, 8), (200, 130, 1, 32),
                                              (90, 70, 3, 32)] + MIXED)
@pytest.mark.parametrize("precision", ["fp64", "fp32", "bf16"])
def test_split_restatement_on_synthetic_partitions(npr, npc, dof, leaf, precision):
    from synth import synthetic_hmat

    arr = synthetic_hmat(npr, npc, dof, seed=npr + npc + leaf, leaf=leaf, rank0_share=0.2)
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=-1, plan_only=True, precisions=(precision,), transpose=True)
    x = np.random.default_rng(3).uniform(-1, 1, arr.n_cols)
    y, _ = narrow_replay(h, x, precision)
    assert _rel(y, oracle_matvec_perm(arr, x, 1)) < TOL[precision]
    g = np.random.default_rng(4).uniform(-1, 1, arr.n_rows)
    yt, _ = narrow_replay(h, g, precision, transposed=True)
    assert _rel(yt, oracle_rmatvec_perm(arr, g, 1)) < TOL[precision]
