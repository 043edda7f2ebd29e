"""The unstaged streaming kernel (narrow_items_kernel), restated lane by lane
in numpy over an exported host plan: the same descriptor words, the same
element indices (column slots of 16-byte row runs for FP64 / FP32, (column,
row-group, column-group) lanes over 8x8 tiles for BF16), the same reductions
over a warp's column lanes and, for CTA-cooperative units (an item's chunks
dealt round robin to 16 warps), over the warps.

Each phase's queue units divide at bw_plan_split: units before n_wide run in
the CTA-wide kernel (restated by planreplay.run_phase), [n_wide, n_coop) a
CTA per unit and the rest warp per unit.  The split is checked against its
rule (by default n_wide = n_coop = one past the last unit with an item of
more than 64 padded rows or 512 columns; with narrow_coop 1, n_wide stops at
the last tall unit and n_coop at the last long one), and the replay of both
launches against the oracle on the golden cases and on synthetic partitions,
H and H^T, every precision within its rounding bound.
"""
import numpy as np
import pytest
from planreplay import build_g2, decode, gather_runs, run_phase

from bigwham_dev_b200 import HmatGpu
from oracle import oracle_matvec_perm, oracle_rmatvec_perm

NARROW_ROWS, NARROW_COLS = 64, 512
TOL = {"fp64": 1e-13, "fp32": 2e-6, "bf16": 1e-2}


def _lanes_fp(hpad, ncols, R):
    """(lane, first row, columns) of a warp over a column-major chunk."""
    lpc = 1
    while lpc * R < hpad:
        lpc *= 2
    cpp = 32 // lpc
    for lane in range(32):
        r0 = (lane % lpc) * R
        if r0 < hpad:
            yield lane, r0, range(lane // lpc, ncols, cpp)


def _lanes_bf16(hpad, ncols):
    """(lane, column group, column, row groups) of a warp over an 8x8-tiled
    chunk."""
    nrg = hpad // 8
    rgl = 1 if nrg <= 1 else 2 if nrg <= 2 else 4
    gpw = 4 // rgl
    ncg = (ncols + 7) // 8
    for lane in range(32):
        c8, rl, cs = lane & 7, (lane >> 3) % rgl, (lane >> 3) // rgl
        rgs = [g for g in (rl, rl + 4) if g < nrg and (g == rl or nrg > 4)]
        for cg in range(cs, ncg, gpw):
            c = 8 * cg + c8
            if c < ncols:
                yield lane, cg, c, rgs


def _warp_chunk(plan, gsrc, precision, d, acc):
    """One warp's pass over one chunk: acc[lane, row] += the lane's products."""
    data = plan["data"]
    hpad, ncols, off, g = d["hpad"], d["ncols"], d["data_off"], d["g_off"]
    assert 0 < hpad <= NARROW_ROWS and hpad % 8 == 0
    if precision == "bf16":
        for lane, cg, c, rgs in _lanes_bf16(hpad, ncols):
            for rg in rgs:
                e = off + cg * 8 * hpad + rg * 64 + (c & 7) * 8
                acc[lane, rg * 8:rg * 8 + 8] += data[e:e + 8] * gsrc[g + c]
    else:
        R = {"fp64": 2, "fp32": 4}[precision]
        for lane, r0, cols in _lanes_fp(hpad, ncols, R):
            for c in cols:
                e = off + c * hpad + r0
                acc[lane, r0:r0 + R] += data[e:e + R] * gsrc[g + c]


def narrow_unit(plan, gsrc, out, precision, cb, ce, cta):
    """One queue unit, warp per unit (cta False) or CTA per unit: warp w of 16
    takes the item's chunks w, w + 16, ..., the warps' rows summed at the end."""
    ds = [decode(plan["chunks"][i]) for i in range(cb, ce)]
    items, start = [], 0
    for k, d in enumerate(ds):
        if d["flags"] & 2:
            items.append(ds[start:k + 1])
            start = k + 1
    assert start == len(ds)
    for item in items:
        assert item[0]["flags"] & 1
        last = item[-1]
        nw = 16 if cta else 1
        acc = np.zeros((nw, 32, last["hpad"]))  # per warp, per lane, per item row
        for k, d in enumerate(item):
            _warp_chunk(plan, gsrc, precision, d, acc[k % nw])
        rows = acc.sum(axis=1).sum(axis=0)[:last["rows"]]  # lanes by shuffles, then warps in order
        out[last["out_off"]:last["out_off"] + last["rows"]] = rows
    return out


def split_rule(plan, rows=NARROW_ROWS, coop=0):
    chunks, units = plan["chunks"], plan["item_ptr"]
    last_tall = last_long = -1
    for u in range(len(units) - 1):
        cols = 0
        for i in range(units[u], units[u + 1]):
            d = decode(chunks[i])
            cols = (0 if d["flags"] & 1 else cols) + d["ncols"]
            last_tall = u if d["hpad"] > rows else last_tall
            last_long = u if cols > NARROW_COLS else last_long
    if coop:
        return last_tall + 1, max(last_tall + 1, last_long + 1)
    return max(last_tall, last_long) + 1, max(last_tall, last_long) + 1


def split_phase(plan, gsrc, out, precision, rows=NARROW_ROWS, coop=0):
    n_wide, n_coop = plan["n_wide"], plan["n_coop"]
    assert (n_wide, n_coop) == split_rule(plan, rows, coop)
    wide = dict(plan, item_ptr=plan["item_ptr"][:n_wide + 1])
    run_phase(wide, gsrc, out, precision == "bf16")
    units = plan["item_ptr"]
    for u in range(n_wide, len(units) - 1):
        narrow_unit(plan, gsrc, out, precision, units[u], units[u + 1], u < n_coop)
    return n_wide, n_coop, len(units) - 1


def narrow_replay(h, x_perm, precision, transposed=False, rows=NARROW_ROWS, coop=0):
    p1 = h.plan_export(precision, 1, transposed)
    p2 = h.plan_export(precision, 2, transposed)
    t = np.zeros(max(1, h.info()["sum_rank"]))
    s1 = split_phase(p1, x_perm, t, precision, rows, coop)
    g2 = build_g2(gather_runs(h, precision, transposed), x_perm, t)
    y = np.full(h.n_cols if transposed else h.n_rows, np.nan)
    s2 = split_phase(p2, g2, y, precision, rows, coop)
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
    if ex["name"] == "2ds0_n256":  # row panels of 62-64 rows, short stacks: every item unstaged
        assert all(w == 0 for w, _, _ in splits), splits
    assert _rel(y, oracle_matvec_perm(arr, x, 1)) < TOL[precision]
    g = np.random.default_rng(2).uniform(-1, 1, arr.n_rows)
    yt, _ = narrow_replay(h, g, precision, transposed=True)
    assert _rel(yt, oracle_rmatvec_perm(arr, g, 1)) < TOL[precision]


def test_split_phases_are_mixed_on_larger_partitions():
    """With narrow_rows 16 the row panels of 24 rows go to the CTA-wide
    kernel, and with narrow_coop 1 items of more than 512 columns run
    CTA-cooperatively: all three modes run, so the replays below cover them."""
    from synth import synthetic_hmat

    modes = set()
    for npr, npc, dof, leaf in MIXED:
        arr = synthetic_hmat(npr, npc, dof, seed=npr + npc + leaf, leaf=leaf, rank0_share=0.2)
        h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                              arr.perm1, device=-1, plan_only=True, precisions=("fp32",), transpose=True,
                              tuning={"narrow_rows": 16, "narrow_coop": 1})
        for ph in (1, 2):
            for t in (False, True):
                p = h.plan_export("fp32", ph, t, with_data=False)
                n = len(p["item_ptr"]) - 1
                modes |= {m for m, k in (("wide", p["n_wide"]), ("coop", p["n_coop"] - p["n_wide"]),
                                         ("warp", n - p["n_coop"])) if k > 0}
    assert modes == {"wide", "coop", "warp"}


MIXED = [(300, 300, 2, 20), (600, 600, 2, 32)]


@pytest.mark.parametrize("npr,npc,dof,leaf", [(40, 25, 2, 4), (96, 96, 2, 16), (17, 60, 3, 8), (200, 130, 1, 32),
                                              (90, 70, 3, 32)] + MIXED)
@pytest.mark.parametrize("precision", ["fp64", "fp32", "bf16"])
@pytest.mark.parametrize("rows,coop", [(64, 0), (64, 1), (16, 1)])
def test_split_restatement_on_synthetic_partitions(npr, npc, dof, leaf, precision, rows, coop):
    from synth import synthetic_hmat

    arr = synthetic_hmat(npr, npc, dof, seed=npr + npc + leaf, leaf=leaf, rank0_share=0.2)
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=-1, plan_only=True, precisions=(precision,), transpose=True,
                          tuning={"narrow_rows": rows, "narrow_coop": coop})
    x = np.random.default_rng(3).uniform(-1, 1, arr.n_cols)
    y, _ = narrow_replay(h, x, precision, rows=rows, coop=coop)
    assert _rel(y, oracle_matvec_perm(arr, x, 1)) < TOL[precision]
    g = np.random.default_rng(4).uniform(-1, 1, arr.n_rows)
    yt, _ = narrow_replay(h, g, precision, transposed=True, rows=rows, coop=coop)
    assert _rel(yt, oracle_rmatvec_perm(arr, g, 1)) < TOL[precision]


def test_launch_count_follows_the_split():
    """bw_matvec_launches: the x gather, the G2 gather and one launch per
    kernel a phase uses."""
    from synth import synthetic_hmat

    arr = synthetic_hmat(600, 600, 2, seed=1264, leaf=32, rank0_share=0.2)
    for tune in ({}, {"narrow_rows": 0}, {"narrow_rows": 16, "narrow_coop": 1}):
        h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                              arr.perm1, device=-1, plan_only=True, precisions=("fp32",), tuning=tune)
        want = 2  # x gather, G2 gather
        for ph in (1, 2):
            p = h.plan_export("fp32", ph, with_data=False)
            n = len(p["item_ptr"]) - 1
            want += (p["n_wide"] > 0) + (p["n_wide"] < n)
        assert h.launches("fp32") == want, tune


def test_batch_split_of_the_48_crack_workload():
    """The 48 x 2DS0-H batch (segments log-uniform in [256, 16,384], seed 3):
    phase 1 splits (long 16-row stacks CTA-wide, the small stacks unstaged),
    phase 2 runs unstaged entirely (row panels of at most 64 rows and 512
    columns); five launches per matvec."""
    from oracle import RefHmat, ref_available
    from bigwham_dev_b200.meshes import straight_crack_2d

    if not ref_available():
        pytest.skip("reference library not built")
    rng = np.random.default_rng(3)
    sizes = np.round(np.exp(rng.uniform(np.log(256), np.log(16384), 48))).astype(int)
    ms = [RefHmat("2DS0-H", *straight_crack_2d(int(n)), [1.0, 0.25], 32, 3.0, 1e-5, n_threads=8).arrays()
          for n in sizes]
    h = HmatGpu.batch(ms, device=-1, precisions=("bf16",), plan_only=True)
    p1 = h.plan_export("bf16", 1, with_data=False)
    p2 = h.plan_export("bf16", 2, with_data=False)
    n1 = len(p1["item_ptr"]) - 1
    assert 0 < p1["n_wide"] < n1 and p1["n_coop"] == p1["n_wide"]
    assert p2["n_wide"] == 0
    assert h.launches("bf16") == 5
