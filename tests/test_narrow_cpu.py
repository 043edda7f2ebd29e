"""The warp-per-item kernel of narrow phases (narrow_items_kernel), restated
lane by lane in numpy over an exported host plan: the same descriptor words,
the same element indices (column slots of 16-byte row runs for FP64 / FP32,
(column, row-group) lanes over 8x8 tiles for BF16), the same reductions over
column slots and the same output rows.  Checked against the oracle on the
2DS0-H golden case (whose phases are all narrow: row panels of 62-64 rows)
and on synthetic partitions with 8- to 64-row items, H and H^T, every
precision within its rounding bound.
"""
import numpy as np
import pytest
from planreplay import build_g2, decode, gather_runs, run_phase

from bigwham_dev_b200 import HmatGpu
from oracle import oracle_matvec_perm, oracle_rmatvec_perm

NARROW_ROWS = 64
TOL = {"fp64": 1e-13, "fp32": 2e-6, "bf16": 1e-2}


def narrow_phase(plan, gsrc, out, precision):
    """Lane-level restatement of narrow_items_kernel for one phase."""
    data, chunks, units = plan["data"], plan["chunks"], plan["item_ptr"]
    R = {"fp64": 2, "fp32": 4, "bf16": 1}[precision]
    for u in range(len(units) - 1):
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


def narrow_replay(h, x_perm, precision, transposed=False):
    p1 = h.plan_export(precision, 1, transposed)
    p2 = h.plan_export(precision, 2, transposed)
    tiled = precision == "bf16"
    t = np.zeros(max(1, h.info()["sum_rank"]))
    narrow = {}
    for ph, p in ((1, p1), (2, p2)):
        hp = [decode(w)["hpad"] for w in p["chunks"]]
        narrow[ph] = not hp or max(hp) <= NARROW_ROWS
    (narrow_phase if narrow[1] else lambda pl, g, o, pr: run_phase(pl, g, o, tiled))(p1, x_perm, t, precision)
    g2 = build_g2(gather_runs(h, precision, transposed), x_perm, t)
    y = np.full(h.n_cols if transposed else h.n_rows, np.nan)
    (narrow_phase if narrow[2] else lambda pl, g, o, pr: run_phase(pl, g, o, tiled))(p2, g2, y, precision)
    return y, narrow


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "bf16"])
def test_narrow_restatement_on_the_2ds0_golden(golden, precision):
    arr, ex = golden
    if ex["name"] != "2ds0_n256":
        pytest.skip("the 2DS0-H golden case is the narrow one")
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=-1, plan_only=True, precisions=(precision,), transpose=True)
    x = np.random.default_rng(1).uniform(-1, 1, arr.n_cols)
    y, narrow = narrow_replay(h, x, precision)
    assert narrow[1] and narrow[2]
    assert _rel(y, oracle_matvec_perm(arr, x, 1)) < TOL[precision]
    g = np.random.default_rng(2).uniform(-1, 1, arr.n_rows)
    yt, _ = narrow_replay(h, g, precision, transposed=True)
    assert _rel(yt, oracle_rmatvec_perm(arr, g, 1)) < TOL[precision]


@pytest.mark.parametrize("npr,npc,dof,leaf", [(40, 25, 2, 4), (96, 96, 2, 16), (17, 60, 3, 8), (200, 130, 1, 32)])
@pytest.mark.parametrize("precision", ["fp64", "fp32", "bf16"])
def test_narrow_restatement_on_synthetic_partitions(npr, npc, dof, leaf, precision):
    from synth import synthetic_hmat

    arr = synthetic_hmat(npr, npc, dof, seed=npr + npc + leaf, leaf=leaf, rank0_share=0.2)
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=-1, plan_only=True, precisions=(precision,), transpose=True)
    x = np.random.default_rng(3).uniform(-1, 1, arr.n_cols)
    y, narrow = narrow_replay(h, x, precision)
    assert narrow[1] and narrow[2]
    assert _rel(y, oracle_matvec_perm(arr, x, 1)) < TOL[precision]
    g = np.random.default_rng(4).uniform(-1, 1, arr.n_rows)
    yt, _ = narrow_replay(h, g, precision, transposed=True)
    assert _rel(yt, oracle_rmatvec_perm(arr, g, 1)) < TOL[precision]
