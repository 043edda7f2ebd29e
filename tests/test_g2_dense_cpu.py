"""gather_g2_kernel's dealing of run values to lanes, restated in numpy: each
warp takes 32 runs (lane k: run k, zero length past the end), an inclusive
scan gives every run its first position in the warp's value list, and each
round of 32 positions [w0, w0 + 32) finds the run of w0 + j as the last run
starting at or before w0 (a ballot) plus the number of run starts inside
(w0, w0 + j] (bits of an OR reduction).  The restated G2 equals
planreplay.build_g2 (the runs applied one by one), every value written once,
on the gather runs of synthetic partitions (H and H^T), whose runs are never
empty, and on hand-made runs; with empty runs (which no layout makes) values
may be skipped but nothing is read or written outside a run.
"""
import numpy as np
import pytest
from planreplay import build_g2, gather_runs

from bigwham_dev_b200 import HmatGpu

KG2RUNS, UNROLL = 32, 4


def dense_g2(runs, x, t, n):
    """Lane-level restatement of gather_g2_kernel over all warps; returns G2,
    the write count per entry and the (source flag, index) of every read."""
    g2 = np.zeros(n)
    written = np.zeros(n, dtype=np.int64)
    reads = []
    for r0 in range(0, len(runs), KG2RUNS):
        w = runs[r0:r0 + KG2RUNS]
        cols = np.zeros(32, dtype=np.int64)
        dst = np.zeros(32, dtype=np.int64)
        off = np.zeros(32, dtype=np.int64)
        src = np.zeros(32, dtype=np.int64)
        sc = np.ones(32)
        cols[:len(w)] = w[:, 2].view(np.uint32) & 0x7FFFFFFF
        src[:len(w)] = w[:, 2].view(np.uint32) >> 31
        dst[:len(w)], off[:len(w)] = w[:, 0], w[:, 1]
        sc[:len(w)] = w[:, 3].view(np.float32)
        incl = np.cumsum(cols)
        start, total = incl - cols, int(incl[-1])
        for base in range(0, total, 32 * UNROLL):
            for u in range(UNROLL):
                w0 = base + 32 * u
                holds = [k for k in range(32) if cols[k] > 0 and start[k] <= w0]
                first = max(holds) if holds else 0
                starts = 0
                for k in range(32):
                    o = start[k] - w0
                    if cols[k] > 0 and 0 < o < 32:
                        starts |= 1 << int(o)
                for lane in range(32):
                    e = w0 + lane
                    r = first + bin(starts & ((2 << lane) - 1)).count("1")
                    assert r < 32
                    k = e - start[r]
                    if e < total and 0 <= k < cols[r]:
                        g2[dst[r] + k] = sc[r] * (t if src[r] else x)[off[r] + k]
                        written[dst[r] + k] += 1
                        reads.append((int(src[r]), int(off[r] + k), int(dst[r] + k)))
    return g2, written, reads


def _check(runs, x, t):
    cols = (runs[:, 2].view(np.uint32) & 0x7FFFFFFF).astype(np.int64)
    assert np.all(cols > 0)  # the layout makes no empty run
    want = build_g2(runs, x, t)
    got, written, _ = dense_g2(runs, x, t, want.size)
    covered = np.zeros(want.size, dtype=np.int64)
    for d, c in zip(runs[:, 0].astype(np.int64), cols):
        covered[d:d + c] += 1
    assert np.array_equal(written, covered)  # every value once, nothing else
    assert np.array_equal(got, want)


def _runs(cols, rng, n_src=5000):
    n = len(cols)
    dst = np.concatenate([[0], np.cumsum(cols)[:-1]])
    runs = np.zeros((n, 4), np.int32)
    runs[:, 0], runs[:, 1] = dst, rng.integers(0, n_src - 100, n)
    src = rng.integers(0, 2, n)
    runs[:, 2] = (np.asarray(cols, dtype=np.uint32) | (src.astype(np.uint32) << 31)).view(np.int32)
    runs[:, 3] = rng.uniform(0.5, 2, n).astype(np.float32).view(np.int32)
    return runs


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_dense_g2_on_synthetic_partitions(precision):
    from synth import synthetic_hmat

    for npr, npc, dof, leaf in [(300, 300, 2, 20), (600, 600, 2, 32), (17, 60, 3, 8)]:
        arr = synthetic_hmat(npr, npc, dof, seed=npr + npc + leaf, leaf=leaf, rank0_share=0.2)
        h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                              arr.perm1, device=-1, plan_only=True, precisions=(precision,), transpose=True)
        rng = np.random.default_rng(npr)
        x = rng.uniform(-1, 1, arr.n_cols)
        t = rng.uniform(-1, 1, max(1, h.info()["sum_rank"]))
        for tr in (False, True):
            _check(gather_runs(h, precision, tr), x if not tr else rng.uniform(-1, 1, arr.n_rows), t)


def test_dense_g2_on_hand_made_runs():
    """Runs of 1 to 99 values, runs longer than a round, a partial last warp."""
    rng = np.random.default_rng(5)
    cols = rng.integers(1, 40, 75)
    cols[[3, 40]] = [97, 99]
    x, t = rng.uniform(-1, 1, 5000), rng.uniform(-1, 1, 5000)
    _check(_runs(cols, rng), x, t)


def test_dense_g2_with_empty_runs_stays_inside_the_runs():
    """Empty runs (no layout makes them) may cost values, but every read and
    write stays inside some run."""
    rng = np.random.default_rng(6)
    cols = rng.integers(1, 40, 75)
    cols[[0, 1, 17, 31, 32, 63, 74]] = 0
    runs = _runs(cols, rng)
    x, t = rng.uniform(-1, 1, 5000), rng.uniform(-1, 1, 5000)
    n = int((runs[:, 0] + cols).max())
    _, written, reads = dense_g2(runs, x, t, n)
    assert written.max() <= 1
    src = (runs[:, 2].view(np.uint32) >> 31).astype(np.int64)
    for s_flag, i, d in reads:
        assert any(src[q] == s_flag and runs[q, 1] <= i < runs[q, 1] + cols[q] and runs[q, 0] <= d < runs[q, 0] + cols[q]
                   for q in range(len(runs)))
