"""gather_g2_kernel's dealing of run values to lanes, restated in numpy: each
warp takes 32 runs (lane k: run k, zero length past the end), an inclusive
scan gives every run its first position in the warp's value list, and value e
finds its run by a 5-step binary search over the starts (the last run whose
start is <= e).  The restated G2 equals planreplay.build_g2 (the runs applied
one by one), every value written once, on the gather runs of synthetic
partitions (H and H^T) and on hand-made runs with zero-length ones mixed in.
"""
import numpy as np
import pytest
from planreplay import build_g2, gather_runs

from bigwham_dev_b200 import HmatGpu

KG2RUNS, UNROLL = 32, 4


def dense_g2(runs, x, t, n):
    """Lane-level restatement of gather_g2_kernel over all warps."""
    g2 = np.zeros(n)
    written = np.zeros(n, dtype=np.int64)
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
                for lane in range(32):
                    e = base + 32 * u + lane
                    r = 0
                    for step in (16, 8, 4, 2, 1):
                        if start[r + step] <= e:
                            r += step
                    if e < total:
                        k = e - start[r]
                        assert 0 <= k < cols[r]
                        g2[dst[r] + k] = sc[r] * (t if src[r] else x)[off[r] + k]
                        written[dst[r] + k] += 1
    return g2, written


def _check(runs, x, t):
    want = build_g2(runs, x, t)
    got, written = dense_g2(runs, x, t, want.size)
    cols = (runs[:, 2].view(np.uint32) & 0x7FFFFFFF).astype(np.int64)
    covered = np.zeros(want.size, dtype=np.int64)
    for d, c in zip(runs[:, 0].astype(np.int64), cols):
        covered[d:d + c] += 1
    assert np.array_equal(written, covered)  # every value once, nothing else
    assert np.array_equal(got, want)


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


def test_dense_g2_with_empty_runs():
    """Zero-length runs (start equal to the next run's) at the warp's start,
    middle and end, and a partial last warp."""
    rng = np.random.default_rng(5)
    n_runs = 75
    cols = rng.integers(1, 40, n_runs)
    cols[[0, 1, 17, 31, 32, 63, 74]] = 0
    dst = np.concatenate([[0], np.cumsum(cols)[:-1]])
    src = rng.integers(0, 2, n_runs)
    x, t = rng.uniform(-1, 1, 5000), rng.uniform(-1, 1, 5000)
    off = rng.integers(0, 4000, n_runs)
    runs = np.zeros((n_runs, 4), np.int32)
    runs[:, 0], runs[:, 1] = dst, off
    runs[:, 2] = (cols.astype(np.uint32) | (src.astype(np.uint32) << 31)).view(np.int32)
    runs[:, 3] = rng.uniform(0.5, 2, n_runs).astype(np.float32).view(np.int32)
    _check(runs, x, t)
