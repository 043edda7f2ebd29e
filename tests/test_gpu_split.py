"""Phases split between the CTA-wide streaming kernel and the unstaged kernel
(-m gpu).

A phase's queue units, in decreasing cost order, run in stream_panels_kernel
up to the last one with an item of more than narrow_rows padded rows or 512
columns, and warp per unit in narrow_items_kernel after it; with narrow_coop
1 the long units after the last tall one run a CTA per unit in
narrow_items_kernel instead.  Checked against the oracle (oracle_matvec /
oracle_rmatvec, the reference's Hmat::matvec,
src/hmat/hmatrix/hmat.cc:496-558) on synthetic partitions under four
tunings that between them use every mode, every precision within its
rounding bound, and against the same blocks with narrow_rows 0 (every item in
the CTA-wide kernel): the plans differ only in summation order.  The 48-member
2DS0-H batch the same way.
"""
import numpy as np
import pytest
from conftest import rel
from synth import synthetic_hmat

from bigwham_dev_b200 import HmatGpu
from oracle import oracle_matvec, oracle_rmatvec

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-13, "fp32": 2e-6, "bf16": 1e-2}
ORDER = {"fp64": 1e-14, "fp32": 1e-6, "bf16": 1e-3}  # split vs all-wide: summation order only


TUNINGS = [{}, {"narrow_rows": 16}, {"narrow_coop": 1}, {"narrow_rows": 16, "narrow_coop": 1}]


def _handles(arr, precs):
    """The same blocks under each tuning, and with every item CTA-wide."""
    args = (arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0, arr.perm1)
    return [HmatGpu.from_flat(*args, device=0, precisions=precs, transpose=True, tuning=t)
            for t in TUNINGS + [{"narrow_rows": 0}]]


@pytest.mark.parametrize("npr,npc,dof,leaf", [(300, 300, 2, 20), (600, 600, 2, 32), (400, 260, 3, 16)])
def test_split_phases_against_the_oracle(npr, npc, dof, leaf):
    arr = synthetic_hmat(npr, npc, dof, seed=npr + npc + leaf, leaf=leaf, rank0_share=0.2)
    precs = ("fp64", "fp32", "bf16")
    *hs, wide = _handles(arr, precs)
    p2 = wide.plan_export("fp32", 2, with_data=False)
    assert p2["n_wide"] == len(p2["item_ptr"]) - 1
    x = np.random.default_rng(5).uniform(-1, 1, arr.n_cols)
    g = np.random.default_rng(6).uniform(-1, 1, arr.n_rows)
    y_or, yt_or = oracle_matvec(arr, x, 1), oracle_rmatvec(arr, g, 1)
    for p in precs:
        yw, ytw = wide.matvec(x, p), wide.rmatvec(g, p)
        for t, h in zip(TUNINGS, hs):
            y, yt = h.matvec(x, p), h.rmatvec(g, p)
            assert rel(y, y_or) < TOL[p], (p, t)
            assert rel(yt, yt_or) < TOL[p], (p, t)
            assert rel(y, yw) < ORDER[p], (p, t)
            assert rel(yt, ytw) < ORDER[p], (p, t)
            assert np.array_equal(h.matvec(x, p), y), (p, t)  # repeatable bits
    for h in hs + [wide]:
        h.close()


def test_split_batch_against_the_all_wide_handle():
    from test_gpu_batch import c4a_members

    ms = c4a_members()
    precs = ("fp64", "fp32", "bf16")
    hs = [HmatGpu.batch(ms, device=0, precisions=precs, tuning=t) for t in TUNINGS + [{"narrow_rows": 0}]]
    x = np.random.default_rng(7).uniform(-1, 1, hs[0].n_cols)
    for p in precs:
        yw = hs[-1].matvec(x, p)
        for t, h in zip(TUNINGS, hs):
            y = h.matvec(x, p)
            assert np.all(np.isfinite(y)), (p, t)
            assert rel(y, yw) < ORDER[p], (p, t)
    for h in hs:
        h.close()
