"""Phases split between the CTA-wide streaming kernel and the warp-per-item
kernel (-m gpu).

Each phase's large items (more than 64 padded rows or 512 columns, first in
the queue's cost order) run in stream_panels_kernel and the small items after
them in narrow_items_kernel, two launches in one phase.  Checked against the
oracle (oracle_matvec / oracle_rmatvec, the reference's Hmat::matvec,
src/hmat/hmatrix/hmat.cc:496-558) on synthetic partitions whose phases mix
both kinds and on the 48-member 2DS0-H batch, every precision within its
rounding bound, and against the same handle built with narrow_rows=0 (every
item in the CTA-wide kernel): the two differ only in summation order.
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


def _pair(arr, precs):
    """The same blocks twice: the default split, and every item CTA-wide."""
    args = (arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0, arr.perm1)
    return [HmatGpu.from_flat(*args, device=0, precisions=precs, transpose=True, tuning=t)
            for t in ({}, {"narrow_rows": 0})]


@pytest.mark.parametrize("npr,npc,dof,leaf", [(300, 300, 2, 20), (600, 600, 1, 64), (400, 260, 3, 16)])
def test_split_phases_against_the_oracle(npr, npc, dof, leaf):
    arr = synthetic_hmat(npr, npc, dof, seed=npr + npc + leaf, leaf=leaf, rank0_share=0.2)
    precs = ("fp64", "fp32", "bf16")
    split, wide = _pair(arr, precs)
    p2 = split.plan_export("fp32", 2, with_data=False)
    assert wide.plan_export("fp32", 2, with_data=False)["n_wide"] == len(p2["item_ptr"]) - 1
    x = np.random.default_rng(5).uniform(-1, 1, arr.n_cols)
    g = np.random.default_rng(6).uniform(-1, 1, arr.n_rows)
    y_or, yt_or = oracle_matvec(arr, x, 1), oracle_rmatvec(arr, g, 1)
    for p in precs:
        y, yt = split.matvec(x, p), split.rmatvec(g, p)
        assert rel(y, y_or) < TOL[p], p
        assert rel(yt, yt_or) < TOL[p], p
        assert rel(y, wide.matvec(x, p)) < ORDER[p], p
        assert rel(yt, wide.rmatvec(g, p)) < ORDER[p], p
    split.close()
    wide.close()


def test_split_batch_against_the_all_wide_handle():
    from test_gpu_batch import c4a_members

    ms = c4a_members()
    precs = ("fp64", "fp32", "bf16")
    split = HmatGpu.batch(ms, device=0, precisions=precs)
    wide = HmatGpu.batch(ms, device=0, precisions=precs, tuning={"narrow_rows": 0})
    x = np.random.default_rng(7).uniform(-1, 1, split.n_cols)
    for p in precs:
        ys, yw = split.matvec(x, p), wide.matvec(x, p)
        assert np.all(np.isfinite(ys)), p
        assert rel(ys, yw) < ORDER[p], p
    split.close()
    wide.close()
