"""Batched H-matrices on the GPU (-m gpu): 48 independent 2DS0-H straight
cracks on [-1,1], segment counts log-uniform in [256, 16,384] (numpy
default_rng(3)), E = 1, nu = 0.25, leaf 32, eta = 3, eps = 1e-5, applied by
one bw_matvec on one handle (bw_create_batch).  Each member's slice of y must
equal the reference-restated product of that member alone (FP64 1e-12, FP32
2e-6, BF16 8e-3 relative), forward and transposed, and the batched FP64
product must equal 48 separate handles' products."""
import numpy as np
import pytest
from conftest import rel

from bigwham_dev_b200 import HmatGpu
from bigwham_dev_b200.meshes import straight_crack_2d
from oracle import RefHmat, oracle_matvec, oracle_rmatvec

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 2e-6, "bf16": 8e-3}


def c4a_members(count=48, lo=256, hi=16384, seed=3):
    rng = np.random.default_rng(seed)
    sizes = np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), count))).astype(int)
    out = []
    for n in sizes:
        coor, conn = straight_crack_2d(int(n))
        out.append(RefHmat("2DS0-H", coor, conn, [1.0, 0.25], 32, 3.0, 1e-5, n_threads=16).arrays())
    return out


@pytest.fixture(scope="module")
def batch():
    ms = c4a_members()
    h = HmatGpu.batch(ms, device=0, precisions=("fp64", "fp32", "bf16"), transpose=True)
    return ms, h


@pytest.mark.parametrize("prec", ["fp64", "fp32", "bf16"])
def test_batch_matches_each_member(batch, prec):
    ms, h = batch
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, h.n_cols)
    y = h.matvec(x, prec)
    g = rng.uniform(-1, 1, h.n_rows)
    yt = h.rmatvec(g, prec)
    for k, m in enumerate(ms):
        r0, r1 = h.row_offsets[k], h.row_offsets[k + 1]
        c0, c1 = h.col_offsets[k], h.col_offsets[k + 1]
        assert rel(y[r0:r1], oracle_matvec(m, x[c0:c1], 16)) < TOL[prec], (k, m.n_rows)
        assert rel(yt[c0:c1], oracle_rmatvec(m, g[r0:r1], 16)) < TOL[prec], (k, m.n_rows)


def test_batch_equals_separate_handles(batch):
    import torch

    ms, h = batch
    x = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, h.n_cols)).cuda()
    y = h.matvec(x)
    for k, m in enumerate(ms[:8]):
        s = HmatGpu.from_flat(m.dof, m.n_rows, m.n_cols, m.fr, m.lr, m.fr_data, m.lr_data, m.perm0, m.perm1,
                              device=0, precisions=("fp64",))
        c0, c1 = int(h.col_offsets[k]), int(h.col_offsets[k + 1])
        ys = s.matvec(x[c0:c1].contiguous())
        r0, r1 = int(h.row_offsets[k]), int(h.row_offsets[k + 1])
        assert rel(y[r0:r1].cpu().numpy(), ys.cpu().numpy()) < 1e-14
        s.close()
    h.sync()
