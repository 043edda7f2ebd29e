"""Failure detection on the GPU without faulting it (-m gpu).

bw_test_withhold_chunk makes CTA 0 of the next streaming launch skip staging
one chunk: a barrier that nothing completes.  With a 20 ms wait limit
(bw_set_wait_limit) the wait for it runs out.  The timed-out kernel:
* writes an error word;
* lets its bulk copies and tensor-core work finish (those waits keep a fixed
  2 s bound);
* frees its TMEM and returns.
The next sync reports BW_ERR_DEVICE.  With the default limit restored the same
handle gives the bitwise-same results as before: no state is left behind
(error word, work-queue counters, TMEM).
"""
import numpy as np
import pytest

from bigwham_dev_b200 import BigWhamError, HmatGpu
from bigwham_dev_b200 import _capi as A
from bigwham_dev_b200.meshes import square_crack_3d
from oracle import RefHmat

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handle():
    coor, conn = square_crack_3d(48)
    arr = RefHmat("3DR0-H", coor, conn, [1.0, 0.25], 32, 3.0, 1e-5, n_threads=16).arrays()
    return HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                             arr.perm1, device=0, precisions=("fp64", "bf16"), matmat=True)


def test_timeout_reported_and_handle_recovers(handle):
    import torch

    h = handle
    x = torch.from_numpy(np.random.default_rng(0).uniform(-1, 1, h.n_cols)).cuda()
    X = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, (h.n_cols, 8))).cuda()
    good = {p: h.matvec(x, p).clone() for p in ("fp64", "bf16")}
    good_mm = h.matmat(X, "bf16").clone()
    h.sync()
    h.set_wait_limit(20_000_000)
    for run in (lambda: h.matvec(x, "fp64"), lambda: h.matvec(x, "bf16"), lambda: h.matmat(X, "bf16")):
        A.check(A.lib().bw_test_withhold_chunk(h._h, 1), h._h)
        run()
        with pytest.raises(BigWhamError) as e:
            h.sync()
        assert e.value.status == A.BW_ERR_DEVICE
        assert "error word" in str(e.value)
    h.set_wait_limit(2_000_000_000)
    for p in ("fp64", "bf16"):
        assert torch.equal(h.matvec(x, p), good[p])
    assert torch.equal(h.matmat(X, "bf16"), good_mm)
    h.sync()


def test_wait_limit_range_checked(handle):
    for bad in (0, -5, 10 ** 12):
        with pytest.raises(BigWhamError) as e:
            handle.set_wait_limit(bad)
        assert e.value.status == A.BW_ERR_ARG
