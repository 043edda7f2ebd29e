"""Block files on the GPU (run on a B200: -m gpu).

A handle made by bw_create_from_file from a block file of a golden case must
give the same bits as the handle made from the same flat arrays, for every
precision and for H^T, and match the golden reference product (FP64 to 1e-12
relative, as in test_gpu_matvec).
"""
import numpy as np
import pytest
from conftest import rel

from bigwham_dev_b200 import HmatGpu, blockfile

pytestmark = pytest.mark.gpu

PRECS = ("fp64", "fp32", "bf16")


def test_handle_from_file_matches_the_flat_upload(golden, tmp_path):
    arr, ex = golden
    flat = {"dof": arr.dof, "n_rows": arr.n_rows, "n_cols": arr.n_cols, "fr": arr.fr, "lr": arr.lr,
            "fr_data": arr.fr_data, "lr_data": arr.lr_data, "perm0": arr.perm0, "perm1": arr.perm1}
    path = tmp_path / "golden.bwb"
    blockfile.write(path, flat)
    kw = dict(device=0, precisions=PRECS, transpose=True)
    h_flat = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data,
                               arr.perm0, arr.perm1, **kw)
    h_file = HmatGpu.from_file(path, verify=True, **kw)
    x = ex["x"]
    xr = np.random.default_rng(9).uniform(-1, 1, arr.n_rows)
    for p in PRECS:
        assert np.array_equal(h_file.matvec(x, p), h_flat.matvec(x, p)), p
        assert np.array_equal(h_file.rmatvec(xr, p), h_flat.rmatvec(xr, p)), p
    assert rel(h_file.matvec(x), ex["y_ref"]) < 1e-12
    assert np.array_equal(h_file.diagonal(), ex["diag_ref"])
    h_file.sync()
    h_flat.sync()
