"""bw_matvec_static_scratch: the matvec for callers that cannot let a library
allocate device memory (their memory belongs to another allocator, or
cudaMalloc/cudaFree's possible device-wide synchronization is not allowed on
their path).  Its scratch lives in a fixed 64 MiB device array compiled into
the library instead of memory allocated per handle.

Checked through the C ABI against bw_matvec on the same handle, two calls in a
row (the array keeps the previous call's contents): within the tolerances the
other GPU tests use, and bit for bit (the same kernels take the same steps;
only the scratch address differs), in all precisions, for H and H^T, original
and permuted ordering.  After a first call, further calls leave the device's
free memory unchanged.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from bigwham_dev_b200 import BigWhamError, HmatGpu
from bigwham_dev_b200 import _capi as A

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 2e-6, "bf16": 8e-3}


def _static_matvec(h, x, y, flags, stream):
    st = A.lib().bw_matvec_static_scratch(h._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), flags,
                                          C.c_void_p(stream))
    A.check(st, h._h)


@pytest.mark.parametrize("transpose", [False, True])
def test_static_scratch_matches_bw_matvec(golden, transpose):
    import torch

    arr, ex = golden
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=0, precisions=("fp64", "fp32", "bf16"), transpose=transpose)
    nin, nout = (arr.n_rows, arr.n_cols) if transpose else (arr.n_cols, arr.n_rows)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(21)
    for prec, permuted in (("fp64", False), ("fp32", False), ("bf16", False), ("fp64", True), ("bf16", True)):
        flags = A.PRECISIONS[prec] | (A.BW_TRANSPOSE if transpose else 0) | (A.BW_PERMUTED if permuted else 0)
        for call in range(2):
            x = torch.from_numpy(rng.uniform(-1, 1, nin)).cuda()
            y_ref = torch.empty(nout, dtype=torch.float64, device="cuda")
            y = torch.full((nout,), float("nan"), dtype=torch.float64, device="cuda")
            A.check(A.lib().bw_matvec(h._h, C.c_void_p(x.data_ptr()), C.c_void_p(y_ref.data_ptr()), flags,
                                      C.c_void_p(stream)), h._h)
            _static_matvec(h, x, y, flags, stream)
            h.sync(stream)
            err = float(torch.linalg.norm(y - y_ref) / torch.linalg.norm(y_ref))
            assert err <= TOL[prec], (prec, call, err)
            assert torch.equal(y, y_ref), (prec, permuted, call)


def test_static_scratch_allocates_nothing(golden):
    """Once the first call has run on the device, further calls do not change
    the device's free memory."""
    import torch

    arr, ex = golden
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=0, precisions=("fp64", "bf16"))
    stream = torch.cuda.current_stream().cuda_stream
    x = torch.from_numpy(ex["x"]).cuda()
    y = torch.empty(arr.n_rows, dtype=torch.float64, device="cuda")
    _static_matvec(h, x, y, A.BW_FP64, stream)
    h.sync(stream)
    free0, _ = torch.cuda.mem_get_info()
    for prec in ("fp64", "bf16", "fp64"):
        _static_matvec(h, x, y, A.PRECISIONS[prec], stream)
    h.sync(stream)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    h.close()


def test_static_scratch_rejects_oversize():
    import torch

    # one rank-1 block over n x n: the gathered input alone (8 bytes per input
    # in FP64) exceeds the 64 MiB static scratch
    n = 9_000_000
    h = HmatGpu(1, n, n, np.arange(n), np.arange(n), device=0)
    h.add_lowrank(0, 0, np.ones((n, 1)), np.ones((1, n)))
    h.finalize(precisions=("fp64",))
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(BigWhamError, match="static maximum") as e:
        _static_matvec(h, x, y, A.BW_FP64, torch.cuda.current_stream().cuda_stream)
    assert e.value.status == A.BW_ERR_ARG
    h.close()
