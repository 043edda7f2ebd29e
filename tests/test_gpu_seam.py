"""The drop-in seam on the GPU (-m gpu): BigWhamIO built by the reference's own
host code inside libbigwham_host.so, HmatGpu installed with setHmat
(bwh_attach_gpu), then every reference-facing product entry.

Cases: C1 (2DS0-H, 4,000 segments, 8,000 DoF, x ~ U(-1,1) seed 0) and C2
(3DR0-H 128 x 128, 49,152 DoF, seed 1), E = 1, nu = 0.25, leaf 32, eta 3,
eps 1e-5.  The oracle is the reference compiled unmodified (RefHmat, its own
OpenMP matvec on its own build of the same mesh).  FP64 storage, relative
(L2) error <= 1e-12 for:
* BigWhamIO::MatVec(il::ArrayView), host arrays (py_bigwham.cc:204-212);
* BigWhamIO::MatVec(double*, double*) with device pointers, the pybind11
  matvec_raw_ptr (py_bigwham.cc:213-222), which reaches
  HmatGpu::matvecOriginal(double*, double*);
* BigWhamIO::MatVecPerm (bigwham_io.cc:965-971), permuted ordering;
and BigWhamIO::GetDiagonal (bigwham_io.cc:907-916) bitwise.
"""
import numpy as np
import pytest
from conftest import rel

from bigwham_dev_b200.bigwham4py import BigWhamIOGpu
from bigwham_dev_b200.meshes import square_crack_3d, straight_crack_2d
from oracle import RefHmat

pytestmark = pytest.mark.gpu

PROPS = [1.0, 0.25]


def _case(kind):
    if kind == "C1":
        coor, conn = straight_crack_2d(4000)
        return "2DS0-H", coor, conn, 0
    coor, conn = square_crack_3d(128)
    return "3DR0-H", coor, conn, 1


@pytest.mark.parametrize("kind", ["C1", "C2"])
def test_reference_entries_through_the_host_library(kind):
    import torch

    kernel, coor, conn, seed = _case(kind)
    R = RefHmat(kernel, coor, conn, PROPS, 32, 3.0, 1e-5, n_threads=16)
    io = BigWhamIOGpu(coor, conn, kernel, PROPS, 16, useCuda=False)
    io.build_hierarchical_matrix(32, 3.0, 1e-5)
    io.use_cuda = True
    io.attach_gpu(("fp64", "fp32"))
    n = io.matrix_size(1)
    assert (io.matrix_size(0), n) == R.shape
    x = np.random.default_rng(seed).uniform(-1, 1, n)
    y_ref = R.matvec(x)
    # host arrays, original ordering
    assert rel(io.matvec(x), y_ref) < 1e-12
    # permuted ordering
    assert rel(io.matvec_permute(x), R.matvec_perm(x)) < 1e-12
    # device pointers (CuPy / torch / JAX callers of the reference)
    xd = torch.from_numpy(x).cuda()
    yd = torch.full((io.matrix_size(0),), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    io.matvec_raw_ptr(xd.data_ptr(), yd.data_ptr())  # returns once y is complete
    y_dev = yd.cpu().numpy()
    assert rel(y_dev, y_ref) < 1e-12
    # the host and device entries run the same kernels: same bits
    assert np.array_equal(y_dev, io.matvec(x))
    # diagonal: the reference's rule over the FR blocks, bitwise
    assert np.array_equal(io.get_diagonal(), R.diagonal())
    # FP32 storage through the same seam
    io.set_precision("fp32")
    assert rel(io.matvec(x), y_ref) < 2e-6
    io.close()
