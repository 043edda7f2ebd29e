"""Penny-shaped crack, 3DT0-H, on the GPU (-m gpu).

Workload: a crack of radius 1 in z = 0.
* Mesh: points on a hexagonal lattice of spacing h, clipped to the disk,
  jittered by U(-0.1h, 0.1h) (numpy default_rng(2)), then Delaunay-triangulated.
* Kernel: E = 1, nu = 0.2, leaf 64, eta 3, ACA eps 1e-4.
* Load: unit internal pressure, a normal traction of 1 on every element.
Sizes:
* h = 0.0128 by default (~44 K triangles, ~133 K DoF);
* BW_C3_H=0.0064 runs the full size (177 K triangles, 531 K DoF), whose
  reference build takes minutes.

Checks:
* FP32 / BF16 matvecs against the FP64 dense operator on 2,049 sampled rows
  (683 collocation points x 3 components)
  (the exact kernel, no H-matrix approximation, evaluated by the reference's
  kernel in the oracle).  The bound is the ACA tolerance plus the storage
  rounding (relative 2e-3).
* FP64-refined GMRES with FP32 and with BF16 inner solves: relative residual
  1e-8 on the FP64 H-matrix, solution within 1e-6 of the FP64 GMRES solution.
  The dense-row residual of the solution stays at the ACA level (<= 1e-3).
* Sneddon's opening of a penny crack under uniform pressure,
  w(r) = 8 (1 - nu^2) / (pi E) sqrt(1 - r^2), matched by the normal
  displacement discontinuity away from the rim (r <= 0.8) to 3%.
"""
import os

import numpy as np
import pytest
from conftest import rel

from bigwham_dev_b200 import HmatGpu
from bigwham_dev_b200.meshes import penny_crack_3d
from bigwham_dev_b200.solve import Gmres, refine
from oracle import RefHmat

pytestmark = pytest.mark.gpu

H = float(os.environ.get("BW_C3_H", "0.0128"))
PROPS = [1.0, 0.2]


@pytest.fixture(scope="module")
def penny():
    import torch

    coor, conn = penny_crack_3d(H, seed=2)
    R = RefHmat("3DT0-H", coor, conn, PROPS, 64, 3.0, 1e-4, n_threads=os.cpu_count() or 8)
    arr = R.arrays()
    h = HmatGpu.from_flat(arr.dof, arr.n_rows, arr.n_cols, arr.fr, arr.lr, arr.fr_data, arr.lr_data, arr.perm0,
                          arr.perm1, device=0, precisions=("fp64", "fp32", "bf16"))
    npts = arr.n_rows // 3
    # 683 collocation points = 2,049 sampled rows of the dense operator
    sample = np.sort(np.random.default_rng(7).choice(npts, size=min(683, npts), replace=False))
    D = R.dense_rows("3DT0-H", PROPS, sample)
    rows = (3 * sample[:, None] + np.arange(3)[None, :]).ravel()
    cp = R.collocation_points().reshape(-1, 3)
    b = np.zeros(arr.n_rows)
    b[2::3] = 1.0
    minv = torch.from_numpy(1.0 / h.diagonal()).cuda()
    return {"h": h, "D": D, "rows": rows, "cp": cp, "b": b, "minv": minv}


@pytest.mark.parametrize("prec", ["fp64", "fp32", "bf16"])
def test_matvec_against_dense_rows(penny, prec):
    x = np.random.default_rng(11).uniform(-1, 1, penny["h"].n_cols)
    y = penny["h"].matvec(x, prec)
    err = rel(y[penny["rows"]], penny["D"] @ x)
    print(f"C3 h={H} n={penny['h'].n_rows} {prec} matvec vs dense rows: {err:.3e}")
    assert err < 2e-3


def test_refined_gmres_pressurised_penny(penny):
    import torch

    h, minv = penny["h"], penny["minv"]
    b = torch.from_numpy(penny["b"]).cuda()
    ops = {p: (lambda x, y, p=p: h.matvec(x, p, out=y)) for p in ("fp64", "fp32", "bf16")}
    x64, info = Gmres(ops["fp64"], h.n_rows, restart=50, minv=minv).solve(b, tol=1e-8, maxiter=5000)
    assert info.converged
    X = x64.cpu().numpy()
    for p in ("fp32", "bf16"):
        xr, inf = refine(ops["fp64"], ops[p], b, h.n_rows, minv=minv, tol=1e-8, inner_tol=1e-3, restart=50)
        assert inf.converged, (p, inf.residuals)
        print(f"C3 refine {p}: outer {inf.outer}, inner iterations {inf.iterations}, "
              f"rel err vs FP64 GMRES {rel(xr.cpu().numpy(), X):.2e}")
        r = torch.empty_like(b)
        ops["fp64"](xr, r)
        assert float(torch.linalg.vector_norm(b - r) / torch.linalg.vector_norm(b)) <= 1e-8
        assert rel(xr.cpu().numpy(), X) <= 1e-6, p
    # the solution against the exact operator on the sampled rows
    assert rel(penny["D"] @ X, penny["b"][penny["rows"]]) <= 1e-3
    # Sneddon: w(r) = 8 (1 - nu^2) / (pi E) sqrt(1 - r^2) for unit pressure
    r = np.hypot(penny["cp"][:, 0], penny["cp"][:, 1])
    inner = r <= 0.8
    w = 8 * (1 - PROPS[1] ** 2) / (np.pi * PROPS[0]) * np.sqrt(1 - r[inner] ** 2)
    wn = np.abs(X[2::3][inner])
    print(f"C3 FP64 GMRES iterations {info.iterations}; dense-row residual {rel(penny['D'] @ X, penny['b'][penny['rows']]):.2e}; "
          f"Sneddon rel diff {rel(wn, w):.2e}")
    assert rel(wn, w) < 0.03
