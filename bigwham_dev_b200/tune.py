"""Plan autotuner: sweeps the plan parameters of bw_set_tuning on one GPU and
writes the measured table and the best configuration as JSON.

    python -m bigwham_dev_b200.tune --mesh 256 --precision bf16    # matvec
    python -m bigwham_dev_b200.tune --mesh 256 --matmat            # 64-RHS matmat
        -> bigwham_dev_b200/tuning/3dr0_256x256.json

Workload: the 3DR0-H square crack of bench.py.
* Mesh and kernel: n x n rectangles on [-1,1]^2, E = 1, nu = 0.25, leaf 32,
  eta 3, ACA eps 1e-5.
* The H-matrix is built once by the reference's host code.
* Each configuration uploads the blocks with its parameters, then times
  `--steps` matvecs with CUDA events after `--warmup` untimed ones.  x is
  U(-1,1), seed 1.

Parameters (they move item and chunk boundaries, and with them the order of
the additions that make an output row, so results agree to rounding; for
fixed parameters they are repeatable bit for bit):
* items_per_cta_phase1 / items_per_cta_phase2: granularity of the work queue
  (items per CTA share; more items balance better but cost more item ends);
* chunk_bytes: block data per pipeline chunk (fewer bytes mean more chunks
  and more descriptor overhead);
* mm_items_per_cta (--matmat): granularity of the matmat's phase 1.

bench.py applies the best configuration of its workload when the file exists.
"""
from __future__ import annotations

import argparse
import itertools
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TUNING_DIR = os.path.join(HERE, "tuning")
GRID = {"items_per_cta_phase1": [1, 2, 4, 8], "items_per_cta_phase2": [2, 4, 8],
        "chunk_bytes": [24576, 32768]}
MM_GRID = {"mm_items_per_cta": [1, 2, 4, 8, 16]}


def tuning_path(mesh: int) -> str:
    return os.path.join(TUNING_DIR, f"3dr0_{mesh}x{mesh}.json")


def load_best(mesh: int, precision: str = "bf16") -> dict | None:
    """The committed best configuration for the 3DR0-H mesh (the matvec entry
    of `precision` merged with the matmat entry), or None."""
    try:
        with open(tuning_path(mesh)) as f:
            best = json.load(f)["best"]
    except (OSError, KeyError, ValueError):
        return None
    out = {**best.get(precision, {}), **best.get("matmat_bf16", {})}
    return out or None


def main(argv=None) -> int:
    import torch

    from . import HmatGpu
    from .bigwham4py import BigWhamIOGpu
    from .meshes import square_crack_3d

    ap = argparse.ArgumentParser()
    ap.add_argument("--mesh", type=int, default=256)
    ap.add_argument("--precision", default="bf16", choices=["fp64", "fp32", "bf16"])
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--out", default=None)
    ap.add_argument("--matmat", action="store_true",
                    help="tune the 64-right-hand-side tensor-core matmat (BF16) instead of the matvec")
    a = ap.parse_args(argv)

    t0 = time.time()
    coor, conn = square_crack_3d(a.mesh)
    io = BigWhamIOGpu(coor, conn, "3DR0-H", [1.0, 0.25], os.cpu_count() or 1, useCuda=False)
    io.build_hierarchical_matrix(32, 3.0, 1e-5)
    ex = io.export_blocks()
    io.close()
    build_s = time.time() - t0
    grid = MM_GRID if a.matmat else GRID
    entry = "matmat_bf16" if a.matmat else a.precision
    k = 64 if a.matmat else 1
    x = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, (k, ex["n_cols"]))).cuda().t()
    y = torch.empty(k, ex["n_rows"], dtype=torch.float64, device="cuda").t()
    x1, y1 = x[:, 0].contiguous(), y[:, 0].contiguous()

    def step(h):
        if a.matmat:
            h.matmat(x, "bf16", out=y)
        else:
            h.matvec(x1, a.precision, out=y1)

    rows = []
    keys = list(grid)
    for vals in itertools.product(*(grid[kk] for kk in keys)):
        cfg = dict(zip(keys, vals))
        h = HmatGpu.from_flat(ex["dof"], ex["n_rows"], ex["n_cols"], ex["fr"], ex["lr"], ex["fr_data"],
                              ex["lr_data"], ex["perm0"], ex["perm1"], device=0,
                              precisions=("bf16",) if a.matmat else (a.precision,), matmat=a.matmat, tuning=cfg)
        for _ in range(a.warmup):
            step(h)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(a.steps):
            step(h)
        e1.record()
        torch.cuda.synchronize()
        h.sync()
        ms = e0.elapsed_time(e1) / a.steps
        rows.append({**cfg, "ms_per_matmat64" if a.matmat else "ms_per_matvec": ms})
        print(json.dumps(rows[-1]), flush=True)
        h.close()
    metric = "ms_per_matmat64" if a.matmat else "ms_per_matvec"
    best = min(rows, key=lambda r: r[metric])
    out = a.out or tuning_path(a.mesh)
    prev = {}
    if os.path.exists(out):
        with open(out) as f:
            prev = json.load(f)
    doc = {"workload": f"3DR0-H square crack {a.mesh}x{a.mesh} ({3 * a.mesh * a.mesh:,} DoF), leaf 32, eta 3, "
                       "ACA eps 1e-5, x ~ U(-1,1) seed 1",
           "device": torch.cuda.get_device_name(0), "host_build_s": round(build_s, 1),
           "timing": f"CUDA events, {a.steps} products after {a.warmup} warm-up",
           "results": {**prev.get("results", {}), entry: rows},
           "best": {**prev.get("best", {}), entry: {kk: best[kk] for kk in keys}}}
    os.makedirs(os.path.dirname(out), exist_ok=True)
    with open(out, "w") as f:
        json.dump(doc, f, indent=1)
    print("best", entry, json.dumps(doc["best"][entry]), f"{best[metric]:.4f} ms", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
