#!/usr/bin/env python
"""H-matvec benchmark on one node (one process per GPU).

Workload: 3DR0-H planar square crack, 256 x 256 rectangles on [-1,1]^2 in
z = 0 (196,608 DoF), E = 1, nu = 0.25, leaf 32, eta 3, ACA eps 1e-5; the
reference's own host code builds the H-matrix (mesh, kernel, cluster tree,
ACA: libbigwham_host.so), the blocks are uploaded once in FP64, FP32 and BF16
(per-block FP32 scale), and one step is one H x over the whole matrix with
x ~ U(-1,1) (seed 1) resident in HBM.  The headline value is the FP32-storage
(FP32 accumulation) rate: the storage whose matvec stays within 1e-6 of the
FP64 GPU matvec.  The FP64 and BF16 rates ride along; BF16 reaches 1e-6 only
through FP64-refined GMRES (the north-star solve checks in the same line).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

N > 1 runs N independent replicas (weak scaling, no collective on the data
path): rank 0 builds the H-matrix once and shares the flat blocks through
shared memory; every rank uploads and applies its own copy.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("H-matvec/s & %HBM roofline, 3DR0-H 196,608 DoF, mixed (FP32 blocks, FP32 accumulation) vs FP64 GPU "
          "at <=1e-6 rel err; FP64 and BF16 alongside")
HEAD = "fp32"  # headline storage precision
UNIT = "matvec/s"
PROPS = [1.0, 0.25]
LEAF, ETA, EPS = 32, 3.0, 1e-5
L2_NOTE = "inputs larger than L2: every step streams all block data (GB-scale) from HBM"


def workload(n):
    return {"workload": f"3DR0-H square crack {n}x{n} rectangles ({3 * n * n:,} DoF), E=1 nu=0.25, "
                        f"leaf {LEAF}, eta {ETA:g}, ACA eps {EPS:g}, one H x per step, x~U(-1,1) seed 1",
            "mesh": f"{n}x{n}", "dof": 3 * n * n,
            # FP64 block bytes grow ~ 0.3 GB per 10^4 DoF here; below ~64x64 the blocks fit in the 126 MB L2
            "l2": L2_NOTE if n >= 64 else "small mesh: the block data may be L2-resident (not a bandwidth figure)"}


def read_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def read_traffic(kernel_key):
    """Per-launch DRAM traffic of the dominant kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f).get(kernel_key)
    except Exception:
        return None


class ClockSampler:
    """SM clock and clock-event reasons of the GPU polled through NVML by a
    thread every 2 ms; window()/end() bracket the timed loops, and the report
    covers the samples inside them."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, device_index, period_s=0.002):
        self.dev, self.period = int(device_index), period_s
        self.samples, self.windows = [], []
        self.nv, self.h, self.thread, self.err = None, None, None, None
        self._stop = False

    def _handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:  # the CUDA device's NVML handle, whatever CUDA_VISIBLE_DEVICES says
            pr = torch.cuda.get_device_properties(self.dev)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def start(self):
        import threading

        try:
            self.nv, self.h = self._handle()
        except Exception as e:  # no NVML: the report says so
            self.err = f"NVML unavailable: {e}"
            return

        def run():
            nv = self.nv
            while not self._stop:
                try:
                    self.samples.append((time.perf_counter(), nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM),
                                         nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)))
                except Exception as e:
                    self.err = str(e)
                    return
                time.sleep(self.period)

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def window(self):
        self.windows.append([time.perf_counter(), None])

    def end(self):
        if self.windows and self.windows[-1][1] is None:
            self.windows[-1][1] = time.perf_counter()

    def stop(self):
        if self.thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.err or "not sampled"], "samples": 0}
        self._stop = True
        self.thread.join(timeout=5)
        inside = [s for s in self.samples if any(w0 <= s[0] <= (w1 or s[0]) for w0, w1 in self.windows)]
        use = inside or self.samples
        sm = [float(s[1]) for s in use]
        mask = 0
        for s in use:
            mask |= int(s[2])
        reasons = sorted(n for n, attr in self.REASONS if mask & int(getattr(self.nv, attr, 0)))
        try:
            mx = float(self.nv.nvmlDeviceGetMaxClockInfo(self.h, self.nv.NVML_CLOCK_SM))
        except Exception:
            mx = max(sm) if sm else None
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(use), "source": "NVML, every 2 ms, inside the timed loops"
                if inside else "NVML, every 2 ms (no sample inside the timed loops)"}


def dist_setup(n_gpus, backend="nccl"):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=900), device_id=None)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(v, world, device="cuda"):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shared_block_file(world, rank, path, build, keep=False):
    """Replicas share one H-matrix build through a block file: rank 0 runs
    build(path), which writes it (BigWhamIOGpu.write_to_file), unless `path`
    already exists; then every rank maps it (HmatGpu.from_file).  Returns
    release(); release() (all ranks, after their upload) removes the file
    unless keep."""
    if rank == 0 and not os.path.exists(path):
        build(path)
    barrier(world)

    def release():
        barrier(world)
        if rank == 0 and not keep:
            os.unlink(path)

    return release


# ----------------------------------------------------------------------------- reference arm
def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from bigwham_dev_b200.meshes import square_crack_3d

    base = {"impl": "reference", "metric": METRIC, "unit": UNIT, "higher_is_better": True,
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup}
    try:
        from oracle import RefHmat, ref_available
    except Exception as e:  # pragma: no cover
        print(json.dumps({**base, "unavailable": f"oracle import failed: {e}"}))
        return 0
    if not ref_available():
        print(json.dumps({**base, "unavailable": "reference library oracle/_ref/libbigwham_ref.so not built"}))
        return 0
    threads = os.cpu_count() or 1
    coor, conn = square_crack_3d(a.mesh)
    t0 = time.time()
    R = RefHmat("3DR0-H", coor, conn, PROPS, LEAF, ETA, EPS, n_threads=threads)
    build_s = time.time() - t0
    x = np.random.default_rng(1).uniform(-1.0, 1.0, R.shape[1])
    t0 = time.perf_counter()
    R.matvec(x)
    est = time.perf_counter() - t0
    for _ in range(max(0, min(a.warmup, int(5.0 / max(est, 1e-6))) - 1)):
        R.matvec(x)
    k = max(1, min(a.steps, int(a.ref_budget_s / max(est, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(k):
        R.matvec(x)
    dt = time.perf_counter() - t0
    v = k / dt
    sample = (f"{k} of {a.steps} steps timed (each a full BigWhamIO::MatVec of the {3 * a.mesh * a.mesh:,}-DoF "
              f"H-matrix, OpenMP over {threads} threads, 1 BLAS thread); H-matrix build {build_s:.1f} s untimed")
    print(json.dumps({**base, "value": v, "ms_per_step": 1e3 * dt / k, "scaling": "weak", "vs_baseline": None,
                      "dtype": "f64", "data": "synthetic mesh (no dataset)", "config": workload(a.mesh),
                      "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                                       "sample": sample},
                      "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


# ----------------------------------------------------------------------------- our arm
def build_hmatrix(a, world, rank, local):
    """Returns (io or None, HmatGpu, setup info).  N = 1: the product host path
    (BigWhamIO built by the reference's code, HmatGpu installed via setHmat).
    N > 1: rank 0 builds once and shares the flat blocks in /dev/shm."""
    from bigwham_dev_b200 import HmatGpu
    from bigwham_dev_b200.bigwham4py import BigWhamIOGpu
    from bigwham_dev_b200.meshes import square_crack_3d

    from bigwham_dev_b200.tune import load_best

    precs = tuple(a.precisions)
    tuning = load_best(a.mesh, "bf16")  # committed autotuner result for this mesh, if any
    if a.tune:
        tuning = {**(tuning or {}), **a.tune}
    info = {"tuning": tuning or "defaults"}
    coor, conn = square_crack_3d(a.mesh)
    if world == 1:
        if a.block_file and os.path.exists(a.block_file):
            # blocks saved by an earlier run: no host rebuild, e2e through HmatGpu.matvec(host arrays)
            from bigwham_dev_b200 import blockfile

            head = blockfile.info(a.block_file)
            t0 = time.time()
            h = HmatGpu.from_file(a.block_file, device=local, verify=True, precisions=precs, transpose=False,
                                  matmat=a.matmat, tuning=tuning)
            info["upload_s"] = round(time.time() - t0, 2)
            info["block_file"] = f"{a.block_file} (read; host build skipped)"
            info["compression"] = (head["fr_entries"] + head["lr_entries"]) / (head["n_rows"] * head["n_cols"])
            return None, h, info
        t0 = time.time()
        io = BigWhamIOGpu(coor, conn, "3DR0-H", PROPS, os.cpu_count() or 1, useCuda=False, device=local)
        io.build_hierarchical_matrix(LEAF, ETA, EPS)
        info["host_build_s"] = round(time.time() - t0, 2)
        if a.block_file:
            io.write_to_file(a.block_file)
            info["block_file"] = f"{a.block_file} (written)"
        t0 = time.time()
        io.use_cuda = True
        h = io.attach_gpu(precs, transpose=False, matmat=a.matmat, tuning=tuning)
        info["upload_s"] = round(time.time() - t0, 2)
        info["compression"] = io.get_compression_ratio()
        return io, h, info
    # replicas: one build, shared as a block file (in /dev/shm unless --block-file names one)
    tag = os.environ.get("TORCHELASTIC_RUN_ID", "bench") + f"_{a.mesh}"
    path = a.block_file or os.path.join("/dev/shm", f"bw_blocks_{tag}.bwb")
    reused = os.path.exists(path)

    def build(p):
        t0 = time.time()
        io = BigWhamIOGpu(coor, conn, "3DR0-H", PROPS, os.cpu_count() or 1, useCuda=False, device=local)
        io.build_hierarchical_matrix(LEAF, ETA, EPS)
        io.write_to_file(p)
        info["host_build_s"] = round(time.time() - t0, 2)
        io.close()

    release = shared_block_file(world, rank, path, build, keep=a.block_file is not None)
    t0 = time.time()
    h = HmatGpu.from_file(path, device=local, verify=reused, precisions=precs, matmat=a.matmat, tuning=tuning)
    info["upload_s"] = round(time.time() - t0, 2)
    release()
    return None, h, info


def _events_ms(fn, steps):
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def time_matmat(a, h, dev, peak, ms_bf16_matvec):
    """H X for 64 right-hand sides on the tensor cores (BF16 matmat layout):
    3 launches per product (X gather, phase 1, phase 2).  Returns the report
    and (X, Y[:, [0, 63]]) on the host for the oracle check."""
    import torch

    k = 64
    X_host = np.random.default_rng(5).uniform(-1, 1, (h.n_cols, k))
    X = torch.from_numpy(X_host).to(dev).t().contiguous().t()
    Y = torch.empty(k, h.n_rows, dtype=torch.float64, device=dev).t()
    for _ in range(a.warmup):
        h.matmat(X, "bf16", out=Y)
    steps = max(3, min(a.steps, 50))
    ms = _events_ms(lambda: h.matmat(X, "bf16", out=Y), steps)
    ref = next(p for p in ("fp64", "fp32", "bf16") if p in a.precisions)  # most accurate stored matvec
    errs = []
    for j in (0, k - 1):
        yr = h.matvec(X[:, j].contiguous(), ref)
        errs.append(float(torch.linalg.vector_norm(Y[:, j] - yr) / torch.linalg.vector_norm(yr)))
    block = 0
    for phase in (1, 2):
        c = h.mm_plan_export(phase)["chunks"].astype(np.int64)
        block += int((c[:, 2] * c[:, 3] * 2).sum())
    cols = Y[:, [0, k - 1]].cpu().numpy()
    return ({"workload": f"3DR0-H {a.mesh}x{a.mesh}, 64 right-hand sides ~U(-1,1) seed 5, BF16 blocks and X, "
                         "FP32 accumulate (tcgen05, TMEM accumulators)",
             "steps": steps, "ms_per_matmat": ms, "rhs_per_s": k / (ms * 1e-3),
             "per_rhs_speedup_vs_bf16_matvec": ms_bf16_matvec * k / ms, "block_bytes": block,
             "block_gbs": block / (ms * 1e-3) / 1e9,
             "roofline_frac_of_measured_hbm": block / (ms * 1e-3) / 1e9 / peak,
             f"rel_err_vs_{ref}_gpu_columns_0_63": errs, "launches_per_matmat": 3},
            (X_host, cols))


def c4a_members(a):
    """The 48 independent 2DS0-H straight cracks on [-1,1] of the batched
    workload: segment counts log-uniform in [256, 16,384] (seed 3), leaf 32,
    eta 3, eps 1e-5, each built by the reference's host code."""
    from types import SimpleNamespace

    from bigwham_dev_b200.bigwham4py import BigWhamIOGpu
    from bigwham_dev_b200.meshes import straight_crack_2d

    rng = np.random.default_rng(3)
    sizes = np.round(np.exp(rng.uniform(np.log(256), np.log(16384), 48))).astype(int)
    members = []
    for n in sizes:
        coor, conn = straight_crack_2d(int(n))
        io = BigWhamIOGpu(coor, conn, "2DS0-H", PROPS, os.cpu_count() or 1, useCuda=False)
        io.build_hierarchical_matrix(LEAF, ETA, EPS)
        members.append(SimpleNamespace(**io.export_blocks()))
        io.close()
    return sizes, members


def run_batch_only(a):
    """--batch-only: the batched matvec of the 48 x 2DS0-H workload alone (one
    handle, the listed precisions), W warm-ups then K timed steps, with the
    per-launch times; one JSON line.  A short, self-contained command for
    profiling the batched kernels."""
    import torch

    from bigwham_dev_b200 import HmatGpu

    torch.cuda.set_device(0)
    sizes, members = c4a_members(a)
    out = {"workload": f"48 x 2DS0-H straight cracks ({int(sizes.sum()):,} segments), one batched matvec per step"}
    for p in a.precisions:
        hb = HmatGpu.batch(members, device=0, precisions=(p,), tuning=a.tune or None)
        x = torch.from_numpy(np.random.default_rng(0).uniform(-1, 1, hb.n_cols)).cuda()
        y = torch.empty(hb.n_rows, dtype=torch.float64, device="cuda")
        for _ in range(a.warmup):
            hb.matvec(x, p, out=y)
        hb.sync()
        ms = _events_ms(lambda: hb.matvec(x, p, out=y), a.steps)
        hb.set_timing(True)  # the per-launch split, from a second run with events between the launches
        for _ in range(a.steps):
            hb.matvec(x, p, out=y)
        l6, nrec = hb.timing_read_launches()
        hb.set_timing(False)
        b1, b2 = hb.phase_bytes(p)
        l6 = [v / max(1, nrec) for v in l6]
        pe = [l6[0], l6[1] + l6[2], l6[3], l6[4] + l6[5]]
        out[p] = {"ms_per_matvec": ms, "launches": hb.launches(p), "launch_ms": pe, "phase_bytes": [b1, b2],
                  "launch_ms_detail": dict(zip(["x_gather", "p1_cta_wide", "p1_unstaged", "g2_gather",
                                                "p2_cta_wide", "p2_unstaged"], l6)),
                  "phase_gbs": [b1 / (pe[1] * 1e-3) / 1e9, b2 / (pe[3] * 1e-3) / 1e9],
                  "algorithmic_bytes": hb.algorithmic_bytes(p)}
        hb.sync()
        hb.close()
    print(json.dumps(out))
    return 0


def time_penny(a, dev):
    """C3: a pressurised penny-shaped crack, 3DT0-H (radius 1, hexagonal
    lattice of spacing h clipped to the disk, jitter U(+-0.1h) seed 2,
    Delaunay; E = 1, nu = 0.2, leaf 64, eta 3, eps 1e-4), built by the
    reference's host code; one matvec per step in FP64, FP32 and BF16, with
    the reduced precisions' distance from the FP64 GPU matvec."""
    import torch

    from bigwham_dev_b200 import HmatGpu
    from bigwham_dev_b200.bigwham4py import BigWhamIOGpu
    from bigwham_dev_b200.meshes import penny_crack_3d

    t0 = time.time()
    coor, conn = penny_crack_3d(a.c3_h, seed=2)
    io = BigWhamIOGpu(coor, conn, "3DT0-H", [1.0, 0.2], os.cpu_count() or 1, useCuda=False)
    io.build_hierarchical_matrix(64, 3.0, 1e-4)
    ex = io.export_blocks()
    io.close()
    build_s = time.time() - t0
    precs = ("fp64", "fp32", "bf16")
    h = HmatGpu.from_flat(ex["dof"], ex["n_rows"], ex["n_cols"], ex["fr"], ex["lr"], ex["fr_data"], ex["lr_data"],
                          ex["perm0"], ex["perm1"], device=dev.index or 0, precisions=precs)
    del ex
    x = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, h.n_cols)).to(dev)
    out = {"workload": f"3DT0-H penny-shaped crack, h = {a.c3_h} ({len(conn):,} triangles, {h.n_rows:,} DoF), "
                       "E=1 nu=0.2, leaf 64, eta 3, ACA eps 1e-4, x~U(-1,1) seed 1",
           "host_build_s": round(build_s, 1)}
    ys = {}
    steps = max(3, min(a.steps, 50))
    for p in precs:
        y = torch.empty(h.n_rows, dtype=torch.float64, device=dev)
        for _ in range(a.warmup):
            h.matvec(x, p, out=y)
        ms = _events_ms(lambda: h.matvec(x, p, out=y), steps)
        ys[p] = y
        ab = h.algorithmic_bytes(p)
        out[p] = {"ms_per_matvec": ms, "matvec_per_s": 1e3 / ms, "algorithmic_bytes": ab,
                  "gbs": ab / (ms * 1e-3) / 1e9, "launches": h.launches(p)}
    for p in ("fp32", "bf16"):
        out[p]["rel_err_vs_fp64_gpu"] = float(torch.linalg.vector_norm(ys[p] - ys["fp64"]) /
                                              torch.linalg.vector_norm(ys["fp64"]))
    h.close()
    return out


def time_batch(a, dev):
    """48 independent 2DS0-H straight cracks on [-1,1], segment counts
    log-uniform in [256, 16,384] (seed 3), leaf 32, eta 3, eps 1e-5, built by
    the reference's host code: one batched matvec (one launch sequence for all
    48) against 48 separate handles (a launch sequence each)."""
    import torch

    from bigwham_dev_b200 import HmatGpu

    t0 = time.time()
    sizes, members = c4a_members(a)
    build_s = time.time() - t0
    precs = ("fp64", "bf16")
    hb = HmatGpu.batch(members, device=dev.index or 0, precisions=precs, tuning=a.tune or None)
    hs = [HmatGpu.from_flat(m.dof, m.n_rows, m.n_cols, m.fr, m.lr, m.fr_data, m.lr_data, m.perm0, m.perm1,
                            device=dev.index or 0, precisions=precs, tuning=a.tune or None) for m in members]
    x = torch.from_numpy(np.random.default_rng(0).uniform(-1, 1, hb.n_cols)).to(dev)
    y = torch.empty(hb.n_rows, dtype=torch.float64, device=dev)
    xs = [x[int(hb.col_offsets[k]):int(hb.col_offsets[k + 1])].contiguous() for k in range(len(hs))]
    ys = [torch.empty(hs[k].n_rows, dtype=torch.float64, device=dev) for k in range(len(hs))]
    out = {"workload": "48 x 2DS0-H straight cracks, segments log-uniform in [256, 16384] seed 3 "
                       f"({int(sizes.sum()):,} segments, {hb.n_rows:,} DoF in total), x~U(-1,1) seed 0",
           "host_build_s": round(build_s, 2)}
    steps = max(3, min(a.steps, 50))
    for p in precs:
        for _ in range(a.warmup):
            hb.matvec(x, p, out=y)
            for k in range(len(hs)):
                hs[k].matvec(xs[k], p, out=ys[k])
        ms_b = _events_ms(lambda: hb.matvec(x, p, out=y), steps)

        def separate():
            for k in range(len(hs)):
                hs[k].matvec(xs[k], p, out=ys[k])

        ms_s = _events_ms(separate, steps)
        yb = y.clone()
        separate()
        diff = max(float(torch.linalg.vector_norm(yb[int(hb.row_offsets[k]):int(hb.row_offsets[k + 1])] - ys[k]) /
                         torch.linalg.vector_norm(ys[k])) for k in range(len(hs)))
        out[p] = {"ms_per_batched_matvec": ms_b, "batches_per_s": 1e3 / ms_b, "ms_48_separate_handles": ms_s,
                  "speedup_batched_vs_separate": ms_s / ms_b, "algorithmic_bytes": hb.algorithmic_bytes(p),
                  "batched_gbs": hb.algorithmic_bytes(p) / (ms_b * 1e-3) / 1e9,
                  "max_member_rel_diff_batched_vs_separate": diff, "launches": {"batched": hb.launches(p), "separate": sum(hk.launches(p) for hk in hs)}}
    hb.close()
    for h in hs:
        h.close()
    return out


def cpu_baseline(a, x_host, y_fp64):
    """The reference's own OpenMP CPU matvec (oracle/_ref) on the same
    H-matrix definition and x, on this host's cores; bounded sample.  Returns
    (report, FP64 parity, the reference object for the checks that follow)."""
    try:
        from oracle import RefHmat, ref_available
    except Exception as e:
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}, None, None
    if not ref_available():
        return ({"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                 "sample": "unavailable: oracle/_ref not built"}, None, None)
    from bigwham_dev_b200.meshes import square_crack_3d

    threads = os.cpu_count() or 1
    coor, conn = square_crack_3d(a.mesh)
    t0 = time.time()
    R = RefHmat("3DR0-H", coor, conn, PROPS, LEAF, ETA, EPS, n_threads=threads)
    build_s = time.time() - t0
    y_ref = R.matvec(x_host)
    t0 = time.perf_counter()
    R.matvec(x_host)
    est = time.perf_counter() - t0
    k = max(2, min(50, int(a.cpu_budget_s / max(est, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(k):
        R.matvec(x_host)
    dt = time.perf_counter() - t0
    parity = float(np.linalg.norm(y_fp64 - y_ref) / np.linalg.norm(y_ref)) if y_fp64 is not None else None
    return ({"value": k / dt, "unit": UNIT, "cores": threads, "kind": "reference",
             "sample": f"{k} full BigWhamIO::MatVec calls on the same {3 * a.mesh * a.mesh:,}-DoF H-matrix "
                       f"(reference build {build_s:.1f} s, untimed), {threads} OpenMP threads, 1 BLAS thread"},
            parity, R)


def device_build(a, h, x_host, host_build_s):
    """The same H-matrix built on the device (devbuild.build_r0: the host
    builds the cluster tree and pattern, bw_r0_assemble_fr the full-rank
    blocks, bw_r0_aca the low-rank ones) and laid out on the device
    (bw_add_flat_device), against the host build of the reference's code:
    wall times and the FP64 matvecs' relative difference (ACA pivots differ
    in the last bits, ranks may differ by a block)."""
    import torch

    from bigwham_dev_b200 import HmatGpu
    from bigwham_dev_b200.bigwham4py import BigWhamIOGpu
    from bigwham_dev_b200.devbuild import build_r0, ex_args
    from bigwham_dev_b200.meshes import square_crack_3d

    coor, conn = square_crack_3d(a.mesh)
    io = BigWhamIOGpu(coor, conn, "3DR0-H", PROPS, os.cpu_count() or 1, useCuda=False)
    torch.cuda.synchronize()
    t0 = time.time()
    ex = build_r0(io, LEAF, ETA, EPS, PROPS[0], PROPS[1], on_device=True)
    torch.cuda.synchronize()
    t_build = time.time() - t0
    io.close()
    t0 = time.time()
    hd = HmatGpu.from_device_flat(**ex_args(ex), device=torch.cuda.current_device(), precisions=("fp64",))
    torch.cuda.synchronize()
    t_layout = time.time() - t0
    entries = int(ex["fr_data"].numel() + ex["lr_data"].numel())
    del ex
    x = torch.from_numpy(x_host).cuda()
    yd, yh = hd.matvec(x, "fp64"), h.matvec(x, "fp64")
    diff = float(torch.linalg.vector_norm(yd - yh) / torch.linalg.vector_norm(yh))
    hd.close()
    return {"workload": f"3DR0-H {a.mesh}x{a.mesh}: blocks computed on the device from the reference's pattern",
            "device_build_s": round(t_build, 3), "device_layout_s": round(t_layout, 3),
            "host_build_s": host_build_s, "entries_device_vs_host": [entries, h.info()["entries"]],
            "fp64_matvec_rel_diff_vs_host_build": diff}


def northstar_checks(a, h, R, x_host, mm_cols):
    """Accuracy of the target configuration against the FP64 dense oracle of
    the same kernel on a sampled row subset (683 collocation points = 2,049
    rows, numpy default_rng(7); the reference's own influence() per entry),
    outside every timed region:
    * every storage precision's matvec on those rows;
    * FP64 Jacobi GMRES(50) to 1e-8 and FP64-refined GMRES with FP32 / BF16
      inner solves to 1e-8 for a uniform unit normal traction: iterations,
      residuals, the solution's residual on the dense rows, its difference
      from the FP64 solution, wall time;
    * the 64-right-hand-side matmat's columns 0 and 63 against the
      reference's own FP64 matvec of the same columns."""
    import torch

    from bigwham_dev_b200.solve import Gmres, refine

    out = {"workload": "uniform unit normal traction; dense rows: 683 collocation points (2,049 rows) x all columns"}
    npts = h.n_rows // 3
    sample = np.sort(np.random.default_rng(7).choice(npts, size=min(683, npts), replace=False))
    t0 = time.time()
    D = R.dense_rows("3DR0-H", PROPS, sample)
    out["dense_rows_s"] = round(time.time() - t0, 2)
    rows = (3 * sample[:, None] + np.arange(3)[None, :]).ravel()

    def rel(u, v):
        return float(np.linalg.norm(u - v) / np.linalg.norm(v))

    yd = D @ x_host
    out["matvec_rel_err_vs_dense_rows"] = {p: rel(h.matvec(x_host, p)[rows], yd) for p in a.precisions}
    if "fp64" not in a.precisions:
        return out
    dev = torch.device("cuda", torch.cuda.current_device())
    b_np = np.zeros(h.n_rows)
    b_np[2::3] = 1.0
    b = torch.from_numpy(b_np).to(dev)
    minv = torch.from_numpy(1.0 / h.diagonal()).to(dev)
    ops = {p: (lambda x, y, p=p: h.matvec(x, p, out=y)) for p in a.precisions}
    r = torch.empty_like(b)

    def true_res(x):
        ops["fp64"](x, r)
        return float(torch.linalg.vector_norm(b - r) / torch.linalg.vector_norm(b))

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    x64, info = Gmres(ops["fp64"], h.n_rows, restart=50, minv=minv).solve(b, tol=1e-8, maxiter=5000)
    torch.cuda.synchronize()
    X64 = x64.cpu().numpy()
    out["fp64_gmres"] = {"converged": info.converged, "arnoldi_steps": info.iterations,
                         "s": round(time.perf_counter() - t0, 3), "rel_residual": true_res(x64),
                         "dense_row_residual": rel(D @ X64, b_np[rows])}
    out["refined"] = {}
    for p in (q for q in ("fp32", "bf16") if q in a.precisions):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        xr, inf = refine(ops["fp64"], ops[p], b, h.n_rows, minv=minv, tol=1e-8, inner_tol=1e-3, restart=50)
        torch.cuda.synchronize()
        Xr = xr.cpu().numpy()
        out["refined"][p] = {"converged": inf.converged, "outer_steps": inf.outer, "inner_arnoldi_steps": inf.iterations,
                             "s": round(time.perf_counter() - t0, 3), "rel_residual": true_res(xr),
                             "rel_err_vs_fp64_solution": rel(Xr, X64),
                             "dense_row_residual": rel(D @ Xr, b_np[rows])}
    if mm_cols is not None:
        X, cols = mm_cols
        out["matmat_columns_vs_reference_matvec"] = [rel(cols[:, q], R.matvec(np.ascontiguousarray(X[:, j])))
                                                     for q, j in enumerate((0, X.shape[1] - 1))]
    return out


def run_ours(a):
    import torch

    world, rank, local = dist_setup(a.gpus)
    torch.cuda.set_device(local)
    if world > 1:  # the matmat and batch lines run on one GPU only
        a.matmat, a.no_batch, a.c3_h = False, True, 0.0
    io, h, setup = build_hmatrix(a, world, rank, local)
    dev = torch.device("cuda", local)
    n_in, n_out = h.n_cols, h.n_rows
    x_host = np.random.default_rng(1).uniform(-1.0, 1.0, n_in)
    x = torch.from_numpy(x_host).to(dev)
    ys = {p: torch.empty(n_out, dtype=torch.float64, device=dev) for p in a.precisions}
    stream = torch.cuda.current_stream(dev)
    peak, peak_kind = read_peak()
    clocks = ClockSampler(local)
    res = {}
    clocks.start()
    # the headline precision first, then the others
    for p in sorted(a.precisions, key=lambda q: q != HEAD):
        y = ys[p]
        for _ in range(a.warmup):
            h.matvec(x, p, out=y)
        h.sync(stream)
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clocks.window()
        e0.record(stream)
        for _ in range(a.steps):
            h.matvec(x, p, out=y)
        e1.record(stream)
        torch.cuda.synchronize()
        clocks.end()
        ms_total = e0.elapsed_time(e1)
        # the per-launch split, from a second run with events between the launches
        h.set_timing(True)
        for _ in range(a.steps):
            h.matvec(x, p, out=y)
        launch_ms, nrec = h.timing_read()
        h.set_timing(False)
        h.sync(stream)
        ms_total = max_over_ranks(ms_total, world)
        b1, b2 = h.phase_bytes(p)
        t_stream = (launch_ms[1] + launch_ms[3]) / max(1, nrec)  # ms per step in the streaming kernel
        res[p] = {"ms_per_step": ms_total / a.steps, "value": world * a.steps / (ms_total / 1e3),
                  "launches_per_step": h.launches(p),
                  "algorithmic_bytes": h.algorithmic_bytes(p), "phase_bytes": [b1, b2],
                  "launch_ms_per_step": [v / max(1, nrec) for v in launch_ms],
                  "stream_kernel_gbs": (b1 + b2) / (t_stream * 1e-3) / 1e9,
                  "matvec_gbs": h.algorithmic_bytes(p) / (ms_total / a.steps * 1e-3) / 1e9}
    # end to end through the reference-facing call with host buffers, every precision
    e2e_steps = max(1, min(a.steps, 200))
    y_e2e = {}
    for p in sorted(a.precisions, key=lambda q: q != HEAD):
        if io is not None:
            io.set_precision(p)
            call = lambda: io.matvec(x_host)  # noqa: E731  BigWhamIO::MatVec -> HmatGpu -> bw_matvec_host
            path = "BigWhamIO::MatVec(host arrays) -> HmatGpu::matvecOriginal -> bw_matvec_host"
        else:
            call = lambda p=p: h.matvec(x_host, p)  # noqa: E731  bw_matvec_host
            path = "bw_matvec_host (host arrays)"
        for _ in range(min(3, a.warmup)):
            call()
        torch.cuda.synchronize()
        barrier(world)
        clocks.window()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            y_e2e[p] = call()
        dt = time.perf_counter() - t0
        clocks.end()
        dt = max_over_ranks(dt, world)
        res[p]["e2e"] = {"value": world * e2e_steps / dt, "unit": UNIT, "ms_per_call": 1e3 * dt / e2e_steps,
                         "h2d_bytes_per_step": 8 * n_in, "d2h_bytes_per_step": 8 * n_out, "path": path,
                         "timer": "host wall clock, synchronous calls"}
    clk = clocks.stop()
    yref = ys["fp64" if "fp64" in ys else HEAD].cpu().numpy()
    y64 = yref if "fp64" in ys else None
    errs = {p: float(np.linalg.norm(ys[p].cpu().numpy() - yref) / np.linalg.norm(yref)) for p in ys if p != "fp64"}
    for p in y_e2e:
        errs[f"e2e_{p}_vs_device_{p}"] = float(np.linalg.norm(y_e2e[p] - ys[p].cpu().numpy()) / np.linalg.norm(yref))
    extra, mm_cols = {}, None
    if world == 1 and a.matmat:
        extra["matmat_64rhs"], mm_cols = time_matmat(a, h, dev, peak, res["bf16"]["ms_per_step"])
    if world == 1 and not a.no_batch:
        extra["batched_2ds0_48"] = time_batch(a, dev)
    if world == 1 and a.c3_h > 0:
        extra["penny_3dt0"] = time_penny(a, dev)
    if world == 1 and not a.no_devbuild:
        extra["device_build_3dr0"] = device_build(a, h, x_host, setup.get("host_build_s"))
    if rank != 0:
        return 0
    cpu, parity = (None, None)
    if world == 1 and not a.no_cpu_baseline:
        cpu, parity, R = cpu_baseline(a, x_host, y64)
        if R is not None and not a.no_checks:
            extra["northstar_checks"] = northstar_checks(a, h, R, x_host, mm_cols)
        del R
    if io is not None:
        io.close()
    head = res[HEAD]
    b1, b2 = head["phase_bytes"]
    t_stream = head["launch_ms_per_step"][1] + head["launch_ms_per_step"][3]
    achieved = (b1 + b2) / (t_stream * 1e-3) / 1e9
    tkey = {"fp64": "stream_panels_fp64", "fp32": "stream_panels_fp32", "bf16": "stream_panels_bf16"}[HEAD]
    kname = {"fp64": "double", "fp32": "float", "bf16": "Bf16"}[HEAD]
    out = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"fp64": "f64", "fp32": "f32", "bf16": "bf16"}[HEAD],
        "data": "synthetic mesh (generated; no dataset), x ~ U(-1,1) seed 1",
        "config": workload(a.mesh),
        "setup": {"parallelism": f"replicas x{world}" if world > 1 else "single GPU", **setup},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                     else "fallback 6650 GB/s",
                     "kernel": f"stream_panels_kernel<{kname}> (phase 1 + phase 2 launches of one step)",
                     "bytes_per_step": b1 + b2, "traffic": read_traffic(tkey)},
        "cpu_baseline": cpu,
        "e2e": {k: v for k, v in head["e2e"].items() if k != "ms_per_call"},
        "gpu_launches": head["launches_per_step"] * a.steps,
        "launches_per_step": head["launches_per_step"],
        "clocks": clk,
        "precisions": {p: {k: v for k, v in res[p].items()} for p in res},
        "speedup_fp32_vs_fp64": res["fp32"]["value"] / res["fp64"]["value"] if {"fp32", "fp64"} <= set(res) else None,
        "speedup_bf16_vs_fp64": res["bf16"]["value"] / res["fp64"]["value"] if {"bf16", "fp64"} <= set(res) else None,
        "rel_err_vs_fp64_gpu": errs,
        "fp64_gpu_vs_reference_rel_err": parity,
        **extra,
    }
    print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--mesh", type=int, default=256, help="rectangles per side (256 -> 196,608 DoF)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precisions", default="fp64,fp32,bf16",
                    help="storage precisions to upload and time (comma list; must include fp32, the headline, "
                         "and bf16)")
    ap.add_argument("--no-matmat", dest="matmat", action="store_false",
                    help="skip the 64-right-hand-side tensor-core matmat line (N = 1 only)")
    ap.add_argument("--no-batch", action="store_true", help="skip the 48 x 2DS0 batched line (N = 1 only)")
    ap.add_argument("--c3-h", type=float, default=0.0128,
                    help="mesh spacing of the 3DT0-H penny line (0.0128: 132,690 DoF; 0.0064: 531,111 DoF; "
                         "0 skips it; N = 1 only)")
    ap.add_argument("--tune", action="append", default=[], metavar="KEY=VALUE",
                    help="plan parameter (bw_set_tuning) for every handle of the run, e.g. narrow_rows=0; repeatable")
    ap.add_argument("--no-devbuild", action="store_true",
                    help="skip the device build of the same H-matrix (N = 1 only)")
    ap.add_argument("--batch-only", action="store_true",
                    help="time only the 48 x 2DS0 batched matvec in the listed precisions (one GPU)")
    ap.add_argument("--block-file", default=None,
                    help="block file of the H-matrix: read it when it exists (no host rebuild), else write it "
                         "after the build")
    ap.add_argument("--no-checks", action="store_true",
                    help="skip the accuracy checks against the dense rows (refined GMRES, N = 1 only)")
    ap.add_argument("--cpu-budget-s", type=float, default=10.0)
    ap.add_argument("--ref-budget-s", type=float, default=60.0)
    a = ap.parse_args(argv)
    if a.warmup < 3:
        ap.error("--warmup must be >= 3")
    a.precisions = [p for p in a.precisions.split(",") if p]
    try:
        a.tune = {k: int(v) for k, v in (t.split("=", 1) for t in a.tune)}
    except ValueError:
        ap.error("--tune takes KEY=INTEGER")
    if not set(a.precisions) <= {"fp64", "fp32", "bf16"}:
        ap.error("--precisions must be a subset of fp64,fp32,bf16")
    if a.batch_only:
        return run_batch_only(a)
    if not {HEAD, "bf16"} <= set(a.precisions):
        ap.error("--precisions must include fp32 (the headline) and bf16")
    if a.impl == "reference":
        return run_reference(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
