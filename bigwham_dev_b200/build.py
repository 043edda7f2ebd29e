"""Build the in-tree shared libraries of the package.

    python -m bigwham_dev_b200.build          # CUDA backend only
    python -m bigwham_dev_b200.build --host   # + the BigWham host adapter (needs the reference sources)

* ``_lib/libbigwham_b200.so``: the CUDA kernels and the C ABI
  (include/bigwham_b200.h), compiled for sm_100a only.
* ``_lib/libbigwham_host.so``: the reference's unmodified host code (mesh,
  kernels, cluster tree, ACA) plus the ``HmatGpu`` adapter that installs the
  CUDA backend behind ``BigWhamIO`` (host/Makefile; needs the reference tree
  at build time only).
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIBDIR = os.path.join(HERE, "_lib")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CUDA_SOURCES = ["csrc/bw_capi.cu", "csrc/bw_layout.cpp", "csrc/bw_file.cpp"]
CUDA_DEPS = CUDA_SOURCES + ["csrc/bw_kernels.cuh", "csrc/bw_mm_kernels.cuh", "csrc/bw_layout.h", "csrc/bw_file.h", "csrc/bw_r0.h", "csrc/bw_assemble_kernels.cuh", "csrc/bw_aca.h", "csrc/bw_aca_kernels.cuh", "csrc/bw_pack.h", "csrc/bw_devlayout_kernels.cuh", "csrc/bw_s0.h", "csrc/bw_r0_fields.h", "csrc/bw_fields_kernels.cuh", "../include/bigwham_b200.h"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(os.path.join(HERE, d)) > t for d in deps)


def build_cuda(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    out = os.path.join(LIBDIR, "libbigwham_b200.so")
    if not force and not _newer(out, CUDA_DEPS):
        return out
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-ccbin", "g++", "-Xcompiler", "-fPIC,-fopenmp",
           "-shared", f"-I{os.path.join(ROOT, 'include')}", *[os.path.join(HERE, s) for s in CUDA_SOURCES],
           "-o", out, "-lgomp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return out


def reference_tree() -> str | None:
    """The BigWham source tree the host adapter and the oracle compile from:
    $BIGWHAM_REF when set, else a ``reference`` directory beside the
    repository; None when neither holds the reference sources."""
    cands = [os.environ["BIGWHAM_REF"]] if os.environ.get("BIGWHAM_REF") else []
    cands.append(os.path.join(os.path.dirname(ROOT), "reference"))
    for c in cands:
        if os.path.isdir(os.path.join(c, "src", "hmat")):
            return os.path.abspath(c)
    return None


def build_host(force: bool = False) -> str | None:
    """Builds the host adapter when the reference tree is present; returns the
    library path (None when the reference tree is absent and no prebuilt
    library exists)."""
    out = os.path.join(LIBDIR, "libbigwham_host.so")
    ref = reference_tree()
    if ref is None:
        return out if os.path.exists(out) else None
    args = ["make", "-C", os.path.join(HERE, "host"), f"REF={ref}", "-j", str(os.cpu_count() or 8)]
    if force:
        args.insert(1, "-B")
    subprocess.run(args, check=True)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--host", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build_cuda(a.force, a.verbose))
    if a.host:
        print(build_host(a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
