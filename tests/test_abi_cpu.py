"""The C ABI on CPU: each library loads and exports every function its header
declares, and the ctypes bindings cover them with the declared arity.

include/bigwham_b200.h -> bigwham_dev_b200/_lib/libbigwham_b200.so
include/bigwham_host.h -> bigwham_dev_b200/_lib/libbigwham_host.so
No function is called, so no GPU is needed.
"""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBS = {"bigwham_b200.h": "libbigwham_b200.so", "bigwham_host.h": "libbigwham_host.so"}


def declared(header):
    """{name: number of parameters} of the functions a header declares."""
    with open(os.path.join(ROOT, "include", header)) as f:
        src = f.read()
    src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
    src = re.sub(r"//[^\n]*", " ", src)
    src = re.sub(r"#[^\n]*", " ", src)
    out = {}
    for m in re.finditer(r"\b(bwh?_\w+)\s*\(([^()]*)\)\s*;", src):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


@pytest.mark.parametrize("header", sorted(LIBS))
def test_library_exports_every_declared_function(header):
    path = os.path.join(ROOT, "bigwham_dev_b200", "_lib", LIBS[header])
    if not os.path.exists(path):
        pytest.skip(f"{LIBS[header]} not built")
    names = declared(header)
    assert len(names) > 10
    lib = C.CDLL(path)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"{LIBS[header]} lacks {missing}"


def test_backend_bindings_match_the_header():
    from bigwham_dev_b200 import _capi as A

    names = declared("bigwham_b200.h")
    assert set(A._SIGS) <= set(names), sorted(set(A._SIGS) - set(names))
    for n, (_, args) in A._SIGS.items():
        assert len(args) == names[n], f"{n}: {len(args)} ctypes arguments, header declares {names[n]}"
    assert sorted(set(names) - set(A._SIGS)) == [], "every backend entry has a ctypes binding"
    lib = A.lib()
    for n in A._SIGS:
        assert hasattr(lib, n)


def test_host_bindings_match_the_header():
    from bigwham_dev_b200 import bigwham4py as B

    names = declared("bigwham_host.h")
    sigs = B._HSIGS
    assert set(sigs) == set(names), sorted(set(sigs) ^ set(names))
    for n, (_, args) in sigs.items():
        assert len(args) == names[n], f"{n}: {len(args)} ctypes arguments, header declares {names[n]}"


def test_every_backend_header_is_a_build_dependency():
    """build_cuda rebuilds when any header under csrc/ changes: each one is
    listed among its dependencies."""
    import glob

    from bigwham_dev_b200 import build as B

    here = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bigwham_dev_b200")
    headers = {os.path.relpath(p, here) for p in glob.glob(os.path.join(here, "csrc", "*.h")) +
               glob.glob(os.path.join(here, "csrc", "*.cuh"))}
    assert headers <= set(B.CUDA_DEPS), sorted(headers - set(B.CUDA_DEPS))
