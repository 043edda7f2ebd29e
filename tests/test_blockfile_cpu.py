"""Block files on CPU (bw_file_* / bwh_write_to_file / bw_create_from_file).

A block file holds what the reference's Hmat::writeToFile stores
(src/hmat/hmatrix/hmat.cc:749-835).  Checked here:
* round trips are bitwise, through the flat writer (bwh_export's form) and
  through the host writer (the CPU Hmat's own blocks, HPattern spots and ACA
  error estimates);
* a handle built from the file plans the same operator as one built from
  the flat arrays: the replayed matvecs agree bitwise and match the oracle;
* padded leading dimensions, sections spanning several checksum blocks, and
  empty patterns;
* corrupt, truncated, foreign and missing files, and inconsistent arguments,
  are rejected with BW_ERR_IO / BW_ERR_ARG, and a failed write leaves no file;
* the header checksum follows the documented algorithm (a Python restatement);
* the C++ API (write_block_file, HmatGpu(filename)) restores the Hmat state
  and BigWhamIO's queries bitwise (tests/cpp/hmat_file_check.cc, built from
  the reference sources when they are present).
"""
import ctypes as C
import os
import struct
import subprocess

import numpy as np
import pytest

from planreplay import replay

from bigwham_dev_b200.build import reference_tree

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST_LIB = os.path.join(ROOT, "bigwham_dev_b200", "_lib", "libbigwham_host.so")
needs_host = pytest.mark.skipif(not os.path.exists(HOST_LIB), reason="host adapter not built")

FLAT = ("fr", "lr", "fr_data", "lr_data", "perm0", "perm1")


@pytest.fixture(scope="module")
def crack(tmp_path_factory):
    """3DR0-H 12 x 12 square crack built by the reference's host code, its
    flat export, and a block file written by the host writer."""
    if not os.path.exists(HOST_LIB):
        pytest.skip("host adapter not built")
    from bigwham_dev_b200.bigwham4py import BigWhamIOGpu
    from bigwham_dev_b200.meshes import square_crack_3d

    coor, conn = square_crack_3d(12)
    io = BigWhamIOGpu(coor, conn, "3DR0-H", [1.0, 0.25], 2, useCuda=False)
    io.build_hierarchical_matrix(32, 3.0, 1e-5)
    ex = io.export_blocks()
    path = tmp_path_factory.mktemp("bf") / "host.bwb"
    io.write_to_file(path)
    nblk = io.n_blocks()
    io.close()
    return ex, str(path), nblk


REF = reference_tree() or ""


@needs_host
@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src")), reason="reference sources not present")
def test_cpp_file_constructor_restores_the_hmat(tmp_path):
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "bigwham_dev_b200", "host"), f"REF={REF}", "check"],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    r = subprocess.run([os.path.join(ROOT, "_build", "hmat_file_check"), str(tmp_path / "c.bwb")],
                       capture_output=True, text=True, timeout=300)
    lines = r.stdout.strip().splitlines()
    assert r.returncode == 0 and lines and lines[-1].startswith("ok "), r.stdout + r.stderr


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@needs_host
def test_flat_round_trip_is_bitwise(crack, tmp_path):
    from bigwham_dev_b200 import blockfile

    ex, _, _ = crack
    err = np.linspace(1e-7, 2e-6, ex["lr"].shape[0])
    p = tmp_path / "flat.bwb"
    blockfile.write(p, ex, lr_error=err)
    h = blockfile.info(p)
    assert (h["dof"], h["n_rows"], h["n_cols"]) == (ex["dof"], ex["n_rows"], ex["n_cols"])
    assert (h["n_fr"], h["n_lr"]) == (ex["fr"].shape[0], ex["lr"].shape[0])
    assert (h["fr_entries"], h["lr_entries"]) == (ex["fr_data"].size, ex["lr_data"].size)
    assert h["has_lr_error"] == 1 and h["file_bytes"] == os.path.getsize(p)
    r = blockfile.read(p, patterns=True)
    for k in FLAT:
        assert r[k].dtype == ex[k].dtype and np.array_equal(r[k], ex[k]), k
    assert np.array_equal(r["lr_error"], err)
    # flat writer: spot = block index, FR flag 0, LR flag = rank
    assert np.array_equal(r["fr_pattern"][:, 0], np.arange(h["n_fr"]))
    assert np.array_equal(r["fr_pattern"][:, 5], np.zeros(h["n_fr"]))
    assert np.array_equal(r["lr_pattern"][:, 1:], ex["lr"])


@needs_host
def test_host_writer_matches_the_export(crack):
    from bigwham_dev_b200 import blockfile

    ex, path, (nfr, nlr) = crack
    r = blockfile.read(path, patterns=True)
    for k in FLAT:
        assert np.array_equal(r[k], ex[k]), k
    assert r["fr_pattern"].shape == (nfr, 6) and r["lr_pattern"].shape == (nlr, 6)
    # HPattern spots are tree node indices (h_pattern.cc), not block numbers
    assert len(np.unique(np.concatenate([r["fr_pattern"][:, 0], r["lr_pattern"][:, 0]]))) == nfr + nlr
    # ACA error estimates of LowRank::error_on_approximation: small, positive
    e = r["lr_error"]
    assert blockfile.info(path)["has_lr_error"] == 1
    assert np.all(e >= 0) and e.max() > 0 and e.max() < 1e-2


@needs_host
@pytest.mark.parametrize("precision", ["fp64", "fp32", "bf16"])
def test_handle_from_file_plans_the_same_operator(crack, precision):
    from bigwham_dev_b200 import HmatGpu
    from oracle import HmatArrays, oracle_matvec_perm

    ex, path, _ = crack
    kw = dict(device=-1, plan_only=True, precisions=(precision,), transpose=True)
    h_flat = HmatGpu.from_flat(ex["dof"], ex["n_rows"], ex["n_cols"], ex["fr"], ex["lr"], ex["fr_data"],
                               ex["lr_data"], ex["perm0"], ex["perm1"], **kw)
    h_file = HmatGpu.from_file(path, **kw)
    assert (h_file.dof, h_file.n_rows, h_file.n_cols) == (ex["dof"], ex["n_rows"], ex["n_cols"])
    x = np.random.default_rng(7).uniform(-1, 1, ex["n_cols"])
    for tr in (False, True):
        assert np.array_equal(replay(h_file, x, precision, tr), replay(h_flat, x, precision, tr))
    assert np.array_equal(h_file.diagonal(), h_flat.diagonal())
    if precision == "fp64":
        arr = HmatArrays(ex["dof"], ex["n_rows"], ex["n_cols"], ex["fr"], ex["lr"], ex["fr_data"], ex["lr_data"],
                         ex["perm0"], ex["perm1"])
        assert _rel(replay(h_file, x, "fp64"), oracle_matvec_perm(arr, x, 1)) < 1e-14
    h_flat.close()
    h_file.close()


def _write_blocks(path, dof, n_rows, n_cols, p0, p1, fr_pat, fr_blocks, lr_pat, lr_a, lr_b, err=None):
    """bw_file_write_blocks with per-block pointers and leading dimensions
    (arrays are Fortran-ordered views, possibly of taller buffers)."""
    from bigwham_dev_b200 import _capi as A

    def ptrs(blocks):
        return ((C.c_void_p * max(1, len(blocks)))(*[b.ctypes.data for b in blocks]),
                np.array([b.strides[1] // 8 for b in blocks] or [0], dtype=np.int64))

    fp, fl = ptrs(fr_blocks)
    ap, al = ptrs(lr_a)
    bp, bl = ptrs(lr_b)
    fr_pat = np.ascontiguousarray(fr_pat, dtype=np.int64).reshape(-1, 6)
    lr_pat = np.ascontiguousarray(lr_pat, dtype=np.int64).reshape(-1, 6)
    return A.lib().bw_file_write_blocks(os.fsencode(str(path)), dof, n_rows, n_cols, p0.ctypes.data, p1.ctypes.data,
                                        fr_pat.shape[0], fr_pat.ctypes.data, fp, fl.ctypes.data, lr_pat.shape[0],
                                        lr_pat.ctypes.data, ap, al.ctypes.data, bp, bl.ctypes.data,
                                        None if err is None else err.ctypes.data)


def test_padded_blocks_and_multi_block_checksums(tmp_path):
    """A 1,100 x 1,100 FR block stored with leading dimension 1,107 (9.7 MB:
    10 checksum blocks) and a rank-7 LR block whose factors are padded too."""
    from bigwham_dev_b200 import blockfile

    rng = np.random.default_rng(3)
    n = 1100
    p = np.arange(n + 300, dtype=np.int64)[::-1].copy()
    big = np.asfortranarray(rng.standard_normal((n + 7, n)))[:n, :]
    a_buf = np.asfortranarray(rng.standard_normal((300 + 5, 7)))
    b_buf = np.asfortranarray(rng.standard_normal((7 + 2, n)))
    fr_pat = [[5, 0, 0, n, n, 0]]
    lr_pat = [[9, n, 0, n + 300, n, 7]]
    err = np.array([3.5e-6])
    path = tmp_path / "pad.bwb"
    assert _write_blocks(path, 1, n + 300, n + 300, p, p, fr_pat, [big], lr_pat, [a_buf[:300]], [b_buf[:7]],
                         err) == 0
    r = blockfile.read(path, patterns=True)
    assert np.array_equal(r["fr_data"], big.ravel(order="F"))
    assert np.array_equal(r["lr_data"], np.concatenate([a_buf[:300].ravel(order="F"), b_buf[:7].ravel(order="F")]))
    assert np.array_equal(r["fr_pattern"], np.array(fr_pat)) and np.array_equal(r["lr_pattern"], np.array(lr_pat))
    assert np.array_equal(r["lr_error"], err)
    assert np.array_equal(r["perm0"], p) and np.array_equal(r["perm1"], p)


def test_empty_pattern_round_trip(tmp_path):
    from bigwham_dev_b200 import blockfile

    ex = {"dof": 2, "n_rows": 6, "n_cols": 4, "fr": np.zeros((0, 4)), "lr": np.zeros((0, 5)),
          "fr_data": np.zeros(0), "lr_data": np.zeros(0), "perm0": [2, 0, 1], "perm1": [1, 0]}
    blockfile.write(tmp_path / "e.bwb", ex)
    r = blockfile.read(tmp_path / "e.bwb")
    assert r["fr"].shape == (0, 4) and r["lr"].shape == (0, 5) and r["fr_data"].size == 0
    assert list(r["perm0"]) == [2, 0, 1] and list(r["perm1"]) == [1, 0]
    assert blockfile.info(tmp_path / "e.bwb")["has_lr_error"] == 0


def _small(tmp_path, name="s.bwb"):
    """Two 4 x 4 FR blocks (dof 1) and a rank-1 LR block: a valid small file."""
    from bigwham_dev_b200 import blockfile

    rng = np.random.default_rng(11)
    ex = {"dof": 1, "n_rows": 8, "n_cols": 8, "fr": np.array([[0, 0, 4, 4], [4, 4, 8, 8]]),
          "lr": np.array([[0, 4, 4, 8, 1]]), "fr_data": rng.standard_normal(32), "lr_data": rng.standard_normal(8),
          "perm0": np.arange(8)[::-1], "perm1": np.arange(8)}
    path = tmp_path / name
    blockfile.write(path, ex)
    return ex, path


def _status(fn):
    from bigwham_dev_b200 import _capi as A

    with pytest.raises(A.BigWhamError) as e:
        fn()
    return e.value.status, str(e.value)


def _flip(path, offset):
    b = bytearray(open(path, "rb").read())
    b[offset] ^= 0x40
    open(path, "wb").write(bytes(b))


def _section(path, s):
    """(offset, bytes) of section s from the raw header."""
    raw = open(path, "rb").read(256)
    off, nbytes, _ = struct.unpack_from("<qqQ", raw, 80 + 24 * s)
    return off, nbytes


def test_corruption_is_detected(tmp_path):
    from bigwham_dev_b200 import _capi as A
    from bigwham_dev_b200 import blockfile

    ex, path = _small(tmp_path)
    off, _ = _section(path, 5)  # fr_data
    _flip(path, off + 8 * 3)
    st, msg = _status(lambda: blockfile.read(path, verify=True))
    assert st == A.BW_ERR_IO and "checksum mismatch in section fr_data" in msg
    st, msg = _status(lambda: A.check(A.lib().bw_create_from_file(os.fsencode(str(path)), -1, 1,
                                                                   C.byref(C.c_void_p())), None))
    assert st == A.BW_ERR_IO and "fr_data" in msg
    r = blockfile.read(path, verify=False)  # the data checksums are skipped on request
    assert np.count_nonzero(r["fr_data"] != ex["fr_data"]) == 1
    # pattern and permutations are checked always
    _, path2 = _small(tmp_path, "p.bwb")
    off, _ = _section(path2, 2)
    _flip(path2, off + 8 * 3)
    st, msg = _status(lambda: blockfile.read(path2, verify=False))
    assert st == A.BW_ERR_IO and "fr_pattern" in msg
    # header
    _, path3 = _small(tmp_path, "h.bwb")
    _flip(path3, 20)
    st, msg = _status(lambda: blockfile.info(path3))
    assert st == A.BW_ERR_IO and "header checksum" in msg


def test_truncated_foreign_and_missing_files(tmp_path):
    from bigwham_dev_b200 import _capi as A
    from bigwham_dev_b200 import blockfile

    _, path = _small(tmp_path)
    raw = open(path, "rb").read()
    (tmp_path / "t.bwb").write_bytes(raw[:-8])
    st, msg = _status(lambda: blockfile.info(tmp_path / "t.bwb"))
    assert st == A.BW_ERR_IO and "truncated" in msg
    (tmp_path / "x.bwb").write_bytes(b"\x89HDF\r\n\x1a\n" + raw[8:])
    st, msg = _status(lambda: blockfile.info(tmp_path / "x.bwb"))
    assert st == A.BW_ERR_IO and "not a block file" in msg
    (tmp_path / "z.bwb").write_bytes(b"BW")
    assert _status(lambda: blockfile.info(tmp_path / "z.bwb"))[0] == A.BW_ERR_IO
    st, msg = _status(lambda: blockfile.info(tmp_path / "none.bwb"))
    assert st == A.BW_ERR_IO and "cannot open" in msg


def test_bad_arguments_leave_no_file(tmp_path):
    from bigwham_dev_b200 import _capi as A
    from bigwham_dev_b200 import blockfile

    ex, _ = _small(tmp_path)
    bad = dict(ex, fr=np.array([[0, 0, 4, 4], [5, 4, 9, 8]]))  # same size, i_end past the last point
    st, msg = _status(lambda: blockfile.write(tmp_path / "b1.bwb", bad))
    assert st == A.BW_ERR_ARG and "outside the matrix" in msg
    bad = dict(ex, perm0=np.array([0, 1, 2, 3, 4, 5, 6, 8]))
    st, msg = _status(lambda: blockfile.write(tmp_path / "b2.bwb", bad))
    assert st == A.BW_ERR_ARG and "perm0" in msg
    with pytest.raises(ValueError):
        blockfile.write(tmp_path / "b3.bwb", dict(ex, fr_data=ex["fr_data"][:-1]))
    assert sorted(os.listdir(tmp_path)) == ["s.bwb"]  # nothing half-written, no temporaries
    # overwriting an existing file replaces it
    ex2 = dict(ex, fr_data=ex["fr_data"] * 2)
    blockfile.write(tmp_path / "s.bwb", ex2)
    assert np.array_equal(blockfile.read(tmp_path / "s.bwb")["fr_data"], ex2["fr_data"])


# --------------------------------------------------------------------------- format pin
M64 = (1 << 64) - 1
GOLDEN = 0x9E3779B97F4A7C15
SEED = 0x42574C4F434B5331


def _mix64(x):  # splitmix64 output function (Steele, Lea, Flood 2014)
    x = (x + GOLDEN) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


def _rotl(x, r):
    return ((x << r) | (x >> (64 - r))) & M64


def _section_hash_py(data: bytes) -> int:
    """Restatement of the documented checksum for data within one block:
    four lanes (word i -> lane i mod 4), lane = rotl(lane ^ w * golden, 31) *
    0xBF58476D1CE4E5B9, block = mix over (count, lanes), folded from SEED and
    finished with the byte count."""
    words = struct.unpack(f"<{len(data) // 8}Q", data)
    assert len(words) <= 1 << 17
    acc = SEED
    if words:
        s = [_mix64((SEED + i) & M64) for i in range(4)]
        for i, w in enumerate(words):
            s[i & 3] = (_rotl(s[i & 3] ^ ((w * GOLDEN) & M64), 31) * 0xBF58476D1CE4E5B9) & M64
        h = _mix64(len(words))
        for v in s:
            h = _mix64(h ^ v)
        acc = _mix64(acc ^ h)
    return _mix64(acc ^ len(data))


def test_header_layout_and_checksums_follow_the_format(tmp_path):
    ex, path = _small(tmp_path)
    raw = open(path, "rb").read()
    assert raw[:8] == b"BWBLOCKS"
    version, hbytes = struct.unpack_from("<II", raw, 8)
    dof, n_rows, n_cols, n_fr, n_lr, fr_e, lr_e, flags = struct.unpack_from("<8q", raw, 16)
    assert (version, hbytes) == (1, 256)
    assert (dof, n_rows, n_cols, n_fr, n_lr, fr_e, lr_e, flags) == (1, 8, 8, 2, 1, 32, 8, 0)
    (hh,) = struct.unpack_from("<Q", raw, 248)
    assert hh == _section_hash_py(raw[:248])
    expect = [np.asarray(ex["perm0"], np.int64).tobytes(), np.asarray(ex["perm1"], np.int64).tobytes(), None, None,
              b"", ex["fr_data"].tobytes(), ex["lr_data"].tobytes()]
    end = 256
    for s in range(7):
        off, nbytes, hs = struct.unpack_from("<qqQ", raw, 80 + 24 * s)
        assert off % 4096 == 0 and off >= end
        body = raw[off:off + nbytes]
        if expect[s] is not None:
            assert body == expect[s], s
        assert hs == _section_hash_py(body), s
        end = off + nbytes
    assert end == len(raw)


def test_rank_zero_blocks_round_trip_and_plan(tmp_path):
    """Low-rank blocks of rank 0 (no factors) survive the file bitwise, and a
    handle made from the file plans the same operator as the flat upload."""
    from bigwham_dev_b200 import HmatGpu, blockfile
    from planreplay import replay
    from synth import synthetic_hmat

    arr = synthetic_hmat(30, 22, 3, seed=31, lr_share=0.8, rank0_share=0.5)
    assert (arr.lr[:, 4] == 0).any()
    ex = {"dof": arr.dof, "n_rows": arr.n_rows, "n_cols": arr.n_cols, "fr": arr.fr, "lr": arr.lr,
          "fr_data": arr.fr_data, "lr_data": arr.lr_data, "perm0": arr.perm0, "perm1": arr.perm1}
    p = tmp_path / "r0.bwb"
    blockfile.write(p, ex)
    r = blockfile.read(p)
    for k in FLAT:
        assert np.array_equal(r[k], np.asarray(ex[k])), k
    x = np.random.default_rng(2).uniform(-1, 1, arr.n_cols)
    h1 = HmatGpu.from_file(p, device=-1, precisions=("fp64", "bf16"), plan_only=True)
    h2 = HmatGpu(arr.dof, arr.n_rows, arr.n_cols, arr.perm0, arr.perm1, device=-1)
    h2.add_flat(arr.fr, arr.lr, arr.fr_data, arr.lr_data)
    h2.finalize(plan_only=True, precisions=("fp64", "bf16"))
    for prec in ("fp64", "bf16"):
        assert np.array_equal(replay(h1, x, prec), replay(h2, x, prec))
