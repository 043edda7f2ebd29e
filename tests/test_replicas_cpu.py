"""The N > 1 path of bench.py (replicas) on CPU: 2 processes over gloo.

bench.py --gpus N runs N independent replicas.
* Rank 0 builds the H-matrix once with the reference's host code and writes
  it as a block file (/dev/shm by default).
* Every rank maps the file and lays out its own copy (HmatGpu.from_file).
* Timings are reduced with a max over ranks.
Here each rank lays the blocks out as a host plan and replays a matvec.  The
two ranks must agree bitwise and match the oracle.  max_over_ranks must return
the largest rank value, and the shared file must be gone afterwards.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST_LIB = os.path.join(ROOT, "bigwham_dev_b200", "_lib", "libbigwham_host.so")


def _worker(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist

    import bench
    from bigwham_dev_b200 import HmatGpu, blockfile
    from bigwham_dev_b200.bigwham4py import BigWhamIOGpu
    from bigwham_dev_b200.meshes import square_crack_3d
    from oracle import HmatArrays, oracle_matvec_perm
    from planreplay import replay

    w, r, _ = bench.dist_setup(world, backend="gloo")
    coor, conn = square_crack_3d(12)

    def build(path):
        io = BigWhamIOGpu(coor, conn, "3DR0-H", [1.0, 0.25], 2, useCuda=False)
        io.build_hierarchical_matrix(32, 3.0, 1e-5)
        io.write_to_file(path)
        io.close()

    path = os.path.join(out_dir, f"blocks_{port}.bwb")
    release = bench.shared_block_file(w, r, path, build)
    h = HmatGpu.from_file(path, device=-1, plan_only=True, precisions=("fp64",))
    ex = blockfile.read(path)
    x = np.random.default_rng(0).uniform(-1, 1, ex["n_cols"])
    y = replay(h, x, "fp64")
    flat = HmatArrays(ex["dof"], ex["n_rows"], ex["n_cols"], ex["fr"], ex["lr"], ex["fr_data"], ex["lr_data"],
                      ex["perm0"], ex["perm1"])
    y_or = oracle_matvec_perm(flat, x, 1)
    release()
    m = bench.max_over_ranks(float(r + 1), w, device="cpu")
    np.save(os.path.join(out_dir, f"y{r}.npy"), y)
    np.save(os.path.join(out_dir, f"info{r}.npy"),
            np.array([m, np.linalg.norm(y - y_or) / np.linalg.norm(y_or), float(os.path.exists(path))]))
    dist.destroy_process_group()


@pytest.mark.skipif(not os.path.exists(HOST_LIB), reason="host adapter not built")
def test_two_replicas_share_one_build(tmp_path):
    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    y0, y1 = np.load(tmp_path / "y0.npy"), np.load(tmp_path / "y1.npy")
    assert np.array_equal(y0, y1)
    for r in (0, 1):
        m, err, left = np.load(tmp_path / f"info{r}.npy")
        assert m == 2.0
        assert err < 1e-14
        assert left == 0.0
