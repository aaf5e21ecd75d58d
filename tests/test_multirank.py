"""Multi-rank host logic on CPU: LPT sharding of a batch over GPUs, the rank
reductions bench.py times with, and the y-slab halo exchange of one grid split
over ranks, as gloo ranks launched by torch.distributed.run (the N > 1 paths
without a GPU), plus the loss of a rank between steps."""
import os
import socket
import subprocess
import sys

import pytest

from mhd_gpu_acc_b200.batch import lpt_partition, orszag_tang_batch_spec

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WORKER = os.path.join(ROOT, "tests", "multirank_worker.py")


def test_lpt_partition():
    assert lpt_partition([5, 4, 3, 3, 3], 2) == [[0, 3], [1, 2, 4]]
    assert lpt_partition([1, 1, 1], 5) == [[0], [1], [2], [], []]
    descs, _, _ = orszag_tang_batch_spec(0, 256)
    w = [int(d.nx) * int(d.ny) for d in descs]
    for parts in (1, 2, 3, 4, 8):
        plan = lpt_partition(w, parts)
        assert sorted(i for p in plan for i in p) == list(range(256))
        loads = [sum(w[i] for i in p) for p in plan]
        assert max(loads) - min(loads) <= max(w)
        assert plan == lpt_partition(w, parts)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _torchrun(mode: str, nproc: int = 2):
    cmd = ["timeout", "-k", "10", "150", sys.executable, "-m", "torch.distributed.run", "--nnodes", "1",
           "--nproc-per-node", str(nproc), "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), WORKER,
           mode]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="1")
    return subprocess.run(cmd, capture_output=True, text=True, timeout=200, env=env, cwd=ROOT)


def test_two_gloo_ranks_shard_and_reduce():
    r = _torchrun("ok")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "rank 0 ok" in r.stdout and "rank 1 ok" in r.stdout


def test_lost_rank_is_detected_not_hung():
    r = _torchrun("fail")
    assert r.returncode != 0
    assert r.returncode != 124, "the surviving rank hung"


@pytest.mark.parametrize("mode,nproc", [("halo", 2), ("halo", 3), ("halo_periodic", 2), ("halo_periodic", 3)])
def test_slab_halo_exchange_between_ranks(mode, nproc):
    """The y-slab exchange of one grid split over ranks (mhd_gpu_acc_b200.slabs.exchange_rows)."""
    r = _torchrun(mode, nproc)
    assert r.returncode == 0, r.stdout + r.stderr
    assert all(f"rank {k} ok" in r.stdout for k in range(nproc))
