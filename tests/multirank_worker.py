"""Rank body of tests/test_multirank.py, launched by torch.distributed.run with
the gloo backend on CPU: the batch shard plan and the rank reductions that
bench.py uses, and (mode "fail") a rank that dies between steps."""
import datetime
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import torch.distributed as dist  # noqa: E402

import bench  # noqa: E402
from mhd_gpu_acc_b200.batch import orszag_tang_batch_spec  # noqa: E402


def main(mode: str) -> int:
    world, rank, _ = bench.dist_setup()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=20))
    descs, _, _ = orszag_tang_batch_spec(0, 256)
    cells = [int(d.nx) * int(d.ny) for d in descs]
    mine = bench.batch_shard(descs, world, rank)
    plans = [None] * world
    dist.all_gather_object(plans, mine)
    flat = sorted(i for p in plans for i in p)
    assert flat == list(range(len(descs))), "shards must cover the batch exactly once"
    loads = [sum(cells[i] for i in p) for p in plans]
    assert max(loads) - min(loads) <= max(cells), loads
    # the reductions bench.py times with: max of per-rank times, sum of updates
    assert bench.max_over_ranks(float(rank + 1), world) == float(world)
    assert bench.sum_over_ranks(float(rank + 1), world) == world * (world + 1) / 2
    my_updates = float(sum(cells[i] for i in mine) * 10)
    assert bench.sum_over_ranks(my_updates, world) == float(sum(cells) * 10)
    bench.barrier(world)
    if mode == "fail":
        if rank == 1:
            raise SystemExit(3)  # leaves between steps, with nothing in flight
        try:
            bench.max_over_ranks(1.0, world)  # the peer never joins this step
        except Exception as e:  # noqa: BLE001 - any collective error is the detection
            print(f"rank {rank} detected the lost peer: {type(e).__name__}", flush=True)
            return 4
        return 0
    dist.destroy_process_group()
    print(f"rank {rank} ok: {len(mine)} instances, {loads[rank]} cells", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1] if len(sys.argv) > 1 else "ok"))
