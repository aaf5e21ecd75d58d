"""Rank body of tests/test_multirank.py, launched by torch.distributed.run with
the gloo backend on CPU: the batch shard plan and the rank reductions that
bench.py uses, (mode "fail") a rank that dies between steps, and (modes
"halo" / "halo_periodic") the y-slab halo exchange of one grid split over the
ranks."""
import datetime
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import torch.distributed as dist  # noqa: E402

import bench  # noqa: E402
from mhd_gpu_acc_b200.batch import orszag_tang_batch_spec  # noqa: E402


def halo(periodic: bool) -> int:
    """Each rank holds its slab of a marked global array (value = 1000 * global
    storage row + field); after exchange_rows every ghost row next to a
    neighbour holds that neighbour's rows, the others are untouched."""
    import torch

    from mhd_gpu_acc_b200.slabs import exchange_rows, neighbours, slab_rows

    world, rank, _ = bench.dist_setup()
    ng, ny, width = 3, 23, 5
    rows = slab_rows(ny, world)
    r0, r1 = rows[rank]
    n = r1 - r0
    f = torch.arange(9, dtype=torch.float64).view(9, 1, 1)
    g = torch.arange(r0, r1 + 2 * ng, dtype=torch.float64).view(1, -1, 1)  # global storage rows
    state = (1000 * g + f).expand(9, n + 2 * ng, width).clone()
    state[:, :ng, :] = -1.0  # ghost rows start invalid
    state[:, ng + n:, :] = -1.0
    below, above = neighbours(rank, world, periodic)
    exchange_rows(state, n, ng, below, above, dist)
    tny = ny + 2 * ng

    def expect(global_storage_row):  # periodic wrap of interior rows
        if periodic:
            global_storage_row = ng + (global_storage_row - ng) % ny
        return 1000 * global_storage_row + f.view(9, 1)

    for k in range(ng - 2, ng):  # bottom ghost rows the y-sweep reads
        got = state[:, k, :]
        if below is None:
            assert torch.all(got == -1.0)
        else:
            assert torch.all(got == expect(r0 + k)), (rank, k, got[:, 0])
    for k in range(ng + n, ng + n + 2):
        got = state[:, k, :]
        if above is None:
            assert torch.all(got == -1.0)
        else:
            assert torch.all(got == expect(r0 + k)), (rank, k, got[:, 0])
    assert torch.all(state[:, :ng - 2, :] == -1.0) and torch.all(state[:, ng + n + 2:, :] == -1.0)
    assert tny > 0
    print(f"rank {rank} ok: halo rows of slab {r0}..{r1}", flush=True)
    return 0


def main(mode: str) -> int:
    world, rank, _ = bench.dist_setup()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=20))
    if mode in ("halo", "halo_periodic"):
        rc = halo(mode == "halo_periodic")
        dist.destroy_process_group()
        return rc
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
