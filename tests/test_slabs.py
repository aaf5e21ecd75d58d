"""One grid split into y-slabs (mhd_gpu_acc_b200.slabs): the plan on the CPU,
and on the GPU the slabbed step -- per-slab device-clocked sweeps, the halo
exchange on a second stream while the y-sweeps do the rows that need no halo,
and a global CFL maximum reduced on the device -- against the single-grid
device loop (mhd_run), bit for bit in FP64 and FP32."""
import numpy as np
import pytest

from helpers import device_loop
from mhd_gpu_acc_b200 import F32, F64, get_n_case_config, initialise, set_gpu_physics_ch, set_gpu_physics_gamma
from mhd_gpu_acc_b200.slabs import (
    EXCHANGED,
    SWEEP_NO_ADVANCE,
    SWEEP_NO_GATHER,
    SlabGrid,
    halo_copies,
    neighbours,
    slab_bc,
    slab_extent,
    slab_rows,
    y_windows,
)


def test_slab_plan():
    assert slab_rows(10, 3) == [(0, 4), (4, 7), (7, 10)]
    with pytest.raises(ValueError):
        slab_rows(5, 3)
    assert neighbours(0, 3, False) == (None, 1) and neighbours(2, 3, False) == (1, None)
    assert neighbours(0, 3, True) == (2, 1) and neighbours(0, 1, True) == (None, None)
    assert slab_bc((2, 1, 1, 2), 0, 3) == (2, 1, 1, EXCHANGED)
    assert slab_bc((2, 1, 1, 2), 2, 3) == (2, 1, EXCHANGED, 2)
    assert slab_bc((0, 0, 0, 0), 0, 3) == (0, 0, EXCHANGED, EXCHANGED)
    assert slab_bc((0, 0, 0, 0), 0, 1) == (0, 0, 0, 0)
    # slab 1 (rows 4..6, 3 rows) sends its top rows to slab 2's bottom ghost rows
    # and its bottom rows to slab 0's top ghost rows (ng = 2)
    assert (1, 3, 2, 0) in halo_copies(slab_rows(10, 3), 2, False)
    assert (1, 2, 0, 6) in halo_copies(slab_rows(10, 3), 2, False)
    assert len(halo_copies(slab_rows(10, 3), 2, True)) == 6
    assert slab_extent(0.0, 1.0, 8, 2, 6) == (0.25, 0.75)
    # y-sweep launches: interior rows during the exchange, the edge rows after it;
    # exactly one launch gathers Dirichlet ghosts and advances the clock
    quiet = SWEEP_NO_GATHER | SWEEP_NO_ADVANCE
    assert y_windows(10, True) == ([(2, 6, quiet)], [(0, 2, quiet), (8, 2, 0)])
    assert y_windows(4, True) == ([], [(0, 0, 0)])
    assert y_windows(10, False) == ([], [(0, 0, 0)])
    for n in range(5, 40):
        early, late = y_windows(n, True)
        rows = sorted(r for r0, k, _ in early + late for r in range(r0, r0 + k))
        assert rows == list(range(n))
        assert [f for *_, f in early + late].count(0) == 1


def _single(case, nx, ny, bc, steps, dtype, limiter):
    """The single-grid device loop (mhd_run) for `steps` steps."""
    cfg = get_n_case_config(case, 1)
    U0 = initialise(case, nx, ny, 2, cfg.extent)
    out, info = device_loop(U0, nx, ny, 2, cfg.extent, cfg.gamma, cfg.cfl, 2, bc, limiter=limiter,
                            max_steps=steps, t_end=cfg.t_end, dtype=dtype)
    return U0, out, info


@pytest.mark.gpu
@pytest.mark.parametrize("case,nx,ny,bc,parts,dtype", [
    (4, 128, 128, (0, 0, 0, 0), 2, F64),   # Orszag-Tang, periodic: a ring of slabs
    (4, 128, 128, (0, 0, 0, 0), 3, F64),
    (4, 96, 130, (0, 0, 0, 0), 4, F32),
    (5, 96, 80, (1, 1, 1, 1), 3, F64),     # shock-bubble, transmissive outer sides
    (1, 64, 90, (2, 1, 2, 1), 5, F64),     # reflecting / transmissive mix
    (4, 64, 12, (0, 0, 0, 0), 3, F64),     # 4-row slabs: no interior-only rows
])
def test_slabbed_step_matches_single_grid(case, nx, ny, bc, parts, dtype):
    cfg = get_n_case_config(case, 1)
    steps = 12
    U0, ref, info = _single(case, nx, ny, bc, steps, dtype, 1)
    sg = SlabGrid(nx, ny, 2, cfg.extent, parts, dtype)
    sg.upload(U0)
    sg.configure(cfg.gamma, 1)
    sg.start(cfg.cfl, cfg.t_end)
    for _ in range(steps):
        sg.step(2, bc)
    got = sg.info()
    out = sg.download()
    sg.destroy()
    assert (got.steps, got.t, got.last_dt, got.ch) == (info.steps, info.t, info.last_dt, info.ch)
    np.testing.assert_array_equal(out[:, 2:-2, :], ref[:, 2:-2, :])


@pytest.mark.gpu
def test_rank_slab_runner_single_rank_matches_single_grid():
    """DistSlabRun on a one-rank NCCL group (the device tensor views of the state
    and of the clock slots, the all-reduce and the clocked sweeps of the rank
    path) equals the single-grid device loop."""
    import socket

    import torch
    import torch.distributed as dist

    from mhd_gpu_acc_b200.slabs import DistSlabRun

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        cfg = get_n_case_config(4, 1)
        U0, ref, info = _single(4, 96, 96, (0, 0, 0, 0), 8, F64, 1)
        run = DistSlabRun(96, 96, 2, cfg.extent, F64)
        run.upload(U0)
        set_gpu_physics_gamma(run.ws, cfg.gamma)
        set_gpu_physics_ch(run.ws, 0.0)
        run.ws.set_limiter(1)
        run.start(cfg.cfl, cfg.t_end)
        for _ in range(8):
            run.step(2, (0, 0, 0, 0))
        got = run.info()
        out = run.U.download()
        run.destroy()
        torch.cuda.synchronize()
        assert (got.steps, got.t, got.ch) == (info.steps, info.t, info.ch)
        np.testing.assert_array_equal(out[:, 2:-2, :], ref[:, 2:-2, :])
    finally:
        dist.destroy_process_group()
