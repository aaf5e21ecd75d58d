"""One grid split into y-slabs (mhd_gpu_acc_b200.slabs): the plan on the CPU,
and on the GPU the slabbed step -- per-slab sweeps with the halo exchange
between them and a global CFL maximum -- against the single-grid drop-in step,
bit for bit in FP64 and FP32."""
import numpy as np
import pytest

from mhd_gpu_acc_b200 import (
    F32,
    F64,
    GpuWorkspace,
    Grid2DGPU,
    advance_second_order_gpu,
    compute_dt_gpu,
    get_n_case_config,
    init_gpu_workspace,
    initialise,
    set_gpu_physics_ch,
    set_gpu_physics_gamma,
)
from mhd_gpu_acc_b200.slabs import EXCHANGED, SlabGrid, halo_copies, neighbours, slab_bc, slab_extent, slab_rows


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


def _single(case, nx, ny, bc, steps, dtype, limiter):
    cfg = get_n_case_config(case, 1)
    U0 = initialise(case, nx, ny, 2, cfg.extent)
    U, T, N = (Grid2DGPU(nx, ny, 2, *cfg.extent, dtype) for _ in range(3))
    for g in (U, T, N):
        g.upload(U0)
    ws = GpuWorkspace()
    init_gpu_workspace(ws, U)
    set_gpu_physics_gamma(ws, cfg.gamma)
    set_gpu_physics_ch(ws, 0.0)
    ws.set_limiter(limiter)
    dts = []
    for _ in range(steps):
        dt = compute_dt_gpu(U, ws, cfg.cfl)
        advance_second_order_gpu(U, T, N, ws, dt, 2, bc)
        U.swap(N)
        dts.append(dt)
    out = U.download()
    ws.destroy()
    return U0, out, dts


@pytest.mark.gpu
@pytest.mark.parametrize("case,nx,ny,bc,parts,dtype", [
    (4, 128, 128, (0, 0, 0, 0), 2, F64),   # Orszag-Tang, periodic: a ring of slabs
    (4, 128, 128, (0, 0, 0, 0), 3, F64),
    (4, 96, 130, (0, 0, 0, 0), 4, F32),
    (5, 96, 80, (1, 1, 1, 1), 3, F64),     # shock-bubble, transmissive outer sides
    (1, 64, 90, (2, 1, 2, 1), 5, F64),     # reflecting / transmissive mix
])
def test_slabbed_step_matches_single_grid(case, nx, ny, bc, parts, dtype):
    cfg = get_n_case_config(case, 1)
    steps = 12
    U0, ref, dts = _single(case, nx, ny, bc, steps, dtype, 1)
    sg = SlabGrid(nx, ny, 2, cfg.extent, parts, dtype)
    sg.upload(U0)
    sg.configure(cfg.gamma, 1)
    got_dts = [sg.step(cfg.cfl, 2, bc) for _ in range(steps)]
    out = sg.download()
    sg.destroy()
    assert got_dts == dts
    np.testing.assert_array_equal(out[:, 2:-2, :], ref[:, 2:-2, :])


@pytest.mark.gpu
def test_rank_slab_runner_single_rank_matches_single_grid():
    """DistSlabRun on a one-rank NCCL group (the device tensor views, the
    all-reduce and the sweeps of the rank path) equals the single-grid step."""
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
        U0, ref, dts = _single(4, 96, 96, (0, 0, 0, 0), 8, F64, 1)
        run = DistSlabRun(96, 96, 2, cfg.extent, F64)
        run.upload(U0)
        load_ws = run.ws
        set_gpu_physics_gamma(load_ws, cfg.gamma)
        set_gpu_physics_ch(load_ws, 0.0)
        load_ws.set_limiter(1)
        got = [run.step(cfg.cfl, 2, (0, 0, 0, 0)) for _ in range(8)]
        out = run.U.download()
        run.destroy()
        torch.cuda.synchronize()
        assert got == dts
        np.testing.assert_array_equal(out[:, 2:-2, :], ref[:, 2:-2, :])
    finally:
        dist.destroy_process_group()
