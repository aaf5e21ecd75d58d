"""The TMA-staged y-sweep's bounded waits, made to run out on purpose.

Every wait of the staged y-sweep (ystage 1) for a box of rows is bounded by the
GPU's global timer.  With the limit set to 1 ns (mhd_set_tma_wait_limit), the
first wave of CTAs -- which queue tens of MB of box copies at launch -- gives up
on boxes still in flight: each such CTA raises its abort flag, waits (with the
full 2 s limit) for the copies it has in flight, and returns, and the next
synchronising call reports MHD_ERR_TIMEOUT.  Nothing faults and the context
stays usable: with the limit back at its default the same workspace then
computes the same step bit for bit as the per-thread-load sweep (FP64) or as a
fresh workspace running the same staged kernels (FP32).
"""
import time

import numpy as np
import pytest

from mhd_gpu_acc_b200 import (
    F32,
    F64,
    GpuWorkspace,
    Grid2DGPU,
    MhdError,
    advance_second_order_gpu,
    compute_dt_gpu,
    get_n_case_config,
    init_gpu_workspace,
    initialise,
    set_gpu_physics_ch,
    set_gpu_physics_gamma,
)

pytestmark = pytest.mark.gpu
TIMEOUT = -8  # MHD_ERR_TIMEOUT


def _workspace(U, cfg, ystage):
    ws = GpuWorkspace()
    init_gpu_workspace(ws, U)
    set_gpu_physics_gamma(ws, cfg.gamma)
    set_gpu_physics_ch(ws, 0.0)
    ws.set_limiter(1)
    ws.set_sweep_shape(8, 0, ystage)
    return ws


@pytest.mark.parametrize("dtype", [F64, F32])
def test_tma_wait_runs_out_and_the_workspace_recovers(dtype):
    n = 2048
    cfg = get_n_case_config(4, 1)
    U0 = initialise(4, n, n, 2, cfg.extent)
    grids = [Grid2DGPU(n, n, 2, *cfg.extent, dtype) for _ in range(3)]
    Uold, Utmp, Unew = grids
    for g in grids:
        g.upload(U0)
    bc = (0, 0, 0, 0)

    # the reference result: per-thread loads (FP64) or a fresh staged workspace (FP32)
    ws_ref = _workspace(Uold, cfg, 0 if dtype == F64 else 1)
    dt = compute_dt_gpu(Uold, ws_ref, cfg.cfl)
    advance_second_order_gpu(Uold, Utmp, Unew, ws_ref, dt, 2, bc)
    ws_ref.synchronize()
    want = Unew.download()
    ws_ref.destroy()

    ws = _workspace(Uold, cfg, 1)
    assert compute_dt_gpu(Uold, ws, cfg.cfl) == dt
    ws.set_tma_wait_limit(1)
    t0 = time.perf_counter()
    advance_second_order_gpu(Uold, Utmp, Unew, ws, dt, 2, bc)
    with pytest.raises(MhdError) as err:
        ws.synchronize()
    assert err.value.code == TIMEOUT
    assert time.perf_counter() - t0 < 10.0
    ws.synchronize()  # the fault word was read and cleared

    ws.set_tma_wait_limit(0)
    advance_second_order_gpu(Uold, Utmp, Unew, ws, dt, 2, bc)
    ws.synchronize()
    np.testing.assert_array_equal(Unew.download(), want)
    ws.destroy()
