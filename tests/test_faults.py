"""Faults injected into the initial state, on the GPU (the failure happens in
the data, not in the device: no kernel is made to fault or wait).

The reference's guards are the positivity fallbacks of the reconstruction, the
HLL fallback of the solvers, the revert of a cell whose update is not finite
(src/cpu/solver_cpu.cpp:49-70, 391-392, 429-430), compute_dt skipping
non-physical cells (:291-300) and the driver's dt checks
(scripts/gpu/main_gpu.cu:219-232).  With a NaN density in one cell and a
negative pressure in another, the FP64 step through the drop-in loop equals the
oracle bit for bit (the NaN in the same place; the oracle follows the reference
build on this state, tests/test_oracle.py); the device-resident loop matches it
too and counts the reverted cells (mhd_run_info.fallbacks), where a clean run
counts none.  A state without a physical cell and one whose first dt falls
under 1e-8 t_end stop the device loop with MHD_ERR_NO_SPEED / MHD_ERR_TINY_DT
(include/mhd_b200.h) after no step, the state untouched.
"""
import numpy as np
import pytest

from helpers import device_loop, gpu_driver_loop, hot_cell, inject_faults, rel_l1
from mhd_gpu_acc_b200 import (
    F64,
    GpuWorkspace,
    Grid2DGPU,
    get_n_case_config,
    init_gpu_workspace,
    initialise,
    set_gpu_physics_ch,
    set_gpu_physics_gamma,
)

pytestmark = pytest.mark.gpu

MHD_ERR_NO_SPEED, MHD_ERR_TINY_DT = -3, -5
N, NG, BC, STEPS = 32, 2, (0, 0, 0, 0), 6


def _case():
    cfg = get_n_case_config(4, 1)
    return cfg, initialise(4, N, N, NG, cfg.extent)


@pytest.mark.parametrize("limiter", [0, 1])
def test_injected_faults_drop_in_loop_bit_exact(oracle, limiter):
    cfg, U0 = _case()
    Ub = inject_faults(U0, NG)
    a = oracle.run(Ub, NG, 1 / N, 1 / N, cfg.gamma, cfg.cfl, 2, limiter, BC, max_steps=STEPS, t_end=cfg.t_end)
    U, t, steps, dts, ch = gpu_driver_loop(Ub, N, N, NG, cfg.extent, cfg.gamma, cfg.cfl, 2, BC, max_steps=STEPS,
                                           t_end=cfg.t_end, limiter=limiter)
    assert steps == a[3] == STEPS and ch == a[4]
    np.testing.assert_array_equal(dts, a[5])
    np.testing.assert_array_equal(U, a[1])  # NaN positions included
    assert np.isnan(U).sum() == 1


def test_device_loop_counts_reverted_cells(oracle):
    cfg, U0 = _case()
    Ub = inject_faults(U0, NG)
    U, info = device_loop(Ub, N, N, NG, cfg.extent, cfg.gamma, cfg.cfl, 2, BC, limiter=1, max_steps=STEPS,
                          t_end=cfg.t_end)
    _, clean = device_loop(U0, N, N, NG, cfg.extent, cfg.gamma, cfg.cfl, 2, BC, limiter=1, max_steps=STEPS,
                           t_end=cfg.t_end)
    assert info.status == 0 and info.steps == STEPS
    # the NaN cell alone is reverted by both sweeps of every step
    assert clean.fallbacks == 0 and info.fallbacks >= 2 * STEPS
    a = oracle.run(Ub, NG, 1 / N, 1 / N, cfg.gamma, cfg.cfl, 2, 1, BC, max_steps=STEPS, t_end=cfg.t_end)
    nan = np.isnan(a[1])
    np.testing.assert_array_equal(np.isnan(U), nan)
    # the device loop's damping factor uses the device exp(): 1e-12 instead of bit equality
    assert rel_l1(np.where(nan, 0.0, U), np.where(nan, 0.0, a[1])).max() <= 1e-12


@pytest.mark.parametrize("what,status", [("no physical cell", MHD_ERR_NO_SPEED), ("hot cell", MHD_ERR_TINY_DT)])
def test_device_loop_stop_statuses(what, status):
    cfg, U0 = _case()
    Us = np.zeros_like(U0) if what == "no physical cell" else hot_cell(U0, NG)
    U = Grid2DGPU(N, N, NG, *cfg.extent, F64)
    T = Grid2DGPU(N, N, NG, *cfg.extent, F64)
    U.upload(Us)
    T.upload(Us)
    ws = GpuWorkspace()
    init_gpu_workspace(ws, U)
    set_gpu_physics_gamma(ws, cfg.gamma)
    set_gpu_physics_ch(ws, 0.0)
    info = ws.run(U, T, cfg.cfl, cfg.t_end, 3, 2, BC, raise_on_stop=False)
    out = U.download()
    ws.destroy()
    assert info.status == status and info.steps == 0
    np.testing.assert_array_equal(out, Us)
