"""The FP32 y-sweep's CFL fold skips the fast speeds of cells whose cheap upper
bound stays under the c_h floor of the reduction.  The c_h the device loop
carries into step k (the fold over the state after step k - 1) must equal the
standalone maximum of that state (every cell's exact speed, the same floor),
computed by mhd_compute_dt (src/gpu/solver_gpu.cu:578-605) on the state of a
(k - 1)-step run."""
from __future__ import annotations

import numpy as np
import pytest

from mhd_gpu_acc_b200 import (
    F32,
    CaseId,
    GpuWorkspace,
    Grid2DGPU,
    compute_dt_gpu,
    get_n_case_config,
    init_gpu_workspace,
    initialise,
    set_gpu_physics_ch,
    set_gpu_physics_gamma,
)

HLLD, VANLEER = 2, 1


def _run(U0, n, cfg, steps):
    U = Grid2DGPU(n, n, 2, *cfg.extent, F32)
    T = Grid2DGPU(n, n, 2, *cfg.extent, F32)
    U.upload(U0)
    T.upload(U0)
    ws = GpuWorkspace()
    init_gpu_workspace(ws, U)
    set_gpu_physics_gamma(ws, cfg.gamma)
    set_gpu_physics_ch(ws, 0.0)
    ws.set_limiter(VANLEER)
    info = ws.run(U, T, cfg.cfl, cfg.t_end, steps, HLLD, (0, 0, 0, 0))
    return U, T, ws, info


@pytest.mark.gpu
@pytest.mark.parametrize("case,rises", [(CaseId.OrszagTangUnit, True), (CaseId.KelvinHelmholtz, False)])
def test_skipped_fold_equals_the_exact_maximum(case, rises):
    """Orszag-Tang's maximum rises above the floor in some of these steps (the
    skipped cells must not hide the new maximum); Kelvin-Helmholtz's stays at
    the floor (nearly every cell skipped)."""
    n = 192
    cfg = get_n_case_config(case, 1)
    U0 = initialise(case, n, n, 2, cfg.extent)
    above = 0
    for k in range(2, 26):
        U, T, ws, info = _run(U0, n, cfg, k)
        folded = info.ch  # c_h of step k: the y-sweep fold of step k - 1
        ws.destroy()
        U.release()
        T.release()
        U, T, ws, info = _run(U0, n, cfg, k - 1)
        floor = ws.ch  # c_h of step k - 1, the fold's floor
        compute_dt_gpu(U, ws, cfg.cfl)  # every cell's exact speed, floored by the same c_h
        exact = ws.ch
        ws.destroy()
        U.release()
        T.release()
        # FP32 speeds from differently contracted kernels: within 2^-20
        assert abs(folded - exact) <= 1e-6 * exact, (k, folded, exact)
        above += exact > floor * (1 + 1e-6)
    assert (above > 0) == rises
