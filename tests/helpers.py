"""Shared helpers for the parity tests."""
from __future__ import annotations

import hashlib

import numpy as np

from mhd_gpu_acc_b200 import (
    F64,
    GpuWorkspace,
    Grid2DGPU,
    advance_second_order_gpu,
    compute_dt_gpu,
    init_gpu_workspace,
    set_gpu_physics_ch,
    set_gpu_physics_gamma,
)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def rel_l1(a: np.ndarray, b: np.ndarray, ng: int = 2) -> np.ndarray:
    """Per-field relative L1 of the interiors: sum|a-b| / sum|b| (0 where b is all zero)."""
    ai = a[:, ng:-ng, ng:-ng].reshape(9, -1)
    bi = b[:, ng:-ng, ng:-ng].reshape(9, -1)
    num = np.abs(ai - bi).sum(axis=1)
    den = np.abs(bi).sum(axis=1)
    return np.where(den > 0, num / np.where(den > 0, den, 1.0), num)


def rel_linf(a: np.ndarray, b: np.ndarray, ng: int = 2) -> np.ndarray:
    ai = a[:, ng:-ng, ng:-ng].reshape(9, -1)
    bi = b[:, ng:-ng, ng:-ng].reshape(9, -1)
    scale = np.abs(bi).max(axis=1)
    return np.abs(ai - bi).max(axis=1) / np.where(scale > 0, scale, 1.0)


def gpu_driver_loop(U0, nx, ny, ng, extent, gamma, cfl, solver, bc, max_steps=0, t_end=1.0, limiter=0, ch=0.0):
    """The reference GPU driver loop (scripts/gpu/main_gpu.cu:208-236) through the
    drop-in API, FP64, without the initial apply_boundary (the CPU driver's
    policy: ghosts hold initial-condition values).  Returns (U, t, steps, dts, ch)."""
    x0, x1, y0, y1 = extent
    Uold = Grid2DGPU(nx, ny, ng, x0, x1, y0, y1, F64)
    Utmp = Grid2DGPU(nx, ny, ng, x0, x1, y0, y1, F64)
    Unew = Grid2DGPU(nx, ny, ng, x0, x1, y0, y1, F64)
    Uold.upload(U0)
    Utmp.upload(U0)
    Unew.upload(U0)
    ws = GpuWorkspace()
    init_gpu_workspace(ws, Uold)
    set_gpu_physics_gamma(ws, gamma)
    set_gpu_physics_ch(ws, ch)
    ws.set_limiter(limiter)
    t, steps, dts = 0.0, 0, []
    while t < t_end and (max_steps <= 0 or steps < max_steps):
        dt_raw = compute_dt_gpu(Uold, ws, cfl)
        dt = min(dt_raw, t_end - t)
        if not np.isfinite(dt) or dt <= 0.0 or dt < 1e-8 * t_end:
            break
        advance_second_order_gpu(Uold, Utmp, Unew, ws, dt, solver, bc)
        Uold.swap(Unew)
        dts.append(dt)
        t += dt
        steps += 1
    out = Uold.download()
    ch = ws.ch
    ws.destroy()
    return out, t, steps, np.array(dts), ch


def device_loop(U0, nx, ny, ng, extent, gamma, cfl, solver, bc, limiter=0, max_steps=0, t_end=1.0, dtype=F64):
    """The device-resident CUDA-graph driver loop (mhd_run) from the same initial
    array as gpu_driver_loop.  Returns (U, run_info)."""
    from mhd_gpu_acc_b200 import GpuWorkspace as _W

    U = Grid2DGPU(nx, ny, ng, *extent, dtype)
    T = Grid2DGPU(nx, ny, ng, *extent, dtype)
    U.upload(U0)
    T.upload(U0)
    ws = _W()
    init_gpu_workspace(ws, U)
    set_gpu_physics_gamma(ws, gamma)
    set_gpu_physics_ch(ws, 0.0)
    ws.set_limiter(limiter)
    info = ws.run(U, T, cfl, t_end, max_steps, solver, bc)
    out = U.download()
    ws.destroy()
    U.release()
    T.release()
    return out, info


def inject_faults(U0: np.ndarray, ng: int) -> np.ndarray:
    """A copy of U0 with a NaN density in one interior cell and, in another, an
    energy below the kinetic + magnetic energy (negative pressure)."""
    U = U0.copy()
    U[0, ng + 12, ng + 9] = np.nan
    j, i = ng + 20, ng + 22
    ke = 0.5 * (U[1, j, i] ** 2 + U[2, j, i] ** 2 + U[3, j, i] ** 2) / U[0, j, i]
    me = 0.5 * (U[4, j, i] ** 2 + U[5, j, i] ** 2 + U[6, j, i] ** 2)
    U[7, j, i] = 0.5 * (ke + me)
    return U


def hot_cell(U0: np.ndarray, ng: int) -> np.ndarray:
    """A copy of U0 with E = 1e30 in one cell: its sound speed makes the first dt
    ~1e-17, under 1e-8 t_end."""
    U = U0.copy()
    U[7, ng + 5, ng + 5] = 1e30
    return U
