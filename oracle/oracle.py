"""ctypes loaders for the CPU checkers (test infrastructure only).

``Oracle`` wraps ``oracle/libmhd_oracle.so`` (this project's plain-C FP64
restatement, ``oracle/mhd_oracle.c``); ``Reference`` wraps
``oracle/_ref/libmhdref.so`` (the reference's own CPU/OpenMP step compiled from
its unmodified sources by ``oracle/Makefile``).  Only tests/, the fixture
generator under tests/golden, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline / reference legs may import this module.

All state arrays are float64 of shape (9, ny + 2 ng, nx + 2 ng): the SoA plane
order rho, rhou, rhov, rhow, Bx, By, Bz, E, psi (reference head/types.hpp:16-41),
row-major with ghost cells (head/cpu/grid_cpu.hpp:85-87).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libmhd_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmhdref.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_D = C.c_double
_I = C.c_int
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int)


def build(ref: bool = True) -> None:
    """Compile the oracle (and the reference build when its sources exist)."""
    target = "all" if ref else "oracle"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def _state(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    assert a.ndim == 3 and a.shape[0] == 9, a.shape
    return a


def _bc(bc):
    return np.ascontiguousarray(np.asarray(bc, dtype=np.int32).reshape(4))


class Oracle:
    """This project's C restatement (supports the van Leer limiter too)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(ref=False)
        lib = C.CDLL(path)
        lib.orc_compute_dt_c.argtypes = [_dp, _I, _I, _I, _D, _D, _D, _D, _pd, _pd]
        lib.orc_compute_dt_c.restype = _I
        lib.orc_advance_c.argtypes = [_dp, _dp, _dp, _I, _I, _I, _D, _D, _D, _D, _D, _D, _I, _I, _ip]
        lib.orc_advance_c.restype = None
        lib.orc_apply_boundary_c.argtypes = [_dp, _I, _I, _I, _ip]
        lib.orc_apply_boundary_c.restype = None
        lib.orc_run_c.argtypes = [_dp, _I, _I, _I, _D, _D, _D, _D, _D, _I, _I, _ip, _I, _D, _pd, _pd, _pi, _pd]
        lib.orc_run_c.restype = _I
        lib.orc_riemann_c.argtypes = [_dp, _dp, _I, _I, _D, _D, _dp]
        lib.orc_riemann_c.restype = None
        lib.orc_set_threads.argtypes = [_I]
        self.lib = lib

    def set_threads(self, n: int) -> None:
        self.lib.orc_set_threads(int(n))

    def compute_dt(self, U, ng, dx, dy, gamma, cfl, ch_prev):
        U = _state(U)
        ny, nx = U.shape[1] - 2 * ng, U.shape[2] - 2 * ng
        ch, dt = _D(ch_prev), _D(0.0)
        rc = self.lib.orc_compute_dt_c(U, nx, ny, ng, dx, dy, gamma, cfl, C.byref(ch), C.byref(dt))
        return rc, dt.value, ch.value

    def advance(self, Uold, ng, dx, dy, gamma, ch, dt, solver, limiter, bc, cr=0.18, Utmp=None, Unew=None):
        Uold = _state(Uold)
        ny, nx = Uold.shape[1] - 2 * ng, Uold.shape[2] - 2 * ng
        Utmp = np.zeros_like(Uold) if Utmp is None else _state(Utmp).copy()
        Unew = np.zeros_like(Uold) if Unew is None else _state(Unew).copy()
        self.lib.orc_advance_c(Uold, Utmp, Unew, nx, ny, ng, dx, dy, gamma, ch, cr, dt, solver, limiter, _bc(bc))
        return Utmp, Unew

    def apply_boundary(self, U, ng, bc):
        U = _state(U).copy()
        ny, nx = U.shape[1] - 2 * ng, U.shape[2] - 2 * ng
        self.lib.orc_apply_boundary_c(U, nx, ny, ng, _bc(bc))
        return U

    def run(self, U, ng, dx, dy, gamma, cfl, solver, limiter, bc, max_steps=0, t_end=1e300, ch=0.0, cr=0.18):
        """Driver loop; returns (rc, U_final, t, steps, ch, dt_log)."""
        U = _state(U).copy()
        ny, nx = U.shape[1] - 2 * ng, U.shape[2] - 2 * ng
        cap = max_steps if max_steps > 0 else 1_000_000
        dtlog = np.zeros(cap, dtype=np.float64)
        chv, tv, st = _D(ch), _D(0.0), _I(0)
        rc = self.lib.orc_run_c(U, nx, ny, ng, dx, dy, gamma, cfl, cr, solver, limiter, _bc(bc), max_steps,
                                t_end, C.byref(chv), C.byref(tv), C.byref(st), dtlog.ctypes.data_as(_pd))
        return rc, U, tv.value, st.value, chv.value, dtlog[: st.value].copy()

    def riemann(self, UL, UR, direction, solver, ch, gamma):
        F = np.zeros(9)
        self.lib.orc_riemann_c(np.ascontiguousarray(UL, dtype=np.float64),
                               np.ascontiguousarray(UR, dtype=np.float64), direction, solver, ch, gamma, F)
        return F


class Reference:
    """The reference's own CPU path (minmod only), built into oracle/_ref."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = C.CDLL(path)
        geo = [_I, _I, _I, _D, _D, _D, _D]
        lib.ref_compute_dt.argtypes = [_dp] + geo + [_D, _D, _pd, _pd]
        lib.ref_compute_dt.restype = _I
        lib.ref_advance.argtypes = [_dp, _dp, _dp] + geo + [_D, _D, _D, _I, _ip]
        lib.ref_advance.restype = _I
        lib.ref_apply_boundary.argtypes = [_dp, _I, _I, _I, _ip]
        lib.ref_apply_boundary.restype = _I
        lib.ref_run.argtypes = [_dp] + geo + [_D, _D, _I, _ip, _I, _D, _pd, _pd, _pi, _pd]
        lib.ref_run.restype = _I
        lib.ref_run_timed.argtypes = [_dp] + geo + [_D, _D, _I, _ip, _I, _D, _pd, _pd, _pi]
        lib.ref_run_timed.restype = _I
        lib.ref_initial_state.argtypes = [_I, _D, _D, _dp]
        lib.ref_initial_state.restype = None
        lib.ref_case_config.argtypes = [_I, _I, _dp]
        lib.ref_case_config.restype = _I
        lib.ref_riemann.argtypes = [_dp, _dp, _I, _I, _D, _D, _dp]
        lib.ref_riemann.restype = None
        lib.ref_initialise_orszag_tang_unit.argtypes = [_I, _I, _I, _dp]
        lib.ref_initialise_orszag_tang_unit.restype = _I
        lib.ref_set_threads.argtypes = [_I]
        lib.ref_max_threads.restype = _I
        self.lib = lib

    def set_threads(self, n: int) -> None:
        self.lib.ref_set_threads(int(n))

    def max_threads(self) -> int:
        return int(self.lib.ref_max_threads())

    def run(self, U, ng, extent, gamma, cfl, solver, bc, max_steps=0, t_end=1e300, ch=0.0):
        U = _state(U).copy()
        ny, nx = U.shape[1] - 2 * ng, U.shape[2] - 2 * ng
        cap = max_steps if max_steps > 0 else 1_000_000
        dtlog = np.zeros(cap, dtype=np.float64)
        chv, tv, st = _D(ch), _D(0.0), _I(0)
        x0, x1, y0, y1 = extent
        rc = self.lib.ref_run(U, nx, ny, ng, x0, x1, y0, y1, gamma, cfl, solver, _bc(bc), max_steps, t_end,
                              C.byref(chv), C.byref(tv), C.byref(st), dtlog.ctypes.data_as(_pd))
        return rc, U, tv.value, st.value, chv.value, dtlog[: st.value].copy()

    def run_timed(self, U, ng, extent, gamma, cfl, solver, bc, steps, t_end, ch=0.0):
        """Driver loop with per-step wall time; U is advanced in place.
        Returns (rc, steps_done, step_seconds, ch)."""
        assert U.flags.c_contiguous and U.dtype == np.float64
        ny, nx = U.shape[1] - 2 * ng, U.shape[2] - 2 * ng
        secs = np.zeros(max(1, steps))
        chv, st = _D(ch), _I(0)
        rc = self.lib.ref_run_timed(U, nx, ny, ng, *extent, gamma, cfl, solver, _bc(bc), steps, t_end, C.byref(chv),
                                    secs.ctypes.data_as(_pd), C.byref(st))
        return rc, st.value, secs[: st.value].copy(), chv.value

    def compute_dt(self, U, ng, extent, gamma, cfl, ch_prev):
        U = _state(U)
        ny, nx = U.shape[1] - 2 * ng, U.shape[2] - 2 * ng
        ch, dt = _D(ch_prev), _D(0.0)
        rc = self.lib.ref_compute_dt(U, nx, ny, ng, *extent, gamma, cfl, C.byref(ch), C.byref(dt))
        return rc, dt.value, ch.value

    def advance(self, Uold, ng, extent, gamma, ch, dt, solver, bc, Utmp=None, Unew=None):
        Uold = _state(Uold)
        ny, nx = Uold.shape[1] - 2 * ng, Uold.shape[2] - 2 * ng
        Utmp = np.zeros_like(Uold) if Utmp is None else _state(Utmp).copy()
        Unew = np.zeros_like(Uold) if Unew is None else _state(Unew).copy()
        self.lib.ref_advance(Uold, Utmp, Unew, nx, ny, ng, *extent, gamma, ch, dt, solver, _bc(bc))
        return Utmp, Unew

    def apply_boundary(self, U, ng, bc):
        U = _state(U).copy()
        ny, nx = U.shape[1] - 2 * ng, U.shape[2] - 2 * ng
        self.lib.ref_apply_boundary(U, nx, ny, ng, _bc(bc))
        return U

    def initial_state(self, case_id: int, x: float, y: float):
        out = np.zeros(9)
        self.lib.ref_initial_state(case_id, x, y, out)
        return out

    def initialise_orszag_tang_unit(self, nx: int, ny: int, ng: int = 2):
        """The Orszag-Tang [0,1]^2 initial state (ghosts hold initial-condition
        values) built by the reference build alone: its Grid2D cell centres and
        its prim_to_cons.  Returns the (9, ny + 2 ng, nx + 2 ng) SoA array."""
        U = np.zeros((9, ny + 2 * ng, nx + 2 * ng))
        if self.lib.ref_initialise_orszag_tang_unit(nx, ny, ng, U) != 0:
            raise ValueError((nx, ny, ng))
        return U

    def case_config(self, case_id: int, n: int = 1):
        out = np.zeros(14)
        if self.lib.ref_case_config(case_id, n, out) != 0:
            raise ValueError(case_id)
        return out

    def riemann(self, UL, UR, direction, solver, ch, gamma):
        F = np.zeros(9)
        self.lib.ref_riemann(np.ascontiguousarray(UL, dtype=np.float64),
                             np.ascontiguousarray(UR, dtype=np.float64), direction, solver, ch, gamma, F)
        return F
