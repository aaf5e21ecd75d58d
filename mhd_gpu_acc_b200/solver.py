"""Python mirror of the reference's GPU-path API on top of the C ABI.

Names and argument meanings follow the reference's C++ interface
(head/gpu/grid_gpu.cuh, head/gpu/solver_gpu.cuh, head/gpu/boundary_gpu.cuh,
head/riemann.hpp, head/test_cases.hpp) so that tests read like the
reference's own driver (scripts/gpu/main_gpu.cu):

    cfg = get_n_case_config(CaseId.BrioWu, 1)
    host = make_n_grid(CaseId.BrioWu, 1)
    Uold = Grid2DGPU(cfg.nx, cfg.ny, cfg.ng, cfg.x_min, cfg.x_max, cfg.y_min, cfg.y_max)
    Uold.upload(host)
    ws = GpuWorkspace(); init_gpu_workspace(ws, Uold)
    set_gpu_physics_gamma(ws, cfg.gamma); set_gpu_physics_ch(ws, 0.0)
    dt = compute_dt_gpu(Uold, ws, cfg.cfl)
    advance_second_order_gpu(Uold, Utmp, Unew, ws, dt, RiemannSolver.HLLD, cfg.bc)

Unlike the reference, gamma and ch live in the workspace (the reference keeps
them as per-translation-unit device globals, head/physics.hpp:27-42), so the
setters take the workspace.  Host states are float64 numpy arrays of shape
(9, ny + 2 ng, nx + 2 ng) in the field order rho, rhou, rhov, rhow, Bx, By, Bz,
E, psi.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
import sys
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check, load, mhd_grid, mhd_run_info, mhd_state_meta

F64, F32 = 0, 1


class RiemannSolver(enum.IntEnum):  # head/riemann.hpp:23
    HLL = 0
    HLLC = 1
    HLLD = 2
    FORCE = 3


class Limiter(enum.IntEnum):
    MINMOD = 0   # src/cpu/solver_cpu.cpp:26-43
    VANLEER = 1  # no counterpart in the reference


class BoundaryType(enum.IntEnum):  # head/test_cases.hpp:11-16
    Periodic = 0
    Transmissive = 1
    Reflecting = 2
    Dirichlet = 3


@dataclass
class BoundaryConfig:  # head/test_cases.hpp:18-23
    left: int = BoundaryType.Transmissive
    right: int = BoundaryType.Transmissive
    bottom: int = BoundaryType.Transmissive
    top: int = BoundaryType.Transmissive

    def as_array(self):
        return (C.c_int * 4)(int(self.left), int(self.right), int(self.bottom), int(self.top))

    @staticmethod
    def of(bc) -> "BoundaryConfig":
        if isinstance(bc, BoundaryConfig):
            return bc
        b = list(bc)
        return BoundaryConfig(*b)


class CaseId(enum.IntEnum):  # head/test_cases.hpp:28-33 plus this build's configurations
    KelvinHelmholtz = 0
    ShockBubble = 1
    BrioWu = 2
    OrszagTang = 3
    OrszagTangUnit = 4
    ShockBubbleMHD = 5
    BrioWuCFL08 = 6


@dataclass
class CaseConfig:  # head/test_cases.hpp:38-55
    nx: int
    ny: int
    ng: int
    x_min: float
    x_max: float
    y_min: float
    y_max: float
    cfl: float
    t_end: float
    gamma: float
    bc: BoundaryConfig = field(default_factory=BoundaryConfig)

    @property
    def dx(self) -> float:
        return (self.x_max - self.x_min) / self.nx

    @property
    def dy(self) -> float:
        return (self.y_max - self.y_min) / self.ny

    @property
    def extent(self):
        return (self.x_min, self.x_max, self.y_min, self.y_max)


def get_n_case_config(case: int, n: int = 1) -> CaseConfig:
    """get_n_case_config (src/test_cases.cpp:275-282)."""
    out = (C.c_double * 14)()
    check(load().mhd_case_config(int(case), int(n), out), "mhd_case_config")
    v = list(out)
    return CaseConfig(int(v[0]), int(v[1]), int(v[2]), v[3], v[4], v[5], v[6], v[7], v[8], v[9],
                      BoundaryConfig(int(v[10]), int(v[11]), int(v[12]), int(v[13])))


def get_case_config(case: int) -> CaseConfig:
    return get_n_case_config(case, 1)


def initial_state_at(case: int, x: float, y: float) -> np.ndarray:
    """initial_state_at (src/test_cases.cpp:288-296)."""
    out = np.zeros(9)
    check(load().mhd_initial_state(int(case), float(x), float(y), out.ctypes.data_as(_lib._pd)), "mhd_initial_state")
    return out


def initialise(case: int, nx: int, ny: int, ng: int, extent) -> np.ndarray:
    """initialise_grid (src/init.cpp:34-43) into a host SoA array."""
    host = np.zeros((9, ny + 2 * ng, nx + 2 * ng))
    x0, x1, y0, y1 = extent
    check(load().mhd_initialise(int(case), nx, ny, ng, x0, x1, y0, y1, host.ctypes.data), "mhd_initialise")
    return host


def make_n_grid(case: int, n: int = 1) -> np.ndarray:
    """make_n_grid (src/init.cpp:58-61): the initial host state of a case."""
    cfg = get_n_case_config(case, n)
    return initialise(case, cfg.nx, cfg.ny, cfg.ng, cfg.extent)


class Grid2DGPU:
    """Device state (Grid2DGPU, head/gpu/grid_gpu.cuh:17-226): one padded slab of 9 planes."""

    def __init__(self, nx: int, ny: int, ng: int = 2, x_min: float = 0.0, x_max: float = 1.0,
                 y_min: float = 0.0, y_max: float = 1.0, dtype: int = F64):
        self.g = mhd_grid()
        check(load().mhd_grid_alloc(C.byref(self.g), nx, ny, ng, dtype, x_min, x_max, y_min, y_max), "mhd_grid_alloc")

    # accessors of the reference class
    nx = property(lambda s: s.g.nx)
    ny = property(lambda s: s.g.ny)
    ng = property(lambda s: s.g.ng)
    dtype = property(lambda s: s.g.dtype)
    total_nx = property(lambda s: s.g.nx + 2 * s.g.ng)
    total_ny = property(lambda s: s.g.ny + 2 * s.g.ng)
    dx = property(lambda s: (s.g.x_max - s.g.x_min) / s.g.nx)
    dy = property(lambda s: (s.g.y_max - s.g.y_min) / s.g.ny)

    @property
    def shape(self):
        return (9, self.total_ny, self.total_nx)

    def upload(self, host: np.ndarray) -> None:
        h = np.ascontiguousarray(host, dtype=np.float64)
        assert h.shape == self.shape, (h.shape, self.shape)
        check(load().mhd_grid_upload(C.byref(self.g), h.ctypes.data), "mhd_grid_upload")

    def download(self) -> np.ndarray:
        h = np.empty(self.shape)
        check(load().mhd_grid_download(C.byref(self.g), h.ctypes.data), "mhd_grid_download")
        return h

    def upload_from_aos(self, aos: np.ndarray) -> None:
        h = np.ascontiguousarray(aos, dtype=np.float64)
        assert h.size == 9 * self.total_nx * self.total_ny
        check(load().mhd_grid_upload_aos(C.byref(self.g), h.ctypes.data), "mhd_grid_upload_aos")

    def download_to_aos(self) -> np.ndarray:
        h = np.empty((self.total_ny * self.total_nx, 9))
        check(load().mhd_grid_download_aos(C.byref(self.g), h.ctypes.data), "mhd_grid_download_aos")
        return h

    def swap(self, other: "Grid2DGPU") -> None:
        check(load().mhd_grid_swap(C.byref(self.g), C.byref(other.g)), "mhd_grid_swap")

    def save(self, path: str, t: float = 0.0, ch: float = 0.0, steps: int = 0) -> None:
        """Binary state dump (mhd_state_save): the grid in its own precision, ghosts
        included, with the time, c_h and step count a resumed run needs."""
        meta = mhd_state_meta(float(t), float(ch), int(steps))
        check(load().mhd_state_save(C.byref(self.g), os.fsencode(path), C.byref(meta)), "mhd_state_save")

    def load_state(self, path: str) -> mhd_state_meta:
        """Reads a mhd_state_save file into this grid (same shape and precision);
        returns its (t, ch, steps)."""
        meta = mhd_state_meta()
        check(load().mhd_state_load(C.byref(self.g), os.fsencode(path), C.byref(meta)), "mhd_state_load")
        return meta

    def release(self) -> None:
        if getattr(self, "g", None) is not None and self.g.data:
            load().mhd_grid_free(C.byref(self.g))

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class GpuWorkspace:
    """Workspace (GpuWorkspace, head/gpu/solver_gpu.cuh:9-19) plus the per-run physics scalars."""

    def __init__(self):
        self.ptr = C.c_void_p()

    def _req(self) -> C.c_void_p:
        if not self.ptr:
            raise RuntimeError("workspace not initialised")
        return self.ptr

    def set_stream(self, stream_handle: int) -> None:
        check(load().mhd_workspace_set_stream(self._req(), C.c_void_p(stream_handle)), "mhd_workspace_set_stream")

    def set_limiter(self, limiter: int) -> None:
        check(load().mhd_set_limiter(self._req(), int(limiter)), "mhd_set_limiter")

    def set_cr(self, cr: float) -> None:
        check(load().mhd_set_cr(self._req(), float(cr)), "mhd_set_cr")

    def set_tma_wait_limit(self, ns: int) -> None:
        """Limit (ns) of each wait for a TMA-staged y-sweep box; 0 = the 2 s default."""
        check(load().mhd_set_tma_wait_limit(self._req(), int(ns)), "mhd_set_tma_wait_limit")

    def set_sweep_shape(self, xrpw: int = 0, yband: int = 0, ystage: int = 0) -> None:
        """Launch shape only: x-sweep work per warp (row segments of 128 * xrpw - 4
        cells; 0: the precision's default), y-sweep rows per warp band (0: the
        precision's default), y-sweep rows staged by TMA (1) or loaded per thread (0)."""
        check(load().mhd_set_sweep_shape(self._req(), int(xrpw), int(yband), int(ystage)), "mhd_set_sweep_shape")

    @property
    def ch(self) -> float:
        v = C.c_double()
        check(load().mhd_get_ch(self._req(), C.byref(v)), "mhd_get_ch")
        return v.value

    def run(self, U: Grid2DGPU, T: Grid2DGPU, cfl: float, t_end: float, max_steps: int, solver: int, bc,
            raise_on_stop: bool = True) -> mhd_run_info:
        """Device-resident driver loop (scripts/gpu/main_gpu.cu:208-264) as a CUDA graph."""
        info = mhd_run_info()
        rc = load().mhd_run(self._req(), C.byref(U.g), C.byref(T.g), float(cfl), float(t_end), int(max_steps),
                            int(solver), BoundaryConfig.of(bc).as_array(), C.byref(info))
        if raise_on_stop:
            check(rc, "mhd_run")
        return info

    def step_async(self, U: Grid2DGPU, T: Grid2DGPU, cfl: float, t_end: float, solver: int, bc) -> None:
        """One step of U (T holds the x-swept state), queued on the workspace
        stream with no host round trip: mhd_clock_start (U's CFL maximum, and
        from it dt and c_h, stay on the GPU), then the x-sweep U -> T and the
        y-sweep T -> U (mhd_sweep_clocked, step parity 0).  The same kernels and
        results as run(U, T, cfl, t_end, 1, ...), which instead waits for the
        step to read its clock; clock_read() gives dt, c_h and the status."""
        lib, ws = load(), self._req()
        bca = BoundaryConfig.of(bc).as_array()
        check(lib.mhd_clock_start(ws, C.byref(U.g), float(cfl), float(t_end)), "mhd_clock_start")
        check(lib.mhd_sweep_clocked(ws, C.byref(U.g), C.byref(T.g), int(solver), bca, 0, 0, 0, 0, 0),
              "mhd_sweep_clocked")
        check(lib.mhd_sweep_clocked(ws, C.byref(T.g), C.byref(U.g), int(solver), bca, 1, 0, 0, 0, 0),
              "mhd_sweep_clocked")

    def clock_read(self) -> mhd_run_info:
        """The device clock after the queued steps (synchronises the workspace stream)."""
        info = mhd_run_info()
        check(load().mhd_clock_read(self._req(), C.byref(info)), "mhd_clock_read")
        return info

    def profile_sweeps(self, U: Grid2DGPU, T: Grid2DGPU, cfl: float, t_end: float, solver: int, bc,
                       nrep: int) -> tuple[float, float]:
        """Mean x- and y-sweep kernel times (ms) over nrep device-clock steps (advances U)."""
        out = (C.c_float * 2)()
        check(load().mhd_profile_sweeps(self._req(), C.byref(U.g), C.byref(T.g), float(cfl), float(t_end),
                                        int(solver), BoundaryConfig.of(bc).as_array(), int(nrep), out),
              "mhd_profile_sweeps")
        return float(out[0]), float(out[1])

    def upload(self, grid: Grid2DGPU, host: np.ndarray) -> None:
        check(load().mhd_upload(self._req(), C.byref(grid.g), host.ctypes.data), "mhd_upload")

    def download(self, grid: Grid2DGPU, host: np.ndarray) -> None:
        check(load().mhd_download(self._req(), C.byref(grid.g), host.ctypes.data), "mhd_download")

    def upload_f32(self, grid: Grid2DGPU, host: np.ndarray) -> None:
        """FP32 host array (9, ny+2ng, nx+2ng) -> FP32 grid, asynchronous on the workspace stream."""
        assert host.dtype == np.float32 and host.flags.c_contiguous and host.shape == grid.shape
        check(load().mhd_upload_f32(self._req(), C.byref(grid.g), host.ctypes.data), "mhd_upload_f32")

    def download_f32(self, grid: Grid2DGPU, host: np.ndarray) -> None:
        assert host.dtype == np.float32 and host.flags.c_contiguous and host.shape == grid.shape
        check(load().mhd_download_f32(self._req(), C.byref(grid.g), host.ctypes.data), "mhd_download_f32")

    def synchronize(self) -> None:
        check(load().mhd_synchronize(self._req()), "mhd_synchronize")

    def diagnostics(self, grid: Grid2DGPU) -> np.ndarray:
        out = (C.c_double * 6)()
        check(load().mhd_diagnostics(self._req(), C.byref(grid.g), out), "mhd_diagnostics")
        return np.array(list(out))

    def destroy(self) -> None:
        if self.ptr:
            load().mhd_workspace_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def init_gpu_workspace(ws: GpuWorkspace, grid: Grid2DGPU) -> None:
    """init_gpu_workspace (src/gpu/solver_gpu.cu:549-566)."""
    ws.destroy()
    check(load().mhd_workspace_create(C.byref(grid.g), C.byref(ws.ptr)), "mhd_workspace_create")


def free_gpu_workspace(ws: GpuWorkspace) -> None:
    """free_gpu_workspace (src/gpu/solver_gpu.cu:568-573)."""
    ws.destroy()


def set_gpu_physics_gamma(ws: GpuWorkspace, gamma: float) -> None:
    """set_gpu_physics_gamma (src/gpu/solver_gpu.cu:536-539), per workspace."""
    check(load().mhd_set_gamma(ws._req(), float(gamma)), "mhd_set_gamma")


def set_gpu_physics_ch(ws: GpuWorkspace, ch: float) -> None:
    """set_gpu_physics_ch (src/gpu/solver_gpu.cu:541-544), per workspace."""
    check(load().mhd_set_ch(ws._req(), float(ch)), "mhd_set_ch")


def compute_dt_gpu(grid: Grid2DGPU, ws: GpuWorkspace, cfl: float) -> float:
    """compute_dt_gpu (src/gpu/solver_gpu.cu:578-605).

    Returns sys.float_info.max when the maximum wave speed is not positive,
    as the reference GPU path does; raises RuntimeError when the workspace does
    not match the grid (solver_gpu.cu:579-580)."""
    dt = C.c_double()
    rc = load().mhd_compute_dt(ws._req(), C.byref(grid.g), float(cfl), C.byref(dt))
    if rc == -3:
        return sys.float_info.max
    check(rc, "mhd_compute_dt")
    return dt.value


def advance_second_order_gpu(Uold: Grid2DGPU, Utmp: Grid2DGPU, Unew: Grid2DGPU, ws: GpuWorkspace, dt: float,
                             solver: int, bc) -> None:
    """advance_second_order_gpu (src/gpu/solver_gpu.cu:617-690)."""
    check(load().mhd_advance(ws._req(), C.byref(Uold.g), C.byref(Utmp.g), C.byref(Unew.g), float(dt), int(solver),
                             BoundaryConfig.of(bc).as_array()), "mhd_advance")


def apply_boundary_gpu(grid: Grid2DGPU, bc, ws: GpuWorkspace | None = None) -> None:
    """apply_boundary_gpu (src/gpu/boundary_gpu.cu:158-176), in place."""
    check(load().mhd_apply_boundary(ws._req() if ws is not None else None, C.byref(grid.g),
                                    BoundaryConfig.of(bc).as_array()), "mhd_apply_boundary")


def launch_count() -> int:
    return int(load().mhd_launch_count())
