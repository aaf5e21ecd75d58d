"""Batched instances: many independent MHD problems of uneven size advanced by
one persistent launch per sweep phase and a CUDA-graph step loop (mhd_batch_*
in include/mhd_b200.h)."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import check, load, mhd_batch_tuning, mhd_grid, mhd_instance_desc, mhd_run_info
from .solver import F32

SQRT_4PI = math.sqrt(4.0 * math.pi)


def instance(nx, ny, gamma, cfl, t_end, bc=(0, 0, 0, 0), extent=(0.0, 1.0, 0.0, 1.0), ng=2, cr=0.18):
    d = mhd_instance_desc()
    d.nx, d.ny, d.ng = int(nx), int(ny), int(ng)
    for k in range(4):
        d.bc[k] = int(bc[k])
    d.x_min, d.x_max, d.y_min, d.y_max = (float(v) for v in extent)
    d.gamma, d.cfl, d.cr, d.t_end = float(gamma), float(cfl), float(cr), float(t_end)
    return d


def orszag_tang_batch_spec(seed: int, n: int = 256, t_end: float = 0.5):
    """The batched Orszag-Tang configuration: sides uniform over {64, 96, ..., 1024},
    B0 ~ U[0.5, 1.5]/sqrt(4 pi), gamma in {5/3, 2}, CFL ~ U[0.3, 0.5], drawn
    from numpy's default generator with `seed`.  Returns (descs, b0s, gammas)."""
    rng = np.random.default_rng(seed)
    sides = rng.choice(np.arange(64, 1025, 32), size=n)
    b0 = rng.uniform(0.5, 1.5, size=n) / SQRT_4PI
    gam = rng.choice([5.0 / 3.0, 2.0], size=n)
    cfl = rng.uniform(0.3, 0.5, size=n)
    descs = [instance(s, s, g, c, t_end) for s, g, c in zip(sides, gam, cfl)]
    return descs, b0, gam


def lpt_partition(weights, parts: int) -> list[list[int]]:
    """Longest-processing-time-first split of independent instances over `parts`
    GPUs: instances in decreasing weight (cells; ties by index) go one by one to
    the part with the least weight so far (lowest part on ties).  Deterministic,
    so every rank computes the same plan without communication; each part's
    index list is returned sorted.  The heaviest part exceeds the lightest by at
    most the largest single weight."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    w = [float(x) for x in weights]
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    load = [0.0] * parts
    out: list[list[int]] = [[] for _ in range(parts)]
    for i in order:
        p = min(range(parts), key=lambda q: (load[q], q))
        out[p].append(i)
        load[p] += w[i]
    return [sorted(s) for s in out]


class Batch:
    def __init__(self, descs, dtype=F32, solver=2, limiter=1):
        self.n = len(descs)
        arr = (mhd_instance_desc * self.n)(*descs)
        self.ptr = C.c_void_p()
        check(load().mhd_batch_create(arr, self.n, int(dtype), int(solver), int(limiter), C.byref(self.ptr)),
              "mhd_batch_create")
        self.descs = list(descs)

    def grid(self, i: int) -> mhd_grid:
        g = mhd_grid()
        check(load().mhd_batch_grid(self.ptr, int(i), C.byref(g)), "mhd_batch_grid")
        return g

    @property
    def cells(self) -> int:
        v = C.c_longlong()
        check(load().mhd_batch_cells(self.ptr, C.byref(v)), "mhd_batch_cells")
        return int(v.value)

    def set_stream(self, handle: int) -> None:
        check(load().mhd_batch_set_stream(self.ptr, C.c_void_p(handle)), "mhd_batch_set_stream")

    def upload(self, i: int, host: np.ndarray) -> None:
        g = self.grid(i)
        h = np.ascontiguousarray(host, dtype=np.float64)
        check(load().mhd_grid_upload(C.byref(g), h.ctypes.data), "mhd_grid_upload")

    def download(self, i: int) -> np.ndarray:
        g = self.grid(i)
        h = np.empty((9, g.ny + 2 * g.ng, g.nx + 2 * g.ng))
        check(load().mhd_grid_download(C.byref(g), h.ctypes.data), "mhd_grid_download")
        return h

    def init_orszag_tang(self, i: int, b0: float, gamma: float, amp=None) -> None:
        g = self.grid(i)
        a = None if amp is None else np.ascontiguousarray(amp, dtype=np.float64)
        check(load().mhd_initialise_orszag_tang(None, C.byref(g), float(b0), float(gamma),
                                                None if a is None else a.ctypes.data), "mhd_initialise_orszag_tang")

    def run(self, max_steps: int, raise_on_stop: bool = True):
        info = (mhd_run_info * self.n)()
        rc = load().mhd_batch_run(self.ptr, int(max_steps), info)
        if raise_on_stop:
            check(rc, "mhd_batch_run")
        return list(info)

    def tune(self, reps: int = 3) -> mhd_batch_tuning:
        t = mhd_batch_tuning()
        check(load().mhd_batch_tune(self.ptr, int(reps), C.byref(t)), "mhd_batch_tune")
        return t

    @staticmethod
    def tune_candidates(which: int) -> list[int]:
        """The autotuner's candidates: 0 x work per warp (xrpw), 1 y segment lengths,
        2 CTAs per SM."""
        n = load().mhd_batch_tune_candidates(int(which), None, 0)
        check(min(n, 0), "mhd_batch_tune_candidates")
        out = (C.c_int * n)()
        load().mhd_batch_tune_candidates(int(which), C.cast(out, C.POINTER(C.c_int)), n)
        return list(out)

    def get_tuning(self) -> mhd_batch_tuning:
        t = mhd_batch_tuning()
        check(load().mhd_batch_get_tuning(self.ptr, C.byref(t)), "mhd_batch_get_tuning")
        return t

    def set_tuning(self, xrpw: int, yseg: int, ctas_x: int = 0, ctas_y: int = 0) -> None:
        t = mhd_batch_tuning(int(xrpw), int(yseg), int(ctas_x), int(ctas_y))
        check(load().mhd_batch_set_tuning(self.ptr, C.byref(t)), "mhd_batch_set_tuning")

    def destroy(self) -> None:
        if self.ptr:
            load().mhd_batch_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
