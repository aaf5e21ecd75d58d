"""Discrete adjoint of the Orszag-Tang gradient problem (mhd_adjoint_* in
include/mhd_b200.h): J(a) = 1/2 sum (rho(t_N; a) - rho_target)^2 over the
interior, a = 16 Fourier amplitudes of the initial velocity and field."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, load
from .solver import F64, Limiter, RiemannSolver


def amplitudes(seed: int, sigma: float = 0.01) -> np.ndarray:
    """16 amplitudes a_k ~ N(0, sigma^2) from numpy's default generator."""
    return np.random.default_rng(seed).normal(0.0, sigma, 16)


class OTAdjoint:
    def __init__(self, n: int = 512, nsteps: int = 400, dtype: int = F64, limiter: int = Limiter.VANLEER,
                 gamma: float = 5.0 / 3.0, cfl: float = 0.4, cr: float = 0.18, checkpoint_every: int = 0,
                 solver: int = RiemannSolver.HLL):
        self.n, self.nsteps = n, nsteps
        self.ptr = C.c_void_p()
        check(load().mhd_adjoint_create(n, n, int(dtype), int(limiter), gamma, cfl, cr, nsteps, checkpoint_every,
                                        C.byref(self.ptr)), "mhd_adjoint_create")
        if int(solver) != int(RiemannSolver.HLL):
            check(load().mhd_adjoint_set_solver(self.ptr, int(solver)), "mhd_adjoint_set_solver")

    def set_target(self, rho: np.ndarray) -> None:
        r = np.ascontiguousarray(rho, dtype=np.float64)
        assert r.shape == (self.n, self.n)
        check(load().mhd_adjoint_set_target(self.ptr, r.ctypes.data), "mhd_adjoint_set_target")

    def forward(self, amp, want_rho: bool = False):
        a = np.ascontiguousarray(amp, dtype=np.float64)
        J = C.c_double()
        rho = np.empty((self.n, self.n)) if want_rho else None
        check(load().mhd_adjoint_forward(self.ptr, a.ctypes.data, C.byref(J),
                                         rho.ctypes.data if want_rho else None), "mhd_adjoint_forward")
        return (J.value, rho) if want_rho else J.value

    def gradient(self, amp):
        a = np.ascontiguousarray(amp, dtype=np.float64)
        J = C.c_double()
        g = np.zeros(16)
        check(load().mhd_adjoint_gradient(self.ptr, a.ctypes.data, C.byref(J), g.ctypes.data),
              "mhd_adjoint_gradient")
        return J.value, g

    def destroy(self) -> None:
        if self.ptr:
            load().mhd_adjoint_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
