"""FP64 parity at the benchmark's grid sizes, and FP32-bulk accuracy to t_end.

The FP64 GPU step against the CPU checkers on the configurations the benchmark
quotes, through the C ABI:
  * the reference's own CPU/OpenMP step (oracle/_ref/libmhdref.so, minmod -- the
    reference's only limiter; src/cpu/solver_cpu.cpp:327-440);
  * the oracle restatement (oracle/mhd_oracle.c, van Leer), itself pinned bit
    for bit to the reference build in minmod mode (tests/test_oracle.py).
The drop-in loop (compute_dt + advance_second_order, host dt and damping
factor) must be bit-exact.  The device-resident graph loop (mhd_run) computes
the psi damping factor with the device exp(), so it is held to a relative L1 of
1e-12 per conserved field.

Sizes: Orszag-Tang [0,1]^2 512^2 to t_end = 0.5 (1691 steps), 2048^2 for 20
steps and 4096^2 for 3 steps (HLLD); the Mach-10 shock-bubble 2048^2 for 20
steps (HLLC and HLLD, transmissive sides).  The CPU checkers use every host
core.
"""
import os
import sys

import numpy as np
import pytest

from helpers import device_loop, gpu_driver_loop, rel_l1, rel_linf
from mhd_gpu_acc_b200 import F32, get_n_case_config, initialise

pytestmark = pytest.mark.gpu

FP64_DEVICE_LOOP_RTOL = 1e-12
OT, SB = 4, 5  # CaseId.OrszagTangUnit, CaseId.ShockBubbleMhd
HLLC, HLLD = 1, 2
MINMOD, VANLEER = 0, 1
FIELDS = ("rho", "rhou", "rhov", "rhow", "Bx", "By", "Bz", "E", "psi")


@pytest.fixture(scope="module")
def cpu_oracle():
    from oracle.oracle import Oracle

    o = Oracle()
    o.set_threads(os.cpu_count() or 1)
    return o


@pytest.fixture(scope="module")
def cpu_ref():
    from oracle.oracle import REF_SO, Reference

    if not os.path.exists(REF_SO):
        pytest.fail("oracle/_ref/libmhdref.so was not built (run __graft_entry__.build() where the reference "
                    "checkout is present)")
    r = Reference()
    r.set_threads(os.cpu_count() or 1)
    return r


def _setup(case, n):
    cfg = get_n_case_config(case, 1)
    U0 = initialise(case, n, n, 2, cfg.extent)
    bc = (cfg.bc.left, cfg.bc.right, cfg.bc.bottom, cfg.bc.top)
    return cfg, U0, bc


def _check_device_loop(U0, n, cfg, solver, bc, limiter, steps, t_end, want, want_steps):
    got, info = device_loop(U0, n, n, 2, cfg.extent, cfg.gamma, cfg.cfl, solver, bc, limiter=limiter,
                            max_steps=steps, t_end=t_end)
    assert info.steps == want_steps
    err = rel_l1(got, want)
    assert err.max() <= FP64_DEVICE_LOOP_RTOL, dict(zip(FIELDS, err))


@pytest.fixture(scope="module")
def ot512_fp64(cpu_oracle):
    """Orszag-Tang 512^2, HLLD + van Leer, FP64 to t_end: the drop-in loop on the
    GPU and the oracle on the CPU."""
    cfg, U0, bc = _setup(OT, 512)
    gpu = gpu_driver_loop(U0, 512, 512, 2, cfg.extent, cfg.gamma, cfg.cfl, HLLD, bc, t_end=cfg.t_end,
                          limiter=VANLEER)
    orc = cpu_oracle.run(U0, 2, 1 / 512, 1 / 512, cfg.gamma, cfg.cfl, HLLD, VANLEER, bc, t_end=cfg.t_end)
    return cfg, U0, bc, gpu, orc


def test_ot512_fp64_to_t_end_bit_exact_vs_oracle(ot512_fp64):
    cfg, U0, bc, (U, t, steps, dts, ch), (rc, want, t_o, steps_o, ch_o, dts_o) = ot512_fp64
    assert rc == 0 and steps == steps_o > 1000 and t == t_o and abs(t - cfg.t_end) <= 1e-15
    np.testing.assert_array_equal(dts, dts_o)
    assert ch == ch_o
    np.testing.assert_array_equal(U, want)
    _check_device_loop(U0, 512, cfg, HLLD, bc, VANLEER, 0, cfg.t_end, want, steps_o)


def test_ot512_fp64_minmod_to_t_end_bit_exact_vs_reference(cpu_ref):
    cfg, U0, bc = _setup(OT, 512)
    rc, want, t_r, steps_r, ch_r, dts_r = cpu_ref.run(U0, 2, cfg.extent, cfg.gamma, cfg.cfl, HLLD, bc,
                                                      t_end=cfg.t_end)
    U, t, steps, dts, ch = gpu_driver_loop(U0, 512, 512, 2, cfg.extent, cfg.gamma, cfg.cfl, HLLD, bc,
                                           t_end=cfg.t_end, limiter=MINMOD)
    assert rc == 0 and steps == steps_r > 1000 and t == t_r and ch == ch_r
    np.testing.assert_array_equal(dts, dts_r)
    np.testing.assert_array_equal(U, want)


def test_ot512_fp32_bulk_to_t_end_per_field(ot512_fp64):
    """FP32-bulk against the FP64 step at t_end: the per-field relative L1 / Linf
    table (printed), density relative L1 <= 1e-5."""
    cfg, U0, bc, (U64, *_), _ = ot512_fp64
    U32, info = device_loop(U0, 512, 512, 2, cfg.extent, cfg.gamma, cfg.cfl, HLLD, bc, limiter=VANLEER,
                            t_end=cfg.t_end, dtype=F32)
    assert abs(info.t - cfg.t_end) <= 1e-12
    l1, linf = rel_l1(U32, U64), rel_linf(U32, U64)
    print("Orszag-Tang 512^2 to t = 0.5, FP32-bulk vs FP64 (relative L1 / Linf):", file=sys.stderr)
    for k, f in enumerate(FIELDS):
        print(f"  {f:5s} L1 {l1[k]:.3e}  Linf {linf[k]:.3e}", file=sys.stderr)
    assert l1[0] <= 1e-5
    assert np.isfinite(U32).all()


@pytest.mark.parametrize("n,steps", [(2048, 20), (4096, 3)])
def test_ot_large_fp64_bit_exact(cpu_oracle, cpu_ref, n, steps):
    cfg, U0, bc = _setup(OT, n)
    # van Leer: the oracle restatement
    rc, want, *_, dts_o = cpu_oracle.run(U0, 2, 1 / n, 1 / n, cfg.gamma, cfg.cfl, HLLD, VANLEER, bc,
                                         max_steps=steps, t_end=cfg.t_end)
    U, t, k, dts, ch = gpu_driver_loop(U0, n, n, 2, cfg.extent, cfg.gamma, cfg.cfl, HLLD, bc, max_steps=steps,
                                       t_end=cfg.t_end, limiter=VANLEER)
    assert rc == 0 and k == steps
    np.testing.assert_array_equal(dts, dts_o)
    np.testing.assert_array_equal(U, want)
    del U
    _check_device_loop(U0, n, cfg, HLLD, bc, VANLEER, steps, cfg.t_end, want, steps)
    del want
    # minmod: the reference's own CPU step
    rc, want, *_, dts_r = cpu_ref.run(U0, 2, cfg.extent, cfg.gamma, cfg.cfl, HLLD, bc, max_steps=steps,
                                      t_end=cfg.t_end)
    U, t, k, dts, ch = gpu_driver_loop(U0, n, n, 2, cfg.extent, cfg.gamma, cfg.cfl, HLLD, bc, max_steps=steps,
                                       t_end=cfg.t_end, limiter=MINMOD)
    assert rc == 0 and k == steps
    np.testing.assert_array_equal(dts, dts_r)
    np.testing.assert_array_equal(U, want)


@pytest.mark.parametrize("solver", [HLLC, HLLD])
def test_shock_bubble_mhd_2048_fp64_bit_exact_vs_reference(cpu_ref, solver):
    n, steps = 2048, 20
    cfg, U0, bc = _setup(SB, n)
    rc, want, *_, dts_r = cpu_ref.run(U0, 2, cfg.extent, cfg.gamma, cfg.cfl, solver, bc, max_steps=steps,
                                      t_end=cfg.t_end)
    U, t, k, dts, ch = gpu_driver_loop(U0, n, n, 2, cfg.extent, cfg.gamma, cfg.cfl, solver, bc, max_steps=steps,
                                       t_end=cfg.t_end, limiter=MINMOD)
    assert rc == 0 and k == steps
    np.testing.assert_array_equal(dts, dts_r)
    np.testing.assert_array_equal(U, want)
    del U
    _check_device_loop(U0, n, cfg, solver, bc, MINMOD, steps, cfg.t_end, want, steps)
