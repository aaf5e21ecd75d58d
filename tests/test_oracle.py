"""The oracle (oracle/mhd_oracle.c) pinned against the reference.

1. Against the committed golden fixtures, which were produced by the reference's
   own CPU code (tests/golden/make_golden.py): bit-exact final states, dt
   sequences, Riemann fluxes and boundary fills.
2. Against the reference build itself (oracle/_ref, present in the build
   container only) on further cases: ghost widths 3 and 4, random states.
"""
import numpy as np
import pytest

from helpers import hot_cell, inject_faults, sha
from mhd_gpu_acc_b200 import get_n_case_config, initialise


def _run_oracle(oracle, rec, limiter=0):
    U0 = initialise(rec["case"], rec["nx"], rec["ny"], rec["ng"], rec["extent"])
    assert sha(U0) == rec["sha_initial"], "initial condition changed"
    x0, x1, y0, y1 = rec["extent"]
    dx, dy = (x1 - x0) / rec["nx"], (y1 - y0) / rec["ny"]
    return oracle.run(U0, rec["ng"], dx, dy, rec["gamma"], rec["cfl"], rec["solver"], limiter, rec["bc"],
                      max_steps=rec["max_steps"], t_end=rec["t_end"], ch=0.0)


def test_oracle_matches_golden_runs(oracle, golden):
    runs, _ = golden
    for name, rec in runs.items():
        rc, U, t, steps, ch, dts = _run_oracle(oracle, rec)
        assert rc == rec["rc"] and steps == rec["steps"], name
        assert t == rec["t"] and ch == rec["ch"], name
        assert sha(dts) == rec["sha_dt"], name
        assert sha(U) == rec["sha_final"], name


def test_oracle_full_states(oracle, golden):
    runs, states = golden
    for key, ref_state in states.items():
        if not key.startswith("state_"):
            continue
        rc, U, *_ = _run_oracle(oracle, runs[key[len("state_"):]])
        np.testing.assert_array_equal(U, ref_state)


def test_oracle_riemann_kats(oracle, golden):
    _, st = golden
    UL, UR, F = st["riemann_UL"], st["riemann_UR"], st["riemann_F"]
    g, ch = float(st["riemann_gamma"]), float(st["riemann_ch"])
    for s in range(4):
        for d in range(2):
            for k in range(UL.shape[0]):
                got = oracle.riemann(UL[k], UR[k], d, s, ch, g)
                np.testing.assert_array_equal(got, F[s, d, k], err_msg=f"solver {s} dir {d} face {k}")


def test_oracle_boundary_kats(oracle, golden):
    _, st = golden
    for c, want in zip(st["bc_combos"], st["bc_out"]):
        np.testing.assert_array_equal(oracle.apply_boundary(st["bc_in"], 2, c), want, err_msg=str(c))


@pytest.mark.parametrize("ng", [3, 4])
def test_oracle_vs_reference_wide_ghosts(oracle, ref, ng):
    cfg = get_n_case_config(5, 1)
    nx, ny = 21, 13
    U0 = initialise(5, nx, ny, ng, cfg.extent)
    for solver, bc in [(2, (2, 1, 0, 0)), (1, (3, 2, 1, 3)), (3, (0, 0, 2, 2))]:
        a = ref.run(U0, ng, cfg.extent, cfg.gamma, cfg.cfl, solver, bc, max_steps=6, t_end=cfg.t_end)
        b = oracle.run(U0, ng, cfg.dx * 1.0 if False else (cfg.x_max - cfg.x_min) / nx,
                       (cfg.y_max - cfg.y_min) / ny, cfg.gamma, cfg.cfl, solver, 0, bc, max_steps=6,
                       t_end=cfg.t_end)
        assert a[0] == b[0] and a[3] == b[3]
        np.testing.assert_array_equal(a[1], b[1])


def test_oracle_vs_reference_random_states(oracle, ref):
    """Smooth random perturbations of the Orszag-Tang state, every solver."""
    rng = np.random.default_rng(7)
    cfg = get_n_case_config(4, 1)
    nx, ny, ng = 24, 20, 2
    U0 = initialise(4, nx, ny, ng, cfg.extent)
    U0 = U0 * (1.0 + 0.05 * rng.standard_normal(U0.shape))
    U0[8] = 0.01 * rng.standard_normal(U0[8].shape)  # non-zero psi
    dx, dy = (cfg.x_max - cfg.x_min) / nx, (cfg.y_max - cfg.y_min) / ny
    for solver in range(4):
        a = ref.run(U0, ng, cfg.extent, cfg.gamma, cfg.cfl, solver, (0, 0, 0, 0), max_steps=8, t_end=cfg.t_end, ch=0.3)
        b = oracle.run(U0, ng, dx, dy, cfg.gamma, cfg.cfl, solver, 0, (0, 0, 0, 0), max_steps=8, t_end=cfg.t_end,
                       ch=0.3)
        np.testing.assert_array_equal(a[1], b[1], err_msg=f"solver {solver}")
        assert a[4] == b[4]


@pytest.mark.parametrize("limiter", [0, 1])
def test_periodic_mass_and_the_ghost_psi_order(oracle, ref, limiter):
    """Periodic Orszag-Tang conserves mass to round-off when psi damping is off
    (c_r -> inf).  With damping, the reference damps psi in the interior AFTER
    filling the ghost cells (src/cpu/solver_cpu.cpp:434-439), so ghost psi is
    undamped, the two periodic boundary faces stop telescoping and mass drifts
    at ~1e-7 after 30 steps -- in the reference build (minmod) and, by design,
    identically in the oracle."""
    cfg = get_n_case_config(4, 1)
    nx = ny = 32
    U0 = initialise(4, nx, ny, 2, cfg.extent)
    args = (U0, 2, 1.0 / nx, 1.0 / ny, cfg.gamma, cfg.cfl, 2, limiter, (0, 0, 0, 0))
    m0 = U0[0, 2:-2, 2:-2].sum()
    rc, U, *_ = oracle.run(*args, max_steps=30, t_end=cfg.t_end, cr=1e300)
    assert rc == 0 and abs(U[0, 2:-2, 2:-2].sum() - m0) / m0 < 1e-14
    rc, Ud, *_ = oracle.run(*args, max_steps=30, t_end=cfg.t_end)
    drift = abs(Ud[0, 2:-2, 2:-2].sum() - m0) / m0
    assert 1e-9 < drift < 1e-5
    if limiter == 0:
        a = ref.run(U0, 2, cfg.extent, cfg.gamma, cfg.cfl, 2, (0, 0, 0, 0), max_steps=30, t_end=cfg.t_end)
        np.testing.assert_array_equal(a[1], Ud)


def test_van_leer_differs_from_minmod(oracle):
    cfg = get_n_case_config(4, 1)
    U0 = initialise(4, 32, 32, 2, cfg.extent)
    runs = [oracle.run(U0, 2, 1 / 32, 1 / 32, cfg.gamma, cfg.cfl, 2, lim, (0, 0, 0, 0), max_steps=10,
                       t_end=cfg.t_end)[1] for lim in (0, 1)]
    assert not np.array_equal(runs[0], runs[1])
    assert np.abs(runs[0] - runs[1]).max() < 0.05


def test_oracle_no_speed_error(oracle):
    """compute_dt on a state without any physical cell: the reference throws (rc -1)."""
    U = np.zeros((9, 8, 8))
    rc, dt, ch = oracle.compute_dt(U, 2, 0.1, 0.1, 5.0 / 3.0, 0.4, 0.0)
    assert rc == -1


@pytest.mark.parametrize("nx,ny,ng", [(64, 48, 2), (33, 17, 3)])
def test_reference_side_orszag_tang_unit_initial_state(ref, nx, ny, ng):
    """The [0,1]^2 Orszag-Tang state built by the reference build alone (its
    Grid2D cell centres and prim_to_cons) equals this library's initial data
    bit for bit, so the reference arm of the benchmark needs no other library."""
    cfg = get_n_case_config(4, 1)
    np.testing.assert_array_equal(ref.initialise_orszag_tang_unit(nx, ny, ng), initialise(4, nx, ny, ng, cfg.extent))


def test_reference_arm_loads_only_the_reference_build(ref):
    """bench.py's reference leg (the timed CPU baseline) maps no library of this
    repository's package: the initial state, the step and the timing all come
    from oracle/_ref."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys; sys.path.insert(0, %r); import bench\n"
            "secs, threads, err = bench.cpu_reference_run(32, 2, 1, None)\n"
            "assert err is None and len(secs) == 2, err\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'libmhdref.so' in maps\n"
            "assert 'libmhd_b200' not in maps, 'the repository library was loaded'\n"
            "assert 'mhd_gpu_acc_b200' not in sys.modules\n" % root)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr


def test_injected_faults_oracle_matches_reference(oracle, ref):
    """The reference's guards (positivity fallbacks, HLL fallback, revert of a
    non-finite update, src/cpu/solver_cpu.cpp:49-70, 391-392, 429-430; compute_dt
    skipping non-physical cells, :291-300) on a state with a NaN cell and a
    negative-pressure cell: the oracle follows the reference build bit for bit
    (the NaN stays in its cell), and both stop the loop the same way on a state
    without a physical cell (no speed) and on one whose first dt is under
    1e-8 t_end (scripts/cpu/main_cpu.cpp:205-216)."""
    cfg = get_n_case_config(4, 1)
    n, ng, bc = 32, 2, (0, 0, 0, 0)
    U0 = initialise(4, n, n, ng, cfg.extent)
    Ub = inject_faults(U0, ng)
    a = oracle.run(Ub, ng, 1 / n, 1 / n, cfg.gamma, cfg.cfl, 2, 0, bc, max_steps=6, t_end=cfg.t_end)
    b = ref.run(Ub, ng, cfg.extent, cfg.gamma, cfg.cfl, 2, bc, max_steps=6, t_end=cfg.t_end)
    assert a[0] == b[0] == 0 and a[3] == b[3] == 6 and a[2] == b[2] and a[4] == b[4]
    np.testing.assert_array_equal(a[5], b[5])
    np.testing.assert_array_equal(a[1], b[1])  # NaN positions included
    assert np.isnan(a[1]).sum() == 1
    clean = oracle.run(U0, ng, 1 / n, 1 / n, cfg.gamma, cfg.cfl, 2, 0, bc, max_steps=6, t_end=cfg.t_end)
    assert a[4] != clean[4]  # the negative-pressure cell changed the run
    for U, rc in ((np.zeros_like(U0), -1), (hot_cell(U0, ng), -3)):
        ra = oracle.run(U, ng, 1 / n, 1 / n, cfg.gamma, cfg.cfl, 2, 0, bc, max_steps=3, t_end=cfg.t_end)
        rb = ref.run(U, ng, cfg.extent, cfg.gamma, cfg.cfl, 2, bc, max_steps=3, t_end=cfg.t_end)
        assert ra[0] == rb[0] == rc and ra[3] == rb[3] == 0

