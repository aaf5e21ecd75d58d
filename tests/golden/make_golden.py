"""Generate the golden fixtures in this directory from the reference itself.

Runs the reference's own CPU/OpenMP step, compiled from its unmodified sources
into oracle/_ref/libmhdref.so (oracle/Makefile), on initial data produced by
this package's initial-condition functions (which the tests check bit for bit
against the reference's initial_state_at for the reference's own cases).

Outputs (committed):
  golden.json  -- per run: configuration, SHA-256 of the initial and final
                  states (float64 C-order (9, ny+2ng, nx+2ng), ghosts
                  included), SHA-256 of the dt sequence, t, steps, ch and the
                  per-field sums of the final interior
  states.npz   -- a few small final states, Riemann-flux known answers and
                  apply_boundary known answers

Usage (needs the reference checkout, i.e. only in the build container):
    MHD_REFERENCE_ROOT=<reference checkout> make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mhd_gpu_acc_b200 import CaseId, get_n_case_config, initialise  # noqa: E402
from oracle.oracle import Reference  # noqa: E402

P, T, R, D = 0, 1, 2, 3


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


# name: (case, nx, ny, extent or None (= case extent), solver, bc or None, max_steps, t_end or None)
RUNS = {
    # the Brio-Wu configuration of the benchmark (800x4, CFL 0.8, transmissive) to t_end
    "bw_cfl08_hlld_tend": (CaseId.BrioWuCFL08, 800, 4, None, 2, None, 0, None),
    # the reference's own cases (reduced grids where the reference's is large)
    "bw_ref_hll_100": (CaseId.BrioWu, 800, 4, None, 0, None, 100, None),
    "bw_ref_hllc_100": (CaseId.BrioWu, 800, 4, None, 1, None, 100, None),
    "bw_ref_hlld_100": (CaseId.BrioWu, 800, 4, None, 2, None, 100, None),
    "bw_ref_force_100": (CaseId.BrioWu, 800, 4, None, 3, None, 100, None),
    "ot_ref_48_hlld_25": (CaseId.OrszagTang, 48, 48, None, 2, None, 25, None),
    "kh_ref_40x80_hllc_12": (CaseId.KelvinHelmholtz, 40, 80, None, 1, None, 12, None),
    "sb_ref_100x40_hllc_15": (CaseId.ShockBubble, 100, 40, None, 1, None, 15, None),
    # the Orszag-Tang [0,1]^2 configuration, every solver (minmod: the reference's limiter)
    "ot_unit_32_hll_20": (CaseId.OrszagTangUnit, 32, 32, None, 0, None, 20, None),
    "ot_unit_32_hllc_20": (CaseId.OrszagTangUnit, 32, 32, None, 1, None, 20, None),
    "ot_unit_32_hlld_20": (CaseId.OrszagTangUnit, 32, 32, None, 2, None, 20, None),
    "ot_unit_32_force_20": (CaseId.OrszagTangUnit, 32, 32, None, 3, None, 20, None),
    "ot_unit_64_hlld_60": (CaseId.OrszagTangUnit, 64, 64, None, 2, None, 60, None),
    # odd sizes and every boundary type, incl. mixed and Dirichlet sides
    "sbmhd_37x23_hlld_refl": (CaseId.ShockBubbleMHD, 37, 23, None, 2, (R, R, R, R), 12, None),
    "sbmhd_37x23_hllc_mixed": (CaseId.ShockBubbleMHD, 37, 23, None, 1, (D, T, R, D), 12, None),
    "sbmhd_37x23_hll_pmix": (CaseId.ShockBubbleMHD, 37, 23, None, 0, (P, P, R, T), 12, None),
    "ot_unit_17x5_force_dir": (CaseId.OrszagTangUnit, 17, 5, None, 3, (D, D, P, P), 9, None),
    "sbmhd_64_hlld_tend": (CaseId.ShockBubbleMHD, 64, 64, None, 2, None, 0, None),
}

FULL_STATES = ["ot_unit_32_hlld_20", "sbmhd_37x23_hllc_mixed", "ot_unit_17x5_force_dir"]


def run_one(ref: Reference, name, spec):
    case, nx, ny, extent, solver, bc, max_steps, t_end = spec
    cfg = get_n_case_config(case, 1)
    extent = extent or cfg.extent
    bc = list(bc) if bc is not None else [cfg.bc.left, cfg.bc.right, cfg.bc.bottom, cfg.bc.top]
    t_end = cfg.t_end if t_end is None else t_end
    ng = 2
    U0 = initialise(case, nx, ny, ng, extent)
    rc, U, t, steps, ch, dts = ref.run(U0, ng, extent, cfg.gamma, cfg.cfl, solver, bc, max_steps=max_steps,
                                       t_end=t_end, ch=0.0)
    inner = U[:, ng:ng + ny, ng:ng + nx]
    rec = dict(case=int(case), nx=nx, ny=ny, ng=ng, extent=list(extent), gamma=cfg.gamma, cfl=cfg.cfl,
               solver=solver, bc=[int(b) for b in bc], max_steps=max_steps, t_end=t_end, rc=rc, t=t, steps=steps,
               ch=ch, sha_initial=sha(U0), sha_final=sha(U), sha_dt=sha(dts), dt_first=float(dts[0]),
               dt_last=float(dts[-1]), field_sums=[float(v) for v in inner.reshape(9, -1).sum(axis=1)])
    return rec, U


def riemann_kats(ref: Reference, rng):
    """Single-face fluxes on random physical states (and a few unphysical ones)."""
    n = 24
    UL = np.zeros((n, 9)); UR = np.zeros((n, 9))
    gamma = 5.0 / 3.0
    for k in range(n):
        for side in (UL, UR):
            rho = rng.uniform(0.1, 3.0); u, v, w = rng.normal(0, 1.0, 3)
            bx, by, bz = rng.normal(0, 0.8, 3); p = rng.uniform(0.05, 2.0); psi = rng.normal(0, 0.1)
            ke = 0.5 * rho * (u * u + v * v + w * w); b2 = bx * bx + by * by + bz * bz
            side[k] = [rho, rho * u, rho * v, rho * w, bx, by, bz, p / (gamma - 1) + ke + 0.5 * b2, psi]
    UL[3, 7] = 0.01  # negative pressure on the left
    UR[5, 0] = -0.2  # negative density on the right
    UR[7] = UL[7]    # identical states
    F = np.zeros((4, 2, n, 9))
    for s in range(4):
        for d in range(2):
            for k in range(n):
                F[s, d, k] = ref.riemann(UL[k], UR[k], d, s, 1.7, gamma)
    return UL, UR, F, gamma, 1.7


def boundary_kats(ref: Reference, rng):
    nx, ny, ng = 7, 5, 2
    combos = np.array([[P, P, P, P], [T, T, T, T], [R, R, R, R], [D, D, D, D], [R, T, P, D], [D, R, T, P],
                       [P, D, D, R]], dtype=np.int32)
    U = rng.normal(0, 1, (9, ny + 2 * ng, nx + 2 * ng))
    out = np.stack([ref.apply_boundary(U, ng, c) for c in combos])
    return U, combos, out


def main() -> int:
    ref = Reference()
    ref.set_threads(min(8, os.cpu_count() or 1))
    golden, states = {}, {}
    for name, spec in RUNS.items():
        rec, U = run_one(ref, name, spec)
        golden[name] = rec
        if name in FULL_STATES:
            states["state_" + name] = U
        print(f"{name:28s} rc={rec['rc']} steps={rec['steps']:4d} t={rec['t']:.6g}")
    rng = np.random.default_rng(20240611)
    UL, UR, F, g, ch = riemann_kats(ref, rng)
    states.update(riemann_UL=UL, riemann_UR=UR, riemann_F=F, riemann_gamma=np.array(g), riemann_ch=np.array(ch))
    U, combos, out = boundary_kats(ref, rng)
    states.update(bc_in=U, bc_combos=combos, bc_out=out)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)
    np.savez_compressed(os.path.join(HERE, "states.npz"), **states)
    return 0


if __name__ == "__main__":
    sys.exit(main())
