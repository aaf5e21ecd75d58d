"""C-ABI library checks that need no GPU: it loads, exports every declared
entry point, and its host-side functions (case configurations, initial data,
argument validation) behave like the reference's."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from helpers import sha
from mhd_gpu_acc_b200 import CaseId, get_n_case_config, initial_state_at, initialise, make_n_grid
from mhd_gpu_acc_b200._lib import PROTOTYPES, mhd_grid

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            src = open(os.path.join(inc, fn)).read()
            names |= set(re.findall(r"\b(mhd_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol(lib):
    decl = declared_symbols()
    assert len(decl) >= 25
    for name in decl:
        assert hasattr(lib, name), name
    assert decl == set(PROTOTYPES), decl ^ set(PROTOTYPES)


def test_version_and_error_string(lib):
    assert b"sm_100a" in lib.mhd_version()
    g = mhd_grid()
    assert lib.mhd_grid_alloc(C.byref(g), 10, 10, 1, 0, 0.0, 1.0, 0.0, 1.0) == -1  # ng < 2: no CUDA call
    assert b"bad sizes" in lib.mhd_last_error()
    assert lib.mhd_grid_alloc(C.byref(g), 10, 10, 2, 7, 0.0, 1.0, 0.0, 1.0) == -1
    assert lib.mhd_case_config(99, 1, (C.c_double * 14)()) == -1


def test_case_configs_match_reference(ref):
    for case in range(4):
        cfg = get_n_case_config(case, 3)
        want = ref.case_config(case, 3)
        got = [cfg.nx, cfg.ny, cfg.ng, cfg.x_min, cfg.x_max, cfg.y_min, cfg.y_max, cfg.cfl, cfg.t_end, cfg.gamma,
               cfg.bc.left, cfg.bc.right, cfg.bc.bottom, cfg.bc.top]
        np.testing.assert_array_equal(np.array(got, dtype=float), want)


@pytest.mark.parametrize("case", [0, 1, 2, 3])
def test_initial_states_match_reference(ref, case):
    cfg = get_n_case_config(case, 1)
    host = make_n_grid(case, 1)
    rng = np.random.default_rng(case)
    for _ in range(400):
        j = int(rng.integers(0, host.shape[1])); i = int(rng.integers(0, host.shape[2]))
        x = cfg.x_min + ((i - cfg.ng) + 0.5) * cfg.dx
        y = cfg.y_min + ((j - cfg.ng) + 0.5) * cfg.dy
        np.testing.assert_array_equal(host[:, j, i], ref.initial_state(case, x, y))
        np.testing.assert_array_equal(initial_state_at(case, x, y), host[:, j, i])


def test_initial_states_match_golden(golden):
    runs, _ = golden
    for name, rec in runs.items():
        U0 = initialise(rec["case"], rec["nx"], rec["ny"], rec["ng"], rec["extent"])
        assert sha(U0) == rec["sha_initial"], name


def test_baseline_case_definitions():
    cfg = get_n_case_config(CaseId.OrszagTangUnit, 8)
    assert (cfg.nx, cfg.ny, cfg.gamma, cfg.cfl, cfg.t_end) == (4096, 4096, 5.0 / 3.0, 0.4, 0.5)
    U = initialise(CaseId.OrszagTangUnit, 16, 16, 2, cfg.extent)
    assert np.allclose(U[0], 25.0 / (36.0 * np.pi))
    p = (5 / 3 - 1) * (U[7] - 0.5 * (U[1] ** 2 + U[2] ** 2) / U[0] - 0.5 * (U[4] ** 2 + U[5] ** 2))
    assert np.allclose(p, 5.0 / (12.0 * np.pi))
    bw = get_n_case_config(CaseId.BrioWuCFL08, 1)
    assert (bw.nx, bw.ny, bw.cfl, bw.t_end) == (800, 4, 0.8, 0.1)
    assert (bw.bc.left, bw.bc.right, bw.bc.bottom, bw.bc.top) == (1, 1, 1, 1)
    sb = get_n_case_config(CaseId.ShockBubbleMHD, 8)
    assert (sb.nx, sb.ny, sb.t_end) == (2048, 2048, 0.06)
    S = initialise(CaseId.ShockBubbleMHD, 64, 64, 2, sb.extent)
    # Rankine-Hugoniot density jump for Mach 10, gamma 5/3, and the rho = 10 bubble
    g, M = 5.0 / 3.0, 10.0
    assert np.isclose(S[0, 40, 5], (g + 1) * M * M / ((g - 1) * M * M + 2))
    assert np.isclose(S[0, 2 + 32, 2 + 51], 10.0)
    assert np.allclose(S[5], 2.0 / np.sqrt(4 * np.pi))


def test_batch_tune_candidates_exported():
    """The autotuner's candidate lists come from the library itself (host-only
    call), so tests and callers cannot drift from what mhd_batch_tune tries."""
    from mhd_gpu_acc_b200.batch import Batch

    assert Batch.tune_candidates(0) == [2, 4, 8, 16]
    assert Batch.tune_candidates(1) == [16, 24, 32, 48, 64, 128]
    assert Batch.tune_candidates(2) == [2, 3, 4]
    from mhd_gpu_acc_b200 import load

    assert load().mhd_batch_tune_candidates(7, None, 0) < 0


def test_state_file_header_checks_need_no_gpu(tmp_path, lib):
    """mhd_state_load rejects a file that is not a state file, or one written
    for another shape or precision, from its 128-byte header alone -- before
    any device copy (so this runs without a GPU; the grid's data pointer is a
    host stand-in that must never be dereferenced)."""
    import struct

    from mhd_gpu_acc_b200._lib import mhd_state_meta

    g = mhd_grid()
    stand_in = C.create_string_buffer(16)
    g.data = C.cast(stand_in, C.c_void_p)
    g.nx, g.ny, g.ng, g.dtype = 8, 6, 2, 0
    g.pitch, g.plane = 32, 32 * 10
    g.x_min, g.x_max, g.y_min, g.y_max = 0.0, 1.0, 0.0, 1.0
    bad = tmp_path / "bad.mhd"
    bad.write_bytes(b"not a state file" * 10)
    meta = mhd_state_meta()
    assert lib.mhd_state_load(C.byref(g), str(bad).encode(), C.byref(meta)) == -1
    assert b"not a state file" in lib.mhd_last_error()
    other = tmp_path / "other.mhd"
    header = b"MHDB200S" + struct.pack("<II3i", 1, 0, 9, 6, 2) + bytes(128 - 28)
    other.write_bytes(header)
    assert lib.mhd_state_load(C.byref(g), str(other).encode(), C.byref(meta)) == -1
    assert b"differs" in lib.mhd_last_error()
    assert lib.mhd_state_load(C.byref(g), str(tmp_path / "missing.mhd").encode(), None) == -1
