"""Binary state dump / load (mhd_state_save / mhd_state_load): checkpoint and
resume.  The reference has write-only CSV snapshots only
(scripts/cpu/main_cpu.cpp:36-91); a saved state reloads bit for bit, and a run
resumed from a mid-run save ends exactly where the uninterrupted run ends."""
import os

import numpy as np
import pytest

from helpers import gpu_driver_loop
from mhd_gpu_acc_b200 import F32, F64, Grid2DGPU, MhdError, get_n_case_config, initialise

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [F64, F32])
def test_state_round_trip(tmp_path, dtype):
    rng = np.random.default_rng(2)
    g = Grid2DGPU(37, 21, 3, -1.0, 2.0, 0.5, 1.5, dtype)
    host = rng.standard_normal(g.shape)
    g.upload(host)
    path = str(tmp_path / "s.mhd")
    g.save(path, t=0.125, ch=1.75, steps=42)
    assert not os.path.exists(path + ".tmp")
    assert os.path.getsize(path) == 128 + 9 * 27 * 43 * (8 if dtype == F64 else 4)
    h = Grid2DGPU(37, 21, 3, -1.0, 2.0, 0.5, 1.5, dtype)
    meta = h.load_state(path)
    assert (meta.t, meta.ch, meta.steps) == (0.125, 1.75, 42)
    np.testing.assert_array_equal(h.download(), g.download())
    with pytest.raises(MhdError):  # another shape
        Grid2DGPU(36, 21, 3, -1.0, 2.0, 0.5, 1.5, dtype).load_state(path)
    with pytest.raises(MhdError):  # another precision
        Grid2DGPU(37, 21, 3, -1.0, 2.0, 0.5, 1.5, F32 if dtype == F64 else F64).load_state(path)


def test_resume_from_a_saved_state_is_bit_exact(tmp_path):
    cfg = get_n_case_config(4, 1)
    n = 96
    U0 = initialise(4, n, n, 2, cfg.extent)
    full, t_full, steps_full, _, ch_full = gpu_driver_loop(U0, n, n, 2, cfg.extent, cfg.gamma, cfg.cfl, 2,
                                                           (0, 0, 0, 0), max_steps=20, t_end=cfg.t_end, limiter=1)
    half, t_half, steps_half, _, ch_half = gpu_driver_loop(U0, n, n, 2, cfg.extent, cfg.gamma, cfg.cfl, 2,
                                                           (0, 0, 0, 0), max_steps=12, t_end=cfg.t_end, limiter=1)
    g = Grid2DGPU(n, n, 2, *cfg.extent, F64)
    g.upload(half)
    path = str(tmp_path / "ckpt.mhd")
    g.save(path, t=t_half, ch=ch_half, steps=steps_half)
    r = Grid2DGPU(n, n, 2, *cfg.extent, F64)
    meta = r.load_state(path)
    rest, t_rest, steps_rest, _, ch_rest = gpu_driver_loop(r.download(), n, n, 2, cfg.extent, cfg.gamma, cfg.cfl, 2,
                                                           (0, 0, 0, 0), max_steps=20 - meta.steps,
                                                           t_end=cfg.t_end - meta.t, limiter=1, ch=meta.ch)
    assert meta.steps + steps_rest == steps_full and ch_rest == ch_full
    np.testing.assert_array_equal(rest, full)
