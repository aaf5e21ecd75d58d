"""Batched instances against the single-grid device loop.

The batch runs the same per-tile device functions with each instance's own
parameters and clock, so every instance must equal -- bit for bit -- the same
problem advanced alone by mhd_run, in FP64 and in FP32-bulk, whatever launch
shape the autotuner picks."""
import ctypes as C

import numpy as np
import pytest

from mhd_gpu_acc_b200 import F32, F64, GpuWorkspace, Grid2DGPU, init_gpu_workspace, load, set_gpu_physics_gamma
from mhd_gpu_acc_b200.batch import SQRT_4PI, Batch, instance, orszag_tang_batch_spec


def test_batch_spec_is_deterministic():
    d1, b1, g1 = orszag_tang_batch_spec(3, n=256)
    d2, b2, g2 = orszag_tang_batch_spec(3, n=256)
    assert [d.nx for d in d1] == [d.nx for d in d2] and np.array_equal(b1, b2)
    sides = np.array([d.nx for d in d1])
    assert sides.min() >= 64 and sides.max() <= 1024 and np.all(sides % 32 == 0)
    assert np.all((b1 * SQRT_4PI >= 0.5) & (b1 * SQRT_4PI <= 1.5))
    assert set(np.unique(g1)) <= {5.0 / 3.0, 2.0}
    cfl = np.array([d.cfl for d in d1])
    assert cfl.min() >= 0.3 and cfl.max() <= 0.5


def _alone(desc, b0, gamma, dtype, steps, solver=2, limiter=1):
    ext = (desc.x_min, desc.x_max, desc.y_min, desc.y_max)
    U = Grid2DGPU(desc.nx, desc.ny, desc.ng, *ext, dtype)
    T = Grid2DGPU(desc.nx, desc.ny, desc.ng, *ext, dtype)
    assert load().mhd_initialise_orszag_tang(None, C.byref(U.g), b0, gamma, None) == 0
    ws = GpuWorkspace()
    init_gpu_workspace(ws, U)
    set_gpu_physics_gamma(ws, desc.gamma)
    ws.set_limiter(limiter)
    ws.set_cr(desc.cr)
    info = ws.run(U, T, desc.cfl, desc.t_end, steps, solver, tuple(desc.bc))
    out = U.download()
    ws.destroy()
    return out, info


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [F64, F32])
def test_batch_equals_single_grid_runs(dtype):
    descs = [instance(40, 40, 5 / 3, 0.4, 0.5), instance(96, 64, 2.0, 0.3, 0.5, bc=(1, 1, 2, 2)),
             instance(33, 70, 5 / 3, 0.45, 0.5, bc=(0, 0, 1, 1)), instance(128, 128, 2.0, 0.35, 0.02)]
    b0 = [1.0 / SQRT_4PI, 0.7 / SQRT_4PI, 1.3 / SQRT_4PI, 1.0 / SQRT_4PI]
    gam = [d.gamma for d in descs]
    batch = Batch(descs, dtype=dtype)
    for i in range(len(descs)):
        batch.init_orszag_tang(i, b0[i], gam[i])
    infos = batch.run(25)
    for i, d in enumerate(descs):
        want, info = _alone(d, b0[i], gam[i], dtype, 25)
        got = batch.download(i)
        assert infos[i].steps == info.steps, i
        if dtype == F64:  # --fmad=false code: identical in every kernel that inlines it
            assert infos[i].t == info.t, i
            np.testing.assert_array_equal(got, want, err_msg=f"instance {i}")
        else:  # FP32 code may contract into FMAs differently inside the batch kernels
            assert abs(infos[i].t - info.t) <= 1e-6 * info.t, i
            I = (slice(None), slice(2, -2), slice(2, -2))
            num = np.abs(got[I] - want[I]).reshape(9, -1).sum(1)
            den = np.maximum(np.abs(want[I]).reshape(9, -1).sum(1), 1e-300)
            assert np.all(num / den <= 1e-4), (i, num / den)  # last-bit differences grown over 25 steps
    # the last instance has a short t_end: it stopped there, the others ran 25 steps
    assert infos[3].t == 0.02 and infos[3].steps < 25 and infos[0].steps == 25
    batch.destroy()


@pytest.mark.gpu
def test_tuning_changes_speed_not_results():
    # the launch shape moves work between warps and CTAs but no cell's arithmetic
    descs, b0, gam = orszag_tang_batch_spec(11, n=12)
    runs = []
    for tuning in [(8, 64), (2, 16), (16, 128)]:
        batch = Batch(descs, dtype=F32)
        batch.set_tuning(*tuning)
        for i in range(len(descs)):
            batch.init_orszag_tang(i, b0[i], gam[i])
        batch.run(6)
        runs.append([batch.download(i) for i in range(len(descs))])
        batch.destroy()
    for other in runs[1:]:
        for a, b in zip(runs[0], other):
            np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
def test_autotuner_picks_a_valid_shape():
    descs, b0, gam = orszag_tang_batch_spec(5, n=16)
    batch = Batch(descs, dtype=F32)
    for i in range(len(descs)):
        batch.init_orszag_tang(i, b0[i], gam[i])
    t = batch.tune(2)
    per_sm = Batch.tune_candidates(2)
    import torch

    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    assert t.xrpw in Batch.tune_candidates(0) and t.yseg in Batch.tune_candidates(1)
    assert t.ctas_x in [c * nsm for c in per_sm] and t.ctas_y in [c * nsm for c in per_sm]
    got = batch.get_tuning()
    assert (got.xrpw, got.yseg) == (t.xrpw, t.yseg)
    info = batch.run(4)
    assert all(i.steps == 4 for i in info)
    batch.destroy()


@pytest.mark.gpu
def test_256_instance_batch_per_instance_error_vs_fp64():
    """The batch configuration: 256 Orszag-Tang instances (sides U{64..1024},
    B0 ~ U[0.5, 1.5]/sqrt(4 pi), gamma in {5/3, 2}, CFL ~ U[0.3, 0.5]; seed 0),
    HLLD + van Leer, autotuned FP32-bulk launch shapes: after 40 steps every
    instance's density relative L1 against the same batch in FP64 is <= 1e-4."""
    descs, b0, gam = orszag_tang_batch_spec(0, n=256, t_end=5.0)

    def make(dtype):
        b = Batch(descs, dtype=dtype, solver=2, limiter=1)
        for i in range(len(descs)):
            b.init_orszag_tang(i, b0[i], gam[i])
        return b

    b32 = make(F32)
    b32.tune(1)
    for i in range(len(descs)):  # the tuner advanced the states: start again
        b32.init_orszag_tang(i, b0[i], gam[i])
    i32 = b32.run(40)
    b64 = make(F64)
    i64 = b64.run(40)
    errs = []
    for i in range(len(descs)):
        assert i32[i].steps == i64[i].steps == 40, i
        r32, r64 = b32.download(i)[0, 2:-2, 2:-2], b64.download(i)[0, 2:-2, 2:-2]
        errs.append(np.abs(r32 - r64).sum() / np.abs(r64).sum())
    b32.destroy()
    b64.destroy()
    errs = np.array(errs)
    print(f"256 instances x 40 steps: rho rel L1 FP32-bulk vs FP64 median {np.median(errs):.2e}, "
          f"max {errs.max():.2e}")
    assert errs.max() <= 1e-4
