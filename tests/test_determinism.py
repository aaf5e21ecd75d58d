"""Race and out-of-bounds checks that need no sanitizer (compute-sanitizer is
not available on this GPU pool):

* determinism: the same run twice, in fresh workspaces, is bit-identical in
  FP64 and FP32-bulk (the only atomics are order-independent maxima and
  counters), on a ragged grid whose strips, bands and x segments end mid-way;
* NaN canaries: every byte of each allocation outside the logical
  (ny + 2 ng) x (nx + 2 ng) planes -- the row padding up to the pitch and the
  plane padding -- is set to NaN before the run; a kernel that read any of it
  would carry the NaN into the state, so the run must equal the same run on
  zero-padded allocations bit for bit.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import sha
from mhd_gpu_acc_b200 import F32, F64, GpuWorkspace, Grid2DGPU, get_n_case_config, init_gpu_workspace, initialise
from mhd_gpu_acc_b200 import set_gpu_physics_ch, set_gpu_physics_gamma

pytestmark = pytest.mark.gpu


class _Bytes:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (int(ptr), False), "version": 3}


def _fill_slab(g: Grid2DGPU, byte: int) -> None:
    import torch

    es = 8 if g.g.dtype == F64 else 4
    n = 9 * int(g.g.plane) * es
    torch.as_tensor(_Bytes(g.g.data, n), device="cuda").fill_(byte)
    torch.cuda.synchronize()


def _run(case, nx, ny, dtype, steps, canary, solver=2, limiter=1, shape=None):
    cfg = get_n_case_config(case, 1)
    U0 = initialise(case, nx, ny, 2, cfg.extent)
    U = Grid2DGPU(nx, ny, 2, *cfg.extent, dtype)
    T = Grid2DGPU(nx, ny, 2, *cfg.extent, dtype)
    for g in (U, T):
        _fill_slab(g, 0xFF if canary else 0x00)  # 0xFF bytes: a NaN in either precision
    U.upload(U0)
    ws = GpuWorkspace()
    init_gpu_workspace(ws, U)
    set_gpu_physics_gamma(ws, cfg.gamma)
    set_gpu_physics_ch(ws, 0.0)
    ws.set_limiter(limiter)
    if shape is not None:
        ws.set_sweep_shape(*shape)
    info = ws.run(U, T, cfg.cfl, cfg.t_end, steps, solver, cfg.bc)
    out = U.download()
    ws.destroy()
    return out, info


@pytest.mark.parametrize("dtype", [F64, F32])
@pytest.mark.parametrize("case,nx,ny", [(4, 203, 137), (5, 131, 77)])
def test_runs_are_deterministic(dtype, case, nx, ny):
    a, ia = _run(case, nx, ny, dtype, 30, False)
    b, ib = _run(case, nx, ny, dtype, 30, False)
    assert (ia.steps, ia.t, ia.ch) == (ib.steps, ib.t, ib.ch)
    assert sha(a) == sha(b)


@pytest.mark.parametrize("dtype", [F64, F32])
@pytest.mark.parametrize("shape", [None, (1, 7, 0), (8, 0, 1)])
def test_padding_is_never_read(dtype, shape):
    """Orszag-Tang 203 x 137 (rows padded from 207 to 224 / 256 elements):
    default launch shape, short x segments with odd y bands, and the
    TMA-staged y rows."""
    ref, iref = _run(4, 203, 137, dtype, 20, False, shape=shape)
    got, igot = _run(4, 203, 137, dtype, 20, True, shape=shape)
    assert np.isfinite(got).all()
    assert (igot.steps, igot.t) == (iref.steps, iref.t)
    np.testing.assert_array_equal(got, ref)
