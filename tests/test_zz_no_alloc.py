"""mhd_advance_noalloc -- the split step for callers that cannot allocate device
memory (an application whose own pool allocator owns all device memory, or a
loop that cannot absorb an allocation's synchronisation).  Its intermediate
state lives in a fixed 32 MiB array inside the library instead of a workspace.

Called through the C ABI and compared with mhd_advance (the workspace path) on
two steps in a row; both run the same kernels, so the tolerance is exact
equality, as for the other FP64 parity tests.  This file is collected last so
that a run stopping at the first failure has run every other test already; it
also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from mhd_gpu_acc_b200 import (
    F32,
    F64,
    GpuWorkspace,
    Grid2DGPU,
    MhdError,
    advance_second_order_gpu,
    compute_dt_gpu,
    get_n_case_config,
    init_gpu_workspace,
    initialise,
    load,
    set_gpu_physics_ch,
    set_gpu_physics_gamma,
)
from mhd_gpu_acc_b200.solver import BoundaryConfig

pytestmark = pytest.mark.gpu


def _noalloc(Uold, Unew, gamma, ch, cr, dt, solver, limiter, bc):
    return load().mhd_advance_noalloc(C.byref(Uold.g), C.byref(Unew.g), gamma, ch, cr, dt, solver, limiter,
                                      BoundaryConfig.of(bc).as_array(), None)


@pytest.mark.parametrize("dtype", [F64, F32])
@pytest.mark.parametrize("case,nx,ny,solver,limiter,bc", [
    (4, 48, 40, 2, 1, (0, 0, 0, 0)),   # Orszag-Tang, HLLD, van Leer, periodic
    (5, 37, 23, 1, 0, (3, 1, 2, 3)),   # shock-bubble, HLLC, Dirichlet/transmissive/reflecting
])
def test_noalloc_matches_workspace_step_twice(dtype, case, nx, ny, solver, limiter, bc):
    cfg = get_n_case_config(case, 1)
    U0 = initialise(case, nx, ny, 2, cfg.extent)
    grids = [Grid2DGPU(nx, ny, 2, *cfg.extent, dtype) for _ in range(5)]
    Uold, Utmp, Unew, A, B = grids
    for g in grids:
        g.upload(U0)
    ws = GpuWorkspace()
    init_gpu_workspace(ws, Uold)
    set_gpu_physics_gamma(ws, cfg.gamma)
    set_gpu_physics_ch(ws, 0.0)
    ws.set_limiter(limiter)
    for call in range(2):
        dt = compute_dt_gpu(Uold, ws, cfg.cfl)
        ch = ws.ch
        advance_second_order_gpu(Uold, Utmp, Unew, ws, dt, solver, bc)
        assert _noalloc(A, B, cfg.gamma, ch, 0.18, dt, solver, limiter, bc) == 0, load().mhd_last_error()
        want, got = Unew.download(), B.download()
        np.testing.assert_array_equal(got, want, err_msg=f"call {call}")
        Uold.swap(Unew)
        A.swap(B)
    ws.destroy()


LIMIT = 32 << 20  # MHD_NOALLOC_SCRATCH_BYTES


def _need(nx, ny, ng, elem):
    """Bytes of the intermediate state: 9 planes, rows padded to 256 bytes."""
    per = 256 // elem
    pitch = -(-(nx + 2 * ng) // per) * per
    plane = -(-(pitch * (ny + 2 * ng)) // per) * per
    return 9 * plane * elem


def _largest_ny(nx, elem, ng=2):
    ny = 1
    while _need(nx, ny + 1, ng, elem) <= LIMIT:
        ny += 1
    return ny


@pytest.mark.parametrize("dtype,n_square,nx_tight", [(F64, 668, 668), (F32, 956, 956)])
def test_noalloc_at_the_size_limit(dtype, n_square, nx_tight):
    """The largest square grid whose intermediate state fits (668^2 FP64, 956^2
    FP32), and the tallest grid of the same width (its state within 0.1 % of the
    32 MiB array, so the sweeps write the array's last plane up to its end):
    bit-equal to mhd_advance on two steps.  One row more is rejected."""
    elem = 8 if dtype == F64 else 4
    assert _need(n_square, n_square, 2, elem) <= LIMIT < _need(n_square + 1, n_square + 1, 2, elem)
    ny_tight = _largest_ny(nx_tight, elem)
    assert _need(nx_tight, ny_tight, 2, elem) > 0.999 * LIMIT
    cfg = get_n_case_config(4, 1)
    for nx, ny in ((n_square, n_square), (nx_tight, ny_tight)):
        U0 = initialise(4, nx, ny, 2, cfg.extent)
        grids = [Grid2DGPU(nx, ny, 2, *cfg.extent, dtype) for _ in range(5)]
        Uold, Utmp, Unew, A, B = grids
        for g in grids:
            g.upload(U0)
        ws = GpuWorkspace()
        init_gpu_workspace(ws, Uold)
        set_gpu_physics_gamma(ws, cfg.gamma)
        set_gpu_physics_ch(ws, 0.0)
        ws.set_limiter(1)
        for call in range(2):
            dt = compute_dt_gpu(Uold, ws, cfg.cfl)
            ch = ws.ch
            advance_second_order_gpu(Uold, Utmp, Unew, ws, dt, 2, (0, 0, 0, 0))
            assert _noalloc(A, B, cfg.gamma, ch, 0.18, dt, 2, 1, (0, 0, 0, 0)) == 0, load().mhd_last_error()
            np.testing.assert_array_equal(B.download(), Unew.download(), err_msg=f"{nx}x{ny} call {call}")
            Uold.swap(Unew)
            A.swap(B)
        ws.destroy()
        for g in grids:
            g.release()
    over = [Grid2DGPU(nx_tight, ny_tight + 1, 2, *cfg.extent, dtype) for _ in range(2)]
    assert _noalloc(over[0], over[1], cfg.gamma, 1.0, 0.18, 1e-4, 2, 1, (0, 0, 0, 0)) == -1
    assert b"limit" in load().mhd_last_error()


def test_noalloc_rejects_grids_above_the_limit():
    big = Grid2DGPU(1024, 1024, 2, 0.0, 1.0, 0.0, 1.0, F64)  # 9 x 1056 x 1028 x 8 B > 32 MiB
    out = Grid2DGPU(1024, 1024, 2, 0.0, 1.0, 0.0, 1.0, F64)
    rc = _noalloc(big, out, 5.0 / 3.0, 1.0, 0.18, 1e-4, 2, 1, (0, 0, 0, 0))
    assert rc == -1
    assert b"limit" in load().mhd_last_error()
    with pytest.raises(MhdError):
        from mhd_gpu_acc_b200._lib import check

        check(rc, "mhd_advance_noalloc")
