"""Discrete adjoint: local derivatives (CPU) and the full gradient (GPU) against
FP64 central finite differences, FP32 against FP64, checkpoint independence,
and a torch.autograd.Function wrapper checked with torch.autograd.gradcheck.

The gradient problem: Orszag-Tang on periodic [0,1]^2, HLL (or HLLD) + van Leer, 16
Fourier amplitudes a ~ N(0, 0.01^2) (seed s) perturbing v and B, target density
from a second amplitude set (seed s + 1), J = 1/2 sum (rho - rho_target)^2.
"""
import os
import subprocess

import numpy as np
import pytest

from mhd_gpu_acc_b200 import F32, F64
from mhd_gpu_acc_b200.adjoint import OTAdjoint, amplitudes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# gradient agreement with central differences (relative, 2-norm)
FD_RTOL = 1e-4


def test_local_adjoints_against_finite_differences(tmp_path):
    exe = str(tmp_path / "adjchk")
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-x", "cu", "-I", os.path.join(ROOT, "mhd_gpu_acc_b200", "csrc"),
                    os.path.join(ROOT, "tests", "adj_local_check.cu"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout


def _problem(n, steps, dtype=F64, seed=0, every=0, solver=0):
    adj = OTAdjoint(n=n, nsteps=steps, dtype=dtype, checkpoint_every=every, solver=solver)
    _, target = adj.forward(amplitudes(seed + 1), want_rho=True)
    adj.set_target(target)
    return adj, amplitudes(seed)


def _fd(adj, a, h=1e-6):
    g = np.zeros(16)
    for k in range(16):
        e = np.zeros(16)
        e[k] = h
        g[k] = (adj.forward(a + e) - adj.forward(a - e)) / (2 * h)
    return g


@pytest.mark.gpu
def test_gradient_matches_central_differences_small():
    adj, a = _problem(64, 40)
    J, g = adj.gradient(a)
    fd = _fd(adj, a)
    assert J > 0
    assert np.linalg.norm(g - fd) / np.linalg.norm(fd) <= FD_RTOL, (g, fd)


@pytest.mark.gpu
def test_hlld_gradient_matches_central_differences():
    """The HLLD adjoint (star / double-star regions, HLL fallbacks, GLM
    overwrite) on the same problem: FP64 against central differences, FP32
    against FP64."""
    adj, a = _problem(64, 40, solver=2)
    J, g = adj.gradient(a)
    fd = _fd(adj, a)
    assert J > 0
    assert np.linalg.norm(g - fd) / np.linalg.norm(fd) <= FD_RTOL, (g, fd)
    adj32, _ = _problem(64, 40, F32, solver=2)
    _, g32 = adj32.gradient(a)
    assert np.linalg.norm(g32 - g) / np.linalg.norm(g) <= 1e-2


@pytest.mark.gpu
def test_checkpoint_interval_does_not_change_the_gradient():
    """Recomputation from checkpoints reproduces the trajectory bit for bit; J and
    the gradient agree to the rounding of their atomically summed reductions."""
    ref, a = _problem(48, 30, every=1)
    J1, g1 = ref.gradient(a)
    for every in (5, 7, 30):
        adj, _ = _problem(48, 30, every=every)
        J2, g2 = adj.gradient(a)
        assert abs(J1 - J2) <= 1e-14 * abs(J1)
        np.testing.assert_allclose(g2, g1, rtol=1e-10, atol=1e-14 * np.abs(g1).max())


@pytest.mark.gpu
def test_configuration_512_400_fp64_and_fp32():
    """The gradient configuration: 512^2, 400 steps, HLL + van Leer."""
    adj64, a = _problem(512, 400, F64)
    J64, g64 = adj64.gradient(a)
    fd = _fd(adj64, a)
    rel_fd = np.linalg.norm(g64 - fd) / np.linalg.norm(fd)
    adj32, _ = _problem(512, 400, F32)
    J32, g32 = adj32.gradient(a)
    rel_32 = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    print(f"512^2 x 400: J {J64:.6e}  FP64 adjoint vs FD {rel_fd:.2e}  FP32 adjoint vs FP64 {rel_32:.2e}")
    assert rel_fd <= FD_RTOL
    assert rel_32 <= 1e-2


@pytest.mark.gpu
def test_torch_autograd_function_gradcheck():
    """The wrapper's backward is the adjoint; gradcheck's own central differences
    (eps 1e-6) on a coarse 48^2 grid, where an occasional van Leer kink within eps
    limits agreement to ~1e-3 (the strict FD checks are above)."""
    torch = pytest.importorskip("torch")
    adj, a0 = _problem(48, 16)

    class OTObjective(torch.autograd.Function):
        """J(a) with the adjoint as its backward (check harness only)."""

        @staticmethod
        def forward(ctx, a):
            J, g = adj.gradient(a.detach().numpy())
            ctx.save_for_backward(torch.from_numpy(g))
            return a.new_tensor(J)

        @staticmethod
        def backward(ctx, gJ):
            (g,) = ctx.saved_tensors
            return gJ * g

    a = torch.tensor(a0, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(OTObjective.apply, (a,), eps=1e-6, atol=1e-6, rtol=1e-3)


def _best_of(fn, reps=3):
    import time

    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        best = min(best, time.perf_counter() - t0)
    return best


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [F32, F64])
def test_gradient_costs_at_most_four_forward_solves(dtype):
    """The gradient configuration (512^2, 400 steps, HLL + van Leer): the
    gradient (forward with checkpoints + reverse sweep) costs at most 4x one
    forward solve, wall time, best of 3 after a warm-up."""
    adj, a = _problem(512, 400, dtype)
    adj.forward(a)
    adj.gradient(a)
    t_fwd = _best_of(lambda: adj.forward(a))
    t_grad = _best_of(lambda: adj.gradient(a))
    print(f"{'FP32' if dtype == F32 else 'FP64'} 512^2 x 400 HLL: forward {t_fwd:.4f} s, gradient {t_grad:.4f} s, "
          f"ratio {t_grad / t_fwd:.2f}")
    assert t_grad / t_fwd <= 4.0
