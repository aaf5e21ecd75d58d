"""The FP32-bulk HLLD degeneracy rule, isolated on near-degenerate faces.

HLLD's single-star state divides by d = rho (S - u_n)(S - S_M) - B_n^2
(head/riemann.hpp:340-373).  The reference takes its degenerate branch when
|d| < 1e-14 (head/riemann.hpp:342-345, 354-357), which FP64 resolves.  On the
faces built here -- B_t, B_w ~ 1e-9..1e-6 and the two sides equal to within
1e-8..1e-5, with B_n^2 / rho above the sound speed squared, so the fast wave is
the Alfven wave (the switch-on limit) -- d is ~1e-6 of its terms: FP64 takes
the regular branch, while in FP32 d is rounding noise, and the reference's
absolute test would divide by it.  The FP32 step takes the degenerate branch
when |d| <= 1e-5 (rho (|S| + |u_n| + |S_M|)^2 + B_n^2) (star_degenerate in
csrc/mhd_common.cuh).  The check: on these faces the FP32 flux, evaluated by
the FP32 step's own solver functions on the GPU (mhd_riemann_flux_device), is
finite and agrees with the FP64 flux to 1e-4 of the face's flux scale.
"""
import ctypes as C

import numpy as np
import pytest

from mhd_gpu_acc_b200 import F32, F64, load
from mhd_gpu_acc_b200._lib import check

GAMMA = 5.0 / 3.0
HLLD = 2


def near_degenerate_faces(n, seed, dir_):
    """Primitive left / right states (9, n) of near-switch-on faces, normal = dir_."""
    rng = np.random.default_rng(seed)
    rho = rng.uniform(0.5, 2.0, n)
    p = rng.uniform(0.01, 0.05, n)
    bn = rng.uniform(0.8, 1.5, n) * rng.choice([-1.0, 1.0], n)
    vel = rng.uniform(-0.5, 0.5, (3, n))
    dv = 10.0 ** rng.uniform(-8, -5, n)   # relative jump across the face
    bt = 10.0 ** rng.uniform(-9, -6, n)   # transverse field scale

    def side():
        W = np.zeros((9, n))
        W[0] = rho * (1 + dv * rng.standard_normal(n))
        W[1:4] = vel + dv * rng.standard_normal((3, n))
        W[4 + dir_] = bn
        W[5 - dir_] = bt * rng.standard_normal(n)
        W[6] = bt * rng.standard_normal(n)
        W[7] = p * (1 + dv * rng.standard_normal(n))
        return W

    return side(), side()


def prim_to_cons(W):
    U = W.copy()
    U[1:4] = W[0] * W[1:4]
    U[7] = W[7] / (GAMMA - 1) + 0.5 * W[0] * (W[1:4] ** 2).sum(0) + 0.5 * (W[4:7] ** 2).sum(0)
    return U


def star_d(WL, WR, dir_):
    """d of each side's single-star state and the FP32 rule's threshold (FP64 numpy)."""
    def cf(W):
        a2 = GAMMA * W[7] / W[0]
        b2 = (W[4:7] ** 2).sum(0) / W[0]
        bn2 = W[4 + dir_] ** 2 / W[0]
        s = a2 + b2
        return np.sqrt(0.5 * (s + np.sqrt(np.maximum(s * s - 4 * a2 * bn2, 0))))

    unL, unR = WL[1 + dir_], WR[1 + dir_]
    cL, cR = cf(WL), cf(WR)
    SL, SR = np.minimum(unL - cL, unR - cR), np.maximum(unL + cL, unR + cR)
    pt = lambda W: W[7] + 0.5 * (W[4:7] ** 2).sum(0)  # noqa: E731
    SM = ((SR - unR) * WR[0] * unR - (SL - unL) * WL[0] * unL + pt(WL) - pt(WR)) / \
         ((SR - unR) * WR[0] - (SL - unL) * WL[0])
    out = []
    for W, S, un in ((WL, SL, unL), (WR, SR, unR)):
        bn = W[4 + dir_]
        d = W[0] * (S - un) * (S - SM) - bn ** 2
        m = np.abs(S) + np.abs(un) + np.abs(SM)
        out.append((d, 1e-5 * (W[0] * m * m + bn ** 2)))
    return out


def device_flux(dtype, UL, UR, dir_, ch):
    import torch

    n = UL.shape[1]
    dl = torch.from_numpy(np.ascontiguousarray(UL.T)).cuda()
    dr = torch.from_numpy(np.ascontiguousarray(UR.T)).cuda()
    df = torch.empty_like(dl)
    check(load().mhd_riemann_flux_device(None, dtype, n, C.c_void_p(dl.data_ptr()), C.c_void_p(dr.data_ptr()),
                                         dir_, HLLD, float(ch), GAMMA, C.c_void_p(df.data_ptr())),
          "mhd_riemann_flux_device")
    torch.cuda.synchronize()
    return df.cpu().numpy().T.copy()


@pytest.mark.gpu
@pytest.mark.parametrize("dir_", [0, 1])
def test_fp32_hlld_near_degenerate_faces(dir_):
    n = 8192
    WL, WR = near_degenerate_faces(n, 11 + dir_, dir_)
    # the face set exercises the rule: FP32 degenerate branch, FP64 regular branch
    for d, thr in star_d(WL, WR, dir_):
        assert np.mean(np.abs(d) <= thr) > 0.95
        assert np.mean(np.abs(d) < 1e-14) < 0.01
    UL, UR = prim_to_cons(WL), prim_to_cons(WR)
    ch = 2.0
    F64_ = device_flux(F64, UL, UR, dir_, ch)
    # the FP64 device solver is the host one (the reference's operand order)
    lib = load()
    F = np.zeros(9)
    for k in range(0, n, 997):
        a, b = np.ascontiguousarray(UL[:, k]), np.ascontiguousarray(UR[:, k])
        assert lib.mhd_riemann_flux(a.ctypes.data, b.ctypes.data, dir_, HLLD, ch, GAMMA, F.ctypes.data) == 0
        np.testing.assert_array_equal(F, F64_[:, k])
    F32_ = device_flux(F32, UL, UR, dir_, ch)
    assert np.isfinite(F32_).all()
    scale = np.abs(F64_).max(axis=0)
    err = (np.abs(F32_ - F64_).max(axis=0) / scale)
    print(f"dir {dir_}: FP32 vs FP64 flux on {n} near-degenerate faces: max {err.max():.2e}, "
          f"median {np.median(err):.2e} (relative to each face's flux scale)")
    assert err.max() <= 1e-4


@pytest.mark.gpu
def test_device_flux_all_solvers_fp64_equals_host():
    """mhd_riemann_flux_device in FP64 is the host riemann_flux bit for bit, for
    every solver, on random smooth faces."""
    rng = np.random.default_rng(5)
    n = 64
    WL = np.stack([rng.uniform(0.5, 2, n), *rng.uniform(-1, 1, (3, n)), *rng.uniform(-1, 1, (3, n)),
                   rng.uniform(0.1, 1, n), rng.uniform(-0.1, 0.1, n)])
    WR = WL * (1 + 0.1 * rng.standard_normal(WL.shape))
    WR[0] = np.abs(WR[0]); WR[7] = np.abs(WR[7])
    UL, UR = prim_to_cons(WL), prim_to_cons(WR)
    lib = load()
    import torch

    for solver in range(4):
        for dir_ in (0, 1):
            dl = torch.from_numpy(np.ascontiguousarray(UL.T)).cuda()
            dr = torch.from_numpy(np.ascontiguousarray(UR.T)).cuda()
            df = torch.empty_like(dl)
            check(lib.mhd_riemann_flux_device(None, F64, n, C.c_void_p(dl.data_ptr()), C.c_void_p(dr.data_ptr()),
                                              dir_, solver, 0.7, GAMMA, C.c_void_p(df.data_ptr())), "flux")
            got = df.cpu().numpy()
            F = np.zeros(9)
            for k in range(n):
                a, b = np.ascontiguousarray(UL[:, k]), np.ascontiguousarray(UR[:, k])
                lib.mhd_riemann_flux(a.ctypes.data, b.ctypes.data, dir_, solver, 0.7, GAMMA, F.ctypes.data)
                np.testing.assert_array_equal(got[k], F, err_msg=f"solver {solver} dir {dir_} face {k}")
