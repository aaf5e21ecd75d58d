// adj_physics.cuh -- local forward functions of the split step and their
// hand-written reverse-mode (adjoint) counterparts, for the HLL solver with the
// van Leer or minmod limiter.
//
// The forward functions restate, in the primitive (W) form, the reference's
// cons_to_prim / prim_to_cons / flux_x / fast_speed_x (head/physics.hpp:69-191),
// hll_flux (head/riemann.hpp:70-107) and the MUSCL-Hancock predictor with c_h
// (src/cpu/solver_cpu.cpp:88-119).  Every *_adj function takes the forward
// inputs and an output cotangent and ADDS the input cotangents (vector-Jacobian
// products).  Branches (limiter sign tests, positivity fallbacks, the HLL wave
// region, min/max selections) are re-evaluated from the same inputs, so the
// adjoint follows exactly the branches the forward took.
//
// Everything is written for the x direction; the y direction swaps (u, v) and
// (Bx, By) on the way in and the flux components on the way out (rot()).
#pragma once

#include <cmath>

#include "mhd_common.cuh"

// Host and device: the host build lets tests check every *_adj against
// finite differences on the CPU.
#ifdef __CUDACC__
#define ADJ_HD __host__ __device__ __forceinline__
#else
#define ADJ_HD inline
#endif

namespace mhd {
namespace adj {

template <typename R>
struct S9 {
    R v[NV];
};

template <typename R>
ADJ_HD void zero(R* a) {
#pragma unroll
    for (int k = 0; k < NV; ++k) a[k] = R(0);
}

// swap the normal and tangential components (u <-> v, Bx <-> By); an involution
template <typename R>
ADJ_HD void rot(R* a) {
    R t = a[1]; a[1] = a[2]; a[2] = t;
    t = a[4]; a[4] = a[5]; a[5] = t;
}

template <typename R>
ADJ_HD void c2p(const R* U, R g, R* W) {
    const R ir = R(1) / U[RHO];
    const R u = U[MX] * ir, v = U[MY] * ir, w = U[MZ] * ir;
    W[RHO] = U[RHO]; W[PU] = u; W[PV] = v; W[PW] = w;
    W[BX] = U[BX]; W[BY] = U[BY]; W[BZ] = U[BZ];
    W[PP] = (g - R(1)) * (U[EN] - R(0.5) * U[RHO] * (u * u + v * v + w * w) -
                          R(0.5) * (U[BX] * U[BX] + U[BY] * U[BY] + U[BZ] * U[BZ]));
    W[PSI] = U[PSI];
}

// lU += (dW/dU)^T lW
template <typename R>
ADJ_HD void c2p_adj(const R* U, const R* W, R g, const R* lW, R* lU) {
    const R ir = R(1) / U[RHO], gm = g - R(1), lp = lW[PP];
    const R u = W[PU], v = W[PV], w = W[PW];
    lU[EN] += gm * lp;
    lU[MX] += lW[PU] * ir - gm * lp * u;
    lU[MY] += lW[PV] * ir - gm * lp * v;
    lU[MZ] += lW[PW] * ir - gm * lp * w;
    lU[RHO] += lW[RHO] - (lW[PU] * u + lW[PV] * v + lW[PW] * w) * ir + gm * lp * R(0.5) * (u * u + v * v + w * w);
    lU[BX] += lW[BX] - gm * lp * W[BX];
    lU[BY] += lW[BY] - gm * lp * W[BY];
    lU[BZ] += lW[BZ] - gm * lp * W[BZ];
    lU[PSI] += lW[PSI];
}

template <typename R>
ADJ_HD void p2c(const R* W, R g, R* U) {
    const R r = W[RHO];
    U[RHO] = r; U[MX] = r * W[PU]; U[MY] = r * W[PV]; U[MZ] = r * W[PW];
    U[BX] = W[BX]; U[BY] = W[BY]; U[BZ] = W[BZ];
    U[EN] = W[PP] / (g - R(1)) + R(0.5) * r * (W[PU] * W[PU] + W[PV] * W[PV] + W[PW] * W[PW]) +
            R(0.5) * (W[BX] * W[BX] + W[BY] * W[BY] + W[BZ] * W[BZ]);
    U[PSI] = W[PSI];
}

template <typename R>
ADJ_HD void p2c_adj(const R* W, R g, const R* lU, R* lW) {
    const R r = W[RHO], u = W[PU], v = W[PV], w = W[PW], lE = lU[EN];
    lW[RHO] += lU[RHO] + lU[MX] * u + lU[MY] * v + lU[MZ] * w + lE * R(0.5) * (u * u + v * v + w * w);
    lW[PU] += (lU[MX] + lE * u) * r;
    lW[PV] += (lU[MY] + lE * v) * r;
    lW[PW] += (lU[MZ] + lE * w) * r;
    lW[BX] += lU[BX] + lE * W[BX];
    lW[BY] += lU[BY] + lE * W[BY];
    lW[BZ] += lU[BZ] + lE * W[BZ];
    lW[PP] += lE / (g - R(1));
    lW[PSI] += lU[PSI];
}

// GLM-MHD x-flux of a primitive state (head/physics.hpp:105-127 in W form)
template <typename R>
ADJ_HD void flux(const R* W, R ch, R g, R* F) {
    const R r = W[RHO], u = W[PU], v = W[PV], w = W[PW], bx = W[BX], by = W[BY], bz = W[BZ], p = W[PP];
    const R B2 = bx * bx + by * by + bz * bz, pt = p + R(0.5) * B2, uB = u * bx + v * by + w * bz;
    const R E = p / (g - R(1)) + R(0.5) * r * (u * u + v * v + w * w) + R(0.5) * B2;
    F[0] = r * u;
    F[1] = r * u * u + pt - bx * bx;
    F[2] = r * u * v - bx * by;
    F[3] = r * u * w - bx * bz;
    F[4] = W[PSI];
    F[5] = by * u - bx * v;
    F[6] = bz * u - bx * w;
    F[7] = (E + pt) * u - bx * uB;
    F[8] = ch * ch * bx;
}

// lW += (dF/dW)^T lF ;  lch += (dF/dch) . lF
template <typename R>
ADJ_HD void flux_adj(const R* W, R ch, R g, const R* lF, R* lW, R& lch) {
    const R r = W[RHO], u = W[PU], v = W[PV], w = W[PW], bx = W[BX], by = W[BY], bz = W[BZ], p = W[PP];
    const R B2 = bx * bx + by * by + bz * bz, uB = u * bx + v * by + w * bz;
    const R H = p * g / (g - R(1)) + R(0.5) * r * (u * u + v * v + w * w) + B2;  // E + p_tot
    lW[RHO] += lF[0] * u + lF[1] * u * u + lF[2] * u * v + lF[3] * u * w + lF[7] * u * R(0.5) * (u * u + v * v + w * w);
    lW[PU] += lF[0] * r + lF[1] * R(2) * r * u + lF[2] * r * v + lF[3] * r * w + lF[5] * by + lF[6] * bz +
              lF[7] * (H + r * u * u - bx * bx);
    lW[PV] += lF[2] * r * u - lF[5] * bx + lF[7] * (r * u * v - bx * by);
    lW[PW] += lF[3] * r * u - lF[6] * bx + lF[7] * (r * u * w - bx * bz);
    lW[BX] += -lF[1] * bx - lF[2] * by - lF[3] * bz - lF[5] * v - lF[6] * w + lF[7] * (bx * u - uB) + lF[8] * ch * ch;
    lW[BY] += lF[1] * by - lF[2] * bx + lF[5] * u + lF[7] * (R(2) * by * u - bx * v);
    lW[BZ] += lF[1] * bz - lF[3] * bx + lF[6] * u + lF[7] * (R(2) * bz * u - bx * w);
    lW[PP] += lF[1] + lF[7] * u * g / (g - R(1));
    lW[PSI] += lF[4];
    lch += lF[8] * R(2) * ch * bx;
}

// fast magnetosonic speed in x (head/physics.hpp:175-181)
template <typename R>
ADJ_HD R fast(const R* W, R g) {
    const R ir = R(1) / W[RHO];
    const R a2 = g * W[PP] * ir, b2 = (W[BX] * W[BX] + W[BY] * W[BY] + W[BZ] * W[BZ]) * ir;
    const R bn2 = W[BX] * W[BX] * ir, s = a2 + b2, disc = s * s - R(4) * a2 * bn2;
    return sqrt(R(0.5) * (s + sqrt(disc > R(0) ? disc : R(0))));
}

template <typename R>
ADJ_HD void fast_adj(const R* W, R g, R lcf, R* lW) {
    const R ir = R(1) / W[RHO];
    const R a2 = g * W[PP] * ir, b2 = (W[BX] * W[BX] + W[BY] * W[BY] + W[BZ] * W[BZ]) * ir;
    const R bn2 = W[BX] * W[BX] * ir, s = a2 + b2, disc = s * s - R(4) * a2 * bn2;
    const R rt = sqrt(disc > R(0) ? disc : R(0));
    const R cf = sqrt(R(0.5) * (s + rt));
    const R lq = lcf / (R(2) * cf);
    R ls = R(0.5) * lq;
    const R lr = R(0.5) * lq;
    const R ld = (disc > R(0)) ? lr / (R(2) * rt) : R(0);
    ls += ld * R(2) * s;
    const R la2 = ls - R(4) * bn2 * ld, lb2 = ls, lbn2 = -R(4) * a2 * ld;
    lW[PP] += la2 * g * ir;
    lW[RHO] -= (la2 * a2 + lb2 * b2 + lbn2 * bn2) * ir;
    lW[BX] += (lb2 + lbn2) * R(2) * W[BX] * ir;
    lW[BY] += lb2 * R(2) * W[BY] * ir;
    lW[BZ] += lb2 * R(2) * W[BZ] * ir;
}

template <typename R>
ADJ_HD bool riemann_ok(const R* W) {
    return isfinite(W[RHO]) && isfinite(W[PP]) && W[RHO] > R(0) && W[PP] > R(0);
}

// HLL in x (head/riemann.hpp:70-107) from conserved side states.
template <typename R>
ADJ_HD void hll(const R* UL, const R* UR, R ch, R g, R* F) {
    R WL[NV], WR[NV], FL[NV], FR[NV];
    c2p(UL, g, WL);
    c2p(UR, g, WR);
    flux(WL, ch, g, FL);
    flux(WR, ch, g, FR);
    if (!riemann_ok(WL) || !riemann_ok(WR)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = R(0.5) * (FL[k] + FR[k]);
        return;
    }
    const R cL = fast(WL, g), cR = fast(WR, g);
    const R SL = fmin(fmin(WL[PU] - cL, WR[PU] - cR), -ch);
    const R SR = fmax(fmax(WL[PU] + cL, WR[PU] + cR), ch);
    if (SL >= R(0)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = FL[k];
        return;
    }
    if (SR <= R(0)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = FR[k];
        return;
    }
    const R D = SR - SL;
    if (fabs(D) < R(1e-14)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = R(0.5) * (FL[k] + FR[k]);
        return;
    }
    const R iD = R(1) / D;
#pragma unroll
    for (int k = 0; k < NV; ++k) F[k] = iD * (SR * FL[k] - SL * FR[k] + SL * SR * (UR[k] - UL[k]));
}

template <typename R>
ADJ_HD void hll_adj(const R* UL, const R* UR, R ch, R g, const R* lF, R* lUL, R* lUR, R& lch) {
    R WL[NV], WR[NV], FL[NV], FR[NV], lWL[NV], lWR[NV], lFL[NV], lFR[NV];
    c2p(UL, g, WL);
    c2p(UR, g, WR);
    flux(WL, ch, g, FL);
    flux(WR, ch, g, FR);
    zero(lWL);
    zero(lWR);
    if (!riemann_ok(WL) || !riemann_ok(WR)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) lFL[k] = lFR[k] = R(0.5) * lF[k];
    } else {
        const R cL = fast(WL, g), cR = fast(WR, g);
        const R aL = WL[PU] - cL, aR = WR[PU] - cR, bL = WL[PU] + cL, bR = WR[PU] + cR;
        const R SL = fmin(fmin(aL, aR), -ch);
        const R SR = fmax(fmax(bL, bR), ch);
        const R D = SR - SL;
        if (SL >= R(0)) {
#pragma unroll
            for (int k = 0; k < NV; ++k) { lFL[k] = lF[k]; lFR[k] = R(0); }
        } else if (SR <= R(0)) {
#pragma unroll
            for (int k = 0; k < NV; ++k) { lFL[k] = R(0); lFR[k] = lF[k]; }
        } else if (fabs(D) < R(1e-14)) {
#pragma unroll
            for (int k = 0; k < NV; ++k) lFL[k] = lFR[k] = R(0.5) * lF[k];
        } else {
            const R iD = R(1) / D;
            R lSL = R(0), lSR = R(0);
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                const R dU = UR[k] - UL[k];
                const R Fk = iD * (SR * FL[k] - SL * FR[k] + SL * SR * dU);
                lFL[k] = lF[k] * SR * iD;
                lFR[k] = -lF[k] * SL * iD;
                lUR[k] += lF[k] * SL * SR * iD;
                lUL[k] -= lF[k] * SL * SR * iD;
                lSR += lF[k] * (FL[k] + SL * dU - Fk) * iD;
                lSL += lF[k] * (-FR[k] + SR * dU + Fk) * iD;
            }
            // SL = fmin(fmin(aL, aR), -ch): route to the selected argument
            const R m1 = fmin(aL, aR);
            if (m1 <= -ch) {
                if (aL <= aR) { lWL[PU] += lSL; fast_adj(WL, g, -lSL, lWL); }
                else { lWR[PU] += lSL; fast_adj(WR, g, -lSL, lWR); }
            } else {
                lch -= lSL;
            }
            const R m2 = fmax(bL, bR);
            if (m2 >= ch) {
                if (bL >= bR) { lWL[PU] += lSR; fast_adj(WL, g, lSR, lWL); }
                else { lWR[PU] += lSR; fast_adj(WR, g, lSR, lWR); }
            } else {
                lch += lSR;
            }
        }
    }
    flux_adj(WL, ch, g, lFL, lWL, lch);
    flux_adj(WR, ch, g, lFR, lWR, lch);
    c2p_adj(UL, WL, g, lWL, lUL);
    c2p_adj(UR, WR, g, lWR, lUR);
}

template <int LIM, typename R>
ADJ_HD R limit(R a, R b) {
    if (a * b <= R(0)) return R(0);
    if (LIM == VANLEER) return R(2) * a * b / (a + b);
    return (a > R(0)) ? ((b < a) ? b : a) : ((a < b) ? b : a);
}

// d limit / d a, d limit / d b
template <int LIM, typename R>
ADJ_HD void limit_adj(R a, R b, R ls, R& la, R& lb) {
    if (a * b <= R(0)) return;
    if (LIM == VANLEER) {
        const R s = a + b, is2 = R(1) / (s * s);
        la += ls * R(2) * b * b * is2;
        lb += ls * R(2) * a * a * is2;
    } else {
        if (a > R(0)) { if (b < a) lb += ls; else la += ls; }
        else { if (a < b) lb += ls; else la += ls; }
    }
}

template <typename R>
ADJ_HD bool physical(const R* V) {
    bool ok = V[RHO] > R(1e-12) && V[PP] > R(1e-12);
#pragma unroll
    for (int k = 0; k < NV; ++k) ok = ok && isfinite(V[k]);
    return ok;
}

// MUSCL-Hancock predictor of one cell in x: (Wm, Wc, Wp) -> (UL*, UR*).
template <int LIM, typename R>
ADJ_HD void recon(const R* Wm, const R* Wc, const R* Wp, R dtd, R ch, R g, R* Ls, R* Rs) {
    R WL[NV], WR[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const R s = limit<LIM>(Wc[k] - Wm[k], Wp[k] - Wc[k]);
        WL[k] = Wc[k] - R(0.5) * s;
        WR[k] = Wc[k] + R(0.5) * s;
    }
    if (!physical(WL)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) WL[k] = Wc[k];
    }
    if (!physical(WR)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) WR[k] = Wc[k];
    }
    R UL[NV], UR[NV], FL[NV], FR[NV], V[NV];
    p2c(WL, g, UL);
    p2c(WR, g, UR);
    flux(WL, ch, g, FL);
    flux(WR, ch, g, FR);
    const R h = R(0.5) * dtd;
#pragma unroll
    for (int k = 0; k < NV; ++k) Ls[k] = UL[k] - h * (FR[k] - FL[k]);
    c2p(Ls, g, V);
    if (!physical(V)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) Ls[k] = UL[k];
    }
#pragma unroll
    for (int k = 0; k < NV; ++k) Rs[k] = UR[k] - h * (FR[k] - FL[k]);
    c2p(Rs, g, V);
    if (!physical(V)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) Rs[k] = UR[k];
    }
}

// Adjoint of recon: adds to lWm, lWc, lWp and the scalar cotangents of
// dtd (= dt/d) and ch.
template <int LIM, typename R>
ADJ_HD void recon_adj(const R* Wm, const R* Wc, const R* Wp, R dtd, R ch, R g, const R* lLs,
                                          const R* lRs, R* lWm, R* lWc, R* lWp, R& ldtd, R& lch) {
    R WL[NV], WR[NV], sl[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        sl[k] = limit<LIM>(Wc[k] - Wm[k], Wp[k] - Wc[k]);
        WL[k] = Wc[k] - R(0.5) * sl[k];
        WR[k] = Wc[k] + R(0.5) * sl[k];
    }
    const bool okL = physical(WL), okR = physical(WR);
    if (!okL) {
#pragma unroll
        for (int k = 0; k < NV; ++k) WL[k] = Wc[k];
    }
    if (!okR) {
#pragma unroll
        for (int k = 0; k < NV; ++k) WR[k] = Wc[k];
    }
    R UL[NV], UR[NV], FL[NV], FR[NV], V[NV], tmp[NV];
    p2c(WL, g, UL);
    p2c(WR, g, UR);
    flux(WL, ch, g, FL);
    flux(WR, ch, g, FR);
    const R h = R(0.5) * dtd;
#pragma unroll
    for (int k = 0; k < NV; ++k) tmp[k] = UL[k] - h * (FR[k] - FL[k]);
    c2p(tmp, g, V);
    const bool okLs = physical(V);
#pragma unroll
    for (int k = 0; k < NV; ++k) tmp[k] = UR[k] - h * (FR[k] - FL[k]);
    c2p(tmp, g, V);
    const bool okRs = physical(V);
    // U*_side = U_side - h (FR - FL) unless the predictor fallback was taken
    R lUL[NV], lUR[NV], lD[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        lUL[k] = lLs[k];
        lUR[k] = lRs[k];
        lD[k] = (okLs ? -lLs[k] : R(0)) + (okRs ? -lRs[k] : R(0));  // cotangent of h (FR - FL)
    }
    R lFL[NV], lFR[NV], lWL[NV], lWR[NV];
    R lh = R(0);
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        lFR[k] = h * lD[k];
        lFL[k] = -h * lD[k];
        lh += lD[k] * (FR[k] - FL[k]);
    }
    ldtd += R(0.5) * lh;
    zero(lWL);
    zero(lWR);
    p2c_adj(WL, g, lUL, lWL);
    p2c_adj(WR, g, lUR, lWR);
    flux_adj(WL, ch, g, lFL, lWL, lch);
    flux_adj(WR, ch, g, lFR, lWR, lch);
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        lWc[k] += lWL[k] + lWR[k];
        const R ls = (okL ? -R(0.5) * lWL[k] : R(0)) + (okR ? R(0.5) * lWR[k] : R(0));
        R la = R(0), lb = R(0);
        limit_adj<LIM>(Wc[k] - Wm[k], Wp[k] - Wc[k], ls, la, lb);
        lWm[k] -= la;
        lWc[k] += la - lb;
        lWp[k] += lb;
    }
}

// Raw CFL speed of a cell (src/cpu/solver_cpu.cpp:291-300 without the c_h
// floor): max(|u| + cf_x, |v| + cf_y), or -1 for a skipped cell.
template <typename R>
ADJ_HD R raw_speed(const R* U, R g, int* branch) {
    R W[NV];
    c2p(U, g, W);
    if (!isfinite(W[RHO]) || !isfinite(W[PP]) || W[RHO] <= R(0) || W[PP] <= R(0)) return R(-1);
    const R sx = fabs(W[PU]) + fast(W, g);
    rot(W);
    const R sy = fabs(W[PU]) + fast(W, g);
    if (!isfinite(sx) || !isfinite(sy)) return R(-1);
    *branch = (sx < sy) ? 1 : 0;
    return (sx < sy) ? sy : sx;
}

// lU += lm * d raw_speed / dU (the branch the max took)
template <typename R>
ADJ_HD void raw_speed_adj(const R* U, R g, int branch, R lm, R* lU) {
    R W[NV], lW[NV];
    c2p(U, g, W);
    zero(lW);
    if (branch == 1) rot(W);
    lW[PU] += (W[PU] >= R(0)) ? lm : -lm;
    fast_adj(W, g, lm, lW);
    if (branch == 1) rot(lW);
    if (branch == 1) rot(W);
    c2p_adj(U, W, g, lW, lU);
}

}  // namespace adj
}  // namespace mhd
