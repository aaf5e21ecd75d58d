// adj_physics.cuh -- local forward functions of the split step and their
// hand-written reverse-mode (adjoint) counterparts, for the HLL and HLLD
// solvers with the van Leer or minmod limiter.
//
// The forward functions restate, in the primitive (W) form, the reference's
// cons_to_prim / prim_to_cons / flux_x / fast_speed_x (head/physics.hpp:69-191),
// hll_flux (head/riemann.hpp:70-107), hlld_flux with the GLM overwrite
// (head/riemann.hpp:253-592) and the MUSCL-Hancock predictor with c_h
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

// ---------------------------------------------------------------------------
// HLLD (head/riemann.hpp:253-480) with the GLM psi/Bn overwrite and the
// non-finite fallback of riemann_flux (head/riemann.hpp:544-592), and their
// adjoints.  The forward follows the FP64 kernel's HLLD (phys_exact.cuh) step
// for step: the same fallbacks to HLL, region tests and star states.
// ---------------------------------------------------------------------------

// One side of a face in the x frame: primitive components and the conserved E.
template <typename R>
struct HSide {
    R rho, un, ut, uw, Bn, Bt, Bw, p, psi, E;
};

template <typename R>
ADJ_HD HSide<R> hside(const R* W, const R* U) {
    return HSide<R>{W[RHO], W[PU], W[PV], W[PW], W[BX], W[BY], W[BZ], W[PP], W[PSI], U[EN]};
}

// side cotangents -> lW (primitive) and lU[EN]
template <typename R>
ADJ_HD void hside_scatter(const HSide<R>& l, R* lW, R* lU) {
    lW[RHO] += l.rho; lW[PU] += l.un; lW[PV] += l.ut; lW[PW] += l.uw;
    lW[BX] += l.Bn; lW[BY] += l.Bt; lW[BZ] += l.Bw; lW[PP] += l.p; lW[PSI] += l.psi;
    lU[EN] += l.E;
}

// Single-star tangential velocity and field of a side (head/riemann.hpp:340-373).
template <typename R>
ADJ_HD void star_tan(const HSide<R>& s, R S, R SM, R& uts, R& uws, R& Bts, R& Bws) {
    const R d = s.rho * (S - s.un) * (S - SM) - s.Bn * s.Bn;
    if (star_degenerate(d, s.rho, s.un, S, SM, s.Bn)) { uts = s.ut; uws = s.uw; Bts = s.Bt; Bws = s.Bw; return; }
    uts = s.ut - s.Bn * s.Bt * (SM - s.un) / d;
    uws = s.uw - s.Bn * s.Bw * (SM - s.un) / d;
    Bts = s.Bt * (s.rho * (S - s.un) * (S - s.un) - s.Bn * s.Bn) / d;
    Bws = s.Bw * (s.rho * (S - s.un) * (S - s.un) - s.Bn * s.Bn) / d;
}

template <typename R>
ADJ_HD void star_tan_adj(const HSide<R>& s, R S, R SM, R luts, R luws, R lBts, R lBws, HSide<R>& ls, R& lS,
                         R& lSM) {
    const R q = S - s.un, d = s.rho * q * (S - SM) - s.Bn * s.Bn;
    if (star_degenerate(d, s.rho, s.un, S, SM, s.Bn)) {
        ls.ut += luts; ls.uw += luws; ls.Bt += lBts; ls.Bw += lBws;
        return;
    }
    const R e = SM - s.un, f = s.rho * q * q - s.Bn * s.Bn, id = R(1) / d;
    const R A = luts * s.Bt + luws * s.Bw;  // from -Bn (Bt, Bw) e / d
    const R Bc = lBts * s.Bt + lBws * s.Bw; // from (Bt, Bw) f / d
    ls.ut += luts;
    ls.uw += luws;
    ls.Bt += -luts * s.Bn * e * id + lBts * f * id;
    ls.Bw += -luws * s.Bn * e * id + lBws * f * id;
    R lBn = -A * e * id;
    const R le = -A * s.Bn * id;
    const R lf = Bc * id;
    const R ld = (A * s.Bn * e - Bc * f) * id * id;
    R lun = -le;  // e = SM - un
    lSM += le;
    ls.rho += lf * q * q + ld * q * (S - SM);  // f = rho q^2 - Bn^2, d = rho q (S - SM) - Bn^2
    R lq = lf * R(2) * s.rho * q + ld * s.rho * (S - SM);
    lBn -= (lf + ld) * R(2) * s.Bn;
    lS += ld * s.rho * q;
    lSM -= ld * s.rho * q;
    lS += lq;  // q = S - un
    lun -= lq;
    ls.un += lun;
    ls.Bn += lBn;
}

// Star energy of a side: (E (S - un) - pt un + ptstar SM + Bn (B.u* - B.u)) / (S - SM);
// BdUs receives B.u* = Bn SM + Bt* ut* + Bw* uw*.
template <typename R>
ADJ_HD R star_energy(const HSide<R>& s, R pt, R S, R SM, R ptstar, R uts, R uws, R Bts, R Bws, R& BdUs) {
    const R BdU = s.Bn * s.un + s.Bt * s.ut + s.Bw * s.uw;
    BdUs = s.Bn * SM + Bts * uts + Bws * uws;
    return (s.E * (S - s.un) - pt * s.un + ptstar * SM + s.Bn * (BdUs - BdU)) / (S - SM);
}

// lBdUs: a cotangent of B.u* from elsewhere (the double-star energy).
template <typename R>
ADJ_HD void star_energy_adj(const HSide<R>& s, R pt, R S, R SM, R ptstar, R uts, R uws, R Bts, R Bws, R Es, R lEs,
                            R lBdUs_in, HSide<R>& ls, R& lpt, R& lS, R& lSM, R& lptstar, R& luts, R& luws, R& lBts,
                            R& lBws) {
    const R den = S - SM;
    const R BdU = s.Bn * s.un + s.Bt * s.ut + s.Bw * s.uw;
    const R BdUs = s.Bn * SM + Bts * uts + Bws * uws;
    const R lnum = lEs / den, lden = -lEs * Es / den;
    lS += lden;
    lSM -= lden;
    ls.E += lnum * (S - s.un);
    lS += lnum * s.E;
    ls.un -= lnum * s.E + lnum * pt;
    lpt -= lnum * s.un;
    lptstar += lnum * SM;
    lSM += lnum * ptstar;
    ls.Bn += lnum * (BdUs - BdU);
    const R lBdUs = lnum * s.Bn + lBdUs_in, lBdU = -lnum * s.Bn;
    ls.Bn += lBdUs * SM + lBdU * s.un;
    lSM += lBdUs * s.Bn;
    lBts += lBdUs * uts;
    luts += lBdUs * Bts;
    lBws += lBdUs * uws;
    luws += lBdUs * Bws;
    ls.un += lBdU * s.Bn;
    ls.Bt += lBdU * s.ut;
    ls.ut += lBdU * s.Bt;
    ls.Bw += lBdU * s.uw;
    ls.uw += lBdU * s.Bw;
}

// Double-star tangential state (head/riemann.hpp:375-413), a = sqrt(rho*_L),
// b = sqrt(rho*_R) with a + b >= 1e-14.
template <typename R>
struct Tan4 {
    R ut, uw, Bt, Bw;
};

template <typename R>
ADJ_HD Tan4<R> dstar(R a, R b, R sg, const Tan4<R>& L, const Tan4<R>& Rr) {
    const R iD = R(1) / (a + b);
    return Tan4<R>{(a * L.ut + b * Rr.ut + sg * (Rr.Bt - L.Bt)) * iD, (a * L.uw + b * Rr.uw + sg * (Rr.Bw - L.Bw)) * iD,
                   (a * Rr.Bt + b * L.Bt + sg * a * b * (Rr.ut - L.ut)) * iD,
                   (a * Rr.Bw + b * L.Bw + sg * a * b * (Rr.uw - L.uw)) * iD};
}

template <typename R>
ADJ_HD void dstar_adj(R a, R b, R sg, const Tan4<R>& L, const Tan4<R>& Rr, const Tan4<R>& l, R& la, R& lb,
                      Tan4<R>& lL, Tan4<R>& lR) {
    const R iD = R(1) / (a + b);
    const R nut = a * L.ut + b * Rr.ut + sg * (Rr.Bt - L.Bt);
    const R nuw = a * L.uw + b * Rr.uw + sg * (Rr.Bw - L.Bw);
    const R nBt = a * Rr.Bt + b * L.Bt + sg * a * b * (Rr.ut - L.ut);
    const R nBw = a * Rr.Bw + b * L.Bw + sg * a * b * (Rr.uw - L.uw);
    const R lD = -(l.ut * nut + l.uw * nuw + l.Bt * nBt + l.Bw * nBw) * iD * iD;
    la += lD;
    lb += lD;
    const R put = l.ut * iD, puw = l.uw * iD, pBt = l.Bt * iD, pBw = l.Bw * iD;
    la += put * L.ut + puw * L.uw + pBt * (Rr.Bt + sg * b * (Rr.ut - L.ut)) + pBw * (Rr.Bw + sg * b * (Rr.uw - L.uw));
    lb += put * Rr.ut + puw * Rr.uw + pBt * (L.Bt + sg * a * (Rr.ut - L.ut)) + pBw * (L.Bw + sg * a * (Rr.uw - L.uw));
    lL.ut += put * a - pBt * sg * a * b;
    lR.ut += put * b + pBt * sg * a * b;
    lL.uw += puw * a - pBw * sg * a * b;
    lR.uw += puw * b + pBw * sg * a * b;
    lR.Bt += put * sg + pBt * a;
    lL.Bt += -put * sg + pBt * b;
    lR.Bw += puw * sg + pBw * a;
    lL.Bw += -puw * sg + pBw * b;
}

// Conserved star state in the x frame.
template <typename R>
ADJ_HD void star_u(R rhos, R SM, const Tan4<R>& t, R Bn, R Es, R psiM, R* U) {
    U[RHO] = rhos; U[MX] = rhos * SM; U[MY] = rhos * t.ut; U[MZ] = rhos * t.uw;
    U[BX] = Bn; U[BY] = t.Bt; U[BZ] = t.Bw; U[EN] = Es; U[PSI] = psiM;
}

template <typename R>
ADJ_HD void star_u_adj(R rhos, R SM, const Tan4<R>& t, const R* lU, R& lrhos, R& lSM, Tan4<R>& lt, R& lBn, R& lEs,
                       R& lpsiM) {
    lrhos += lU[RHO] + lU[MX] * SM + lU[MY] * t.ut + lU[MZ] * t.uw;
    lSM += lU[MX] * rhos;
    lt.ut += lU[MY] * rhos;
    lt.uw += lU[MZ] * rhos;
    lBn += lU[BX];
    lt.Bt += lU[BY];
    lt.Bw += lU[BZ];
    lEs += lU[EN];
    lpsiM += lU[PSI];
}

// Region of an HLLD face after its fallbacks: -1 = HLL, 0 = F_L, 1 = F_R,
// 2 = L*, 3 = L**, 4 = R*, 5 = R**.  Fills the quantities the branches use.
template <typename R>
struct HlldState {
    R WL[NV], WR[NV];
    HSide<R> L, Rr;
    R cfL, cfR, SL, SR, ptL, ptR, SM, rhoLs, rhoRs, ptstar, sqL, sqR, psiM;
    int region;
};

template <typename R>
ADJ_HD void hlld_state(const R* UL, const R* UR, R ch, R g, HlldState<R>& h) {
    c2p(UL, g, h.WL);
    c2p(UR, g, h.WR);
    h.region = -1;
    if (!riemann_ok(h.WL) || !riemann_ok(h.WR)) return;
    h.L = hside(h.WL, UL);
    h.Rr = hside(h.WR, UR);
    const HSide<R>& L = h.L;
    const HSide<R>& Rr = h.Rr;
    h.cfL = fast(h.WL, g);
    h.cfR = fast(h.WR, g);
    h.SL = fmin(L.un - h.cfL, Rr.un - h.cfR);
    h.SR = fmax(L.un + h.cfL, Rr.un + h.cfR);
    if (fabs(h.SR - h.SL) < R(1e-14)) return;
    h.ptL = L.p + R(0.5) * (L.Bn * L.Bn + L.Bt * L.Bt + L.Bw * L.Bw);
    h.ptR = Rr.p + R(0.5) * (Rr.Bn * Rr.Bn + Rr.Bt * Rr.Bt + Rr.Bw * Rr.Bw);
    const R numer = (h.SR - Rr.un) * Rr.rho * Rr.un - (h.SL - L.un) * L.rho * L.un + h.ptL - h.ptR;
    const R denom = (h.SR - Rr.un) * Rr.rho - (h.SL - L.un) * L.rho;
    if (fabs(denom) < R(1e-14)) return;
    h.SM = numer / denom;
    h.rhoLs = L.rho * (h.SL - L.un) / (h.SL - h.SM);
    h.rhoRs = Rr.rho * (h.SR - Rr.un) / (h.SR - h.SM);
    if (h.rhoLs <= R(0) || h.rhoRs <= R(0) || !isfinite(h.rhoLs) || !isfinite(h.rhoRs)) return;
    if (h.SL >= R(0)) { h.region = 0; return; }
    if (h.SR <= R(0)) { h.region = 1; return; }
    h.ptstar = h.ptL + L.rho * (h.SL - L.un) * (h.SM - L.un);
    h.sqL = sqrt(h.rhoLs);
    h.sqR = sqrt(h.rhoRs);
    h.psiM = R(0.5) * (L.psi + Rr.psi) - R(0.5) * ch * (Rr.Bn - L.Bn);
    if (h.SM >= R(0)) h.region = (h.SM - fabs(L.Bn) / h.sqL >= R(0)) ? 2 : 3;
    else h.region = (h.SM + fabs(Rr.Bn) / h.sqR <= R(0)) ? 4 : 5;
}

template <typename R>
ADJ_HD void hlld(const R* UL, const R* UR, R ch, R g, R* F) {
    HlldState<R> h;
    hlld_state(UL, UR, ch, g, h);
    if (h.region < 0) { hll(UL, UR, ch, g, F); return; }
    if (h.region == 0) { flux(h.WL, ch, g, F); return; }
    if (h.region == 1) { flux(h.WR, ch, g, F); return; }
    const bool left = h.region <= 3;
    const HSide<R>& s = left ? h.L : h.Rr;
    const R S = left ? h.SL : h.SR, pt = left ? h.ptL : h.ptR, rhos = left ? h.rhoLs : h.rhoRs;
    const R* Uside = left ? UL : UR;
    Tan4<R> ts;
    star_tan(s, S, h.SM, ts.ut, ts.uw, ts.Bt, ts.Bw);
    R BdUs;
    const R Es = star_energy(s, pt, S, h.SM, h.ptstar, ts.ut, ts.uw, ts.Bt, ts.Bw, BdUs);
    R Us[NV], Fs[NV];
    star_u(rhos, h.SM, ts, s.Bn, Es, h.psiM, Us);
    flux(left ? h.WL : h.WR, ch, g, Fs);
    if (h.region == 2 || h.region == 4) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = Fs[k] + S * (Us[k] - Uside[k]);
        return;
    }
    const R Sss = left ? h.SM - fabs(h.L.Bn) / h.sqL : h.SM + fabs(h.Rr.Bn) / h.sqR;
    Tan4<R> tL, tR;  // both single-star states
    star_tan(h.L, h.SL, h.SM, tL.ut, tL.uw, tL.Bt, tL.Bw);
    star_tan(h.Rr, h.SR, h.SM, tR.ut, tR.uw, tR.Bt, tR.Bw);
    const R sg = (h.L.Bn >= R(0)) ? R(1) : R(-1);
    Tan4<R> tss = ts;
    R Ess = Es;
    if (fabs(h.sqL + h.sqR) >= R(1e-14)) {
        tss = dstar(h.sqL, h.sqR, sg, tL, tR);
        const R BdUss = s.Bn * h.SM + tss.Bt * tss.ut + tss.Bw * tss.uw;
        Ess = left ? Es - h.sqL * sg * (BdUss - BdUs) : Es + h.sqR * sg * (BdUss - BdUs);
    }
    R Uss[NV];
    star_u(rhos, h.SM, tss, s.Bn, Ess, h.psiM, Uss);
#pragma unroll
    for (int k = 0; k < NV; ++k) F[k] = Fs[k] + S * (Us[k] - Uside[k]) + Sss * (Uss[k] - Us[k]);
}

template <typename R>
ADJ_HD void hlld_adj(const R* UL, const R* UR, R ch, R g, const R* lF, R* lUL, R* lUR, R& lch) {
    HlldState<R> h;
    hlld_state(UL, UR, ch, g, h);
    if (h.region < 0) { hll_adj(UL, UR, ch, g, lF, lUL, lUR, lch); return; }
    R lWL[NV], lWR[NV];
    zero(lWL);
    zero(lWR);
    if (h.region <= 1) {
        flux_adj(h.region == 0 ? h.WL : h.WR, ch, g, lF, h.region == 0 ? lWL : lWR, lch);
        c2p_adj(UL, h.WL, g, lWL, lUL);
        c2p_adj(UR, h.WR, g, lWR, lUR);
        return;
    }
    const HSide<R>& L = h.L;
    const HSide<R>& Rr = h.Rr;
    const bool left = h.region <= 3;
    const HSide<R>& s = left ? L : Rr;
    const R S = left ? h.SL : h.SR, pt = left ? h.ptL : h.ptR, rhos = left ? h.rhoLs : h.rhoRs;
    const R* Uside = left ? UL : UR;
    R* lUside = left ? lUL : lUR;
    // ---- forward values of the selected branch
    Tan4<R> ts;
    star_tan(s, S, h.SM, ts.ut, ts.uw, ts.Bt, ts.Bw);
    R BdUs;
    const R Es = star_energy(s, pt, S, h.SM, h.ptstar, ts.ut, ts.uw, ts.Bt, ts.Bw, BdUs);
    R Us[NV];
    star_u(rhos, h.SM, ts, s.Bn, Es, h.psiM, Us);
    // ---- cotangents of the intermediates
    HSide<R> lL{}, lR{};
    HSide<R>& ls = left ? lL : lR;
    R lSL = R(0), lSR = R(0), lSM = R(0), lrhoLs = R(0), lrhoRs = R(0), lptL = R(0), lptR = R(0);
    R lptstar = R(0), lsqL = R(0), lsqR = R(0), lpsiM = R(0);
    R& lS = left ? lSL : lSR;
    R& lpt = left ? lptL : lptR;
    R& lrhos = left ? lrhoLs : lrhoRs;
    R lFs[NV], lUs[NV];
    Tan4<R> lts{};
    R lEs = R(0), lBdUs_extra = R(0), lBn_side = R(0);
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        lFs[k] = lF[k];
        lS += lF[k] * (Us[k] - Uside[k]);
        lUside[k] -= S * lF[k];  // direct conserved dependence
    }
    if (h.region == 2 || h.region == 4) {
#pragma unroll
        for (int k = 0; k < NV; ++k) lUs[k] = S * lF[k];
    } else {
        const R Sss = left ? h.SM - fabs(L.Bn) / h.sqL : h.SM + fabs(Rr.Bn) / h.sqR;
        Tan4<R> tL, tR;
        star_tan(L, h.SL, h.SM, tL.ut, tL.uw, tL.Bt, tL.Bw);
        star_tan(Rr, h.SR, h.SM, tR.ut, tR.uw, tR.Bt, tR.Bw);
        const R sg = (L.Bn >= R(0)) ? R(1) : R(-1);
        const bool ds = fabs(h.sqL + h.sqR) >= R(1e-14);
        Tan4<R> tss = ts;
        R Ess = Es, BdUss = R(0);
        if (ds) {
            tss = dstar(h.sqL, h.sqR, sg, tL, tR);
            BdUss = s.Bn * h.SM + tss.Bt * tss.ut + tss.Bw * tss.uw;
            Ess = left ? Es - h.sqL * sg * (BdUss - BdUs) : Es + h.sqR * sg * (BdUss - BdUs);
        }
        R Uss[NV], lUss[NV];
        star_u(rhos, h.SM, tss, s.Bn, Ess, h.psiM, Uss);
        R lSss = R(0);
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            lUs[k] = (S - Sss) * lF[k];
            lUss[k] = Sss * lF[k];
            lSss += lF[k] * (Uss[k] - Us[k]);
        }
        // Sss = SM -/+ |Bn_side| / sq_side
        lSM += lSss;
        const R sgn_side = (s.Bn >= R(0)) ? R(1) : R(-1);
        if (left) {
            lBn_side -= lSss * sgn_side / h.sqL;
            lsqL += lSss * fabs(L.Bn) / (h.sqL * h.sqL);
        } else {
            lBn_side += lSss * sgn_side / h.sqR;
            lsqR -= lSss * fabs(Rr.Bn) / (h.sqR * h.sqR);
        }
        // Uss = star(rhos, SM, tss, Bn, Ess, psiM)
        Tan4<R> ltss{};
        R lEss = R(0);
        star_u_adj(rhos, h.SM, tss, lUss, lrhos, lSM, ltss, lBn_side, lEss, lpsiM);
        if (ds) {
            lEs += lEss;
            R lBdUss;
            if (left) {
                lsqL -= sg * (BdUss - BdUs) * lEss;
                lBdUss = -h.sqL * sg * lEss;
                lBdUs_extra += h.sqL * sg * lEss;
            } else {
                lsqR += sg * (BdUss - BdUs) * lEss;
                lBdUss = h.sqR * sg * lEss;
                lBdUs_extra -= h.sqR * sg * lEss;
            }
            lBn_side += lBdUss * h.SM;
            lSM += lBdUss * s.Bn;
            ltss.Bt += lBdUss * tss.ut;
            ltss.ut += lBdUss * tss.Bt;
            ltss.Bw += lBdUss * tss.uw;
            ltss.uw += lBdUss * tss.Bw;
            Tan4<R> ltL{}, ltR{};
            dstar_adj(h.sqL, h.sqR, sg, tL, tR, ltss, lsqL, lsqR, ltL, ltR);
            // the side's own single-star state is tL or tR: its cotangent joins lts below
            Tan4<R>& lown = left ? ltL : ltR;
            lts.ut += lown.ut; lts.uw += lown.uw; lts.Bt += lown.Bt; lts.Bw += lown.Bw;
            Tan4<R>& loth = left ? ltR : ltL;
            const HSide<R>& o = left ? Rr : L;
            HSide<R>& lo = left ? lR : lL;
            star_tan_adj(o, left ? h.SR : h.SL, h.SM, loth.ut, loth.uw, loth.Bt, loth.Bw, lo, left ? lSR : lSL, lSM);
        } else {
            lEs += lEss;
            lts.ut += ltss.ut; lts.uw += ltss.uw; lts.Bt += ltss.Bt; lts.Bw += ltss.Bw;
        }
    }
    // Us = star(rhos, SM, ts, Bn, Es, psiM)
    star_u_adj(rhos, h.SM, ts, lUs, lrhos, lSM, lts, lBn_side, lEs, lpsiM);
    // Es and the single-star tangential state of the side
    star_energy_adj(s, pt, S, h.SM, h.ptstar, ts.ut, ts.uw, ts.Bt, ts.Bw, Es, lEs, lBdUs_extra, ls, lpt, lS, lSM,
                    lptstar, lts.ut, lts.uw, lts.Bt, lts.Bw);
    star_tan_adj(s, S, h.SM, lts.ut, lts.uw, lts.Bt, lts.Bw, ls, lS, lSM);
    ls.Bn += lBn_side;
    // Fs = flux(W_side)
    flux_adj(left ? h.WL : h.WR, ch, g, lFs, left ? lWL : lWR, lch);
    // psiM = (psiL + psiR) / 2 - ch (BnR - BnL) / 2
    lL.psi += R(0.5) * lpsiM;
    lR.psi += R(0.5) * lpsiM;
    lch -= R(0.5) * (Rr.Bn - L.Bn) * lpsiM;
    lR.Bn -= R(0.5) * ch * lpsiM;
    lL.Bn += R(0.5) * ch * lpsiM;
    // sq = sqrt(rho*)
    lrhoLs += lsqL / (R(2) * h.sqL);
    lrhoRs += lsqR / (R(2) * h.sqR);
    // ptstar = ptL + rhoL (SL - unL) (SM - unL)
    {
        const R qL = h.SL - L.un, e = h.SM - L.un;
        lptL += lptstar;
        lL.rho += lptstar * qL * e;
        const R lqL = lptstar * L.rho * e;
        lSM += lptstar * L.rho * qL;
        lL.un -= lptstar * L.rho * qL;
        lSL += lqL;
        lL.un -= lqL;
    }
    // rho*_X = rho_X (S_X - un_X) / (S_X - SM)
    {
        const R qL = h.SL - L.un, dL = h.SL - h.SM;
        lL.rho += lrhoLs * qL / dL;
        const R lqL = lrhoLs * L.rho / dL, ldL = -lrhoLs * h.rhoLs / dL;
        lSL += lqL + ldL;
        lL.un -= lqL;
        lSM -= ldL;
        const R qR = h.SR - Rr.un, dR = h.SR - h.SM;
        lR.rho += lrhoRs * qR / dR;
        const R lqR = lrhoRs * Rr.rho / dR, ldR = -lrhoRs * h.rhoRs / dR;
        lSR += lqR + ldR;
        lR.un -= lqR;
        lSM -= ldR;
    }
    // SM = numer / denom
    {
        const R qL = h.SL - L.un, qR = h.SR - Rr.un;
        const R denom = qR * Rr.rho - qL * L.rho;
        const R lnum = lSM / denom, lden = -lSM * h.SM / denom;
        // numer = qR rhoR unR - qL rhoL unL + ptL - ptR ; denom = qR rhoR - qL rhoL
        const R lqR = lnum * Rr.rho * Rr.un + lden * Rr.rho;
        const R lqL = -lnum * L.rho * L.un - lden * L.rho;
        lR.rho += lnum * qR * Rr.un + lden * qR;
        lR.un += lnum * qR * Rr.rho;
        lL.rho -= lnum * qL * L.un + lden * qL;
        lL.un -= lnum * qL * L.rho;
        lptL += lnum;
        lptR -= lnum;
        lSR += lqR;
        lR.un -= lqR;
        lSL += lqL;
        lL.un -= lqL;
    }
    // pt = p + |B|^2 / 2
    lL.p += lptL; lL.Bn += lptL * L.Bn; lL.Bt += lptL * L.Bt; lL.Bw += lptL * L.Bw;
    lR.p += lptR; lR.Bn += lptR * Rr.Bn; lR.Bt += lptR * Rr.Bt; lR.Bw += lptR * Rr.Bw;
    // SL = min(unL - cfL, unR - cfR), SR = max(unL + cfL, unR + cfR)
    R lcfL = R(0), lcfR = R(0);
    if (L.un - h.cfL <= Rr.un - h.cfR) { lL.un += lSL; lcfL -= lSL; }
    else { lR.un += lSL; lcfR -= lSL; }
    if (L.un + h.cfL >= Rr.un + h.cfR) { lL.un += lSR; lcfL += lSR; }
    else { lR.un += lSR; lcfR += lSR; }
    hside_scatter(lL, lWL, lUL);
    hside_scatter(lR, lWR, lUR);
    fast_adj(h.WL, g, lcfL, lWL);
    fast_adj(h.WR, g, lcfR, lWR);
    c2p_adj(UL, h.WL, g, lWL, lUL);
    c2p_adj(UR, h.WR, g, lWR, lUR);
}

// GLM overwrite of the psi / normal-field flux (head/riemann.hpp:544-563).
template <typename R>
ADJ_HD void glm_fix(const R* UL, const R* UR, R ch, R* F) {
    if (ch <= R(0)) return;
    const R Bns = R(0.5) * (UL[BX] + UR[BX]) - R(0.5) / ch * (UR[PSI] - UL[PSI]);
    const R psis = R(0.5) * (UL[PSI] + UR[PSI]) - R(0.5) * ch * (UR[BX] - UL[BX]);
    F[BX] = psis;
    F[PSI] = ch * ch * Bns;
}

// Face flux of the dispatcher (head/riemann.hpp:568-592): HLL as is; HLLD with
// the non-finite fallback to HLL and then the GLM overwrite.
template <int SOLVER, typename R>
ADJ_HD void face(const R* UL, const R* UR, R ch, R g, R* F) {
    if (SOLVER == HLL) { hll(UL, UR, ch, g, F); return; }
    hlld(UL, UR, ch, g, F);
    if (!isfinite(F[RHO]) || !isfinite(F[EN]) || !isfinite(F[BX]) || !isfinite(F[PSI])) {
        hll(UL, UR, ch, g, F);
        return;
    }
    glm_fix(UL, UR, ch, F);
}

template <int SOLVER, typename R>
ADJ_HD void face_adj(const R* UL, const R* UR, R ch, R g, const R* lF, R* lUL, R* lUR, R& lch) {
    if (SOLVER == HLL) { hll_adj(UL, UR, ch, g, lF, lUL, lUR, lch); return; }
    R F[NV];
    hlld(UL, UR, ch, g, F);
    if (!isfinite(F[RHO]) || !isfinite(F[EN]) || !isfinite(F[BX]) || !isfinite(F[PSI])) {
        hll_adj(UL, UR, ch, g, lF, lUL, lUR, lch);
        return;
    }
    R lH[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) lH[k] = lF[k];
    if (ch > R(0)) {
        lH[BX] = R(0);
        lH[PSI] = R(0);
        const R Bns = R(0.5) * (UL[BX] + UR[BX]) - R(0.5) / ch * (UR[PSI] - UL[PSI]);
        const R lps = lF[BX], lBns = lF[PSI] * ch * ch;
        lch += lF[PSI] * R(2) * ch * Bns;
        lUL[PSI] += R(0.5) * lps + R(0.5) / ch * lBns;
        lUR[PSI] += R(0.5) * lps - R(0.5) / ch * lBns;
        lUL[BX] += R(0.5) * ch * lps + R(0.5) * lBns;
        lUR[BX] += -R(0.5) * ch * lps + R(0.5) * lBns;
        lch += -R(0.5) * (UR[BX] - UL[BX]) * lps + R(0.5) * (UR[PSI] - UL[PSI]) / (ch * ch) * lBns;
    }
    hlld_adj(UL, UR, ch, g, lH, lUL, lUR, lch);
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
