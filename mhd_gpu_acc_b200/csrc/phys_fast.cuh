// phys_fast.cuh -- FP32-bulk GLM-MHD physics for the fast step.
//
// Same algorithm as the FP64 path (reference head/physics.hpp, head/riemann.hpp,
// src/cpu/solver_cpu.cpp:88-119), restructured for single precision:
//   * a reconstructed side state carries both its conserved (U) and primitive
//     (W) form, so cons_to_prim runs once per state instead of once per use,
//     and physical fluxes are evaluated from (U, W) directly;
//   * the pressure recovery p = (g-1)(E - rho|u|^2/2 - |B|^2/2) is computed
//     in FP32 unless the internal energy is a small fraction of E (low-beta
//     or hypersonic cells), where cancellation would cost more than FP32's
//     24 bits; those cells take a flagged FP64 branch;
//   * the translation unit is built with --use_fast_math (approximate
//     reciprocal / square root, FMA contraction).
// Accuracy is checked against the FP64 path per field (relative L1 / Linf).
#pragma once

#include "mhd_common.cuh"

namespace mhd {
namespace fast {

constexpr float kRhoFloor = 1.0e-12f;  // src/cpu/solver_cpu.cpp:19
constexpr float kPFloor = 1.0e-12f;    // src/cpu/solver_cpu.cpp:20
// Internal energy below this fraction of E takes the FP64 pressure branch.
constexpr float kLowBetaFrac = 0.02f;

// x * 0 is 0 for finite x and NaN for an infinity or a NaN, so an FMA chain of
// the values times zero tells whether all are finite with FMA-pipe work and a
// single comparison (instead of one ALU test per value).
__device__ __forceinline__ bool both_finite(float a, float b) { return fmaf(a, 0.0f, b * 0.0f) == 0.0f; }

// A face-side state: [0, 9) U, [9, 18) W and two values of the x-sweep.
// [18]: 1 when the reconstruction's test of the advanced state has already
// shown W physical in is_physical's sense (rho and p above their floors, every
// value finite), which implies riemann_physical, so the solver skips that test
// (0: not known, test it -- a fallback state, a state made by PH::side, and
// every y-sweep state).  [19]: the fast magnetosonic speed of W in x, which
// the reconstruction computes for both faces of a cell at once on paired FP32
// instructions (x 0.514 -> 0.506 ms at 4096^2).  The two ride in the fifth
// 16-byte slot of the x-sweep's ring entry, which has room for them.  The
// y-sweep, at its register limit, carries U and W only (NSY) and its solver
// computes the speed: with both values its single-grid sweep measured 0.565
// -> 0.570 ms, and the batched y-sweep 8.95 -> 9.69 ms per step.
struct Side {
    float v[2 * NV + 2];
    __device__ __forceinline__ float* U() { return v; }
    __device__ __forceinline__ float* W() { return v + NV; }
    __device__ __forceinline__ const float* U() const { return v; }
    __device__ __forceinline__ const float* W() const { return v + NV; }
    __device__ __forceinline__ bool known_physical() const { return v[2 * NV] != 0.0f; }
    __device__ __forceinline__ float cf() const { return v[2 * NV + 1]; }
};

template <int DIR>
__device__ __forceinline__ float fast_speed(const float* W, float g);
// The solvers' fast magnetosonic speed of a face-side state.
template <int DIR>
__device__ __forceinline__ float side_speed(const Side& S, float g) {
    return (DIR == 0) ? S.cf() : fast_speed<DIR>(S.W(), g);
}

// cons_to_prim with the flagged FP64 pressure recovery.
__device__ __forceinline__ void c2p(const float* U, float g, float* W) {
    const float inv_rho = 1.0f / U[RHO];
    const float ux = U[MX] * inv_rho, uy = U[MY] * inv_rho, uz = U[MZ] * inv_rho;
    const float B2 = U[BX] * U[BX] + U[BY] * U[BY] + U[BZ] * U[BZ];
    const float ke = 0.5f * (U[MX] * ux + U[MY] * uy + U[MZ] * uz);
    float eint = U[EN] - ke - 0.5f * B2;
    if (eint < kLowBetaFrac * U[EN]) {
        const double mx = U[MX], my = U[MY], mz = U[MZ], r = U[RHO];
        const double bx = U[BX], by = U[BY], bz = U[BZ];
        const double ke_d = 0.5 * (mx * mx + my * my + mz * mz) / r;
        eint = (float)((double)U[EN] - ke_d - 0.5 * (bx * bx + by * by + bz * bz));
    }
    W[RHO] = U[RHO]; W[PU] = ux; W[PV] = uy; W[PW] = uz;
    W[BX] = U[BX]; W[BY] = U[BY]; W[BZ] = U[BZ]; W[PP] = (g - 1.0f) * eint; W[PSI] = U[PSI];
}

__device__ __forceinline__ void p2c(const float* W, float g, float* U) {
    const float B2 = W[BX] * W[BX] + W[BY] * W[BY] + W[BZ] * W[BZ];
    const float ke = 0.5f * W[RHO] * (W[PU] * W[PU] + W[PV] * W[PV] + W[PW] * W[PW]);
    U[RHO] = W[RHO]; U[MX] = W[RHO] * W[PU]; U[MY] = W[RHO] * W[PV]; U[MZ] = W[RHO] * W[PW];
    U[BX] = W[BX]; U[BY] = W[BY]; U[BZ] = W[BZ];
    U[EN] = W[PP] / (g - 1.0f) + ke + 0.5f * B2;
    U[PSI] = W[PSI];
}

// GLM-MHD physical flux (head/physics.hpp:105-164) from a consistent (U, W) pair.
template <int DIR>
__device__ __forceinline__ void flux(const float* U, const float* W, float ch, float* F) {
    const float B2 = W[BX] * W[BX] + W[BY] * W[BY] + W[BZ] * W[BZ];
    const float pt = W[PP] + 0.5f * B2;
    const float uB = W[PU] * W[BX] + W[PV] * W[BY] + W[PW] * W[BZ];
    if (DIR == 0) {
        F[0] = U[MX];
        F[1] = U[MX] * W[PU] + pt - W[BX] * W[BX];
        F[2] = U[MX] * W[PV] - W[BX] * W[BY];
        F[3] = U[MX] * W[PW] - W[BX] * W[BZ];
        F[4] = W[PSI];
        F[5] = W[BY] * W[PU] - W[BX] * W[PV];
        F[6] = W[BZ] * W[PU] - W[BX] * W[PW];
        F[7] = (U[EN] + pt) * W[PU] - W[BX] * uB;
        F[8] = ch * ch * W[BX];
    } else {
        F[0] = U[MY];
        F[1] = U[MY] * W[PU] - W[BY] * W[BX];
        F[2] = U[MY] * W[PV] + pt - W[BY] * W[BY];
        F[3] = U[MY] * W[PW] - W[BY] * W[BZ];
        F[4] = W[BX] * W[PV] - W[BY] * W[PU];
        F[5] = W[PSI];
        F[6] = W[BZ] * W[PV] - W[BY] * W[PW];
        F[7] = (U[EN] + pt) * W[PV] - W[BY] * uB;
        F[8] = ch * ch * W[BY];
    }
}

// fast magnetosonic speed (head/physics.hpp:175-191)
template <int DIR>
__device__ __forceinline__ float fast_speed(const float* W, float g) {
    const float inv_rho = 1.0f / W[RHO];
    const float a2 = g * W[PP] * inv_rho;
    const float b2 = (W[BX] * W[BX] + W[BY] * W[BY] + W[BZ] * W[BZ]) * inv_rho;
    const float Bn = (DIR == 0) ? W[BX] : W[BY];
    const float bn2 = Bn * Bn * inv_rho;
    const float s = a2 + b2;
    const float disc = s * s - 4.0f * a2 * bn2;
    return sqrtf(0.5f * (s + sqrtf(fmaxf(disc, 0.0f))));
}

__device__ __forceinline__ bool riemann_physical(const float* W) {
    return both_finite(W[RHO], W[PP]) && W[RHO] > 0.0f && W[PP] > 0.0f;
}
__device__ __forceinline__ bool riemann_physical(const Side& S) {
    if (S.known_physical()) return true;
    return riemann_physical(S.W());
}

template <int DIR>
__device__ __forceinline__ void rotate(const float* W, float& un, float& ut, float& uw, float& Bn, float& Bt,
                                       float& Bw) {
    if (DIR == 0) { un = W[PU]; ut = W[PV]; uw = W[PW]; Bn = W[BX]; Bt = W[BY]; Bw = W[BZ]; }
    else          { un = W[PV]; ut = W[PU]; uw = W[PW]; Bn = W[BY]; Bt = W[BX]; Bw = W[BZ]; }
}

template <int DIR>
__device__ __forceinline__ void build_star(float rhos, float uns, float uts, float uws, float Bns, float Bts,
                                           float Bws, float Es, float psis, float* U) {
    U[RHO] = rhos;
    if (DIR == 0) {
        U[MX] = rhos * uns; U[MY] = rhos * uts; U[MZ] = rhos * uws;
        U[BX] = Bns; U[BY] = Bts; U[BZ] = Bws;
    } else {
        U[MX] = rhos * uts; U[MY] = rhos * uns; U[MZ] = rhos * uws;
        U[BX] = Bts; U[BY] = Bns; U[BZ] = Bws;
    }
    U[EN] = Es; U[PSI] = psis;
}

// hll_flux (head/riemann.hpp:70-107)
template <int DIR>
__device__ __forceinline__ void hll(const Side& L, const Side& R, float ch, float g, float* F) {
    float FL[NV], FR[NV];
    flux<DIR>(L.U(), L.W(), ch, FL);
    flux<DIR>(R.U(), R.W(), ch, FR);
    if (!riemann_physical(L) || !riemann_physical(R)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = 0.5f * (FL[k] + FR[k]);
        return;
    }
    const float cfL = side_speed<DIR>(L, g), cfR = side_speed<DIR>(R, g);
    const float unL = (DIR == 0) ? L.W()[PU] : L.W()[PV];
    const float unR = (DIR == 0) ? R.W()[PU] : R.W()[PV];
    const float SL = fminf(fminf(unL - cfL, unR - cfR), -ch);
    const float SR = fmaxf(fmaxf(unL + cfL, unR + cfR), ch);
    if (SL >= 0.0f) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = FL[k];
        return;
    }
    if (SR <= 0.0f) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = FR[k];
        return;
    }
    const float denom = SR - SL;
    if (fabsf(denom) < 1.0e-14f) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = 0.5f * (FL[k] + FR[k]);
        return;
    }
    const float inv = 1.0f / denom;
    const float SLSR = SL * SR;
#pragma unroll
    for (int k = 0; k < NV; ++k) F[k] = inv * (SR * FL[k] - SL * FR[k] + SLSR * (R.U()[k] - L.U()[k]));
}

// hllc_flux (head/riemann.hpp:122-241)
template <int DIR>
__device__ __forceinline__ bool hllc_star(const Side& L, const Side& R, float ch, float g, float* F) {
    const float* VL = L.W();
    const float* VR = R.W();
    if (!riemann_physical(L) || !riemann_physical(R)) return false;
    const float rhoL = VL[RHO], rhoR = VR[RHO], pL = VL[PP], pR = VR[PP];
    float unL, unR, utL, utR, uwL, uwR, BnL, BnR, BtL, BtR, BwL, BwR;
    rotate<DIR>(VL, unL, utL, uwL, BnL, BtL, BwL);
    rotate<DIR>(VR, unR, utR, uwR, BnR, BtR, BwR);
    const float cfL = side_speed<DIR>(L, g), cfR = side_speed<DIR>(R, g);
    const float SL = fminf(unL - cfL, unR - cfR);
    const float SR = fmaxf(unL + cfL, unR + cfR);
    if (SL >= 0.0f) { flux<DIR>(L.U(), VL, ch, F); return true; }
    if (SR <= 0.0f) { flux<DIR>(R.U(), VR, ch, F); return true; }
    const float ptL = pL + 0.5f * (BnL * BnL + BtL * BtL + BwL * BwL);
    const float ptR = pR + 0.5f * (BnR * BnR + BtR * BtR + BwR * BwR);
    const float numerSM = (SR - unR) * rhoR * unR - (SL - unL) * rhoL * unL + ptL - ptR;
    const float denomSM = (SR - unR) * rhoR - (SL - unL) * rhoL;
    if (fabsf(denomSM) < 1.0e-14f) return false;
    const float SM = numerSM / denomSM;
    const float rhoLs = rhoL * (SL - unL) / (SL - SM);
    const float rhoRs = rhoR * (SR - unR) / (SR - SM);
    if (rhoLs <= 0.0f || rhoRs <= 0.0f || !both_finite(rhoLs, rhoRs)) return false;
    const float psiM = 0.5f * (VL[PSI] + VR[PSI]) - 0.5f * ch * (BnR - BnL);
    float Us[NV], Fs[NV];
    if (SM >= 0.0f) {
        const float ptLs = ptL + rhoL * (SL - unL) * (SM - unL);
        const float ELs = ((SL - unL) * L.U()[EN] - ptL * unL + ptLs * SM + BnL * (BnL * SM - BnL * unL)) / (SL - SM);
        build_star<DIR>(rhoLs, SM, utL, uwL, BnL, BtL, BwL, ELs, psiM, Us);
        flux<DIR>(L.U(), VL, ch, Fs);
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = Fs[k] + SL * (Us[k] - L.U()[k]);
    } else {
        const float ptRs = ptR + rhoR * (SR - unR) * (SM - unR);
        const float ERs = ((SR - unR) * R.U()[EN] - ptR * unR + ptRs * SM + BnR * (BnR * SM - BnR * unR)) / (SR - SM);
        build_star<DIR>(rhoRs, SM, utR, uwR, BnR, BtR, BwR, ERs, psiM, Us);
        flux<DIR>(R.U(), VR, ch, Fs);
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = Fs[k] + SR * (Us[k] - R.U()[k]);
    }
    return true;
}

// Single-star state of one side (head/riemann.hpp:340-373), with the FP32
// degeneracy test of star_degenerate.
__device__ __forceinline__ void star_state(float rho, float un, float ut, float uw, float Bn, float Bt, float Bw,
                                           float S, float SM, float& uts, float& uws, float& Bts, float& Bws) {
    const float d = rho * (S - un) * (S - SM) - Bn * Bn;
    if (star_degenerate(d, rho, un, S, SM, Bn)) {
        uts = ut; uws = uw; Bts = Bt; Bws = Bw;
    } else {
        const float inv_d = 1.0f / d;
        const float a = Bn * (SM - un) * inv_d;
        const float b = (rho * (S - un) * (S - un) - Bn * Bn) * inv_d;
        uts = ut - Bt * a;
        uws = uw - Bw * a;
        Bts = Bt * b;
        Bws = Bw * b;
    }
}

// hlld_flux (head/riemann.hpp:253-480)
template <int DIR>
__device__ __forceinline__ bool hlld_star(const Side& L, const Side& R, float ch, float g, float* F) {
    const float* VL = L.W();
    const float* VR = R.W();
    if (!riemann_physical(L) || !riemann_physical(R)) return false;
    const float rhoL = VL[RHO], rhoR = VR[RHO], pL = VL[PP], pR = VR[PP];
    float unL, unR, utL, utR, uwL, uwR, BnL, BnR, BtL, BtR, BwL, BwR;
    rotate<DIR>(VL, unL, utL, uwL, BnL, BtL, BwL);
    rotate<DIR>(VR, unR, utR, uwR, BnR, BtR, BwR);
    const float cfL = side_speed<DIR>(L, g), cfR = side_speed<DIR>(R, g);
    const float SL = fminf(unL - cfL, unR - cfR);
    const float SR = fmaxf(unL + cfL, unR + cfR);
    if (fabsf(SR - SL) < 1.0e-14f) return false;
    const float ptL = pL + 0.5f * (BnL * BnL + BtL * BtL + BwL * BwL);
    const float ptR = pR + 0.5f * (BnR * BnR + BtR * BtR + BwR * BwR);
    const float numerSM = (SR - unR) * rhoR * unR - (SL - unL) * rhoL * unL + ptL - ptR;
    const float denomSM = (SR - unR) * rhoR - (SL - unL) * rhoL;
    if (fabsf(denomSM) < 1.0e-14f) return false;
    const float SM = numerSM / denomSM;
    const float rhoLs = rhoL * (SL - unL) / (SL - SM);
    const float rhoRs = rhoR * (SR - unR) / (SR - SM);
    if (rhoLs <= 0.0f || rhoRs <= 0.0f || !both_finite(rhoLs, rhoRs)) return false;
    if (SL >= 0.0f) { flux<DIR>(L.U(), VL, ch, F); return true; }
    if (SR <= 0.0f) { flux<DIR>(R.U(), VR, ch, F); return true; }
    const float ptstar = ptL + rhoL * (SL - unL) * (SM - unL);
    const float psiM = 0.5f * (VL[PSI] + VR[PSI]) - 0.5f * ch * (BnR - BnL);
    const float signBn = (BnL >= 0.0f) ? 1.0f : -1.0f;
    // The side that owns the face (S_M >= 0: left).  Its single-star state is
    // all a single-star face needs; the other side's star state and square
    // root are computed only for a double-star face.  The values are those of
    // the symmetric evaluation (both star states, then a selection), which
    // measured 2 % slower in both sweeps (4096^2: x 0.558 / y 0.644 ms against
    // 0.547 / 0.630 ms; early in a run most faces are single-star).
    const bool left = (SM >= 0.0f);
    const float rho_ = left ? rhoL : rhoR, un_ = left ? unL : unR, S_ = left ? SL : SR;
    const float Bn_ = left ? BnL : BnR, pt_ = left ? ptL : ptR;
    const float ut_ = left ? utL : utR, uw_ = left ? uwL : uwR, Bt_ = left ? BtL : BtR, Bw_ = left ? BwL : BwR;
    const float rhos = left ? rhoLs : rhoRs;
    float uts, uws, Bts, Bws;
    star_state(rho_, un_, ut_, uw_, Bn_, Bt_, Bw_, S_, SM, uts, uws, Bts, Bws);
    const float sq = sqrtf(rhos);
    const float* Uside = left ? L.U() : R.U();
    const float* Wside = left ? VL : VR;
    const float BdU = Bn_ * un_ + Bt_ * ut_ + Bw_ * uw_;
    const float BdUs = Bn_ * SM + Bts * uts + Bws * uws;
    const float Es = (Uside[EN] * (S_ - un_) - pt_ * un_ + ptstar * SM + Bn_ * (BdUs - BdU)) / (S_ - SM);
    float Us[NV], Fs[NV];
    build_star<DIR>(rhos, SM, uts, uws, Bn_, Bts, Bws, Es, psiM, Us);
    flux<DIR>(Uside, Wside, ch, Fs);
    const float Sstar = left ? SM - fabsf(Bn_) / sq : SM + fabsf(Bn_) / sq;
    const bool single = left ? (Sstar >= 0.0f) : (Sstar <= 0.0f);
    if (single) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = Fs[k] + S_ * (Us[k] - Uside[k]);
        return true;
    }
    // double-star state (head/riemann.hpp:375-413): the other side's star state
    float uto, uwo, Bto, Bwo;
    star_state(left ? rhoR : rhoL, left ? unR : unL, left ? utR : utL, left ? uwR : uwL, left ? BnR : BnL,
               left ? BtR : BtL, left ? BwR : BwL, left ? SR : SL, SM, uto, uwo, Bto, Bwo);
    const float sqo = sqrtf(left ? rhoRs : rhoLs);
    const float sqL = left ? sq : sqo, sqR = left ? sqo : sq;
    const float utLs = left ? uts : uto, uwLs = left ? uws : uwo, BtLs = left ? Bts : Bto, BwLs = left ? Bws : Bwo;
    const float utRs = left ? uto : uts, uwRs = left ? uwo : uws, BtRs = left ? Bto : Bts, BwRs = left ? Bwo : Bws;
    const float denom2 = sqL + sqR;
    float utss = uts, uwss = uws, Btss = Bts, Bwss = Bws, Ess = Es;
    if (fabsf(denom2) >= 1.0e-14f) {
        const float inv_d2 = 1.0f / denom2;
        utss = (sqL * utLs + sqR * utRs + signBn * (BtRs - BtLs)) * inv_d2;
        uwss = (sqL * uwLs + sqR * uwRs + signBn * (BwRs - BwLs)) * inv_d2;
        Btss = (sqL * BtRs + sqR * BtLs + signBn * sqL * sqR * (utRs - utLs)) * inv_d2;
        Bwss = (sqL * BwRs + sqR * BwLs + signBn * sqL * sqR * (uwRs - uwLs)) * inv_d2;
        const float BdUss = Bn_ * SM + Btss * utss + Bwss * uwss;
        Ess = left ? Es - sq * signBn * (BdUss - BdUs) : Es + sq * signBn * (BdUss - BdUs);
    }
    float Uss[NV];
    build_star<DIR>(rhos, SM, utss, uwss, Bn_, Btss, Bwss, Ess, psiM, Uss);
#pragma unroll
    for (int k = 0; k < NV; ++k) F[k] = Fs[k] + S_ * (Us[k] - Uside[k]) + Sstar * (Uss[k] - Us[k]);
    return true;
}

// force_flux (head/riemann.hpp:486-525)
template <int DIR>
__device__ __forceinline__ void force(const Side& L, const Side& R, float ch, float g, float* F) {
    float FL[NV], FR[NV];
    flux<DIR>(L.U(), L.W(), ch, FL);
    flux<DIR>(R.U(), R.W(), ch, FR);
    if (!riemann_physical(L) || !riemann_physical(R)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = 0.5f * (FL[k] + FR[k]);
        return;
    }
    const float cfL = side_speed<DIR>(L, g), cfR = side_speed<DIR>(R, g);
    const float unL = (DIR == 0) ? L.W()[PU] : L.W()[PV];
    const float unR = (DIR == 0) ? R.W()[PU] : R.W()[PV];
    const float alpha = fmaxf(fmaxf(fabsf(unL) + cfL, fabsf(unR) + cfR), ch);
    if (alpha < 1.0e-14f) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = 0.5f * (FL[k] + FR[k]);
        return;
    }
    float Flf[NV], Uri[NV], Wri[NV];
    const float ha = 0.5f * alpha, hia = 0.5f / alpha;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        Flf[k] = 0.5f * (FL[k] + FR[k]) - ha * (R.U()[k] - L.U()[k]);
        Uri[k] = 0.5f * (L.U()[k] + R.U()[k]) - hia * (FR[k] - FL[k]);
    }
    c2p(Uri, g, Wri);
    if (!riemann_physical(Wri)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = Flf[k];
        return;
    }
    flux<DIR>(Uri, Wri, ch, FR);
#pragma unroll
    for (int k = 0; k < NV; ++k) F[k] = 0.5f * (Flf[k] + FR[k]);
}

// apply_glm_flux (head/riemann.hpp:544-563)
template <int DIR>
__device__ __forceinline__ void glm_overwrite(float* F, const Side& L, const Side& R, float ch) {
    if (ch <= 0.0f) return;
    const float BnL = (DIR == 0) ? L.U()[BX] : L.U()[BY];
    const float BnR = (DIR == 0) ? R.U()[BX] : R.U()[BY];
    const float psiL = L.U()[PSI], psiR = R.U()[PSI];
    const float Bn_star = 0.5f * (BnL + BnR) - (0.5f / ch) * (psiR - psiL);
    const float psi_star = 0.5f * (psiL + psiR) - 0.5f * ch * (BnR - BnL);
    if (DIR == 0) F[BX] = psi_star; else F[BY] = psi_star;
    F[PSI] = ch * ch * Bn_star;
}

__device__ __forceinline__ bool flux_finite(const float* F) {
    return fmaf(F[RHO], 0.0f, fmaf(F[EN], 0.0f, fmaf(F[BX], 0.0f, F[PSI] * 0.0f))) == 0.0f;
}

// riemann_flux dispatcher (head/riemann.hpp:568-592).  HLLC and HLLD report a
// fallback instead of computing HLL themselves, so one inlined HLL serves every
// fallback: a star-state solver that gave up (the reference's solver then
// returns hll_flux, which riemann_flux still checks and, if finite, overwrites
// with the GLM psi / Bn flux) and a non-finite solver result (HLL, returned
// without the overwrite).
template <int DIR, int SOLVER>
__device__ __forceinline__ void riemann(const Side& L, const Side& R, float ch, float g, float* F) {
    if (SOLVER == HLL) { hll<DIR>(L, R, ch, g, F); return; }
    bool ok = true;
    if (SOLVER == HLLC) ok = hllc_star<DIR>(L, R, ch, g, F);
    else if (SOLVER == HLLD) ok = hlld_star<DIR>(L, R, ch, g, F);
    else force<DIR>(L, R, ch, g, F);
    bool overwrite = true;
    if (ok && !flux_finite(F)) overwrite = false;
    if (!ok || !overwrite) hll<DIR>(L, R, ch, g, F);
    if (!ok && !flux_finite(F)) overwrite = false;
    if (overwrite) glm_overwrite<DIR>(F, L, R, ch);
}

__device__ __forceinline__ float minmod(float a, float b) {
    if (a * b <= 0.0f) return 0.0f;
    return (a > 0.0f) ? fminf(a, b) : fmaxf(a, b);
}
// van Leer without a compare-and-select: ab + |ab| is 2ab where the slopes
// agree in sign and 0 where they do not; the 1e-30 keeps a + b = 0 (then also
// ab <= 0) from producing 0 / 0, and is below the rounding of any a + b that
// meets a non-zero numerator (with flush-to-zero, |a|, |b| > 1e-19 there).
// Results equal the select form bit for bit; measured x 0.548 -> 0.545 ms.
__device__ __forceinline__ float vanleer(float a, float b) {
    const float ab = a * b;
    return (ab + fabsf(ab)) / (a + b + 1.0e-30f);
}

// ---------------------------------------------------------------------------
// Packed face pairs.  A cell's MUSCL-Hancock predictor produces its left-face
// and right-face states together and treats them identically, so they are
// carried as float2 (.x = left face, .y = right face) and advanced with the
// sm_100 paired FP32 instructions (one issue slot for both faces).  Per
// component the arithmetic is the scalar code's (round-to-nearest FMA / add /
// multiply), only the contraction pattern differs.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(1.0f / a.x, 1.0f / a.y); }

// p2c of both faces.
__device__ __forceinline__ void p2c2(const float2* W, float inv_gm1, float2* U) {
    const float2 B2 = fma2(W[BZ], W[BZ], fma2(W[BY], W[BY], mul2(W[BX], W[BX])));
    const float2 v2 = fma2(W[PW], W[PW], fma2(W[PV], W[PV], mul2(W[PU], W[PU])));
    const float2 half = dup2(0.5f);
    U[RHO] = W[RHO];
    U[MX] = mul2(W[RHO], W[PU]); U[MY] = mul2(W[RHO], W[PV]); U[MZ] = mul2(W[RHO], W[PW]);
    U[BX] = W[BX]; U[BY] = W[BY]; U[BZ] = W[BZ];
    U[EN] = fma2(W[PP], dup2(inv_gm1), fma2(half, B2, mul2(mul2(half, W[RHO]), v2)));
    U[PSI] = W[PSI];
}

// GLM-MHD physical flux of both faces from consistent (U, W) pairs.
template <int DIR>
__device__ __forceinline__ void flux2(const float2* U, const float2* W, float ch, float2* F) {
    const float2 B2 = fma2(W[BZ], W[BZ], fma2(W[BY], W[BY], mul2(W[BX], W[BX])));
    const float2 pt = fma2(dup2(0.5f), B2, W[PP]);
    const float2 uB = fma2(W[PW], W[BZ], fma2(W[PV], W[BY], mul2(W[PU], W[BX])));
    const float2 c2 = dup2(ch * ch);
    if (DIR == 0) {
        F[0] = U[MX];
        F[1] = fma2(U[MX], W[PU], sub2(pt, mul2(W[BX], W[BX])));
        F[2] = fma2(U[MX], W[PV], mul2(make_float2(-W[BX].x, -W[BX].y), W[BY]));
        F[3] = fma2(U[MX], W[PW], mul2(make_float2(-W[BX].x, -W[BX].y), W[BZ]));
        F[4] = W[PSI];
        F[5] = fma2(W[BY], W[PU], mul2(make_float2(-W[BX].x, -W[BX].y), W[PV]));
        F[6] = fma2(W[BZ], W[PU], mul2(make_float2(-W[BX].x, -W[BX].y), W[PW]));
        F[7] = fma2(add2(U[EN], pt), W[PU], mul2(make_float2(-W[BX].x, -W[BX].y), uB));
        F[8] = mul2(c2, W[BX]);
    } else {
        F[0] = U[MY];
        F[1] = fma2(U[MY], W[PU], mul2(make_float2(-W[BY].x, -W[BY].y), W[BX]));
        F[2] = fma2(U[MY], W[PV], sub2(pt, mul2(W[BY], W[BY])));
        F[3] = fma2(U[MY], W[PW], mul2(make_float2(-W[BY].x, -W[BY].y), W[BZ]));
        F[4] = fma2(W[BX], W[PV], mul2(make_float2(-W[BY].x, -W[BY].y), W[PU]));
        F[5] = W[PSI];
        F[6] = fma2(W[BZ], W[PV], mul2(make_float2(-W[BY].x, -W[BY].y), W[PW]));
        F[7] = fma2(add2(U[EN], pt), W[PV], mul2(make_float2(-W[BY].x, -W[BY].y), uB));
        F[8] = mul2(c2, W[BY]);
    }
}

// Scalar FP64 pressure recovery of one face (the flagged low-internal-energy branch of c2p).
__device__ __forceinline__ float eint_fp64(float r, float mx, float my, float mz, float bx, float by, float bz, float E) {
    const double ke = 0.5 * ((double)mx * mx + (double)my * my + (double)mz * mz) / (double)r;
    return (float)((double)E - ke - 0.5 * ((double)bx * bx + (double)by * by + (double)bz * bz));
}

// c2p of both faces, with c2p's FP64 branch per face.
__device__ __forceinline__ void c2p2(const float2* U, float gm1, float2* W) {
    const float2 inv_rho = rcp2(U[RHO]);
    const float2 ux = mul2(U[MX], inv_rho), uy = mul2(U[MY], inv_rho), uz = mul2(U[MZ], inv_rho);
    const float2 B2 = fma2(U[BZ], U[BZ], fma2(U[BY], U[BY], mul2(U[BX], U[BX])));
    const float2 mu = fma2(U[MZ], uz, fma2(U[MY], uy, mul2(U[MX], ux)));
    float2 eint = fma2(dup2(-0.5f), add2(mu, B2), U[EN]);
    const float2 lim = mul2(dup2(kLowBetaFrac), U[EN]);
    if (eint.x < lim.x)
        eint.x = eint_fp64(U[RHO].x, U[MX].x, U[MY].x, U[MZ].x, U[BX].x, U[BY].x, U[BZ].x, U[EN].x);
    if (eint.y < lim.y)
        eint.y = eint_fp64(U[RHO].y, U[MX].y, U[MY].y, U[MZ].y, U[BX].y, U[BY].y, U[BZ].y, U[EN].y);
    W[RHO] = U[RHO]; W[PU] = ux; W[PV] = uy; W[PW] = uz;
    W[BX] = U[BX]; W[BY] = U[BY]; W[BZ] = U[BZ]; W[PP] = mul2(dup2(gm1), eint); W[PSI] = U[PSI];
}

// is_physical (rho and p above their floors, every value finite) of both faces.
__device__ __forceinline__ void is_physical2(const float2* V, bool& okx, bool& oky) {
    float2 z = mul2(V[0], dup2(0.0f));
#pragma unroll
    for (int k = 1; k < NV; ++k) z = fma2(V[k], dup2(0.0f), z);
    okx = V[RHO].x > kRhoFloor && V[PP].x > kPFloor && z.x == 0.0f;
    oky = V[RHO].y > kRhoFloor && V[PP].y > kPFloor && z.y == 0.0f;
}

// MUSCL-Hancock half step (src/cpu/solver_cpu.cpp:88-119; c_h in the predictor)
// on packed face pairs.  The fallbacks (first-order face values, or the
// unadvanced face state) are rare, so they are taken as a branch guarded by a
// vote of the active lanes instead of as per-component selects.
template <int DIR, int LIMITER>
__device__ __forceinline__ void reconstruct(const float* Wm, const float* Wc, const float* Wp, float dtd, float ch,
                                            float g, Side& Ls, Side& Rs) {
    float2 W[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const float a = Wc[k] - Wm[k], b = Wp[k] - Wc[k];
        const float s = (LIMITER == VANLEER) ? vanleer(a, b) : minmod(a, b);
        W[k] = make_float2(fmaf(-0.5f, s, Wc[k]), fmaf(0.5f, s, Wc[k]));
    }
    const unsigned active = __activemask();
    bool okL1, okR1;
    is_physical2(W, okL1, okR1);
    if (__any_sync(active, !(okL1 && okR1))) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            if (!okL1) W[k].x = Wc[k];
            if (!okR1) W[k].y = Wc[k];
        }
    }
    float2 U0[NV], F[NV];
    p2c2(W, 1.0f / (g - 1.0f), U0);
    flux2<DIR>(U0, W, ch, F);
    const float s = 0.5f * dtd;
    float2 U[NV], V[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const float d = s * (F[k].y - F[k].x);
        U[k] = make_float2(U0[k].x - d, U0[k].y - d);
    }
    c2p2(U, g - 1.0f, V);
    bool okL, okR;
    is_physical2(V, okL, okR);
    if (__any_sync(active, !(okL && okR))) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            if (!okL) { V[k].x = W[k].x; U[k].x = U0[k].x; }
            if (!okR) { V[k].y = W[k].y; U[k].y = U0[k].y; }
        }
    }
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        Ls.U()[k] = U[k].x; Ls.W()[k] = V[k].x;
        Rs.U()[k] = U[k].y; Rs.W()[k] = V[k].y;
    }
    if (DIR != 0) {  // the y-sweep's solver tests the states and computes their speeds itself
        Ls.v[2 * NV] = 0.0f; Ls.v[2 * NV + 1] = 0.0f;
        Rs.v[2 * NV] = 0.0f; Rs.v[2 * NV + 1] = 0.0f;
        return;
    }
    // known physical when V passed the second test (a fallback state is tested by the solver)
    Ls.v[2 * NV] = okL ? 1.0f : 0.0f;
    Rs.v[2 * NV] = okR ? 1.0f : 0.0f;
    // fast_speed<DIR> of both faces, paired
    const float2 inv_rho = rcp2(V[RHO]);
    const float2 a2 = mul2(mul2(dup2(g), V[PP]), inv_rho);
    const float2 b2 = mul2(fma2(V[BZ], V[BZ], fma2(V[BY], V[BY], mul2(V[BX], V[BX]))), inv_rho);
    const float2 Bn = (DIR == 0) ? V[BX] : V[BY];
    const float2 bn2 = mul2(mul2(Bn, Bn), inv_rho);
    const float2 sum = add2(a2, b2);
    const float2 disc = fma2(sum, sum, mul2(dup2(-4.0f), mul2(a2, bn2)));
    Ls.v[2 * NV + 1] = sqrtf(0.5f * (sum.x + sqrtf(fmaxf(disc.x, 0.0f))));
    Rs.v[2 * NV + 1] = sqrtf(0.5f * (sum.y + sqrtf(fmaxf(disc.y, 0.0f))));
}

// Per-cell CFL speed (src/cpu/solver_cpu.cpp:291-300); -1 for skipped cells.
__device__ __forceinline__ double cell_speed(const float* U, float g, double ch) {
    float W[NV];
    c2p(U, g, W);
    if (!isfinite(W[RHO]) || !isfinite(W[PP]) || W[RHO] <= 0.0f || W[PP] <= 0.0f) return -1.0;
    const double sx = fmax((double)(fabsf(W[PU]) + fast_speed<0>(W, g)), ch);
    const double sy = fmax((double)(fabsf(W[PV]) + fast_speed<1>(W, g)), ch);
    if (isfinite(sx) && isfinite(sy)) return (sx < sy) ? sy : sx;
    return -1.0;
}

// Folds one updated cell's CFL speed into acc without cell_speed's c_h floor
// and FP64 arithmetic: the maximum over cells of max(s_x, s_y, c_h) equals
// max(c_h, maximum over cells of max(s_x, s_y)), so the caller applies the
// floor once (acc < 0: no cell counted).  Cells cell_speed skips leave acc
// unchanged; a NaN directional speed counts as c_h, as fmax makes it there.
// (Skipping the fast speeds of cells whose cheap upper bound max(|u|, |v|) +
// sqrt(a^2 + b^2) stays under the running maximum measured no faster: 0.630
// against 0.631 ms for the 4096^2 y-sweep.)
__device__ __forceinline__ void fold_cell_speed(const float* U, float g, float& acc) {
    float W[NV];
    c2p(U, g, W);
    if (!(W[RHO] > 0.0f && W[PP] > 0.0f && both_finite(W[RHO], W[PP]))) return;
    const float a = fabsf(W[PU]) + fast_speed<0>(W, g);
    const float b = fabsf(W[PV]) + fast_speed<1>(W, g);
    if (a == INFINITY || b == INFINITY) return;
    acc = fmaxf(acc, fmaxf(fmaxf(a, b), 0.0f));
}

// fold_cell_speed for a reduction whose result is floored by c_h (speed_of),
// as every y-sweep's is: a cell whose speed provably stays under the floor
// cannot change the result, so its fast speeds are not computed.  The test is
// an upper bound from the conserved state, max(|u|, |v|) + sqrt(a^2 + b^2) >=
// max(|u| + c_fx, |v| + c_fy) (c_f^2 = (s + sqrt(s^2 - 4 a^2 b_n^2)) / 2 <= s =
// a^2 + b^2), with a relative margin of 1e-5 over the rounding of both forms.
// Only physical cells whose internal energy is above 1/40 of E are skipped, so
// that c2p would take its FP32 branch and count the cell too (a skipped cell
// is counted: acc >= 0); the others, and any non-finite cell, take the exact
// path.  Measured on B200 (Orszag-Tang 4096^2, HLLD, van Leer): y-sweep
// 0.582 -> 0.567 ms (bit-identical results).
__device__ __forceinline__ void fold_cell_speed_floored(const float* U, float g, float floor_f, float& acc) {
    const float r = U[RHO];
    const float ir = 1.0f / r;
    const float m2 = U[MX] * U[MX] + U[MY] * U[MY] + U[MZ] * U[MZ];
    const float B2 = U[BX] * U[BX] + U[BY] * U[BY] + U[BZ] * U[BZ];
    const float eint = U[EN] - 0.5f * (m2 * ir + B2);
    const float bound = fmaxf(fabsf(U[MX]), fabsf(U[MY])) * ir + sqrtf((g * (g - 1.0f) * eint + B2) * ir);
    if (r > 0.0f && eint > 0.025f * fabsf(U[EN]) && bound * 1.00001f < floor_f) {
        acc = fmaxf(acc, 0.0f);
        return;
    }
    fold_cell_speed(U, g, acc);
}

}  // namespace fast
}  // namespace mhd
