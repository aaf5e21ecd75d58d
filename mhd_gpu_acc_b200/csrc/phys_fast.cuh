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
__device__ __forceinline__ bool all_finite(const float* v, int n) {
    float z = v[0] * 0.0f;
    for (int k = 1; k < n; ++k) z = fmaf(v[k], 0.0f, z);
    return z == 0.0f;
}
__device__ __forceinline__ bool both_finite(float a, float b) { return fmaf(a, 0.0f, b * 0.0f) == 0.0f; }

struct Side {
    float v[2 * NV];  // [0, 9): U, [9, 18): W
    __device__ __forceinline__ float* U() { return v; }
    __device__ __forceinline__ float* W() { return v + NV; }
    __device__ __forceinline__ const float* U() const { return v; }
    __device__ __forceinline__ const float* W() const { return v + NV; }
};

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
    if (!riemann_physical(L.W()) || !riemann_physical(R.W())) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = 0.5f * (FL[k] + FR[k]);
        return;
    }
    const float cfL = fast_speed<DIR>(L.W(), g), cfR = fast_speed<DIR>(R.W(), g);
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
__device__ __forceinline__ void hllc(const Side& L, const Side& R, float ch, float g, float* F) {
    const float* VL = L.W();
    const float* VR = R.W();
    if (!riemann_physical(VL) || !riemann_physical(VR)) { hll<DIR>(L, R, ch, g, F); return; }
    const float rhoL = VL[RHO], rhoR = VR[RHO], pL = VL[PP], pR = VR[PP];
    float unL, unR, utL, utR, uwL, uwR, BnL, BnR, BtL, BtR, BwL, BwR;
    rotate<DIR>(VL, unL, utL, uwL, BnL, BtL, BwL);
    rotate<DIR>(VR, unR, utR, uwR, BnR, BtR, BwR);
    const float cfL = fast_speed<DIR>(VL, g), cfR = fast_speed<DIR>(VR, g);
    const float SL = fminf(unL - cfL, unR - cfR);
    const float SR = fmaxf(unL + cfL, unR + cfR);
    if (SL >= 0.0f) { flux<DIR>(L.U(), VL, ch, F); return; }
    if (SR <= 0.0f) { flux<DIR>(R.U(), VR, ch, F); return; }
    const float ptL = pL + 0.5f * (BnL * BnL + BtL * BtL + BwL * BwL);
    const float ptR = pR + 0.5f * (BnR * BnR + BtR * BtR + BwR * BwR);
    const float numerSM = (SR - unR) * rhoR * unR - (SL - unL) * rhoL * unL + ptL - ptR;
    const float denomSM = (SR - unR) * rhoR - (SL - unL) * rhoL;
    if (fabsf(denomSM) < 1.0e-14f) { hll<DIR>(L, R, ch, g, F); return; }
    const float SM = numerSM / denomSM;
    const float rhoLs = rhoL * (SL - unL) / (SL - SM);
    const float rhoRs = rhoR * (SR - unR) / (SR - SM);
    if (rhoLs <= 0.0f || rhoRs <= 0.0f || !both_finite(rhoLs, rhoRs)) { hll<DIR>(L, R, ch, g, F); return; }
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
}

// Single-star state of one side (head/riemann.hpp:340-373).
__device__ __forceinline__ void star_state(float rho, float un, float ut, float uw, float Bn, float Bt, float Bw,
                                           float S, float SM, float& uts, float& uws, float& Bts, float& Bws) {
    const float d = rho * (S - un) * (S - SM) - Bn * Bn;
    if (fabsf(d) < 1.0e-14f) {
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
__device__ __forceinline__ void hlld(const Side& L, const Side& R, float ch, float g, float* F) {
    const float* VL = L.W();
    const float* VR = R.W();
    if (!riemann_physical(VL) || !riemann_physical(VR)) { hll<DIR>(L, R, ch, g, F); return; }
    const float rhoL = VL[RHO], rhoR = VR[RHO], pL = VL[PP], pR = VR[PP];
    float unL, unR, utL, utR, uwL, uwR, BnL, BnR, BtL, BtR, BwL, BwR;
    rotate<DIR>(VL, unL, utL, uwL, BnL, BtL, BwL);
    rotate<DIR>(VR, unR, utR, uwR, BnR, BtR, BwR);
    const float cfL = fast_speed<DIR>(VL, g), cfR = fast_speed<DIR>(VR, g);
    const float SL = fminf(unL - cfL, unR - cfR);
    const float SR = fmaxf(unL + cfL, unR + cfR);
    if (fabsf(SR - SL) < 1.0e-14f) { hll<DIR>(L, R, ch, g, F); return; }
    const float ptL = pL + 0.5f * (BnL * BnL + BtL * BtL + BwL * BwL);
    const float ptR = pR + 0.5f * (BnR * BnR + BtR * BtR + BwR * BwR);
    const float numerSM = (SR - unR) * rhoR * unR - (SL - unL) * rhoL * unL + ptL - ptR;
    const float denomSM = (SR - unR) * rhoR - (SL - unL) * rhoL;
    if (fabsf(denomSM) < 1.0e-14f) { hll<DIR>(L, R, ch, g, F); return; }
    const float SM = numerSM / denomSM;
    const float rhoLs = rhoL * (SL - unL) / (SL - SM);
    const float rhoRs = rhoR * (SR - unR) / (SR - SM);
    if (rhoLs <= 0.0f || rhoRs <= 0.0f || !both_finite(rhoLs, rhoRs)) { hll<DIR>(L, R, ch, g, F); return; }
    if (SL >= 0.0f) { flux<DIR>(L.U(), VL, ch, F); return; }
    if (SR <= 0.0f) { flux<DIR>(R.U(), VR, ch, F); return; }
    const float ptstar = ptL + rhoL * (SL - unL) * (SM - unL);
    const float sqL = sqrtf(rhoLs), sqR = sqrtf(rhoRs);
    const float psiM = 0.5f * (VL[PSI] + VR[PSI]) - 0.5f * ch * (BnR - BnL);
    const float signBn = (BnL >= 0.0f) ? 1.0f : -1.0f;
    float utLs, uwLs, BtLs, BwLs, utRs, uwRs, BtRs, BwRs;
    star_state(rhoL, unL, utL, uwL, BnL, BtL, BwL, SL, SM, utLs, uwLs, BtLs, BwLs);
    star_state(rhoR, unR, utR, uwR, BnR, BtR, BwR, SR, SM, utRs, uwRs, BtRs, BwRs);
    const bool left = (SM >= 0.0f);
    // the side that owns the face
    const float rho_ = left ? rhoL : rhoR, un_ = left ? unL : unR, S_ = left ? SL : SR;
    const float Bn_ = left ? BnL : BnR, pt_ = left ? ptL : ptR;
    const float ut_ = left ? utL : utR, uw_ = left ? uwL : uwR, Bt_ = left ? BtL : BtR, Bw_ = left ? BwL : BwR;
    const float uts = left ? utLs : utRs, uws = left ? uwLs : uwRs, Bts = left ? BtLs : BtRs, Bws = left ? BwLs : BwRs;
    const float rhos = left ? rhoLs : rhoRs, sq = left ? sqL : sqR;
    const float* Uside = left ? L.U() : R.U();
    const float* Wside = left ? VL : VR;
    const float BdU = Bn_ * un_ + Bt_ * ut_ + Bw_ * uw_;
    const float BdUs = Bn_ * SM + Bts * uts + Bws * uws;
    const float Es = (Uside[EN] * (S_ - un_) - pt_ * un_ + ptstar * SM + Bn_ * (BdUs - BdU)) / (S_ - SM);
    float Us[NV], Fs[NV];
    build_star<DIR>(rhos, SM, uts, uws, Bn_, Bts, Bws, Es, psiM, Us);
    flux<DIR>(Uside, Wside, ch, Fs);
    const float Sstar = left ? SM - fabsf(BnL) / sqL : SM + fabsf(BnR) / sqR;
    const bool single = left ? (Sstar >= 0.0f) : (Sstar <= 0.0f);
    if (single) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = Fs[k] + S_ * (Us[k] - Uside[k]);
        return;
    }
    // double-star state (head/riemann.hpp:375-413)
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
}

// force_flux (head/riemann.hpp:486-525)
template <int DIR>
__device__ __forceinline__ void force(const Side& L, const Side& R, float ch, float g, float* F) {
    float FL[NV], FR[NV];
    flux<DIR>(L.U(), L.W(), ch, FL);
    flux<DIR>(R.U(), R.W(), ch, FR);
    if (!riemann_physical(L.W()) || !riemann_physical(R.W())) {
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = 0.5f * (FL[k] + FR[k]);
        return;
    }
    const float cfL = fast_speed<DIR>(L.W(), g), cfR = fast_speed<DIR>(R.W(), g);
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

// riemann_flux dispatcher (head/riemann.hpp:568-592)
template <int DIR, int SOLVER>
__device__ __forceinline__ void riemann(const Side& L, const Side& R, float ch, float g, float* F) {
    if (SOLVER == HLL) { hll<DIR>(L, R, ch, g, F); return; }
    if (SOLVER == HLLC) hllc<DIR>(L, R, ch, g, F);
    else if (SOLVER == HLLD) hlld<DIR>(L, R, ch, g, F);
    else force<DIR>(L, R, ch, g, F);
    if (!(fmaf(F[RHO], 0.0f, fmaf(F[EN], 0.0f, fmaf(F[BX], 0.0f, F[PSI] * 0.0f))) == 0.0f)) {
        hll<DIR>(L, R, ch, g, F);
        return;
    }
    glm_overwrite<DIR>(F, L, R, ch);
}

__device__ __forceinline__ float minmod(float a, float b) {
    if (a * b <= 0.0f) return 0.0f;
    return (a > 0.0f) ? fminf(a, b) : fmaxf(a, b);
}
__device__ __forceinline__ float vanleer(float a, float b) {
    const float ab = a * b;
    if (ab <= 0.0f) return 0.0f;
    return 2.0f * ab / (a + b);
}

__device__ __forceinline__ bool is_physical(const float* V) {
    return V[RHO] > kRhoFloor && V[PP] > kPFloor && all_finite(V, NV);
}

// MUSCL-Hancock half step (src/cpu/solver_cpu.cpp:88-119; c_h in the predictor).
template <int DIR, int LIMITER>
__device__ __forceinline__ void reconstruct(const float* Wm, const float* Wc, const float* Wp, float dtd, float ch,
                                            float g, Side& Ls, Side& Rs) {
    float* WL = Ls.W();
    float* WR = Rs.W();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const float a = Wc[k] - Wm[k], b = Wp[k] - Wc[k];
        const float s = (LIMITER == VANLEER) ? vanleer(a, b) : minmod(a, b);
        WL[k] = Wc[k] - 0.5f * s;
        WR[k] = Wc[k] + 0.5f * s;
    }
    if (!is_physical(WL)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) WL[k] = Wc[k];
    }
    if (!is_physical(WR)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) WR[k] = Wc[k];
    }
    float UL[NV], UR[NV], FL[NV], FR[NV];
    p2c(WL, g, UL);
    p2c(WR, g, UR);
    flux<DIR>(UL, WL, ch, FL);
    flux<DIR>(UR, WR, ch, FR);
    const float s = 0.5f * dtd;
    float V[NV];
    {
        float* U = Ls.U();
#pragma unroll
        for (int k = 0; k < NV; ++k) U[k] = UL[k] - s * (FR[k] - FL[k]);
        c2p(U, g, V);
        if (is_physical(V)) {
#pragma unroll
            for (int k = 0; k < NV; ++k) WL[k] = V[k];
        } else {
#pragma unroll
            for (int k = 0; k < NV; ++k) U[k] = UL[k];  // WL already matches UL
        }
    }
    {
        float* U = Rs.U();
#pragma unroll
        for (int k = 0; k < NV; ++k) U[k] = UR[k] - s * (FR[k] - FL[k]);
        c2p(U, g, V);
        if (is_physical(V)) {
#pragma unroll
            for (int k = 0; k < NV; ++k) WR[k] = V[k];
        } else {
#pragma unroll
            for (int k = 0; k < NV; ++k) U[k] = UR[k];
        }
    }
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

}  // namespace fast
}  // namespace mhd
