/*
 * mhd_oracle.c -- CPU restatement (FP64, plain C99) of the reference's 2D
 * Dedner GLM-MHD finite-volume time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * path: it may be loaded by tests/, by __graft_entry__.smoke() and by the
 * cpu_baseline leg of bench.py, never by the product.  The product (the
 * libmhd_b200 CUDA library) does not link, load or call it.
 *
 * Parity is pinned: tests/test_oracle_pin.py checks this restatement
 * bit-for-bit against the reference's own CPU code compiled from source into
 * oracle/_ref (see oracle/Makefile), and tests/golden holds fixtures made by
 * that build.
 *
 * Every function follows the reference's expression order literally (same
 * operands, same association), because IEEE double arithmetic is only
 * reproducible when the expression trees agree.  Compile with
 * -ffp-contract=off so that no multiply-add is fused.
 *
 * State layout: 9 SoA planes of (nx+2ng)*(ny+2ng) doubles, row-major
 * (j*(nx+2ng)+i), plane order rho, rhou, rhov, rhow, Bx, By, Bz, E, psi
 * (head/types.hpp:16-41 gives the field order; head/cpu/grid_cpu.hpp:85-87 the
 * row-major index).
 *
 * Additions that the reference does not have (documented as such):
 *   - a van Leer slope limiter (limiter = 1); minmod (limiter = 0) is the
 *     reference's only limiter (src/cpu/solver_cpu.cpp:26-43).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

enum { RHO = 0, MX = 1, MY = 2, MZ = 3, BX = 4, BY = 5, BZ = 6, EN = 7, PSI = 8 };
/* primitive slots share the indices: u=1, v=2, w=3, p=7 */
enum { PU = 1, PV = 2, PW = 3, PP = 7 };
enum { DIR_X = 0, DIR_Y = 1 };
enum { ORC_HLL = 0, ORC_HLLC = 1, ORC_HLLD = 2, ORC_FORCE = 3 };
enum { ORC_MINMOD = 0, ORC_VANLEER = 1 };
enum { ORC_PERIODIC = 0, ORC_TRANSMISSIVE = 1, ORC_REFLECTING = 2, ORC_DIRICHLET = 3 };

#define NV 9
#define RHO_FLOOR 1.0e-12 /* src/cpu/solver_cpu.cpp:19 */
#define P_FLOOR 1.0e-12   /* src/cpu/solver_cpu.cpp:20 */

typedef struct {
    int nx, ny, ng;
    double dx, dy;
} orc_grid;

static inline int tnx(const orc_grid *g) { return g->nx + 2 * g->ng; }
static inline int tny(const orc_grid *g) { return g->ny + 2 * g->ng; }
static inline size_t plane(const orc_grid *g) { return (size_t)tnx(g) * (size_t)tny(g); }
static inline size_t cidx(const orc_grid *g, int i, int j) { return (size_t)j * (size_t)tnx(g) + (size_t)i; }

static inline void load9(const double *U, const orc_grid *g, size_t k, double *out) {
    const size_t ps = plane(g);
    for (int f = 0; f < NV; ++f) out[f] = U[(size_t)f * ps + k];
}
static inline void store9(double *U, const orc_grid *g, size_t k, const double *in) {
    const size_t ps = plane(g);
    for (int f = 0; f < NV; ++f) U[(size_t)f * ps + k] = in[f];
}

/* ------------------------------------------------------------------ */
/* Physics: head/physics.hpp                                            */
/* ------------------------------------------------------------------ */

/* cons_to_prim, head/physics.hpp:69-78 */
static inline void c2p(const double *U, double gam, double *W) {
    const double inv_rho = 1.0 / U[RHO];
    const double ux = U[MX] * inv_rho;
    const double uy = U[MY] * inv_rho;
    const double uz = U[MZ] * inv_rho;
    const double Bmag2 = U[BX] * U[BX] + U[BY] * U[BY] + U[BZ] * U[BZ];
    const double ke = 0.5 * U[RHO] * (ux * ux + uy * uy + uz * uz);
    const double p = (gam - 1.0) * (U[EN] - ke - 0.5 * Bmag2);
    W[RHO] = U[RHO]; W[PU] = ux; W[PV] = uy; W[PW] = uz;
    W[BX] = U[BX]; W[BY] = U[BY]; W[BZ] = U[BZ]; W[PP] = p; W[PSI] = U[PSI];
}

/* prim_to_cons, head/physics.hpp:83-90 */
static inline void p2c(const double *V, double gam, double *U) {
    const double Bmag2 = V[BX] * V[BX] + V[BY] * V[BY] + V[BZ] * V[BZ];
    const double ke = 0.5 * V[RHO] * (V[PU] * V[PU] + V[PV] * V[PV] + V[PW] * V[PW]);
    const double E = V[PP] / (gam - 1.0) + ke + 0.5 * Bmag2;
    U[RHO] = V[RHO]; U[MX] = V[RHO] * V[PU]; U[MY] = V[RHO] * V[PV]; U[MZ] = V[RHO] * V[PW];
    U[BX] = V[BX]; U[BY] = V[BY]; U[BZ] = V[BZ]; U[EN] = E; U[PSI] = V[PSI];
}

/* flux_x / flux_y, head/physics.hpp:105-127 and :142-164 */
static inline void flux(const double *U, double ch, double gam, int dir, double *F) {
    const double inv_rho = 1.0 / U[RHO];
    const double ux = U[MX] * inv_rho;
    const double uy = U[MY] * inv_rho;
    const double uz = U[MZ] * inv_rho;
    const double Bmag2 = U[BX] * U[BX] + U[BY] * U[BY] + U[BZ] * U[BZ];
    const double ke = 0.5 * U[RHO] * (ux * ux + uy * uy + uz * uz);
    const double p = (gam - 1.0) * (U[EN] - ke - 0.5 * Bmag2);
    const double p_tot = p + 0.5 * Bmag2;
    const double BdotU = U[BX] * ux + U[BY] * uy + U[BZ] * uz;
    if (dir == DIR_X) {
        F[0] = U[MX];
        F[1] = U[MX] * ux + p_tot - U[BX] * U[BX];
        F[2] = U[MX] * uy - U[BX] * U[BY];
        F[3] = U[MX] * uz - U[BX] * U[BZ];
        F[4] = U[PSI];
        F[5] = U[BY] * ux - U[BX] * uy;
        F[6] = U[BZ] * ux - U[BX] * uz;
        F[7] = (U[EN] + p_tot) * ux - U[BX] * BdotU;
        F[8] = ch * ch * U[BX];
    } else {
        F[0] = U[MY];
        F[1] = U[MY] * ux - U[BY] * U[BX];
        F[2] = U[MY] * uy + p_tot - U[BY] * U[BY];
        F[3] = U[MY] * uz - U[BY] * U[BZ];
        F[4] = U[BX] * uy - U[BY] * ux;
        F[5] = U[PSI];
        F[6] = U[BZ] * uy - U[BY] * uz;
        F[7] = (U[EN] + p_tot) * uy - U[BY] * BdotU;
        F[8] = ch * ch * U[BY];
    }
}

/* fast_speed_x / fast_speed_y, head/physics.hpp:175-191 */
static inline double fast_speed(const double *V, double gam, int dir) {
    const double a2 = gam * V[PP] / V[RHO];
    const double b2 = (V[BX] * V[BX] + V[BY] * V[BY] + V[BZ] * V[BZ]) / V[RHO];
    const double Bn = (dir == DIR_X) ? V[BX] : V[BY];
    const double bn2 = Bn * Bn / V[RHO];
    const double disc = (a2 + b2) * (a2 + b2) - 4.0 * a2 * bn2;
    return sqrt(0.5 * (a2 + b2 + sqrt(disc > 0.0 ? disc : 0.0)));
}

/* primitive_is_physical, head/riemann.hpp:54-57 */
static inline int prim_physical_riemann(const double *V) {
    return isfinite(V[RHO]) && isfinite(V[PP]) && V[RHO] > 0.0 && V[PP] > 0.0;
}

/* ------------------------------------------------------------------ */
/* Riemann solvers: head/riemann.hpp                                    */
/* ------------------------------------------------------------------ */

/* hll_flux, head/riemann.hpp:70-107 */
static void hll(const double *UL, const double *UR, int dir, double ch, double gam, double *F) {
    double VL[NV], VR[NV], FL[NV], FR[NV];
    c2p(UL, gam, VL);
    c2p(UR, gam, VR);
    flux(UL, ch, gam, dir, FL);
    flux(UR, ch, gam, dir, FR);
    if (!prim_physical_riemann(VL) || !prim_physical_riemann(VR)) {
        for (int k = 0; k < NV; ++k) F[k] = 0.5 * (FL[k] + FR[k]);
        return;
    }
    const double cfL = fast_speed(VL, gam, dir);
    const double cfR = fast_speed(VR, gam, dir);
    const double unL = (dir == DIR_X) ? VL[PU] : VL[PV];
    const double unR = (dir == DIR_X) ? VR[PU] : VR[PV];
    const double SL = fmin(fmin(unL - cfL, unR - cfR), -ch);
    const double SR = fmax(fmax(unL + cfL, unR + cfR), ch);
    if (SL >= 0.0) { memcpy(F, FL, sizeof FL); return; }
    if (SR <= 0.0) { memcpy(F, FR, sizeof FR); return; }
    const double denom = SR - SL;
    if (fabs(denom) < 1.0e-14) {
        for (int k = 0; k < NV; ++k) F[k] = 0.5 * (FL[k] + FR[k]);
        return;
    }
    /* Conserved operator/ multiplies by the reciprocal: head/types.hpp:104-106 */
    const double inv = 1.0 / denom;
    const double SLSR = SL * SR;
    for (int k = 0; k < NV; ++k)
        F[k] = inv * (SR * FL[k] - SL * FR[k] + SLSR * (UR[k] - UL[k]));
}

/* Star-state builder with the direction rotation, head/riemann.hpp:219-230 and :417-437 */
static inline void build_star(int dir, double rhos, double uns, double uts, double uws,
                              double Bns, double Bts, double Bws, double Es, double psis, double *U) {
    U[RHO] = rhos;
    if (dir == DIR_X) {
        U[MX] = rhos * uns; U[MY] = rhos * uts; U[MZ] = rhos * uws;
        U[BX] = Bns; U[BY] = Bts; U[BZ] = Bws;
    } else {
        U[MX] = rhos * uts; U[MY] = rhos * uns; U[MZ] = rhos * uws;
        U[BX] = Bts; U[BY] = Bns; U[BZ] = Bws;
    }
    U[EN] = Es; U[PSI] = psis;
}

/* Normal/tangential split, head/riemann.hpp:141-155 and :274-288 */
static inline void rotate(const double *V, int dir, double *un, double *ut, double *uw,
                          double *Bn, double *Bt, double *Bw) {
    if (dir == DIR_X) {
        *un = V[PU]; *ut = V[PV]; *uw = V[PW]; *Bn = V[BX]; *Bt = V[BY]; *Bw = V[BZ];
    } else {
        *un = V[PV]; *ut = V[PU]; *uw = V[PW]; *Bn = V[BY]; *Bt = V[BX]; *Bw = V[BZ];
    }
}

/* hllc_flux, head/riemann.hpp:122-241 */
static void hllc(const double *UL, const double *UR, int dir, double ch, double gam, double *F) {
    double VL[NV], VR[NV];
    c2p(UL, gam, VL);
    c2p(UR, gam, VR);
    if (!prim_physical_riemann(VL) || !prim_physical_riemann(VR)) { hll(UL, UR, dir, ch, gam, F); return; }
    const double rhoL = VL[RHO], rhoR = VR[RHO];
    const double pL = VL[PP], pR = VR[PP];
    double unL, unR, utL, utR, uwL, uwR, BnL, BnR, BtL, BtR, BwL, BwR;
    rotate(VL, dir, &unL, &utL, &uwL, &BnL, &BtL, &BwL);
    rotate(VR, dir, &unR, &utR, &uwR, &BnR, &BtR, &BwR);
    const double cfL = fast_speed(VL, gam, dir);
    const double cfR = fast_speed(VR, gam, dir);
    const double SL = fmin(unL - cfL, unR - cfR);
    const double SR = fmax(unL + cfL, unR + cfR);
    double FL[NV], FR[NV];
    flux(UL, ch, gam, dir, FL);
    flux(UR, ch, gam, dir, FR);
    if (SL >= 0.0) { memcpy(F, FL, sizeof FL); return; }
    if (SR <= 0.0) { memcpy(F, FR, sizeof FR); return; }
    const double BmagL2 = BnL * BnL + BtL * BtL + BwL * BwL;
    const double BmagR2 = BnR * BnR + BtR * BtR + BwR * BwR;
    const double ptL = pL + 0.5 * BmagL2;
    const double ptR = pR + 0.5 * BmagR2;
    const double numerSM = (SR - unR) * rhoR * unR - (SL - unL) * rhoL * unL + ptL - ptR;
    const double denomSM = (SR - unR) * rhoR - (SL - unL) * rhoL;
    if (fabs(denomSM) < 1.0e-14) { hll(UL, UR, dir, ch, gam, F); return; }
    const double SM = numerSM / denomSM;
    const double rhoLs = rhoL * (SL - unL) / (SL - SM);
    const double rhoRs = rhoR * (SR - unR) / (SR - SM);
    if (rhoLs <= 0.0 || rhoRs <= 0.0 || !isfinite(rhoLs) || !isfinite(rhoRs)) {
        hll(UL, UR, dir, ch, gam, F);
        return;
    }
    const double ptLs = ptL + rhoL * (SL - unL) * (SM - unL);
    const double ptRs = ptR + rhoR * (SR - unR) * (SM - unR);
    const double psiM = 0.5 * (VL[PSI] + VR[PSI]) - 0.5 * ch * (BnR - BnL);
    const double BdotUL = BnL * unL + BtL * utL + BwL * uwL;
    const double BdotULs = BnL * SM + BtL * utL + BwL * uwL;
    const double BdotUR = BnR * unR + BtR * utR + BwR * uwR;
    const double BdotURs = BnR * SM + BtR * utR + BwR * uwR;
    const double ELs = ((SL - unL) * UL[EN] - ptL * unL + ptLs * SM + BnL * (BdotULs - BdotUL)) / (SL - SM);
    const double ERs = ((SR - unR) * UR[EN] - ptR * unR + ptRs * SM + BnR * (BdotURs - BdotUR)) / (SR - SM);
    double Us[NV];
    if (SM >= 0.0) {
        build_star(dir, rhoLs, SM, utL, uwL, BnL, BtL, BwL, ELs, psiM, Us);
        for (int k = 0; k < NV; ++k) F[k] = FL[k] + SL * (Us[k] - UL[k]);
    } else {
        build_star(dir, rhoRs, SM, utR, uwR, BnR, BtR, BwR, ERs, psiM, Us);
        for (int k = 0; k < NV; ++k) F[k] = FR[k] + SR * (Us[k] - UR[k]);
    }
}

/* hlld_flux, head/riemann.hpp:253-480 */
static void hlld(const double *UL, const double *UR, int dir, double ch, double gam, double *F) {
    double VL[NV], VR[NV];
    c2p(UL, gam, VL);
    c2p(UR, gam, VR);
    if (!prim_physical_riemann(VL) || !prim_physical_riemann(VR)) { hll(UL, UR, dir, ch, gam, F); return; }
    const double rhoL = VL[RHO], rhoR = VR[RHO];
    const double pL = VL[PP], pR = VR[PP];
    double unL, unR, utL, utR, uwL, uwR, BnL, BnR, BtL, BtR, BwL, BwR;
    rotate(VL, dir, &unL, &utL, &uwL, &BnL, &BtL, &BwL);
    rotate(VR, dir, &unR, &utR, &uwR, &BnR, &BtR, &BwR);
    const double cfL = fast_speed(VL, gam, dir);
    const double cfR = fast_speed(VR, gam, dir);
    const double SL = fmin(unL - cfL, unR - cfR);
    const double SR = fmax(unL + cfL, unR + cfR);
    const double denom_RL = SR - SL;
    if (fabs(denom_RL) < 1.0e-14) { hll(UL, UR, dir, ch, gam, F); return; }
    const double BmagL2 = BnL * BnL + BtL * BtL + BwL * BwL;
    const double BmagR2 = BnR * BnR + BtR * BtR + BwR * BwR;
    const double ptL = pL + 0.5 * BmagL2;
    const double ptR = pR + 0.5 * BmagR2;
    const double numerSM = (SR - unR) * rhoR * unR - (SL - unL) * rhoL * unL + ptL - ptR;
    const double denomSM = (SR - unR) * rhoR - (SL - unL) * rhoL;
    if (fabs(denomSM) < 1.0e-14) { hll(UL, UR, dir, ch, gam, F); return; }
    const double SM = numerSM / denomSM;
    const double rhoLs = rhoL * (SL - unL) / (SL - SM);
    const double rhoRs = rhoR * (SR - unR) / (SR - SM);
    if (rhoLs <= 0.0 || rhoRs <= 0.0 || !isfinite(rhoLs) || !isfinite(rhoRs)) {
        hll(UL, UR, dir, ch, gam, F);
        return;
    }
    const double ptstar = ptL + rhoL * (SL - unL) * (SM - unL);
    const double sqrtRhoLs = sqrt(rhoLs);
    const double sqrtRhoRs = sqrt(rhoRs);
    const double SLs = SM - fabs(BnL) / sqrtRhoLs;
    const double SRs = SM + fabs(BnR) / sqrtRhoRs;

    double utLs, uwLs, BtLs, BwLs, ELs;
    {
        const double BdotUL = BnL * unL + BtL * utL + BwL * uwL;
        const double d = rhoL * (SL - unL) * (SL - SM) - BnL * BnL;
        if (fabs(d) < 1.0e-14) {
            utLs = utL; uwLs = uwL; BtLs = BtL; BwLs = BwL;
        } else {
            utLs = utL - BnL * BtL * (SM - unL) / d;
            uwLs = uwL - BnL * BwL * (SM - unL) / d;
            BtLs = BtL * (rhoL * (SL - unL) * (SL - unL) - BnL * BnL) / d;
            BwLs = BwL * (rhoL * (SL - unL) * (SL - unL) - BnL * BnL) / d;
        }
        const double BdotULs = BnL * SM + BtLs * utLs + BwLs * uwLs;
        ELs = (UL[EN] * (SL - unL) - ptL * unL + ptstar * SM + BnL * (BdotULs - BdotUL)) / (SL - SM);
    }
    double utRs, uwRs, BtRs, BwRs, ERs;
    {
        const double BdotUR = BnR * unR + BtR * utR + BwR * uwR;
        const double d = rhoR * (SR - unR) * (SR - SM) - BnR * BnR;
        if (fabs(d) < 1.0e-14) {
            utRs = utR; uwRs = uwR; BtRs = BtR; BwRs = BwR;
        } else {
            utRs = utR - BnR * BtR * (SM - unR) / d;
            uwRs = uwR - BnR * BwR * (SM - unR) / d;
            BtRs = BtR * (rhoR * (SR - unR) * (SR - unR) - BnR * BnR) / d;
            BwRs = BwR * (rhoR * (SR - unR) * (SR - unR) - BnR * BnR) / d;
        }
        const double BdotURs = BnR * SM + BtRs * utRs + BwRs * uwRs;
        ERs = (UR[EN] * (SR - unR) - ptR * unR + ptstar * SM + BnR * (BdotURs - BdotUR)) / (SR - SM);
    }
    const double signBn = (BnL >= 0.0) ? 1.0 : -1.0;
    const double sqRhoLs = sqrtRhoLs, sqRhoRs = sqrtRhoRs;
    const double denom2 = sqRhoLs + sqRhoRs;
    double utLss, uwLss, BtLss, BwLss, utRss, uwRss, BtRss, BwRss, ELss, ERss;
    if (fabs(denom2) < 1.0e-14) {
        utLss = utLs; uwLss = uwLs; BtLss = BtLs; BwLss = BwLs; ELss = ELs;
        utRss = utRs; uwRss = uwRs; BtRss = BtRs; BwRss = BwRs; ERss = ERs;
    } else {
        const double inv_d2 = 1.0 / denom2;
        utLss = utRss = (sqRhoLs * utLs + sqRhoRs * utRs + signBn * (BtRs - BtLs)) * inv_d2;
        uwLss = uwRss = (sqRhoLs * uwLs + sqRhoRs * uwRs + signBn * (BwRs - BwLs)) * inv_d2;
        BtLss = BtRss = (sqRhoLs * BtRs + sqRhoRs * BtLs + signBn * sqRhoLs * sqRhoRs * (utRs - utLs)) * inv_d2;
        BwLss = BwRss = (sqRhoLs * BwRs + sqRhoRs * BwLs + signBn * sqRhoLs * sqRhoRs * (uwRs - uwLs)) * inv_d2;
        /* the first ELss/ERss estimate (head/riemann.hpp:398-403) is overwritten by :406-412 */
        const double BdotULss = BnL * SM + BtLss * utLss + BwLss * uwLss;
        const double BdotULs = BnL * SM + BtLs * utLs + BwLs * uwLs;
        ELss = ELs - sqRhoLs * signBn * (BdotULss - BdotULs);
        const double BdotURss = BnR * SM + BtRss * utRss + BwRss * uwRss;
        const double BdotURs = BnR * SM + BtRs * utRs + BwRs * uwRs;
        ERss = ERs + sqRhoRs * signBn * (BdotURss - BdotURs);
    }
    const double psiM = 0.5 * (VL[PSI] + VR[PSI]) - 0.5 * ch * (BnR - BnL);
    double FL[NV], FR[NV];
    flux(UL, ch, gam, dir, FL);
    flux(UR, ch, gam, dir, FR);
    if (SL >= 0.0) { memcpy(F, FL, sizeof FL); return; }
    if (SR <= 0.0) { memcpy(F, FR, sizeof FR); return; }
    double Us[NV], Uss[NV];
    if (SM >= 0.0) {
        build_star(dir, rhoLs, SM, utLs, uwLs, BnL, BtLs, BwLs, ELs, psiM, Us);
        if (SLs >= 0.0) {
            for (int k = 0; k < NV; ++k) F[k] = FL[k] + SL * (Us[k] - UL[k]);
        } else {
            build_star(dir, rhoLs, SM, utLss, uwLss, BnL, BtLss, BwLss, ELss, psiM, Uss);
            for (int k = 0; k < NV; ++k) F[k] = FL[k] + SL * (Us[k] - UL[k]) + SLs * (Uss[k] - Us[k]);
        }
    } else {
        build_star(dir, rhoRs, SM, utRs, uwRs, BnR, BtRs, BwRs, ERs, psiM, Us);
        if (SRs <= 0.0) {
            for (int k = 0; k < NV; ++k) F[k] = FR[k] + SR * (Us[k] - UR[k]);
        } else {
            build_star(dir, rhoRs, SM, utRss, uwRss, BnR, BtRss, BwRss, ERss, psiM, Uss);
            for (int k = 0; k < NV; ++k) F[k] = FR[k] + SR * (Us[k] - UR[k]) + SRs * (Uss[k] - Us[k]);
        }
    }
}

/* force_flux, head/riemann.hpp:486-525 */
static void force(const double *UL, const double *UR, int dir, double ch, double gam, double *F) {
    double VL[NV], VR[NV], FL[NV], FR[NV];
    c2p(UL, gam, VL);
    c2p(UR, gam, VR);
    flux(UL, ch, gam, dir, FL);
    flux(UR, ch, gam, dir, FR);
    if (!prim_physical_riemann(VL) || !prim_physical_riemann(VR)) {
        for (int k = 0; k < NV; ++k) F[k] = 0.5 * (FL[k] + FR[k]);
        return;
    }
    const double cfL = fast_speed(VL, gam, dir);
    const double cfR = fast_speed(VR, gam, dir);
    const double unL = (dir == DIR_X) ? VL[PU] : VL[PV];
    const double unR = (dir == DIR_X) ? VR[PU] : VR[PV];
    const double alpha = fmax(fmax(fabs(unL) + cfL, fabs(unR) + cfR), ch);
    if (alpha < 1.0e-14) {
        for (int k = 0; k < NV; ++k) F[k] = 0.5 * (FL[k] + FR[k]);
        return;
    }
    double Flf[NV], Uri[NV], Vri[NV], Fri[NV];
    const double ha = 0.5 * alpha;
    const double hia = 0.5 * (1.0 / alpha);
    for (int k = 0; k < NV; ++k) {
        Flf[k] = 0.5 * (FL[k] + FR[k]) - ha * (UR[k] - UL[k]);
        Uri[k] = 0.5 * (UL[k] + UR[k]) - hia * (FR[k] - FL[k]);
    }
    c2p(Uri, gam, Vri);
    if (!prim_physical_riemann(Vri)) { memcpy(F, Flf, sizeof Flf); return; }
    flux(Uri, ch, gam, dir, Fri);
    for (int k = 0; k < NV; ++k) F[k] = 0.5 * (Flf[k] + Fri[k]);
}

/* apply_glm_flux, head/riemann.hpp:544-563 */
static inline void glm_overwrite(double *F, const double *UL, const double *UR, int dir, double ch) {
    if (ch <= 0.0) return;
    const double BnL = (dir == DIR_X) ? UL[BX] : UL[BY];
    const double BnR = (dir == DIR_X) ? UR[BX] : UR[BY];
    const double psiL = UL[PSI], psiR = UR[PSI];
    const double Bn_star = 0.5 * (BnL + BnR) - 0.5 / ch * (psiR - psiL);
    const double psi_star = 0.5 * (psiL + psiR) - 0.5 * ch * (BnR - BnL);
    if (dir == DIR_X) F[BX] = psi_star; else F[BY] = psi_star;
    F[PSI] = ch * ch * Bn_star;
}

/* riemann_flux (explicit ch form), head/riemann.hpp:568-592 */
static void riemann(const double *UL, const double *UR, int dir, int solver, double ch, double gam, double *F) {
    if (solver == ORC_HLL) { hll(UL, UR, dir, ch, gam, F); return; }
    if (solver == ORC_HLLC) hllc(UL, UR, dir, ch, gam, F);
    else if (solver == ORC_HLLD) hlld(UL, UR, dir, ch, gam, F);
    else force(UL, UR, dir, ch, gam, F);
    if (!isfinite(F[RHO]) || !isfinite(F[EN]) || !isfinite(F[BX]) || !isfinite(F[PSI])) {
        hll(UL, UR, dir, ch, gam, F);
        return;
    }
    glm_overwrite(F, UL, UR, dir, ch);
}

/* ------------------------------------------------------------------ */
/* MUSCL-Hancock: src/cpu/solver_cpu.cpp                                */
/* ------------------------------------------------------------------ */

/* minmod_scalar, src/cpu/solver_cpu.cpp:26-29 (std::min/std::max spelled out) */
static inline double minmod(double a, double b) {
    if (a * b <= 0.0) return 0.0;
    return (a > 0.0) ? ((b < a) ? b : a) : ((a < b) ? b : a);
}

/* van Leer harmonic-mean limiter (no counterpart in the reference) */
static inline double vanleer(double a, double b) {
    if (a * b <= 0.0) return 0.0;
    return 2.0 * a * b / (a + b);
}

/* is_physical, src/cpu/solver_cpu.cpp:49-56 */
static inline int is_physical(const double *V) {
    return isfinite(V[RHO]) && V[RHO] > RHO_FLOOR && isfinite(V[PP]) && V[PP] > P_FLOOR &&
           isfinite(V[PU]) && isfinite(V[PV]) && isfinite(V[PW]) && isfinite(V[BX]) &&
           isfinite(V[BY]) && isfinite(V[BZ]) && isfinite(V[PSI]);
}

/* reconstruct_cell_muscl_hancock, src/cpu/solver_cpu.cpp:88-119 (ch in the predictor) */
static void reconstruct(const double *Wm, const double *Wc, const double *Wp, double dt_over_d, int dir,
                        double ch, double gam, int limiter, double *Ul_star, double *Ur_star) {
    double slope[NV], Wl[NV], Wr[NV], Ul[NV], Ur[NV], Fl[NV], Fr[NV], tmp[NV], Vtmp[NV];
    for (int k = 0; k < NV; ++k) {
        const double a = Wc[k] - Wm[k];
        const double b = Wp[k] - Wc[k];
        slope[k] = (limiter == ORC_VANLEER) ? vanleer(a, b) : minmod(a, b);
    }
    for (int k = 0; k < NV; ++k) {
        Wl[k] = Wc[k] - 0.5 * slope[k];
        Wr[k] = Wc[k] + 0.5 * slope[k];
    }
    /* enforce_physical_primitive, src/cpu/solver_cpu.cpp:58-63 */
    if (!is_physical(Wl)) memcpy(Wl, Wc, sizeof Wl);
    if (!is_physical(Wr)) memcpy(Wr, Wc, sizeof Wr);
    p2c(Wl, gam, Ul);
    p2c(Wr, gam, Ur);
    flux(Ul, ch, gam, dir, Fl);
    flux(Ur, ch, gam, dir, Fr);
    const double s = 0.5 * dt_over_d;
    /* enforce_physical_conserved, src/cpu/solver_cpu.cpp:65-70 */
    for (int k = 0; k < NV; ++k) tmp[k] = Ul[k] - s * (Fr[k] - Fl[k]);
    c2p(tmp, gam, Vtmp);
    memcpy(Ul_star, is_physical(Vtmp) ? tmp : Ul, sizeof tmp);
    for (int k = 0; k < NV; ++k) tmp[k] = Ur[k] - s * (Fr[k] - Fl[k]);
    c2p(tmp, gam, Vtmp);
    memcpy(Ur_star, is_physical(Vtmp) ? tmp : Ur, sizeof tmp);
}

/* ------------------------------------------------------------------ */
/* Boundary conditions: head/cpu/boundary_cpu.hpp                       */
/* ------------------------------------------------------------------ */

static inline void copy_cell(double *U, const orc_grid *g, int di, int dj, int si, int sj) {
    const size_t ps = plane(g);
    const size_t d = cidx(g, di, dj), s = cidx(g, si, sj);
    for (int f = 0; f < NV; ++f) U[f * ps + d] = U[f * ps + s];
}

/* copy_ghost_cells, head/cpu/boundary_cpu.hpp:12-32 */
void orc_copy_ghost_cells(const double *src, double *dst, const orc_grid *g) {
    const size_t ps = plane(g);
    const int ng = g->ng, ib = ng, ie = ng + g->nx, jb = ng, je = ng + g->ny;
    for (int j = 0; j < tny(g); ++j)
        for (int q = 0; q < ng; ++q) {
            const size_t a = cidx(g, ib - 1 - q, j), b = cidx(g, ie + q, j);
            for (int f = 0; f < NV; ++f) { dst[f * ps + a] = src[f * ps + a]; dst[f * ps + b] = src[f * ps + b]; }
        }
    for (int i = ib; i < ie; ++i)
        for (int q = 0; q < ng; ++q) {
            const size_t a = cidx(g, i, jb - 1 - q), b = cidx(g, i, je + q);
            for (int f = 0; f < NV; ++f) { dst[f * ps + a] = src[f * ps + a]; dst[f * ps + b] = src[f * ps + b]; }
        }
}

/* apply_boundary, head/cpu/boundary_cpu.hpp:45-149 (left, right, bottom, top in that order) */
void orc_apply_boundary(double *U, const orc_grid *g, const int bc[4]) {
    const size_t ps = plane(g);
    const int ng = g->ng, ib = ng, ie = ng + g->nx, jb = ng, je = ng + g->ny;
    if (bc[0] != ORC_DIRICHLET)
        for (int j = 0; j < tny(g); ++j)
            for (int q = 0; q < ng; ++q) {
                if (bc[0] == ORC_PERIODIC) copy_cell(U, g, ib - 1 - q, j, ie - 1 - q, j);
                else if (bc[0] == ORC_TRANSMISSIVE) copy_cell(U, g, ib - 1 - q, j, ib, j);
                else if (bc[0] == ORC_REFLECTING) {
                    copy_cell(U, g, ib - 1 - q, j, ib + q, j);
                    const size_t d = cidx(g, ib - 1 - q, j);
                    U[MX * ps + d] = -U[MX * ps + d];
                    U[BX * ps + d] = -U[BX * ps + d];
                }
            }
    if (bc[1] != ORC_DIRICHLET)
        for (int j = 0; j < tny(g); ++j)
            for (int q = 0; q < ng; ++q) {
                if (bc[1] == ORC_PERIODIC) copy_cell(U, g, ie + q, j, ib + q, j);
                else if (bc[1] == ORC_TRANSMISSIVE) copy_cell(U, g, ie + q, j, ie - 1, j);
                else if (bc[1] == ORC_REFLECTING) {
                    copy_cell(U, g, ie + q, j, ie - 1 - q, j);
                    const size_t d = cidx(g, ie + q, j);
                    U[MX * ps + d] = -U[MX * ps + d];
                    U[BX * ps + d] = -U[BX * ps + d];
                }
            }
    if (bc[2] != ORC_DIRICHLET)
        for (int i = 0; i < tnx(g); ++i)
            for (int q = 0; q < ng; ++q) {
                if (bc[2] == ORC_PERIODIC) copy_cell(U, g, i, jb - 1 - q, i, je - 1 - q);
                else if (bc[2] == ORC_TRANSMISSIVE) copy_cell(U, g, i, jb - 1 - q, i, jb);
                else if (bc[2] == ORC_REFLECTING) {
                    copy_cell(U, g, i, jb - 1 - q, i, jb + q);
                    const size_t d = cidx(g, i, jb - 1 - q);
                    U[MY * ps + d] = -U[MY * ps + d];
                    U[BY * ps + d] = -U[BY * ps + d];
                }
            }
    if (bc[3] != ORC_DIRICHLET)
        for (int i = 0; i < tnx(g); ++i)
            for (int q = 0; q < ng; ++q) {
                if (bc[3] == ORC_PERIODIC) copy_cell(U, g, i, je + q, i, jb + q);
                else if (bc[3] == ORC_TRANSMISSIVE) copy_cell(U, g, i, je + q, i, je - 1);
                else if (bc[3] == ORC_REFLECTING) {
                    copy_cell(U, g, i, je + q, i, je - 1 - q);
                    const size_t d = cidx(g, i, je + q);
                    U[MY * ps + d] = -U[MY * ps + d];
                    U[BY * ps + d] = -U[BY * ps + d];
                }
            }
}

/* ------------------------------------------------------------------ */
/* CFL time step: src/cpu/solver_cpu.cpp:283-312                        */
/* ------------------------------------------------------------------ */

/* Returns 0 on success, -1 when the maximum wave speed is not positive
 * (the reference throws std::runtime_error there, solver_cpu.cpp:304-306).
 * *ch is read as the floor (previous ch_glm) and overwritten with the new
 * maximum, as the reference does with phys::ch_glm (solver_cpu.cpp:309). */
int orc_compute_dt(const double *U, const orc_grid *g, double gam, double cfl, double *ch, double *dt) {
    const int ng = g->ng;
    const double ch_prev = *ch;
    double max_speed = 0.0;
#ifdef _OPENMP
#pragma omp parallel for reduction(max : max_speed) schedule(static)
#endif
    for (int j = ng; j < ng + g->ny; ++j) {
        for (int i = ng; i < ng + g->nx; ++i) {
            double Uc[NV], V[NV];
            load9(U, g, cidx(g, i, j), Uc);
            c2p(Uc, gam, V);
            if (!isfinite(V[RHO]) || !isfinite(V[PP]) || V[RHO] <= 0.0 || V[PP] <= 0.0) continue;
            const double sx = fmax(fabs(V[PU]) + fast_speed(V, gam, DIR_X), ch_prev);
            const double sy = fmax(fabs(V[PV]) + fast_speed(V, gam, DIR_Y), ch_prev);
            if (isfinite(sx) && isfinite(sy)) {
                const double m = (sx < sy) ? sy : sx;
                if (max_speed < m) max_speed = m;
            }
        }
    }
    if (max_speed <= 0.0) return -1;
    *ch = max_speed;
    const double dmin = (g->dy < g->dx) ? g->dy : g->dx;
    *dt = cfl * dmin / max_speed;
    return 0;
}

/* ------------------------------------------------------------------ */
/* One split step: src/cpu/solver_cpu.cpp:327-440                       */
/* ------------------------------------------------------------------ */

/* One directional sweep Uin -> Uout over the interior: primitive cache,
 * face fluxes from reconstructed states, conservative update with the
 * non-finite revert (solver_cpu.cpp:363-394 for x, :404-432 for y).
 * Each cell is reconstructed once; the reference reconstructs it once per
 * adjacent face, with identical (deterministic) results. */
static void sweep(const double *Uin, double *Uout, const orc_grid *g, int dir, double dt, double ch, double gam,
                  int solver, int limiter) {
    const size_t ps = plane(g);
    const int TX = tnx(g), TY = tny(g);
    const int ng = g->ng, ib = ng, ie = ng + g->nx, jb = ng, je = ng + g->ny;
    const double dt_over_d = (dir == DIR_X) ? dt / g->dx : dt / g->dy;
    double *W = (double *)malloc(sizeof(double) * NV * ps);
    double *RL = (double *)malloc(sizeof(double) * NV * ps); /* left-biased recon state per cell */
    double *RR = (double *)malloc(sizeof(double) * NV * ps); /* right-biased recon state per cell */
    double *FF = (double *)malloc(sizeof(double) * NV * ps); /* flux at face (cell, cell+1) */
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int j = 0; j < TY; ++j)
        for (int i = 0; i < TX; ++i) {
            double Uc[NV], Wc[NV];
            load9(Uin, g, cidx(g, i, j), Uc);
            c2p(Uc, gam, Wc);
            store9(W, g, cidx(g, i, j), Wc);
        }
    /* reconstruct cells ib-1..ie (x) or jb-1..je (y) on interior lines */
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int j = 0; j < TY; ++j)
        for (int i = 0; i < TX; ++i) {
            int need;
            if (dir == DIR_X) need = (j >= jb && j < je && i >= ib - 1 && i <= ie);
            else need = (i >= ib && i < ie && j >= jb - 1 && j <= je);
            if (!need) continue;
            double Wm[NV], Wc[NV], Wp[NV], l[NV], r[NV];
            const int di = (dir == DIR_X) ? 1 : 0, dj = (dir == DIR_X) ? 0 : 1;
            load9(W, g, cidx(g, i - di, j - dj), Wm);
            load9(W, g, cidx(g, i, j), Wc);
            load9(W, g, cidx(g, i + di, j + dj), Wp);
            reconstruct(Wm, Wc, Wp, dt_over_d, dir, ch, gam, limiter, l, r);
            store9(RL, g, cidx(g, i, j), l);
            store9(RR, g, cidx(g, i, j), r);
        }
    /* face (c, c+1) for c = ib-1..ie-1 (x) / jb-1..je-1 (y) */
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int j = 0; j < TY; ++j)
        for (int i = 0; i < TX; ++i) {
            int need;
            if (dir == DIR_X) need = (j >= jb && j < je && i >= ib - 1 && i < ie);
            else need = (i >= ib && i < ie && j >= jb - 1 && j < je);
            if (!need) continue;
            double a[NV], b[NV], f[NV];
            const int di = (dir == DIR_X) ? 1 : 0, dj = (dir == DIR_X) ? 0 : 1;
            load9(RR, g, cidx(g, i, j), a);
            load9(RL, g, cidx(g, i + di, j + dj), b);
            riemann(a, b, dir, solver, ch, gam, f);
            store9(FF, g, cidx(g, i, j), f);
        }
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int j = jb; j < je; ++j)
        for (int i = ib; i < ie; ++i) {
            double Uc[NV], Fp[NV], Fm[NV], Un[NV];
            const int di = (dir == DIR_X) ? 1 : 0, dj = (dir == DIR_X) ? 0 : 1;
            load9(Uin, g, cidx(g, i, j), Uc);
            load9(FF, g, cidx(g, i, j), Fp);
            load9(FF, g, cidx(g, i - di, j - dj), Fm);
            for (int k = 0; k < NV; ++k) Un[k] = Uc[k] - dt_over_d * (Fp[k] - Fm[k]);
            if (!isfinite(Un[RHO]) || !isfinite(Un[EN])) memcpy(Un, Uc, sizeof Un);
            store9(Uout, g, cidx(g, i, j), Un);
        }
    free(W); free(RL); free(RR); free(FF);
    (void)ps;
}

/* psi damping, src/cpu/solver_cpu.cpp:263-275 */
static void psi_damping(double *U, const orc_grid *g, double dt, double ch, double cr) {
    const double factor = exp(-dt * ch / cr);
    if (factor >= 1.0) return;
    const size_t ps = plane(g);
    for (int j = g->ng; j < g->ng + g->ny; ++j)
        for (int i = g->ng; i < g->ng + g->nx; ++i) U[PSI * ps + cidx(g, i, j)] *= factor;
}

/* advance_second_order, src/cpu/solver_cpu.cpp:327-440 */
void orc_advance(const double *Uold, double *Utmp, double *Unew, const orc_grid *g, double gam, double ch,
                 double cr, double dt, int solver, int limiter, const int bc[4]) {
    sweep(Uold, Utmp, g, DIR_X, dt, ch, gam, solver, limiter);
    orc_copy_ghost_cells(Uold, Utmp, g);
    orc_apply_boundary(Utmp, g, bc);
    sweep(Utmp, Unew, g, DIR_Y, dt, ch, gam, solver, limiter);
    orc_copy_ghost_cells(Utmp, Unew, g);
    orc_apply_boundary(Unew, g, bc);
    psi_damping(Unew, g, dt, ch, cr);
}

/* Driver loop of scripts/cpu/main_cpu.cpp:196-222: compute_dt, clamp to
 * t_end, the dt guards, advance, swap.  U is updated in place.  Stops after
 * max_steps steps (if > 0) or when t reaches t_end.  Returns 0, or -1 when
 * compute_dt fails, -2 when dt is non-finite or non-positive, -3 when dt falls
 * below 1e-8 t_end (main_cpu.cpp:205-216).  dt_log (optional, max_steps long)
 * receives each step's dt. */
int orc_run(double *U, const orc_grid *g, double gam, double cfl, double cr, int solver, int limiter,
            const int bc[4], int max_steps, double t_end, double *ch, double *t_out, int *steps_out,
            double *dt_log) {
    const size_t n = (size_t)NV * plane(g);
    double *A = U;
    double *T = (double *)malloc(sizeof(double) * n);
    double *B = (double *)malloc(sizeof(double) * n);
    memcpy(T, U, sizeof(double) * n);
    memcpy(B, U, sizeof(double) * n);
    double t = 0.0;
    int step = 0, rc = 0;
    while (t < t_end && (max_steps <= 0 || step < max_steps)) {
        double dt_raw = 0.0;
        if (orc_compute_dt(A, g, gam, cfl, ch, &dt_raw) != 0) { rc = -1; break; }
        const double rem = t_end - t;
        const double dt = (rem < dt_raw) ? rem : dt_raw;
        if (!isfinite(dt) || dt <= 0.0) { rc = -2; break; }
        if (dt < 1.0e-8 * t_end) { rc = -3; break; }
        orc_advance(A, T, B, g, gam, *ch, cr, dt, solver, limiter, bc);
        double *s = A; A = B; B = s;
        if (dt_log) dt_log[step] = dt;
        t += dt;
        step += 1;
    }
    if (A != U) memcpy(U, A, sizeof(double) * n);
    free(T);
    free(A == U ? B : A);
    *t_out = t;
    *steps_out = step;
    return rc;
}

/* Exported single-function wrappers for ctypes (plain scalars and pointers). */
int orc_compute_dt_c(const double *U, int nx, int ny, int ng, double dx, double dy, double gam, double cfl,
                     double *ch, double *dt) {
    orc_grid g = {nx, ny, ng, dx, dy};
    return orc_compute_dt(U, &g, gam, cfl, ch, dt);
}
void orc_advance_c(const double *Uold, double *Utmp, double *Unew, int nx, int ny, int ng, double dx, double dy,
                   double gam, double ch, double cr, double dt, int solver, int limiter, const int *bc) {
    orc_grid g = {nx, ny, ng, dx, dy};
    orc_advance(Uold, Utmp, Unew, &g, gam, ch, cr, dt, solver, limiter, bc);
}
void orc_apply_boundary_c(double *U, int nx, int ny, int ng, const int *bc) {
    orc_grid g = {nx, ny, ng, 1.0, 1.0};
    orc_apply_boundary(U, &g, bc);
}
int orc_run_c(double *U, int nx, int ny, int ng, double dx, double dy, double gam, double cfl, double cr,
              int solver, int limiter, const int *bc, int max_steps, double t_end, double *ch, double *t_out,
              int *steps_out, double *dt_log) {
    orc_grid g = {nx, ny, ng, dx, dy};
    return orc_run(U, &g, gam, cfl, cr, solver, limiter, bc, max_steps, t_end, ch, t_out, steps_out, dt_log);
}
/* Single Riemann flux (for unit tests of the solvers). */
void orc_riemann_c(const double *UL, const double *UR, int dir, int solver, double ch, double gam, double *F) {
    riemann(UL, UR, dir, solver, ch, gam, F);
}
void orc_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : 1);
#else
    (void)n;
#endif
}
