// Host-side finite-difference check of the local adjoint functions in
// mhd_gpu_acc_b200/csrc/adj_physics.cuh (built and run by test_adjoint.py).
// For each function f and random inputs x, cotangent w: compares the adjoint's
// <J^T w, d> with the central difference (w . (f(x + h d) - f(x - h d))) / 2h
// for random directions d.  Prints the worst relative error and exits 1 above
// the threshold.
#include <cmath>
#include <cstdio>
#include <random>

#include "adj_physics.cuh"

using namespace mhd;
using namespace mhd::adj;

static std::mt19937_64 rng(12345);
static double uni(double a, double b) { return std::uniform_real_distribution<double>(a, b)(rng); }

static void rand_prim(double* W) {
    W[RHO] = uni(0.3, 2.0); W[PU] = uni(-1, 1); W[PV] = uni(-1, 1); W[PW] = uni(-0.5, 0.5);
    W[BX] = uni(-1, 1); W[BY] = uni(-1, 1); W[BZ] = uni(-0.5, 0.5); W[PP] = uni(0.2, 2.0); W[PSI] = uni(-0.1, 0.1);
}

static double worst = 0.0;
static void report(const char* name, double adj, double fd) {
    const double e = std::fabs(adj - fd) / std::fmax(1e-8, std::fabs(fd) + std::fabs(adj));
    if (e > worst) worst = e;
    if (e > 1e-6) std::printf("%-10s adj %.12e fd %.12e rel %.2e\n", name, adj, fd, e);
}

// HLLD degeneracy rule: FP64 keeps the reference's |d| < 1e-14; FP32 compares
// |d| with 1e-5 of rho (|S| + |un| + |SM|)^2 + Bn^2 (here 9 + 0.25 = 9.25).
static bool degeneracy_rule_ok() {
    bool ok = true;
    ok &= star_degenerate(1e-15, 1.0, 0.5, 1.5, 1.0, 0.5);
    ok &= !star_degenerate(1e-13, 1.0, 0.5, 1.5, 1.0, 0.5);
    ok &= star_degenerate(-1e-15, 1.0, 0.5, 1.5, 1.0, 0.5);
    ok &= star_degenerate(3e-8f, 1.0f, 0.5f, 1.5f, 1.0f, 0.5f);   // rounding-noise size in FP32
    ok &= star_degenerate(-9e-5f, 1.0f, 0.5f, 1.5f, 1.0f, 0.5f);  // |d| <= 9.25e-5
    ok &= !star_degenerate(1e-4f, 1.0f, 0.5f, 1.5f, 1.0f, 0.5f);
    ok &= star_degenerate(0.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f);    // all terms zero
    ok &= !star_degenerate(std::nanf(""), 1.0f, 0.5f, 1.5f, 1.0f, 0.5f);  // NaN: the non-degenerate path
    return ok;
}

int main() {
    if (!degeneracy_rule_ok()) {
        std::printf("star_degenerate: a known answer failed\n");
        return 1;
    }
    const double g = 5.0 / 3.0, h = 1e-6;
    for (int trial = 0; trial < 200; ++trial) {
        double W[NV], U[NV], d[NV], w[NV];
        rand_prim(W);
        p2c(W, g, U);
        for (int k = 0; k < NV; ++k) { d[k] = uni(-1, 1); w[k] = uni(-1, 1); }
        // c2p
        {
            double lU[NV] = {0}, Wc[NV], a[NV], b[NV], Up[NV], Um[NV];
            c2p(U, g, Wc);
            c2p_adj(U, Wc, g, w, lU);
            for (int k = 0; k < NV; ++k) { Up[k] = U[k] + h * d[k]; Um[k] = U[k] - h * d[k]; }
            c2p(Up, g, a); c2p(Um, g, b);
            double fd = 0, ad = 0;
            for (int k = 0; k < NV; ++k) { fd += w[k] * (a[k] - b[k]) / (2 * h); ad += lU[k] * d[k]; }
            report("c2p", ad, fd);
        }
        // p2c
        {
            double lW[NV] = {0}, a[NV], b[NV], Wp[NV], Wm[NV];
            p2c_adj(W, g, w, lW);
            for (int k = 0; k < NV; ++k) { Wp[k] = W[k] + h * d[k]; Wm[k] = W[k] - h * d[k]; }
            p2c(Wp, g, a); p2c(Wm, g, b);
            double fd = 0, ad = 0;
            for (int k = 0; k < NV; ++k) { fd += w[k] * (a[k] - b[k]) / (2 * h); ad += lW[k] * d[k]; }
            report("p2c", ad, fd);
        }
        // flux (with ch)
        {
            const double ch = uni(0.5, 2.0), dch = uni(-1, 1);
            double lW[NV] = {0}, lch = 0, a[NV], b[NV], Wp[NV], Wm[NV];
            flux_adj(W, ch, g, w, lW, lch);
            for (int k = 0; k < NV; ++k) { Wp[k] = W[k] + h * d[k]; Wm[k] = W[k] - h * d[k]; }
            flux(Wp, ch + h * dch, g, a); flux(Wm, ch - h * dch, g, b);
            double fd = 0, ad = lch * dch;
            for (int k = 0; k < NV; ++k) { fd += w[k] * (a[k] - b[k]) / (2 * h); ad += lW[k] * d[k]; }
            report("flux", ad, fd);
        }
        // fast speed
        {
            double lW[NV] = {0}, Wp[NV], Wm[NV];
            fast_adj(W, g, 1.3, lW);
            for (int k = 0; k < NV; ++k) { Wp[k] = W[k] + h * d[k]; Wm[k] = W[k] - h * d[k]; }
            const double fd = 1.3 * (fast(Wp, g) - fast(Wm, g)) / (2 * h);
            double ad = 0;
            for (int k = 0; k < NV; ++k) ad += lW[k] * d[k];
            report("fast", ad, fd);
        }
        // hll (both sides and ch), smooth region of the inputs
        {
            double W2[NV], U2[NV], d2[NV];
            rand_prim(W2);
            p2c(W2, g, U2);
            for (int k = 0; k < NV; ++k) d2[k] = uni(-1, 1);
            const double ch = uni(0.2, 3.0), dch = uni(-1, 1);
            double lL[NV] = {0}, lR[NV] = {0}, lch = 0, a[NV], b[NV], Lp[NV], Lm[NV], Rp[NV], Rm[NV];
            hll_adj(U, U2, ch, g, w, lL, lR, lch);
            for (int k = 0; k < NV; ++k) {
                Lp[k] = U[k] + h * d[k]; Lm[k] = U[k] - h * d[k];
                Rp[k] = U2[k] + h * d2[k]; Rm[k] = U2[k] - h * d2[k];
            }
            hll(Lp, Rp, ch + h * dch, g, a); hll(Lm, Rm, ch - h * dch, g, b);
            double fd = 0, ad = lch * dch;
            for (int k = 0; k < NV; ++k) { fd += w[k] * (a[k] - b[k]) / (2 * h); ad += lL[k] * d[k] + lR[k] * d2[k]; }
            report("hll", ad, fd);
        }
        // reconstruction (van Leer and minmod), dtd and ch
        for (int lim = 0; lim < 2; ++lim) {
            double Wm_[NV], Wp_[NV], dm[NV], dp[NV], w2[NV];
            rand_prim(Wm_);
            rand_prim(Wp_);
            for (int k = 0; k < NV; ++k) {
                Wm_[k] = 0.7 * W[k] + 0.3 * Wm_[k];  // keep neighbours close: smooth limiter region
                Wp_[k] = 0.7 * W[k] + 0.3 * Wp_[k];
                dm[k] = uni(-1, 1); dp[k] = uni(-1, 1); w2[k] = uni(-1, 1);
            }
            const double dtd = uni(0.05, 0.3), ch = uni(0.5, 2.0), ddt = uni(-1, 1), dch = uni(-1, 1);
            double lWm[NV] = {0}, lWc[NV] = {0}, lWp[NV] = {0}, ldtd = 0, lch = 0;
            double Lp[NV], Rp[NV], Lm[NV], Rm[NV], A[NV], B[NV], C_[NV], A2[NV], B2[NV], C2[NV];
            if (lim) recon_adj<VANLEER>(Wm_, W, Wp_, dtd, ch, g, w, w2, lWm, lWc, lWp, ldtd, lch);
            else recon_adj<MINMOD>(Wm_, W, Wp_, dtd, ch, g, w, w2, lWm, lWc, lWp, ldtd, lch);
            for (int k = 0; k < NV; ++k) {
                A[k] = Wm_[k] + h * dm[k]; B[k] = W[k] + h * d[k]; C_[k] = Wp_[k] + h * dp[k];
                A2[k] = Wm_[k] - h * dm[k]; B2[k] = W[k] - h * d[k]; C2[k] = Wp_[k] - h * dp[k];
            }
            if (lim) {
                recon<VANLEER>(A, B, C_, dtd + h * ddt, ch + h * dch, g, Lp, Rp);
                recon<VANLEER>(A2, B2, C2, dtd - h * ddt, ch - h * dch, g, Lm, Rm);
            } else {
                recon<MINMOD>(A, B, C_, dtd + h * ddt, ch + h * dch, g, Lp, Rp);
                recon<MINMOD>(A2, B2, C2, dtd - h * ddt, ch - h * dch, g, Lm, Rm);
            }
            double fd = 0, ad = ldtd * ddt + lch * dch;
            for (int k = 0; k < NV; ++k) {
                fd += (w[k] * (Lp[k] - Lm[k]) + w2[k] * (Rp[k] - Rm[k])) / (2 * h);
                ad += lWm[k] * dm[k] + lWc[k] * d[k] + lWp[k] * dp[k];
            }
            report(lim ? "recon_vl" : "recon_mm", ad, fd);
        }
        // CFL speed
        {
            int br = 0;
            raw_speed(U, g, &br);
            double lU[NV] = {0}, Up[NV], Um[NV];
            raw_speed_adj(U, g, br, 0.7, lU);
            for (int k = 0; k < NV; ++k) { Up[k] = U[k] + h * d[k]; Um[k] = U[k] - h * d[k]; }
            int b1 = 0, b2 = 0;
            const double fd = 0.7 * (raw_speed(Up, g, &b1) - raw_speed(Um, g, &b2)) / (2 * h);
            double ad = 0;
            for (int k = 0; k < NV; ++k) ad += lU[k] * d[k];
            if (b1 == br && b2 == br) report("speed", ad, fd);
        }
    }
    // HLLD face (with the GLM overwrite and the HLL fallbacks): states spread so
    // that every region is taken; a check counts only when both perturbed
    // evaluations stay in the region of the base point.
    int hits[7] = {0};
    for (int trial = 0; trial < 6000; ++trial) {
        double WL[NV], WR[NV], UL[NV], UR[NV], dL[NV], dR[NV], w[NV];
        rand_prim(WL);
        rand_prim(WR);
        WL[PU] = uni(-2.5, 2.5);
        WR[PU] = WL[PU] + uni(-1.5, 1.5);
        WL[BX] = uni(-1.5, 1.5);
        WR[BX] = WL[BX] + uni(-0.2, 0.2);
        WL[PP] = uni(0.05, 2.0);
        p2c(WL, g, UL);
        p2c(WR, g, UR);
        for (int k = 0; k < NV; ++k) { dL[k] = uni(-1, 1); dR[k] = uni(-1, 1); w[k] = uni(-1, 1); }
        const double ch = uni(0.2, 3.0), dch = uni(-1, 1);
        HlldState<double> s0, sp, sm;
        double Lp[NV], Lm[NV], Rp[NV], Rm[NV];
        for (int k = 0; k < NV; ++k) {
            Lp[k] = UL[k] + h * dL[k]; Lm[k] = UL[k] - h * dL[k];
            Rp[k] = UR[k] + h * dR[k]; Rm[k] = UR[k] - h * dR[k];
        }
        hlld_state(UL, UR, ch, g, s0);
        hlld_state(Lp, Rp, ch + h * dch, g, sp);
        hlld_state(Lm, Rm, ch - h * dch, g, sm);
        if (sp.region != s0.region || sm.region != s0.region) continue;
        hits[s0.region + 1]++;
        double lL[NV] = {0}, lR[NV] = {0}, lch = 0, a[NV], b[NV];
        face_adj<HLLD>(UL, UR, ch, g, w, lL, lR, lch);
        face<HLLD>(Lp, Rp, ch + h * dch, g, a);
        face<HLLD>(Lm, Rm, ch - h * dch, g, b);
        double fd = 0, ad = lch * dch;
        for (int k = 0; k < NV; ++k) { fd += w[k] * (a[k] - b[k]) / (2 * h); ad += lL[k] * dL[k] + lR[k] * dR[k]; }
        static const char* names[7] = {"hlld_hll", "hlld_FL", "hlld_FR", "hlld_L*", "hlld_L**", "hlld_R*", "hlld_R**"};
        report(names[s0.region + 1], ad, fd);
    }
    std::printf("HLLD regions checked (HLL, FL, FR, L*, L**, R*, R**): %d %d %d %d %d %d %d\n", hits[0], hits[1],
                hits[2], hits[3], hits[4], hits[5], hits[6]);
    for (int r = 1; r < 7; ++r)
        if (hits[r] < 20) {
            std::printf("HLLD region %d checked only %d times\n", r - 1, hits[r]);
            return 1;
        }
    std::printf("worst relative error %.3e\n", worst);
    return worst < 1e-5 ? 0 : 1;
}
