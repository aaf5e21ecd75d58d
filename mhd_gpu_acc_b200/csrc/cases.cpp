// cases.cpp -- test-case configurations and initial states.
//
// The reference's four cases keep its formulas and constants term for term
// (src/test_cases.cpp:24-148, configs :178-269), so the initial grids agree
// bit for bit with the reference's initialise_grid (src/init.cpp:34-43).  Three
// configurations are added:
//   MHD_CASE_ORSZAG_TANG_UNIT  Orszag-Tang on periodic [0,1]^2: rho = 25/(36 pi),
//                              p = 5/(12 pi), v = (-sin 2pi y, sin 2pi x, 0),
//                              B = B0 (-sin 2pi y, sin 4pi x, 0), B0 = 1/sqrt(4 pi),
//                              gamma 5/3, CFL 0.4, t_end 0.5; base 512^2.
//   MHD_CASE_SHOCK_BUBBLE_MHD  Mach-10 planar shock at x = 0.6 on [0,1]^2 with
//                              outflow boundaries; pre-shock rho = 1, p = 1, v = 0,
//                              B = (0, 2/sqrt(4 pi), 0) everywhere; post-shock rho,
//                              u, p from the hydrodynamic Rankine-Hugoniot
//                              relations (gamma 5/3) on the x < 0.6 side, so the
//                              shock runs toward the dense bubble (radius 0.15 at
//                              (0.8, 0.5), rho = 10, p = 1); CFL 0.4, t_end 0.06;
//                              base 256^2 (n = 8 gives 2048^2).
//   MHD_CASE_BRIO_WU_CFL08     the Brio-Wu state on 800x4 with CFL 0.8 and all
//                              sides transmissive, t_end 0.1.
#include <cmath>
#include <cstring>

#include "../../include/mhd_b200.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace {

struct Cons { double rho, rhou, rhov, rhow, Bx, By, Bz, E, psi; };

// make_mhd (src/test_cases.cpp:24-35): psi = 0.
Cons make_mhd(double rho, double ux, double uy, double uz, double Bx, double By, double Bz, double p,
              double gamma) {
    const double Bmag2 = Bx * Bx + By * By + Bz * Bz;
    const double ke = 0.5 * rho * (ux * ux + uy * uy + uz * uz);
    const double E = p / (gamma - 1.0) + ke + 0.5 * Bmag2;
    return Cons{rho, rho * ux, rho * uy, rho * uz, Bx, By, Bz, E, 0.0};
}

// kh_state (src/test_cases.cpp:43-63)
Cons kelvin_helmholtz(double x, double y) {
    constexpr double gamma = 1.4;
    const double ux = 5.0 * (tanh(20.0 * (y + 0.5)) - (tanh(20.0 * (y - 0.5)) + 1.0));
    const double uy = 0.25 * sin(2.0 * M_PI * x) *
                      (exp(-100.0 * (y + 0.5) * (y + 0.5)) - exp(-100.0 * (y - 0.5) * (y - 0.5)));
    return make_mhd(1.0, ux, uy, 0.0, 1.0, 0.0, 0.0, 50.0, gamma);
}

// shock_bubble_state (src/test_cases.cpp:76-106): Mach 1.22 air / helium, B = 0.
Cons shock_bubble(double x, double y) {
    constexpr double gamma = 1.4, rho_air = 1.29, rho_He = 0.214, p0 = 1.01325e5, Ms = 1.22;
    constexpr double xc = 0.035, yc = 0.0445, R = 0.025, xs = 0.005;
    static const double c1 = std::sqrt(gamma * p0 / rho_air);
    static const double vs = Ms * c1;
    static const double rho2 = rho_air * (gamma + 1.0) * Ms * Ms / ((gamma - 1.0) * Ms * Ms + 2.0);
    static const double p2 = p0 * (2.0 * gamma * Ms * Ms - (gamma - 1.0)) / (gamma + 1.0);
    static const double u2 = vs * (1.0 - rho_air / rho2);
    if (x < xs) return make_mhd(rho2, u2, 0.0, 0.0, 0.0, 0.0, 0.0, p2, gamma);
    const double r2 = (x - xc) * (x - xc) + (y - yc) * (y - yc);
    if (r2 < R * R) return make_mhd(rho_He, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, p0, gamma);
    return make_mhd(rho_air, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, p0, gamma);
}

// brio_wu_state (src/test_cases.cpp:117-126)
Cons brio_wu(double x, double) {
    constexpr double gamma = 2.0, Bx = 0.75;
    if (x < 0.5) return make_mhd(1.0, 0.0, 0.0, 0.0, Bx, 1.0, 0.0, 1.0, gamma);
    return make_mhd(0.125, 0.0, 0.0, 0.0, Bx, -1.0, 0.0, 0.1, gamma);
}

// orszag_tang_state (src/test_cases.cpp:139-148): [0, 2pi]^2, rho = gamma^2, p = gamma.
Cons orszag_tang(double x, double y) {
    constexpr double gamma = 5.0 / 3.0;
    const double rho = gamma * gamma;
    const double p = gamma;
    const double u = -std::sin(y);
    const double v = std::sin(x);
    const double Bx = -std::sin(y);
    const double By = std::sin(2.0 * x);
    return make_mhd(rho, u, v, 0.0, Bx, By, 0.0, p, gamma);
}

// Orszag-Tang on [0,1]^2 (the [0,2pi]^2 flow under the ideal-MHD scaling).
Cons orszag_tang_unit(double x, double y) {
    constexpr double gamma = 5.0 / 3.0;
    const double rho = 25.0 / (36.0 * M_PI);
    const double p = 5.0 / (12.0 * M_PI);
    const double B0 = 1.0 / std::sqrt(4.0 * M_PI);
    const double u = -std::sin(2.0 * M_PI * y);
    const double v = std::sin(2.0 * M_PI * x);
    const double Bx = -B0 * std::sin(2.0 * M_PI * y);
    const double By = B0 * std::sin(4.0 * M_PI * x);
    return make_mhd(rho, u, v, 0.0, Bx, By, 0.0, p, gamma);
}

// Mach-10 MHD shock - dense bubble.
Cons shock_bubble_mhd(double x, double y) {
    constexpr double gamma = 5.0 / 3.0, rho1 = 1.0, p1 = 1.0, M = 10.0;
    const double By = 2.0 / std::sqrt(4.0 * M_PI);
    static const double c1 = std::sqrt(gamma * p1 / rho1);
    static const double vs = M * c1;
    static const double rho2 = rho1 * (gamma + 1.0) * M * M / ((gamma - 1.0) * M * M + 2.0);
    static const double p2 = p1 * (2.0 * gamma * M * M - (gamma - 1.0)) / (gamma + 1.0);
    static const double u2 = vs * (1.0 - rho1 / rho2);
    if (x < 0.6) return make_mhd(rho2, u2, 0.0, 0.0, 0.0, By, 0.0, p2, gamma);
    const double r2 = (x - 0.8) * (x - 0.8) + (y - 0.5) * (y - 0.5);
    if (r2 < 0.15 * 0.15) return make_mhd(10.0, 0.0, 0.0, 0.0, 0.0, By, 0.0, p1, gamma);
    return make_mhd(rho1, 0.0, 0.0, 0.0, 0.0, By, 0.0, p1, gamma);
}

bool state_at(int id, double x, double y, Cons& c) {
    switch (id) {
        case MHD_CASE_KELVIN_HELMHOLTZ: c = kelvin_helmholtz(x, y); return true;
        case MHD_CASE_SHOCK_BUBBLE: c = shock_bubble(x, y); return true;
        case MHD_CASE_BRIO_WU:
        case MHD_CASE_BRIO_WU_CFL08: c = brio_wu(x, y); return true;
        case MHD_CASE_ORSZAG_TANG: c = orszag_tang(x, y); return true;
        case MHD_CASE_ORSZAG_TANG_UNIT: c = orszag_tang_unit(x, y); return true;
        case MHD_CASE_SHOCK_BUBBLE_MHD: c = shock_bubble_mhd(x, y); return true;
        default: return false;
    }
}

void put(const Cons& c, double* o) {
    o[0] = c.rho; o[1] = c.rhou; o[2] = c.rhov; o[3] = c.rhow; o[4] = c.Bx;
    o[5] = c.By; o[6] = c.Bz; o[7] = c.E; o[8] = c.psi;
}

}  // namespace

extern "C" {

int mhd_case_config(int id, int n, double* o) {
    if (!o || n < 1) return MHD_ERR_ARG;
    const double P = MHD_BC_PERIODIC, T = MHD_BC_TRANSMISSIVE;
    double nx, ny, x0, x1, y0, y1, cfl, tend, gam, b0, b1, b2, b3;
    switch (id) {
        case MHD_CASE_KELVIN_HELMHOLTZ:  // src/test_cases.cpp:181-192
            nx = 200; ny = 400; x0 = 0.0; x1 = 1.0; y0 = -1.0; y1 = 1.0; cfl = 0.3; tend = 0.5; gam = 1.4;
            b0 = b1 = b2 = b3 = P;
            break;
        case MHD_CASE_SHOCK_BUBBLE: {  // src/test_cases.cpp:194-234 (t_end = last snapshot time)
            nx = 500; ny = 197; x0 = 0.0; x1 = 0.225; y0 = 0.0; y1 = 0.089; cfl = 0.4; gam = 1.4;
            const double vs = 1.22 * std::sqrt(1.4 * 1.01325e5 / 1.29);
            const double T0 = (0.035 - 0.025 - 0.005) / vs;
            const double tau = 0.025 / vs;
            tend = T0 + 19.0 * tau;
            b0 = b1 = b2 = b3 = T;
            break;
        }
        case MHD_CASE_BRIO_WU:  // src/test_cases.cpp:236-247
            nx = 800; ny = 4; x0 = 0.0; x1 = 1.0; y0 = 0.0; y1 = 4.0 / 800.0; cfl = 0.4; tend = 0.1; gam = 2.0;
            b0 = b1 = T; b2 = b3 = P;
            break;
        case MHD_CASE_ORSZAG_TANG:  // src/test_cases.cpp:249-266
            nx = 192; ny = 192; x0 = 0.0; x1 = 2.0 * M_PI; y0 = 0.0; y1 = 2.0 * M_PI; cfl = 0.4;
            tend = 2.0 * M_PI; gam = 5.0 / 3.0;
            b0 = b1 = b2 = b3 = P;
            break;
        case MHD_CASE_ORSZAG_TANG_UNIT:
            nx = 512; ny = 512; x0 = 0.0; x1 = 1.0; y0 = 0.0; y1 = 1.0; cfl = 0.4; tend = 0.5; gam = 5.0 / 3.0;
            b0 = b1 = b2 = b3 = P;
            break;
        case MHD_CASE_SHOCK_BUBBLE_MHD:
            nx = 256; ny = 256; x0 = 0.0; x1 = 1.0; y0 = 0.0; y1 = 1.0; cfl = 0.4; tend = 0.06; gam = 5.0 / 3.0;
            b0 = b1 = b2 = b3 = T;
            break;
        case MHD_CASE_BRIO_WU_CFL08:
            nx = 800; ny = 4; x0 = 0.0; x1 = 1.0; y0 = 0.0; y1 = 4.0 / 800.0; cfl = 0.8; tend = 0.1; gam = 2.0;
            b0 = b1 = b2 = b3 = T;
            break;
        default: return MHD_ERR_ARG;
    }
    // get_n_case_config scales both directions by n (src/test_cases.cpp:275-282)
    const double vals[14] = {nx * n, ny * n, 2.0, x0, x1, y0, y1, cfl, tend, gam, b0, b1, b2, b3};
    std::memcpy(o, vals, sizeof vals);
    return MHD_OK;
}

int mhd_initial_state(int id, double x, double y, double* out9) {
    if (!out9) return MHD_ERR_ARG;
    Cons c;
    if (!state_at(id, x, y, c)) return MHD_ERR_ARG;
    put(c, out9);
    return MHD_OK;
}

// initialise_grid (src/init.cpp:34-43) with cell centres x_min + (i - ng + 0.5) dx
// (head/cpu/grid_cpu.hpp:54-60), ghosts included.
int mhd_initialise(int id, int nx, int ny, int ng, double x_min, double x_max, double y_min, double y_max,
                   double* host) {
    if (!host || nx < 1 || ny < 1 || ng < 0) return MHD_ERR_ARG;
    Cons probe;
    if (!state_at(id, 0.0, 0.0, probe)) return MHD_ERR_ARG;
    const double dx = (x_max - x_min) / static_cast<double>(nx);
    const double dy = (y_max - y_min) / static_cast<double>(ny);
    const long long tnx = nx + 2LL * ng, tny = ny + 2LL * ng, np = tnx * tny;
    for (long long j = 0; j < tny; ++j) {
        const double y = y_min + (static_cast<double>(j - ng) + 0.5) * dy;
        for (long long i = 0; i < tnx; ++i) {
            const double x = x_min + (static_cast<double>(i - ng) + 0.5) * dx;
            Cons c;
            state_at(id, x, y, c);
            double v[9];
            put(c, v);
            const long long k = j * tnx + i;
            for (int f = 0; f < 9; ++f) host[f * np + k] = v[f];
        }
    }
    return MHD_OK;
}

}  // extern "C"
