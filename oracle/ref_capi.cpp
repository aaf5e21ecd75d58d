// ref_capi.cpp -- C-ABI shim that drives the reference's OWN CPU/OpenMP step.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference's unmodified sources (src/cpu/solver_cpu.cpp,
// src/test_cases.cpp, src/init.cpp and the head/ headers, read where they lie
// in the reference checkout) into oracle/_ref/libmhdref.so.  Nothing of the
// reference is copied into this repository.  Only tests/, tests/golden's
// fixture generator and bench.py's reference / cpu_baseline legs load it.
//
// The shim converts between this project's SoA layout (9 planes of
// (nx+2ng)*(ny+2ng) doubles, row-major) and the reference's AoS Grid2D, and
// resets the reference's process globals phys::gamma and phys::ch_glm
// (head/physics.hpp:30,41) before every call.
#include <chrono>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "cpu/boundary_cpu.hpp"
#include "cpu/grid_cpu.hpp"
#include "cpu/solver_cpu.hpp"
#include "physics.hpp"
#include "riemann.hpp"
#include "test_cases.hpp"

namespace {

Grid2D make_grid(int nx, int ny, int ng, double x0, double x1, double y0, double y1) {
    return Grid2D(nx, ny, ng, x0, x1, y0, y1);
}

void soa_to_grid(const double* U, Grid2D& g) {
    const std::size_t n = static_cast<std::size_t>(g.total_nx()) * g.total_ny();
    auto& d = g.data();
    for (std::size_t k = 0; k < n; ++k) {
        d[k] = Conserved(U[0 * n + k], U[1 * n + k], U[2 * n + k], U[3 * n + k], U[4 * n + k],
                         U[5 * n + k], U[6 * n + k], U[7 * n + k], U[8 * n + k]);
    }
}

void grid_to_soa(const Grid2D& g, double* U) {
    const std::size_t n = static_cast<std::size_t>(g.total_nx()) * g.total_ny();
    const auto& d = g.data();
    for (std::size_t k = 0; k < n; ++k) {
        U[0 * n + k] = d[k].rho;  U[1 * n + k] = d[k].rhou; U[2 * n + k] = d[k].rhov;
        U[3 * n + k] = d[k].rhow; U[4 * n + k] = d[k].Bx;   U[5 * n + k] = d[k].By;
        U[6 * n + k] = d[k].Bz;   U[7 * n + k] = d[k].E;    U[8 * n + k] = d[k].psi;
    }
}

BoundaryConfig to_bc(const int* bc) {
    BoundaryConfig c;
    c.left = static_cast<BoundaryType>(bc[0]);
    c.right = static_cast<BoundaryType>(bc[1]);
    c.bottom = static_cast<BoundaryType>(bc[2]);
    c.top = static_cast<BoundaryType>(bc[3]);
    return c;
}

void put9(const Conserved& c, double* o) {
    o[0] = c.rho; o[1] = c.rhou; o[2] = c.rhov; o[3] = c.rhow; o[4] = c.Bx;
    o[5] = c.By;  o[6] = c.Bz;   o[7] = c.E;    o[8] = c.psi;
}

Conserved get9(const double* o) {
    return Conserved(o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7], o[8]);
}

}  // namespace

extern "C" {

void ref_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : 1);
#else
    (void)n;
#endif
}

int ref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// compute_dt (src/cpu/solver_cpu.cpp:283-312).  *ch: in = previous ch_glm,
// out = new ch_glm.  Returns -1 where the reference throws.
int ref_compute_dt(const double* U, int nx, int ny, int ng, double x0, double x1, double y0, double y1,
                   double gamma, double cfl, double* ch, double* dt) {
    Grid2D g = make_grid(nx, ny, ng, x0, x1, y0, y1);
    soa_to_grid(U, g);
    phys::gamma = gamma;
    phys::ch_glm = *ch;
    try {
        *dt = compute_dt(g, cfl);
    } catch (const std::exception&) {
        return -1;
    }
    *ch = phys::ch_glm;
    return 0;
}

// advance_second_order (src/cpu/solver_cpu.cpp:327-440) with ch_glm = ch.
int ref_advance(const double* Uold, double* Utmp, double* Unew, int nx, int ny, int ng, double x0, double x1,
                double y0, double y1, double gamma, double ch, double dt, int solver, const int* bc) {
    Grid2D a = make_grid(nx, ny, ng, x0, x1, y0, y1);
    Grid2D t = make_grid(nx, ny, ng, x0, x1, y0, y1);
    Grid2D b = make_grid(nx, ny, ng, x0, x1, y0, y1);
    soa_to_grid(Uold, a);
    soa_to_grid(Utmp, t);
    soa_to_grid(Unew, b);
    phys::gamma = gamma;
    phys::ch_glm = ch;
    CpuWorkspace ws;
    ws.init(nx, ny);
    advance_second_order(a, t, b, dt, ws, static_cast<RiemannSolver>(solver), to_bc(bc));
    grid_to_soa(t, Utmp);
    grid_to_soa(b, Unew);
    return 0;
}

// apply_boundary (head/cpu/boundary_cpu.hpp:45-149), in place.
int ref_apply_boundary(double* U, int nx, int ny, int ng, const int* bc) {
    Grid2D g = make_grid(nx, ny, ng, 0.0, 1.0, 0.0, 1.0);
    soa_to_grid(U, g);
    apply_boundary(g, to_bc(bc));
    grid_to_soa(g, U);
    return 0;
}

// The time loop of scripts/cpu/main_cpu.cpp:196-222 (dt clamp and guards;
// no snapshots).  Return codes: 0 ok, -1 compute_dt threw, -2 dt non-finite or
// non-positive, -3 dt below 1e-8 t_end.
int ref_run(double* U, int nx, int ny, int ng, double x0, double x1, double y0, double y1, double gamma,
            double cfl, int solver, const int* bc, int max_steps, double t_end, double* ch, double* t_out,
            int* steps_out, double* dt_log) {
    Grid2D Uold = make_grid(nx, ny, ng, x0, x1, y0, y1);
    soa_to_grid(U, Uold);
    Grid2D Unew = Uold;
    Grid2D Utmp = Uold;
    CpuWorkspace ws;
    ws.init(nx, ny);
    phys::gamma = gamma;
    phys::ch_glm = *ch;
    const RiemannSolver rs = static_cast<RiemannSolver>(solver);
    const BoundaryConfig bcc = to_bc(bc);
    double t = 0.0;
    int step = 0, rc = 0;
    while (t < t_end && (max_steps <= 0 || step < max_steps)) {
        double dt_raw;
        try {
            dt_raw = compute_dt(Uold, cfl);
        } catch (const std::exception&) {
            rc = -1;
            break;
        }
        const double dt = std::min(dt_raw, t_end - t);
        if (!std::isfinite(dt) || dt <= 0.0) { rc = -2; break; }
        if (dt < 1.0e-8 * t_end) { rc = -3; break; }
        advance_second_order(Uold, Utmp, Unew, dt, ws, rs, bcc);
        std::swap(Uold, Unew);
        if (dt_log) dt_log[step] = dt;
        t += dt;
        step += 1;
    }
    grid_to_soa(Uold, U);
    *ch = phys::ch_glm;
    *t_out = t;
    *steps_out = step;
    return rc;
}

// Same loop with each step's wall time (steady_clock around compute_dt +
// advance + swap, the span the reference's [TIMING] line covers,
// scripts/cpu/main_cpu.cpp:191-257) written to step_seconds[max_steps].
int ref_run_timed(double* U, int nx, int ny, int ng, double x0, double x1, double y0, double y1, double gamma,
                  double cfl, int solver, const int* bc, int max_steps, double t_end, double* ch,
                  double* step_seconds, int* steps_out) {
    Grid2D Uold = make_grid(nx, ny, ng, x0, x1, y0, y1);
    soa_to_grid(U, Uold);
    Grid2D Unew = Uold;
    Grid2D Utmp = Uold;
    CpuWorkspace ws;
    ws.init(nx, ny);
    phys::gamma = gamma;
    phys::ch_glm = *ch;
    const RiemannSolver rs = static_cast<RiemannSolver>(solver);
    const BoundaryConfig bcc = to_bc(bc);
    double t = 0.0;
    int step = 0, rc = 0;
    while (t < t_end && step < max_steps) {
        const auto t0 = std::chrono::steady_clock::now();
        double dt_raw;
        try {
            dt_raw = compute_dt(Uold, cfl);
        } catch (const std::exception&) {
            rc = -1;
            break;
        }
        const double dt = std::min(dt_raw, t_end - t);
        if (!std::isfinite(dt) || dt <= 0.0) { rc = -2; break; }
        advance_second_order(Uold, Utmp, Unew, dt, ws, rs, bcc);
        std::swap(Uold, Unew);
        step_seconds[step] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        t += dt;
        step += 1;
    }
    grid_to_soa(Uold, U);
    *ch = phys::ch_glm;
    *steps_out = step;
    return rc;
}

// initial_state_at (src/test_cases.cpp:288-296) for the reference's own cases.
// case_id follows CaseId (head/test_cases.hpp:28-33).
void ref_initial_state(int case_id, double x, double y, double* out9) {
    put9(initial_state_at(static_cast<CaseId>(case_id), x, y), out9);
}

// The Orszag-Tang vortex on periodic [0,1]^2 (rho = 25/(36 pi), p = 5/(12 pi),
// v = (-sin 2 pi y, sin 2 pi x, 0), B = B0 (-sin 2 pi y, sin 4 pi x, 0),
// B0 = 1/sqrt(4 pi), gamma 5/3, psi = 0) -- a configuration the reference does
// not have -- evaluated at the reference Grid2D's own cell centres
// (head/cpu/grid_cpu.hpp:54-60, ghosts included) and converted with the
// reference's prim_to_cons (head/physics.hpp:83-90), so that the reference's
// CPU step can be driven on this configuration without any other library.
// U: SoA, 9 planes of (nx + 2 ng) x (ny + 2 ng) doubles.
int ref_initialise_orszag_tang_unit(int nx, int ny, int ng, double* U) {
    if (!U || nx < 1 || ny < 1 || ng < 0) return -1;
    const double pi = 3.14159265358979323846;
    Grid2D g = make_grid(nx, ny, ng, 0.0, 1.0, 0.0, 1.0);
    phys::gamma = 5.0 / 3.0;
    const double rho = 25.0 / (36.0 * pi);
    const double p = 5.0 / (12.0 * pi);
    const double B0 = 1.0 / std::sqrt(4.0 * pi);
    for (int j = 0; j < g.total_ny(); ++j) {
        const double y = g.y_center(j);
        for (int i = 0; i < g.total_nx(); ++i) {
            const double x = g.x_center(i);
            Primitive V;
            V.rho = rho; V.u = -std::sin(2.0 * pi * y); V.v = std::sin(2.0 * pi * x); V.w = 0.0;
            V.Bx = -B0 * std::sin(2.0 * pi * y); V.By = B0 * std::sin(4.0 * pi * x); V.Bz = 0.0;
            V.p = p; V.psi = 0.0;
            g(i, j) = phys::prim_to_cons(V);
        }
    }
    grid_to_soa(g, U);
    return 0;
}

// get_n_case_config (src/test_cases.cpp:275-282): grid and physics scalars.
// out: nx, ny, ng (as doubles), x_min, x_max, y_min, y_max, cfl, t_end, gamma,
// bc[4] (as doubles)  -> 14 values.
int ref_case_config(int case_id, int n, double* out) {
    CaseConfig c;
    try {
        c = get_n_case_config(static_cast<CaseId>(case_id), n);
    } catch (const std::exception&) {
        return -1;
    }
    out[0] = c.nx; out[1] = c.ny; out[2] = c.ng;
    out[3] = c.x_min; out[4] = c.x_max; out[5] = c.y_min; out[6] = c.y_max;
    out[7] = c.cfl; out[8] = c.t_end; out[9] = c.gamma;
    out[10] = static_cast<int>(c.bc.left); out[11] = static_cast<int>(c.bc.right);
    out[12] = static_cast<int>(c.bc.bottom); out[13] = static_cast<int>(c.bc.top);
    return 0;
}

// riemann_flux (head/riemann.hpp:568-592) on one face, for solver unit tests.
void ref_riemann(const double* UL, const double* UR, int dir, int solver, double ch, double gamma, double* F) {
    phys::gamma = gamma;
    const Conserved f = riemann_flux(get9(UL), get9(UR), dir == 0 ? Direction::X : Direction::Y,
                                     static_cast<RiemannSolver>(solver), ch);
    put9(f, F);
}

}  // extern "C"
