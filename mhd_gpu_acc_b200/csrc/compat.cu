// compat.cu -- the reference's C++ API (include/mhd_b200/*.hpp, *.cuh) on top
// of the C ABI.  Host code only: the physics and Riemann functions reuse the
// FP64 functions the kernels run (phys_exact.cuh, compiled here for the host),
// so phys::cons_to_prim or riemann_flux agree bit for bit with the reference's
// header-inline versions.
#include <cmath>
#include <iomanip>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>

#include "../../include/mhd_b200.h"
#include "../../include/mhd_b200/gpu/boundary_gpu.cuh"
#include "../../include/mhd_b200/gpu/solver_gpu.cuh"
#include "../../include/mhd_b200/init.hpp"
#include "phys_exact.cuh"

namespace phys {
double gamma = 5.0 / 3.0;  // head/physics.hpp:28
double ch_glm = 0.0;       // head/physics.hpp:38
double cr_glm = 0.18;      // head/physics.hpp:39
}  // namespace phys

namespace {

const double* ptr(const Conserved& c) { return &c.rho; }
const double* ptr(const Primitive& p) { return &p.rho; }

Conserved to_cons(const double* v) { return Conserved(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8]); }
Primitive to_prim(const double* v) { return Primitive(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8]); }

Limiter g_limiter = Limiter::Minmod;

template <int DIR>
Conserved solve(const Conserved& UL, const Conserved& UR, int which, double ch, double g) {
    double F[9];
    switch (which) {
        case 0: mhd::exact::hll<DIR>(ptr(UL), ptr(UR), ch, g, F); break;
        case 1: mhd::exact::hllc<DIR>(ptr(UL), ptr(UR), ch, g, F); break;
        case 2: mhd::exact::hlld<DIR>(ptr(UL), ptr(UR), ch, g, F); break;
        case 3: mhd::exact::force<DIR>(ptr(UL), ptr(UR), ch, g, F); break;
        case 10: mhd::exact::riemann<DIR, 0>(ptr(UL), ptr(UR), ch, g, F); break;
        case 11: mhd::exact::riemann<DIR, 1>(ptr(UL), ptr(UR), ch, g, F); break;
        case 12: mhd::exact::riemann<DIR, 2>(ptr(UL), ptr(UR), ch, g, F); break;
        default: mhd::exact::riemann<DIR, 3>(ptr(UL), ptr(UR), ch, g, F); break;
    }
    return to_cons(F);
}

Conserved solve_dir(const Conserved& UL, const Conserved& UR, Direction d, int which, double ch,
                    double g = phys::gamma) {
    return d == Direction::X ? solve<0>(UL, UR, which, ch, g) : solve<1>(UL, UR, which, ch, g);
}

int bc_array(const BoundaryConfig& b, int* out) {
    out[0] = static_cast<int>(b.left);
    out[1] = static_cast<int>(b.right);
    out[2] = static_cast<int>(b.bottom);
    out[3] = static_cast<int>(b.top);
    return 0;
}

}  // namespace

// ---- physics (head/physics.hpp) ----
namespace phys {
Primitive cons_to_prim(const Conserved& U) {
    double W[9];
    mhd::exact::c2p(ptr(U), gamma, W);
    return to_prim(W);
}
Conserved prim_to_cons(const Primitive& V) {
    double U[9];
    mhd::exact::p2c(ptr(V), gamma, U);
    return to_cons(U);
}
Conserved flux_x(const Conserved& U, double ch) {
    double F[9];
    mhd::exact::flux<0>(ptr(U), ch, gamma, F);
    return to_cons(F);
}
Conserved flux_y(const Conserved& U, double ch) {
    double F[9];
    mhd::exact::flux<1>(ptr(U), ch, gamma, F);
    return to_cons(F);
}
double fast_speed_x(const Primitive& V) { return mhd::exact::fast_speed<0>(ptr(V), gamma); }
double fast_speed_y(const Primitive& V) { return mhd::exact::fast_speed<1>(ptr(V), gamma); }
double sound_speed(const Primitive& V) { return std::sqrt(gamma * V.p / V.rho); }
double max_signal_speed_x(const Primitive& V, double ch) { return std::fmax(std::fabs(V.u) + fast_speed_x(V), ch); }
double max_signal_speed_y(const Primitive& V, double ch) { return std::fmax(std::fabs(V.v) + fast_speed_y(V), ch); }
}  // namespace phys

// ---- Riemann solvers (head/riemann.hpp) ----
Conserved physical_flux(const Conserved& U, Direction dir) {
    return dir == Direction::X ? phys::flux_x(U, phys::ch_glm) : phys::flux_y(U, phys::ch_glm);
}
Conserved hll_flux(const Conserved& UL, const Conserved& UR, Direction d, double ch) { return solve_dir(UL, UR, d, 0, ch); }
Conserved hllc_flux(const Conserved& UL, const Conserved& UR, Direction d, double ch) { return solve_dir(UL, UR, d, 1, ch); }
Conserved hlld_flux(const Conserved& UL, const Conserved& UR, Direction d, double ch) { return solve_dir(UL, UR, d, 2, ch); }
Conserved force_flux(const Conserved& UL, const Conserved& UR, Direction d, double ch) { return solve_dir(UL, UR, d, 3, ch); }
void apply_glm_flux(Conserved& F, const Conserved& UL, const Conserved& UR, Direction d, double ch) {
    if (d == Direction::X) mhd::exact::glm_overwrite<0>(&F.rho, ptr(UL), ptr(UR), ch);
    else mhd::exact::glm_overwrite<1>(&F.rho, ptr(UL), ptr(UR), ch);
}
Conserved riemann_flux(const Conserved& UL, const Conserved& UR, Direction d, RiemannSolver s, double ch) {
    return solve_dir(UL, UR, d, 10 + static_cast<int>(s), ch);
}
Conserved riemann_flux(const Conserved& UL, const Conserved& UR, Direction d, RiemannSolver s) {
    return riemann_flux(UL, UR, d, s, phys::ch_glm);
}

// ---- test cases (head/test_cases.hpp, src/test_cases.cpp:156-296) ----
CaseId parse_case_id(const std::string& name) {
    if (name == "kelvin_helmholtz") return CaseId::KelvinHelmholtz;
    if (name == "shock_bubble") return CaseId::ShockBubble;
    if (name == "brio_wu") return CaseId::BrioWu;
    if (name == "orszag_tang") return CaseId::OrszagTang;
    if (name == "orszag_tang_unit") return CaseId::OrszagTangUnit;
    if (name == "shock_bubble_mhd") return CaseId::ShockBubbleMHD;
    if (name == "brio_wu_cfl08") return CaseId::BrioWuCFL08;
    throw std::runtime_error("Unknown MHD test case: '" + name +
                             "'. Valid names: kelvin_helmholtz, shock_bubble, brio_wu, orszag_tang, "
                             "orszag_tang_unit, shock_bubble_mhd, brio_wu_cfl08.");
}

std::string case_id_to_string(CaseId id) {
    switch (id) {
        case CaseId::KelvinHelmholtz: return "kelvin_helmholtz";
        case CaseId::ShockBubble: return "shock_bubble";
        case CaseId::BrioWu: return "brio_wu";
        case CaseId::OrszagTang: return "orszag_tang";
        case CaseId::OrszagTangUnit: return "orszag_tang_unit";
        case CaseId::ShockBubbleMHD: return "shock_bubble_mhd";
        case CaseId::BrioWuCFL08: return "brio_wu_cfl08";
    }
    throw std::runtime_error("Unhandled CaseId in case_id_to_string.");
}

CaseConfig get_n_case_config(CaseId id, int n) {
    if (n < 1) throw std::runtime_error("get_n_case_config: n must be >= 1.");
    double v[14];
    if (mhd_case_config(static_cast<int>(id), n, v) != MHD_OK) throw std::runtime_error("get_n_case_config: bad case");
    CaseConfig c{static_cast<int>(v[0]), static_cast<int>(v[1]), static_cast<int>(v[2]), v[3], v[4], v[5], v[6],
                 v[7], v[8], v[9],
                 BoundaryConfig{static_cast<BoundaryType>(static_cast<int>(v[10])),
                                static_cast<BoundaryType>(static_cast<int>(v[11])),
                                static_cast<BoundaryType>(static_cast<int>(v[12])),
                                static_cast<BoundaryType>(static_cast<int>(v[13]))}};
    if (id == CaseId::ShockBubble) {
        // Haas & Sturtevant snapshot schedule (src/test_cases.cpp:215-231)
        const double vs = 1.22 * std::sqrt(1.4 * 1.01325e5 / 1.29);
        const double T0 = (0.035 - 0.025 - 0.005) / vs;
        const double tau = 0.025 / vs;
        const double t_paper[] = {0.6, 1.2, 1.8, 3.0, 4.6, 6.2, 7.8, 12.6, 19.0};
        for (double tp : t_paper) {
            c.snapshot_times.push_back(T0 + tp * tau);
            std::ostringstream oss;
            oss << "t" << std::setw(3) << std::setfill('0') << static_cast<int>(std::round(tp * 10.0));
            c.snapshot_tags.push_back(oss.str());
        }
    } else if (id == CaseId::OrszagTang) {  // src/test_cases.cpp:263-264
        c.snapshot_times = {M_PI, 2.0 * M_PI};
        c.snapshot_tags = {"tpi", "t2pi"};
    }
    return c;
}
CaseConfig get_n_case_config(const std::string& name, int n) { return get_n_case_config(parse_case_id(name), n); }
CaseConfig get_case_config(CaseId id) { return get_n_case_config(id, 1); }
CaseConfig get_case_config(const std::string& name) { return get_case_config(parse_case_id(name)); }

Conserved initial_state_at(CaseId id, double x, double y) {
    double v[9];
    if (mhd_initial_state(static_cast<int>(id), x, y, v) != MHD_OK) throw std::runtime_error("initial_state_at");
    return to_cons(v);
}
Conserved initial_state_at(const std::string& name, double x, double y) {
    return initial_state_at(parse_case_id(name), x, y);
}

// ---- init (head/init.hpp, src/init.cpp:18-65) ----
void initialise_grid(Grid2D& grid, CaseId id) {
    for (int j = 0; j < grid.total_ny(); ++j)
        for (int i = 0; i < grid.total_nx(); ++i) grid(i, j) = initial_state_at(id, grid.x_center(i), grid.y_center(j));
}
void initialise_grid(Grid2D& grid, const std::string& name) { initialise_grid(grid, parse_case_id(name)); }

Grid2D make_n_grid(CaseId id, int n) {
    const CaseConfig c = get_n_case_config(id, n);
    phys::gamma = c.gamma;
    Grid2D g(c.nx, c.ny, c.ng, c.x_min, c.x_max, c.y_min, c.y_max);
    initialise_grid(g, id);
    return g;
}
Grid2D make_n_grid(const std::string& name, int n) { return make_n_grid(parse_case_id(name), n); }
Grid2D make_initial_grid(CaseId id) { return make_n_grid(id, 1); }
Grid2D make_initial_grid(const std::string& name) { return make_initial_grid(parse_case_id(name)); }

// ---- GPU step (head/gpu/solver_gpu.cuh, head/gpu/boundary_gpu.cuh) ----
void set_gpu_physics_gamma(double gamma) { phys::gamma = gamma; }
void set_gpu_physics_ch(double ch) { phys::ch_glm = ch; }
void set_gpu_limiter(Limiter limiter) { g_limiter = limiter; }

void init_gpu_workspace(GpuWorkspace& ws, const Grid2DGPU& grid) {
    free_gpu_workspace(ws);
    mhd_throw_if(mhd_workspace_create(grid.c_grid(), &ws.impl), "init_gpu_workspace");
    ws.nx = grid.nx();
    ws.ny = grid.ny();
}

void free_gpu_workspace(GpuWorkspace& ws) {
    if (ws.impl) mhd_workspace_destroy(ws.impl);
    ws = GpuWorkspace{};
}

static void sync_physics(GpuWorkspace& ws) {
    mhd_throw_if(mhd_set_gamma(ws.impl, phys::gamma), "set_gpu_physics_gamma");
    mhd_throw_if(mhd_set_ch(ws.impl, phys::ch_glm), "set_gpu_physics_ch");
    mhd_throw_if(mhd_set_cr(ws.impl, phys::cr_glm), "cr_glm");
    mhd_throw_if(mhd_set_limiter(ws.impl, static_cast<int>(g_limiter)), "set_gpu_limiter");
}

double compute_dt_gpu(const Grid2DGPU& grid, GpuWorkspace& ws, double cfl) {
    if (!ws.impl || ws.nx != grid.nx() || ws.ny != grid.ny())
        throw std::runtime_error("compute_dt_gpu: workspace not initialised.");
    sync_physics(ws);
    double dt = 0.0;
    const int rc = mhd_compute_dt(ws.impl, grid.c_grid(), cfl, &dt);
    if (rc == MHD_ERR_NO_SPEED) return std::numeric_limits<double>::max();
    mhd_throw_if(rc, "compute_dt_gpu");
    mhd_throw_if(mhd_get_ch(ws.impl, &phys::ch_glm), "compute_dt_gpu");
    return dt;
}

void advance_second_order_gpu(const Grid2DGPU& Uold, Grid2DGPU& Utmp, Grid2DGPU& Unew, GpuWorkspace& ws, double dt,
                              RiemannSolver solver, const BoundaryConfig& bc) {
    if (!ws.impl || ws.nx != Uold.nx() || ws.ny != Uold.ny())
        throw std::runtime_error("advance_second_order_gpu: workspace not initialised.");
    sync_physics(ws);
    int b[4];
    bc_array(bc, b);
    mhd_throw_if(mhd_advance(ws.impl, Uold.c_grid(), Utmp.c_grid(), Unew.c_grid(), dt, static_cast<int>(solver), b),
                 "advance_second_order_gpu");
}

void apply_boundary_gpu(Grid2DGPU& grid, const BoundaryConfig& bc) {
    int b[4];
    bc_array(bc, b);
    mhd_throw_if(mhd_apply_boundary(nullptr, grid.c_grid(), b), "apply_boundary_gpu");
}

// Single-face Riemann flux through the C ABI (FP64, the reference's riemann_flux
// with explicit c_h, head/riemann.hpp:568-592).
extern "C" int mhd_riemann_flux(const double* UL, const double* UR, int dir, int solver, double ch, double gamma,
                                double* F) {
    if (!UL || !UR || !F || dir < 0 || dir > 1 || solver < MHD_HLL || solver > MHD_FORCE) return MHD_ERR_ARG;
    const Conserved f = solve_dir(to_cons(UL), to_cons(UR), dir == 0 ? Direction::X : Direction::Y, 10 + solver, ch,
                                  gamma);
    const double* p = &f.rho;
    for (int k = 0; k < 9; ++k) F[k] = p[k];
    return MHD_OK;
}
