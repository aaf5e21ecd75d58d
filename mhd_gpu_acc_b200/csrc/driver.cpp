// driver.cpp -- init / step / output driver on libmhd_b200 (the role of the
// reference's scripts/gpu/main_gpu.cu and scripts/cpu/main_cpu.cpp).
//
//   mhd_run_case [case] [N] [--n N] [--solver hll|hllc|hlld|force]
//                [--limiter minmod|vanleer] [--precision fp64|fp32]
//                [--out DIR] [--no-out] [--device-loop] [--device-ic]
//                [--initial-bc] [--max-steps K]
//
// Defaults follow the reference drivers: case kelvin_helmholtz, HLLD, minmod,
// FP64, scale 1.  The time loop clamps dt to the next snapshot time and t_end
// and stops on a non-finite, non-positive or tiny dt (main_cpu.cpp:196-222).
// Fields are written as the reference writes them (main_cpu.cpp:36-91): one CSV
// per field, rows top first, %.8e, through a temporary file and a rename.
// --device-loop keeps dt and c_h on the GPU (mhd_run) between snapshots;
// --initial-bc applies the boundary conditions to the initial data first, as
// the reference GPU driver does (main_gpu.cu:195); without it the ghost cells
// hold initial-condition values, as in the CPU driver.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mhd_b200.h"
#include "../../include/mhd_b200/physics.hpp"
#include "../../include/mhd_b200/test_cases.hpp"

namespace {

struct Args {
    std::string case_name = "kelvin_helmholtz";
    int n = 1;
    int solver = MHD_HLLD;
    int limiter = MHD_LIMITER_MINMOD;
    int dtype = MHD_F64;
    std::string out = "output";
    bool write = false;
    bool device_loop = false;
    bool device_ic = false;
    bool initial_bc = false;
    int max_steps = 0;
};

void die(const std::string& msg) {
    std::cerr << "error: " << msg << "\n";
    std::exit(1);
}

void check(int rc, const char* what) {
    if (rc != MHD_OK) die(std::string(what) + ": " + mhd_last_error());
}

Args parse(int argc, char** argv) {
    Args a;
    for (int i = 1; i < argc; ++i) {
        const std::string s = argv[i];
        auto next = [&]() -> std::string {
            if (i + 1 >= argc) die("missing value after " + s);
            return argv[++i];
        };
        if (s == "--n") a.n = std::stoi(next());
        else if (s == "--case") a.case_name = next();
        else if (s == "--solver") {
            const std::string v = next();
            if (v == "hll") a.solver = MHD_HLL;
            else if (v == "hllc") a.solver = MHD_HLLC;
            else if (v == "hlld") a.solver = MHD_HLLD;
            else if (v == "force") a.solver = MHD_FORCE;
            else die("unknown solver " + v);
        } else if (s == "--limiter") {
            const std::string v = next();
            a.limiter = (v == "vanleer") ? MHD_LIMITER_VANLEER : MHD_LIMITER_MINMOD;
        } else if (s == "--precision") a.dtype = (next() == "fp32") ? MHD_F32 : MHD_F64;
        else if (s == "--out" || s == "--output") {
            if (s == "--out") a.out = next();
            a.write = true;
        } else if (s == "--no-out") a.write = false;
        else if (s == "--device-loop") a.device_loop = true;
        else if (s == "--device-ic") a.device_ic = true;
        else if (s == "--initial-bc") a.initial_bc = true;
        else if (s == "--max-steps") a.max_steps = std::stoi(next());
        else if (!s.empty() && s[0] != '-') {
            if (std::isdigit(static_cast<unsigned char>(s[0]))) a.n = std::stoi(s);
            else a.case_name = s;
        } else die("unknown argument " + s);
    }
    if (a.n < 1) die("--n must be >= 1");
    return a;
}

void write_field(const std::vector<double>& h, int nx, int ny, int ng, int f, const std::string& path,
                 double gamma) {
    const long long tnx = nx + 2LL * ng, np = tnx * (ny + 2LL * ng);
    const std::string tmp = path + ".tmp";
    FILE* fp = std::fopen(tmp.c_str(), "w");
    if (!fp) die("cannot open " + tmp);
    for (int j = ng + ny - 1; j >= ng; --j) {
        for (int i = ng; i < ng + nx; ++i) {
            const long long k = j * tnx + i;
            double v;
            const Conserved U(h[k], h[np + k], h[2 * np + k], h[3 * np + k], h[4 * np + k], h[5 * np + k],
                              h[6 * np + k], h[7 * np + k], h[8 * np + k]);
            switch (f) {
                case 1: v = U.rhou / U.rho; break;
                case 2: v = U.rhov / U.rho; break;
                case 3: v = U.rhow / U.rho; break;
                case 9: v = phys::cons_to_prim(U).p; break;
                default: v = (&U.rho)[f]; break;
            }
            std::fprintf(fp, i > ng ? ",%.8e" : "%.8e", v);
        }
        std::fputc('\n', fp);
    }
    if (std::fclose(fp) != 0) die("write error " + tmp);
    std::filesystem::rename(tmp, path);
    (void)gamma;
}

void write_all(const mhd_grid& g, const std::string& dir, const std::string& prefix) {
    std::filesystem::create_directories(dir);
    std::vector<double> h(static_cast<size_t>(9) * (g.nx + 2 * g.ng) * (g.ny + 2 * g.ng));
    check(mhd_grid_download(&g, h.data()), "download");
    static const char* names[10] = {"rho", "u", "v", "w", "Bx", "By", "Bz", "E", "psi", "p"};
    for (int f = 0; f < 10; ++f)
        write_field(h, g.nx, g.ny, g.ng, f, dir + "/" + prefix + "_" + names[f] + ".csv", phys::gamma);
    std::cout << "  Wrote fields to " << dir << "/" << prefix << "_*.csv\n";
}

}  // namespace

int main(int argc, char** argv) {
    const Args a = parse(argc, argv);
    CaseConfig cfg;
    try {
        cfg = get_n_case_config(a.case_name, a.n);
    } catch (const std::exception& e) {
        die(e.what());
    }
    phys::gamma = cfg.gamma;
    const int cid = static_cast<int>(parse_case_id(a.case_name));
    const int bc[4] = {static_cast<int>(cfg.bc.left), static_cast<int>(cfg.bc.right), static_cast<int>(cfg.bc.bottom),
                       static_cast<int>(cfg.bc.top)};
    std::cout << "=== MHD GLM step on libmhd_b200 (" << mhd_version() << ") ===\n"
              << "  Case      : " << a.case_name << "  (" << cfg.nx << " x " << cfg.ny << ")\n"
              << "  Precision : " << (a.dtype == MHD_F64 ? "fp64" : "fp32-bulk") << "\n";

    mhd_grid U{}, T{}, N{};
    check(mhd_grid_alloc(&U, cfg.nx, cfg.ny, cfg.ng, a.dtype, cfg.x_min, cfg.x_max, cfg.y_min, cfg.y_max), "alloc");
    check(mhd_grid_alloc(&T, cfg.nx, cfg.ny, cfg.ng, a.dtype, cfg.x_min, cfg.x_max, cfg.y_min, cfg.y_max), "alloc");
    check(mhd_grid_alloc(&N, cfg.nx, cfg.ny, cfg.ng, a.dtype, cfg.x_min, cfg.x_max, cfg.y_min, cfg.y_max), "alloc");
    mhd_workspace* ws = nullptr;
    check(mhd_workspace_create(&U, &ws), "workspace");
    if (a.device_ic) {
        check(mhd_initialise_device(ws, &U, cid), "initialise_device");
    } else {
        std::vector<double> h(static_cast<size_t>(9) * (cfg.nx + 2 * cfg.ng) * (cfg.ny + 2 * cfg.ng));
        check(mhd_initialise(cid, cfg.nx, cfg.ny, cfg.ng, cfg.x_min, cfg.x_max, cfg.y_min, cfg.y_max, h.data()),
              "initialise");
        check(mhd_grid_upload(&U, h.data()), "upload");
    }
    check(mhd_set_gamma(ws, cfg.gamma), "gamma");
    check(mhd_set_ch(ws, 0.0), "ch");
    check(mhd_set_limiter(ws, a.limiter), "limiter");
    if (a.initial_bc) check(mhd_apply_boundary(ws, &U, bc), "initial boundary");
    check(mhd_synchronize(ws), "sync");
    if (a.write) write_all(U, a.out, a.case_name + "_gpu_t0");

    const bool snaps = !cfg.snapshot_times.empty();
    size_t snap = 0;
    double t = 0.0;
    int step = 0;
    const auto t0 = std::chrono::steady_clock::now();
    while (t < cfg.t_end && (a.max_steps <= 0 || step < a.max_steps)) {
        double t_next = cfg.t_end;
        if (snaps && snap < cfg.snapshot_times.size()) t_next = std::min(t_next, cfg.snapshot_times[snap]);
        if (a.device_loop) {
            mhd_run_info info{};
            const int left = a.max_steps > 0 ? a.max_steps - step : 0;
            const int rc = mhd_run(ws, &U, &T, cfg.cfl, t_next - t, left, a.solver, bc, &info);
            step += info.steps;
            t += info.t;
            if (rc != MHD_OK) {
                std::cerr << "[WARN] step loop stopped: " << mhd_last_error() << "\n";
                break;
            }
        } else {
            double dt_raw = 0.0;
            if (mhd_compute_dt(ws, &U, cfg.cfl, &dt_raw) != MHD_OK) {
                std::cerr << "[ERROR] " << mhd_last_error() << " at step " << step << "\n";
                break;
            }
            const double dt = std::min(dt_raw, t_next - t);
            if (!std::isfinite(dt) || dt <= 0.0) {
                std::cerr << "[ERROR] dt=" << dt << " at step=" << step << ". Aborting.\n";
                break;
            }
            if (dt < 1.0e-8 * cfg.t_end) {
                std::cerr << "[WARN]  dt=" << dt << " below 1e-8 t_end at step=" << step << ", stopping.\n";
                break;
            }
            check(mhd_advance(ws, &U, &T, &N, dt, a.solver, bc), "advance");
            check(mhd_grid_swap(&U, &N), "swap");
            t += dt;
            step += 1;
        }
        if (a.write && snaps) {
            while (snap < cfg.snapshot_times.size() && t >= cfg.snapshot_times[snap] - 1e-12) {
                check(mhd_synchronize(ws), "sync");
                write_all(U, a.out, a.case_name + "_gpu_" + cfg.snapshot_tags[snap]);
                ++snap;
            }
        }
    }
    check(mhd_synchronize(ws), "sync");
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cout << "[GPU] Total steps= " << step << "\n";
    std::cout << "[TIMING] n=" << a.n << " nx=" << cfg.nx << " ny=" << cfg.ny << " steps=" << step << std::fixed
              << std::setprecision(4) << " elapsed_s=" << elapsed << std::setprecision(2)
              << " steps_per_s=" << step / elapsed << std::setprecision(1)
              << " Mcell_updates_s=" << static_cast<double>(step) * cfg.nx * cfg.ny / elapsed / 1.0e6 << "\n";
    if (a.write && !snaps)
        write_all(U, a.out, a.case_name + "_gpu_t" + std::to_string(static_cast<int>(std::round(cfg.t_end * 100))));
    mhd_workspace_destroy(ws);
    mhd_grid_free(&U);
    mhd_grid_free(&T);
    mhd_grid_free(&N);
    return 0;
}
