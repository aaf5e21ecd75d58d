// gpu_step_timer.cu -- times the split step through the reference's C++ GPU API
// (Grid2DGPU, init_gpu_workspace, set_gpu_physics_*, apply_boundary_gpu,
// compute_dt_gpu, advance_second_order_gpu; the loop of the reference driver
// scripts/gpu/main_gpu.cu:197-236 without output) on the reference's own
// Orszag-Tang case scaled by n (192n x 192n cells on [0, 2 pi]^2, HLLD).
//
// Measurement infrastructure, built twice by oracle/Makefile from this one
// source: against the reference's headers and src/gpu sources
// (_ref/ref_gpu_timer: the reference's GPU step) and against this
// repository's drop-in headers and libmhd_b200 (_ref/dropin_gpu_timer: the
// same host loop on the B200 kernels).  Prints one JSON line.
//
// usage: gpu_step_timer N_SCALE WARMUP STEPS
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "gpu/boundary_gpu.cuh"
#include "gpu/grid_gpu.cuh"
#include "gpu/solver_gpu.cuh"
#include "init.hpp"
#include "test_cases.hpp"

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s N_SCALE WARMUP STEPS\n", argv[0]);
        return 2;
    }
    const int n = std::atoi(argv[1]), warmup = std::atoi(argv[2]), steps = std::atoi(argv[3]);
    const std::string name = "orszag_tang";
    CaseConfig cfg = get_n_case_config(name, n);
    Grid2D cpu = make_n_grid(name, n);
    phys::gamma = cfg.gamma;

    Grid2DGPU Uold(cfg.nx, cfg.ny, cfg.ng, cfg.x_min, cfg.x_max, cfg.y_min, cfg.y_max);
    Grid2DGPU Utmp(cfg.nx, cfg.ny, cfg.ng, cfg.x_min, cfg.x_max, cfg.y_min, cfg.y_max);
    Grid2DGPU Unew(cfg.nx, cfg.ny, cfg.ng, cfg.x_min, cfg.x_max, cfg.y_min, cfg.y_max);
    Uold.upload_from_aos(cpu.data());
    GpuWorkspace ws;
    init_gpu_workspace(ws, Uold);
    set_gpu_physics_gamma(cfg.gamma);
    set_gpu_physics_ch(0.0);
    apply_boundary_gpu(Uold, cfg.bc);

    double t = 0.0;
    auto step = [&]() {
        const double dt = compute_dt_gpu(Uold, ws, cfg.cfl);
        advance_second_order_gpu(Uold, Utmp, Unew, ws, dt, RiemannSolver::HLLD, cfg.bc);
        Uold.swap(Unew);
        t += dt;
    };
    for (int k = 0; k < warmup; ++k) step();
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    const auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < steps; ++k) step();
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const double cells = (double)cfg.nx * cfg.ny;
    std::printf("{\"nx\": %d, \"ny\": %d, \"warmup\": %d, \"steps\": %d, \"seconds\": %.6f, "
                "\"ms_per_step\": %.6f, \"cell_updates_per_s\": %.6e, \"t\": %.9e}\n",
                cfg.nx, cfg.ny, warmup, steps, s, 1e3 * s / steps, cells * steps / s, t);
    free_gpu_workspace(ws);
    return 0;
}
