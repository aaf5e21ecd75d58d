// gpu/solver_gpu.cuh -- the reference's GPU step API (head/gpu/solver_gpu.cuh:9-53)
// on libmhd_b200.
//
// As in the reference, gamma and ch are process-global (phys::gamma,
// phys::ch_glm): set_gpu_physics_* write them, compute_dt_gpu sets ch_glm to
// the CFL maximum, and advance_second_order_gpu uses both.  Failures throw
// std::runtime_error (the reference throws for a workspace mismatch and exits
// the process on CUDA errors; this library never exits).
#pragma once

#include <cstddef>

#include "../riemann.hpp"
#include "../test_cases.hpp"
#include "grid_gpu.cuh"

struct GpuWorkspace {
    int nx = 0;
    int ny = 0;
    mhd_workspace* impl = nullptr;  // the library's workspace (device scratch, CUDA graph cache)
};

void set_gpu_physics_gamma(double gamma);   // src/gpu/solver_gpu.cu:536-539
void set_gpu_physics_ch(double ch);         // src/gpu/solver_gpu.cu:541-544
// Slope limiter for later steps (process-global, default minmod as the reference).
void set_gpu_limiter(Limiter limiter);

void init_gpu_workspace(GpuWorkspace& ws, const Grid2DGPU& grid);  // src/gpu/solver_gpu.cu:549-566
void free_gpu_workspace(GpuWorkspace& ws);                         // src/gpu/solver_gpu.cu:568-573

// CFL time step; sets phys::ch_glm to the maximum signal speed.  Returns
// std::numeric_limits<double>::max() when no cell has a positive speed
// (src/gpu/solver_gpu.cu:598-599).
double compute_dt_gpu(const Grid2DGPU& grid, GpuWorkspace& ws, double cfl);

// x-sweep, boundary conditions, y-sweep, boundary conditions, psi damping
// (src/gpu/solver_gpu.cu:617-690).
void advance_second_order_gpu(const Grid2DGPU& Uold, Grid2DGPU& Utmp, Grid2DGPU& Unew, GpuWorkspace& ws, double dt,
                              RiemannSolver solver, const BoundaryConfig& bc);
