// mhd_common.cuh -- layout, parameter blocks and small device helpers shared
// by every kernel of the B200 GLM-MHD step.
//
// HBM layout of one state ("grid"): ONE allocation holding 9 SoA planes
// (rho, rhou, rhov, rhow, Bx, By, Bz, E, psi -- the field order of the
// reference's Conserved, head/types.hpp:16-41).  Each plane is (ny+2ng) rows
// of `pitch` elements; cell (i, j) of plane f (i, j counting ghosts, as in
// head/gpu/grid_gpu.cuh:314-316) sits at data[f*plane + j*pitch + i].  The
// allocator pads `pitch` to a multiple of 256 bytes and `plane` to a multiple
// of 256 bytes, so every row start is 16-byte aligned (TMA- and
// vector-load-legal) and the 9 planes can be described by one 3-D tensor map.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

namespace mhd {

constexpr int NV = 9;
enum Field : int { RHO = 0, MX = 1, MY = 2, MZ = 3, BX = 4, BY = 5, BZ = 6, EN = 7, PSI = 8 };
// primitive slots reuse the indices: u = 1, v = 2, w = 3, p = 7
enum PrimSlot : int { PU = 1, PV = 2, PW = 3, PP = 7 };

// Same numbering as the reference enums so values pass through unchanged:
// RiemannSolver (head/riemann.hpp:23), BoundaryType (head/test_cases.hpp:11-16).
enum Solver : int { HLL = 0, HLLC = 1, HLLD = 2, FORCE = 3 };
enum Limiter : int { MINMOD = 0, VANLEER = 1 };
enum Bc : int { PERIODIC = 0, TRANSMISSIVE = 1, REFLECTING = 2, DIRICHLET = 3 };

constexpr int MAX_NG = 4;  // ghost layers supported by the kernels (>= 2 needed)

#ifdef __CUDACC__
#define MHD_HD_RULE __host__ __device__ __forceinline__
#else
#define MHD_HD_RULE inline
#endif

// Degenerate single-star state of HLLD (head/riemann.hpp:342-345, 354-357):
// d = rho (S - un)(S - SM) - Bn^2 vanishing.  The reference tests |d| < 1e-14,
// which FP64 resolves (d's rounding noise is ~1e-16 of its terms).  In FP32 the
// inputs S, un and SM carry noise of ~1e-7 of their size, so near the
// degenerate state d is that noise and the star state 1 / noise; FP32-bulk
// therefore takes the degenerate branch when |d| is within 1e-5 of the size of
// the terms that form it (NaN stays on the non-degenerate path, whose
// non-finite flux the dispatcher replaces by HLL, as in FP64).
constexpr float kStarDegenRel = 1.0e-5f;
MHD_HD_RULE bool star_degenerate(double d, double, double, double, double, double) { return fabs(d) < 1.0e-14; }
MHD_HD_RULE bool star_degenerate(float d, float rho, float un, float S, float SM, float Bn) {
    const float m = fabsf(S) + fabsf(un) + fabsf(SM);
    return fabsf(d) <= kStarDegenRel * (rho * m * m + Bn * Bn);
}
constexpr int kDefaultXRpw = 0;  // x-sweep work per warp: 0 = the policy's kXRpw
constexpr int kDefaultBatchXRpw = 8;  // batched x-sweep work per warp before tuning
constexpr int kDefaultYSeg = 64; // batched y-sweep rows per warp segment
constexpr int kDefaultYBand = 0;  // single-grid y-sweep rows per warp band: 0 = the policy's kYBand

struct DevGrid {
    void* data;          // plane 0, element (0, 0)
    long long pitch;     // elements per row
    long long plane;     // elements per plane
    int nx, ny, ng;
    int pad_;
    __host__ __device__ int tnx() const { return nx + 2 * ng; }
    __host__ __device__ int tny() const { return ny + 2 * ng; }
    __host__ __device__ long long idx(int i, int j) const { return (long long)j * pitch + i; }
};

// Device-resident time-step clock: lets a captured step loop pick dt and ch on
// the GPU.  Slot `parity` is read by step n (parity = n % 2); the y-sweep of
// step n accumulates the next maximum signal speed into slot parity ^ 1 as the
// bit pattern of a non-negative double (ordered like an unsigned integer).
struct DevClock {
    unsigned long long maxbits[2];
    double t[2];
    double last_dt;
    double last_ch;
    int steps;
    int status;          // 0 running, else one of ClockStatus
    unsigned int lowbeta_hits;   // FP32-bulk: FP64 pressure-recovery branch count
    unsigned int flux_fallbacks; // cells reverted by the non-finite update guard
};

enum ClockStatus : int {
    CLK_OK = 0,
    CLK_NO_SPEED = 1,     // max wave speed <= 0 (the reference throws, solver_cpu.cpp:304-306)
    CLK_BAD_DT = 2,       // dt non-finite or <= 0 (scripts/cpu/main_cpu.cpp:205-209)
    CLK_TINY_DT = 3,      // dt < 1e-8 t_end (scripts/cpu/main_cpu.cpp:210-216)
    CLK_DONE = 8,         // t reached t_end: later steps of a captured loop are no-ops
    CLK_TIMEOUT = 16,     // a bounded device wait gave up
};

// Everything a sweep needs besides the two grids.
struct StepParams {
    double gamma;
    double cr;        // c_r = c_p^2 / c_h, 0.18 in the reference (head/physics.hpp:39)
    double cfl;
    double dx, dy;
    double dmin;      // min(dx, dy)
    double t_end;
    // explicit mode (clock == nullptr): dt, ch and the psi damping factor
    double dt, ch, damp;
    DevClock* clock;  // device mode when non-null
    int parity;
    int solver, limiter;
    int bc[4];        // left, right, bottom, top
    int any_dirichlet;
    int accumulate;   // y-sweep: also fold the next max signal speed into maxbits
    unsigned long long* max_out;  // explicit mode accumulation target (may be null)
    int* fault;       // ClockStatus bits of a bounded device wait that gave up (may be null)
    unsigned long long tma_wait_ns;  // limit of each wait for a TMA-staged box (0: the default, 2 s)
    // y-sweep row window: interior rows [row0, row0 + nrows) (nrows 0: every row)
    int row0, nrows;
    int no_gather;    // skip the Dirichlet ghost gather (another launch of the step does it)
    int no_advance;   // device mode: do not advance the clock (another launch of the step does)
};

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// Positive doubles compare like their bit patterns.
__device__ __forceinline__ void atomic_max_pos(unsigned long long* addr, double v) {
    if (v > 0.0) atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

// dt / ch / damping for this step, computed identically by every thread.
// Returns false when the step must be skipped.  Mirrors the driver loop of
// scripts/cpu/main_cpu.cpp:196-216 and compute_dt (src/cpu/solver_cpu.cpp:304-311).
__device__ __forceinline__ bool step_scalars(const StepParams& P, double& dt, double& ch, double& damp) {
    if (P.clock == nullptr) {
        dt = P.dt; ch = P.ch; damp = P.damp;
        return true;
    }
    const DevClock* c = P.clock;
    if (*(volatile const int*)&c->status != CLK_OK) return false;
    const double t = *(volatile const double*)&c->t[P.parity];
    if (!(t < P.t_end)) return false;
    const double mx = __longlong_as_double(
        (long long)*(volatile const unsigned long long*)&c->maxbits[P.parity]);
    if (!(mx > 0.0)) return false;
    ch = mx;
    const double dt_raw = P.cfl * P.dmin / mx;
    const double rem = P.t_end - t;
    dt = (rem < dt_raw) ? rem : dt_raw;
    if (!isfinite(dt) || dt <= 0.0) return false;
    if (dt < 1.0e-8 * P.t_end) return false;
    damp = exp(-dt * ch / P.cr);
    return true;
}

// Status for a skipped device-mode step (called by one thread).
__device__ __forceinline__ void clock_flag_skip(const StepParams& P) {
    DevClock* c = P.clock;
    if (c == nullptr || c->status != CLK_OK) return;
    const double t = c->t[P.parity];
    if (!(t < P.t_end)) { c->status = CLK_DONE; return; }
    const double mx = __longlong_as_double((long long)c->maxbits[P.parity]);
    if (!(mx > 0.0)) { c->status = CLK_NO_SPEED; return; }
    const double dt_raw = P.cfl * P.dmin / mx;
    const double rem = P.t_end - t;
    const double dt = (rem < dt_raw) ? rem : dt_raw;
    if (!isfinite(dt) || dt <= 0.0) { c->status = CLK_BAD_DT; return; }
    if (dt < 1.0e-8 * P.t_end) { c->status = CLK_TINY_DT; return; }
}

// ---------------------------------------------------------------------------
// Boundary rules (head/cpu/boundary_cpu.hpp:12-149): where a ghost cell's value
// comes from.  Column/row indices are storage coordinates (ghosts included).
// ---------------------------------------------------------------------------

// Source column of left ghost column ib-1-q (bc = left type).
__host__ __device__ __forceinline__ int src_left(int bc, int q, int ib, int ie) {
    return bc == PERIODIC ? ie - 1 - q : (bc == TRANSMISSIVE ? ib : ib + q);
}
// Source column of right ghost column ie+q.
__host__ __device__ __forceinline__ int src_right(int bc, int q, int ib, int ie) {
    return bc == PERIODIC ? ib + q : (bc == TRANSMISSIVE ? ie - 1 : ie - 1 - q);
}

// Source column for ghost column x (x < ib or x >= ie) on side bc.
__host__ __device__ __forceinline__ int ghost_src_x(int x, int ib, int ie, const int* bc) {
    return (x < ib) ? src_left(bc[0], ib - 1 - x, ib, ie) : src_right(bc[1], x - ie, ib, ie);
}
__host__ __device__ __forceinline__ int ghost_src_y(int y, int jb, int je, const int* bc) {
    return (y < jb) ? src_left(bc[2], jb - 1 - y, jb, je) : src_right(bc[3], y - je, jb, je);
}

}  // namespace mhd
