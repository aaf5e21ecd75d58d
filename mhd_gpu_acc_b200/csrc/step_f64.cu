// step_f64.cu -- the FP64 ("plain") GLM-MHD step: the reference-faithful
// physics of phys_exact.cuh driven by the fused sweeps of sweep.cuh.
//
// Build this translation unit with --fmad=false: together with the reference
// operand order in phys_exact.cuh it makes the GPU step reproduce the
// reference's CPU/OpenMP FP64 step (src/cpu/solver_cpu.cpp) bit for bit.
#include "launch.h"
#include "phys_exact.cuh"
#include "dispatch.cuh"
#include "batch.cuh"

namespace mhd {

template <int SOLVER, int LIMITER>
struct ExactPolicy {
    using Real = double;
    static constexpr int NW = NV;  // primitive values per cell
    static constexpr int NS = NV;  // values per reconstructed side state (U*)
    static constexpr int NSY = NV;  // the same in the y-sweep's carried window
    template <class S>
    __device__ static void y_side_rest(S&) {}
    static constexpr int kYWarps = 4;   // y-sweep warps per CTA (side by side)
    // y-sweep window in shared memory (y_segment_carried), 2 CTAs per SM.
    // Measured at 4096^2 (HLLD, van Leer): 2.97 ms, against 3.11 ms for the
    // register window (255 registers, spills) and 3.06 ms for the shared-memory
    // window at 3 CTAs (168 registers, spills).
    static constexpr bool kYCarry = true;
    // FP64 slots for the updated row would take the CTA's static shared memory
    // past 48 KB: that row is reloaded from global memory.
    static constexpr bool kYURing = false;
    static constexpr int kYBlocks = 2;  // y-sweep CTAs per SM the register budget is cut for
    static constexpr int kYTBlocks = 2; // the same for the TMA-staged y-sweep
    // Default y band (shorter bands at the end of the launch, y_plan).
    // Measured at 4096^2 (HLLD, van Leer) with the guided phases and the fold
    // skip: 56 rows 2.62 ms, 48 rows 2.63, 64 rows 2.63, 80 rows 2.64, 40 rows
    // 2.65, 32 rows 2.68, 128 rows 2.89 (FP32 runs fastest at 28: its faster
    // sweep is the more sensitive to the DRAM locality of short bands); with
    // one band height: 32 rows 2.97 ms, 24 rows 2.98, 48 rows 2.98.
    static constexpr int kYBand = 56;
    // x-sweep (row march): 4 warps per CTA, 2 CTAs per SM (238 registers, no
    // spills), the updated cell reloaded at the top of each step.  Measured at
    // 4096^2 (HLLD, van Leer): 2.21 ms, against 2.27 ms reloading just before
    // the update and 2.39 / 2.64 ms (early / late reload) at 3 CTAs per SM
    // (168 registers, 128 / 360 bytes of spills).
    static constexpr int kXWarps = 4;
    static constexpr int kXBlocks = 2;
    static constexpr bool kXEarlyReload = true;
    // The updated cell from a fourth ring instead (the early reload is then
    // not made; 2 CTAs x 80 KB of rings): measured at 4096^2 2.174 -> 2.147 ms
    // (step 4.795 -> 4.766 ms), bit-identical results.
    static constexpr bool kXURing = true;
    // Default x work per warp: segments of 2044 cells (the last quarter of a
    // row in 668-cell ones).  Measured at 4096^2: 2.175 ms, against 2.210 ms
    // for 1020-cell segments.
    static constexpr int kXRpw = 16;
    struct Prim { double v[NV]; };
    struct Side { double v[NV]; };

    __device__ static void prim(const double* U, double g, double* W) { exact::c2p(U, g, W); }
    // A face-side state made directly from a conserved cell (the solvers' input).
    template <int DIR>
    __device__ static void side(const double* U, double, Side& S) {
#pragma unroll
        for (int k = 0; k < NV; ++k) S.v[k] = U[k];
    }

    template <int DIR>
    __device__ static void recon(const Prim& Wm, const Prim& Wc, const Prim& Wp, double dtd, double ch, double g,
                                 Side& L, Side& R) {
        exact::reconstruct<DIR, LIMITER>(Wm.v, Wc.v, Wp.v, dtd, ch, g, L.v, R.v);
    }

    template <int DIR>
    __device__ static void face(const Side& Rl, const Side& Lr, double ch, double g, double* F) {
        exact::riemann<DIR, SOLVER>(Rl.v, Lr.v, ch, g, F);
    }

    __device__ static double speed(const double* U, double g, double ch) { return exact::cell_speed(U, g, ch); }

    // The y-sweep's running CFL maximum (cell_speed per cell, as the reference;
    // the fast speeds of cells provably under the floor ch are skipped, which
    // leaves the maximum unchanged bit for bit).
    using SpeedAcc = double;
    __device__ static SpeedAcc no_speed() { return 0.0; }
    __device__ static void fold_speed(const double* U, double g, double ch, SpeedAcc& acc) {
        exact::fold_cell_speed_floored(U, g, ch, acc);
    }
    __device__ static double speed_of(SpeedAcc acc, double) { return acc; }
};

cudaError_t launch_step_f64(const DevGrid& in, const DevGrid& tmp, const DevGrid& out, const StepParams& P,
                            cudaStream_t st, int yseg, int which, int xrpw, int ystage) {
    return dispatch_step<ExactPolicy>(in, tmp, out, P, st, yseg, which, xrpw, ystage);
}

cudaError_t launch_batch_f64(const BatchInst* inst, const int* first, int n, int parity, int which, int solver,
                             int limiter, int xrpw, int yseg, int ctas, cudaStream_t st) {
    return dispatch_batch<ExactPolicy>(inst, first, n, parity, which, solver, limiter, xrpw, yseg, ctas, st);
}

cudaError_t launch_faces_f64(const double* UL, const double* UR, long long n, int dir, int solver, double ch,
                             double gamma, double* F, cudaStream_t st) {
    return launch_faces_policy<ExactPolicy>(UL, UR, n, dir, solver, ch, gamma, F, st);
}

cudaError_t launch_argmax_f64(const DevGrid& g, double gamma, double ch, double m, int* idx, cudaStream_t st) {
    return launch_argmax_policy<ExactPolicy<HLL, MINMOD>>(g, gamma, ch, m, idx, st);
}

cudaError_t launch_max_speed_f64(const DevGrid& g, double gamma, double ch, unsigned long long* out,
                                 cudaStream_t st, int nsm) {
    return launch_max_policy<ExactPolicy<HLL, MINMOD>>(g, gamma, ch, out, st, nsm);
}

}  // namespace mhd
