// step_f32.cu -- the FP32-bulk GLM-MHD step: FP32 storage and arithmetic with
// the flagged FP64 pressure recovery (phys_fast.cuh), FP64 time step and CFL
// reduction, driven by the same fused sweeps as the FP64 step (sweep.cuh).
//
// Build this translation unit with --use_fast_math.
#include "launch.h"
#include "phys_fast.cuh"
#include "dispatch.cuh"
#include "batch.cuh"

namespace mhd {

template <int SOLVER, int LIMITER>
struct FastPolicy {
    using Real = float;
    static constexpr int NW = NV;
    static constexpr int NS = 2 * NV + 2;  // U, W, the known-physical flag and c_f (fast::Side)
    // The y-sweep's face states carry U and W only: its reconstruction leaves
    // the flag and c_f at 0 (its solver tests the states and computes the
    // speeds), and two more carried values made the batched y-sweep spill.
    static constexpr int NSY = 2 * NV;
    __device__ static void y_side_rest(fast::Side& S) { S.v[2 * NV] = 0.0f; S.v[2 * NV + 1] = 0.0f; }
    static constexpr int kYWarps = 4;   // y-sweep warps per CTA (side by side)
    // y-sweep window in shared memory (y_segment_carried), 4 CTAs per SM (128
    // registers, no spills).  Measured at 4096^2 (HLLD, van Leer): 0.674 ms,
    // against 0.702 ms for the register window at 3 CTAs (168 registers) and
    // 0.729 ms for the shared-memory window at 3 CTAs.
    static constexpr bool kYCarry = true;
    // The updated row from the slots rather than reloaded from global memory:
    // 40 KB of slots per CTA; measured 0.618 ms against 0.631 ms.
    static constexpr bool kYURing = true;
    static constexpr int kYBlocks = 4;  // y-sweep CTAs per SM the register budget is cut for
    static constexpr int kYTBlocks = 3; // the same for the TMA-staged y-sweep
    // Default y band (rows one warp marches; shorter bands at the end of the
    // launch, y_plan).  Measured at 4096^2 (HLLD, van Leer) with the guided
    // phases: 28 rows 0.566 ms, 24 rows 0.567, 32 rows 0.586 (before the CFL
    // fold skip), 20 rows 0.594 (the same); with one band height: 24 rows
    // 0.659 ms, 16 rows 0.664, 32 rows 0.667, 48 rows 0.698.
    static constexpr int kYBand = 28;
    // x-sweep (row march, segments of 1020 cells): 4 warps per CTA, 4 CTAs per
    // SM (128 registers, 56 KB of rings per CTA).  Measured at 4096^2 (HLLD, van
    // Leer): 0.549 ms; segments of 508 cells 0.545 ms, of 2044 cells 0.588 ms.
    // (The lane-per-cell tile it replaced: 0.574 ms.)
    static constexpr int kXWarps = 4;
    static constexpr int kXBlocks = 4;
    // Default x work per warp: segments of 1020 cells (the last quarter of a
    // row in 316-cell ones); 2044-cell segments measured 0.520 ms, 508-cell 0.551.
    static constexpr int kXRpw = 8;
    // Reloading the updated cell at the top of each x-march step needs 9 more
    // registers across the solve: at 128 registers that spills, and measured
    // 0.576 ms against 0.549 ms for the reload just before the update.
    static constexpr bool kXEarlyReload = false;
    // The updated cell instead comes back from a fourth ring (3 more 16-byte
    // slots per entry; 4 CTAs x 56 KB fill the SM's 228 KB with the per-CTA
    // reserve): measured at 4096^2 0.506 -> 0.473 ms (step 1.066 -> 1.033 ms),
    // bit-identical results.
    static constexpr bool kXURing = true;
    struct Prim { float v[NV]; };
    using Side = fast::Side;

    __device__ static void prim(const float* U, double g, float* W) { fast::c2p(U, (float)g, W); }
    // A face-side state made directly from a conserved cell: (U, c2p(U)), not
    // known physical, with its fast speed in direction DIR.
    template <int DIR>
    __device__ static void side(const float* U, double g, Side& S) {
#pragma unroll
        for (int k = 0; k < NV; ++k) S.v[k] = U[k];
        fast::c2p(U, (float)g, S.W());
        S.v[2 * NV] = 0.0f;  // not known physical: the solvers test it
        S.v[2 * NV + 1] = fast::fast_speed<DIR>(S.W(), (float)g);
    }

    template <int DIR>
    __device__ static void recon(const Prim& Wm, const Prim& Wc, const Prim& Wp, double dtd, double ch, double g,
                                 Side& L, Side& R) {
        fast::reconstruct<DIR, LIMITER>(Wm.v, Wc.v, Wp.v, (float)dtd, (float)ch, (float)g, L, R);
    }

    template <int DIR>
    __device__ static void face(const Side& Rl, const Side& Lr, double ch, double g, float* F) {
        fast::riemann<DIR, SOLVER>(Rl, Lr, (float)ch, (float)g, F);
    }

    __device__ static double speed(const float* U, double g, double ch) { return fast::cell_speed(U, (float)g, ch); }

    // The y-sweep's running CFL maximum: FP32, floored by c_h once at the end.
    using SpeedAcc = float;
    __device__ static SpeedAcc no_speed() { return -1.0f; }
    __device__ static void fold_speed(const float* U, double g, double ch, SpeedAcc& acc) {
        fast::fold_cell_speed_floored(U, (float)g, (float)ch, acc);
    }
    __device__ static double speed_of(SpeedAcc acc, double ch) { return acc < 0.0f ? 0.0 : fmax((double)acc, ch); }
};

cudaError_t launch_step_f32(const DevGrid& in, const DevGrid& tmp, const DevGrid& out, const StepParams& P,
                            cudaStream_t st, int yseg, int which, int xrpw, int ystage) {
    return dispatch_step<FastPolicy>(in, tmp, out, P, st, yseg, which, xrpw, ystage);
}

cudaError_t launch_batch_f32(const BatchInst* inst, const int* first, int n, int parity, int which, int solver,
                             int limiter, int xrpw, int yseg, int ctas, cudaStream_t st) {
    return dispatch_batch<FastPolicy>(inst, first, n, parity, which, solver, limiter, xrpw, yseg, ctas, st);
}

cudaError_t launch_faces_f32(const double* UL, const double* UR, long long n, int dir, int solver, double ch,
                             double gamma, double* F, cudaStream_t st) {
    return launch_faces_policy<FastPolicy>(UL, UR, n, dir, solver, ch, gamma, F, st);
}

cudaError_t launch_argmax_f32(const DevGrid& g, double gamma, double ch, double m, int* idx, cudaStream_t st) {
    return launch_argmax_policy<FastPolicy<HLL, MINMOD>>(g, gamma, ch, m, idx, st);
}

cudaError_t launch_max_speed_f32(const DevGrid& g, double gamma, double ch, unsigned long long* out,
                                 cudaStream_t st, int nsm) {
    return launch_max_policy<FastPolicy<HLL, MINMOD>>(g, gamma, ch, out, st, nsm);
}

}  // namespace mhd
