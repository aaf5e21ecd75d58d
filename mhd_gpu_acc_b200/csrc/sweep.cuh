// sweep.cuh -- the fused directional sweep kernels of one split step.
//
// One launch per sweep replaces the reference's x/y kernels, its two boundary
// kernels per sweep, the psi-damping kernel and the CFL block-max kernel + CUB
// reduction (src/gpu/solver_gpu.cu:188-251, 265-528; src/gpu/boundary_gpu.cu).
//
// x-sweep  (Uin -> Uout): one warp per interior row segment.  Lane l holds the
//          cell at storage column x0 + l (x0 = ng - 2 + TX*blockIdx.x); the
//          stencil neighbours are exchanged with warp shuffles, so primitive,
//          reconstruction, face flux and update each run once per cell, in
//          registers, with no shared-memory staging.
// y-sweep  (Uin -> Uout): one thread per column; each warp marches down a
//          segment of rows with a sliding window (W(r-2), W(r-1), the last
//          right-biased state and the last face flux), held in registers or,
//          when the policy asks (kYCarry), in per-lane shared-memory slots.
//          Row loads are fully coalesced.
//
// Both sweeps write the complete ghost ring of their output with the
// reference's copy_ghost_cells + apply_boundary semantics
// (head/cpu/boundary_cpu.hpp:12-149): the thread that produces an interior
// source cell scatters it to every ghost cell that copies it; ghost cells
// that come from the input grid (Dirichlet sides) are gathered by a
// grid-stride pass.  The y-sweep additionally applies psi damping to interior
// cells only, after the ghost copy (src/cpu/solver_cpu.cpp:434-439), and folds
// the next CFL maximum (src/cpu/solver_cpu.cpp:283-303) into one atomic per
// warp.
#pragma once

#include "mhd_common.cuh"

namespace mhd {

constexpr unsigned FULL = 0xffffffffu;
constexpr int XS_TX = 28;       // interior cells per warp in the x-sweep (32 lanes - 4 halo)
constexpr int XS_ROWS = 8;      // warps (rows) per x-sweep CTA
// rows each x-sweep warp processes (with one-row prefetch) and the rows a
// y-sweep warp takes are launch parameters (kDefaultXRpw, kDefaultYBand and, for
// batches, kDefaultYSeg in mhd_common.cuh; the batch autotuner may pick others).
constexpr int YS_WARPS = 4;     // warps (row segments) per y-sweep CTA

template <int N, typename T>
__device__ __forceinline__ void shfl_up_n(const T* in, T* out, int d) {
#pragma unroll
    for (int k = 0; k < N; ++k) out[k] = __shfl_up_sync(FULL, in[k], d);
}
template <int N, typename T>
__device__ __forceinline__ void shfl_down_n(const T* in, T* out, int d) {
#pragma unroll
    for (int k = 0; k < N; ++k) out[k] = __shfl_down_sync(FULL, in[k], d);
}

template <typename R>
__device__ __forceinline__ void load_cell(const DevGrid& g, int x, int y, R* U) {
    const R* b = static_cast<const R*>(g.data) + g.idx(x, y);
#pragma unroll
    for (int f = 0; f < NV; ++f) U[f] = __ldg(b + f * g.plane);
}

template <typename R>
__device__ __forceinline__ void store_cell(const DevGrid& g, int x, int y, const R* U) {
    R* b = static_cast<R*>(g.data) + g.idx(x, y);
#pragma unroll
    for (int f = 0; f < NV; ++f) b[f * g.plane] = U[f];
}

// Writes interior cell (x, y)'s value to every ghost cell of `out` whose
// boundary rule copies it (non-Dirichlet sides), corners by composition.
// Inlined (on the rare near-edge path) so that neither the cell nor the kernel
// parameter block holding `bc` has to be spilled to the stack for a call.
template <typename R>
__device__ __forceinline__ void scatter_ghosts(const DevGrid& out, int x, int y, const R* v, const int* bc) {
    const int ng = out.ng, ib = ng, ie = ng + out.nx, jb = ng, je = ng + out.ny;
    for (int a = 0; a <= 2 * ng; ++a) {
        int gx = x, fx = 0;
        if (a > 0) {
            const int q = (a - 1) >> 1;
            if (((a - 1) & 1) == 0) {
                if (bc[0] == DIRICHLET || src_left(bc[0], q, ib, ie) != x) continue;
                gx = ib - 1 - q; fx = (bc[0] == REFLECTING);
            } else {
                if (bc[1] == DIRICHLET || src_right(bc[1], q, ib, ie) != x) continue;
                gx = ie + q; fx = (bc[1] == REFLECTING);
            }
        }
        for (int b = 0; b <= 2 * ng; ++b) {
            if (a == 0 && b == 0) continue;
            int gy = y, fy = 0;
            if (b > 0) {
                const int q = (b - 1) >> 1;
                if (((b - 1) & 1) == 0) {
                    if (bc[2] == DIRICHLET || src_left(bc[2], q, jb, je) != y) continue;
                    gy = jb - 1 - q; fy = (bc[2] == REFLECTING);
                } else {
                    if (bc[3] == DIRICHLET || src_right(bc[3], q, jb, je) != y) continue;
                    gy = je + q; fy = (bc[3] == REFLECTING);
                }
            }
            R w[NV];
#pragma unroll
            for (int k = 0; k < NV; ++k) w[k] = v[k];
            if (fx) { w[MX] = -w[MX]; w[BX] = -w[BX]; }
            if (fy) { w[MY] = -w[MY]; w[BY] = -w[BY]; }
            store_cell(out, gx, gy, w);
        }
    }
}

__device__ __forceinline__ bool near_edge(const DevGrid& g, int x, int y) {
    const int ng = g.ng;
    return x < 2 * ng || x >= g.nx || y < 2 * ng || y >= g.ny;  // within ng of an interior edge
}

// Ghost cells of the sweep output that come from the INPUT grid: Dirichlet
// sides (copy_ghost_cells) and corners whose rule passes through a Dirichlet
// side.  Grid-stride over all ghost cells.
template <typename R>
__device__ __forceinline__ void gather_dirichlet_ghosts(const DevGrid& in, const DevGrid& out, const int* bc) {
    const int ng = in.ng, ib = ng, ie = ng + in.nx, jb = ng, je = ng + in.ny;
    const int tx = in.tnx(), ty = in.tny();
    const long long nthreads = (long long)gridDim.x * gridDim.y * blockDim.x * blockDim.y;
    const long long tid = ((long long)blockIdx.y * gridDim.x + blockIdx.x) * (blockDim.x * blockDim.y) +
                          threadIdx.y * blockDim.x + threadIdx.x;
    const long long total = (long long)tx * ty;
    for (long long k = tid; k < total; k += nthreads) {
        const int y = (int)(k / tx), x = (int)(k - (long long)y * tx);
        const bool xg = (x < ib || x >= ie), yg = (y < jb || y >= je);
        if (!xg && !yg) continue;
        const int bcx = (x < ib) ? bc[0] : bc[1], bcy = (y < jb) ? bc[2] : bc[3];
        int srcx = x, srcy = y, fx = 0, fy = 0;
        if (xg && !yg) {
            if (bcx != DIRICHLET) continue;
        } else if (yg && !xg) {
            if (bcy != DIRICHLET) continue;
        } else {
            if (bcy != DIRICHLET) {
                if (bcx != DIRICHLET) continue;  // produced by the scatter
                srcy = ghost_src_y(y, jb, je, bc);
                fy = (bcy == REFLECTING);
            } else if (bcx != DIRICHLET) {
                srcx = ghost_src_x(x, ib, ie, bc);
                fx = (bcx == REFLECTING);
            }
        }
        R w[NV];
        load_cell(in, srcx, srcy, w);
        if (fx) { w[MX] = -w[MX]; w[BX] = -w[BX]; }
        if (fy) { w[MY] = -w[MY]; w[BY] = -w[BY]; }
        store_cell(out, x, y, w);
    }
}

// Conservative update with the CPU path's revert rule (non-finite rho or E
// keeps the old cell, src/cpu/solver_cpu.cpp:386-392).
template <typename R>
__device__ __forceinline__ bool update_cell(const R* U, const R* Fp, const R* Fm, R dtd, R* Un) {
#pragma unroll
    for (int k = 0; k < NV; ++k) Un[k] = U[k] - dtd * (Fp[k] - Fm[k]);
    if (!isfinite(Un[RHO]) || !isfinite(Un[EN])) {
#pragma unroll
        for (int k = 0; k < NV; ++k) Un[k] = U[k];
        return true;
    }
    return false;
}

// ---------------------------------------------------------------------------
// x-sweep
// ---------------------------------------------------------------------------
// One CTA of WARPS warps handles a 28-column tile over WARPS * rpw rows:
// warp w takes rows  row_block*WARPS*rpw + w + k*WARPS  (k < rpw) and loads
// the next row's cells before computing the current one, so the load latency
// overlaps the arithmetic.
template <class PH, int WARPS = XS_ROWS>
__device__ __forceinline__ void x_tile(const DevGrid& in, const DevGrid& out, const StepParams& P, double dt,
                                       double ch, int tile_x, int row_block, int rpw) {
    using R = typename PH::Real;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int row0 = row_block * WARPS * rpw;
    const int row_end = min(in.ny, row0 + WARPS * rpw);
    int row = row0 + warp;
    if (row >= row_end) return;  // whole warp: no block-level synchronisation follows
    const int ng = in.ng, ib = ng, ie = ng + in.nx;
    const int x = ib - 2 + tile_x * XS_TX + lane;
    const bool xin = x < in.tnx();
    const double g = P.gamma;
    const double dtd = dt / P.dx;
    const bool do_recon = lane >= 1 && lane <= 30 && x >= ib - 1 && x <= ie;
    const bool do_face = lane >= 1 && lane <= 29 && x >= ib - 1 && x <= ie - 1;
    const bool do_update = lane >= 2 && lane <= 29 && x >= ib && x < ie;

    R Unext[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) Unext[k] = R(0);
    Unext[RHO] = R(1);
    if (xin) load_cell(in, x, ng + row, Unext);

#pragma unroll 1
    for (; row < row_end; row += WARPS) {
        const int y = ng + row;
        R U[NV], W[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) U[k] = Unext[k];
        if (xin && row + WARPS < row_end) load_cell(in, x, y + WARPS, Unext);  // prefetch
        PH::prim(U, g, W);

        typename PH::Side L, Rt;
#pragma unroll
        for (int k = 0; k < PH::NS; ++k) { L.v[k] = R(0); Rt.v[k] = R(0); }
        {
            typename PH::Prim Wm, Wp, Wc;
            shfl_up_n<PH::NW>(W, Wm.v, 1);
            shfl_down_n<PH::NW>(W, Wp.v, 1);
#pragma unroll
            for (int k = 0; k < PH::NW; ++k) Wc.v[k] = W[k];
            if (do_recon) PH::template recon<0>(Wm, Wc, Wp, dtd, ch, g, L, Rt);
        }
        typename PH::Side Ln;
        shfl_down_n<PH::NS>(L.v, Ln.v, 1);
        R F[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) F[k] = R(0);
        if (do_face) PH::template face<0>(Rt, Ln, ch, g, F);
        R Fm[NV];
        shfl_up_n<NV>(F, Fm, 1);
        if (do_update) {
            R Un[NV];
            const bool reverted = update_cell<R>(U, F, Fm, R(dtd), Un);
            if (reverted && P.clock) atomicAdd(&P.clock->flux_fallbacks, 1u);
            store_cell(out, x, y, Un);
            if (near_edge(out, x, y)) scatter_ghosts<R>(out, x, y, Un, P.bc);
        }
    }
}

// CTA shape and register budget per policy: PH::kXWarps warps per CTA,
// PH::kXBlocks CTAs per SM.
template <class PH>
__global__ void __launch_bounds__(32 * PH::kXWarps, PH::kXBlocks)
    sweep_x_kernel(DevGrid in, DevGrid out, StepParams P, int rpw) {
    using R = typename PH::Real;
    double dt, ch, damp;
    const bool first = (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0);
    if (!step_scalars(P, dt, ch, damp)) {
        if (first) clock_flag_skip(P);
        return;
    }
    if (first && P.clock) P.clock->maxbits[P.parity ^ 1] = 0ull;
    if (P.any_dirichlet) gather_dirichlet_ghosts<R>(in, out, P.bc);
    x_tile<PH, PH::kXWarps>(in, out, P, dt, ch, blockIdx.x, blockIdx.y, rpw);
}

// ---------------------------------------------------------------------------
// y-sweep
// ---------------------------------------------------------------------------
// One warp marches down interior rows [j0, j0 + count) (ghost offset included)
// of a 32-column strip (lane = column x = strip*32 + lane), folding the CFL
// speed of every updated cell into vmax (when P.accumulate) and counting
// reverted cells.  Called by whole warps; y_fold publishes the two results.
template <class PH>
__device__ __forceinline__ void y_segment(const DevGrid& in, const DevGrid& out, const StepParams& P, double dt,
                                          double ch, double damp, int strip, int j0, int count, double& vmax,
                                          unsigned& reverts) {
    using R = typename PH::Real;
    const int lane = threadIdx.x & 31;
    const int ng = in.ng, ib = ng, ie = ng + in.nx;
    const int x = strip * 32 + lane;
    const int j1 = j0 + count;
    const bool active = (x >= ib && x < ie && count > 0);
    const double g = P.gamma;
    const double dtd = dt / P.dy;
    typename PH::SpeedAcc acc = PH::no_speed();

    if (active) {
        typename PH::Prim Wm, Wc, Wp;
        typename PH::Side Rprev, L, Rt;
        R Fprev[NV], F[NV], U[NV];
        R Unext[NV];
        load_cell(in, x, j0 - 2, U);
        load_cell(in, x, j0 - 1, Unext);
        PH::prim(U, g, Wm.v);
        PH::prim(Unext, g, Wc.v);
        load_cell(in, x, j0, Unext);
#pragma unroll 1
        for (int r = j0; r <= j1 + 1; ++r) {
#pragma unroll
            for (int k = 0; k < NV; ++k) U[k] = Unext[k];
            if (r <= j1) load_cell(in, x, r + 1, Unext);  // prefetch the next row
            R Uc[NV];
            if (r >= j0 + 2) load_cell(in, x, r - 2, Uc);  // the row updated below
            PH::prim(U, g, Wp.v);
            PH::template recon<1>(Wm, Wc, Wp, dtd, ch, g, L, Rt);  // cell r-1
            if (r >= j0 + 1) {
                PH::template face<1>(Rprev, L, ch, g, F);  // face (r-2 | r-1)
                if (r >= j0 + 2) {
                    const int yc = r - 2;
                    R Un[NV];
                    reverts += update_cell<R>(Uc, F, Fprev, R(dtd), Un) ? 1u : 0u;
                    if (near_edge(out, x, yc)) scatter_ghosts<R>(out, x, yc, Un, P.bc);
                    Un[PSI] = Un[PSI] * R(damp);
                    store_cell(out, x, yc, Un);
                    if (P.accumulate) PH::fold_speed(Un, g, ch, acc);
                }
#pragma unroll
                for (int k = 0; k < NV; ++k) Fprev[k] = F[k];
            }
            Rprev = Rt;
            Wm = Wc;
            Wc = Wp;
        }
    }
    if (P.accumulate) {
        const double v = PH::speed_of(acc, ch);
        vmax = (vmax < v) ? v : vmax;
    }
}

// The same march with its loop-carried values -- the two previous primitive
// rows (a ring indexed by row parity), the last right-biased state and the
// last face flux -- kept in per-lane shared-memory slots instead of registers.
// Slot s of a lane is carry[s * 32 + lane]: a warp's access is one
// conflict-free row and no other thread reads it, so no synchronisation is
// needed.  Moving these 2*NW + NS + NV values out of the register file lets
// the sweep run at the x-sweep's register budget (more resident warps) for a
// few shared-memory loads and stores per cell; values and operation order are
// those of y_segment, so results are identical.
template <class PH>
struct YCarry {
    static constexpr int kSlots = 2 * PH::NW + PH::NS + NV;
};

template <class PH>
__device__ __forceinline__ void y_segment_carried(const DevGrid& in, const DevGrid& out, const StepParams& P,
                                                  double dt, double ch, double damp, int strip, int j0, int count,
                                                  double& vmax, unsigned& reverts, typename PH::Real* carry) {
    using R = typename PH::Real;
    const int lane = threadIdx.x & 31;
    const int ng = in.ng, ib = ng, ie = ng + in.nx;
    const int x = strip * 32 + lane;
    const int j1 = j0 + count;
    const bool active = (x >= ib && x < ie && count > 0);
    const double g = P.gamma;
    const double dtd = dt / P.dy;
    typename PH::SpeedAcc acc = PH::no_speed();
    R* const wring = carry + lane;                    // W of row k: slots (k & 1) * NW + [0, NW)
    R* const rslot = carry + 2 * PH::NW * 32 + lane;  // last right-biased state: NS slots
    R* const fslot = rslot + PH::NS * 32;             // last face flux: NV slots

    if (active) {
        typename PH::Prim Wm, Wc, Wp;
        typename PH::Side Rprev, L, Rt;
        R F[NV], U[NV];
        R Unext[NV];
        load_cell(in, x, j0 - 2, U);
        load_cell(in, x, j0 - 1, Unext);
        PH::prim(U, g, Wp.v);
#pragma unroll
        for (int k = 0; k < PH::NW; ++k) wring[(((j0 - 2) & 1) * PH::NW + k) * 32] = Wp.v[k];
        PH::prim(Unext, g, Wp.v);
#pragma unroll
        for (int k = 0; k < PH::NW; ++k) wring[(((j0 - 1) & 1) * PH::NW + k) * 32] = Wp.v[k];
        load_cell(in, x, j0, Unext);
#pragma unroll 1
        for (int r = j0; r <= j1 + 1; ++r) {
#pragma unroll
            for (int k = 0; k < NV; ++k) U[k] = Unext[k];
            if (r <= j1) load_cell(in, x, r + 1, Unext);  // prefetch the next row
            R Uc[NV];
            if (r >= j0 + 2) load_cell(in, x, r - 2, Uc);  // the row updated below
            PH::prim(U, g, Wp.v);
            R* const wm = wring + (r & 1) * PH::NW * 32;        // row r - 2, overwritten by row r
            R* const wc = wring + ((r - 1) & 1) * PH::NW * 32;  // row r - 1
#pragma unroll
            for (int k = 0; k < PH::NW; ++k) { Wm.v[k] = wm[k * 32]; Wc.v[k] = wc[k * 32]; }
#pragma unroll
            for (int k = 0; k < PH::NW; ++k) wm[k * 32] = Wp.v[k];
            PH::template recon<1>(Wm, Wc, Wp, dtd, ch, g, L, Rt);  // cell r-1
            if (r >= j0 + 1) {
#pragma unroll
                for (int k = 0; k < PH::NS; ++k) Rprev.v[k] = rslot[k * 32];
                PH::template face<1>(Rprev, L, ch, g, F);  // face (r-2 | r-1)
                if (r >= j0 + 2) {
                    const int yc = r - 2;
                    R Fprev[NV], Un[NV];
#pragma unroll
                    for (int k = 0; k < NV; ++k) Fprev[k] = fslot[k * 32];
                    reverts += update_cell<R>(Uc, F, Fprev, R(dtd), Un) ? 1u : 0u;
                    if (near_edge(out, x, yc)) scatter_ghosts<R>(out, x, yc, Un, P.bc);
                    Un[PSI] = Un[PSI] * R(damp);
                    store_cell(out, x, yc, Un);
                    if (P.accumulate) PH::fold_speed(Un, g, ch, acc);
                }
#pragma unroll
                for (int k = 0; k < NV; ++k) fslot[k * 32] = F[k];
            }
#pragma unroll
            for (int k = 0; k < PH::NS; ++k) rslot[k * 32] = Rt.v[k];
        }
    }
    if (P.accumulate) {
        const double v = PH::speed_of(acc, ch);
        vmax = (vmax < v) ? v : vmax;
    }
}

// y_segment or y_segment_carried, as the policy asks (kYCarry).
template <class PH>
__device__ __forceinline__ void y_march(const DevGrid& in, const DevGrid& out, const StepParams& P, double dt,
                                        double ch, double damp, int strip, int j0, int count, double& vmax,
                                        unsigned& reverts, typename PH::Real* carry) {
    if constexpr (PH::kYCarry)
        y_segment_carried<PH>(in, out, P, dt, ch, damp, strip, j0, count, vmax, reverts, carry);
    else
        y_segment<PH>(in, out, P, dt, ch, damp, strip, j0, count, vmax, reverts);
}

// Warp-wide CFL maximum into one atomic (when P.accumulate) and the revert
// count into the clock.  Called by whole warps.
__device__ __forceinline__ void y_fold(const StepParams& P, double vmax, unsigned reverts) {
    const int lane = threadIdx.x & 31;
    if (P.accumulate) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double t = __shfl_xor_sync(FULL, vmax, o);
            vmax = (vmax < t) ? t : vmax;
        }
        if (lane == 0) {
            unsigned long long* tgt = P.clock ? &P.clock->maxbits[P.parity ^ 1] : P.max_out;
            if (tgt) atomic_max_pos(tgt, vmax);
        }
    }
    if (P.clock && reverts) atomicAdd(&P.clock->flux_fallbacks, reverts);
}

// Clock advance of a completed device-mode step (one thread per step).
__device__ __forceinline__ void clock_advance(const StepParams& P, double dt, double ch) {
    DevClock* c = P.clock;
    c->t[P.parity ^ 1] = c->t[P.parity] + dt;
    c->steps += 1;
    c->last_dt = dt;
    c->last_ch = ch;
}

// The y-sweep's work is `strips` column strips, each cut into row bands of
// `per` rows (the policy's kYBand by default).  Warp w takes strip w % strips,
// band w / strips: the warps of a CTA sit side by side on one band and
// consecutive CTAs walk across the width first, so the resident CTAs cover a
// narrow window of full-width rows that moves down the grid.  Measured on B200
// (4096^2, FP32, register window): 32-row bands 0.72 ms, 64 rows 0.78 ms, 128
// rows 0.96 ms, and one wave of ~300-row bands 1.31 ms -- short bands in a
// moving window keep the segment
// halos and the pages in use shared.
__host__ __device__ __forceinline__ int y_strips(const DevGrid& g) { return (g.ng + g.nx + 31) / 32; }

template <class PH>
__global__ void __launch_bounds__(32 * PH::kYWarps, PH::kYBlocks) sweep_y_kernel(DevGrid in, DevGrid out,
                                                                            StepParams P, int per) {
    using R = typename PH::Real;
    double dt, ch, damp;
    const bool first = (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0);
    if (!step_scalars(P, dt, ch, damp)) {
        if (first) clock_flag_skip(P);
        return;
    }
    if (P.any_dirichlet) gather_dirichlet_ghosts<R>(in, out, P.bc);
    const int strips = y_strips(in);
    const int w = blockIdx.x * PH::kYWarps + threadIdx.y;
    const int r0 = (w / strips) * per;
    __shared__ R carry[PH::kYCarry ? PH::kYWarps * YCarry<PH>::kSlots * 32 : 1];
    double vmax = 0.0;
    unsigned reverts = 0;
    if (r0 < in.ny)
        y_march<PH>(in, out, P, dt, ch, damp, w % strips, in.ng + r0, min(per, in.ny - r0), vmax, reverts,
                    carry + threadIdx.y * YCarry<PH>::kSlots * 32);
    y_fold(P, vmax, reverts);
    if (P.clock && first) clock_advance(P, dt, ch);
}

// Standalone CFL maximum over the interior (compute_dt, src/cpu/solver_cpu.cpp:283-303)
// with `ch` as the floor; one atomic per warp.
template <class PH>
__global__ void __launch_bounds__(256) max_speed_kernel(DevGrid gd, double gamma, double ch,
                                                       unsigned long long* out) {
    using R = typename PH::Real;
    const long long n = (long long)gd.nx * gd.ny;
    double vmax = 0.0;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(k / gd.nx), i = (int)(k - (long long)j * gd.nx);
        R U[NV];
        load_cell(gd, gd.ng + i, gd.ng + j, U);
        const double s = PH::speed(U, gamma, ch);
        vmax = (vmax < s) ? s : vmax;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double t = __shfl_xor_sync(FULL, vmax, o);
        vmax = (vmax < t) ? t : vmax;
    }
    if ((threadIdx.x & 31) == 0) atomic_max_pos(out, vmax);
}

}  // namespace mhd
