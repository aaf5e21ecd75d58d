// sweep.cuh -- the fused directional sweep kernels of one split step.
//
// One launch per sweep replaces the reference's x/y kernels, its two boundary
// kernels per sweep, the psi-damping kernel and the CFL block-max kernel + CUB
// reduction (src/gpu/solver_gpu.cu:188-251, 265-528; src/gpu/boundary_gpu.cu).
//
// x-sweep  (Uin -> Uout): one warp marches along a row segment in chunks of
//          32 consecutive cells; the stencil neighbours come from per-warp
//          shared-memory rings, so primitive, reconstruction, face flux and
//          update each run once per cell with every lane busy.
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
// the x-sweep segment a warp marches and the rows a y-sweep warp takes are
// launch parameters (kDefaultXRpw, kDefaultYBand and, for batches, kDefaultYSeg
// in mhd_common.cuh; the batch autotuner may pick others).
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
// side.  Grid-stride over the ghost ring only -- the 2 ng full-width ghost rows,
// then the 2 ng ghost columns of the interior rows -- so that a launch with few
// threads (an edge-row window of the slab step) does not walk the interior.
template <typename R>
__device__ __forceinline__ void gather_dirichlet_ghosts(const DevGrid& in, const DevGrid& out, const int* bc) {
    const int ng = in.ng, ib = ng, ie = ng + in.nx, jb = ng, je = ng + in.ny;
    const int tx = in.tnx();
    const long long nthreads = (long long)gridDim.x * gridDim.y * blockDim.x * blockDim.y;
    const long long tid = ((long long)blockIdx.y * gridDim.x + blockIdx.x) * (blockDim.x * blockDim.y) +
                          threadIdx.y * blockDim.x + threadIdx.x;
    const long long nrow = 2LL * ng * tx;  // ghost rows 0 .. ng-1 and je .. je+ng-1, full width
    const long long total = nrow + 2LL * ng * in.ny;
    for (long long k = tid; k < total; k += nthreads) {
        int x, y;
        if (k < nrow) {
            const int r = (int)(k / tx);
            x = (int)(k - (long long)r * tx);
            y = r < ng ? r : in.ny + r;
        } else {
            const long long c = k - nrow;
            const int r = (int)(c / (2 * ng)), q = (int)(c - (long long)r * 2 * ng);
            y = jb + r;
            x = q < ng ? q : in.nx + q;
        }
        const bool xg = (x < ib || x >= ie), yg = (y < jb || y >= je);
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

// 16-byte shared-memory slots (four FP32 or two FP64 values): the sweeps keep
// per-lane values in shared memory in these units, so a group of values moves
// with one 128-bit access.
template <typename R>
struct Slot16;
template <>
struct Slot16<float> {
    static constexpr int E = 4;
    using V = float4;
    __device__ static V pack(const float* v, int n, int g) {
        const int k = 4 * g;
        return make_float4(v[k], k + 1 < n ? v[k + 1] : 0.f, k + 2 < n ? v[k + 2] : 0.f, k + 3 < n ? v[k + 3] : 0.f);
    }
    __device__ static void unpack(V t, float* v, int n, int g) {
        const int k = 4 * g;
        v[k] = t.x;
        if (k + 1 < n) v[k + 1] = t.y;
        if (k + 2 < n) v[k + 2] = t.z;
        if (k + 3 < n) v[k + 3] = t.w;
    }
};
template <>
struct Slot16<double> {
    static constexpr int E = 2;
    using V = double2;
    __device__ static V pack(const double* v, int n, int g) {
        const int k = 2 * g;
        return make_double2(v[k], k + 1 < n ? v[k + 1] : 0.0);
    }
    __device__ static void unpack(V t, double* v, int n, int g) {
        const int k = 2 * g;
        v[k] = t.x;
        if (k + 1 < n) v[k + 1] = t.y;
    }
};

// N values <-> ceil(N / E) slots of slot group g0 on, `stride` slots apart.
template <typename R, int N, int STRIDE>
__device__ __forceinline__ void slots_put(typename Slot16<R>::V* base, int g0, const R* v) {
#pragma unroll
    for (int g = 0; g < (N + Slot16<R>::E - 1) / Slot16<R>::E; ++g) base[(g0 + g) * STRIDE] = Slot16<R>::pack(v, N, g);
}
template <typename R, int N, int STRIDE>
__device__ __forceinline__ void slots_get(const typename Slot16<R>::V* base, int g0, R* v) {
#pragma unroll
    for (int g = 0; g < (N + Slot16<R>::E - 1) / Slot16<R>::E; ++g) {
        const typename Slot16<R>::V t = base[(g0 + g) * STRIDE];
        Slot16<R>::unpack(t, v, N, g);
    }
}

// ---------------------------------------------------------------------------
// x-sweep
// ---------------------------------------------------------------------------
// A march along a row.  A warp takes one row segment of `len` interior cells
// starting at interior column c0 and walks it in chunks of 32 consecutive
// cells, lane l holding cell xs + q, q = 32 k + l (xs = ng + c0 - 2, two cells
// before the segment).  At step q a lane computes the primitive state of cell
// q, the reconstruction of cell q - 1, the face flux between cells q - 2 and
// q - 1 and the update of cell q - 2 -- every cell and every face exactly once,
// with all 32 lanes doing useful work except in the last, partial chunk of a
// segment (segments are 32 m - 4 cells long, so a full segment fills its chunks
// exactly).  The neighbour values a lane needs (W of cells q - 2 and q - 1, the
// right-face state of cell q - 2, the flux of face (q - 3 | q - 2)) come from
// three per-warp shared-memory rings of 64 entries, written one step earlier by
// the neighbouring lane or, for lanes 0 and 1, by lanes 30 and 31 of the
// previous chunk; a __syncwarp orders each write before the neighbouring lane's
// read.  The conserved cell updated at step q was loaded two steps before; when
// the policy asks (kXURing) it rides in a fourth ring and comes back from shared
// memory, else it is reloaded from the input (L1-resident), at the top of the
// step when the policy has the registers to hold it across the solve
// (kXEarlyReload), or just before the update.
template <class PH>
struct XRing {
    using R = typename PH::Real;
    static constexpr int E = Slot16<R>::E;
    static constexpr int GW = (PH::NW + E - 1) / E;   // slot groups of a primitive state
    static constexpr int GS = (PH::NS + E - 1) / E;   // of a face-side state
    static constexpr int GF = (NV + E - 1) / E;       // of a face flux
    static constexpr bool kURing = PH::kXURing;       // the conserved cell in the ring too
    static constexpr int GU = kURing ? (NV + E - 1) / E : 0;  // of a conserved cell
    static constexpr int kEntries = 64;
    static constexpr int kGroups = GW + GS + GF + GU;
    static constexpr int kWarpBytes = kGroups * kEntries * 16;
};

template <typename R>
__device__ __forceinline__ void load_cell_or_rest(const DevGrid& g, int x, int y, R* U) {
    if (x < g.tnx()) {
        load_cell(g, x, y, U);
    } else {  // past the grid: a state at rest that only feeds lanes storing nothing
#pragma unroll
        for (int k = 0; k < NV; ++k) U[k] = R(0);
        U[RHO] = R(1);
        U[EN] = R(1);
    }
}

template <class PH>
__device__ __forceinline__ void x_segment(const DevGrid& in, const DevGrid& out, const StepParams& P, double dt,
                                          double ch, int y, int c0, int len,
                                          typename Slot16<typename PH::Real>::V* ring) {
    using R = typename PH::Real;
    using X = XRing<PH>;
    constexpr int NE = X::kEntries;
    const int lane = threadIdx.x & 31;
    const int xs = in.ng + c0 - 2;        // storage column of step q = 0
    const int nk = (len + 4 + 31) >> 5;   // chunks: steps q = 0 .. len + 3
    const double g = P.gamma;
    const double dtd = dt / P.dx;
    unsigned reverts = 0;
    R Unext[NV];
    __syncwarp();  // a warp that marched a segment before may still be reading its ring
    load_cell_or_rest(in, xs + lane, y, Unext);
#pragma unroll 1
    for (int k = 0; k < nk; ++k) {
        const int q = 32 * k + lane;
        const int x = xs + q;
        typename PH::Prim Wm, Wc, Wp;
        R U[NV];
#pragma unroll
        for (int f = 0; f < NV; ++f) U[f] = Unext[f];
        if (k + 1 < nk) load_cell_or_rest(in, x + 32, y, Unext);  // prefetch the next chunk
        PH::prim(U, g, Wp.v);
        const int cell = q - 4;  // segment cell updated at this step: storage column x - 2
        const bool upd = cell >= 0 && cell < len;
        R Uc[NV];
        if (PH::kXEarlyReload && !X::kURing && upd) load_cell(in, x - 2, y, Uc);  // its latency hides behind the solve
        typename Slot16<R>::V* const e0 = ring + (q & 63);
        typename Slot16<R>::V* const e1 = ring + ((q - 1) & 63);
        typename Slot16<R>::V* const e2 = ring + ((q - 2) & 63);
        slots_put<R, PH::NW, NE>(e0, 0, Wp.v);
        __syncwarp();
        // After the first barrier of the step: the entry's previous occupant was
        // last read (by lanes 0 and 1, at their update) in the chunk before.
        if constexpr (X::kURing) slots_put<R, NV, NE>(e0, X::GW + X::GS + X::GF, U);
        slots_get<R, PH::NW, NE>(e2, 0, Wm.v);
        slots_get<R, PH::NW, NE>(e1, 0, Wc.v);
        typename PH::Side L, Rt;
        PH::template recon<0>(Wm, Wc, Wp, dtd, ch, g, L, Rt);  // cell q - 1 (valid for q >= 2)
        slots_put<R, PH::NS, NE>(e1, X::GW, Rt.v);
        __syncwarp();
        R F[NV];
        {
            typename PH::Side Rl;
            slots_get<R, PH::NS, NE>(e2, X::GW, Rl.v);
            PH::template face<0>(Rl, L, ch, g, F);  // face (q - 2 | q - 1) (valid for q >= 3)
        }
        slots_put<R, NV, NE>(e1, X::GW + X::GS, F);
        __syncwarp();
        if (upd) {
            R Fm[NV], Un[NV];
            slots_get<R, NV, NE>(e2, X::GW + X::GS, Fm);  // face (q - 3 | q - 2)
            if constexpr (X::kURing) slots_get<R, NV, NE>(e2, X::GW + X::GS + X::GF, Uc);  // cell q - 2
            else if (!PH::kXEarlyReload) load_cell(in, x - 2, y, Uc);
            reverts += update_cell<R>(Uc, F, Fm, R(dtd), Un) ? 1u : 0u;
            store_cell(out, x - 2, y, Un);
            if (near_edge(out, x - 2, y)) scatter_ghosts<R>(out, x - 2, y, Un, P.bc);
        }
    }
    if (reverts && P.clock) atomicAdd(&P.clock->flux_fallbacks, reverts);
}

// Interior cells per x-sweep segment of `chunks` 32-cell chunks.
__host__ __device__ __forceinline__ int x_seg_len(int chunks) { return 32 * chunks - 4; }

// Guided task sizes.  A sweep launches several waves of tasks (4096^2 FP32:
// ~7 waves of x segments, ~9 of y bands), and the tasks of the last wave end at
// staggered times, which leaves SMs idle for up to one task's duration at the
// end of the kernel.  So each sweep's work is cut into three phases of falling
// task length, issued in order: long tasks for most of the grid, then shorter
// ones, so that the long tasks' stragglers overlap short tasks and the kernel
// ends on short tasks.  Phase p covers [lo[p], lo[p+1]) -- interior columns of
// every row (x) or rows of every column strip (y) -- in n[p] tasks of len[p]
// (the last task of phase 2 may be shorter); tasks run phase by phase, the
// row (x) or strip (y) index fastest.
struct SweepPlan {
    int lo[4];
    int len[3];
    int n[3];
};

// Phase 0 ends at the last multiple of len0 at or below e0/64 of `total`,
// phase 1 at the last multiple of len1 after that at or below e1/64 of it.
__host__ __device__ inline SweepPlan guided_plan(int total, int len0, int len1, int len2, int e0, int e1) {
    SweepPlan pl;
    pl.len[0] = len0; pl.len[1] = len1; pl.len[2] = len2;
    pl.lo[0] = 0;
    pl.lo[1] = (int)(((long long)total * e0 / 64) / len0 * len0);
    const int t1 = (int)((long long)total * e1 / 64);
    pl.lo[2] = pl.lo[1] + (t1 > pl.lo[1] ? (t1 - pl.lo[1]) / len1 * len1 : 0);
    pl.lo[3] = total;
    pl.n[0] = pl.lo[1] / len0;
    pl.n[1] = (pl.lo[2] - pl.lo[1]) / len1;
    pl.n[2] = (total - pl.lo[2] + len2 - 1) / len2;
    return pl;
}

__host__ __device__ inline long long plan_tasks(const SweepPlan& pl, int width) {
    return (long long)(pl.n[0] + pl.n[1] + pl.n[2]) * width;
}

// Task k of a plan over `width` rows (x) or strips (y): its row / strip, first
// column / row and length.  False past the last task.  (Host-callable for the
// plan coverage check, tests/plan_check.cu.)
__host__ __device__ __forceinline__ bool plan_task(const SweepPlan& pl, long long k, int width, int& idx, int& start,
                                          int& len) {
    // selects rather than an indexed read, so the plan stays in the parameter bank
    const long long n0 = (long long)pl.n[0] * width, n1 = (long long)pl.n[1] * width;
    const long long n2 = (long long)pl.n[2] * width;
    if (k >= n0 + n1 + n2) return false;
    const bool p0 = k < n0, p1 = !p0 && k < n0 + n1;
    k -= p0 ? 0 : (p1 ? n0 : n0 + n1);
    const int lo = p0 ? pl.lo[0] : (p1 ? pl.lo[1] : pl.lo[2]);
    const int hi = p0 ? pl.lo[1] : (p1 ? pl.lo[2] : pl.lo[3]);
    const int l = p0 ? pl.len[0] : (p1 ? pl.len[1] : pl.len[2]);
    idx = (int)(k % width);
    start = lo + (int)(k / width) * l;
    len = min(l, hi - start);
    return true;
}

// Phase ends in 1/64 of the extent.  x: segments of the requested chunks up
// to 3/4 of the row, then of 1/3 of them, the remainder (under one of those)
// in segments of 1/9.  y: bands of the requested rows up to 7/8 of the rows,
// then of 1/2 of them up to 31/32, then of 1/4 (a band carries a halo of four
// rows, so the short phases stay small).  Measured on B200 at 4096^2 (HLLD,
// van Leer; FP32 / FP64 ms): x 0.543 / 2.209 with one segment length, 0.513 /
// 2.206 with these phases, 0.524 / 2.258 with a third phase of 92-cell
// segments from 15/16 of the row; y 0.617 / 2.973 with one band height, 0.594 /
// 2.919 with two phases (24 then 12 rows from 7/8), 0.582 / 2.891 with these,
// 0.586 / 2.906 with the phases ending at 13/16 and 61/64.
constexpr int kXPhase0End = 48, kXPhase1End = 64;
constexpr int kYPhase0End = 56, kYPhase1End = 62;

__host__ __device__ inline SweepPlan x_plan(int nx, int chunks) {
    const int c1 = chunks / 3 > 1 ? chunks / 3 : 1, c2 = chunks / 9 > 1 ? chunks / 9 : 1;
    return guided_plan(nx, x_seg_len(chunks), x_seg_len(c1), x_seg_len(c2), kXPhase0End, kXPhase1End);
}

__host__ __device__ inline SweepPlan y_plan(int rows, int per) {
    const int p1 = per / 2 > 1 ? per / 2 : 1, p2 = per / 4 > 1 ? per / 4 : 1;
    return guided_plan(rows, per, p1, p2, kYPhase0End, kYPhase1End);
}

// CTA shape and register budget per policy: PH::kXWarps warps per CTA,
// PH::kXBlocks CTAs per SM; each warp takes one (row, segment) task of the
// plan (x_plan), consecutive tasks on adjacent rows.  The rings live in dynamic
// shared memory: kXWarps * XRing<PH>::kWarpBytes.
template <class PH>
__global__ void __launch_bounds__(32 * PH::kXWarps, PH::kXBlocks)
    sweep_x_kernel(DevGrid in, DevGrid out, StepParams P, SweepPlan pl) {
    using R = typename PH::Real;
    using V = typename Slot16<R>::V;
    extern __shared__ __align__(16) unsigned char xs_smem[];
    double dt, ch, damp;
    const bool first = (blockIdx.x == 0 && threadIdx.x == 0);
    if (!step_scalars(P, dt, ch, damp)) {
        if (first) clock_flag_skip(P);
        return;
    }
    if (first && P.clock) P.clock->maxbits[P.parity ^ 1] = 0ull;
    if (P.any_dirichlet && !P.no_gather) gather_dirichlet_ghosts<R>(in, out, P.bc);
    const int warp = threadIdx.x >> 5;
    const long long task = (long long)blockIdx.x * PH::kXWarps + warp;
    int row, c0, len;
    if (!plan_task(pl, task, in.ny, row, c0, len)) return;  // whole warp: no block-level synchronisation follows
    V* ring = reinterpret_cast<V*>(xs_smem + warp * XRing<PH>::kWarpBytes);
    x_segment<PH>(in, out, P, dt, ch, in.ng + row, c0, len, ring);
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
// Slot group g of a lane is carry[g * 32 + lane] (16 bytes: four FP32 or two
// FP64 values move with one 128-bit access); a warp's access is one contiguous,
// conflict-free row of 512 bytes and no other thread reads it, so no
// synchronisation is needed.  Moving these 2*NW + NS + NV values out of the
// register file lets the sweep run at the x-sweep's register budget (more
// resident warps) for a few shared-memory loads and stores per cell; values and
// operation order are those of y_segment, so results are identical.  When the
// policy asks (kYURing), the conserved row r - 2 that step r updates also comes
// from the slots (rows r - 2 and r share a slot pair by row parity) instead of
// a second global load of that row.
template <class PH>
struct YCarry {
    using R = typename PH::Real;
    static constexpr int E = Slot16<R>::E;
    static constexpr int GW = (PH::NW + E - 1) / E;  // slot groups of one primitive row
    static constexpr int GS = (PH::NSY + E - 1) / E;  // of one side state (the values a y-face uses)
    static constexpr int GF = (NV + E - 1) / E;      // of one face flux
    static constexpr bool kURing = PH::kYURing;       // conserved rows r - 2 / r in the slots too
    static constexpr int GU = (NV + E - 1) / E;      // of one conserved row
    static constexpr int kGroups = 2 * GW + GS + GF + (kURing ? 2 * GU : 0);
    static constexpr int kSlots = kGroups * E;        // R values per lane (the shared array's unit)
};

template <class PH>
__device__ __forceinline__ void y_segment_carried(const DevGrid& in, const DevGrid& out, const StepParams& P,
                                                  double dt, double ch, double damp, int strip, int j0, int count,
                                                  double& vmax, unsigned& reverts, typename PH::Real* carry) {
    using R = typename PH::Real;
    using C = YCarry<PH>;
    using V = typename Slot16<R>::V;
    const int lane = threadIdx.x & 31;
    const int ng = in.ng, ib = ng, ie = ng + in.nx;
    const int x = strip * 32 + lane;
    const int j1 = j0 + count;
    const bool active = (x >= ib && x < ie && count > 0);
    const double g = P.gamma;
    const double dtd = dt / P.dy;
    typename PH::SpeedAcc acc = PH::no_speed();
    V* const lb = reinterpret_cast<V*>(carry) + lane;  // this lane's slot groups, 32 slots apart
    constexpr int RS = 2 * C::GW;                      // last right-biased state
    constexpr int FS = RS + C::GS;                     // last face flux
    constexpr int US = FS + C::GF;                     // conserved rows r - 2 / r (ring by row parity)

    if (active) {
        typename PH::Prim Wm, Wc, Wp;
        typename PH::Side Rprev, L, Rt;
        R F[NV], U[NV];
        R Unext[NV];
        load_cell(in, x, j0 - 2, U);
        load_cell(in, x, j0 - 1, Unext);
        PH::prim(U, g, Wp.v);
        slots_put<R, PH::NW, 32>(lb, ((j0 - 2) & 1) * C::GW, Wp.v);
        PH::prim(Unext, g, Wp.v);
        slots_put<R, PH::NW, 32>(lb, ((j0 - 1) & 1) * C::GW, Wp.v);
        if constexpr (C::kURing) slots_put<R, NV, 32>(lb, US + ((j0 - 1) & 1) * C::GU, Unext);
        load_cell(in, x, j0, Unext);
#pragma unroll 1
        for (int r = j0; r <= j1 + 1; ++r) {
#pragma unroll
            for (int k = 0; k < NV; ++k) U[k] = Unext[k];
            if (r <= j1) load_cell(in, x, r + 1, Unext);  // prefetch the next row
            R Uc[NV];
            if constexpr (C::kURing) {
                if (r >= j0 + 2) slots_get<R, NV, 32>(lb, US + (r & 1) * C::GU, Uc);  // the row updated below
                slots_put<R, NV, 32>(lb, US + (r & 1) * C::GU, U);
            } else if (r >= j0 + 2) {
                load_cell(in, x, r - 2, Uc);
            }
            PH::prim(U, g, Wp.v);
            const int gm = (r & 1) * C::GW;          // row r - 2, overwritten by row r
            const int gc = ((r - 1) & 1) * C::GW;    // row r - 1
            slots_get<R, PH::NW, 32>(lb, gm, Wm.v);
            slots_get<R, PH::NW, 32>(lb, gc, Wc.v);
            slots_put<R, PH::NW, 32>(lb, gm, Wp.v);
            PH::template recon<1>(Wm, Wc, Wp, dtd, ch, g, L, Rt);  // cell r-1
            if (r >= j0 + 1) {
                slots_get<R, PH::NSY, 32>(lb, RS, Rprev.v);
                PH::y_side_rest(Rprev);
                PH::template face<1>(Rprev, L, ch, g, F);  // face (r-2 | r-1)
                if (r >= j0 + 2) {
                    const int yc = r - 2;
                    R Fprev[NV], Un[NV];
                    slots_get<R, NV, 32>(lb, FS, Fprev);
                    reverts += update_cell<R>(Uc, F, Fprev, R(dtd), Un) ? 1u : 0u;
                    if (near_edge(out, x, yc)) scatter_ghosts<R>(out, x, yc, Un, P.bc);
                    Un[PSI] = Un[PSI] * R(damp);
                    store_cell(out, x, yc, Un);
                    if (P.accumulate) PH::fold_speed(Un, g, ch, acc);
                }
                slots_put<R, NV, 32>(lb, FS, F);
            }
            slots_put<R, PH::NSY, 32>(lb, RS, Rt.v);
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

// The y-sweep's work is `strips` column strips, each cut into row bands (the
// policy's kYBand rows by default, shorter bands at the end: y_plan).  Warp w
// takes task w of the plan, strip-fastest: the warps of a CTA sit side by side
// on one band and consecutive CTAs walk across the width first, so the resident
// CTAs cover a narrow window of full-width rows that moves down the grid.
// Measured on B200 (4096^2, FP32, register window, one band height): 32-row
// bands 0.72 ms, 64 rows 0.78 ms, 128 rows 0.96 ms, and one wave of ~300-row
// bands 1.31 ms -- short bands in a moving window keep the segment halos and
// the pages in use shared.
__host__ __device__ __forceinline__ int y_strips(const DevGrid& g) { return (g.ng + g.nx + 31) / 32; }

template <class PH>
__global__ void __launch_bounds__(32 * PH::kYWarps, PH::kYBlocks) sweep_y_kernel(DevGrid in, DevGrid out,
                                                                            StepParams P, SweepPlan pl) {
    using R = typename PH::Real;
    double dt, ch, damp;
    const bool first = (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0);
    if (!step_scalars(P, dt, ch, damp)) {
        if (first) clock_flag_skip(P);
        return;
    }
    if (P.any_dirichlet && !P.no_gather) gather_dirichlet_ghosts<R>(in, out, P.bc);
    const int w = blockIdx.x * PH::kYWarps + threadIdx.y;
    int strip, r0, count;  // r0: first row of the band within the launch's interior row window (y_plan)
    __shared__ __align__(16) R carry[PH::kYCarry ? PH::kYWarps * YCarry<PH>::kSlots * 32 : 1];
    double vmax = 0.0;
    unsigned reverts = 0;
    if (plan_task(pl, w, y_strips(in), strip, r0, count))
        y_march<PH>(in, out, P, dt, ch, damp, strip, in.ng + P.row0 + r0, count, vmax, reverts,
                    carry + threadIdx.y * YCarry<PH>::kSlots * 32);
    y_fold(P, vmax, reverts);
    if (P.clock && first && !P.no_advance) clock_advance(P, dt, ch);
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
