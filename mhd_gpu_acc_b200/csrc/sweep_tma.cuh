// sweep_tma.cuh -- y-sweep with its input rows staged in shared memory by TMA.
//
// Same arithmetic and the same per-thread register window as sweep_y_kernel
// (sweep.cuh), but the rows it marches down are not fetched by per-thread
// loads: a CTA of YT_WARPS warps side by side covers 32*YT_WARPS columns of one
// row band, and the band's rows (two halo rows above, two below) arrive as
// {32*YT_WARPS columns x ROWS rows x 9 fields} boxes of one 3D tensor map
// (x, row, field) over the x-swept state, through a ring of STAGES shared-memory
// buffers.  Each thread reads its cell of row r, and row r-2 again for the
// update, from shared memory; the registers that held the one-row prefetch and
// the reloaded row are freed, and the copy engine runs a chunk of rows ahead.
//
// Pipeline: box k goes to stage k % STAGES and completes on mbarrier full[s]
// (phase k / STAGES).  A warp releases box k once it no longer reads it (when
// row r-2 has moved into box k+1); the last of the CTA's warps to release a
// stage issues the box STAGES later into it, so no warp waits on another's
// release and no producer warp is needed.  Every wait is bounded by the global
// timer (StepParams::tma_wait_ns, default kTmaWaitNs).  A warp whose wait gives
// up records CLK_TIMEOUT in the fault word (and the clock) and raises a
// CTA-wide abort flag in shared memory, so the other warps stop waiting at
// once instead of each sitting out its own limit on boxes that the aborted
// warp will never release.  Before the CTA exits, one thread waits (bounded by
// kTmaWaitNs) for the last box issued into every stage, so no copy can land in
// the CTA's shared memory after it is gone.  Lanes of a warp agree on every
// wait's outcome (a vote), so the warp never splits around a __syncwarp.
//
// Box coordinates: x = CTA column start (a multiple of 32*YT_WARPS, so 16-byte
// aligned for both element sizes), row >= 0 (the band starts at ng - 2 or
// later), field 0.  Rows or columns past the grid are zero-filled by the copy
// engine and only ever feed lanes or rows that store nothing.
#pragma once

#include <cuda.h>

#include "sweep.cuh"

namespace mhd {

constexpr int YT_WARPS = 4;
constexpr int YT_COLS = 32 * YT_WARPS;
// A wait on a box gives up after this many nanoseconds (a box lands in microseconds).
constexpr unsigned long long kTmaWaitNs = 2000000000ull;

template <typename R> struct YTShape;
template <> struct YTShape<float> { static constexpr int ROWS = 8, STAGES = 2; };
template <> struct YTShape<double> { static constexpr int ROWS = 4, STAGES = 3; };

template <typename R>
__host__ __device__ constexpr int yt_stage_bytes() { return YT_COLS * YTShape<R>::ROWS * NV * (int)sizeof(R); }
template <typename R>
__host__ __device__ constexpr int yt_smem_bytes() { return YTShape<R>::STAGES * yt_stage_bytes<R>() + 128; }

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of `bar`, bounded by limit_ns of the global timer and
// cut short when *abort becomes non-zero (abort may be null); false when it
// gave up.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, const volatile int* abort,
                                          unsigned long long limit_ns) {
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_test(bar, parity))
        if ((abort && *abort) || global_ns() - t0 > limit_ns) return false;
    return true;
}

// One box of the 3D map into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_box(void* dst, const CUtensorMap* map, int x, int y, int z,
                                        unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void record_fault(const StepParams& P) {
    if (P.fault) atomicOr(P.fault, (int)CLK_TIMEOUT);
    if (P.clock) P.clock->status = CLK_TIMEOUT;
}

// One CTA: columns [x0, x0 + YT_COLS) of interior rows [j0, j0 + count) (ghost
// offset included).  Called by all YT_WARPS warps of the CTA.
template <class PH>
__device__ __forceinline__ void y_band_tma(const CUtensorMap* map, const DevGrid& in, const DevGrid& out,
                                           const StepParams& P, double dt, double ch, double damp, int x0, int j0,
                                           int count, unsigned char* smem, double& vmax, unsigned& reverts) {
    using R = typename PH::Real;
    constexpr int ROWS = YTShape<R>::ROWS, STAGES = YTShape<R>::STAGES;
    constexpr int ROW_ELEMS = YT_COLS;                  // one field row of a box
    constexpr int FIELD_ELEMS = YT_COLS * ROWS;         // one field of a box
    constexpr int STAGE_ELEMS = FIELD_ELEMS * NV;
    R* stage = reinterpret_cast<R*>(smem);
    unsigned long long* full = reinterpret_cast<unsigned long long*>(smem + STAGES * yt_stage_bytes<R>());
    int* released = reinterpret_cast<int*>(full + STAGES);
    int* last_box = released + STAGES;                 // last box issued into each stage (-1: none)
    volatile int* abort_flag = last_box + STAGES;      // a warp gave up: stop waiting
    static_assert(STAGES * (8 + 4 + 4) + 4 <= 128, "barrier block exceeds its 128-byte reserve");
    const unsigned long long wait_ns = P.tma_wait_ns ? P.tma_wait_ns : kTmaWaitNs;

    const int lane = threadIdx.x & 31, warp = threadIdx.y;
    const int col = warp * 32 + lane;
    const int x = x0 + col;
    const int ng = in.ng, ib = ng, ie = ng + in.nx;
    const int top = j0 - 2;                             // first row of box 0
    const int nrows = count + 4;                        // rows j0-2 .. j0+count+1
    const int nbox = (nrows + ROWS - 1) / ROWS;
    const bool active = (x >= ib && x < ie);
    const bool lead = (lane == 0 && warp == 0);

    if (lead) {
        for (int s = 0; s < STAGES; ++s) { mbar_init(&full[s], 1); released[s] = 0; last_box[s] = -1; }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int k = 0; k < STAGES && k < nbox; ++k) {
            mbar_expect_tx(&full[k], (unsigned)yt_stage_bytes<R>());
            tma_box(stage + k * STAGE_ELEMS, map, x0, top + k * ROWS, 0, &full[k]);
            last_box[k] = k;
        }
    }
    __syncthreads();

    // Row q (0-based from `top`) of field f as seen by this thread.
    auto at = [&](int q, int f) -> R {
        const int k = q / ROWS;
        return stage[(k % STAGES) * STAGE_ELEMS + f * FIELD_ELEMS + (q - k * ROWS) * ROW_ELEMS + col];
    };
    auto row = [&](int q, R* U) {
#pragma unroll
        for (int f = 0; f < NV; ++f) U[f] = at(q, f);
    };
    int ready = -1;   // boxes [0, ready] have landed (as far as this warp knows)
    bool ok = true;
    auto need = [&](int q) -> bool {           // make box q / ROWS readable (whole warp)
        const int k = q / ROWS;
        while (ready < k) {
            ++ready;
            const bool got = mbar_wait(&full[ready % STAGES], (unsigned)((ready / STAGES) & 1), abort_flag, wait_ns);
            if (!__all_sync(FULL, got)) {
                if (lane == 0) *abort_flag = 1;
                return false;
            }
        }
        return true;
    };
    auto release = [&](int k) {                 // this warp is done with box k
        __syncwarp();
        if (lane == 0) {
            __threadfence_block();
            const int s = k % STAGES;
            // released[s] counts every release of stage s; the warp completing a
            // multiple of YT_WARPS is the last one out of box k
            if ((atomicAdd(&released[s], 1) + 1) % YT_WARPS == 0) {
                if (k + STAGES < nbox) {
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    mbar_expect_tx(&full[s], (unsigned)yt_stage_bytes<R>());
                    tma_box(stage + s * STAGE_ELEMS, map, x0, top + (k + STAGES) * ROWS, 0, &full[s]);
                    last_box[s] = k + STAGES;
                }
            }
        }
    };

    const double g = P.gamma;
    const double dtd = dt / P.dy;
    typename PH::Prim Wm, Wc, Wp;
    typename PH::Side Rprev, L, Rt;
    R Fprev[NV], F[NV], U[NV];
    ok = need(1);
    if (ok) {
        row(0, U);
        PH::prim(U, g, Wm.v);
        row(1, U);
        PH::prim(U, g, Wc.v);
    }
    for (int q = 2; ok && q < nrows; ++q) {     // q = r - top: row r = j0 - 2 + q
        if (!need(q)) { ok = false; break; }
        row(q, U);
        if (active) {
            PH::prim(U, g, Wp.v);
            PH::template recon<1>(Wm, Wc, Wp, dtd, ch, g, L, Rt);      // cell r-1
            if (q >= 3) {
                PH::template face<1>(Rprev, L, ch, g, F);              // face (r-2 | r-1)
                if (q >= 4) {
                    const int yc = top + q - 2;
                    R Uc[NV], Un[NV];
                    row(q - 2, Uc);
                    reverts += update_cell<R>(Uc, F, Fprev, R(dtd), Un) ? 1u : 0u;
                    if (near_edge(out, x, yc)) scatter_ghosts<R>(out, x, yc, Un, P.bc);
                    Un[PSI] = Un[PSI] * R(damp);
                    store_cell(out, x, yc, Un);
                    if (P.accumulate) {
                        const double sp = PH::speed(Un, g, ch);
                        vmax = (vmax < sp) ? sp : vmax;
                    }
                }
#pragma unroll
                for (int k = 0; k < NV; ++k) Fprev[k] = F[k];
            }
            Rprev = Rt;
            Wm = Wc;
            Wc = Wp;
        }
        // row q-2 was the last read of box (q-2)/ROWS - 1 once q-2 starts a box
        if (q >= 2 + ROWS && (q - 2) % ROWS == 0) release((q - 2) / ROWS - 1);
    }
    if (!ok && lane == 0) record_fault(P);
    // Drain: every wait above is bounded, so all warps get here.  A box is issued
    // into a stage only after every warp released the stage's previous box, so
    // at most the last box of each stage can still be in flight; wait for it
    // (bounded, with the full limit) before the CTA's shared memory goes away.
    __syncthreads();
    if (lead) {
        for (int s = 0; s < STAGES; ++s)
            if (last_box[s] >= 0 && !mbar_wait(&full[s], (unsigned)((last_box[s] / STAGES) & 1), nullptr, kTmaWaitNs))
                record_fault(P);
    }
}

template <class PH>
__global__ void __launch_bounds__(32 * YT_WARPS, PH::kYTBlocks)
    sweep_y_tma_kernel(const __grid_constant__ CUtensorMap map, DevGrid in, DevGrid out, StepParams P, int per) {
    using R = typename PH::Real;
    extern __shared__ __align__(1024) unsigned char yt_smem[];
    double dt, ch, damp;
    const bool first = (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0);
    if (!step_scalars(P, dt, ch, damp)) {
        if (first) clock_flag_skip(P);
        return;
    }
    if (P.any_dirichlet && !P.no_gather) gather_dirichlet_ghosts<R>(in, out, P.bc);
    const int groups = (y_strips(in) + YT_WARPS - 1) / YT_WARPS;
    const int band = blockIdx.x / groups;
    const int row_end = P.nrows > 0 ? P.row0 + P.nrows : in.ny;  // the launch's interior row window
    const int r0 = P.row0 + band * per;
    double vmax = 0.0;
    unsigned reverts = 0;
    if (r0 < row_end)  // uniform over the CTA
        y_band_tma<PH>(&map, in, out, P, dt, ch, damp, (blockIdx.x % groups) * YT_COLS, in.ng + r0,
                       min(per, row_end - r0), yt_smem, vmax, reverts);
    y_fold(P, vmax, reverts);
    if (P.clock && first && !P.no_advance) clock_advance(P, dt, ch);
}

}  // namespace mhd
