// batch.cuh -- many independent instances of uneven size advanced together.
//
// Each instance (its own grid, gamma, CFL, c_r, boundary types, t_end and
// device clock) is cut into the same work units the single-grid sweeps use:
// x units of BX_WARPS (row, segment) tasks, segments of x_seg_len(4 * rpw)
// cells marched by one warp each (x_segment); y units of YS_WARPS
// consecutive (strip, band) items of an instance, strip-fastest (a strip is 32
// columns, a band seg rows), as the single-grid y-sweep orders its warps.  The units of all instances
// form one global list (prefix offsets in `first`, split by phase: first[0..n]
// for x, first[n+1..2n+1] for y).  A persistent launch per sweep phase -- `ctas` CTAs striding over the
// list -- advances every instance; the kernel boundary between the x and y
// phases is the only synchronisation a step needs, and a CUDA graph of two
// steps replays the loop.  Instance k's unit 0 performs the clock duties the
// single-grid kernels give to CTA (0, 0).
#pragma once

#include "dispatch.cuh"

namespace mhd {

constexpr int BX_WARPS = 4;  // warps per batched x-sweep CTA

struct BatchInst {
    DevGrid U, T;
    StepParams P;  // physics, boundary types, t_end and clock of this instance
    int x_segs, x_pad_;      // x-sweep segments per row
    int y_strips, y_bands;   // 32-column strips; bands of seg rows
    int y_units;             // ceil(strips * bands / YS_WARPS)
    int pad_;
};

// largest k in [0, n) with first[k] <= u (first is non-decreasing, first[0] = 0)
__device__ __forceinline__ int find_instance(const int* first, int n, int u) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(first + mid) <= u) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Dynamic shared memory of the batched x-sweep: one x_segment ring per warp.
template <class PH>
constexpr int bx_smem_bytes() { return BX_WARPS * XRing<PH>::kWarpBytes; }

template <class PH>
__global__ void __launch_bounds__(32 * BX_WARPS, PH::kXBlocks) batch_x_kernel(const BatchInst* __restrict__ inst,
                                                              const int* __restrict__ first, int n, int parity,
                                                              int rpw) {
    using V = typename Slot16<typename PH::Real>::V;
    extern __shared__ __align__(16) unsigned char bx_smem[];
    const int warp = threadIdx.x >> 5;
    V* ring = reinterpret_cast<V*>(bx_smem + warp * XRing<PH>::kWarpBytes);
    const int len = x_seg_len(4 * rpw);
    const int total = __ldg(first + n);
    for (int u = blockIdx.x; u < total; u += gridDim.x) {
        const int k = find_instance(first, n, u);
        const int local = u - __ldg(first + k);
        StepParams P = inst[k].P;
        P.parity = parity;
        double dt, ch, damp;
        if (!step_scalars(P, dt, ch, damp)) {
            if (local == 0 && threadIdx.x == 0) clock_flag_skip(P);
            continue;
        }
        if (local == 0 && threadIdx.x == 0) P.clock->maxbits[parity ^ 1] = 0ull;
        const DevGrid& U = inst[k].U;
        const long long task = (long long)local * BX_WARPS + warp;
        if (task < (long long)inst[k].x_segs * U.ny) {  // whole warp
            const int row = (int)(task % U.ny), c0 = (int)(task / U.ny) * len;
            x_segment<PH>(U, inst[k].T, P, dt, ch, U.ng + row, c0, min(len, U.nx - c0), ring);
        }
    }
}

template <class PH>
__global__ void __launch_bounds__(32 * YS_WARPS, PH::kYBlocks) batch_y_kernel(const BatchInst* __restrict__ inst,
                                                               const int* __restrict__ first, int n, int parity,
                                                               int seg) {
    using R = typename PH::Real;
    __shared__ __align__(16) R carry[PH::kYCarry ? YS_WARPS * YCarry<PH>::kSlots * 32 : 1];
    const int total = __ldg(first + n);
    const bool lead = (threadIdx.x == 0 && threadIdx.y == 0);
    for (int u = blockIdx.x; u < total; u += gridDim.x) {
        const int k = find_instance(first, n, u);
        const int local = u - __ldg(first + k);
        StepParams P = inst[k].P;
        P.parity = parity;
        double dt, ch, damp;
        if (!step_scalars(P, dt, ch, damp)) {
            if (local == 0 && lead) clock_flag_skip(P);
            continue;
        }
        const int strips = inst[k].y_strips;
        const DevGrid& T = inst[k].T;
        const int item = local * YS_WARPS + threadIdx.y;
        const int strip = item % strips, r0 = (item / strips) * seg;
        double vmax = 0.0;
        unsigned reverts = 0;
        if (item < strips * inst[k].y_bands)
            y_march<PH>(T, inst[k].U, P, dt, ch, damp, strip, T.ng + r0, min(seg, T.ny - r0), vmax, reverts,
                        carry + threadIdx.y * YCarry<PH>::kSlots * 32);
        y_fold(P, vmax, reverts);
        if (local == 0 && lead) clock_advance(P, dt, ch);
    }
}

// The x phase's dynamic shared memory opt-in (once per policy and device,
// before any stream capture: mhd_batch_run makes a which = 0 call first).
template <class PH>
cudaError_t bx_setup() {
    static_assert(PH::kXBlocks * (bx_smem_bytes<PH>() + kSmemPerCTAReserve) <= kSmemPerSM,
                  "batched x-phase rings of kXBlocks CTAs exceed an SM's shared memory");
    static PerDeviceOnce once;
    return once.run([] {
        cudaError_t r = cudaFuncSetAttribute(batch_x_kernel<PH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             bx_smem_bytes<PH>());
        if (r == cudaSuccess)
            r = cudaFuncSetAttribute(batch_x_kernel<PH>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared);
        return r;
    });
}

struct BatchLaunch {
    const BatchInst* inst;
    const int* first;
    int n, parity, which, xrpw, yseg, ctas;
    cudaStream_t st;
    template <class PH>
    cudaError_t run() const {
        const cudaError_t attr = bx_setup<PH>();
        if (attr != cudaSuccess || which == 0) return attr;  // which 0: the set-up alone
        if (which == 1) {
            batch_x_kernel<PH><<<ctas, 32 * BX_WARPS, bx_smem_bytes<PH>(), st>>>(inst, first, n, parity, xrpw);
        }
        else batch_y_kernel<PH><<<ctas, dim3(32, YS_WARPS), 0, st>>>(inst, first + n + 1, n, parity, yseg);
        return cudaGetLastError();
    }
};

template <template <int, int> class POL>
cudaError_t dispatch_batch(const BatchInst* inst, const int* first, int n, int parity, int which, int solver,
                           int limiter, int xrpw, int yseg, int ctas, cudaStream_t st) {
    BatchLaunch go{inst, first, n, parity, which, xrpw, yseg, ctas, st};
    return with_policy<POL>(solver, limiter, go);
}

}  // namespace mhd
