// dispatch.cuh -- runtime (solver, limiter) -> template instance dispatch and
// launch geometry of the two sweeps, shared by the FP64 and FP32 translation
// units.  `which` selects the sweeps: 1 = x only, 2 = y only, 3 = both;
// `yband` is the height of a y-sweep warp's row band and `xrpw` the x-sweep rows
// per warp.
#pragma once

#include "launch.h"
#include "sweep_tma.cuh"

namespace mhd {

// Dynamic shared memory opt-in of the TMA y-sweep, once per policy and device,
// with the shared-memory carveout at its maximum so that kYTBlocks CTAs' rings
// fit on an SM.
template <class PH>
cudaError_t y_tma_setup() {
    static PerDeviceOnce once;
    return once.run([] {
        cudaError_t r = cudaFuncSetAttribute(sweep_y_tma_kernel<PH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             yt_smem_bytes<typename PH::Real>());
        if (r == cudaSuccess)
            r = cudaFuncSetAttribute(sweep_y_tma_kernel<PH>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared);
        return r;
    });
}

// Dynamic shared memory of the x-sweep's rings (kXWarps warps per CTA), with
// the carveout at its maximum so that kXBlocks CTAs' rings fit on an SM; once
// per policy and device, outside any stream capture (the which = 0 set-up
// launch).
template <class PH>
constexpr int x_smem_bytes() { return PH::kXWarps * XRing<PH>::kWarpBytes; }

// Shared memory of one sm_100 SM (228 KB, of which the runtime keeps 1 KB per
// resident CTA): the rings of kXBlocks CTAs must fit, or the x-sweep silently
// runs fewer CTAs per SM than its register budget was cut for.
constexpr int kSmemPerSM = 228 * 1024, kSmemPerCTAReserve = 1024;
template <class PH>
constexpr bool x_rings_fit() { return PH::kXBlocks * (x_smem_bytes<PH>() + kSmemPerCTAReserve) <= kSmemPerSM; }

template <class PH>
cudaError_t x_setup() {
    static_assert(x_rings_fit<PH>(), "x-sweep rings of kXBlocks CTAs exceed an SM's shared memory");
    static PerDeviceOnce once;
    return once.run([] {
        cudaError_t r = cudaFuncSetAttribute(sweep_x_kernel<PH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             x_smem_bytes<PH>());
        if (r == cudaSuccess)
            r = cudaFuncSetAttribute(sweep_x_kernel<PH>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared);
        return r;
    });
}

template <class PH>
cudaError_t launch_policy(const DevGrid& in, const DevGrid& tmp, const DevGrid& out, const StepParams& P,
                          cudaStream_t st, int yband, int which, int xrpw, int ystage) {
    using R = typename PH::Real;
    if (ystage == 1) {
        const cudaError_t e = y_tma_setup<PH>();
        if (e != cudaSuccess) return e;
    }
    {
        const cudaError_t e = x_setup<PH>();
        if (e != cudaSuccess) return e;
    }
    if (which & 1) {
        // xrpw sets the x-sweep work per warp: row segments of 4 * xrpw chunks of 32 cells (then shorter
        // ones); 0 = the policy's kXRpw
        const SweepPlan pl = x_plan(in.nx, 4 * (xrpw > 0 ? xrpw : PH::kXRpw));
        const long long ctas = (plan_tasks(pl, in.ny) + PH::kXWarps - 1) / PH::kXWarps;
        sweep_x_kernel<PH><<<(unsigned)ctas, 32 * PH::kXWarps, x_smem_bytes<PH>(), st>>>(in, tmp, P, pl);
    }
    if (which & 2) {
        const int per = yband > 0 ? yband : PH::kYBand;
        const int rows = P.nrows > 0 ? P.nrows : tmp.ny - P.row0;  // the interior row window
        alignas(64) CUtensorMap map;
        if (ystage == 1 && P.fault &&
            rows_tensor_map(&map, tmp, (int)sizeof(R), YT_COLS, YTShape<R>::ROWS)) {
            // the TMA-staged y-sweep: one band height (its CTAs stage fixed boxes)
            const long long bands = (rows + per - 1) / per;
            const long long groups = (y_strips(tmp) + YT_WARPS - 1) / YT_WARPS;
            sweep_y_tma_kernel<PH><<<(unsigned)(groups * bands), dim3(32, YT_WARPS), yt_smem_bytes<R>(), st>>>(
                map, tmp, out, P, per);
        } else {
            const SweepPlan pl = y_plan(rows, per);
            const long long warps = plan_tasks(pl, y_strips(tmp));
            const unsigned grid = (unsigned)((warps + PH::kYWarps - 1) / PH::kYWarps);
            sweep_y_kernel<PH><<<grid, dim3(32, PH::kYWarps), 0, st>>>(tmp, out, P, pl);
        }
    }
    return cudaGetLastError();
}

// Calls F::template run<POL<S, L>>() for the runtime (solver, limiter) pair.
template <template <int, int> class POL, class F>
cudaError_t with_policy(int solver, int limiter, F&& f) {
    switch (solver * 2 + limiter) {
        case 0: return f.template run<POL<HLL, MINMOD>>();
        case 1: return f.template run<POL<HLL, VANLEER>>();
        case 2: return f.template run<POL<HLLC, MINMOD>>();
        case 3: return f.template run<POL<HLLC, VANLEER>>();
        case 4: return f.template run<POL<HLLD, MINMOD>>();
        case 5: return f.template run<POL<HLLD, VANLEER>>();
        case 6: return f.template run<POL<FORCE, MINMOD>>();
        case 7: return f.template run<POL<FORCE, VANLEER>>();
        default: return cudaErrorInvalidValue;
    }
}

struct StepLaunch {
    const DevGrid &in, &tmp, &out;
    const StepParams& P;
    cudaStream_t st;
    int yseg, which, xrpw, ystage;
    template <class PH>
    cudaError_t run() const { return launch_policy<PH>(in, tmp, out, P, st, yseg, which, xrpw, ystage); }
};

template <template <int, int> class POL>
cudaError_t dispatch_step(const DevGrid& in, const DevGrid& tmp, const DevGrid& out, const StepParams& P,
                          cudaStream_t st, int yseg, int which, int xrpw, int ystage) {
    StepLaunch go{in, tmp, out, P, st, yseg, which, xrpw, ystage};
    return with_policy<POL>(P.solver, P.limiter, go);
}

// riemann_flux (head/riemann.hpp:568-592) of n independent faces with the
// sweeps' own solver functions: face k's left / right conserved states are
// UL[9k..9k+8] / UR[9k..9k+8] (FP64, rounded to the policy's precision), its
// flux goes to F[9k..9k+8].  No warp-collective operations are involved, so
// any thread may take any face.
template <class PH, int DIR>
__global__ void __launch_bounds__(256) face_flux_kernel(const double* UL, const double* UR, long long n, double ch,
                                                        double gamma, double* F) {
    using R = typename PH::Real;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        R uL[NV], uR[NV], f[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) { uL[q] = (R)UL[k * NV + q]; uR[q] = (R)UR[k * NV + q]; }
        typename PH::Side L, Rs;
        PH::template side<DIR>(uL, gamma, L);
        PH::template side<DIR>(uR, gamma, Rs);
        PH::template face<DIR>(L, Rs, ch, gamma, f);
#pragma unroll
        for (int q = 0; q < NV; ++q) F[k * NV + q] = (double)f[q];
    }
}

struct FaceLaunch {
    const double *UL, *UR;
    long long n;
    int dir;
    double ch, gamma;
    double* F;
    cudaStream_t st;
    template <class PH>
    cudaError_t run() const {
        long long blocks = (n + 255) / 256;
        if (blocks > 65535) blocks = 65535;
        if (blocks < 1) return cudaSuccess;
        if (dir == 0) face_flux_kernel<PH, 0><<<(unsigned)blocks, 256, 0, st>>>(UL, UR, n, ch, gamma, F);
        else face_flux_kernel<PH, 1><<<(unsigned)blocks, 256, 0, st>>>(UL, UR, n, ch, gamma, F);
        return cudaGetLastError();
    }
};

template <template <int, int> class POL>
cudaError_t launch_faces_policy(const double* UL, const double* UR, long long n, int dir, int solver, double ch,
                                double gamma, double* F, cudaStream_t st) {
    FaceLaunch go{UL, UR, n, dir, ch, gamma, F, st};
    return with_policy<POL>(solver, MINMOD, go);
}

// Smallest linear interior index whose CFL speed (the forward reduction's own
// per-cell function, floor ch) is m -- exactly for FP64; within 2^-20 relative
// for FP32, whose code may be contracted differently in another kernel.
// *idx must start at INT_MAX.
template <class PH>
__global__ void argmax_speed_kernel(DevGrid gd, double gamma, double ch, double m, int* idx) {
    using R = typename PH::Real;
    const double tol = sizeof(R) == 8 ? 0.0 : m * 9.5367431640625e-07;
    const long long n = (long long)gd.nx * gd.ny;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(k / gd.nx), i = (int)(k - (long long)j * gd.nx);
        R U[NV];
        load_cell(gd, gd.ng + i, gd.ng + j, U);
        if (fabs(PH::speed(U, gamma, ch) - m) <= tol) atomicMin(idx, (int)k);
    }
}

template <class PH>
cudaError_t launch_argmax_policy(const DevGrid& g, double gamma, double ch, double m, int* idx, cudaStream_t st) {
    const long long n = (long long)g.nx * g.ny;
    long long blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    argmax_speed_kernel<PH><<<(unsigned)blocks, 256, 0, st>>>(g, gamma, ch, m, idx);
    return cudaGetLastError();
}

template <class PH>
cudaError_t launch_max_policy(const DevGrid& g, double gamma, double ch, unsigned long long* out, cudaStream_t st,
                              int nsm) {
    const long long n = (long long)g.nx * g.ny;
    long long blocks = (n + 255) / 256;
    const long long cap = (long long)nsm * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    max_speed_kernel<PH><<<(unsigned)blocks, 256, 0, st>>>(g, gamma, ch, out);
    return cudaGetLastError();
}

}  // namespace mhd
