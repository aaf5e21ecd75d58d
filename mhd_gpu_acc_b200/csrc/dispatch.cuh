// dispatch.cuh -- runtime (solver, limiter) -> template instance dispatch and
// launch geometry of the two sweeps, shared by the FP64 and FP32 translation
// units.  `which` selects the sweeps: 1 = x only, 2 = y only, 3 = both.
#pragma once

#include "sweep.cuh"

namespace mhd {

template <class PH>
cudaError_t launch_policy(const DevGrid& in, const DevGrid& tmp, const DevGrid& out, const StepParams& P,
                          cudaStream_t st, int yseg, int which) {
    if (which & 1) {
        const int rows_per_cta = XS_ROWS * XS_RPW;
        const dim3 bx(32 * XS_ROWS), gx((in.nx + XS_TX - 1) / XS_TX, (in.ny + rows_per_cta - 1) / rows_per_cta);
        sweep_x_kernel<PH><<<gx, bx, 0, st>>>(in, tmp, P);
    }
    if (which & 2) {
        const int nseg = (in.ny + yseg - 1) / yseg;
        const dim3 by(32, YS_WARPS), gy((in.tnx() + 31) / 32, (nseg + YS_WARPS - 1) / YS_WARPS);
        sweep_y_kernel<PH><<<gy, by, 0, st>>>(tmp, out, P, yseg);
    }
    return cudaGetLastError();
}

template <template <int, int> class POL>
cudaError_t dispatch_step(const DevGrid& in, const DevGrid& tmp, const DevGrid& out, const StepParams& P,
                          cudaStream_t st, int yseg, int which) {
    switch (P.solver * 2 + P.limiter) {
        case 0: return launch_policy<POL<HLL, MINMOD>>(in, tmp, out, P, st, yseg, which);
        case 1: return launch_policy<POL<HLL, VANLEER>>(in, tmp, out, P, st, yseg, which);
        case 2: return launch_policy<POL<HLLC, MINMOD>>(in, tmp, out, P, st, yseg, which);
        case 3: return launch_policy<POL<HLLC, VANLEER>>(in, tmp, out, P, st, yseg, which);
        case 4: return launch_policy<POL<HLLD, MINMOD>>(in, tmp, out, P, st, yseg, which);
        case 5: return launch_policy<POL<HLLD, VANLEER>>(in, tmp, out, P, st, yseg, which);
        case 6: return launch_policy<POL<FORCE, MINMOD>>(in, tmp, out, P, st, yseg, which);
        case 7: return launch_policy<POL<FORCE, VANLEER>>(in, tmp, out, P, st, yseg, which);
        default: return cudaErrorInvalidValue;
    }
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
