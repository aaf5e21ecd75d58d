// launch.h -- host-side entry points of the kernel translation units.  Only
// the C-ABI layer (capi.cu) includes this; it is not part of the public API.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <mutex>

#include "mhd_common.cuh"

namespace mhd {

// NVTX range over one C-ABI call (visible in Nsight Systems / usable as an
// ncu --nvtx-include filter); header-only NVTX v3, a no-op without a tool.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// A kernel's function attributes (its dynamic shared-memory opt-in, its
// carveout) belong to the context of the device they were set on.  run(set)
// calls `set` once per device -- on the first call made with that device
// current -- and returns its result on every later call there.
struct PerDeviceOnce {
    static constexpr int kMaxDevices = 64;
    std::mutex mu;
    bool done[kMaxDevices] = {};
    cudaError_t result[kMaxDevices] = {};

    template <class F>
    cudaError_t run(F&& set) {
        int dev = 0;
        const cudaError_t g = cudaGetDevice(&dev);
        if (g != cudaSuccess) return g;
        if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
        std::lock_guard<std::mutex> lock(mu);
        if (!done[dev]) {
            result[dev] = set();
            done[dev] = true;
        }
        return result[dev];
    }
};

// One split step Uin -> Utmp (x) -> Uout (y), reference semantics.
// which: 1 = x-sweep only, 2 = y-sweep only, 3 = both, 0 = nothing (only the
// one-time kernel attribute setup, so that a later stream capture makes none).
// ystage: 1 = y-sweep rows staged by TMA (needs P.fault and a 16-byte aligned
// slab; other grids use per-thread loads), 0 = per-thread loads.
cudaError_t launch_step_f64(const DevGrid& in, const DevGrid& tmp, const DevGrid& out, const StepParams& P,
                            cudaStream_t st, int yseg, int which = 3, int xrpw = kDefaultXRpw, int ystage = 0);
cudaError_t launch_step_f32(const DevGrid& in, const DevGrid& tmp, const DevGrid& out, const StepParams& P,
                            cudaStream_t st, int yseg, int which = 3, int xrpw = kDefaultXRpw, int ystage = 0);

// 3D tensor map (x, row, field) over the 9 planes of `g` with boxes of
// box_cols x box_rows x 9; false when the slab is not TMA-addressable (base or
// strides not 16-byte multiples) or the driver has no encoder.
bool rows_tensor_map(void* map64, const DevGrid& g, int elem_bytes, int box_cols, int box_rows);

// Batched instances: one persistent launch per sweep over the global work list
// (batch.cuh).  which = 1: x-sweeps of every instance, 2: y-sweeps.
struct BatchInst;
cudaError_t launch_batch_f64(const BatchInst* inst, const int* first, int n, int parity, int which, int solver,
                             int limiter, int xrpw, int yseg, int ctas, cudaStream_t st);
cudaError_t launch_batch_f32(const BatchInst* inst, const int* first, int n, int parity, int which, int solver,
                             int limiter, int xrpw, int yseg, int ctas, cudaStream_t st);

// riemann_flux of n faces (AoS, 9 doubles per face, device memory) with the
// precision's own solver functions; dir 0 = x, 1 = y.
cudaError_t launch_faces_f64(const double* UL, const double* UR, long long n, int dir, int solver, double ch,
                             double gamma, double* F, cudaStream_t st);
cudaError_t launch_faces_f32(const double* UL, const double* UR, long long n, int dir, int solver, double ch,
                             double gamma, double* F, cudaStream_t st);

// CFL maximum (floored by ch) folded into *out with atomicMax on the bits.
cudaError_t launch_max_speed_f64(const DevGrid& g, double gamma, double ch, unsigned long long* out,
                                 cudaStream_t st, int nsm);
cudaError_t launch_max_speed_f32(const DevGrid& g, double gamma, double ch, unsigned long long* out,
                                 cudaStream_t st, int nsm);

// Smallest linear interior index whose CFL speed (floor ch) equals m (atomicMin on *idx).
cudaError_t launch_argmax_f64(const DevGrid& g, double gamma, double ch, double m, int* idx, cudaStream_t st);
cudaError_t launch_argmax_f32(const DevGrid& g, double gamma, double ch, double m, int* idx, cudaStream_t st);

// In-place apply_boundary (head/cpu/boundary_cpu.hpp:45-149), any precision.
cudaError_t launch_apply_boundary(const DevGrid& g, int elem_bytes, const int* bc, cudaStream_t st);

// f64 <-> f32 plane conversion over the whole padded slab.
cudaError_t launch_convert_f64_to_f32(const DevGrid& src, const DevGrid& dst, cudaStream_t st);
cudaError_t launch_convert_f32_to_f64(const DevGrid& src, const DevGrid& dst, cudaStream_t st);

// Dense AoS Conserved array (device) <-> grid of either precision.
cudaError_t launch_aos_to_grid(const double* aos, const DevGrid& dst, int elem_bytes, cudaStream_t st);
cudaError_t launch_grid_to_aos(const DevGrid& src, int elem_bytes, double* aos, cudaStream_t st);

// FP64 diagnostics: out[0] = sum rho dA, out[1] = sum E dA, out[2] = sum |divB| dA,
// out[3] = max |divB|, out[4] = min rho, out[5] = min p.  Deterministic
// (fixed-order) two-pass reduction through `scratch` (>= 6 * 1024 doubles).
cudaError_t launch_diagnostics(const DevGrid& g, int elem_bytes, double gamma, double dx, double dy,
                               double* scratch, double* out, cudaStream_t st);

// Initial data of case `id` evaluated on the device at every cell centre.
cudaError_t launch_initialise(const DevGrid& g, int elem_bytes, int id, double x0, double y0, double dx, double dy,
                              cudaStream_t st);

// Parametrised Orszag-Tang initial data (mhd_initialise_orszag_tang).
cudaError_t launch_initialise_ot(const DevGrid& g, int elem_bytes, double b0, double gamma, const double* amp,
                                 double x0, double y0, double dx, double dy, cudaStream_t st);

// Clock initialisation: maxbits[0] = bits(max0), maxbits[1] = 0, t = 0, steps = 0.
cudaError_t launch_clock_init(DevClock* c, const unsigned long long* max0, cudaStream_t st);

}  // namespace mhd
