// noalloc.cu -- one split step that allocates no device memory.
//
// Some callers of this library cannot call cudaMalloc: applications that hand
// every byte of device memory to their own pool allocator and forbid any other
// allocation, and time-critical loops that cannot afford the device-wide
// synchronisation a cudaMalloc or cudaFree may imply.  mhd_advance needs an
// intermediate (x-swept) state that such a caller would have to allocate;
// mhd_advance_noalloc keeps that state in a fixed device array compiled into
// the library instead, so the caller passes only the input and output states.
//
// The array is a file-scope __device__ variable of MHD_NOALLOC_SCRATCH_BYTES
// (32 MiB): every GPU that loads the library holds it until the process exits.
// Its device address is looked up once per device, on the first call made
// with that device current (cudaGetSymbolAddress); make that first call before
// any stream capture.  The address is kept for the life of the process, so the
// device must not be reset (cudaDeviceReset, or a teardown and re-creation of
// its primary context) between calls.  All calls share the one array, so calls
// whose work can overlap on the GPU (different streams, or different host
// threads on one device) race on it and must be serialised by the caller.  The x-sweep writes
// every cell of the array that the y-sweep then reads, so nothing has to start
// at zero.
#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/mhd_b200.h"
#include "launch.h"

namespace mhd {
int report_error(int code, const char* msg);
void count_launches(unsigned n);
}

namespace {

constexpr size_t kScratchBytes = MHD_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_step_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

int err(int code, const char* fmt, long long a = 0, long long b = 0) {
    char buf[256];
    std::snprintf(buf, sizeof buf, fmt, a, b);
    return mhd::report_error(code, buf);
}

// Device address of the scratch array for the current device (host code may
// not use the symbol itself: on the host it names a stand-in, not device memory).
int scratch_address(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return err(MHD_ERR_CUDA, "mhd_advance_noalloc: no usable current device");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_step_scratch);
        if (e != cudaSuccess || !p)
            return err(MHD_ERR_CUDA, "mhd_advance_noalloc: cudaGetSymbolAddress failed (%lld)", (long long)e);
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return MHD_OK;
}

bool valid(const mhd_grid* g) {
    if (!g || !g->data || g->ng < 2 || g->ng > MHD_MAX_NG || g->nx < g->ng || g->ny < g->ng) return false;
    if (g->dtype != MHD_F64 && g->dtype != MHD_F32) return false;
    const long long tnx = g->nx + 2LL * g->ng, tny = g->ny + 2LL * g->ng;
    return g->pitch >= tnx && g->plane >= g->pitch * tny && g->x_max > g->x_min && g->y_max > g->y_min;
}

}  // namespace

extern "C" int mhd_advance_noalloc(const mhd_grid* Uold, mhd_grid* Unew, double gamma, double ch, double cr,
                                   double dt, int solver, int limiter, const int* bc, void* stream) {
    mhd::NvtxRange nvtx_range("mhd_advance_noalloc");
    if (!valid(Uold) || !valid(Unew)) return err(MHD_ERR_ARG, "mhd_advance_noalloc: invalid grid");
    if (Uold->nx != Unew->nx || Uold->ny != Unew->ny || Uold->ng != Unew->ng || Uold->dtype != Unew->dtype)
        return err(MHD_ERR_ARG, "mhd_advance_noalloc: Uold and Unew differ in shape or precision");
    if (Uold->data == Unew->data) return err(MHD_ERR_ARG, "mhd_advance_noalloc: Uold and Unew must be distinct");
    if (!bc) return err(MHD_ERR_ARG, "mhd_advance_noalloc: null boundary config");
    for (int k = 0; k < 4; ++k)
        if (bc[k] < MHD_BC_PERIODIC || bc[k] > MHD_BC_DIRICHLET)
            return err(MHD_ERR_ARG, "mhd_advance_noalloc: bad boundary type %lld", bc[k]);
    if (solver < MHD_HLL || solver > MHD_FORCE) return err(MHD_ERR_ARG, "mhd_advance_noalloc: bad solver %lld", solver);
    if (limiter != MHD_LIMITER_MINMOD && limiter != MHD_LIMITER_VANLEER)
        return err(MHD_ERR_ARG, "mhd_advance_noalloc: bad limiter %lld", limiter);
    if (!(gamma > 1.0) || !(cr > 0.0) || !(ch >= 0.0))
        return err(MHD_ERR_ARG, "mhd_advance_noalloc: need gamma > 1, cr > 0, ch >= 0");

    // intermediate state: same padded layout as mhd_grid_alloc
    const long long eb = (Uold->dtype == MHD_F32) ? 4 : 8;
    const long long per = 256 / eb;
    const long long tnx = Uold->nx + 2LL * Uold->ng, tny = Uold->ny + 2LL * Uold->ng;
    const long long pitch = (tnx + per - 1) / per * per;
    const long long plane = (pitch * tny + per - 1) / per * per;
    const long long need = plane * MHD_NV * eb;
    if (need > (long long)kScratchBytes)
        return err(MHD_ERR_ARG,
                   "mhd_advance_noalloc: grid needs %lld bytes of intermediate state, above the %lld-byte limit",
                   need, (long long)kScratchBytes);
    void* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;

    mhd::DevGrid in{Uold->data, Uold->pitch, Uold->plane, Uold->nx, Uold->ny, Uold->ng, 0};
    mhd::DevGrid out{Unew->data, Unew->pitch, Unew->plane, Unew->nx, Unew->ny, Unew->ng, 0};
    mhd::DevGrid tmp{scratch, pitch, plane, Uold->nx, Uold->ny, Uold->ng, 0};
    mhd::StepParams P{};
    P.gamma = gamma;
    P.cr = cr;
    P.dx = (Uold->x_max - Uold->x_min) / static_cast<double>(Uold->nx);
    P.dy = (Uold->y_max - Uold->y_min) / static_cast<double>(Uold->ny);
    P.dmin = (P.dy < P.dx) ? P.dy : P.dx;
    P.dt = dt;
    P.ch = ch;
    P.damp = std::exp(-dt * ch / cr);  // host C library exp, as the reference (src/cpu/solver_cpu.cpp:264)
    if (P.damp >= 1.0) P.damp = 1.0;
    P.solver = solver;
    P.limiter = limiter;
    for (int k = 0; k < 4; ++k) P.bc[k] = bc[k];
    P.any_dirichlet = (bc[0] == MHD_BC_DIRICHLET || bc[1] == MHD_BC_DIRICHLET || bc[2] == MHD_BC_DIRICHLET ||
                       bc[3] == MHD_BC_DIRICHLET);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    mhd::count_launches(2);  // the x- and the y-sweep
    const cudaError_t e = (Uold->dtype == MHD_F64) ? mhd::launch_step_f64(in, tmp, out, P, st, mhd::kDefaultYBand, 3)
                                                   : mhd::launch_step_f32(in, tmp, out, P, st, mhd::kDefaultYBand, 3);
    if (e != cudaSuccess) return err(MHD_ERR_CUDA, "mhd_advance_noalloc: launch failed (%lld)", (long long)e);
    return MHD_OK;
}
