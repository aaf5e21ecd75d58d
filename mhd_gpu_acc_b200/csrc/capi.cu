// capi.cu -- implementation of the C ABI in include/mhd_b200.h.
//
// Host-side orchestration only: argument validation, workspaces, the drop-in
// equivalents of the reference's compute_dt_gpu / advance_second_order_gpu /
// apply_boundary_gpu (src/gpu/solver_gpu.cu:578-690, src/gpu/boundary_gpu.cu:158),
// and the device-resident, CUDA-graph-captured step loop.  No function here
// exits the process; every failure becomes an MHD_ERR_* code plus a message.
#include <atomic>
#include <cfloat>
#include <cstdarg>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/mhd_b200.h"
#include "launch.h"

namespace {

thread_local std::string g_err;
std::atomic<unsigned long long> g_launches{0};

int fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) return fail(MHD_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

size_t elem_bytes(int dtype) { return dtype == MHD_F32 ? 4 : 8; }

int check_grid(const mhd_grid* g, const char* what) {
    if (!g) return fail(MHD_ERR_ARG, "%s: null grid", what);
    if (g->ng < 2 || g->ng > MHD_MAX_NG)
        return fail(MHD_ERR_ARG, "%s: ng=%d outside [2, %d]", what, g->ng, MHD_MAX_NG);
    if (g->nx < g->ng || g->ny < g->ng)
        return fail(MHD_ERR_ARG, "%s: nx=%d, ny=%d must be >= ng=%d", what, g->nx, g->ny, g->ng);
    if (g->dtype != MHD_F64 && g->dtype != MHD_F32) return fail(MHD_ERR_ARG, "%s: bad dtype %d", what, g->dtype);
    const long long tnx = g->nx + 2LL * g->ng, tny = g->ny + 2LL * g->ng;
    if (g->pitch < tnx || g->plane < g->pitch * tny)
        return fail(MHD_ERR_ARG, "%s: pitch/plane too small", what);
    if (!g->data) return fail(MHD_ERR_ARG, "%s: null data", what);
    if (!(g->x_max > g->x_min) || !(g->y_max > g->y_min)) return fail(MHD_ERR_ARG, "%s: empty extent", what);
    return MHD_OK;
}

int check_bc(const int* bc) {
    if (!bc) return fail(MHD_ERR_ARG, "null boundary config");
    for (int k = 0; k < 4; ++k)
        if (bc[k] < MHD_BC_PERIODIC || bc[k] > MHD_BC_DIRICHLET) return fail(MHD_ERR_ARG, "bad boundary type %d", bc[k]);
    return MHD_OK;
}

bool same_shape(const mhd_grid* a, const mhd_grid* b) {
    return a->nx == b->nx && a->ny == b->ny && a->ng == b->ng && a->dtype == b->dtype;
}

mhd::DevGrid dev(const mhd_grid* g) {
    mhd::DevGrid d;
    d.data = g->data;
    d.pitch = g->pitch;
    d.plane = g->plane;
    d.nx = g->nx;
    d.ny = g->ny;
    d.ng = g->ng;
    d.pad_ = 0;
    return d;
}

double gdx(const mhd_grid* g) { return (g->x_max - g->x_min) / static_cast<double>(g->nx); }
double gdy(const mhd_grid* g) { return (g->y_max - g->y_min) / static_cast<double>(g->ny); }

}  // namespace

namespace mhd {
// Lets other translation units of the library report through mhd_last_error().
int report_error(int code, const char* msg) {
    g_err = msg;
    return code;
}
// Lets other translation units count their kernel launches in mhd_launch_count().
void count_launches(unsigned n) { g_launches += n; }
}  // namespace mhd

struct mhd_workspace {
    int nx = 0, ny = 0, ng = 0, dtype = 0;
    double gamma = 5.0 / 3.0;  // head/physics.hpp:28 default
    double ch = 0.0;
    double cr = 0.18;          // head/physics.hpp:39
    int limiter = MHD_LIMITER_MINMOD;
    int yseg = mhd::kDefaultYBand;  // y-sweep rows per warp band (0: the precision's default)
    int xrpw = mhd::kDefaultXRpw;  // x-sweep rows per warp
    int ystage = 0;                // y-sweep rows loaded per thread (1: staged by TMA)
    unsigned long long tma_wait_ns = 0;  // limit of each wait for a TMA-staged box (0: 2 s)
    double clk_cfl = 0.0, clk_t_end = 0.0;  // of the clock started by mhd_clock_start
    int clk_started = 0;
    double dx = 0.0, dy = 0.0;     // cell spacing of the step; 0 = from the grid's extent
    int nsm = 148;
    cudaStream_t stream = nullptr;
    unsigned long long* d_max = nullptr;
    mhd::DevClock* d_clock = nullptr;
    int* d_fault = nullptr;       // ClockStatus bits from bounded device waits
    double* d_diag = nullptr;     // 6 * 1024 partials + 6 results
    void* d_stage = nullptr;      // FP64 staging for uploads/downloads
    size_t stage_bytes = 0;
    // graph of two captured steps
    cudaGraphExec_t graph = nullptr;
    struct Key {
        void* u; void* t; int solver, limiter, bc[4], yseg, xrpw, ystage, pad_;
        double gamma, cr, cfl, t_end;
        bool operator==(const Key& o) const { return std::memcmp(this, &o, sizeof(Key)) == 0; }
    } key{};
};

namespace {

// Reads (and clears) the fault word after the stream has drained: a bounded
// device wait that gave up turns into MHD_ERR_TIMEOUT.
int check_fault(mhd_workspace* ws, const char* what) {
    int f = 0;
    if (cudaMemcpyAsync(&f, ws->d_fault, sizeof f, cudaMemcpyDeviceToHost, ws->stream) != cudaSuccess ||
        cudaStreamSynchronize(ws->stream) != cudaSuccess)
        return fail(MHD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(cudaGetLastError()));
    if (f == 0) return MHD_OK;
    cudaMemsetAsync(ws->d_fault, 0, sizeof(int), ws->stream);
    return fail(MHD_ERR_TIMEOUT, "%s: a bounded wait for a staged tile gave up (status %d)", what, f);
}

int ensure_stage(mhd_workspace* ws, size_t bytes) {
    if (ws->stage_bytes >= bytes) return MHD_OK;
    if (ws->d_stage) cudaFree(ws->d_stage);
    ws->d_stage = nullptr;
    ws->stage_bytes = 0;
    if (cudaMalloc(&ws->d_stage, bytes) != cudaSuccess) return fail(MHD_ERR_NOMEM, "staging buffer of %zu bytes", bytes);
    ws->stage_bytes = bytes;
    return MHD_OK;
}

int check_ws_grid(const mhd_workspace* ws, const mhd_grid* g, const char* what) {
    int rc = check_grid(g, what);
    if (rc) return rc;
    if (!ws) return fail(MHD_ERR_STATE, "%s: workspace not initialised", what);
    if (ws->nx != g->nx || ws->ny != g->ny || ws->ng != g->ng || ws->dtype != g->dtype)
        return fail(MHD_ERR_STATE, "%s: workspace not initialised for this grid", what);
    return MHD_OK;
}

mhd::StepParams base_params(const mhd_workspace* ws, const mhd_grid* g, int solver, const int* bc) {
    mhd::StepParams P;
    std::memset(&P, 0, sizeof P);
    P.gamma = ws->gamma;
    P.cr = ws->cr;
    P.dx = ws->dx > 0.0 ? ws->dx : gdx(g);
    P.dy = ws->dy > 0.0 ? ws->dy : gdy(g);
    P.dmin = (P.dy < P.dx) ? P.dy : P.dx;
    P.solver = solver;
    P.limiter = ws->limiter;
    for (int k = 0; k < 4; ++k) P.bc[k] = bc[k];
    P.any_dirichlet = (bc[0] == MHD_BC_DIRICHLET || bc[1] == MHD_BC_DIRICHLET || bc[2] == MHD_BC_DIRICHLET ||
                       bc[3] == MHD_BC_DIRICHLET);
    P.fault = ws->d_fault;
    P.tma_wait_ns = ws->tma_wait_ns;
    return P;
}

cudaError_t launch_step(const mhd_grid* g, const mhd::DevGrid& in, const mhd::DevGrid& tmp, const mhd::DevGrid& out,
                        const mhd::StepParams& P, cudaStream_t st, int yseg, int which = 3,
                        int xrpw = mhd::kDefaultXRpw, int ystage = 0) {
    g_launches += (which == 3) ? 2 : 1;
    return g->dtype == MHD_F64 ? mhd::launch_step_f64(in, tmp, out, P, st, yseg, which, xrpw, ystage)
                               : mhd::launch_step_f32(in, tmp, out, P, st, yseg, which, xrpw, ystage);
}

cudaError_t launch_max(const mhd_workspace* ws, const mhd_grid* g, cudaStream_t st) {
    g_launches += 1;
    return g->dtype == MHD_F64 ? mhd::launch_max_speed_f64(dev(g), ws->gamma, ws->ch, ws->d_max, st, ws->nsm)
                               : mhd::launch_max_speed_f32(dev(g), ws->gamma, ws->ch, ws->d_max, st, ws->nsm);
}

int status_code(int s) {
    switch (s) {
        case mhd::CLK_OK:
        case mhd::CLK_DONE: return MHD_OK;
        case mhd::CLK_NO_SPEED: return MHD_ERR_NO_SPEED;
        case mhd::CLK_BAD_DT: return MHD_ERR_BAD_DT;
        case mhd::CLK_TINY_DT: return MHD_ERR_TINY_DT;
        default: return MHD_ERR_TIMEOUT;
    }
}

}  // namespace

extern "C" {

const char* mhd_last_error(void) { return g_err.c_str(); }
const char* mhd_version(void) { return "mhd_b200 0.1 (sm_100a)"; }
unsigned long long mhd_launch_count(void) { return g_launches.load(); }

int mhd_grid_alloc(mhd_grid* g, int nx, int ny, int ng, int dtype, double x_min, double x_max, double y_min,
                   double y_max) {
    if (!g) return fail(MHD_ERR_ARG, "mhd_grid_alloc: null grid");
    std::memset(g, 0, sizeof *g);
    if (ng < 2 || ng > MHD_MAX_NG || nx < ng || ny < ng) return fail(MHD_ERR_ARG, "mhd_grid_alloc: bad sizes");
    if (dtype != MHD_F64 && dtype != MHD_F32) return fail(MHD_ERR_ARG, "mhd_grid_alloc: bad dtype");
    const size_t eb = elem_bytes(dtype);
    const long long per = 256 / (long long)eb;
    const long long tnx = nx + 2LL * ng, tny = ny + 2LL * ng;
    const long long pitch = (tnx + per - 1) / per * per;
    const long long plane = (pitch * tny + per - 1) / per * per;
    void* p = nullptr;
    if (cudaMalloc(&p, (size_t)(plane * MHD_NV) * eb) != cudaSuccess)
        return fail(MHD_ERR_NOMEM, "mhd_grid_alloc: %lld bytes", (long long)(plane * MHD_NV * eb));
    cudaMemset(p, 0, (size_t)(plane * MHD_NV) * eb);
    g->data = p;
    g->pitch = pitch;
    g->plane = plane;
    g->nx = nx;
    g->ny = ny;
    g->ng = ng;
    g->dtype = dtype;
    g->x_min = x_min;
    g->x_max = x_max;
    g->y_min = y_min;
    g->y_max = y_max;
    return MHD_OK;
}

int mhd_grid_free(mhd_grid* g) {
    if (!g) return MHD_OK;
    if (g->data) CK(cudaFree(g->data));
    g->data = nullptr;
    return MHD_OK;
}

int mhd_grid_swap(mhd_grid* a, mhd_grid* b) {
    if (!a || !b) return fail(MHD_ERR_ARG, "mhd_grid_swap: null grid");
    mhd_grid t = *a;
    *a = *b;
    *b = t;
    return MHD_OK;
}

// Host (dense FP64 SoA) <-> grid on `st`, staging through `stage` for FP32.
static int upload_impl(const mhd_grid* g, const double* host, void* stage, cudaStream_t st) {
    const long long tnx = g->nx + 2LL * g->ng, tny = g->ny + 2LL * g->ng;
    if (g->dtype == MHD_F64) {
        for (int f = 0; f < MHD_NV; ++f)
            CK(cudaMemcpy2DAsync(static_cast<double*>(g->data) + f * g->plane, g->pitch * 8, host + f * tnx * tny,
                                 tnx * 8, tnx * 8, tny, cudaMemcpyHostToDevice, st));
        return MHD_OK;
    }
    CK(cudaMemcpyAsync(stage, host, (size_t)(MHD_NV * tnx * tny) * 8, cudaMemcpyHostToDevice, st));
    mhd::DevGrid s = dev(g);
    s.data = stage;
    s.pitch = tnx;
    s.plane = tnx * tny;
    g_launches += 1;
    CK(mhd::launch_convert_f64_to_f32(s, dev(g), st));
    return MHD_OK;
}

static int download_impl(const mhd_grid* g, double* host, void* stage, cudaStream_t st) {
    const long long tnx = g->nx + 2LL * g->ng, tny = g->ny + 2LL * g->ng;
    if (g->dtype == MHD_F64) {
        for (int f = 0; f < MHD_NV; ++f)
            CK(cudaMemcpy2DAsync(host + f * tnx * tny, tnx * 8, static_cast<const double*>(g->data) + f * g->plane,
                                 g->pitch * 8, tnx * 8, tny, cudaMemcpyDeviceToHost, st));
        return MHD_OK;
    }
    mhd::DevGrid s = dev(g);
    s.data = stage;
    s.pitch = tnx;
    s.plane = tnx * tny;
    g_launches += 1;
    CK(mhd::launch_convert_f32_to_f64(dev(g), s, st));
    CK(cudaMemcpyAsync(host, stage, (size_t)(MHD_NV * tnx * tny) * 8, cudaMemcpyDeviceToHost, st));
    return MHD_OK;
}

int mhd_grid_upload(const mhd_grid* g, const double* host) {
    int rc = check_grid(g, "mhd_grid_upload");
    if (rc) return rc;
    if (!host) return fail(MHD_ERR_ARG, "mhd_grid_upload: null host pointer");
    void* stage = nullptr;
    const size_t n = (size_t)MHD_NV * (g->nx + 2 * g->ng) * (g->ny + 2 * g->ng);
    if (g->dtype == MHD_F32 && cudaMalloc(&stage, n * 8) != cudaSuccess) return fail(MHD_ERR_NOMEM, "staging");
    rc = upload_impl(g, host, stage, nullptr);
    cudaError_t e = cudaStreamSynchronize(nullptr);
    if (stage) cudaFree(stage);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(MHD_ERR_CUDA, "mhd_grid_upload: %s", cudaGetErrorString(e));
    return MHD_OK;
}

int mhd_grid_download(const mhd_grid* g, double* host) {
    int rc = check_grid(g, "mhd_grid_download");
    if (rc) return rc;
    if (!host) return fail(MHD_ERR_ARG, "mhd_grid_download: null host pointer");
    void* stage = nullptr;
    const size_t n = (size_t)MHD_NV * (g->nx + 2 * g->ng) * (g->ny + 2 * g->ng);
    if (g->dtype == MHD_F32 && cudaMalloc(&stage, n * 8) != cudaSuccess) return fail(MHD_ERR_NOMEM, "staging");
    rc = download_impl(g, host, stage, nullptr);
    cudaError_t e = cudaStreamSynchronize(nullptr);
    if (stage) cudaFree(stage);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(MHD_ERR_CUDA, "mhd_grid_download: %s", cudaGetErrorString(e));
    return MHD_OK;
}

int mhd_grid_upload_aos(const mhd_grid* g, const double* host_aos) {
    int rc = check_grid(g, "mhd_grid_upload_aos");
    if (rc) return rc;
    if (!host_aos) return fail(MHD_ERR_ARG, "mhd_grid_upload_aos: null host pointer");
    const size_t n = (size_t)MHD_NV * (g->nx + 2 * g->ng) * (g->ny + 2 * g->ng);
    double* stage = nullptr;
    if (cudaMalloc(&stage, n * 8) != cudaSuccess) return fail(MHD_ERR_NOMEM, "staging");
    cudaError_t e = cudaMemcpy(stage, host_aos, n * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        g_launches += 1;
        e = mhd::launch_aos_to_grid(stage, dev(g), (int)elem_bytes(g->dtype), nullptr);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(nullptr);
    cudaFree(stage);
    if (e != cudaSuccess) return fail(MHD_ERR_CUDA, "mhd_grid_upload_aos: %s", cudaGetErrorString(e));
    return MHD_OK;
}

int mhd_grid_download_aos(const mhd_grid* g, double* host_aos) {
    int rc = check_grid(g, "mhd_grid_download_aos");
    if (rc) return rc;
    if (!host_aos) return fail(MHD_ERR_ARG, "mhd_grid_download_aos: null host pointer");
    const size_t n = (size_t)MHD_NV * (g->nx + 2 * g->ng) * (g->ny + 2 * g->ng);
    double* stage = nullptr;
    if (cudaMalloc(&stage, n * 8) != cudaSuccess) return fail(MHD_ERR_NOMEM, "staging");
    g_launches += 1;
    cudaError_t e = mhd::launch_grid_to_aos(dev(g), (int)elem_bytes(g->dtype), stage, nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(host_aos, stage, n * 8, cudaMemcpyDeviceToHost);
    cudaFree(stage);
    if (e != cudaSuccess) return fail(MHD_ERR_CUDA, "mhd_grid_download_aos: %s", cudaGetErrorString(e));
    return MHD_OK;
}

int mhd_workspace_create(const mhd_grid* g, mhd_workspace** out) {
    if (!out) return fail(MHD_ERR_ARG, "mhd_workspace_create: null output");
    *out = nullptr;
    int rc = check_grid(g, "mhd_workspace_create");
    if (rc) return rc;
    mhd_workspace* ws = new mhd_workspace();
    ws->nx = g->nx;
    ws->ny = g->ny;
    ws->ng = g->ng;
    ws->dtype = g->dtype;
    int dev_id = 0;
    cudaGetDevice(&dev_id);
    cudaDeviceGetAttribute(&ws->nsm, cudaDevAttrMultiProcessorCount, dev_id);
    if (ws->nsm <= 0) ws->nsm = 148;
    if (cudaMalloc(&ws->d_max, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&ws->d_clock, sizeof(mhd::DevClock)) != cudaSuccess ||
        cudaMalloc(&ws->d_fault, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&ws->d_diag, sizeof(double) * (6 * 1024 + 8)) != cudaSuccess) {
        mhd_workspace_destroy(ws);
        return fail(MHD_ERR_NOMEM, "mhd_workspace_create: device scratch");
    }
    cudaMemset(ws->d_clock, 0, sizeof(mhd::DevClock));
    cudaMemset(ws->d_fault, 0, sizeof(int));
    *out = ws;
    return MHD_OK;
}

int mhd_workspace_destroy(mhd_workspace* ws) {
    if (!ws) return MHD_OK;
    if (ws->graph) cudaGraphExecDestroy(ws->graph);
    if (ws->d_max) cudaFree(ws->d_max);
    if (ws->d_clock) cudaFree(ws->d_clock);
    if (ws->d_fault) cudaFree(ws->d_fault);
    if (ws->d_diag) cudaFree(ws->d_diag);
    if (ws->d_stage) cudaFree(ws->d_stage);
    delete ws;
    return MHD_OK;
}

int mhd_workspace_set_stream(mhd_workspace* ws, void* stream) {
    if (!ws) return fail(MHD_ERR_STATE, "mhd_workspace_set_stream: null workspace");
    if (ws->stream != static_cast<cudaStream_t>(stream) && ws->graph) {
        cudaGraphExecDestroy(ws->graph);
        ws->graph = nullptr;
    }
    ws->stream = static_cast<cudaStream_t>(stream);
    return MHD_OK;
}

int mhd_set_gamma(mhd_workspace* ws, double gamma) {
    if (!ws) return fail(MHD_ERR_STATE, "mhd_set_gamma: null workspace");
    if (!(gamma > 1.0)) return fail(MHD_ERR_ARG, "mhd_set_gamma: gamma must exceed 1");
    ws->gamma = gamma;
    return MHD_OK;
}

int mhd_set_ch(mhd_workspace* ws, double ch) {
    if (!ws) return fail(MHD_ERR_STATE, "mhd_set_ch: null workspace");
    if (!(ch >= 0.0)) return fail(MHD_ERR_ARG, "mhd_set_ch: ch must be >= 0");
    ws->ch = ch;
    return MHD_OK;
}

int mhd_get_ch(const mhd_workspace* ws, double* ch) {
    if (!ws || !ch) return fail(MHD_ERR_ARG, "mhd_get_ch: null argument");
    *ch = ws->ch;
    return MHD_OK;
}

int mhd_set_limiter(mhd_workspace* ws, int limiter) {
    if (!ws) return fail(MHD_ERR_STATE, "mhd_set_limiter: null workspace");
    if (limiter != MHD_LIMITER_MINMOD && limiter != MHD_LIMITER_VANLEER) return fail(MHD_ERR_ARG, "bad limiter");
    ws->limiter = limiter;
    return MHD_OK;
}

int mhd_set_cr(mhd_workspace* ws, double cr) {
    if (!ws) return fail(MHD_ERR_STATE, "mhd_set_cr: null workspace");
    if (!(cr > 0.0)) return fail(MHD_ERR_ARG, "mhd_set_cr: cr must be > 0");
    ws->cr = cr;
    return MHD_OK;
}

int mhd_set_sweep_shape(mhd_workspace* ws, int xrpw, int yband, int ystage) {
    if (!ws) return fail(MHD_ERR_STATE, "mhd_set_sweep_shape: null workspace");
    if (xrpw < 0 || xrpw > 64 || yband < 0 || yband > 65536 || ystage < 0 || ystage > 1)
        return fail(MHD_ERR_ARG, "mhd_set_sweep_shape: need 0 <= xrpw <= 64, 0 <= yband <= 65536, ystage 0 or 1");
    ws->xrpw = xrpw;
    ws->yseg = yband;
    ws->ystage = ystage;
    return MHD_OK;
}

int mhd_set_tma_wait_limit(mhd_workspace* ws, unsigned long long ns) {
    if (!ws) return fail(MHD_ERR_STATE, "mhd_set_tma_wait_limit: null workspace");
    ws->tma_wait_ns = ns;
    return MHD_OK;
}

int mhd_set_spacing(mhd_workspace* ws, double dx, double dy) {
    if (!ws) return fail(MHD_ERR_STATE, "mhd_set_spacing: null workspace");
    if (!(dx >= 0.0) || !(dy >= 0.0) || (dx > 0.0) != (dy > 0.0))
        return fail(MHD_ERR_ARG, "mhd_set_spacing: need dx, dy > 0 (or both 0)");
    ws->dx = dx;
    ws->dy = dy;
    return MHD_OK;
}

int mhd_compute_dt(mhd_workspace* ws, const mhd_grid* g, double cfl, double* dt) {
    mhd::NvtxRange nvtx_range("mhd_compute_dt");
    int rc = check_ws_grid(ws, g, "mhd_compute_dt");
    if (rc) return rc;
    if (!dt) return fail(MHD_ERR_ARG, "mhd_compute_dt: null dt");
    CK(cudaMemsetAsync(ws->d_max, 0, sizeof(unsigned long long), ws->stream));
    CK(launch_max(ws, g, ws->stream));
    unsigned long long bits = 0;
    CK(cudaMemcpyAsync(&bits, ws->d_max, sizeof bits, cudaMemcpyDeviceToHost, ws->stream));
    rc = check_fault(ws, "mhd_compute_dt");  // synchronises the stream
    if (rc) return rc;
    double mx;
    std::memcpy(&mx, &bits, sizeof mx);
    if (!(mx > 0.0)) {
        *dt = DBL_MAX;
        return fail(MHD_ERR_NO_SPEED, "mhd_compute_dt: non-positive maximum wave speed");
    }
    ws->ch = mx;
    const double dx = ws->dx > 0.0 ? ws->dx : gdx(g), dy = ws->dy > 0.0 ? ws->dy : gdy(g);
    *dt = cfl * ((dy < dx) ? dy : dx) / mx;
    return MHD_OK;
}

int mhd_advance(mhd_workspace* ws, const mhd_grid* Uold, mhd_grid* Utmp, mhd_grid* Unew, double dt, int solver,
                const int* bc) {
    mhd::NvtxRange nvtx_range("mhd_advance");
    int rc = check_ws_grid(ws, Uold, "mhd_advance(Uold)");
    if (!rc) rc = check_ws_grid(ws, Utmp, "mhd_advance(Utmp)");
    if (!rc) rc = check_ws_grid(ws, Unew, "mhd_advance(Unew)");
    if (!rc) rc = check_bc(bc);
    if (rc) return rc;
    if (solver < MHD_HLL || solver > MHD_FORCE) return fail(MHD_ERR_ARG, "mhd_advance: bad solver %d", solver);
    if (Uold->data == Utmp->data || Uold->data == Unew->data || Utmp->data == Unew->data)
        return fail(MHD_ERR_ARG, "mhd_advance: Uold, Utmp and Unew must be distinct");
    mhd::StepParams P = base_params(ws, Uold, solver, bc);
    P.dt = dt;
    P.ch = ws->ch;
    // psi damping factor on the host with the C library's exp, as the reference
    // does (src/cpu/solver_cpu.cpp:264, src/gpu/solver_gpu.cu:686).
    P.damp = std::exp(-dt * ws->ch / ws->cr);
    if (P.damp >= 1.0) P.damp = 1.0;
    P.t_end = 0.0;
    P.cfl = 0.0;
    CK(launch_step(Uold, dev(Uold), dev(Utmp), dev(Unew), P, ws->stream, ws->yseg, 3, ws->xrpw, ws->ystage));
    return MHD_OK;
}

int mhd_sweep(mhd_workspace* ws, const mhd_grid* in, mhd_grid* out, double dt, int solver, const int* bc, int dir) {
    mhd::NvtxRange nvtx_range("mhd_sweep");
    int rc = check_ws_grid(ws, in, "mhd_sweep(in)");
    if (!rc) rc = check_ws_grid(ws, out, "mhd_sweep(out)");
    if (!rc) rc = check_bc(bc);
    if (rc) return rc;
    if (solver < MHD_HLL || solver > MHD_FORCE) return fail(MHD_ERR_ARG, "mhd_sweep: bad solver %d", solver);
    if (dir != 0 && dir != 1) return fail(MHD_ERR_ARG, "mhd_sweep: dir must be 0 (x) or 1 (y)");
    if (in->data == out->data) return fail(MHD_ERR_ARG, "mhd_sweep: in and out must be distinct");
    mhd::StepParams P = base_params(ws, in, solver, bc);
    P.dt = dt;
    P.ch = ws->ch;
    P.damp = std::exp(-dt * ws->ch / ws->cr);  // as mhd_advance
    if (P.damp >= 1.0) P.damp = 1.0;
    P.t_end = 0.0;
    P.cfl = 0.0;
    if (dir == 0) CK(launch_step(in, dev(in), dev(out), dev(out), P, ws->stream, ws->yseg, 1, ws->xrpw, ws->ystage));
    else CK(launch_step(in, dev(in), dev(in), dev(out), P, ws->stream, ws->yseg, 2, ws->xrpw, ws->ystage));
    return MHD_OK;
}

int mhd_max_speed(mhd_workspace* ws, const mhd_grid* g, double* vmax) {
    int rc = check_ws_grid(ws, g, "mhd_max_speed");
    if (rc) return rc;
    if (!vmax) return fail(MHD_ERR_ARG, "mhd_max_speed: null output");
    CK(cudaMemsetAsync(ws->d_max, 0, sizeof(unsigned long long), ws->stream));
    CK(launch_max(ws, g, ws->stream));
    unsigned long long bits = 0;
    CK(cudaMemcpyAsync(&bits, ws->d_max, sizeof bits, cudaMemcpyDeviceToHost, ws->stream));
    rc = check_fault(ws, "mhd_max_speed");  // synchronises the stream
    if (rc) return rc;
    std::memcpy(vmax, &bits, sizeof *vmax);
    if (!(*vmax > 0.0)) return fail(MHD_ERR_NO_SPEED, "mhd_max_speed: non-positive maximum wave speed");
    return MHD_OK;
}

int mhd_grid_copy_rows(const mhd_grid* src, int src_row, mhd_grid* dst, int dst_row, int nrows, void* stream) {
    int rc = check_grid(src, "mhd_grid_copy_rows(src)");
    if (!rc) rc = check_grid(dst, "mhd_grid_copy_rows(dst)");
    if (rc) return rc;
    if (src->nx != dst->nx || src->ng != dst->ng || src->dtype != dst->dtype || src->pitch != dst->pitch)
        return fail(MHD_ERR_ARG, "mhd_grid_copy_rows: grids differ in nx, ng, dtype or pitch");
    const int sty = src->ny + 2 * src->ng, dty = dst->ny + 2 * dst->ng;
    if (nrows < 0 || src_row < 0 || dst_row < 0 || src_row + nrows > sty || dst_row + nrows > dty)
        return fail(MHD_ERR_ARG, "mhd_grid_copy_rows: rows out of range");
    if (nrows == 0) return MHD_OK;
    const size_t e = elem_bytes(src->dtype);
    const size_t bytes = (size_t)nrows * (size_t)src->pitch * e;  // the rows of one field are contiguous
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // one strided copy: 9 blocks (one per field), a plane apart in each grid
    const char* s = static_cast<const char*>(src->data) + (size_t)src_row * src->pitch * e;
    char* d = static_cast<char*>(dst->data) + (size_t)dst_row * dst->pitch * e;
    CK(cudaMemcpy2DAsync(d, (size_t)dst->plane * e, s, (size_t)src->plane * e, bytes, MHD_NV,
                         cudaMemcpyDeviceToDevice, st));
    return MHD_OK;
}

int mhd_riemann_flux_device(mhd_workspace* ws, int dtype, long long n, const double* UL, const double* UR, int dir,
                            int solver, double ch, double gamma, double* F) {
    if (dtype != MHD_F64 && dtype != MHD_F32) return fail(MHD_ERR_ARG, "mhd_riemann_flux_device: bad dtype %d", dtype);
    if (n < 0 || (n > 0 && (!UL || !UR || !F))) return fail(MHD_ERR_ARG, "mhd_riemann_flux_device: bad arrays");
    if (dir != 0 && dir != 1) return fail(MHD_ERR_ARG, "mhd_riemann_flux_device: dir must be 0 (x) or 1 (y)");
    if (solver < MHD_HLL || solver > MHD_FORCE) return fail(MHD_ERR_ARG, "mhd_riemann_flux_device: bad solver %d", solver);
    if (n == 0) return MHD_OK;
    cudaStream_t st = ws ? ws->stream : nullptr;
    g_launches += 1;
    CK(dtype == MHD_F64 ? mhd::launch_faces_f64(UL, UR, n, dir, solver, ch, gamma, F, st)
                        : mhd::launch_faces_f32(UL, UR, n, dir, solver, ch, gamma, F, st));
    if (!ws) CK(cudaStreamSynchronize(nullptr));
    return MHD_OK;
}

int mhd_apply_boundary(mhd_workspace* ws, mhd_grid* g, const int* bc) {
    int rc = check_grid(g, "mhd_apply_boundary");
    if (!rc) rc = check_bc(bc);
    if (rc) return rc;
    cudaStream_t st = ws ? ws->stream : nullptr;
    g_launches += 1;
    CK(mhd::launch_apply_boundary(dev(g), (int)elem_bytes(g->dtype), bc, st));
    if (!ws) CK(cudaStreamSynchronize(nullptr));
    return MHD_OK;
}

// Validation and device-clock start shared by mhd_run and mhd_profile_sweeps:
// the initial CFL maximum (floored by the current ch) goes to clock slot 0.
static int start_device_loop(mhd_workspace* ws, mhd_grid* U, mhd_grid* T, double cfl, double t_end, int solver,
                             const int* bc, const char* what, mhd::StepParams* P) {
    int rc = check_ws_grid(ws, U, what);
    if (!rc) rc = check_ws_grid(ws, T, what);
    if (!rc) rc = check_bc(bc);
    if (rc) return rc;
    if (solver < MHD_HLL || solver > MHD_FORCE) return fail(MHD_ERR_ARG, "%s: bad solver %d", what, solver);
    if (U->data == T->data) return fail(MHD_ERR_ARG, "%s: U and T must be distinct", what);
    if (!(t_end > 0.0) || !std::isfinite(t_end) || !(cfl > 0.0))
        return fail(MHD_ERR_ARG, "%s: need finite t_end > 0 and cfl > 0", what);
    CK(cudaMemsetAsync(ws->d_max, 0, sizeof(unsigned long long), ws->stream));
    CK(launch_max(ws, U, ws->stream));
    g_launches += 1;
    CK(mhd::launch_clock_init(ws->d_clock, ws->d_max, ws->stream));
    *P = base_params(ws, U, solver, bc);
    P->cfl = cfl;
    P->t_end = t_end;
    P->clock = ws->d_clock;
    P->accumulate = 1;
    return MHD_OK;
}

int mhd_clock_start(mhd_workspace* ws, const mhd_grid* U, double cfl, double t_end) {
    int rc = check_ws_grid(ws, U, "mhd_clock_start");
    if (rc) return rc;
    if (!(t_end > 0.0) || !std::isfinite(t_end) || !(cfl > 0.0))
        return fail(MHD_ERR_ARG, "mhd_clock_start: need finite t_end > 0 and cfl > 0");
    CK(cudaMemsetAsync(ws->d_max, 0, sizeof(unsigned long long), ws->stream));
    CK(launch_max(ws, U, ws->stream));
    g_launches += 1;
    CK(mhd::launch_clock_init(ws->d_clock, ws->d_max, ws->stream));
    ws->clk_cfl = cfl;
    ws->clk_t_end = t_end;
    ws->clk_started = 1;
    return MHD_OK;
}

int mhd_clock_slot(mhd_workspace* ws, int parity, void** dptr) {
    if (!ws || !ws->d_clock) return fail(MHD_ERR_STATE, "mhd_clock_slot: null workspace");
    if (!dptr || (parity != 0 && parity != 1)) return fail(MHD_ERR_ARG, "mhd_clock_slot: need parity 0 or 1");
    *dptr = &ws->d_clock->maxbits[parity];
    return MHD_OK;
}

int mhd_sweep_clocked(mhd_workspace* ws, const mhd_grid* in, mhd_grid* out, int solver, const int* bc, int dir,
                      int parity, int row0, int nrows, int flags) {
    mhd::NvtxRange nvtx_range("mhd_sweep_clocked");
    int rc = check_ws_grid(ws, in, "mhd_sweep_clocked(in)");
    if (!rc) rc = check_ws_grid(ws, out, "mhd_sweep_clocked(out)");
    if (!rc) rc = check_bc(bc);
    if (rc) return rc;
    if (!ws->clk_started) return fail(MHD_ERR_STATE, "mhd_sweep_clocked: no clock (call mhd_clock_start)");
    if (solver < MHD_HLL || solver > MHD_FORCE) return fail(MHD_ERR_ARG, "mhd_sweep_clocked: bad solver %d", solver);
    if ((dir != 0 && dir != 1) || (parity != 0 && parity != 1))
        return fail(MHD_ERR_ARG, "mhd_sweep_clocked: dir and parity must be 0 or 1");
    if (in->data == out->data) return fail(MHD_ERR_ARG, "mhd_sweep_clocked: in and out must be distinct");
    if (row0 < 0 || nrows < 0 || row0 + nrows > in->ny || (nrows == 0 && row0 != 0) || (dir == 0 && nrows != 0))
        return fail(MHD_ERR_ARG, "mhd_sweep_clocked: bad row window %d + %d (y-sweeps only)", row0, nrows);
    if (flags & ~(MHD_SWEEP_NO_GATHER | MHD_SWEEP_NO_ADVANCE))
        return fail(MHD_ERR_ARG, "mhd_sweep_clocked: unknown flags %d", flags);
    mhd::StepParams P = base_params(ws, in, solver, bc);
    P.cfl = ws->clk_cfl;
    P.t_end = ws->clk_t_end;
    P.clock = ws->d_clock;
    P.accumulate = 1;
    P.parity = parity;
    P.row0 = row0;
    P.nrows = nrows;
    P.no_gather = (flags & MHD_SWEEP_NO_GATHER) ? 1 : 0;
    P.no_advance = (flags & MHD_SWEEP_NO_ADVANCE) ? 1 : 0;
    if (dir == 0) CK(launch_step(in, dev(in), dev(out), dev(out), P, ws->stream, ws->yseg, 1, ws->xrpw, ws->ystage));
    else CK(launch_step(in, dev(in), dev(in), dev(out), P, ws->stream, ws->yseg, 2, ws->xrpw, ws->ystage));
    return MHD_OK;
}

int mhd_clock_read(mhd_workspace* ws, mhd_run_info* info) {
    if (!ws || !ws->d_clock) return fail(MHD_ERR_STATE, "mhd_clock_read: null workspace");
    mhd::DevClock hc;
    CK(cudaMemcpyAsync(&hc, ws->d_clock, sizeof hc, cudaMemcpyDeviceToHost, ws->stream));
    CK(cudaStreamSynchronize(ws->stream));
    if (hc.steps > 0) ws->ch = hc.last_ch;
    if (info) {
        info->t = hc.t[hc.steps & 1];
        info->last_dt = hc.last_dt;
        info->ch = ws->ch;
        info->steps = hc.steps;
        info->status = status_code(hc.status);
        info->fallbacks = hc.flux_fallbacks;
        info->pad_ = 0;
    }
    return check_fault(ws, "mhd_clock_read");
}

int mhd_profile_sweeps(mhd_workspace* ws, mhd_grid* U, mhd_grid* T, double cfl, double t_end, int solver,
                       const int* bc, int nrep, float* ms_out) {
    mhd::NvtxRange nvtx_range("mhd_profile_sweeps");
    if (nrep < 1 || !ms_out) return fail(MHD_ERR_ARG, "mhd_profile_sweeps: need nrep >= 1 and an output");
    mhd::StepParams P;
    int rc = start_device_loop(ws, U, T, cfl, t_end, solver, bc, "mhd_profile_sweeps", &P);
    if (rc) return rc;
    cudaStream_t st = ws->stream;
    cudaEvent_t ev[3];
    for (auto& e : ev) CK(cudaEventCreate(&e));
    const mhd::DevGrid dU = dev(U), dT = dev(T);
    float sx = 0.f, sy = 0.f;
    cudaError_t e = cudaSuccess;
    for (int r = 0; r < nrep && e == cudaSuccess; ++r) {
        mhd::StepParams Q = P;
        Q.parity = r & 1;
        cudaEventRecord(ev[0], st);
        e = launch_step(U, dU, dT, dU, Q, st, ws->yseg, 1, ws->xrpw, ws->ystage);
        cudaEventRecord(ev[1], st);
        if (e == cudaSuccess) e = launch_step(U, dU, dT, dU, Q, st, ws->yseg, 2, ws->xrpw, ws->ystage);
        cudaEventRecord(ev[2], st);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[2]);
        float a = 0.f, b = 0.f;
        cudaEventElapsedTime(&a, ev[0], ev[1]);
        cudaEventElapsedTime(&b, ev[1], ev[2]);
        sx += a;
        sy += b;
    }
    for (auto& x : ev) cudaEventDestroy(x);
    if (e != cudaSuccess) return fail(MHD_ERR_CUDA, "mhd_profile_sweeps: %s", cudaGetErrorString(e));
    ms_out[0] = sx / nrep;
    ms_out[1] = sy / nrep;
    return check_fault(ws, "mhd_profile_sweeps");
}

int mhd_run(mhd_workspace* ws, mhd_grid* U, mhd_grid* T, double cfl, double t_end, int max_steps, int solver,
            const int* bc, mhd_run_info* info) {
    mhd::NvtxRange nvtx_range("mhd_run");
    mhd::StepParams P;
    int rc = start_device_loop(ws, U, T, cfl, t_end, solver, bc, "mhd_run", &P);
    if (rc) return rc;
    cudaStream_t st = ws->stream;

    mhd_workspace::Key key{};
    key.u = U->data; key.t = T->data; key.solver = solver; key.limiter = ws->limiter;
    for (int k = 0; k < 4; ++k) key.bc[k] = bc[k];
    key.yseg = ws->yseg; key.xrpw = ws->xrpw; key.ystage = ws->ystage; key.gamma = ws->gamma; key.cr = ws->cr; key.cfl = cfl; key.t_end = t_end;
    const mhd::DevGrid dU = dev(U), dT = dev(T);
    if (!ws->graph || !(ws->key == key)) {
        if (ws->graph) { cudaGraphExecDestroy(ws->graph); ws->graph = nullptr; }
        cudaStream_t cap = st;
        bool own = false;
        if (cap == nullptr) {  // the legacy stream cannot be captured
            CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            own = true;
        }
        cudaGraph_t gr = nullptr;
        // one-time kernel attribute setup happens outside the capture
        CK(launch_step(U, dU, dT, dU, P, cap, ws->yseg, 0, ws->xrpw, ws->ystage));
        CK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        cudaError_t e1 = cudaSuccess, e2 = cudaSuccess;
        for (int par = 0; par < 2 && e1 == cudaSuccess; ++par) {
            mhd::StepParams Q = P;
            Q.parity = par;
            e1 = (U->dtype == MHD_F64) ? mhd::launch_step_f64(dU, dT, dU, Q, cap, ws->yseg, 3, ws->xrpw, ws->ystage)
                                       : mhd::launch_step_f32(dU, dT, dU, Q, cap, ws->yseg, 3, ws->xrpw, ws->ystage);
        }
        e2 = cudaStreamEndCapture(cap, &gr);
        if (own) cudaStreamDestroy(cap);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            if (gr) cudaGraphDestroy(gr);
            return fail(MHD_ERR_CUDA, "mhd_run: capture failed: %s", cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
        }
        cudaError_t e3 = cudaGraphInstantiate(&ws->graph, gr, 0);
        cudaGraphDestroy(gr);
        if (e3 != cudaSuccess) { ws->graph = nullptr; return fail(MHD_ERR_CUDA, "mhd_run: instantiate: %s", cudaGetErrorString(e3)); }
        ws->key = key;
    }

    mhd::DevClock hc;
    std::memset(&hc, 0, sizeof hc);
    if (max_steps > 0) {
        for (int p = 0; p < max_steps / 2; ++p) {
            g_launches += 4;
            CK(cudaGraphLaunch(ws->graph, st));
        }
        if (max_steps & 1) {
            mhd::StepParams Q = P;
            Q.parity = 0;
            CK(launch_step(U, dU, dT, dU, Q, st, ws->yseg, 3, ws->xrpw, ws->ystage));
        }
        CK(cudaMemcpyAsync(&hc, ws->d_clock, sizeof hc, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    } else {
        const int chunk = 32;  // graph launches (64 steps) between host checks
        for (;;) {
            for (int p = 0; p < chunk; ++p) {
                g_launches += 4;
                CK(cudaGraphLaunch(ws->graph, st));
            }
            CK(cudaMemcpyAsync(&hc, ws->d_clock, sizeof hc, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (hc.status != mhd::CLK_OK) break;
        }
    }
    if (hc.steps > 0) ws->ch = hc.last_ch;
    if (info) {
        info->t = hc.t[hc.steps & 1];
        info->last_dt = hc.last_dt;
        info->ch = ws->ch;
        info->steps = hc.steps;
        info->status = status_code(hc.status);
        info->fallbacks = hc.flux_fallbacks;
        info->pad_ = 0;
    }
    const int frc = check_fault(ws, "mhd_run");
    if (frc) return frc;
    const int code = status_code(hc.status);
    if (code != MHD_OK) return fail(code, "mhd_run: step loop stopped with status %d after %d steps", hc.status, hc.steps);
    return MHD_OK;
}

int mhd_upload(mhd_workspace* ws, const mhd_grid* g, const double* host) {
    int rc = check_ws_grid(ws, g, "mhd_upload");
    if (rc) return rc;
    if (!host) return fail(MHD_ERR_ARG, "mhd_upload: null host pointer");
    if (g->dtype == MHD_F32) {
        rc = ensure_stage(ws, (size_t)MHD_NV * (g->nx + 2 * g->ng) * (g->ny + 2 * g->ng) * 8);
        if (rc) return rc;
    }
    return upload_impl(g, host, ws->d_stage, ws->stream);
}

// FP32 host arrays for FP32 grids: one pitched copy per field, no staging.
static int copy_f32(mhd_workspace* ws, const mhd_grid* g, float* host, bool up, const char* what) {
    int rc = check_ws_grid(ws, g, what);
    if (rc) return rc;
    if (!host) return fail(MHD_ERR_ARG, "%s: null host pointer", what);
    if (g->dtype != MHD_F32) return fail(MHD_ERR_ARG, "%s: the grid is not FP32", what);
    const long long tnx = g->nx + 2LL * g->ng, tny = g->ny + 2LL * g->ng;
    for (int f = 0; f < MHD_NV; ++f) {
        float* d = static_cast<float*>(g->data) + f * g->plane;
        float* h = host + f * tnx * tny;
        if (up) CK(cudaMemcpy2DAsync(d, g->pitch * 4, h, tnx * 4, tnx * 4, tny, cudaMemcpyHostToDevice, ws->stream));
        else CK(cudaMemcpy2DAsync(h, tnx * 4, d, g->pitch * 4, tnx * 4, tny, cudaMemcpyDeviceToHost, ws->stream));
    }
    return MHD_OK;
}

int mhd_upload_f32(mhd_workspace* ws, const mhd_grid* g, const float* host) {
    return copy_f32(ws, g, const_cast<float*>(host), true, "mhd_upload_f32");
}

int mhd_download_f32(mhd_workspace* ws, const mhd_grid* g, float* host) {
    return copy_f32(ws, g, host, false, "mhd_download_f32");
}

int mhd_download(mhd_workspace* ws, const mhd_grid* g, double* host) {
    int rc = check_ws_grid(ws, g, "mhd_download");
    if (rc) return rc;
    if (!host) return fail(MHD_ERR_ARG, "mhd_download: null host pointer");
    if (g->dtype == MHD_F32) {
        rc = ensure_stage(ws, (size_t)MHD_NV * (g->nx + 2 * g->ng) * (g->ny + 2 * g->ng) * 8);
        if (rc) return rc;
    }
    return download_impl(g, host, ws->d_stage, ws->stream);
}

int mhd_initialise_device(mhd_workspace* ws, const mhd_grid* g, int case_id) {
    int rc = check_grid(g, "mhd_initialise_device");
    if (rc) return rc;
    if (case_id < MHD_CASE_KELVIN_HELMHOLTZ || case_id > MHD_CASE_BRIO_WU_CFL08)
        return fail(MHD_ERR_ARG, "mhd_initialise_device: unknown case %d", case_id);
    cudaStream_t st = ws ? ws->stream : nullptr;
    g_launches += 1;
    CK(mhd::launch_initialise(dev(g), (int)elem_bytes(g->dtype), case_id, g->x_min, g->y_min, gdx(g), gdy(g), st));
    if (!ws) CK(cudaStreamSynchronize(nullptr));
    return MHD_OK;
}

int mhd_initialise_orszag_tang(mhd_workspace* ws, const mhd_grid* g, double b0, double gamma, const double* amp) {
    int rc = check_grid(g, "mhd_initialise_orszag_tang");
    if (rc) return rc;
    if (!(gamma > 1.0)) return fail(MHD_ERR_ARG, "mhd_initialise_orszag_tang: gamma must exceed 1");
    cudaStream_t st = ws ? ws->stream : nullptr;
    g_launches += 1;
    CK(mhd::launch_initialise_ot(dev(g), (int)elem_bytes(g->dtype), b0, gamma, amp, g->x_min, g->y_min, gdx(g),
                                 gdy(g), st));
    if (!ws) CK(cudaStreamSynchronize(nullptr));
    return MHD_OK;
}

int mhd_synchronize(mhd_workspace* ws) {
    if (!ws) return fail(MHD_ERR_STATE, "mhd_synchronize: null workspace");
    CK(cudaStreamSynchronize(ws->stream));
    return check_fault(ws, "mhd_synchronize");
}

int mhd_diagnostics(mhd_workspace* ws, const mhd_grid* g, double* out6) {
    int rc = check_ws_grid(ws, g, "mhd_diagnostics");
    if (rc) return rc;
    if (!out6) return fail(MHD_ERR_ARG, "mhd_diagnostics: null output");
    g_launches += 2;
    CK(mhd::launch_diagnostics(dev(g), (int)elem_bytes(g->dtype), ws->gamma, gdx(g), gdy(g), ws->d_diag,
                               ws->d_diag + 6 * 1024, ws->stream));
    CK(cudaMemcpyAsync(out6, ws->d_diag + 6 * 1024, 6 * sizeof(double), cudaMemcpyDeviceToHost, ws->stream));
    CK(cudaStreamSynchronize(ws->stream));
    return MHD_OK;
}

}  // extern "C"
