// batch_api.cu -- C ABI of the batched engine (mhd_batch_*) and its autotuner.
//
// A batch owns, per instance, the state U and the x-swept state T (padded slabs
// as mhd_grid_alloc makes them), a device clock, and one shared instance table
// and work list (batch.cuh).  mhd_batch_run starts every clock from the CFL
// maximum of its instance and replays a CUDA graph of two steps (four
// persistent launches) until max_steps steps or every instance's t_end.
//
// Autotuner (mhd_batch_tune): the x-sweep phase maps U -> T and the y-sweep
// phase maps T -> U without touching the clock slots they read, so each phase
// can be launched repeatedly on unchanged input.  The tuner times every x
// candidate (rows per warp x persistent CTAs) and then every y candidate
// (segment length x persistent CTAs) with CUDA events, keeping the fastest of
// each.  The instances end one step ahead of where they started.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mhd_b200.h"
#include "batch.cuh"
#include "launch.h"

namespace mhd {
int report_error(int code, const char* msg);
}

namespace {

int berr(int code, const char* msg) { return mhd::report_error(code, msg); }

#define BCK(call)                                                             \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) return berr(MHD_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)

__global__ void batch_clock_init(mhd::DevClock* c, const unsigned long long* mx, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    mhd::DevClock z{};
    z.maxbits[0] = mx[i];
    c[i] = z;
}

}  // namespace

struct mhd_batch {
    int n = 0, dtype = MHD_F32, solver = MHD_HLLD, limiter = MHD_LIMITER_VANLEER, nsm = 148;
    std::vector<mhd_instance_desc> desc;
    std::vector<mhd_grid> U, T;
    std::vector<double> ch;  // per-instance c_h carried between runs (floor of the next CFL maximum)
    std::vector<mhd::BatchInst> host_inst;
    std::vector<int> first;  // x prefix (n + 1) then y prefix (n + 1)
    mhd::BatchInst* d_inst = nullptr;
    int* d_first = nullptr;
    mhd::DevClock* d_clock = nullptr;
    unsigned long long* d_max = nullptr;
    cudaStream_t stream = nullptr;
    mhd_batch_tuning tune{mhd::kDefaultBatchXRpw, mhd::kDefaultYSeg, 0, 0};
    cudaGraphExec_t graph = nullptr;
    mhd_batch_tuning graph_tune{};
    long long cells = 0;
};

namespace {

// Candidate launch shapes the autotuner times (mhd_batch_tune), exported by
// mhd_batch_tune_candidates.
const int kTuneXrpw[] = {2, 4, 8, 16};             // x-sweep rows per warp
const int kTuneYseg[] = {16, 24, 32, 48, 64, 128};  // y-sweep segment rows
const int kTuneCtasPerSm[] = {2, 3, 4};             // persistent CTAs per SM, both phases

cudaError_t phase(mhd_batch* b, int parity, int which, const mhd_batch_tuning& t, cudaStream_t st) {
    const int ctas = which == 1 ? t.ctas_x : t.ctas_y;
    return b->dtype == MHD_F64 ? mhd::launch_batch_f64(b->d_inst, b->d_first, b->n, parity, which, b->solver,
                                                       b->limiter, t.xrpw, t.yseg, ctas, st)
                               : mhd::launch_batch_f32(b->d_inst, b->d_first, b->n, parity, which, b->solver,
                                                       b->limiter, t.xrpw, t.yseg, ctas, st);
}

// Work decomposition for the current tuning; uploads the table and prefixes.
int build_worklist(mhd_batch* b) {
    b->first.assign(2 * (b->n + 1), 0);
    for (int i = 0; i < b->n; ++i) {
        mhd::BatchInst& I = b->host_inst[i];
        const int len = mhd::x_seg_len(4 * b->tune.xrpw);
        I.x_segs = (b->desc[i].nx + len - 1) / len;
        I.x_pad_ = 0;
        I.y_strips = (b->desc[i].nx + b->desc[i].ng + 31) / 32;  // strips holding interior columns
        I.y_bands = (b->desc[i].ny + b->tune.yseg - 1) / b->tune.yseg;
        I.y_units = (I.y_strips * I.y_bands + mhd::YS_WARPS - 1) / mhd::YS_WARPS;
        I.pad_ = 0;
        b->first[i + 1] = b->first[i] + (int)(((long long)I.x_segs * b->desc[i].ny + mhd::BX_WARPS - 1) / mhd::BX_WARPS);
        b->first[b->n + 1 + i + 1] = b->first[b->n + 1 + i] + I.y_units;
    }
    BCK(cudaMemcpyAsync(b->d_inst, b->host_inst.data(), sizeof(mhd::BatchInst) * b->n, cudaMemcpyHostToDevice,
                        b->stream));
    BCK(cudaMemcpyAsync(b->d_first, b->first.data(), sizeof(int) * b->first.size(), cudaMemcpyHostToDevice,
                        b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return MHD_OK;
}

// Every clock from its instance's CFL maximum (floored by the carried c_h).
int start_clocks(mhd_batch* b) {
    BCK(cudaMemsetAsync(b->d_max, 0, sizeof(unsigned long long) * b->n, b->stream));
    for (int i = 0; i < b->n; ++i) {
        mhd::DevGrid g{b->U[i].data, b->U[i].pitch, b->U[i].plane, b->U[i].nx, b->U[i].ny, b->U[i].ng, 0};
        const cudaError_t e =
            b->dtype == MHD_F64 ? mhd::launch_max_speed_f64(g, b->desc[i].gamma, b->ch[i], b->d_max + i, b->stream, b->nsm)
                                : mhd::launch_max_speed_f32(g, b->desc[i].gamma, b->ch[i], b->d_max + i, b->stream, b->nsm);
        BCK(e);
    }
    batch_clock_init<<<(b->n + 127) / 128, 128, 0, b->stream>>>(b->d_clock, b->d_max, b->n);
    BCK(cudaGetLastError());
    return MHD_OK;
}

void default_ctas(mhd_batch* b) {
    if (b->tune.ctas_x <= 0) b->tune.ctas_x = 3 * b->nsm;
    if (b->tune.ctas_y <= 0) b->tune.ctas_y = 3 * b->nsm;
}

}  // namespace

extern "C" {

int mhd_batch_create(const mhd_instance_desc* desc, int n, int dtype, int solver, int limiter, mhd_batch** out) {
    if (!out || !desc || n < 1) return berr(MHD_ERR_ARG, "mhd_batch_create: need n >= 1 descriptors and an output");
    *out = nullptr;
    if (dtype != MHD_F64 && dtype != MHD_F32) return berr(MHD_ERR_ARG, "mhd_batch_create: bad dtype");
    if (solver < MHD_HLL || solver > MHD_FORCE) return berr(MHD_ERR_ARG, "mhd_batch_create: bad solver");
    if (limiter != MHD_LIMITER_MINMOD && limiter != MHD_LIMITER_VANLEER)
        return berr(MHD_ERR_ARG, "mhd_batch_create: bad limiter");
    for (int i = 0; i < n; ++i) {
        const mhd_instance_desc& d = desc[i];
        if (d.ng < 2 || d.ng > MHD_MAX_NG || d.nx < d.ng || d.ny < d.ng || !(d.gamma > 1.0) || !(d.cfl > 0.0) ||
            !(d.cr > 0.0) || !(d.t_end > 0.0) || !std::isfinite(d.t_end) || !(d.x_max > d.x_min) ||
            !(d.y_max > d.y_min))
            return berr(MHD_ERR_ARG, "mhd_batch_create: invalid instance descriptor");
        for (int k = 0; k < 4; ++k)
            if (d.bc[k] < MHD_BC_PERIODIC || d.bc[k] > MHD_BC_REFLECTING)
                return berr(MHD_ERR_ARG, "mhd_batch_create: boundary types are periodic, transmissive or reflecting");
    }
    mhd_batch* b = new mhd_batch();
    b->n = n;
    b->dtype = dtype;
    b->solver = solver;
    b->limiter = limiter;
    b->desc.assign(desc, desc + n);
    b->U.assign(n, mhd_grid{});
    b->T.assign(n, mhd_grid{});
    b->ch.assign(n, 0.0);
    b->host_inst.assign(n, mhd::BatchInst{});
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, dev);
    if (b->nsm <= 0) b->nsm = 148;
    default_ctas(b);
    int rc = MHD_OK;
    for (int i = 0; i < n && rc == MHD_OK; ++i) {
        const mhd_instance_desc& d = desc[i];
        rc = mhd_grid_alloc(&b->U[i], d.nx, d.ny, d.ng, dtype, d.x_min, d.x_max, d.y_min, d.y_max);
        if (!rc) rc = mhd_grid_alloc(&b->T[i], d.nx, d.ny, d.ng, dtype, d.x_min, d.x_max, d.y_min, d.y_max);
        b->cells += (long long)d.nx * d.ny;
    }
    if (!rc && (cudaMalloc(&b->d_inst, sizeof(mhd::BatchInst) * n) != cudaSuccess ||
                cudaMalloc(&b->d_first, sizeof(int) * 2 * (n + 1)) != cudaSuccess ||
                cudaMalloc(&b->d_clock, sizeof(mhd::DevClock) * n) != cudaSuccess ||
                cudaMalloc(&b->d_max, sizeof(unsigned long long) * n) != cudaSuccess))
        rc = berr(MHD_ERR_NOMEM, "mhd_batch_create: device tables");
    if (rc) {
        mhd_batch_destroy(b);
        return rc;
    }
    for (int i = 0; i < n; ++i) {
        const mhd_instance_desc& d = desc[i];
        mhd::BatchInst& I = b->host_inst[i];
        I.U = mhd::DevGrid{b->U[i].data, b->U[i].pitch, b->U[i].plane, d.nx, d.ny, d.ng, 0};
        I.T = mhd::DevGrid{b->T[i].data, b->T[i].pitch, b->T[i].plane, d.nx, d.ny, d.ng, 0};
        mhd::StepParams& P = I.P;
        std::memset(&P, 0, sizeof P);
        P.gamma = d.gamma;
        P.cr = d.cr;
        P.cfl = d.cfl;
        P.dx = (d.x_max - d.x_min) / d.nx;
        P.dy = (d.y_max - d.y_min) / d.ny;
        P.dmin = (P.dy < P.dx) ? P.dy : P.dx;
        P.t_end = d.t_end;
        P.clock = b->d_clock + i;
        P.solver = solver;
        P.limiter = limiter;
        for (int k = 0; k < 4; ++k) P.bc[k] = d.bc[k];
        P.any_dirichlet = 0;
        P.accumulate = 1;
    }
    rc = build_worklist(b);
    if (rc) {
        mhd_batch_destroy(b);
        return rc;
    }
    *out = b;
    return MHD_OK;
}

int mhd_batch_destroy(mhd_batch* b) {
    if (!b) return MHD_OK;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (auto& g : b->U) mhd_grid_free(&g);
    for (auto& g : b->T) mhd_grid_free(&g);
    if (b->d_inst) cudaFree(b->d_inst);
    if (b->d_first) cudaFree(b->d_first);
    if (b->d_clock) cudaFree(b->d_clock);
    if (b->d_max) cudaFree(b->d_max);
    delete b;
    return MHD_OK;
}

int mhd_batch_set_stream(mhd_batch* b, void* stream) {
    if (!b) return berr(MHD_ERR_STATE, "mhd_batch_set_stream: null batch");
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    b->stream = static_cast<cudaStream_t>(stream);
    return MHD_OK;
}

int mhd_batch_grid(const mhd_batch* b, int i, mhd_grid* out) {
    if (!b || !out || i < 0 || i >= b->n) return berr(MHD_ERR_ARG, "mhd_batch_grid: bad instance");
    *out = b->U[i];
    return MHD_OK;
}

int mhd_batch_cells(const mhd_batch* b, long long* cells) {
    if (!b || !cells) return berr(MHD_ERR_ARG, "mhd_batch_cells: null argument");
    *cells = b->cells;
    return MHD_OK;
}

int mhd_batch_get_tuning(const mhd_batch* b, mhd_batch_tuning* t) {
    if (!b || !t) return berr(MHD_ERR_ARG, "mhd_batch_get_tuning: null argument");
    *t = b->tune;
    return MHD_OK;
}

int mhd_batch_set_tuning(mhd_batch* b, const mhd_batch_tuning* t) {
    if (!b || !t) return berr(MHD_ERR_ARG, "mhd_batch_set_tuning: null argument");
    if (t->xrpw < 1 || t->xrpw > 64 || t->yseg < 4 || t->yseg > 4096 || t->ctas_x < 0 || t->ctas_y < 0)
        return berr(MHD_ERR_ARG, "mhd_batch_set_tuning: out of range");
    b->tune = *t;
    default_ctas(b);
    return build_worklist(b);
}

int mhd_batch_run(mhd_batch* b, int max_steps, mhd_run_info* info) {
    mhd::NvtxRange nvtx_range("mhd_batch_run");
    if (!b) return berr(MHD_ERR_STATE, "mhd_batch_run: null batch");
    if (max_steps < 1) return berr(MHD_ERR_ARG, "mhd_batch_run: max_steps must be >= 1");
    int rc = start_clocks(b);
    if (rc) return rc;
    if (!b->graph || std::memcmp(&b->graph_tune, &b->tune, sizeof b->tune) != 0) {
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
        cudaStream_t cap = b->stream;
        bool own = false;
        if (!cap) {
            BCK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            own = true;
        }
        cudaGraph_t gr = nullptr;
        BCK(phase(b, 0, 0, b->tune, cap));  // kernel attribute set-up, outside the capture
        BCK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int p = 0; p < 2 && e == cudaSuccess; ++p) {
            e = phase(b, p, 1, b->tune, cap);
            if (e == cudaSuccess) e = phase(b, p, 2, b->tune, cap);
        }
        const cudaError_t e2 = cudaStreamEndCapture(cap, &gr);
        if (own) cudaStreamDestroy(cap);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (gr) cudaGraphDestroy(gr);
            return berr(MHD_ERR_CUDA, "mhd_batch_run: graph capture failed");
        }
        const cudaError_t e3 = cudaGraphInstantiate(&b->graph, gr, 0);
        cudaGraphDestroy(gr);
        if (e3 != cudaSuccess) {
            b->graph = nullptr;
            return berr(MHD_ERR_CUDA, "mhd_batch_run: graph instantiation failed");
        }
        b->graph_tune = b->tune;
    }
    for (int p = 0; p < max_steps / 2; ++p) BCK(cudaGraphLaunch(b->graph, b->stream));
    if (max_steps & 1) {
        BCK(phase(b, 0, 1, b->tune, b->stream));
        BCK(phase(b, 0, 2, b->tune, b->stream));
    }
    std::vector<mhd::DevClock> hc(b->n);
    BCK(cudaMemcpyAsync(hc.data(), b->d_clock, sizeof(mhd::DevClock) * b->n, cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    int worst = MHD_OK;
    for (int i = 0; i < b->n; ++i) {
        const mhd::DevClock& c = hc[i];
        if (c.steps > 0) b->ch[i] = c.last_ch;
        int code = MHD_OK;
        if (c.status == mhd::CLK_NO_SPEED) code = MHD_ERR_NO_SPEED;
        else if (c.status == mhd::CLK_BAD_DT) code = MHD_ERR_BAD_DT;
        else if (c.status == mhd::CLK_TINY_DT) code = MHD_ERR_TINY_DT;
        if (code != MHD_OK) worst = code;
        if (info) {
            info[i].t = c.t[c.steps & 1];
            info[i].last_dt = c.last_dt;
            info[i].ch = b->ch[i];
            info[i].steps = c.steps;
            info[i].status = code;
            info[i].fallbacks = c.flux_fallbacks;
            info[i].pad_ = 0;
        }
    }
    if (worst != MHD_OK) return berr(worst, "mhd_batch_run: an instance's step loop stopped (see its info.status)");
    return MHD_OK;
}

int mhd_batch_tune_candidates(int which, int* out, int cap) {
    const int* src = nullptr;
    int n = 0;
    switch (which) {
        case 0: src = kTuneXrpw; n = (int)(sizeof(kTuneXrpw) / sizeof(int)); break;
        case 1: src = kTuneYseg; n = (int)(sizeof(kTuneYseg) / sizeof(int)); break;
        case 2: src = kTuneCtasPerSm; n = (int)(sizeof(kTuneCtasPerSm) / sizeof(int)); break;
        default: return berr(MHD_ERR_ARG, "mhd_batch_tune_candidates: which must be 0, 1 or 2");
    }
    for (int k = 0; out && k < n && k < cap; ++k) out[k] = src[k];
    return n;
}

int mhd_batch_tune(mhd_batch* b, int reps, mhd_batch_tuning* best_out) {
    mhd::NvtxRange nvtx_range("mhd_batch_tune");
    if (!b) return berr(MHD_ERR_STATE, "mhd_batch_tune: null batch");
    if (reps < 1) reps = 3;
    int rc = start_clocks(b);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    mhd_batch_tuning best = b->tune;
    const auto& xr = kTuneXrpw;
    const auto& xc = kTuneCtasPerSm;
    const auto& ys = kTuneYseg;
    const auto& yc = kTuneCtasPerSm;
    auto time_phase = [&](int which, float* ms) -> int {
        BCK(phase(b, 0, which, b->tune, b->stream));  // warm
        BCK(cudaEventRecord(e0, b->stream));
        for (int r = 0; r < reps; ++r) BCK(phase(b, 0, which, b->tune, b->stream));
        BCK(cudaEventRecord(e1, b->stream));
        BCK(cudaEventSynchronize(e1));
        BCK(cudaEventElapsedTime(ms, e0, e1));
        return MHD_OK;
    };
    float best_ms = 1e30f;
    for (int r : xr)
        for (int c : xc) {
            b->tune.xrpw = r;
            b->tune.ctas_x = c * b->nsm;
            if ((rc = build_worklist(b))) return rc;
            float ms = 0.f;
            if ((rc = time_phase(1, &ms))) return rc;
            if (ms < best_ms) {
                best_ms = ms;
                best.xrpw = r;
                best.ctas_x = c * b->nsm;
            }
        }
    b->tune.xrpw = best.xrpw;
    b->tune.ctas_x = best.ctas_x;
    if ((rc = build_worklist(b))) return rc;
    BCK(phase(b, 0, 1, b->tune, b->stream));  // T from U with the chosen x tuning
    best_ms = 1e30f;
    for (int s : ys)
        for (int c : yc) {
            b->tune.yseg = s;
            b->tune.ctas_y = c * b->nsm;
            if ((rc = build_worklist(b))) return rc;
            float ms = 0.f;
            if ((rc = time_phase(2, &ms))) return rc;
            if (ms < best_ms) {
                best_ms = ms;
                best.yseg = s;
                best.ctas_y = c * b->nsm;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->tune = best;
    if ((rc = build_worklist(b))) return rc;
    if (best_out) *best_out = best;
    return MHD_OK;
}

}  // extern "C"
