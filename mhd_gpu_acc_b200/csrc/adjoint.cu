// adjoint.cu -- discrete adjoint of the split GLM-MHD step (HLL or HLLD, van
// Leer or minmod, periodic boundaries) and the Orszag-Tang gradient problem of
// the C ABI (mhd_adjoint_*).
//
// Forward step n (the same kernels as mhd_advance, explicit dt_n and c_h,n):
//   m_n = max(c_h,n-1, max_cells s(U^n)),  c_h,n = m_n,  dt_n = cfl dmin / m_n,
//   T = X(U^n) (x-sweep + ghost fill),  V = Y(T) (y-sweep + ghost fill),
//   U^{n+1} = V with interior psi scaled by f_n = exp(-dt_n c_h,n / c_r)
//   (ghost psi undamped, as the reference orders it).
// Reverse step n, with lambda = dJ/dU^{n+1} on the cells the next x-sweep reads:
//   (a) fold the ghost-column cotangents onto their periodic sources and apply
//       the damping: lambda_V; collect dJ/df_n;
//   (b) recompute T = X(U^n);
//   (c) lambda_T = Y^T lambda_V (recomputing Y locally), + dJ/d(dt/dy), dJ/dc_h;
//   (d) fold the ghost-row cotangents of T onto their sources;
//   (e) lambda_U = X^T lambda_T (recomputing X locally), + dJ/d(dt/dx), dJ/dc_h;
//   (f) dJ/dm_n from dt_n, c_h,n and f_n (plus the next step's floor when it
//       was c_h,n itself) goes to the argmax cell of U^n through the CFL speed.
// Every branch is re-evaluated from the recomputed forward states, i.e. the
// adjoint differentiates the branches the forward took.
// Checkpointing: states every S steps are kept during the forward solve; the
// reverse pass recomputes one segment of S steps at a time from its checkpoint
// (storing the segment), then walks it backwards: 2N forward steps and
// N/S + S + 1 stored states for N steps.
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/mhd_b200.h"
#include "adj_physics.cuh"
#include "launch.h"
#include "sweep.cuh"

namespace mhd {
int report_error(int code, const char* msg);
}

namespace mhd {
namespace adj {

constexpr int AT = 26;  // outputs per warp: 32 lanes minus a 3-cell halo on each side

template <typename R>
__device__ __forceinline__ void ld(const DevGrid& g, int dir, int line, int p, R* v) {
    if (dir == 0) load_cell(g, p, line, v);
    else { load_cell(g, line, p, v); rot(v); }
}
template <typename R>
__device__ __forceinline__ void st(const DevGrid& g, int dir, int line, int p, R* v) {
    if (dir == 1) rot(v);
    if (dir == 0) store_cell(g, p, line, v);
    else store_cell(g, line, p, v);
}

// lamIn = (sweep)^T lamOut along DIR for every interior line; lanes along the
// sweep direction.  Writes lamIn at positions [ng-2, ng+n+2) of each line.
template <typename R, int DIR, int LIM, int SOLVER>
__global__ void __launch_bounds__(256) adj_sweep_kernel(DevGrid U, DevGrid lamOut, DevGrid lamIn, R g, R dtd, R ch,
                                                        double* acc) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int ng = U.ng;
    const int nline = (DIR == 0) ? U.ny : U.nx;
    const int nalong = (DIR == 0) ? U.nx : U.ny;
    const int ntile = (nalong + 4 + AT - 1) / AT;
    const int line_i = warp / ntile, tile = warp - line_i * ntile;
    double sdt = 0.0, sch = 0.0;
    if (line_i < nline) {
        const int line = ng + line_i;
        const int p = ng - 2 + tile * AT + lane - 3;
        const int tn = nalong + 2 * ng;
        R Uc[NV], W[NV];
        zero(Uc);
        Uc[RHO] = R(1);
        if (p >= 0 && p < tn) ld(U, DIR, line, p, Uc);
        c2p(Uc, g, W);
        R Wm[NV], Wp[NV], Ls[NV], Rs[NV];
        shfl_up_n<NV>(W, Wm, 1);
        shfl_down_n<NV>(W, Wp, 1);
        zero(Ls);
        zero(Rs);
        const bool do_recon = lane >= 1 && lane <= 30 && p >= ng - 1 && p <= ng + nalong;
        const bool do_face = lane >= 1 && lane <= 29 && p >= ng - 1 && p <= ng + nalong - 1;
        const bool interior = p >= ng && p < ng + nalong;
        if (do_recon) recon<LIM>(Wm, W, Wp, dtd, ch, g, Ls, Rs);
        R Ln[NV];
        shfl_down_n<NV>(Ls, Ln, 1);  // L* of cell p+1
        R lT[NV], lTn[NV];
        zero(lT);
        if (interior) ld(lamOut, DIR, line, p, lT);
        shfl_down_n<NV>(lT, lTn, 1);
        // Lanes 3..28 own their position p, the face (p | p+1) and the
        // reconstruction of p; only owned work adds to the scalar cotangents,
        // so overlapping halos of neighbouring tiles count nothing twice.
        const bool own = lane >= 3 && lane <= 28;
        R F[NV], lF[NV], lR[NV], lLn[NV];
        zero(F);
        zero(lR);
        zero(lLn);
        R lch = R(0), ldtd = R(0);
        if (do_face) {
            face<SOLVER>(Rs, Ln, ch, g, F);
#pragma unroll
            for (int k = 0; k < NV; ++k) lF[k] = dtd * (lTn[k] - lT[k]);
            R lch_f = R(0);
            face_adj<SOLVER>(Rs, Ln, ch, g, lF, lR, lLn, lch_f);
            if (own) lch += lch_f;
        }
        R Fm[NV], lL[NV];
        shfl_up_n<NV>(F, Fm, 1);    // flux of face (p-1 | p)
        shfl_up_n<NV>(lLn, lL, 1);  // cotangent of L* of cell p
        if (interior && own) {
#pragma unroll
            for (int k = 0; k < NV; ++k) ldtd -= lT[k] * (F[k] - Fm[k]);
        }
        R lWm[NV], lWc[NV], lWp[NV];
        zero(lWm);
        zero(lWc);
        zero(lWp);
        if (do_recon) {
            R ldtd_r = R(0), lch_r = R(0);
            recon_adj<LIM>(Wm, W, Wp, dtd, ch, g, lL, lR, lWm, lWc, lWp, ldtd_r, lch_r);
            if (own) { ldtd += ldtd_r; lch += lch_r; }
        }
        R a[NV], b[NV];
        shfl_up_n<NV>(lWp, a, 1);    // from cell p-1 (its W_{p+1} role)
        shfl_down_n<NV>(lWm, b, 1);  // from cell p+1 (its W_{p-1} role)
        R lW[NV], lU[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) lW[k] = lWc[k] + a[k] + b[k];
        zero(lU);
        if (interior) {
#pragma unroll
            for (int k = 0; k < NV; ++k) lU[k] = lT[k];  // T_p = U_p - dtd (F_{p+1/2} - F_{p-1/2})
        }
        c2p_adj(Uc, W, g, lW, lU);
        const bool out = lane >= 3 && lane <= 28 && p >= ng - 2 && p < ng + nalong + 2;
        if (out) st(lamIn, DIR, line, p, lU);
        sdt = (double)ldtd;
        sch = (double)lch;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sdt += __shfl_xor_sync(FULL, sdt, o);
        sch += __shfl_xor_sync(FULL, sch, o);
    }
    if (lane == 0 && (sdt != 0.0 || sch != 0.0)) {
        atomicAdd(acc, sdt);
        atomicAdd(acc + 1, sch);
    }
}

// Fold the cotangents of ghost cells onto the interior cells they copy
// (periodic, transmissive or reflecting; reflecting flips the normal momentum
// and field).  dir 0: ghost columns of interior rows; dir 1: ghost rows of
// interior columns.  When damp_psi > 0 (step (a)) the interior psi cotangent is
// scaled by f and sum(lambda_psi * Unext_psi / f) is added to acc[2].
template <typename R>
__global__ void fold_kernel(DevGrid lam, DevGrid out, DevGrid Unext, int dir, int b0, int b1, int b2, int b3,
                            double f, double* acc) {
    const int bc[4] = {b0, b1, b2, b3};
    const int ng = lam.ng, ib = ng, ie = ng + lam.nx, jb = ng, je = ng + lam.ny;
    const long long n = (long long)lam.nx * lam.ny;
    double sf = 0.0;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(k / lam.nx) + ng, i = (int)(k % lam.nx) + ng;
        R v[NV];
        load_cell(lam, i, j, v);
        if (f > 0.0) {
            R un[NV];
            load_cell(Unext, i, j, un);
            sf += (double)v[PSI] * (double)un[PSI] / f;
            v[PSI] = v[PSI] * (R)f;
        }
        for (int q = 0; q < ng; ++q) {
            for (int side = 0; side < 2; ++side) {
                const int t = (dir == 0) ? bc[side] : bc[2 + side];
                const int c = (dir == 0) ? i : j;
                const int lo = (dir == 0) ? ib : jb, hi = (dir == 0) ? ie : je;
                const int src = side == 0 ? src_left(t, q, lo, hi) : src_right(t, q, lo, hi);
                if (src != c) continue;
                const int gpos = side == 0 ? lo - 1 - q : hi + q;
                R gv[NV];
                if (dir == 0) load_cell(lam, gpos, j, gv);
                else load_cell(lam, i, gpos, gv);
                if (t == REFLECTING) {
                    if (dir == 0) { gv[MX] = -gv[MX]; gv[BX] = -gv[BX]; }
                    else { gv[MY] = -gv[MY]; gv[BY] = -gv[BY]; }
                }
#pragma unroll
                for (int m = 0; m < NV; ++m) v[m] += gv[m];
            }
        }
        store_cell(out, i, j, v);
    }
    if (f > 0.0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sf += __shfl_xor_sync(FULL, sf, o);
        if ((threadIdx.x & 31) == 0 && sf != 0.0) atomicAdd(acc + 2, sf);
    }
}

template <typename R>
__global__ void fill_kernel(DevGrid g, R v) {
    const long long n = g.plane * NV;
    R* d = static_cast<R*>(g.data);
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        d[k] = v;
}

// J = 1/2 sum_interior (rho - target)^2 (into acc[3]) and lambda_N = (rho - target) e_rho
template <typename R>
__global__ void objective_kernel(DevGrid U, const double* target, DevGrid lam, double* acc) {
    const long long n = (long long)U.nx * U.ny;
    double s = 0.0;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(k / U.nx) + U.ng, i = (int)(k % U.nx) + U.ng;
        const double d = (double)static_cast<const R*>(U.data)[U.idx(i, j)] - target[k];
        s += 0.5 * d * d;
        if (lam.data) static_cast<R*>(lam.data)[lam.idx(i, j)] = (R)d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(acc + 3, s);
}

// Reverse of the CFL speed of the argmax cell (*idx; INT_MAX: none) with weight
// *lm (the step's combined dt / c_h cotangent, from step_scalars_kernel).
template <typename R>
__global__ void speed_adj_kernel(DevGrid U, DevGrid lam, const int* idx_p, R g, const double* lm_p) {
    const int idx = *idx_p;
    if (idx == INT_MAX) return;
    const R lm = (R)*lm_p;
    const int j = idx / U.nx + U.ng, i = idx % U.nx + U.ng;
    R u[NV], l[NV];
    load_cell(U, i, j, u);
    load_cell(lam, i, j, l);
    int branch = 0;
    raw_speed(u, g, &branch);
    raw_speed_adj(u, g, branch, lm, l);
    store_cell(lam, i, j, l);
}

// Per-step scalars of the reverse pass, on the device so the pass needs no
// host round trip.  sc: [0, 1] the y-sweep's dt/dy and c_h cotangent sums,
// [2] sum(lambda_psi * psi / f) of the damping fold, [3, 4] the x-sweep's sums,
// [5] the c_h floor carry between steps, [6] the weight of the argmax cell.
// The expressions and their order are the host code's before it moved here
// (explicit round-to-nearest operations, no contraction).
__global__ void step_scalars_kernel(double* sc, int* idx, double dt, double ch, double f, double cr, double dx,
                                    double dy, int new_max) {
    const double ldt = __dadd_rn(__dadd_rn(__ddiv_rn(sc[3], dx), __ddiv_rn(sc[0], dy)),
                                 __dmul_rn(__dmul_rn(sc[2], f), __ddiv_rn(-ch, cr)));
    const double lch = __dadd_rn(__dadd_rn(__dadd_rn(sc[4], sc[1]), __dmul_rn(__dmul_rn(sc[2], f), __ddiv_rn(-dt, cr))),
                                 sc[5]);
    const double lm = __dadd_rn(lch, __dmul_rn(ldt, __ddiv_rn(-dt, ch)));
    if (new_max) {  // this step's maximum set c_h: its argmax cell takes lm
        sc[6] = lm;
        sc[5] = 0.0;
        *idx = INT_MAX;
    } else {        // the floor c_h,n-1 set this step's maximum: lm carries to step n-1
        sc[5] = lm;
    }
}

__device__ __constant__ int kMX[8] = {1, 0, 1, 1, 2, 0, 2, 1};
__device__ __constant__ int kMY[8] = {0, 1, 1, -1, 0, 2, 1, 2};

// grad_k += sum over every cell (ghosts included) of lambda_0 . dU0/da_k for the
// perturbed Orszag-Tang initial data (mhd_initialise_orszag_tang).
template <typename R>
__global__ void ic_grad_kernel(DevGrid lam, DevGrid U0, double x0, double y0, double dx, double dy, double* grad) {
    const double PI = 3.14159265358979323846;
    const int tx = lam.tnx(), ty = lam.tny();
    const long long n = (long long)tx * ty;
    double gk[16];
    for (int k = 0; k < 16; ++k) gk[k] = 0.0;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(c / tx), i = (int)(c - (long long)j * tx);
        const double x = x0 + ((double)(i - lam.ng) + 0.5) * dx;
        const double y = y0 + ((double)(j - lam.ng) + 0.5) * dy;
        R l[NV], u[NV];
        load_cell(lam, i, j, l);
        load_cell(U0, i, j, u);
        const double rho = u[RHO], uu = u[MX] / rho, vv = u[MY] / rho, bx = u[BX], by = u[BY];
        for (int m = 0; m < 8; ++m) {
            const double mx = kMX[m], my = kMY[m];
            const double s = sin(2.0 * PI * (mx * x + my * y)) / sqrt(mx * mx + my * my);
            const double du = -s * my, dv = s * mx;  // d(u, v)/d amp[m]  and  d(Bx, By)/d amp[8+m]
            gk[m] += (double)l[MX] * rho * du + (double)l[MY] * rho * dv + (double)l[EN] * rho * (uu * du + vv * dv);
            gk[8 + m] += (double)l[BX] * du + (double)l[BY] * dv + (double)l[EN] * (bx * du + by * dv);
        }
    }
    for (int k = 0; k < 16; ++k) {
        double v = gk[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
        if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(grad + k, v);
    }
}

unsigned blocks_for(long long n) {
    long long b = (n + 255) / 256;
    if (b > 8192) b = 8192;
    return (unsigned)(b < 1 ? 1 : b);
}

template <typename R, int SOLVER>
void launch_adj_sweep(int dir, int lim, unsigned blocks, const DevGrid& U, const DevGrid& lout, const DevGrid& lin,
                      double g, double dtd, double ch, double* acc, cudaStream_t st) {
    if (dir == 0 && lim == VANLEER)
        adj_sweep_kernel<R, 0, VANLEER, SOLVER><<<blocks, 256, 0, st>>>(U, lout, lin, (R)g, (R)dtd, (R)ch, acc);
    else if (dir == 0)
        adj_sweep_kernel<R, 0, MINMOD, SOLVER><<<blocks, 256, 0, st>>>(U, lout, lin, (R)g, (R)dtd, (R)ch, acc);
    else if (lim == VANLEER)
        adj_sweep_kernel<R, 1, VANLEER, SOLVER><<<blocks, 256, 0, st>>>(U, lout, lin, (R)g, (R)dtd, (R)ch, acc);
    else
        adj_sweep_kernel<R, 1, MINMOD, SOLVER><<<blocks, 256, 0, st>>>(U, lout, lin, (R)g, (R)dtd, (R)ch, acc);
}

template <typename R>
cudaError_t run_adj_sweep(int dir, int lim, int solver, const DevGrid& U, const DevGrid& lout, const DevGrid& lin,
                          double g, double dtd, double ch, double* acc, cudaStream_t st) {
    const int nline = dir == 0 ? U.ny : U.nx, nalong = dir == 0 ? U.nx : U.ny;
    const long long warps = (long long)nline * ((nalong + 4 + AT - 1) / AT);
    const unsigned blocks = (unsigned)((warps * 32 + 255) / 256);
    if (solver == HLLD) launch_adj_sweep<R, HLLD>(dir, lim, blocks, U, lout, lin, g, dtd, ch, acc, st);
    else launch_adj_sweep<R, HLL>(dir, lim, blocks, U, lout, lin, g, dtd, ch, acc, st);
    return cudaGetLastError();
}

}  // namespace adj
}  // namespace mhd

// ---------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------
struct mhd_adjoint {
    int nx = 0, ny = 0, dtype = MHD_F64, limiter = MHD_LIMITER_VANLEER, solver = MHD_HLL, nsteps = 0, every = 1;
    double gamma = 5.0 / 3.0, cfl = 0.4, cr = 0.18, b0 = 0.0;
    std::vector<mhd_grid> ckpt, seg;
    mhd_grid T{}, lamA{}, lamB{}, lamT{}, lamV{};
    mhd_workspace* ws = nullptr;
    double* d_target = nullptr;  // ny * nx
    double* d_acc = nullptr;     // [dt/dx-or-dy, ch, f, J] cotangent / objective sums
    double* d_grad = nullptr;    // 16
    int* d_idx = nullptr;
    double* d_sc = nullptr;      // 8: per-step scalars of the reverse pass (step_scalars_kernel)
    std::vector<double> dt, ch;  // per step
    bool have_target = false;
};

namespace {

using mhd::DevGrid;

int aerr(int code, const char* msg) { return mhd::report_error(code, msg); }

#define ACK(call)                                                                \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) return aerr(MHD_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)
#define ARC(call)               \
    do {                        \
        int r_ = (call);        \
        if (r_) return r_;      \
    } while (0)

DevGrid dg(const mhd_grid& g) { return DevGrid{g.data, g.pitch, g.plane, g.nx, g.ny, g.ng, 0}; }

bool f64(const mhd_adjoint* a) { return a->dtype == MHD_F64; }

int grid_copy(const mhd_grid& dst, const mhd_grid& src, cudaStream_t st) {
    const size_t eb = src.dtype == MHD_F32 ? 4 : 8;
    ACK(cudaMemcpyAsync(dst.data, src.data, (size_t)src.plane * MHD_NV * eb, cudaMemcpyDeviceToDevice, st));
    return MHD_OK;
}

int zero_grid(const mhd_grid& g, cudaStream_t st) {
    const size_t eb = g.dtype == MHD_F32 ? 4 : 8;
    ACK(cudaMemsetAsync(g.data, 0, (size_t)g.plane * MHD_NV * eb, st));
    return MHD_OK;
}

const int kPeriodic[4] = {MHD_BC_PERIODIC, MHD_BC_PERIODIC, MHD_BC_PERIODIC, MHD_BC_PERIODIC};

// one forward step Uin -> Uout through the library's step with explicit dt / ch
int fwd_step(mhd_adjoint* a, const mhd_grid& Uin, mhd_grid& Uout, double dt, double ch) {
    ARC(mhd_set_ch(a->ws, ch));
    return mhd_advance(a->ws, &Uin, &a->T, &Uout, dt, a->solver, kPeriodic);
}

// Forward solve from amp: checkpoints every `every` steps, per-step dt and ch.
int forward(mhd_adjoint* a, const double* amp, double* J, double* rho_final) {
    cudaStream_t st = nullptr;
    ARC(mhd_initialise_orszag_tang(a->ws, &a->ckpt[0], a->b0, a->gamma, amp));
    ARC(mhd_set_ch(a->ws, 0.0));
    mhd_grid cur = a->seg[0], nxt = a->seg[1];
    ARC(grid_copy(cur, a->ckpt[0], st));
    a->dt.assign(a->nsteps, 0.0);
    a->ch.assign(a->nsteps, 0.0);
    for (int n = 0; n < a->nsteps; ++n) {
        if (n % a->every == 0 && n > 0) ARC(grid_copy(a->ckpt[n / a->every], cur, st));
        double dt = 0.0;
        ARC(mhd_compute_dt(a->ws, &cur, a->cfl, &dt));
        ARC(mhd_get_ch(a->ws, &a->ch[n]));
        a->dt[n] = dt;
        ARC(mhd_advance(a->ws, &cur, &a->T, &nxt, dt, a->solver, kPeriodic));
        std::swap(cur, nxt);
    }
    // keep the final state in seg[0] for the objective
    if (cur.data != a->seg[0].data) ARC(grid_copy(a->seg[0], cur, st));
    ACK(cudaMemsetAsync(a->d_acc, 0, sizeof(double) * 4, st));
    if (a->have_target) {
        const DevGrid U = dg(a->seg[0]);
        const DevGrid none{nullptr, U.pitch, U.plane, U.nx, U.ny, U.ng, 0};
        if (f64(a)) mhd::adj::objective_kernel<double><<<mhd::adj::blocks_for((long long)a->nx * a->ny), 256, 0, st>>>(U, a->d_target, none, a->d_acc);
        else mhd::adj::objective_kernel<float><<<mhd::adj::blocks_for((long long)a->nx * a->ny), 256, 0, st>>>(U, a->d_target, none, a->d_acc);
        ACK(cudaGetLastError());
    }
    double acc[4];
    ACK(cudaMemcpy(acc, a->d_acc, sizeof acc, cudaMemcpyDeviceToHost));
    if (J) *J = acc[3];
    if (rho_final) {
        std::vector<double> h((size_t)MHD_NV * (a->nx + 4) * (a->ny + 4));
        ARC(mhd_grid_download(&a->seg[0], h.data()));
        const int tnx = a->nx + 4;
        for (int j = 0; j < a->ny; ++j)
            for (int i = 0; i < a->nx; ++i) rho_final[(size_t)j * a->nx + i] = h[(size_t)(j + 2) * tnx + i + 2];
    }
    return MHD_OK;
}

template <typename R>
int reverse_step(mhd_adjoint* a, int n, const mhd_grid& Un, const mhd_grid& Un1, mhd_grid& lam_next,
                 mhd_grid& lam_out) {
    cudaStream_t st = nullptr;
    const double dt = a->dt[n], ch = a->ch[n];
    const double f = std::exp(-dt * ch / a->cr) >= 1.0 ? 1.0 : std::exp(-dt * ch / a->cr);
    const double dx = 1.0 / a->nx, dy = 1.0 / a->ny;
    double* sc = a->d_sc;
    ACK(cudaMemsetAsync(sc, 0, sizeof(double) * 5, st));
    // (a) lambda_V from lambda_{n+1}: ghost columns onto sources, damping, dJ/df (into sc[2])
    mhd::adj::fold_kernel<R><<<mhd::adj::blocks_for((long long)a->nx * a->ny), 256, 0, st>>>(
        dg(lam_next), dg(a->lamV), dg(Un1), 0, 0, 0, 0, 0, f, sc);
    ACK(cudaGetLastError());
    // (b) T = X(U^n)
    {
        mhd::StepParams P{};
        P.gamma = a->gamma; P.cr = a->cr; P.dx = dx; P.dy = dy; P.dmin = dx < dy ? dx : dy;
        P.dt = dt; P.ch = ch; P.damp = f; P.solver = a->solver; P.limiter = a->limiter;
        const cudaError_t e = f64(a) ? mhd::launch_step_f64(dg(Un), dg(a->T), dg(a->T), P, st, mhd::kDefaultYBand, 1)
                                     : mhd::launch_step_f32(dg(Un), dg(a->T), dg(a->T), P, st, mhd::kDefaultYBand, 1);
        ACK(e);
    }
    // (c) lambda_T = Y^T lambda_V (dt/dy and c_h sums into sc[0], sc[1])
    ARC(zero_grid(a->lamT, st));
    ACK(mhd::adj::run_adj_sweep<R>(1, a->limiter, a->solver, dg(a->T), dg(a->lamV), dg(a->lamT), a->gamma, dt / dy, ch,
                                   sc, st));
    // (d) ghost rows of T onto their sources (lamV is free again: reuse it; no sums)
    mhd::adj::fold_kernel<R><<<mhd::adj::blocks_for((long long)a->nx * a->ny), 256, 0, st>>>(
        dg(a->lamT), dg(a->lamV), dg(a->lamT), 1, 0, 0, 0, 0, -1.0, sc);
    ACK(cudaGetLastError());
    // (e) lambda_U = X^T lambda_T (sums into sc[3], sc[4])
    ARC(zero_grid(lam_out, st));
    ACK(mhd::adj::run_adj_sweep<R>(0, a->limiter, a->solver, dg(Un), dg(a->lamV), dg(lam_out), a->gamma, dt / dx, ch,
                                   sc + 3, st));
    // (f) the time step and cleaning speed: dt = cfl dmin / c_h with c_h the
    // larger of this step's maximum speed and the previous c_h
    const double ch_prev = n > 0 ? a->ch[n - 1] : 0.0;
    const int new_max = ch > ch_prev;
    mhd::adj::step_scalars_kernel<<<1, 1, 0, st>>>(sc, a->d_idx, dt, ch, f, a->cr, dx, dy, new_max);
    ACK(cudaGetLastError());
    if (new_max) {
        const cudaError_t e = f64(a) ? mhd::launch_argmax_f64(dg(Un), a->gamma, ch_prev, ch, a->d_idx, st)
                                     : mhd::launch_argmax_f32(dg(Un), a->gamma, ch_prev, ch, a->d_idx, st);
        ACK(e);
        mhd::adj::speed_adj_kernel<R><<<1, 1, 0, st>>>(dg(Un), dg(lam_out), a->d_idx, (R)a->gamma, sc + 6);
        ACK(cudaGetLastError());
    }
    return MHD_OK;
}

template <typename R>
int gradient(mhd_adjoint* a, const double* amp, double* J, double* grad) {
    cudaStream_t st = nullptr;
    ARC(forward(a, amp, J, nullptr));
    // lambda_N from the final state (kept in seg[0] by forward())
    ARC(zero_grid(a->lamA, st));
    ACK(cudaMemsetAsync(a->d_acc, 0, sizeof(double) * 4, st));
    mhd::adj::objective_kernel<R><<<mhd::adj::blocks_for((long long)a->nx * a->ny), 256, 0, st>>>(
        dg(a->seg[0]), a->d_target, dg(a->lamA), a->d_acc);
    ACK(cudaGetLastError());
    mhd_grid lam_next = a->lamA, lam_cur = a->lamB;
    ACK(cudaMemsetAsync(a->d_sc, 0, sizeof(double) * 8, st));  // the c_h floor carry starts at zero
    const int nseg = (a->nsteps + a->every - 1) / a->every;
    for (int k = nseg - 1; k >= 0; --k) {
        const int n0 = k * a->every, n1 = std::min(a->nsteps, n0 + a->every);
        ARC(grid_copy(a->seg[0], a->ckpt[k], st));
        for (int n = n0; n < n1; ++n) ARC(fwd_step(a, a->seg[n - n0], a->seg[n - n0 + 1], a->dt[n], a->ch[n]));
        for (int n = n1 - 1; n >= n0; --n) {
            ARC(reverse_step<R>(a, n, a->seg[n - n0], a->seg[n - n0 + 1], lam_next, lam_cur));
            std::swap(lam_next, lam_cur);
        }
    }
    // lam_next now holds dJ/dU^0 (ghosts included); contract with dU^0/da
    ACK(cudaMemsetAsync(a->d_grad, 0, sizeof(double) * 16, st));
    ARC(mhd_initialise_orszag_tang(a->ws, &a->seg[0], a->b0, a->gamma, amp));
    mhd::adj::ic_grad_kernel<R><<<mhd::adj::blocks_for((long long)(a->nx + 4) * (a->ny + 4)), 256, 0, st>>>(
        dg(lam_next), dg(a->seg[0]), 0.0, 0.0, 1.0 / a->nx, 1.0 / a->ny, a->d_grad);
    ACK(cudaGetLastError());
    ACK(cudaMemcpy(grad, a->d_grad, sizeof(double) * 16, cudaMemcpyDeviceToHost));
    return MHD_OK;
}

}  // namespace

extern "C" {

int mhd_adjoint_create(int nx, int ny, int dtype, int limiter, double gamma, double cfl, double cr, int nsteps,
                       int checkpoint_every, mhd_adjoint** out) {
    if (!out || nx < 4 || ny < 4 || nsteps < 1 || (dtype != MHD_F64 && dtype != MHD_F32) ||
        (limiter != MHD_LIMITER_MINMOD && limiter != MHD_LIMITER_VANLEER) || !(gamma > 1.0) || !(cfl > 0.0) ||
        !(cr > 0.0))
        return aerr(MHD_ERR_ARG, "mhd_adjoint_create: invalid arguments");
    *out = nullptr;
    mhd_adjoint* a = new mhd_adjoint();
    a->nx = nx; a->ny = ny; a->dtype = dtype; a->limiter = limiter; a->gamma = gamma; a->cfl = cfl; a->cr = cr;
    a->nsteps = nsteps;
    a->every = checkpoint_every > 0 ? checkpoint_every : std::max(1, (int)std::lround(std::sqrt((double)nsteps)));
    a->b0 = 1.0 / std::sqrt(4.0 * M_PI);
    const int nck = (nsteps + a->every - 1) / a->every;
    a->ckpt.assign(nck, mhd_grid{});
    a->seg.assign(a->every + 1, mhd_grid{});
    int rc = MHD_OK;
    auto alloc = [&](mhd_grid& g) {
        if (!rc) rc = mhd_grid_alloc(&g, nx, ny, 2, dtype, 0.0, 1.0, 0.0, 1.0);
    };
    for (auto& g : a->ckpt) alloc(g);
    for (auto& g : a->seg) alloc(g);
    alloc(a->T); alloc(a->lamA); alloc(a->lamB); alloc(a->lamT); alloc(a->lamV);
    if (!rc) rc = mhd_workspace_create(&a->seg[0], &a->ws);
    if (!rc) rc = mhd_set_gamma(a->ws, gamma);
    if (!rc) rc = mhd_set_limiter(a->ws, limiter);
    if (!rc) rc = mhd_set_cr(a->ws, cr);
    if (!rc && (cudaMalloc(&a->d_target, sizeof(double) * (size_t)nx * ny) != cudaSuccess ||
                cudaMalloc(&a->d_acc, sizeof(double) * 4) != cudaSuccess ||
                cudaMalloc(&a->d_grad, sizeof(double) * 16) != cudaSuccess ||
                cudaMalloc(&a->d_idx, sizeof(int)) != cudaSuccess ||
                cudaMalloc(&a->d_sc, sizeof(double) * 8) != cudaSuccess))
        rc = aerr(MHD_ERR_NOMEM, "mhd_adjoint_create: device buffers");
    if (rc) {
        mhd_adjoint_destroy(a);
        return rc;
    }
    *out = a;
    return MHD_OK;
}

int mhd_adjoint_set_solver(mhd_adjoint* a, int solver) {
    if (!a) return aerr(MHD_ERR_STATE, "mhd_adjoint_set_solver: null adjoint");
    if (solver != MHD_HLL && solver != MHD_HLLD)
        return aerr(MHD_ERR_ARG, "mhd_adjoint_set_solver: the adjoint differentiates HLL or HLLD");
    a->solver = solver;
    return MHD_OK;
}

int mhd_adjoint_destroy(mhd_adjoint* a) {
    if (!a) return MHD_OK;
    for (auto& g : a->ckpt) mhd_grid_free(&g);
    for (auto& g : a->seg) mhd_grid_free(&g);
    mhd_grid_free(&a->T); mhd_grid_free(&a->lamA); mhd_grid_free(&a->lamB);
    mhd_grid_free(&a->lamT); mhd_grid_free(&a->lamV);
    if (a->ws) mhd_workspace_destroy(a->ws);
    if (a->d_target) cudaFree(a->d_target);
    if (a->d_acc) cudaFree(a->d_acc);
    if (a->d_grad) cudaFree(a->d_grad);
    if (a->d_idx) cudaFree(a->d_idx);
    if (a->d_sc) cudaFree(a->d_sc);
    delete a;
    return MHD_OK;
}

int mhd_adjoint_set_target(mhd_adjoint* a, const double* rho_target) {
    if (!a || !rho_target) return aerr(MHD_ERR_ARG, "mhd_adjoint_set_target: null argument");
    ACK(cudaMemcpy(a->d_target, rho_target, sizeof(double) * (size_t)a->nx * a->ny, cudaMemcpyHostToDevice));
    a->have_target = true;
    return MHD_OK;
}

int mhd_adjoint_forward(mhd_adjoint* a, const double* amp16, double* J, double* rho_final) {
    mhd::NvtxRange nvtx_range("mhd_adjoint_forward");
    if (!a) return aerr(MHD_ERR_STATE, "mhd_adjoint_forward: null handle");
    return forward(a, amp16, J, rho_final);
}

int mhd_adjoint_gradient(mhd_adjoint* a, const double* amp16, double* J, double* grad16) {
    mhd::NvtxRange nvtx_range("mhd_adjoint_gradient");
    if (!a || !grad16) return aerr(MHD_ERR_ARG, "mhd_adjoint_gradient: null argument");
    if (!a->have_target) return aerr(MHD_ERR_STATE, "mhd_adjoint_gradient: no target set");
    return f64(a) ? gradient<double>(a, amp16, J, grad16) : gradient<float>(a, amp16, J, grad16);
}

}  // extern "C"
