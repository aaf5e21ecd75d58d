// aux_kernels.cu -- boundary conditions, precision conversion, diagnostics,
// and the tensor maps of the TMA-staged sweep.
#include <cuda.h>

#include <cstdint>
#include <mutex>

#include "launch.h"
#include "sweep.cuh"

namespace mhd {
namespace {

// In-place apply_boundary (head/cpu/boundary_cpu.hpp:45-149).  The reference
// runs left, right, bottom, top in sequence; every ghost cell's final value is
// written here directly in gather form.  The sources are interior cells or
// ghost cells that no rule overwrites (Dirichlet sides), so the in-place
// gather is free of read/write races.
template <typename R>
__global__ void apply_boundary_kernel(DevGrid g, int b0, int b1, int b2, int b3) {
    const int bc[4] = {b0, b1, b2, b3};
    const int ng = g.ng, ib = ng, ie = ng + g.nx, jb = ng, je = ng + g.ny;
    const int tx = g.tnx(), ty = g.tny();
    const long long total = (long long)tx * ty;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(k / tx), x = (int)(k - (long long)y * tx);
        const bool xg = (x < ib || x >= ie), yg = (y < jb || y >= je);
        if (!xg && !yg) continue;
        const int sxs = (x < ib) ? 0 : 1, sys = (y < jb) ? 2 : 3;
        int srcx = x, srcy = y, fx = 0, fy = 0;
        if (xg && !yg) {
            if (bc[sxs] == DIRICHLET) continue;
            srcx = ghost_src_x(x, ib, ie, bc);
            fx = (bc[sxs] == REFLECTING);
        } else if (yg && !xg) {
            if (bc[sys] == DIRICHLET) continue;
            srcy = ghost_src_y(y, jb, je, bc);
            fy = (bc[sys] == REFLECTING);
        } else {
            // corner: the bottom/top pass reads the column after the left/right pass
            if (bc[sys] != DIRICHLET) {
                srcy = ghost_src_y(y, jb, je, bc);
                fy = (bc[sys] == REFLECTING);
                if (bc[sxs] != DIRICHLET) {
                    srcx = ghost_src_x(x, ib, ie, bc);
                    fx = (bc[sxs] == REFLECTING);
                }
            } else {
                if (bc[sxs] == DIRICHLET) continue;
                srcx = ghost_src_x(x, ib, ie, bc);
                fx = (bc[sxs] == REFLECTING);
            }
        }
        R w[NV];
        const R* b = static_cast<const R*>(g.data) + g.idx(srcx, srcy);
#pragma unroll
        for (int f = 0; f < NV; ++f) w[f] = b[f * g.plane];
        if (fx) { w[MX] = -w[MX]; w[BX] = -w[BX]; }
        if (fy) { w[MY] = -w[MY]; w[BY] = -w[BY]; }
        store_cell(g, x, y, w);
    }
}

template <typename S, typename D>
__global__ void convert_kernel(DevGrid src, DevGrid dst) {
    const int tx = src.tnx(), ty = src.tny();
    const long long total = (long long)tx * ty;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(k / tx), x = (int)(k - (long long)y * tx);
        const S* s = static_cast<const S*>(src.data) + src.idx(x, y);
        D* d = static_cast<D*>(dst.data) + dst.idx(x, y);
#pragma unroll
        for (int f = 0; f < NV; ++f) d[f * dst.plane] = static_cast<D>(s[f * src.plane]);
    }
}

// Dense AoS (9 doubles per cell, row-major over the ghosted grid) <-> grid.
template <typename D>
__global__ void aos_to_grid_kernel(const double* __restrict__ aos, DevGrid dst) {
    const int tx = dst.tnx(), ty = dst.tny();
    const long long total = (long long)tx * ty;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(k / tx), x = (int)(k - (long long)y * tx);
        D* d = static_cast<D*>(dst.data) + dst.idx(x, y);
#pragma unroll
        for (int f = 0; f < NV; ++f) d[f * dst.plane] = static_cast<D>(aos[k * NV + f]);
    }
}

template <typename S>
__global__ void grid_to_aos_kernel(DevGrid src, double* __restrict__ aos) {
    const int tx = src.tnx(), ty = src.tny();
    const long long total = (long long)tx * ty;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(k / tx), x = (int)(k - (long long)y * tx);
        const S* s = static_cast<const S*>(src.data) + src.idx(x, y);
#pragma unroll
        for (int f = 0; f < NV; ++f) aos[k * NV + f] = static_cast<double>(s[f * src.plane]);
    }
}

constexpr int DIAG_BLOCKS = 1024;
constexpr int DIAG_THREADS = 256;

// Pass 1: per-block partials (fixed thread->cell assignment, fixed tree order).
template <typename R>
__global__ void __launch_bounds__(DIAG_THREADS) diag_partial_kernel(DevGrid g, double gamma, double dx, double dy,
                                                                   double* part) {
    __shared__ double sh[6][DIAG_THREADS];
    const long long n = (long long)g.nx * g.ny;
    double mass = 0.0, energy = 0.0, divl1 = 0.0, divmax = 0.0, rhomin = 1e300, pmin = 1e300;
    const R* base = static_cast<const R*>(g.data);
    for (long long k = (long long)blockIdx.x * DIAG_THREADS + threadIdx.x; k < n;
         k += (long long)gridDim.x * DIAG_THREADS) {
        const int j = (int)(k / g.nx) + g.ng, i = (int)(k % g.nx) + g.ng;
        double U[NV];
#pragma unroll
        for (int f = 0; f < NV; ++f) U[f] = (double)base[f * g.plane + g.idx(i, j)];
        mass += U[RHO];
        energy += U[EN];
        const double bxp = (double)base[BX * g.plane + g.idx(i + 1, j)];
        const double bxm = (double)base[BX * g.plane + g.idx(i - 1, j)];
        const double byp = (double)base[BY * g.plane + g.idx(i, j + 1)];
        const double bym = (double)base[BY * g.plane + g.idx(i, j - 1)];
        const double div = (bxp - bxm) / (2.0 * dx) + (byp - bym) / (2.0 * dy);
        divl1 += fabs(div);
        divmax = fmax(divmax, fabs(div));
        rhomin = fmin(rhomin, U[RHO]);
        const double ke = 0.5 * (U[MX] * U[MX] + U[MY] * U[MY] + U[MZ] * U[MZ]) / U[RHO];
        const double p = (gamma - 1.0) * (U[EN] - ke - 0.5 * (U[BX] * U[BX] + U[BY] * U[BY] + U[BZ] * U[BZ]));
        pmin = fmin(pmin, p);
    }
    sh[0][threadIdx.x] = mass; sh[1][threadIdx.x] = energy; sh[2][threadIdx.x] = divl1;
    sh[3][threadIdx.x] = divmax; sh[4][threadIdx.x] = rhomin; sh[5][threadIdx.x] = pmin;
    __syncthreads();
    for (int s = DIAG_THREADS / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + s];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + s];
            sh[2][threadIdx.x] += sh[2][threadIdx.x + s];
            sh[3][threadIdx.x] = fmax(sh[3][threadIdx.x], sh[3][threadIdx.x + s]);
            sh[4][threadIdx.x] = fmin(sh[4][threadIdx.x], sh[4][threadIdx.x + s]);
            sh[5][threadIdx.x] = fmin(sh[5][threadIdx.x], sh[5][threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x < 6) part[threadIdx.x * DIAG_BLOCKS + blockIdx.x] = sh[threadIdx.x][0];
}

__global__ void __launch_bounds__(DIAG_THREADS) diag_final_kernel(const double* part, double dA, double* out) {
    __shared__ double sh[6][DIAG_THREADS];
    for (int q = 0; q < 6; ++q) {
        double v = (q < 3) ? 0.0 : (q == 3 ? 0.0 : 1e300);
        for (int b = threadIdx.x; b < DIAG_BLOCKS; b += DIAG_THREADS) {
            const double x = part[q * DIAG_BLOCKS + b];
            if (q < 3) v += x;
            else if (q == 3) v = fmax(v, x);
            else v = fmin(v, x);
        }
        sh[q][threadIdx.x] = v;
    }
    __syncthreads();
    for (int s = DIAG_THREADS / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            for (int q = 0; q < 6; ++q) {
                const double a = sh[q][threadIdx.x], b = sh[q][threadIdx.x + s];
                sh[q][threadIdx.x] = (q < 3) ? a + b : (q == 3 ? fmax(a, b) : fmin(a, b));
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sh[0][0] * dA;
        out[1] = sh[1][0] * dA;
        out[2] = sh[2][0] * dA;
        out[3] = sh[3][0];
        out[4] = sh[4][0];
        out[5] = sh[5][0];
    }
}

__global__ void clock_init_kernel(DevClock* c, const unsigned long long* max0) {
    c->maxbits[0] = *max0;
    c->maxbits[1] = 0ull;
    c->t[0] = 0.0;
    c->t[1] = 0.0;
    c->last_dt = 0.0;
    c->last_ch = 0.0;
    c->steps = 0;
    c->status = CLK_OK;
    c->lowbeta_hits = 0u;
    c->flux_fallbacks = 0u;
}

unsigned grid_for(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    if (b > 65535LL * 4) b = 65535LL * 4;
    if (b < 1) b = 1;
    return (unsigned)b;
}

}  // namespace

cudaError_t launch_apply_boundary(const DevGrid& g, int elem_bytes, const int* bc, cudaStream_t st) {
    const long long n = (long long)g.tnx() * g.tny();
    if (elem_bytes == 8)
        apply_boundary_kernel<double><<<grid_for(n, 256), 256, 0, st>>>(g, bc[0], bc[1], bc[2], bc[3]);
    else
        apply_boundary_kernel<float><<<grid_for(n, 256), 256, 0, st>>>(g, bc[0], bc[1], bc[2], bc[3]);
    return cudaGetLastError();
}

cudaError_t launch_convert_f64_to_f32(const DevGrid& src, const DevGrid& dst, cudaStream_t st) {
    const long long n = (long long)src.tnx() * src.tny();
    convert_kernel<double, float><<<grid_for(n, 256), 256, 0, st>>>(src, dst);
    return cudaGetLastError();
}

cudaError_t launch_convert_f32_to_f64(const DevGrid& src, const DevGrid& dst, cudaStream_t st) {
    const long long n = (long long)src.tnx() * src.tny();
    convert_kernel<float, double><<<grid_for(n, 256), 256, 0, st>>>(src, dst);
    return cudaGetLastError();
}

cudaError_t launch_aos_to_grid(const double* aos, const DevGrid& dst, int elem_bytes, cudaStream_t st) {
    const long long n = (long long)dst.tnx() * dst.tny();
    if (elem_bytes == 8) aos_to_grid_kernel<double><<<grid_for(n, 256), 256, 0, st>>>(aos, dst);
    else aos_to_grid_kernel<float><<<grid_for(n, 256), 256, 0, st>>>(aos, dst);
    return cudaGetLastError();
}

cudaError_t launch_grid_to_aos(const DevGrid& src, int elem_bytes, double* aos, cudaStream_t st) {
    const long long n = (long long)src.tnx() * src.tny();
    if (elem_bytes == 8) grid_to_aos_kernel<double><<<grid_for(n, 256), 256, 0, st>>>(src, aos);
    else grid_to_aos_kernel<float><<<grid_for(n, 256), 256, 0, st>>>(src, aos);
    return cudaGetLastError();
}

cudaError_t launch_diagnostics(const DevGrid& g, int elem_bytes, double gamma, double dx, double dy,
                               double* scratch, double* out, cudaStream_t st) {
    if (elem_bytes == 8)
        diag_partial_kernel<double><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(g, gamma, dx, dy, scratch);
    else
        diag_partial_kernel<float><<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(g, gamma, dx, dy, scratch);
    diag_final_kernel<<<1, DIAG_THREADS, 0, st>>>(scratch, dx * dy, out);
    return cudaGetLastError();
}

cudaError_t launch_clock_init(DevClock* c, const unsigned long long* max0, cudaStream_t st) {
    clock_init_kernel<<<1, 1, 0, st>>>(c, max0);
    return cudaGetLastError();
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links only the CUDA runtime).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

bool rows_tensor_map(void* map64, const DevGrid& g, int elem_bytes, int box_cols, int box_rows) {
    const EncodeTiledFn fn = encode_tiled();
    if (!fn || (reinterpret_cast<std::uintptr_t>(g.data) % 16) || ((g.pitch * elem_bytes) % 16) ||
        ((g.plane * elem_bytes) % 16))
        return false;
    const cuuint64_t dims[3] = {(cuuint64_t)g.tnx(), (cuuint64_t)g.tny(), (cuuint64_t)NV};
    const cuuint64_t strides[2] = {(cuuint64_t)(g.pitch * elem_bytes), (cuuint64_t)(g.plane * elem_bytes)};
    const cuuint32_t box[3] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows, (cuuint32_t)NV};
    const cuuint32_t step[3] = {1, 1, 1};
    return fn(static_cast<CUtensorMap*>(map64),
              elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, g.data, dims,
              strides, box, step, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace mhd
