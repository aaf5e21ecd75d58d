// ic_kernels.cu -- initial data generated on the device, straight into a grid
// of either precision (no host array, no host->device copy).  Same case
// definitions as cases.cpp; the device sin / tanh / exp may differ from the
// host C library in the last bit, so mhd_initialise_device agrees with
// mhd_initialise to rounding, not bit for bit.
#include <cmath>

#include "../../include/mhd_b200.h"
#include "launch.h"

namespace mhd {
namespace {

struct C9 { double v[NV]; };

__device__ C9 make_state(double rho, double ux, double uy, double uz, double Bx, double By, double Bz, double p,
                         double gamma) {
    const double Bmag2 = Bx * Bx + By * By + Bz * Bz;
    const double ke = 0.5 * rho * (ux * ux + uy * uy + uz * uz);
    C9 c;
    c.v[0] = rho; c.v[1] = rho * ux; c.v[2] = rho * uy; c.v[3] = rho * uz;
    c.v[4] = Bx; c.v[5] = By; c.v[6] = Bz; c.v[7] = p / (gamma - 1.0) + ke + 0.5 * Bmag2; c.v[8] = 0.0;
    return c;
}

__device__ C9 state_at(int id, double x, double y) {
    const double PI = 3.14159265358979323846;
    switch (id) {
        case MHD_CASE_KELVIN_HELMHOLTZ: {
            const double ux = 5.0 * (tanh(20.0 * (y + 0.5)) - (tanh(20.0 * (y - 0.5)) + 1.0));
            const double uy = 0.25 * sin(2.0 * PI * x) *
                              (exp(-100.0 * (y + 0.5) * (y + 0.5)) - exp(-100.0 * (y - 0.5) * (y - 0.5)));
            return make_state(1.0, ux, uy, 0.0, 1.0, 0.0, 0.0, 50.0, 1.4);
        }
        case MHD_CASE_SHOCK_BUBBLE: {
            const double g = 1.4, rho_air = 1.29, rho_He = 0.214, p0 = 1.01325e5, Ms = 1.22;
            const double c1 = sqrt(g * p0 / rho_air), vs = Ms * c1;
            const double rho2 = rho_air * (g + 1.0) * Ms * Ms / ((g - 1.0) * Ms * Ms + 2.0);
            const double p2 = p0 * (2.0 * g * Ms * Ms - (g - 1.0)) / (g + 1.0);
            const double u2 = vs * (1.0 - rho_air / rho2);
            if (x < 0.005) return make_state(rho2, u2, 0, 0, 0, 0, 0, p2, g);
            const double r2 = (x - 0.035) * (x - 0.035) + (y - 0.0445) * (y - 0.0445);
            if (r2 < 0.025 * 0.025) return make_state(rho_He, 0, 0, 0, 0, 0, 0, p0, g);
            return make_state(rho_air, 0, 0, 0, 0, 0, 0, p0, g);
        }
        case MHD_CASE_BRIO_WU:
        case MHD_CASE_BRIO_WU_CFL08:
            if (x < 0.5) return make_state(1.0, 0, 0, 0, 0.75, 1.0, 0, 1.0, 2.0);
            return make_state(0.125, 0, 0, 0, 0.75, -1.0, 0, 0.1, 2.0);
        case MHD_CASE_ORSZAG_TANG: {
            const double g = 5.0 / 3.0;
            return make_state(g * g, -sin(y), sin(x), 0.0, -sin(y), sin(2.0 * x), 0.0, g, g);
        }
        case MHD_CASE_ORSZAG_TANG_UNIT: {
            const double B0 = 1.0 / sqrt(4.0 * PI);
            return make_state(25.0 / (36.0 * PI), -sin(2.0 * PI * y), sin(2.0 * PI * x), 0.0,
                              -B0 * sin(2.0 * PI * y), B0 * sin(4.0 * PI * x), 0.0, 5.0 / (12.0 * PI), 5.0 / 3.0);
        }
        default: {  // MHD_CASE_SHOCK_BUBBLE_MHD
            const double g = 5.0 / 3.0, M = 10.0, By = 2.0 / sqrt(4.0 * PI);
            const double vs = M * sqrt(g);
            const double rho2 = (g + 1.0) * M * M / ((g - 1.0) * M * M + 2.0);
            const double p2 = (2.0 * g * M * M - (g - 1.0)) / (g + 1.0);
            const double u2 = vs * (1.0 - 1.0 / rho2);
            if (x < 0.6) return make_state(rho2, u2, 0, 0, 0, By, 0, p2, g);
            const double r2 = (x - 0.8) * (x - 0.8) + (y - 0.5) * (y - 0.5);
            if (r2 < 0.15 * 0.15) return make_state(10.0, 0, 0, 0, 0, By, 0, 1.0, g);
            return make_state(1.0, 0, 0, 0, 0, By, 0, 1.0, g);
        }
    }
}

template <typename R>
__global__ void ic_kernel(DevGrid g, int id, double x0, double y0, double dx, double dy) {
    const int tx = g.tnx(), ty = g.tny();
    const long long total = (long long)tx * ty;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(k / tx), i = (int)(k - (long long)j * tx);
        const double x = x0 + ((double)(i - g.ng) + 0.5) * dx;
        const double y = y0 + ((double)(j - g.ng) + 0.5) * dy;
        const C9 c = state_at(id, x, y);
        R* b = static_cast<R*>(g.data) + g.idx(i, j);
#pragma unroll
        for (int f = 0; f < NV; ++f) b[f * g.plane] = static_cast<R>(c.v[f]);
    }
}

struct OTParams {
    double b0, gamma;
    double amp[16];
    int has_amp;
};

// Fourier modes of the perturbations (mhd_initialise_orszag_tang).
__device__ __constant__ int kModeX[8] = {1, 0, 1, 1, 2, 0, 2, 1};
__device__ __constant__ int kModeY[8] = {0, 1, 1, -1, 0, 2, 1, 2};

template <typename R>
__global__ void ot_kernel(DevGrid g, OTParams prm, double x0, double y0, double dx, double dy) {
    const double PI = 3.14159265358979323846;
    const int tx = g.tnx(), ty = g.tny();
    const long long total = (long long)tx * ty;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(k / tx), i = (int)(k - (long long)j * tx);
        const double x = x0 + ((double)(i - g.ng) + 0.5) * dx;
        const double y = y0 + ((double)(j - g.ng) + 0.5) * dy;
        double u = -sin(2.0 * PI * y), v = sin(2.0 * PI * x);
        double bx = -prm.b0 * sin(2.0 * PI * y), by = prm.b0 * sin(4.0 * PI * x);
        if (prm.has_amp) {
            for (int m = 0; m < 8; ++m) {
                const double mx = kModeX[m], my = kModeY[m];
                const double s = sin(2.0 * PI * (mx * x + my * y)) / sqrt(mx * mx + my * my);
                u -= prm.amp[m] * s * my;
                v += prm.amp[m] * s * mx;
                bx -= prm.amp[8 + m] * s * my;
                by += prm.amp[8 + m] * s * mx;
            }
        }
        const C9 c = make_state(25.0 / (36.0 * PI), u, v, 0.0, bx, by, 0.0, 5.0 / (12.0 * PI), prm.gamma);
        R* b = static_cast<R*>(g.data) + g.idx(i, j);
#pragma unroll
        for (int f = 0; f < NV; ++f) b[f * g.plane] = static_cast<R>(c.v[f]);
    }
}

}  // namespace

cudaError_t launch_initialise_ot(const DevGrid& g, int elem_bytes, double b0, double gamma, const double* amp,
                                 double x0, double y0, double dx, double dy, cudaStream_t st) {
    OTParams prm{};
    prm.b0 = b0;
    prm.gamma = gamma;
    prm.has_amp = amp != nullptr;
    if (amp)
        for (int k = 0; k < 16; ++k) prm.amp[k] = amp[k];
    const long long n = (long long)g.tnx() * g.tny();
    long long blocks = (n + 255) / 256;
    if (blocks > 65535LL * 8) blocks = 65535LL * 8;
    if (elem_bytes == 8) ot_kernel<double><<<(unsigned)blocks, 256, 0, st>>>(g, prm, x0, y0, dx, dy);
    else ot_kernel<float><<<(unsigned)blocks, 256, 0, st>>>(g, prm, x0, y0, dx, dy);
    return cudaGetLastError();
}

cudaError_t launch_initialise(const DevGrid& g, int elem_bytes, int id, double x0, double y0, double dx, double dy,
                              cudaStream_t st) {
    const long long n = (long long)g.tnx() * g.tny();
    long long blocks = (n + 255) / 256;
    if (blocks > 65535LL * 8) blocks = 65535LL * 8;
    if (elem_bytes == 8) ic_kernel<double><<<(unsigned)blocks, 256, 0, st>>>(g, id, x0, y0, dx, dy);
    else ic_kernel<float><<<(unsigned)blocks, 256, 0, st>>>(g, id, x0, y0, dx, dy);
    return cudaGetLastError();
}

}  // namespace mhd
