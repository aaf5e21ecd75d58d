// gpu/grid_gpu.cuh -- the reference's device grid (head/gpu/grid_gpu.cuh:17-305)
// over libmhd_b200's storage: one padded slab of nine SoA planes per grid.
//
// Same constructor, accessors, upload_from_aos / download_to_aos, swap and
// views as the reference.  The views carry `pitch` (elements per row) and
// `plane` (elements per field), and flat_index(i, j) = j * pitch + i; field
// pointers are base + f * plane.  An optional precision argument selects the
// FP32-bulk storage (default FP64, the reference's).
#pragma once

#include <cstddef>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../mhd_b200.h"
#include "../types.hpp"

enum class Precision { FP64 = MHD_F64, FP32 = MHD_F32 };

inline void mhd_throw_if(int rc, const char* what) {
    if (rc != MHD_OK) throw std::runtime_error(std::string(what) + ": " + mhd_last_error());
}

class Grid2DGPU {
public:
    Grid2DGPU() { g_ = mhd_grid{}; }
    Grid2DGPU(int nx, int ny, int ng, double x_min, double x_max, double y_min, double y_max,
              Precision prec = Precision::FP64) {
        g_ = mhd_grid{};
        allocate(nx, ny, ng, x_min, x_max, y_min, y_max, prec);
    }
    Grid2DGPU(const Grid2DGPU&) = delete;
    Grid2DGPU& operator=(const Grid2DGPU&) = delete;
    Grid2DGPU(Grid2DGPU&& o) noexcept : g_(o.g_) { o.g_ = mhd_grid{}; }
    Grid2DGPU& operator=(Grid2DGPU&& o) noexcept {
        if (this != &o) {
            release();
            g_ = o.g_;
            o.g_ = mhd_grid{};
        }
        return *this;
    }
    ~Grid2DGPU() { release(); }

    void allocate(int nx, int ny, int ng, double x_min, double x_max, double y_min, double y_max,
                  Precision prec = Precision::FP64) {
        release();
        mhd_throw_if(mhd_grid_alloc(&g_, nx, ny, ng, static_cast<int>(prec), x_min, x_max, y_min, y_max),
                     "Grid2DGPU::allocate");
    }
    void release() {
        if (g_.data) mhd_grid_free(&g_);
        g_ = mhd_grid{};
    }

    int nx() const { return g_.nx; }
    int ny() const { return g_.ny; }
    int ng() const { return g_.ng; }
    int total_nx() const { return g_.nx + 2 * g_.ng; }
    int total_ny() const { return g_.ny + 2 * g_.ng; }
    double x_min() const { return g_.x_min; }
    double x_max() const { return g_.x_max; }
    double y_min() const { return g_.y_min; }
    double y_max() const { return g_.y_max; }
    double dx() const { return (g_.x_max - g_.x_min) / static_cast<double>(g_.nx); }
    double dy() const { return (g_.y_max - g_.y_min) / static_cast<double>(g_.ny); }
    int i_begin() const { return g_.ng; }
    int i_end() const { return g_.ng + g_.nx; }
    int j_begin() const { return g_.ng; }
    int j_end() const { return g_.ng + g_.ny; }
    std::size_t num_cells() const { return static_cast<std::size_t>(total_nx()) * total_ny(); }
    Precision precision() const { return static_cast<Precision>(g_.dtype); }
    long long pitch() const { return g_.pitch; }
    long long plane() const { return g_.plane; }

    // FP64 field pointers (an FP32 grid has no double planes: these return null)
    double* field_ptr(int f) {
        return g_.dtype == MHD_F64 ? static_cast<double*>(g_.data) + static_cast<long long>(f) * g_.plane : nullptr;
    }
    const double* field_ptr(int f) const { return const_cast<Grid2DGPU*>(this)->field_ptr(f); }
    double* rho_ptr() { return field_ptr(0); }
    double* rhou_ptr() { return field_ptr(1); }
    double* rhov_ptr() { return field_ptr(2); }
    double* rhow_ptr() { return field_ptr(3); }
    double* Bx_ptr() { return field_ptr(4); }
    double* By_ptr() { return field_ptr(5); }
    double* Bz_ptr() { return field_ptr(6); }
    double* E_ptr() { return field_ptr(7); }
    double* psi_ptr() { return field_ptr(8); }
    const double* rho_ptr() const { return field_ptr(0); }
    const double* rhou_ptr() const { return field_ptr(1); }
    const double* rhov_ptr() const { return field_ptr(2); }
    const double* rhow_ptr() const { return field_ptr(3); }
    const double* Bx_ptr() const { return field_ptr(4); }
    const double* By_ptr() const { return field_ptr(5); }
    const double* Bz_ptr() const { return field_ptr(6); }
    const double* E_ptr() const { return field_ptr(7); }
    const double* psi_ptr() const { return field_ptr(8); }

    // host AoS <-> device (head/gpu/grid_gpu.cuh:120-177); the transpose runs on the GPU
    void upload_from_aos(const std::vector<Conserved>& host) {
        if (host.size() != num_cells()) throw std::runtime_error("upload_from_aos: size mismatch");
        mhd_throw_if(mhd_grid_upload_aos(&g_, &host[0].rho), "upload_from_aos");
    }
    void download_to_aos(std::vector<Conserved>& host) const {
        host.resize(num_cells());
        mhd_throw_if(mhd_grid_download_aos(&g_, &host[0].rho), "download_to_aos");
    }
    void swap(Grid2DGPU& o) { std::swap(g_, o.g_); }

    mhd_grid* c_grid() { return &g_; }
    const mhd_grid* c_grid() const { return &g_; }

private:
    mhd_grid g_;
};

// Non-owning views (head/gpu/grid_gpu.cuh:228-277), FP64 grids.
struct Grid2DGPUView {
    int nx, ny, ng;
    double x_min, x_max, y_min, y_max, dx, dy;
    double *rho, *rhou, *rhov, *rhow, *Bx, *By, *Bz, *E, *psi;
    long long pitch;
    HD int total_nx() const { return nx + 2 * ng; }
    HD int total_ny() const { return ny + 2 * ng; }
    HD int i_begin() const { return ng; }
    HD int i_end() const { return ng + nx; }
    HD int j_begin() const { return ng; }
    HD int j_end() const { return ng + ny; }
    HD long long flat_index(int i, int j) const { return static_cast<long long>(j) * pitch + i; }
};

struct ConstGrid2DGPUView {
    int nx, ny, ng;
    double x_min, x_max, y_min, y_max, dx, dy;
    const double *rho, *rhou, *rhov, *rhow, *Bx, *By, *Bz, *E, *psi;
    long long pitch;
    HD int total_nx() const { return nx + 2 * ng; }
    HD int total_ny() const { return ny + 2 * ng; }
    HD int i_begin() const { return ng; }
    HD int i_end() const { return ng + nx; }
    HD int j_begin() const { return ng; }
    HD int j_end() const { return ng + ny; }
    HD long long flat_index(int i, int j) const { return static_cast<long long>(j) * pitch + i; }
};

inline Grid2DGPUView make_view(Grid2DGPU& g) {
    return Grid2DGPUView{g.nx(), g.ny(), g.ng(), g.x_min(), g.x_max(), g.y_min(), g.y_max(), g.dx(), g.dy(),
                         g.rho_ptr(), g.rhou_ptr(), g.rhov_ptr(), g.rhow_ptr(), g.Bx_ptr(), g.By_ptr(),
                         g.Bz_ptr(), g.E_ptr(), g.psi_ptr(), g.pitch()};
}

inline ConstGrid2DGPUView make_view(const Grid2DGPU& g) {
    return ConstGrid2DGPUView{g.nx(), g.ny(), g.ng(), g.x_min(), g.x_max(), g.y_min(), g.y_max(), g.dx(), g.dy(),
                              g.rho_ptr(), g.rhou_ptr(), g.rhov_ptr(), g.rhow_ptr(), g.Bx_ptr(), g.By_ptr(),
                              g.Bz_ptr(), g.E_ptr(), g.psi_ptr(), g.pitch()};
}
