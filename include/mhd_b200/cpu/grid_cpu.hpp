// cpu/grid_cpu.hpp -- host AoS grid with ghost cells, the reference's Grid2D
// (head/cpu/grid_cpu.hpp:14-88): what make_n_grid returns and what
// Grid2DGPU::upload_from_aos reads.
#pragma once

#include <algorithm>
#include <cstddef>
#include <vector>

#include "../types.hpp"

class Grid2D {
public:
    Grid2D() = default;
    Grid2D(int nx, int ny, int ng, double x_min, double x_max, double y_min, double y_max)
        : nx_(nx), ny_(ny), ng_(ng), x_min_(x_min), x_max_(x_max), y_min_(y_min), y_max_(y_max) {
        dx_ = (x_max_ - x_min_) / static_cast<double>(nx_);
        dy_ = (y_max_ - y_min_) / static_cast<double>(ny_);
        U_.assign(static_cast<std::size_t>(total_nx()) * static_cast<std::size_t>(total_ny()), Conserved{});
    }

    int nx() const { return nx_; }
    int ny() const { return ny_; }
    int ng() const { return ng_; }
    int total_nx() const { return nx_ + 2 * ng_; }
    int total_ny() const { return ny_ + 2 * ng_; }
    double x_min() const { return x_min_; }
    double x_max() const { return x_max_; }
    double y_min() const { return y_min_; }
    double y_max() const { return y_max_; }
    double dx() const { return dx_; }
    double dy() const { return dy_; }
    int i_begin() const { return ng_; }
    int i_end() const { return ng_ + nx_; }
    int j_begin() const { return ng_; }
    int j_end() const { return ng_ + ny_; }
    double x_center(int i) const { return x_min_ + (static_cast<double>(i - ng_) + 0.5) * dx_; }
    double y_center(int j) const { return y_min_ + (static_cast<double>(j - ng_) + 0.5) * dy_; }

    Conserved& operator()(int i, int j) { return U_[index(i, j)]; }
    const Conserved& operator()(int i, int j) const { return U_[index(i, j)]; }
    std::vector<Conserved>& data() { return U_; }
    const std::vector<Conserved>& data() const { return U_; }
    void fill(const Conserved& v) { std::fill(U_.begin(), U_.end(), v); }

private:
    int nx_ = 0, ny_ = 0, ng_ = 0;
    double x_min_ = 0.0, x_max_ = 1.0, y_min_ = 0.0, y_max_ = 1.0;
    double dx_ = 0.0, dy_ = 0.0;
    std::vector<Conserved> U_;
    std::size_t index(int i, int j) const {
        return static_cast<std::size_t>(j) * static_cast<std::size_t>(total_nx()) + static_cast<std::size_t>(i);
    }
};
