// gpu/boundary_gpu.cuh -- boundary conditions on a device grid
// (head/gpu/boundary_gpu.cuh:9-14): periodic, transmissive, reflecting,
// Dirichlet (ghost cells left as they are), all nine fields, in place.
#pragma once

#include "../test_cases.hpp"
#include "grid_gpu.cuh"

void apply_boundary_gpu(Grid2DGPU& grid, const BoundaryConfig& bc);

inline void apply_transmissive_boundary_gpu(Grid2DGPU& grid) { apply_boundary_gpu(grid, BoundaryConfig{}); }
