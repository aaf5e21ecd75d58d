"""B200-native 2D Dedner GLM-MHD time step (drop-in for the reference's src/gpu path).

The numerics run in libmhd_b200.so (hand-written sm_100a CUDA kernels behind a
C ABI, include/mhd_b200.h); this package is the Python host-side binding.
"""
from .solver import (  # noqa: F401
    F32,
    F64,
    BoundaryConfig,
    BoundaryType,
    CaseConfig,
    CaseId,
    GpuWorkspace,
    Grid2DGPU,
    Limiter,
    RiemannSolver,
    advance_second_order_gpu,
    apply_boundary_gpu,
    compute_dt_gpu,
    free_gpu_workspace,
    get_case_config,
    get_n_case_config,
    init_gpu_workspace,
    initial_state_at,
    initialise,
    launch_count,
    make_n_grid,
    set_gpu_physics_ch,
    set_gpu_physics_gamma,
)
from ._lib import MhdError, load  # noqa: F401
