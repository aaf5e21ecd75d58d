/*
 * mhd_b200.h -- C ABI of the B200-native 2D Dedner GLM-MHD step.
 *
 * This is the drop-in boundary for the reference's src/gpu path
 * (HarryKKKKK/MHD_gpu_acc).  Every entry point takes plain pointers, sizes
 * and scalars; none exits the process.  Each returns MHD_OK (0) or a negative
 * MHD_ERR_* code; mhd_last_error() returns a message for the calling thread.
 * The C++ drop-in headers under include/mhd_b200/ (types.hpp, riemann.hpp,
 * test_cases.hpp, gpu/grid_gpu.cuh, gpu/solver_gpu.cuh, gpu/boundary_gpu.cuh)
 * implement the reference's C++ API on top of these functions.
 *
 * Device state layout ("grid"): one allocation holding 9 SoA planes in the
 * field order of the reference's Conserved (head/types.hpp:16-41):
 * rho, rhou, rhov, rhow, Bx, By, Bz, E, psi.  Cell (i, j) -- ghosts included,
 * as in Grid2DGPUView::flat_index (head/gpu/grid_gpu.cuh:314-316) -- of field f
 * is element  f*plane + j*pitch + i.  mhd_grid_alloc pads pitch and plane to
 * 256 bytes.  Host arrays exchanged with upload/download are dense FP64 SoA of
 * shape (9, ny+2ng, nx+2ng) (or the reference's AoS Conserved array for the
 * *_aos variants).
 */
#ifndef MHD_B200_H
#define MHD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define MHD_NV 9
#define MHD_MAX_NG 4

/* ---- error codes ---- */
#define MHD_OK 0
#define MHD_ERR_ARG (-1)       /* invalid argument / size / layout */
#define MHD_ERR_CUDA (-2)      /* a CUDA runtime call failed */
#define MHD_ERR_NO_SPEED (-3)  /* max wave speed <= 0 (the reference throws: src/cpu/solver_cpu.cpp:304-306) */
#define MHD_ERR_BAD_DT (-4)    /* dt non-finite or <= 0 (scripts/gpu/main_gpu.cu:219-223) */
#define MHD_ERR_TINY_DT (-5)   /* dt < 1e-8 t_end (scripts/gpu/main_gpu.cu:224-232) */
#define MHD_ERR_STATE (-6)     /* workspace not initialised / mismatched (src/gpu/solver_gpu.cu:579-580, 626-627) */
#define MHD_ERR_NOMEM (-7)     /* device or host allocation failed */
#define MHD_ERR_TIMEOUT (-8)   /* a bounded device wait gave up */

/* ---- enumerations: values equal the reference's enums ---- */
/* RiemannSolver, head/riemann.hpp:23 */
#define MHD_HLL 0
#define MHD_HLLC 1
#define MHD_HLLD 2
#define MHD_FORCE 3
/* BoundaryType, head/test_cases.hpp:11-16 */
#define MHD_BC_PERIODIC 0
#define MHD_BC_TRANSMISSIVE 1
#define MHD_BC_REFLECTING 2
#define MHD_BC_DIRICHLET 3
/* slope limiter: minmod is the reference's (src/cpu/solver_cpu.cpp:26-43); van Leer is new */
#define MHD_LIMITER_MINMOD 0
#define MHD_LIMITER_VANLEER 1
/* storage / arithmetic precision */
#define MHD_F64 0 /* the plain step: matches the reference CPU FP64 path */
#define MHD_F32 1 /* FP32-bulk step with the flagged FP64 pressure recovery */
/* CaseId, head/test_cases.hpp:28-33, plus the configurations this build adds */
#define MHD_CASE_KELVIN_HELMHOLTZ 0
#define MHD_CASE_SHOCK_BUBBLE 1
#define MHD_CASE_BRIO_WU 2
#define MHD_CASE_ORSZAG_TANG 3
#define MHD_CASE_ORSZAG_TANG_UNIT 4   /* Orszag-Tang on periodic [0,1]^2, rho = 25/(36 pi), p = 5/(12 pi) */
#define MHD_CASE_SHOCK_BUBBLE_MHD 5   /* Mach-10 MHD shock - dense bubble on [0,1]^2, gamma 5/3 */
#define MHD_CASE_BRIO_WU_CFL08 6      /* Brio-Wu 800x4, CFL 0.8, all transmissive */

/* ---- device grid (Grid2DGPU / Grid2DGPUView, head/gpu/grid_gpu.cuh:17-277) ---- */
typedef struct mhd_grid {
    void* data;       /* device pointer to field 0, cell (0, 0) */
    long long pitch;  /* elements per row, >= nx + 2 ng */
    long long plane;  /* elements per field plane, >= pitch * (ny + 2 ng) */
    int nx, ny, ng;   /* interior cells and ghost layers (2 <= ng <= MHD_MAX_NG) */
    int dtype;        /* MHD_F64 or MHD_F32 */
    double x_min, x_max, y_min, y_max;  /* dx = (x_max - x_min) / nx, dy likewise */
} mhd_grid;

/* Replaces Grid2DGPU::allocate (head/gpu/grid_gpu.cuh:39-58): one padded slab. */
int mhd_grid_alloc(mhd_grid* g, int nx, int ny, int ng, int dtype, double x_min, double x_max, double y_min,
                   double y_max);
/* Replaces Grid2DGPU::release (head/gpu/grid_gpu.cuh:60-77). */
int mhd_grid_free(mhd_grid* g);
/* Replaces Grid2DGPU::upload_from_aos / download_to_aos (head/gpu/grid_gpu.cuh:120-177),
 * synchronous.  `host` is dense FP64 SoA (9, ny+2ng, nx+2ng); FP32 grids convert on the device. */
int mhd_grid_upload(const mhd_grid* g, const double* host);
int mhd_grid_download(const mhd_grid* g, double* host);
/* Same with the reference's AoS Conserved array (9 doubles per cell, row-major). */
int mhd_grid_upload_aos(const mhd_grid* g, const double* host_aos);
int mhd_grid_download_aos(const mhd_grid* g, double* host_aos);
/* Replaces Grid2DGPU::swap (head/gpu/grid_gpu.cuh:179-189). */
int mhd_grid_swap(mhd_grid* a, mhd_grid* b);

/* ---- workspace (GpuWorkspace, head/gpu/solver_gpu.cuh:9-19) ---- */
typedef struct mhd_workspace mhd_workspace;

/* Replaces init_gpu_workspace (src/gpu/solver_gpu.cu:549-566). */
int mhd_workspace_create(const mhd_grid* g, mhd_workspace** ws);
/* Replaces free_gpu_workspace (src/gpu/solver_gpu.cu:568-573). */
int mhd_workspace_destroy(mhd_workspace* ws);
/* All work of this workspace is queued on `stream` (a cudaStream_t; NULL = legacy default). */
int mhd_workspace_set_stream(mhd_workspace* ws, void* stream);
/* Replaces set_gpu_physics_gamma (src/gpu/solver_gpu.cu:536-539); per workspace, not process-global. */
int mhd_set_gamma(mhd_workspace* ws, double gamma);
/* Replaces set_gpu_physics_ch (src/gpu/solver_gpu.cu:541-544). */
int mhd_set_ch(mhd_workspace* ws, double ch);
int mhd_get_ch(const mhd_workspace* ws, double* ch);
/* Slope limiter for later steps (default minmod, as the reference). */
int mhd_set_limiter(mhd_workspace* ws, int limiter);
/* GLM damping ratio c_r = c_p^2 / c_h (default 0.18, head/physics.hpp:39). */
int mhd_set_cr(mhd_workspace* ws, double cr);
/* Launch shape of the sweeps (no reference counterpart; results do not depend
 * on it): the x-sweep work per warp, xrpw (0 = the precision's default: 8 for
 * FP32, 16 for FP64; one warp marches a row segment of 128 * xrpw - 4 cells,
 * the last quarter of each row in segments of a third of that), the height of
 * the row band one y-sweep warp marches down (0 = the precision's default: 28
 * rows for FP32, 56 for FP64; the last eighth of the rows in bands of a half
 * and a quarter of that), and how the y-sweep gets its rows: ystage 0
 * (default) = per-thread loads, 1 = TMA boxes staged in shared memory, one band
 * height (same results; on B200 at 4096^2 FP32 the staged sweep measured
 * 0.77 ms against 0.62 ms for per-thread loads with one band height). */
int mhd_set_sweep_shape(mhd_workspace* ws, int xrpw, int yband, int ystage);
/* Limit, in nanoseconds of the GPU's global timer, of each wait of the
 * TMA-staged y-sweep (ystage 1) for a box of rows to land; 0 restores the
 * default of 2 s.  A wait that runs out stops the sweep: the CTA waits (with
 * the full 2 s limit) for the copies it has in flight, the step's output is
 * left incomplete, and the next synchronising call on the workspace
 * (mhd_compute_dt, mhd_synchronize, mhd_run ...) returns MHD_ERR_TIMEOUT.
 * Setting a limit of a few nanoseconds makes that path run on purpose (tests). */
int mhd_set_tma_wait_limit(mhd_workspace* ws, unsigned long long ns);
/* Cell spacing the step and compute_dt use instead of the grid's
 * (x_max - x_min) / nx and (y_max - y_min) / ny; (0, 0) restores those.  A slab
 * of a larger grid takes the global spacing, so that its steps equal the
 * unsplit grid's bit for bit (no counterpart in the reference). */
int mhd_set_spacing(mhd_workspace* ws, double dx, double dy);

/* Replaces compute_dt_gpu (src/gpu/solver_gpu.cu:578-605): CFL maximum over the
 * interior floored by the current ch; sets ch to it and returns
 * dt = cfl * min(dx, dy) / max.  Returns MHD_ERR_NO_SPEED where the reference
 * CPU path throws (the reference GPU returned DBL_MAX there); *dt is then DBL_MAX. */
int mhd_compute_dt(mhd_workspace* ws, const mhd_grid* g, double cfl, double* dt);

/* Replaces advance_second_order_gpu (src/gpu/solver_gpu.cu:617-690): x-sweep
 * Uold -> Utmp, boundary conditions, y-sweep Utmp -> Unew, boundary conditions,
 * psi damping -- one fused kernel per sweep.  bc = {left, right, bottom, top}. */
int mhd_advance(mhd_workspace* ws, const mhd_grid* Uold, mhd_grid* Utmp, mhd_grid* Unew, double dt, int solver,
                const int* bc);

/* One sweep of mhd_advance (no reference counterpart): dir 0 = the x-sweep
 * in -> out, dir 1 = the y-sweep in -> out with the psi damping, each with its
 * boundary fill, at dt and the workspace's ch.  mhd_advance is the x-sweep
 * followed by the y-sweep; between them a caller may rewrite ghost rows of the
 * x-swept state (the halo exchange of a grid split into y-slabs). */
int mhd_sweep(mhd_workspace* ws, const mhd_grid* in, mhd_grid* out, double dt, int solver, const int* bc, int dir);
/* The CFL maximum of mhd_compute_dt (interior, floored by the current ch)
 * without changing ch or forming dt: the per-slab term of a global maximum. */
int mhd_max_speed(mhd_workspace* ws, const mhd_grid* g, double* vmax);
/* Copies nrows full storage rows (ghost columns included) of all 9 fields,
 * src rows [src_row, src_row + nrows) -> dst rows [dst_row, ...), between grids
 * of equal nx, ng, dtype and pitch, asynchronously on `stream`. */
int mhd_grid_copy_rows(const mhd_grid* src, int src_row, mhd_grid* dst, int dst_row, int nrows, void* stream);

/* Replaces apply_boundary_gpu (src/gpu/boundary_gpu.cu:158-176), in place. */
int mhd_apply_boundary(mhd_workspace* ws, mhd_grid* g, const int* bc);

/* One split step (as mhd_advance) that allocates no device memory.  No
 * counterpart in the reference.  For callers that cannot call cudaMalloc -- an
 * application whose own pool allocator owns all device memory, or a loop that
 * cannot absorb the synchronisation an allocation may imply -- and therefore
 * cannot create a workspace or an intermediate state: the x-swept state lives
 * in a fixed 32 MiB device array inside the library (held by every GPU that
 * loads it, until exit).  Grids whose intermediate state would not fit
 * (9 planes of pitch x (ny+2ng) elements, pitch = nx+2ng rounded up to 256
 * bytes) are rejected with MHD_ERR_ARG.  The array's device address is looked
 * up on the first call on each device (make that call before any stream
 * capture) and kept until exit, so the device must not be reset between calls.
 * All calls share the array: calls that can overlap on the GPU race and must
 * be serialised by the caller.  gamma, ch and cr are the values a
 * workspace would hold; `stream` is a cudaStream_t (NULL = legacy default). */
#define MHD_NOALLOC_SCRATCH_BYTES (32u << 20)
int mhd_advance_noalloc(const mhd_grid* Uold, mhd_grid* Unew, double gamma, double ch, double cr, double dt,
                        int solver, int limiter, const int* bc, void* stream);

/* ---- device-resident run: the driver loop of scripts/gpu/main_gpu.cu:208-264 ----
 * The time step, its clamp to t_end and the dt guards are evaluated on the GPU
 * (the CFL maximum is folded into the y-sweep), and the step loop is captured
 * once as a CUDA graph of two steps.  U holds the state on entry and exit; T is
 * the intermediate (x-swept) state.  Stops after max_steps steps (if > 0) or at
 * t_end, whichever comes first. */
typedef struct mhd_run_info {
    double t;          /* simulated time reached */
    double last_dt;    /* dt of the last step taken */
    double ch;         /* ch_glm after the last step */
    int steps;         /* steps taken */
    int status;        /* MHD_OK, or MHD_ERR_NO_SPEED / _BAD_DT / _TINY_DT (the step loop stopped) */
    unsigned int fallbacks;  /* cells reverted by the non-finite update guard */
    unsigned int pad_;
} mhd_run_info;
int mhd_run(mhd_workspace* ws, mhd_grid* U, mhd_grid* T, double cfl, double t_end, int max_steps, int solver,
            const int* bc, mhd_run_info* info);

/* ---- device-clocked sweeps: the pieces of a step a caller composes itself
 * (one grid split into y-slabs over several GPUs), with dt, c_h and the psi
 * damping factor evaluated on the GPU as in mhd_run, so that a step makes no
 * host round trip (no reference counterpart: the reference reads dt back to
 * the host every step, src/gpu/solver_gpu.cu:578-605) ----
 * mhd_clock_start: resets the workspace's device clock (t = 0, no steps) and
 * puts U's CFL maximum, floored by the workspace's c_h, in clock slot 0;
 * asynchronous on the workspace stream.  cfl and t_end apply to the sweeps
 * that follow.
 * mhd_clock_slot: device address of clock slot `parity` -- the maximum signal
 * speed as the bit pattern of a non-negative double, which orders like an
 * unsigned (and a signed) 64-bit integer -- so that a caller can max-reduce it
 * across slabs or ranks between steps.
 * mhd_sweep_clocked: one sweep of step n (parity = n % 2) with dt, c_h and
 * damping from slot parity (a step past t_end or with a bad dt is skipped and
 * the clock's status says why).  The x-sweep (dir 0) clears slot parity ^ 1;
 * the y-sweep (dir 1) folds the output's CFL maximum into it.  A y-sweep may
 * be cut into launches over interior row windows [row0, row0 + nrows)
 * (nrows 0: every row): MHD_SWEEP_NO_GATHER skips the copy of Dirichlet ghost
 * cells from the input and MHD_SWEEP_NO_ADVANCE leaves the clock's time and
 * step count alone, so exactly one launch of a step should do each.
 * mhd_clock_read: reads the clock into *info, synchronising the workspace
 * stream, and sets the workspace's c_h to the last step's. */
#define MHD_SWEEP_NO_GATHER 1
#define MHD_SWEEP_NO_ADVANCE 2
int mhd_clock_start(mhd_workspace* ws, const mhd_grid* U, double cfl, double t_end);
int mhd_clock_slot(mhd_workspace* ws, int parity, void** dptr);
int mhd_sweep_clocked(mhd_workspace* ws, const mhd_grid* in, mhd_grid* out, int solver, const int* bc, int dir,
                      int parity, int row0, int nrows, int flags);
int mhd_clock_read(mhd_workspace* ws, mhd_run_info* info);

/* ---- binary state dump / load (no reference counterpart: the reference has
 * write-only CSV snapshots, scripts/cpu/main_cpu.cpp:36-91) ----
 * mhd_state_save writes grid g -- 9 planes in its own precision, ghost cells
 * included -- with the scalars a resumed run needs to `path` (through
 * "<path>.tmp" and a rename); mhd_state_load reads such a file into an
 * allocated grid of the same nx, ny, ng and precision, bit for bit (another
 * shape or precision: MHD_ERR_ARG).  meta may be NULL (saved as zeros / not
 * returned).  Both are synchronous on the legacy stream.  A run resumes by
 * loading the state and setting c_h (mhd_set_ch) to meta.ch. */
typedef struct mhd_state_meta {
    double t;          /* simulated time of the state */
    double ch;         /* GLM c_h carried into the next step */
    long long steps;   /* steps taken */
} mhd_state_meta;
int mhd_state_save(const mhd_grid* g, const char* path, const mhd_state_meta* meta);
int mhd_state_load(mhd_grid* g, const char* path, mhd_state_meta* meta);


/* Measurement aid (no reference counterpart): advances U by nrep device-clock
 * steps like mhd_run, launching each sweep separately between CUDA events on the
 * workspace stream; ms_out[0] / ms_out[1] receive the mean x- / y-sweep kernel
 * time in milliseconds. */
int mhd_profile_sweeps(mhd_workspace* ws, mhd_grid* U, mhd_grid* T, double cfl, double t_end, int solver,
                       const int* bc, int nrep, float* ms_out);

/* Asynchronous host <-> device copies through the workspace's stream and staging
 * buffer (pinned host memory gives full bandwidth).  Same layout as mhd_grid_upload. */
int mhd_upload(mhd_workspace* ws, const mhd_grid* g, const double* host);
int mhd_download(mhd_workspace* ws, const mhd_grid* g, double* host);
/* The same for an FP32 grid with FP32 host arrays (dense (9, ny+2ng, nx+2ng)):
 * half the bytes of the FP64 host format and no device-side conversion.  No
 * reference counterpart. */
int mhd_upload_f32(mhd_workspace* ws, const mhd_grid* g, const float* host);
int mhd_download_f32(mhd_workspace* ws, const mhd_grid* g, float* host);
int mhd_synchronize(mhd_workspace* ws);

/* FP64 diagnostics of a state: out[0] = sum rho dA, out[1] = sum E dA,
 * out[2] = sum |div B| dA (central differences), out[3] = max |div B|,
 * out[4] = min rho, out[5] = min p.  Deterministic reduction order. */
int mhd_diagnostics(mhd_workspace* ws, const mhd_grid* g, double* out6);

/* ---- test cases and initial data (head/test_cases.hpp, head/init.hpp) ---- */
/* get_n_case_config (src/test_cases.cpp:275-282) for case_id, scale n.
 * out14: nx, ny, ng, x_min, x_max, y_min, y_max, cfl, t_end, gamma, bc[4]. */
int mhd_case_config(int case_id, int n, double* out14);
/* initial_state_at (src/test_cases.cpp:288-296): 9 conserved values at (x, y). */
int mhd_initial_state(int case_id, double x, double y, double* out9);
/* initialise_grid (src/init.cpp:34-43): evaluates the initial state at every
 * cell centre, ghosts included, into dense host SoA (9, ny+2ng, nx+2ng). */
int mhd_initialise(int case_id, int nx, int ny, int ng, double x_min, double x_max, double y_min, double y_max,
                   double* host);

/* riemann_flux with explicit c_h (head/riemann.hpp:568-592) on one face, on the
 * host, FP64: the functions the FP64 kernels run.  dir 0 = x, 1 = y. */
int mhd_riemann_flux(const double* UL, const double* UR, int dir, int solver, double ch, double gamma, double* F);
/* riemann_flux (head/riemann.hpp:568-592) of n independent faces on the GPU,
 * with the sweep kernels' own solver functions of the given precision:
 * MHD_F64 (the FP64 step's, bit-equal to mhd_riemann_flux) or MHD_F32 (the
 * FP32-bulk step's: inputs rounded to FP32, cons->prim with the flagged FP64
 * pressure branch, FP32 HLLD degeneracy rule).  UL, UR and F are DEVICE arrays
 * of n x 9 doubles (face k's conserved states / flux at [9k, 9k+9)).  Runs on
 * the workspace's stream (ws NULL: legacy stream, synchronous). */
int mhd_riemann_flux_device(mhd_workspace* ws, int dtype, long long n, const double* UL, const double* UR, int dir,
                            int solver, double ch, double gamma, double* F);

/* Initial data of case_id evaluated on the device at every cell centre of g
 * (ghosts included), without a host array.  Agrees with mhd_initialise to the
 * rounding of the device sin/tanh/exp.  ws may be NULL (then synchronous on the
 * legacy stream). */
int mhd_initialise_device(mhd_workspace* ws, const mhd_grid* g, int case_id);

/* Orszag-Tang on [0,1]^2 with field amplitude b0 (1/sqrt(4 pi) in the standard
 * case) and adiabatic exponent gamma: rho = 25/(36 pi), p = 5/(12 pi),
 * v = (-sin 2pi y, sin 2pi x), B = b0 (-sin 2pi y, sin 4pi x), psi = 0, plus,
 * when amp != NULL (16 values), divergence-free Fourier perturbations:
 * with theta_j = 2 pi (m_j . x) and the modes m_j = (1,0), (0,1), (1,1),
 * (1,-1), (2,0), (0,2), (2,1), (1,2) (j = 0..7),
 *   du = -sum_j amp[j]   sin(theta_j) m_jy/|m_j|,  dv = sum_j amp[j]   sin(theta_j) m_jx/|m_j|,
 *   dBx = -sum_j amp[8+j] sin(theta_j) m_jy/|m_j|, dBy = sum_j amp[8+j] sin(theta_j) m_jx/|m_j|.
 * Evaluated on the device at every cell centre of g (ghosts included). */
int mhd_initialise_orszag_tang(mhd_workspace* ws, const mhd_grid* g, double b0, double gamma, const double* amp);

/* ---- batched instances (no reference counterpart) ----
 * Many independent problems of uneven size advanced together: one persistent
 * launch per sweep phase over a global tile work list, CUDA-graph step loop,
 * per-instance gamma, CFL, c_r, boundary types, t_end, dt and c_h.  Solver,
 * limiter and precision are shared.  Dirichlet sides are not supported. */
typedef struct mhd_instance_desc {
    int nx, ny, ng;
    int bc[4];
    double x_min, x_max, y_min, y_max;
    double gamma, cfl, cr, t_end;
} mhd_instance_desc;
/* Launch shape of the batched sweeps: x-sweep work per warp (xrpw: row
 * segments of 128 * xrpw - 4 cells), y-sweep segment length, persistent CTAs
 * of each phase (0 = default from the SM count). */
typedef struct mhd_batch_tuning {
    int xrpw, yseg, ctas_x, ctas_y;
} mhd_batch_tuning;
typedef struct mhd_batch mhd_batch;

int mhd_batch_create(const mhd_instance_desc* desc, int n, int dtype, int solver, int limiter, mhd_batch** out);
int mhd_batch_destroy(mhd_batch* b);
int mhd_batch_set_stream(mhd_batch* b, void* stream);
/* The state grid of instance i (device memory owned by the batch): fill it with
 * mhd_grid_upload / mhd_initialise_device / mhd_initialise_orszag_tang, read it
 * with mhd_grid_download. */
int mhd_batch_grid(const mhd_batch* b, int i, mhd_grid* out);
/* Total interior cells of all instances. */
int mhd_batch_cells(const mhd_batch* b, long long* cells);
/* Advances every instance by max_steps steps (or to its t_end); info (n
 * entries, may be NULL) receives each instance's t, steps, dt, c_h, status. */
int mhd_batch_run(mhd_batch* b, int max_steps, mhd_run_info* info);
int mhd_batch_get_tuning(const mhd_batch* b, mhd_batch_tuning* t);
int mhd_batch_set_tuning(mhd_batch* b, const mhd_batch_tuning* t);
/* Autotuner: times each sweep phase for every candidate launch shape (x work
 * per warp xrpw 2/4/8/16 x 2-4 CTAs per SM; y segment 16/24/32/48/64/128 x 2-4
 * CTAs per SM) on the batch's current states, `reps` launches each, and keeps
 * the fastest.  Leaves the instances one step ahead. */
int mhd_batch_tune(mhd_batch* b, int reps, mhd_batch_tuning* best);
/* The autotuner's candidate values: which = 0 x work per warp (xrpw), 1 y
 * segment lengths, 2 CTAs per SM (both phases).  Copies up to cap of them into
 * out (may be NULL) and returns how many there are (MHD_ERR_ARG for another
 * `which`). */
int mhd_batch_tune_candidates(int which, int* out, int cap);

/* ---- discrete adjoint (no reference counterpart) ----
 * Gradient of J(a) = 1/2 sum_interior (rho(t_N; a) - rho_target)^2 with respect
 * to the 16 perturbation amplitudes a of mhd_initialise_orszag_tang
 * (b0 = 1/sqrt(4 pi)), after nsteps steps of the split step with HLL (or HLLD,
 * mhd_adjoint_set_solver) and the given limiter on periodic [0,1]^2 (nx x ny,
 * ng = 2).  The reverse pass
 * differentiates the time step and c_h through the CFL argmax cell, the psi
 * damping and every branch the forward took, recomputing the trajectory from
 * checkpoints kept every `checkpoint_every` steps (0: about sqrt(nsteps)).
 * dtype MHD_F64 or MHD_F32 selects the precision of forward and adjoint. */
typedef struct mhd_adjoint mhd_adjoint;
int mhd_adjoint_create(int nx, int ny, int dtype, int limiter, double gamma, double cfl, double cr, int nsteps,
                       int checkpoint_every, mhd_adjoint** out);
int mhd_adjoint_destroy(mhd_adjoint* a);
/* Riemann solver of forward and adjoint: MHD_HLL (default) or MHD_HLLD (its
 * star and double-star regions, its fallbacks to HLL and the GLM psi / Bn
 * overwrite are differentiated). */
int mhd_adjoint_set_solver(mhd_adjoint* a, int solver);
/* rho_target: ny x nx interior densities, row-major (j * nx + i). */
int mhd_adjoint_set_target(mhd_adjoint* a, const double* rho_target);
/* Forward solve only: J (needs a target; else 0) and optionally the final
 * interior density (ny x nx). */
int mhd_adjoint_forward(mhd_adjoint* a, const double* amp16, double* J, double* rho_final);
/* Forward solve and reverse pass: J and dJ/da (16 values). */
int mhd_adjoint_gradient(mhd_adjoint* a, const double* amp16, double* J, double* grad16);

/* ---- misc ---- */
const char* mhd_last_error(void);
/* Library version string. */
const char* mhd_version(void);
/* Number of device kernel launches issued by this library in this process. */
unsigned long long mhd_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* MHD_B200_H */
