/*
 * mhd_b200 — C ABI of the B200 (sm_100a) GLM-MHD backend.
 *
 * This is the drop-in boundary for the reference's accelerator plug-in seam
 * (include/mhd/gpu/device_solver.hpp in the reference project). Each entry point names the
 * reference interface it replaces. Plain C types only: no C++ or torch types cross it, and no
 * exception leaves it. Every call returns an mhdb_status; the message of the last failure on a
 * handle is available from mhdb_last_error().
 *
 * State exchanged with the host uses the reference's StateField layout
 * (include/state/state_field.hpp:9-73): nine planes (rho, mx, my, mz, E, bx, by, bz, psi), each
 * (ny + 2 ng) x (nx + 2 ng) doubles, row-major, including ghost cells. On the device the state
 * lives without ghosts in padded SoA planes; boundary conditions are applied as index maps when
 * tiles are loaded.
 *
 * Threading: one handle per host thread at a time. All work of a handle runs on its own CUDA
 * stream on the device that was current when the handle was created.
 */
#ifndef MHD_B200_H
#define MHD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MHDB_OK = 0,
    MHDB_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference */
    MHDB_MAX_STEPS = 2,        /* "solve: reached max_steps before t_end" */
    MHDB_CUDA_ERROR = 3,       /* std::runtime_error("CUDA: ...") */
    MHDB_NO_DEVICE = 4,        /* factory: no CUDA device */
    MHDB_BAD_TIMESTEP = 5      /* dt not positive (ssp_rk2_step's invalid_argument) */
} mhdb_status;

/* Precision (reference: enum class Precision, device_solver.hpp:28). FP32 selects the
   FP32-mixed form: FP32 arithmetic with the state carried as a compensated hi/lo pair. */
enum { MHDB_FP64 = 0, MHDB_FP32 = 1 };

/* Boundary types, same numbering as the reference's BoundaryConditionType
   (include/boundary_conditions/boundary_conditions.hpp:8). Reflective is rejected, as in the
   reference. */
enum { MHDB_BC_PERIODIC = 0, MHDB_BC_REFLECTIVE = 1, MHDB_BC_OUTFLOW = 2 };

/* Slope limiters: SlopeLimiter::Minmod / MC (include/mhd/mhd_types.hpp:44) plus van Leer. */
enum { MHDB_MINMOD = 0, MHDB_MC = 1, MHDB_VANLEER = 2 };

/* Grid2D (include/grid/grid.hpp:5-26). */
typedef struct {
    int nx, ny, ng;
    double x_min, x_max, y_min, y_max;
} mhdb_grid;

/* SolveParams with its NonIdealConfig flattened (include/mhd/solve_types.hpp:8-16,
   include/physics_config/mhd_config.hpp:13-20). */
typedef struct {
    double t_end, cfl, gamma, glm_alpha;
    int limiter;
    int ohmic, hall, ambipolar;
    double eta_ohm, eta_hall, eta_ambipolar;
    int max_steps;
} mhdb_params;

/* SolveResult (include/mhd/solve_types.hpp:18-22). */
typedef struct {
    double t;
    int steps;
    double c_h;
} mhdb_result;

/* FP64 interior diagnostics: sums of rho*dx*dy and E*dx*dy, central-difference div B
   (max and root-mean-square), minimum rho and p, and whether every value is finite. */
typedef struct {
    double mass, energy, div_b_max, div_b_l2, rho_min, p_min;
    int finite;
} mhdb_diag;

typedef struct mhdb_solver mhdb_solver;

/* Seeded synthetic initial state generated on the device (additive): a smooth periodic field of
   Fourier modes, or four piecewise-constant quadrants split at x = y = 0.5. For the Fourier kind,
   coef holds 5 spectra (vx, vy, A_z, f1, f2), each (2 kmax + 1) rows (ky = -kmax..kmax) by
   (kmax + 1) columns (kx = 0..kmax) of complex values as (re, im) pairs; the device evaluates them
   at cell centres, sets B = curl(A_z), scales v and B to rms 1, and sets rho = 1 + clip(0.2 f1),
   p = 1 + clip(0.1 f2) with f1, f2 scaled to rms 1 and the perturbations clipped to +-0.2. For
   the quadrant kind, quad[q] = (rho, p, vx, vy, By) of quadrant q in the order (x<.5, y<.5),
   (x>=.5, y<.5), (x<.5, y>=.5), (x>=.5, y>=.5), with Bx = 0.75. */
enum { MHDB_INIT_FOURIER = 0, MHDB_INIT_QUADRANTS = 1 };
typedef struct {
    int kind;
    int kmax;
    const double* coef;
    double quad[4][5];
} mhdb_init;

/* mhd::cuda_available() (device_solver.hpp:78): 1 when a CUDA device is usable. */
int mhdb_cuda_available(void);

/* mhd::make_cuda_solver(grid, precision) (device_solver.hpp:82). Fails with
   MHDB_INVALID_ARGUMENT when ng < 2 or the sizes are not positive, MHDB_NO_DEVICE without a
   device. On failure *out is NULL and mhdb_last_error(NULL) holds the message. */
int mhdb_create(const mhdb_grid* grid, int precision, mhdb_solver** out);

/* ~DeviceSolver(). NULL is accepted. */
void mhdb_destroy(mhdb_solver* h);

/* Message of the last failure on h (h == NULL: of the last failed mhdb_create on this thread). */
const char* mhdb_last_error(const mhdb_solver* h);

/* DeviceSolver::device_name() (device_solver.hpp:62), e.g. "CUDA: NVIDIA B200". */
int mhdb_device_name(const mhdb_solver* h, char* buf, size_t len);

/* DeviceSolver::precision() (device_solver.hpp:63). */
int mhdb_precision(const mhdb_solver* h);

/* DeviceSolver::configure(bc, mask, reflective_walls) (device_solver.hpp:66-67). mask is the
   interior fluid mask, row-major ny * nx bytes (1 = fluid), or NULL for all fluid; mask_len must
   then be 0 or nx * ny. */
int mhdb_configure(mhdb_solver* h, int bc_x, int bc_y, const uint8_t* mask, size_t mask_len,
                   int reflective_walls);

/* Additive: configure with a mask rasterised on the device from circles and rectangles instead of
   a host array (no host mask, no upload). The rule of the reference's geometry helpers
   (gui/geometry.py:22-38, :130-156): every interior cell starts fluid; the shapes are applied in
   order, each painting the cells whose centre x_min + (i + 1/2) dx, y_min + (j + 1/2) dy it
   contains solid (solid = 1) or fluid (solid = 0), later shapes overwriting earlier ones; a circle
   contains (x - a)^2 + (y - b)^2 <= c^2, a rectangle min(a, c) <= x <= max(a, c) and
   min(b, d) <= y <= max(b, d), both inclusive. The mask equals the host rasterisation of the same
   shapes bit for bit. count may be 0 (all fluid). */
enum { MHDB_SHAPE_CIRCLE = 0, MHDB_SHAPE_RECTANGLE = 1 };
typedef struct mhdb_shape {
    int kind;          /* MHDB_SHAPE_CIRCLE or MHDB_SHAPE_RECTANGLE */
    int solid;         /* 1: contained cells become solid; 0: fluid */
    double a, b, c, d; /* circle: centre (a, b), radius c; rectangle: corners (a, b), (c, d) */
} mhdb_shape;
int mhdb_configure_shapes(mhdb_solver* h, int bc_x, int bc_y, const mhdb_shape* shapes, int count,
                          int reflective_walls);

/* Additive: the interior fluid mask the handle uses (MHDSolver::mask(), the reference module's
   get_mask), row-major ny * nx bytes, 1 = fluid; len must be nx * ny. */
int mhdb_get_mask(mhdb_solver* h, uint8_t* out, size_t len);

/* DeviceSolver::upload / download (device_solver.hpp:70-71): nine host planes of n_tot =
   (nx + 2 ng)(ny + 2 ng) doubles each. download returns the state with ghosts filled by the
   boundary rule and solid cells wall-filled, as the reference's solve() leaves it. */
int mhdb_upload(mhdb_solver* h, const double* const comps[9], size_t n_tot);
int mhdb_download(mhdb_solver* h, double* const comps[9], size_t n_tot);

/* DeviceSolver::solve(params) (device_solver.hpp:73-74): advances the device state by
   params->t_end (relative), same contract as the reference solve(). */
int mhdb_solve(mhdb_solver* h, const mhdb_params* params, mhdb_result* result);

/* Additive: advance exactly nsteps SSP-RK2 steps (no t_end limit; params->t_end is ignored). */
int mhdb_solve_steps(mhdb_solver* h, const mhdb_params* params, int nsteps, mhdb_result* result);

/* Additive: replace the device state by a generated initial state (gamma from params). The
   state then behaves like the result of a solve: download fills the ghosts, and with a mask the
   next solve wall-fills the solid cells first. */
int mhdb_generate(mhdb_solver* h, const mhdb_init* init, const mhdb_params* params);

/* Additive: FP64 diagnostics of the device state (gamma from params). */
int mhdb_diagnostics(mhdb_solver* h, const mhdb_params* params, mhdb_diag* out);

/* Additive: the handle's CUDA stream (a cudaStream_t) for event timing by the caller. */
void* mhdb_stream(mhdb_solver* h);

/* Additive: per-kernel event timing. While enabled, every stage kernel launch is bracketed by
   events (no CUDA graphs); mhdb_profile_read returns the summed milliseconds and launch counts
   of the two stage kernels since the last reset. */
int mhdb_set_profiling(mhdb_solver* h, int enabled);
int mhdb_profile_read(mhdb_solver* h, double* ms_stage1, int* n_stage1, double* ms_stage2,
                      int* n_stage2, int reset);

/* Additive: number of kernel launches this handle has issued (graph nodes included). */
long long mhdb_launch_count(const mhdb_solver* h);

/* Additive: tile configurations of the stage kernels. Configuration 0 (the shared-memory tile
   kernel) serves every solve; the others serve solves without a mask (the strip-march ones ideal
   and non-ideal solves, the other tile ones ideal solves only; FP32-mixed configurations 11,
   13 and 17 and FP64 configuration 7 also masked solves; a solve they do not serve runs the default of its size, see below) and are
   picked per grid size class by the autotuner
   (mhd_gpu_solver_b200.autotune). mhdb_tile_config_info writes the interior cells one CTA covers
   (tile width and height), threads per CTA and the minimum CTAs per SM of one configuration;
   mhdb_tile_config_kind returns its kernel: MHDB_KERNEL_TILE (shared-memory tile, separate x and
   y sweeps), MHDB_KERNEL_TILE_MERGED (merged sweeps), MHDB_KERNEL_MARCH (warp strip march, 28
   columns per warp), MHDB_KERNEL_MARCH_TMA (the strip march fed by TMA bulk copies into shared
   memory), MHDB_KERNEL_MARCH_TMA_DELTA (the same for the FP32-mixed increment form: stage 1
   stores the FP32 increment dt L instead of U*, stage 2 reads U^n + increment; configuration 17
   takes stage 2's own-cell increment from its halo copies) or
   MHDB_KERNEL_MARCH_TMA_PAIR (the increment form with two columns per lane, 60 columns per warp),
   or -1 for an unknown configuration. */
enum { MHDB_KERNEL_TILE = 0, MHDB_KERNEL_TILE_MERGED = 1, MHDB_KERNEL_MARCH = 2,
       MHDB_KERNEL_MARCH_TMA = 3, MHDB_KERNEL_MARCH_TMA_DELTA = 4, MHDB_KERNEL_MARCH_TMA_PAIR = 5 };
int mhdb_tile_config_count(int precision);
int mhdb_tile_config_info(int precision, int config, int* tile_x, int* tile_y, int* threads,
                          int* min_blocks);
int mhdb_tile_config_kind(int precision, int config);
/* mhdb_set_tile_config(h, -1) restores the default: FP32-mixed solves of at least 1024 x 1024
   cells run the TMA strip march (one warp per block; unmasked solves in the increment form,
   configuration 13; masked ones configuration 11, the TMA strip march that also serves masks),
   smaller FP32-mixed ones configuration 0; FP64 solves of
   at least 2048 x 2048 cells run the FP64 TMA strip march (configuration 7, which also serves
   masks), smaller ones the 320-thread tile kernel (configuration 2, non-ideal ones configuration
   0), smaller masked FP64 solves configuration 0. */
int mhdb_set_tile_config(mhdb_solver* h, int config);

/* Additive, for tests of the error path: every bulk-copy wait of the TMA strip marches is bounded
   (0.5 s); when one runs out the kernel records it in the Ctrl block, lets its copies in flight
   land and stops, and the solve returns MHDB_CUDA_ERROR ("a bulk-copy wait exceeded its limit")
   with the device context intact. With extra_bytes > 0 (at most 4096) the strip marches of this
   handle arm the first row copy of the strip at the grid's origin for extra_bytes transaction
   bytes more than its boxes deliver, so that wait runs out; the copies themselves are unchanged.
   0 (the default) turns it off. Solves on other kernels are unaffected. No reference
   counterpart (the reference has no bulk copies). */
int mhdb_debug_stall_copies(mhdb_solver* h, int extra_bytes);

/* ---------------------------------------------------------------- strips of one grid (additive)

   One grid split into y strips, one solver per strip (on one GPU or on several): each strip's
   solver holds its owned rows plus overlap rows copied from its neighbours (outflow y rule at the
   strip's ends, which only corrupts overlap rows), so every step runs the same kernels as a whole
   grid. The reference has no multi-GPU form; the step rule stays that of
   include/mhd/time_integrator.hpp:62-106 with one global dt:

     mhdb_set_cell_size(h, dx, dy)    the whole grid's cell size (a strip's extent / rows may
                                      round differently; default: the grid's extent / cells)
     mhdb_set_reduce_rows(h, y0, y1)  rows [y0, y1) of this solver's interior are its owned rows:
                                      only they enter the CFL reduction and the diagnostics
     mhdb_strip_begin(h, p, n)        start a deferred solve (n >= 0: n steps; n < 0: to p->t_end)
                                      and reduce the owned rows' signal speed into ch_bits
     (host: ch_bits = max over all strips, written back to each strip)
     mhdb_strip_finish(h)             dt, c_h and the clock from the combined maximum
     mhdb_strip_step(h)               one RK2 step (both stages), its reduction left in ch_bits
     (host: combine, then mhdb_strip_finish, then copy overlap rows between neighbours)
     mhdb_strip_poll / mhdb_strip_end the clock, finished flag and result, as mhdb_solve

   All strips take the same dt, so they finish at the same step. Calls out of this order return
   MHDB_INVALID_ARGUMENT; mhdb_solve / mhdb_solve_steps end a deferred solve. */
typedef struct mhdb_strip_state {
    void* state;      /* device: U^n, planes of `plane` elements, rows of `pitch` elements; the
                         FP32-mixed increment form alternates between two buffers, so query it
                         again after mhdb_strip_step */
    void* ch_bits;    /* device: 8-byte running signal-speed max (IEEE bits of a double >= 0) */
    long long pitch;  /* elements per row (>= nx) */
    long long plane;  /* elements per plane (pitch * ny) */
    int planes;       /* 9 (FP64) or 18 (FP32-mixed: 9 hi planes, then 9 lo planes) */
    int elem_bytes;   /* 8 (FP64) or 4 (FP32-mixed) */
} mhdb_strip_state;

int mhdb_set_cell_size(mhdb_solver* h, double dx, double dy);
int mhdb_set_reduce_rows(mhdb_solver* h, int y0, int y1);
int mhdb_strip_view(mhdb_solver* h, mhdb_strip_state* out);
int mhdb_strip_begin(mhdb_solver* h, const mhdb_params* params, int nsteps);
int mhdb_strip_step(mhdb_solver* h);
int mhdb_strip_finish(mhdb_solver* h);
int mhdb_strip_poll(mhdb_solver* h, int* finished, int* steps, double* t);
int mhdb_strip_end(mhdb_solver* h, mhdb_result* result);

/* ---------------------------------------------------------------- batched form (additive)

   A batch advances many independent solves of uneven sizes together: every RK2 step is one
   persistent launch per stage (per limiter and non-ideal combination present) over a tile
   work-list of all unfinished solves, and chunks of steps are replayed as CUDA graphs. Each solve
   has its own grid, physics parameters, boundary rule, time target and HBM-resident state, and
   its own FP64 clock; results do not depend on what else is in the batch. No fluid masks. */
typedef struct mhdb_batch mhdb_batch;

int mhdb_batch_create(int precision, mhdb_batch** out);
void mhdb_batch_destroy(mhdb_batch* b);
const char* mhdb_batch_last_error(const mhdb_batch* b);

/* Add a solve from a host state in the StateField layout (uploaded during the call). With
   fixed_steps != 0 the solve runs exactly params->max_steps steps (t_end ignored); otherwise it
   runs to params->t_end like mhdb_solve. *id identifies the solve until mhdb_batch_remove. */
int mhdb_batch_add(mhdb_batch* b, const mhdb_grid* grid, const mhdb_params* params, int bc_x,
                   int bc_y, const double* const comps[9], size_t n_tot, int fixed_steps,
                   int* id);
int mhdb_batch_remove(mhdb_batch* b, int id);

/* Add a solve whose initial state is generated on the device (no host state, no upload). */
int mhdb_batch_add_generated(mhdb_batch* b, const mhdb_grid* grid, const mhdb_params* params,
                             int bc_x, int bc_y, const mhdb_init* init, int fixed_steps, int* id);

/* Advance every unfinished solve by up to nsteps steps; *active (optional) = unfinished count. */
int mhdb_batch_step(mhdb_batch* b, int nsteps, int* active);

/* mhdb_batch_step in two halves: mhdb_batch_launch issues the steps and returns without waiting;
   mhdb_batch_poll waits for them and refreshes every solve's status (as mhdb_batch_step does at
   its end). Between the two, solves that the previous poll reported finished can be downloaded
   (mhdb_batch_download copies them beside the running steps) and removed. */
int mhdb_batch_launch(mhdb_batch* b, int nsteps);
int mhdb_batch_poll(mhdb_batch* b, int* active);

/* Batch configurations: the kernel a solve runs with in a batch (tile shape, halo staging and
   threads per work item). mhdb_batch_config_info writes the interior cells of one work item
   (tile width and height), its threads and its kernel kind (MHDB_KERNEL_*). FP32-mixed: 0 = TMA
   strip march, one warp by 32 rows; 1 = register strip march, 4 warps by 32 rows; 2 = TMA strip
   march, one warp by 64 rows; 3 = TMA strip march of the increment form, one warp by 32 rows
   (the default for solves of at least 128 x 128 cells; smaller ones take 1).
   mhdb_batch_set_config picks one for a solve (-1: by the solve's size, the default); once a
   solve has been stepped it cannot change between configuration 3 and the others
   (MHDB_INVALID_ARGUMENT). The batch autotuner (mhd_gpu_solver_b200.autotune.tune_batch) chooses
   per size class. The configurations agree to the FP32 rounding of the form. */
int mhdb_batch_config_count(int precision);
int mhdb_batch_config_info(int precision, int config, int* tile_x, int* tile_y, int* threads,
                           int* kind);
int mhdb_batch_set_config(mhdb_batch* b, int id, int config);

/* t, steps, c_h and whether the solve has finished; MHDB_MAX_STEPS / MHDB_BAD_TIMESTEP as
   mhdb_solve would report them, and MHDB_CUDA_ERROR when one of the solve's bulk-copy waits ran
   out (the solve stopped; the other solves of the batch are unaffected). */
int mhdb_batch_status(mhdb_batch* b, int id, mhdb_result* result, int* finished);

/* Test hook of the bounded bulk-copy waits for one solve of a batch, as mhdb_debug_stall_copies
   (TMA strip-march batch configurations only). */
int mhdb_batch_debug_stall_copies(mhdb_batch* b, int id, int extra_bytes);
int mhdb_batch_download(mhdb_batch* b, int id, double* const comps[9], size_t n_tot);
int mhdb_batch_info(const mhdb_batch* b, size_t* bytes_in_use, int* live, long long* launches);
void* mhdb_batch_stream(mhdb_batch* b);

/* Allocation-free fixed-step solve. No counterpart in the reference.
   For callers that cannot call cudaMalloc: code inside another framework's device memory pool or
   under a fixed memory budget, and code that must not let an allocation synchronise the device.
   Advances an FP64 state that the caller owns in device memory by exactly nsteps SSP-RK2 steps
   (no t_end limit, like mhdb_solve_steps), without a handle and without allocating anything:
   the stage state U* and the step control live in one file-scope device array of 16 MiB + 256 B
   that every GPU loading this library holds until the process exits.
   - u_in, u_out: device pointers to 9 dense planes of nx * ny doubles (rho, mx, my, mz, E, bx,
     by, bz, psi; interior cells only, row-major, no ghosts); u_out must equal u_in or not
     overlap it at all (a partial overlap is rejected with MHDB_INVALID_ARGUMENT). The caller
     passes both; the state is read from u_in and the result written to u_out.
   - Limit: nx * ny <= 233016 interior cells (16 MiB / 72 B); larger grids are rejected with
     MHDB_INVALID_ARGUMENT and a message from mhdb_last_error(NULL). No mask; boundaries
     periodic or outflow; ideal or non-ideal terms, any limiter.
   - Work runs on `stream` (a cudaStream_t, NULL for the legacy default stream). Each call copies
     the step control between host and device through pageable host memory and synchronises
     `stream` before it returns; result then holds t, steps and c_h.
   - The first call on each device looks up the device address of the scratch array
     (cudaGetSymbolAddress) with that device current and keeps it for the life of the process
     (a cudaDeviceReset of that device would leave it stale); make that first call before any
     stream capture.
   - Every call shares the one scratch array, which keeps the last call's contents: the step
     control is reset at the start of each call and U* is fully rewritten before it is read.
     Calls in one process whose work overlaps on the GPU (several streams or threads on the same
     device) race on that array; each process has its own copy. */
int mhdb_solve_steps_noalloc_f64(const mhdb_grid* grid, int bc_x, int bc_y,
                                 const mhdb_params* params, int nsteps, const double* u_in,
                                 double* u_out, mhdb_result* result, void* stream);

#ifdef __cplusplus
}
#endif

#endif
