// Host runtime of the B200 GLM-MHD backend and its C ABI (include/mhd_b200.h).
//
// One mhdb_solver owns, on the device that was current at creation:
//   * the state U^n and the stage state U* as padded SoA planes without ghosts
//     (FP64: 9 double planes each; FP32-mixed: 9 float hi + 9 float lo planes each),
//   * the padded fluid mask, a device Ctrl block (FP64 clock, dt, c_h, step counter),
//   * a ghosted staging buffer for host <-> device exchange in the reference layout,
//   * one CUDA stream and cached CUDA graphs of batches of RK2 steps.
// The time loop keeps dt and the clock on the device: each step is two launches (stage 1, stage 2
// with the CFL reduction fused in), replayed as captured graphs of kGraphBatch steps, and a
// time-based solve reads the Ctrl block back only after each queue of the steps that its current
// dt says remain (steps_to_queue); the device ends the solve.

#include "mhd_b200.h"

#include "physics.cuh"
#include "runtime_types.cuh"
#include "stage_f64.cuh"
#include "stage_mixed.cuh"
#include "diagnostics.cuh"
#include "generate.cuh"
#include "mask_gen.cuh"
#include "stage_select.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <utility>
#include <vector>

using namespace mhdb;

namespace mhdb {
// Message of the last failure not tied to a handle (mhdb_last_error(NULL)).
thread_local std::string g_create_error;
} // namespace mhdb

namespace {

struct CudaFail {
    cudaError_t err;
    const char* what;
};

#define MHDB_CHECK(expr)                                                                           \
    do {                                                                                           \
        const cudaError_t e_ = (expr);                                                             \
        if (e_ != cudaSuccess) {                                                                   \
            throw CudaFail{e_, #expr};                                                             \
        }                                                                                          \
    } while (0)

struct ApiError {
    int code;
    std::string msg;
};

constexpr int kInitThreads = 256;
constexpr int kGraphBatch = 32;
// An even batch: a captured batch of increment-form steps ends in the buffer it started from.
static_assert(kGraphBatch % 2 == 0, "graph batches must hold an even number of steps");

int round_up(int v, int m) { return (v + m - 1) / m * m; }

// ---------------------------------------------------------------- pack / unpack kernels

// Ghosted host layout (reference StateField) -> padded interior planes.
__global__ void unpack_f64(const double* __restrict__ stg, double* __restrict__ u, Geometry g,
                           int ng, int nxt, size_t ntot)
{
    const long long n = static_cast<long long>(g.nx) * g.ny;
    for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(c % g.nx), y = static_cast<int>(c / g.nx);
        const size_t s = static_cast<size_t>(y + ng) * nxt + (x + ng);
        const size_t d = static_cast<size_t>(y) * g.pitch + x;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            u[k * g.plane + d] = stg[k * ntot + s];
        }
    }
}

__global__ void unpack_mixed(const double* __restrict__ stg, MixedState u, Geometry g, int ng,
                             int nxt, size_t ntot)
{
    const long long n = static_cast<long long>(g.nx) * g.ny;
    for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(c % g.nx), y = static_cast<int>(c / g.nx);
        const size_t s = static_cast<size_t>(y + ng) * nxt + (x + ng);
        const size_t d = static_cast<size_t>(y) * g.pitch + x;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            split_store(u, q * g.plane + d, stg[q * ntot + s]);
        }
    }
}

__global__ void pack_mixed(const MixedState u, const uint8_t* __restrict__ mask,
                           double* __restrict__ stg, Geometry g, int ng, int nxt, int nyt,
                           size_t ntot, int fill, double gm1)
{
    const long long n = static_cast<long long>(nxt) * nyt;
    for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(c % nxt), j = static_cast<int>(c / nxt);
        const int gx = i - ng, gy = j - ng;
        const int sx = map_index(gx, g.nx, g.bc_x), sy = map_index(gy, g.ny, g.bc_y);
        const bool interior = gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny;
        double v[9];
        if (fill && interior && is_solid(mask, g, sx, sy)) {
            wall_fill_mx(u, mask, g, sx, sy, gm1, v);
        } else {
            load_cons_mx(u, g, sx, sy, v);
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            stg[q * ntot + static_cast<size_t>(c)] = v[q];
        }
    }
}

// Padded interior planes -> ghosted layout with the final ghost fill and wall fill of the
// reference solve() (include/mhd/time_integrator.hpp:101-104): ghosts copy the (pre-fill)
// stored value of the interior cell their boundary rule maps to; solid interior cells are
// wall-filled.
__global__ void pack_f64(const double* __restrict__ u, const uint8_t* __restrict__ mask,
                         double* __restrict__ stg, Geometry g, int ng, int nxt, int nyt,
                         size_t ntot, int fill, double gm1)
{
    const long long n = static_cast<long long>(nxt) * nyt;
    for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(c % nxt), j = static_cast<int>(c / nxt);
        const int gx = i - ng, gy = j - ng;
        const int sx = map_index(gx, g.nx, g.bc_x), sy = map_index(gy, g.ny, g.bc_y);
        const bool interior = gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny;
        double v[9];
        if (fill && interior && is_solid(mask, g, sx, sy)) {
            wall_fill_f64(u, mask, g, sx, sy, gm1, v);
        } else {
            load_cons_f64(u, g, sx, sy, v);
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            stg[k * ntot + static_cast<size_t>(c)] = v[k];
        }
    }
}

// Wall fill of every solid interior cell in place. Reads fluid cells only and writes solid cells
// only, so the order of cells does not matter (include/mhd/mask.hpp:85-149).
__global__ void fill_solids_f64(double* __restrict__ u, const uint8_t* __restrict__ mask,
                                Geometry g, double gm1)
{
    const long long n = static_cast<long long>(g.nx) * g.ny;
    for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(c % g.nx), y = static_cast<int>(c / g.nx);
        if (!is_solid(mask, g, x, y)) {
            continue;
        }
        double v[9];
        wall_fill_f64(u, mask, g, x, y, gm1, v);
        const size_t o = static_cast<size_t>(y) * g.pitch + x;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            u[k * g.plane + o] = v[k];
        }
    }
}

__global__ void fill_solids_mixed(MixedState u, const uint8_t* __restrict__ mask, Geometry g,
                                  double gm1)
{
    const long long n = static_cast<long long>(g.nx) * g.ny;
    for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(c % g.nx), y = static_cast<int>(c / g.nx);
        if (!is_solid(mask, g, x, y)) {
            continue;
        }
        double v[9];
        wall_fill_mx(u, mask, g, x, y, gm1, v);
        const size_t o = static_cast<size_t>(y) * g.pitch + x;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            split_store(u, k * g.plane + o, v[k]);
        }
    }
}

struct Prof {
    cudaEvent_t a, b;
    int kind;
};

struct StepPlan;

} // namespace

struct mhdb_solver {
    mhdb_grid grid{};
    int precision = MHDB_FP64;
    int device = 0;
    std::string name;
    std::string last_error;
    cudaStream_t stream = nullptr;

    Geometry geom{};
    double dx = 0.0, dy = 0.0; // cell size: the grid's extent / cells unless set explicitly
    int nxt = 0, nyt = 0;
    size_t ntot = 0;

    void* U = nullptr;  // U^n, the current state
    void* Us = nullptr; // U*; in the increment form the other state buffer (swapped with U
                        // after every step)
    float* delta = nullptr; // increment form: 9 float planes of dt L (allocated on first use)
    // increment form: parity of the host-side buffer swaps since the solve started. Steps
    // launched after the solve finished do nothing on the device, so at the end the state is in
    // the buffer of the parity of the steps actually taken (settle_buffers).
    int swap_parity = 0;
    double* staging = nullptr;
    uint8_t* mask = nullptr;
    Ctrl* ctrl = nullptr;
    Ctrl* ctrl_host = nullptr;
    int* flag = nullptr;         // device int of the mask rasteriser (any solid cell)
    double* diag = nullptr;      // kDiagFields * kDiagBlocks partials + kDiagFields results
    double* diag_host = nullptr; // pinned copy of the results

    bool has_mask = false;
    bool walls = true;
    // gamma - 1 of the last solve (the wall fill of download needs it) and whether the device
    // state has been advanced since the last upload; an upload followed directly by a download
    // returns the uploaded array unchanged, ghosts included.
    double last_gm1 = 2.0 / 3.0;
    bool solved_since_upload = false;

    // graph cache for a batch of kGraphBatch steps: two entries, so that the increment form
    // (whose current state buffer alternates with odd step counts) keeps a graph per buffer
    cudaGraphExec_t graph_exec[2] = {nullptr, nullptr};
    std::vector<double> graph_key[2];
    int graph_next = 0; // entry to replace next

    int tile_config = -1; // index into the compiled tile configurations (-1: by grid size)
    int stall_tx = 0;     // test hook of the bounded copy waits (mhdb_debug_stall_copies)
    bool profiling = false;
    std::vector<Prof> prof_pending;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_pool;
    size_t prof_used = 0;
    double prof_ms[2] = {0.0, 0.0};
    int prof_n[2] = {0, 0};
    long long launches = 0;

    // A deferred solve (mhdb_strip_*): its plan, whether it runs a fixed number of steps, its
    // t_end, and which call comes next (a finish after begin / step, a step after finish).
    std::unique_ptr<StepPlan> strip;
    bool strip_fixed = false;
    double strip_t_end = 0.0;
    bool strip_advance = false;
    bool strip_due = false;
};

namespace {

int cuda_status(mhdb_solver* h, const CudaFail& f)
{
    char buf[512];
    std::snprintf(buf, sizeof buf, "CUDA: %s (%s)", cudaGetErrorString(f.err), f.what);
    if (h != nullptr) {
        h->last_error = buf;
    } else {
        g_create_error = buf;
    }
    return MHDB_CUDA_ERROR;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) {
            prev = -1;
        }
        if (prev != dev) {
            MHDB_CHECK(cudaSetDevice(dev));
        }
    }
    ~DeviceGuard()
    {
        if (prev >= 0) {
            cudaSetDevice(prev);
        }
    }
};

Consts make_consts(const mhdb_solver* h, const mhdb_params* p)
{
    Consts k{};
    const double dx = h->dx;
    const double dy = h->dy;
    k.gamma = p->gamma;
    k.gm1 = p->gamma - 1.0;
    k.inv_gm1 = 1.0 / (p->gamma - 1.0);
    k.glm_alpha = p->glm_alpha;
    k.inv_dx = 1.0 / dx;
    k.inv_dy = 1.0 / dy;
    k.inv_2dx = 0.5 / dx;
    k.inv_2dy = 0.5 / dy;
    k.h = (dy < dx) ? dy : dx;
    k.cfl = p->cfl;
    double eta = 0.0;
    auto vmx = [](double a, double b) { return (a < b) ? b : a; };
    if (p->ohmic) eta = vmx(eta, std::fabs(p->eta_ohm));
    if (p->hall) eta = vmx(eta, std::fabs(p->eta_hall));
    if (p->ambipolar) eta = vmx(eta, std::fabs(p->eta_ambipolar));
    k.eta_max = eta;
    k.dt_diff = eta > 0.0 ? p->cfl * k.h * k.h / (2.0 * 2.0 * eta) : 0.0;
    k.ni.ohmic = p->ohmic != 0;
    k.ni.hall = p->hall != 0;
    k.ni.ambipolar = p->ambipolar != 0;
    k.ni.eta_ohm = p->eta_ohm;
    k.ni.eta_hall = p->eta_hall;
    k.ni.eta_ambipolar = p->eta_ambipolar;
    k.ni_any = (p->ohmic && p->eta_ohm != 0.0) || (p->hall && p->eta_hall != 0.0) ||
               (p->ambipolar && p->eta_ambipolar != 0.0);
    k.stall_tx = h->stall_tx;
    return k;
}

void validate_params(const mhdb_params* p, bool time_based)
{
    if (p == nullptr) {
        throw ApiError{MHDB_INVALID_ARGUMENT, "params must not be NULL"};
    }
    if (time_based && p->t_end < 0.0) {
        throw ApiError{MHDB_INVALID_ARGUMENT, "t_end must be non-negative"};
    }
    if (p->cfl <= 0.0) {
        throw ApiError{MHDB_INVALID_ARGUMENT, "CFL number must be positive"};
    }
    if (p->limiter < kMinmod || p->limiter > kVanLeer) {
        throw ApiError{MHDB_INVALID_ARGUMENT, "unknown slope limiter"};
    }
}

// Launch plan of one RK2 step for the current state and parameters.
struct StepPlan {
    bool mixed = false;
    StageFnF64 s1 = nullptr, s2 = nullptr;
    StageArgsF64 a1{}, a2{};
    StageFnMx m1 = nullptr, m2 = nullptr;
    StageArgsMx b1{}, b2{};
    StageFnMxTma t1 = nullptr, t2 = nullptr; // TMA-fed FP32-mixed kernels (m1/m2 unused then)
    StageFnF64Tma d1 = nullptr, d2 = nullptr; // TMA-fed FP64 kernels (s1/s2 unused then)
    StageFnDeltaTma e1 = nullptr, e2 = nullptr; // FP32-mixed increment form (m1/m2 unused then)
    // increment form, by parity q: U^n in buffer q (0: the handle's U at planning time, 1: its
    // Us), U^{n+1} written to buffer 1 - q
    StageArgsDelta c1[2]{}, c2[2]{};
    MarchTmaMaps dm1[2]{}, dm2[2]{};
    const void* p0 = nullptr;
    MarchTmaMaps tm1{}, tm2{};
    dim3 grid, block;
    size_t smem = 0, smem2 = 0; // dynamic shared memory of stage 1 and stage 2
    Consts k{};
};

StepPlan make_plan(mhdb_solver* h, const mhdb_params* p)
{
    StepPlan s;
    s.k = make_consts(h, p);
    const bool ni = s.k.ni_any != 0;
    StageKernels sk{};
    // Configurations other than 0 serve unmasked solves (the tile ones ideal solves only, the
    // strip-march ones non-ideal solves too; FP32-mixed configurations 11, 13 and 17 and
    // FP64 configuration 7 also masked solves). A
    // solve the chosen configuration does not serve (e.g. a masked solve after an autotuner
    // choice made on unmasked grids) uses the default configuration of its size, else 0.
    const long long cells = static_cast<long long>(h->grid.nx) * h->grid.ny;
    const int dflt = h->precision == MHDB_FP64 ? default_stage_config_f64(cells, h->has_mask)
                                               : default_stage_config_mixed(cells, h->has_mask);
    auto serves = [&](int c) {
        return c == 0 || (h->precision == MHDB_FP64
                              ? select_stage_f64(p->limiter, ni, h->has_mask, c)
                              : select_stage_mixed(p->limiter, ni, h->has_mask, c))
                                 .threads != 0;
    };
    int cfg = h->tile_config >= 0 ? h->tile_config : dflt;
    if (!serves(cfg)) {
        cfg = serves(dflt) ? dflt : 0;
    }
    if (h->precision == MHDB_FP64) {
        sk = select_stage_f64(p->limiter, ni, h->has_mask, cfg);
        s.s1 = sk.f64_stage1;
        s.s2 = sk.f64_stage2;
        const double* u = static_cast<const double*>(h->U);
        const double* us = static_cast<const double*>(h->Us);
        s.a1 = StageArgsF64{u, static_cast<double*>(h->Us), h->has_mask ? h->mask : nullptr,
                            h->ctrl, h->geom, s.k, h->walls ? 1 : 0};
        s.a2 = StageArgsF64{us, static_cast<double*>(h->U), h->has_mask ? h->mask : nullptr,
                            h->ctrl, h->geom, s.k, h->walls ? 1 : 0};
        if (sk.f64_tma1 != nullptr) {
            s.d1 = sk.f64_tma1;
            s.d2 = sk.f64_tma2;
            std::string err;
            if (!encode_march_maps_f64(u, us, h->geom, &s.tm1, &err) ||
                !encode_march_maps_f64(us, u, h->geom, &s.tm2, &err)) {
                throw ApiError{MHDB_CUDA_ERROR, err};
            }
        }
    } else {
        s.mixed = true;
        sk = select_stage_mixed(p->limiter, ni, h->has_mask, cfg);
        s.m1 = sk.mx_stage1;
        s.m2 = sk.mx_stage2;
        const MixedState u = mixed_view(h->U, h->geom);
        const MixedState us = mixed_view(h->Us, h->geom);
        s.b1 = StageArgsMx{u, us, h->has_mask ? h->mask : nullptr, h->ctrl, h->geom, s.k,
                           h->walls ? 1 : 0};
        s.b2 = StageArgsMx{us, u, h->has_mask ? h->mask : nullptr, h->ctrl, h->geom, s.k,
                           h->walls ? 1 : 0};
        if (sk.mx_tma1 != nullptr) {
            s.t1 = sk.mx_tma1;
            s.t2 = sk.mx_tma2;
            std::string err;
            if (!encode_march_maps(u, us, h->geom, &s.tm1, &err) ||
                !encode_march_maps(us, u, h->geom, &s.tm2, &err)) {
                throw ApiError{MHDB_CUDA_ERROR, err};
            }
        } else if (sk.dx_tma1 != nullptr) {
            // increment form: the state alternates between the two buffers step by step
            s.e1 = sk.dx_tma1;
            s.e2 = sk.dx_tma2;
            if (h->delta == nullptr) {
                MHDB_CHECK(cudaMalloc(reinterpret_cast<void**>(&h->delta),
                                      9 * h->geom.plane * sizeof(float)));
            }
            const MixedState bufs[2] = {u, us};
            s.p0 = h->U;
            for (int q = 0; q < 2; ++q) {
                s.c1[q] = StageArgsDelta{bufs[q], bufs[1 - q], h->delta,
                                         h->has_mask ? h->mask : nullptr, h->ctrl, h->geom, s.k,
                                         h->walls ? 1 : 0};
                s.c2[q] = s.c1[q];
                std::string err;
                if (!encode_march_maps_delta(bufs[q], h->delta, h->geom, &s.dm1[q], &s.dm2[q],
                                             &err, sk.halo_w, sk.own_w)) {
                    throw ApiError{MHDB_CUDA_ERROR, err};
                }
            }
        }
    }
    if (sk.threads == 0) {
        throw ApiError{MHDB_INVALID_ARGUMENT, "no stage kernel for this configuration"};
    }
    s.grid = dim3((h->grid.nx + sk.tile_x - 1) / sk.tile_x, (h->grid.ny + sk.tile_y - 1) / sk.tile_y);
    s.block = dim3(sk.threads);
    s.smem = sk.smem;
    s.smem2 = sk.smem2;
    const int b1 = static_cast<int>(s.smem), b2 = static_cast<int>(s.smem2);
    if (s.d1 != nullptr) {
        MHDB_CHECK(cudaFuncSetAttribute(s.d1, cudaFuncAttributeMaxDynamicSharedMemorySize, b1));
        MHDB_CHECK(cudaFuncSetAttribute(s.d2, cudaFuncAttributeMaxDynamicSharedMemorySize, b2));
    } else if (s.e1 != nullptr) {
        MHDB_CHECK(cudaFuncSetAttribute(s.e1, cudaFuncAttributeMaxDynamicSharedMemorySize, b1));
        MHDB_CHECK(cudaFuncSetAttribute(s.e2, cudaFuncAttributeMaxDynamicSharedMemorySize, b2));
    } else if (!s.mixed) {
        MHDB_CHECK(cudaFuncSetAttribute(s.s1, cudaFuncAttributeMaxDynamicSharedMemorySize, b1));
        MHDB_CHECK(cudaFuncSetAttribute(s.s2, cudaFuncAttributeMaxDynamicSharedMemorySize, b2));
    } else if (s.t1 != nullptr) {
        MHDB_CHECK(cudaFuncSetAttribute(s.t1, cudaFuncAttributeMaxDynamicSharedMemorySize, b1));
        MHDB_CHECK(cudaFuncSetAttribute(s.t2, cudaFuncAttributeMaxDynamicSharedMemorySize, b2));
    } else {
        MHDB_CHECK(cudaFuncSetAttribute(s.m1, cudaFuncAttributeMaxDynamicSharedMemorySize, b1));
        MHDB_CHECK(cudaFuncSetAttribute(s.m2, cudaFuncAttributeMaxDynamicSharedMemorySize, b2));
    }
    return s;
}

void launch_stage(mhdb_solver* h, const StepPlan& s, int stage)
{
    if (s.d1 != nullptr) {
        (stage == 1 ? s.d1 : s.d2)<<<s.grid, s.block, stage == 1 ? s.smem : s.smem2, h->stream>>>(
            stage == 1 ? s.a1 : s.a2, stage == 1 ? s.tm1 : s.tm2);
    } else if (s.e1 != nullptr) {
        const int q = h->U == s.p0 ? 0 : 1;
        (stage == 1 ? s.e1 : s.e2)<<<s.grid, s.block, stage == 1 ? s.smem : s.smem2, h->stream>>>(
            stage == 1 ? s.c1[q] : s.c2[q], stage == 1 ? s.dm1[q] : s.dm2[q]);
    } else if (!s.mixed) {
        (stage == 1 ? s.s1 : s.s2)<<<s.grid, s.block, stage == 1 ? s.smem : s.smem2, h->stream>>>(
            stage == 1 ? s.a1 : s.a2);
    } else if (s.t1 != nullptr) {
        (stage == 1 ? s.t1 : s.t2)<<<s.grid, s.block, stage == 1 ? s.smem : s.smem2, h->stream>>>(
            stage == 1 ? s.b1 : s.b2, stage == 1 ? s.tm1 : s.tm2);
    } else {
        (stage == 1 ? s.m1 : s.m2)<<<s.grid, s.block, stage == 1 ? s.smem : s.smem2, h->stream>>>(
            stage == 1 ? s.b1 : s.b2);
    }
    ++h->launches;
}

std::pair<cudaEvent_t, cudaEvent_t> prof_events(mhdb_solver* h)
{
    if (h->prof_used == h->prof_pool.size()) {
        cudaEvent_t a, b;
        MHDB_CHECK(cudaEventCreate(&a));
        MHDB_CHECK(cudaEventCreate(&b));
        h->prof_pool.emplace_back(a, b);
    }
    return h->prof_pool[h->prof_used++];
}

void launch_step_direct(mhdb_solver* h, const StepPlan& s)
{
    for (int stage = 1; stage <= 2; ++stage) {
        if (h->profiling) {
            auto ev = prof_events(h);
            MHDB_CHECK(cudaEventRecord(ev.first, h->stream));
            launch_stage(h, s, stage);
            MHDB_CHECK(cudaEventRecord(ev.second, h->stream));
            h->prof_pending.push_back(Prof{ev.first, ev.second, stage - 1});
        } else {
            launch_stage(h, s, stage);
        }
    }
    if (s.e1 != nullptr) {
        std::swap(h->U, h->Us); // the increment form's stage 2 wrote U^{n+1} to the other buffer
        h->swap_parity ^= 1;
    }
}

// After an increment-form solve: point U at the buffer that holds the state after the steps the
// device actually took (the Ctrl block read back by read_ctrl).
void settle_buffers(mhdb_solver* h, const StepPlan& s)
{
    if (s.e1 != nullptr && h->swap_parity != (h->ctrl_host->steps & 1)) {
        std::swap(h->U, h->Us);
    }
    h->swap_parity = 0;
}

// Identity of a captured batch: everything a stage launch depends on, field by field (no
// struct padding enters the comparison).
std::vector<double> plan_key(const mhdb_solver* h, const mhdb_params* p, const StepPlan& s)
{
    return {static_cast<double>(reinterpret_cast<uintptr_t>(h->U)),
            static_cast<double>(reinterpret_cast<uintptr_t>(h->Us)),
            static_cast<double>(s.mixed), static_cast<double>(p->limiter),
            static_cast<double>(h->has_mask), static_cast<double>(h->walls),
            static_cast<double>(h->geom.bc_x), static_cast<double>(h->geom.bc_y),
            p->gamma, p->glm_alpha, p->cfl,
            static_cast<double>(p->ohmic), static_cast<double>(p->hall),
            static_cast<double>(p->ambipolar), p->eta_ohm, p->eta_hall, p->eta_ambipolar,
            static_cast<double>(h->grid.nx), static_cast<double>(h->grid.ny),
            static_cast<double>(h->tile_config),
            h->grid.x_min, h->grid.x_max, h->grid.y_min, h->grid.y_max, h->dx, h->dy,
            static_cast<double>(h->geom.ry0), static_cast<double>(h->geom.ry1),
            static_cast<double>(h->stall_tx)};
}

void launch_steps(mhdb_solver* h, const mhdb_params* p, const StepPlan& s, int n)
{
    if (h->profiling || n < kGraphBatch) {
        for (int i = 0; i < n; ++i) {
            launch_step_direct(h, s);
        }
        MHDB_CHECK(cudaGetLastError());
        return;
    }
    const std::vector<double> key = plan_key(h, p, s);
    int e = -1;
    for (int j = 0; j < 2; ++j) {
        if (h->graph_exec[j] != nullptr && h->graph_key[j] == key) {
            e = j;
        }
    }
    if (e < 0) {
        e = h->graph_next;
        h->graph_next ^= 1;
        if (h->graph_exec[e] != nullptr) {
            cudaGraphExecDestroy(h->graph_exec[e]);
            h->graph_exec[e] = nullptr;
        }
        cudaGraph_t graph = nullptr;
        MHDB_CHECK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        const long long before = h->launches;
        for (int i = 0; i < kGraphBatch; ++i) {
            launch_step_direct(h, s);
        }
        h->launches = before;
        const cudaError_t cap = cudaStreamEndCapture(h->stream, &graph);
        if (cap != cudaSuccess) {
            throw CudaFail{cap, "cudaStreamEndCapture"};
        }
        const cudaError_t ins = cudaGraphInstantiate(&h->graph_exec[e], graph, 0);
        cudaGraphDestroy(graph);
        if (ins != cudaSuccess) {
            h->graph_exec[e] = nullptr;
            throw CudaFail{ins, "cudaGraphInstantiate"};
        }
        h->graph_key[e] = key;
    }
    const int batches = n / kGraphBatch;
    for (int b = 0; b < batches; ++b) {
        MHDB_CHECK(cudaGraphLaunch(h->graph_exec[e], h->stream));
        h->launches += 2 * kGraphBatch;
    }
    for (int i = 0; i < n - batches * kGraphBatch; ++i) {
        launch_step_direct(h, s);
    }
    MHDB_CHECK(cudaGetLastError());
}

void start_solve(mhdb_solver* h, const StepPlan& s, double t_end, int max_steps, int defer = 0)
{
    Ctrl c{};
    c.t = 0.0;
    c.dt = 0.0;
    c.c_h = 0.0;
    c.t_end = t_end;
    c.ch_bits = 0ull;
    c.arrived = 0u;
    c.steps = 0;
    c.max_steps = max_steps;
    c.finished = 0;
    c.status = 0;
    c.defer = defer;
    *h->ctrl_host = c;
    h->swap_parity = 0;
    MHDB_CHECK(cudaMemcpyAsync(h->ctrl, h->ctrl_host, sizeof(Ctrl), cudaMemcpyHostToDevice,
                               h->stream));
    const long long ncell = static_cast<long long>(h->grid.nx) * h->grid.ny;
    const int blocks = static_cast<int>(std::min<long long>((ncell + kInitThreads - 1) / kInitThreads, 148LL * 8));
    if (!s.mixed) {
        cfl_init_kernel_f64<kInitThreads><<<blocks, kInitThreads, 0, h->stream>>>(
            static_cast<const double*>(h->U), h->mask, h->geom, s.k, h->ctrl, h->has_mask ? 1 : 0);
    } else {
        cfl_init_kernel_mixed<kInitThreads><<<blocks, kInitThreads, 0, h->stream>>>(
            mixed_view(h->U, h->geom), h->mask, h->geom, s.k, h->ctrl, h->has_mask ? 1 : 0);
    }
    ++h->launches;
    MHDB_CHECK(cudaGetLastError());
}

void read_ctrl(mhdb_solver* h)
{
    MHDB_CHECK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost,
                               h->stream));
    MHDB_CHECK(cudaStreamSynchronize(h->stream));
}

// Steps to queue before the next read of the Ctrl block in a time-based solve. The device
// decides where the solve ends (finish_step sets `finished`, and steps queued past that point
// return at once), so the host only sizes the queue: the steps that the dt of the step about to
// run says remain, ceil((t_end - t) / dt), capped by the steps max_steps leaves, and rounded up
// to whole captured graph batches once a batch fits (at most kGraphBatch - 1 queued steps then
// do nothing). A dt that shrinks as the flow steepens costs one more round.
int steps_to_queue(const Ctrl& c)
{
    const int left = std::max(1, c.max_steps - c.steps);
    const double need = std::ceil((c.t_end - c.t) / c.dt);
    if (!(need > 0.0) || need >= static_cast<double>(left)) {
        return left;
    }
    int n = static_cast<int>(need);
    if (n >= kGraphBatch) {
        n = static_cast<int>(std::min<long long>(
            left, (static_cast<long long>(n) + kGraphBatch - 1) / kGraphBatch * kGraphBatch));
    }
    return n;
}

void ensure_staging(mhdb_solver* h)
{
    if (h->staging == nullptr) {
        MHDB_CHECK(cudaMalloc(reinterpret_cast<void**>(&h->staging), 9 * h->ntot * sizeof(double)));
        MHDB_CHECK(cudaMemsetAsync(h->staging, 0, 9 * h->ntot * sizeof(double), h->stream));
    }
}

int launch_blocks(long long n, int threads)
{
    return static_cast<int>(std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 16)));
}

template <class F>
int guarded(mhdb_solver* h, F&& f)
{
    if (h == nullptr) {
        g_create_error = "solver handle must not be NULL";
        return MHDB_INVALID_ARGUMENT;
    }
    try {
        DeviceGuard dg(h->device);
        f();
        return MHDB_OK;
    } catch (const ApiError& e) {
        h->last_error = e.msg;
        return e.code;
    } catch (const CudaFail& e) {
        return cuda_status(h, e);
    } catch (const std::bad_alloc&) {
        h->last_error = "out of host memory";
        return MHDB_CUDA_ERROR;
    }
}

void release(mhdb_solver* h)
{
    for (auto& g : h->graph_exec) {
        if (g != nullptr) cudaGraphExecDestroy(g);
    }
    for (auto& e : h->prof_pool) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    if (h->U) cudaFree(h->U);
    if (h->Us) cudaFree(h->Us);
    if (h->delta) cudaFree(h->delta);
    if (h->staging) cudaFree(h->staging);
    if (h->mask) cudaFree(h->mask);
    if (h->ctrl) cudaFree(h->ctrl);
    if (h->ctrl_host) cudaFreeHost(h->ctrl_host);
    if (h->diag) cudaFree(h->diag);
    if (h->flag) cudaFree(h->flag);
    if (h->diag_host) cudaFreeHost(h->diag_host);
    if (h->stream) cudaStreamDestroy(h->stream);
}

// Before a solve: the state left by an earlier solve is wall-filled, as the reference leaves it.
void prepare_solve(mhdb_solver* h, const mhdb_params* p)
{
    if (h->solved_since_upload && h->has_mask && h->walls) {
        // The state is the result of an earlier solve, which the reference leaves wall-filled
        // (time_integrator.hpp:101-104); apply that fill now so that ghosts of solid edge
        // cells see the filled values, as after a download/upload round trip.
        const long long n = static_cast<long long>(h->grid.nx) * h->grid.ny;
        if (h->precision == MHDB_FP64) {
            fill_solids_f64<<<launch_blocks(n, 256), 256, 0, h->stream>>>(
                static_cast<double*>(h->U), h->mask, h->geom, h->last_gm1);
        } else {
            fill_solids_mixed<<<launch_blocks(n, 256), 256, 0, h->stream>>>(
                mixed_view(h->U, h->geom), h->mask, h->geom, h->last_gm1);
        }
        ++h->launches;
        MHDB_CHECK(cudaGetLastError());
    }
    h->last_gm1 = p->gamma - 1.0;
    h->solved_since_upload = true;
}

// After a solve: the Ctrl block read back by read_ctrl into the result, or the solve's error.
void collect_result(mhdb_solver* h, bool time_based, double t_end, mhdb_result* r)
{
    const Ctrl& c = *h->ctrl_host;
    if ((c.status & kStatusWaitTimeout) != 0) {
        throw ApiError{MHDB_CUDA_ERROR, "stage kernel: a bulk-copy wait exceeded its limit"};
    }
    if ((c.status & kStatusBadDt) != 0) {
        throw ApiError{MHDB_BAD_TIMESTEP, "ssp_rk2_step requires positive dt"};
    }
    r->t = c.t;
    r->steps = c.steps;
    r->c_h = c.c_h;
    if (time_based && c.t < t_end) {
        throw ApiError{MHDB_MAX_STEPS, "solve: reached max_steps before t_end"};
    }
}

// finish_step of a deferred solve, after the host has combined ch_bits over the strips.
__global__ void finish_step_kernel(Ctrl* ctrl, Consts k, int advance)
{
    if (blockIdx.x == 0 && threadIdx.x == 0 && ctrl->finished == 0) {
        finish_step(ctrl, k, advance != 0);
    }
}

int run_solve(mhdb_solver* h, const mhdb_params* p, int fixed_steps, mhdb_result* r)
{
    return guarded(h, [&] {
        validate_params(p, fixed_steps < 0);
        if (r == nullptr) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "result must not be NULL"};
        }
        const StepPlan s = make_plan(h, p);
        h->strip.reset(); // a solve ends any deferred solve of this handle
        h->strip_due = false;
        prepare_solve(h, p);
        if (fixed_steps >= 0) {
            start_solve(h, s, static_cast<double>(INFINITY), fixed_steps);
            launch_steps(h, p, s, fixed_steps);
            read_ctrl(h);
        } else {
            start_solve(h, s, p->t_end, p->max_steps);
            read_ctrl(h);
            while (h->ctrl_host->finished == 0) {
                launch_steps(h, p, s, steps_to_queue(*h->ctrl_host));
                read_ctrl(h);
            }
        }
        settle_buffers(h, s);
        collect_result(h, fixed_steps < 0, p->t_end, r);
    });
}

} // namespace

extern "C" {

int mhdb_cuda_available(void)
{
    int count = 0;
    return (cudaGetDeviceCount(&count) == cudaSuccess && count > 0) ? 1 : 0;
}

int mhdb_create(const mhdb_grid* grid, int precision, mhdb_solver** out)
{
    if (out == nullptr || grid == nullptr) {
        g_create_error = "grid and out must not be NULL";
        return MHDB_INVALID_ARGUMENT;
    }
    *out = nullptr;
    if (grid->ng < 2) {
        g_create_error = "CUDA solver requires grid.ng >= 2";
        return MHDB_INVALID_ARGUMENT;
    }
    if (grid->nx < 1 || grid->ny < 1) {
        g_create_error = "grid sizes must be positive";
        return MHDB_INVALID_ARGUMENT;
    }
    if (precision != MHDB_FP64 && precision != MHDB_FP32) {
        g_create_error = "unknown precision";
        return MHDB_INVALID_ARGUMENT;
    }
    if (!mhdb_cuda_available()) {
        g_create_error = "CUDA: no device available";
        return MHDB_NO_DEVICE;
    }
    auto* h = new (std::nothrow) mhdb_solver();
    if (h == nullptr) {
        g_create_error = "out of host memory";
        return MHDB_CUDA_ERROR;
    }
    h->grid = *grid;
    h->precision = precision;
    try {
        MHDB_CHECK(cudaGetDevice(&h->device));
        cudaDeviceProp prop{};
        MHDB_CHECK(cudaGetDeviceProperties(&prop, h->device));
        h->name = std::string("CUDA: ") + prop.name;
        MHDB_CHECK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->nxt = grid->nx + 2 * grid->ng;
        h->nyt = grid->ny + 2 * grid->ng;
        h->ntot = static_cast<size_t>(h->nxt) * h->nyt;
        h->geom.nx = grid->nx;
        h->geom.ny = grid->ny;
        h->geom.pitch = round_up(grid->nx, 32);
        h->geom.bc_x = kPeriodic;
        h->geom.bc_y = kPeriodic;
        h->geom.plane = static_cast<size_t>(h->geom.pitch) * grid->ny;
        h->geom.ry0 = 0;
        h->geom.ry1 = grid->ny;
        h->dx = (grid->x_max - grid->x_min) / static_cast<double>(grid->nx);
        h->dy = (grid->y_max - grid->y_min) / static_cast<double>(grid->ny);
        const size_t bytes = 9 * h->geom.plane * 8; // FP64 or two FP32 halves
        MHDB_CHECK(cudaMalloc(&h->U, bytes));
        MHDB_CHECK(cudaMalloc(&h->Us, bytes));
        MHDB_CHECK(cudaMemsetAsync(h->U, 0, bytes, h->stream));
        MHDB_CHECK(cudaMemsetAsync(h->Us, 0, bytes, h->stream));
        MHDB_CHECK(cudaMalloc(reinterpret_cast<void**>(&h->mask), h->geom.plane));
        MHDB_CHECK(cudaMemsetAsync(h->mask, 1, h->geom.plane, h->stream));
        MHDB_CHECK(cudaMalloc(reinterpret_cast<void**>(&h->ctrl), sizeof(Ctrl)));
        MHDB_CHECK(cudaMemsetAsync(h->ctrl, 0, sizeof(Ctrl), h->stream));
        MHDB_CHECK(cudaMallocHost(reinterpret_cast<void**>(&h->ctrl_host), sizeof(Ctrl)));
        MHDB_CHECK(cudaStreamSynchronize(h->stream));
    } catch (const CudaFail& e) {
        cuda_status(nullptr, e);
        release(h);
        delete h;
        return MHDB_CUDA_ERROR;
    }
    *out = h;
    return MHDB_OK;
}

void mhdb_destroy(mhdb_solver* h)
{
    if (h == nullptr) {
        return;
    }
    {
        int prev = -1;
        cudaGetDevice(&prev);
        cudaSetDevice(h->device);
        if (h->stream) cudaStreamSynchronize(h->stream);
        release(h);
        if (prev >= 0) cudaSetDevice(prev);
    }
    delete h;
}

const char* mhdb_last_error(const mhdb_solver* h)
{
    return h == nullptr ? g_create_error.c_str() : h->last_error.c_str();
}

int mhdb_device_name(const mhdb_solver* h, char* buf, size_t len)
{
    if (h == nullptr || buf == nullptr || len == 0) {
        return MHDB_INVALID_ARGUMENT;
    }
    std::snprintf(buf, len, "%s", h->name.c_str());
    return MHDB_OK;
}

int mhdb_precision(const mhdb_solver* h)
{
    return h == nullptr ? -1 : h->precision;
}

int mhdb_configure(mhdb_solver* h, int bc_x, int bc_y, const uint8_t* mask, size_t mask_len,
                   int reflective_walls)
{
    return guarded(h, [&] {
        if (bc_x == kReflective || bc_y == kReflective) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "Reflective boundary conditions are not implemented yet"};
        }
        if ((bc_x != kPeriodic && bc_x != kOutflow) || (bc_y != kPeriodic && bc_y != kOutflow)) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "unknown boundary condition type"};
        }
        const size_t n = static_cast<size_t>(h->grid.nx) * h->grid.ny;
        bool active = false;
        if (mask != nullptr) {
            if (mask_len != n) {
                throw ApiError{MHDB_INVALID_ARGUMENT, "FluidMask size does not match Grid2D interior"};
            }
            for (size_t i = 0; i < n && !active; ++i) {
                active = mask[i] == 0;
            }
        }
        h->geom.bc_x = bc_x;
        h->geom.bc_y = bc_y;
        h->walls = reflective_walls != 0;
        h->has_mask = active;
        if (active) {
            MHDB_CHECK(cudaMemcpy2DAsync(h->mask, h->geom.pitch, mask, h->grid.nx, h->grid.nx,
                                         h->grid.ny, cudaMemcpyHostToDevice, h->stream));
            MHDB_CHECK(cudaStreamSynchronize(h->stream));
        }
    });
}

int mhdb_configure_shapes(mhdb_solver* h, int bc_x, int bc_y, const mhdb_shape* shapes, int count,
                          int reflective_walls)
{
    return guarded(h, [&] {
        if (bc_x == kReflective || bc_y == kReflective) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "Reflective boundary conditions are not implemented yet"};
        }
        if ((bc_x != kPeriodic && bc_x != kOutflow) || (bc_y != kPeriodic && bc_y != kOutflow)) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "unknown boundary condition type"};
        }
        if (count < 0 || (count > 0 && shapes == nullptr)) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "shapes must not be NULL when count > 0"};
        }
        for (int k = 0; k < count; ++k) {
            if (shapes[k].kind != MHDB_SHAPE_CIRCLE && shapes[k].kind != MHDB_SHAPE_RECTANGLE) {
                throw ApiError{MHDB_INVALID_ARGUMENT, "unknown shape kind"};
            }
        }
        if (h->flag == nullptr) {
            MHDB_CHECK(cudaMalloc(reinterpret_cast<void**>(&h->flag), sizeof(int)));
        }
        ShapeList L{};
        L.x_min = h->grid.x_min;
        L.dx = (h->grid.x_max - h->grid.x_min) / static_cast<double>(h->grid.nx);
        L.y_min = h->grid.y_min;
        L.dy = (h->grid.y_max - h->grid.y_min) / static_cast<double>(h->grid.ny);
        const long long n = static_cast<long long>(h->grid.nx) * h->grid.ny;
        int k0 = 0;
        do { // at least one launch: count == 0 leaves an all-fluid mask
            L.count = std::min(count - k0, kShapesPerLaunch);
            L.first = k0 == 0 ? 1 : 0;
            for (int k = 0; k < L.count; ++k) {
                L.s[k] = shapes[k0 + k];
            }
            // every launch rewrites and checks every cell, so the last one's flag holds
            MHDB_CHECK(cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream));
            rasterize_shapes<<<launch_blocks(n, 256), 256, 0, h->stream>>>(h->mask, h->geom, L,
                                                                           h->flag);
            ++h->launches;
            MHDB_CHECK(cudaGetLastError());
            k0 += L.count;
        } while (k0 < count);
        int any = 0;
        MHDB_CHECK(cudaMemcpyAsync(&any, h->flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        MHDB_CHECK(cudaStreamSynchronize(h->stream));
        h->geom.bc_x = bc_x;
        h->geom.bc_y = bc_y;
        h->walls = reflective_walls != 0;
        h->has_mask = any != 0;
    });
}

int mhdb_get_mask(mhdb_solver* h, uint8_t* out, size_t len)
{
    return guarded(h, [&] {
        if (out == nullptr || len != static_cast<size_t>(h->grid.nx) * h->grid.ny) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "FluidMask size does not match Grid2D interior"};
        }
        if (!h->has_mask) {
            std::memset(out, 1, len);
            return;
        }
        MHDB_CHECK(cudaMemcpy2DAsync(out, h->grid.nx, h->mask, h->geom.pitch, h->grid.nx,
                                     h->grid.ny, cudaMemcpyDeviceToHost, h->stream));
        MHDB_CHECK(cudaStreamSynchronize(h->stream));
    });
}

int mhdb_upload(mhdb_solver* h, const double* const comps[9], size_t n_tot)
{
    return guarded(h, [&] {
        if (comps == nullptr || n_tot != h->ntot) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "StateField size does not match Grid2D"};
        }
        ensure_staging(h);
        for (int c = 0; c < 9; ++c) {
            if (comps[c] == nullptr) {
                throw ApiError{MHDB_INVALID_ARGUMENT, "state component must not be NULL"};
            }
            MHDB_CHECK(cudaMemcpyAsync(h->staging + c * h->ntot, comps[c], h->ntot * sizeof(double),
                                       cudaMemcpyHostToDevice, h->stream));
        }
        const long long n = static_cast<long long>(h->grid.nx) * h->grid.ny;
        if (h->precision == MHDB_FP64) {
            unpack_f64<<<launch_blocks(n, 256), 256, 0, h->stream>>>(
                h->staging, static_cast<double*>(h->U), h->geom, h->grid.ng, h->nxt, h->ntot);
        } else {
            unpack_mixed<<<launch_blocks(n, 256), 256, 0, h->stream>>>(
                h->staging, mixed_view(h->U, h->geom), h->geom, h->grid.ng, h->nxt, h->ntot);
        }
        ++h->launches;
        MHDB_CHECK(cudaGetLastError());
        MHDB_CHECK(cudaStreamSynchronize(h->stream));
        h->solved_since_upload = false;
    });
}

int mhdb_download(mhdb_solver* h, double* const comps[9], size_t n_tot)
{
    return guarded(h, [&] {
        if (comps == nullptr || n_tot != h->ntot) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "StateField size does not match Grid2D"};
        }
        ensure_staging(h);
        // gamma only matters for the wall fill; it is the one of the last solve.
        const double gm1 = h->last_gm1;
        const long long n = static_cast<long long>(h->ntot);
        const int fill = (h->has_mask && h->walls) ? 1 : 0;
        if (!h->solved_since_upload) {
            // staging still holds the uploaded array
        } else if (h->precision == MHDB_FP64) {
            pack_f64<<<launch_blocks(n, 256), 256, 0, h->stream>>>(
                static_cast<const double*>(h->U), h->mask, h->staging, h->geom, h->grid.ng, h->nxt,
                h->nyt, h->ntot, fill, gm1);
        } else {
            pack_mixed<<<launch_blocks(n, 256), 256, 0, h->stream>>>(
                mixed_view(h->U, h->geom), h->mask, h->staging, h->geom, h->grid.ng, h->nxt,
                h->nyt, h->ntot, fill, gm1);
        }
        if (h->solved_since_upload) {
            ++h->launches;
        }
        MHDB_CHECK(cudaGetLastError());
        for (int c = 0; c < 9; ++c) {
            if (comps[c] == nullptr) {
                throw ApiError{MHDB_INVALID_ARGUMENT, "state component must not be NULL"};
            }
            MHDB_CHECK(cudaMemcpyAsync(comps[c], h->staging + c * h->ntot, h->ntot * sizeof(double),
                                       cudaMemcpyDeviceToHost, h->stream));
        }
        MHDB_CHECK(cudaStreamSynchronize(h->stream));
    });
}

int mhdb_solve(mhdb_solver* h, const mhdb_params* params, mhdb_result* result)
{
    return run_solve(h, params, -1, result);
}

int mhdb_solve_steps(mhdb_solver* h, const mhdb_params* params, int nsteps, mhdb_result* result)
{
    if (nsteps < 0) {
        if (h != nullptr) h->last_error = "nsteps must be non-negative";
        return MHDB_INVALID_ARGUMENT;
    }
    return run_solve(h, params, nsteps, result);
}

int mhdb_generate(mhdb_solver* h, const mhdb_init* init, const mhdb_params* params)
{
    return guarded(h, [&] {
        if (init == nullptr || params == nullptr) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "init and params must not be NULL"};
        }
        if (init->kind != MHDB_INIT_FOURIER && init->kind != MHDB_INIT_QUADRANTS) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "unknown initial-state kind"};
        }
        if (init->kind == MHDB_INIT_FOURIER && (init->coef == nullptr || init->kmax < 1)) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "Fourier initial state needs kmax >= 1 and coef"};
        }
        GenSpec spec{};
        spec.kind = init->kind;
        spec.kmax = init->kmax;
        spec.gamma = params->gamma;
        std::memcpy(spec.quad, init->quad, sizeof spec.quad);
        spec.x_min = h->grid.x_min;
        spec.x_max = h->grid.x_max;
        spec.y_min = h->grid.y_min;
        spec.y_max = h->grid.y_max;
        cudaError_t e;
        if (h->precision == MHDB_FP64) {
            e = launch_generate(h->stream, spec, init->coef, h->geom, static_cast<double*>(h->Us),
                                StoreF64{static_cast<double*>(h->U), h->geom.plane});
        } else {
            e = launch_generate(h->stream, spec, init->coef, h->geom, static_cast<double*>(h->Us),
                                StoreMx{mixed_view(h->U, h->geom), h->geom.plane});
        }
        h->launches += init->kind == MHDB_INIT_FOURIER ? 2 : 1;
        MHDB_CHECK(e);
        MHDB_CHECK(cudaStreamSynchronize(h->stream));
        h->last_gm1 = params->gamma - 1.0;
        h->solved_since_upload = true;
    });
}

int mhdb_diagnostics(mhdb_solver* h, const mhdb_params* params, mhdb_diag* out)
{
    return guarded(h, [&] {
        if (params == nullptr || out == nullptr) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "params and out must not be NULL"};
        }
        if (h->diag == nullptr) {
            MHDB_CHECK(cudaMalloc(reinterpret_cast<void**>(&h->diag),
                                  sizeof(double) * kDiagFields * (kDiagBlocks + 1)));
            MHDB_CHECK(cudaMallocHost(reinterpret_cast<void**>(&h->diag_host),
                                      sizeof(double) * kDiagFields));
        }
        const Consts k = make_consts(h, params);
        const double dx = h->dx;
        const double dy = h->dy;
        const long long n = static_cast<long long>(h->grid.nx) * (h->geom.ry1 - h->geom.ry0);
        const int blocks = static_cast<int>(std::min<long long>(kDiagBlocks, (n + kDiagThreads - 1) / kDiagThreads));
        const int fill = (h->has_mask && h->walls) ? 1 : 0;
        if (h->precision == MHDB_FP64) {
            diag_partial<<<blocks, kDiagThreads, 0, h->stream>>>(
                DiagLoaderF64{static_cast<const double*>(h->U)}, h->mask, fill, h->geom, k.gm1,
                k.inv_2dx, k.inv_2dy, h->diag);
        } else {
            diag_partial<<<blocks, kDiagThreads, 0, h->stream>>>(
                DiagLoaderMx{mixed_view(h->U, h->geom)}, h->mask, fill, h->geom, k.gm1, k.inv_2dx,
                k.inv_2dy, h->diag);
        }
        double* res = h->diag + kDiagFields * kDiagBlocks;
        diag_final<<<1, 32, 0, h->stream>>>(h->diag, blocks, dx * dy, n, res);
        h->launches += 2;
        MHDB_CHECK(cudaGetLastError());
        MHDB_CHECK(cudaMemcpyAsync(h->diag_host, res, sizeof(double) * kDiagFields,
                                   cudaMemcpyDeviceToHost, h->stream));
        MHDB_CHECK(cudaStreamSynchronize(h->stream));
        out->mass = h->diag_host[0];
        out->energy = h->diag_host[1];
        out->div_b_max = h->diag_host[2];
        out->div_b_l2 = h->diag_host[3];
        out->rho_min = h->diag_host[4];
        out->p_min = h->diag_host[5];
        out->finite = h->diag_host[6] == 0.0 ? 1 : 0;
    });
}

void* mhdb_stream(mhdb_solver* h)
{
    return h == nullptr ? nullptr : static_cast<void*>(h->stream);
}

int mhdb_set_profiling(mhdb_solver* h, int enabled)
{
    if (h == nullptr) return MHDB_INVALID_ARGUMENT;
    h->profiling = enabled != 0;
    return MHDB_OK;
}

int mhdb_profile_read(mhdb_solver* h, double* ms1, int* n1, double* ms2, int* n2, int reset)
{
    return guarded(h, [&] {
        MHDB_CHECK(cudaStreamSynchronize(h->stream));
        for (const Prof& p : h->prof_pending) {
            float ms = 0.f;
            MHDB_CHECK(cudaEventElapsedTime(&ms, p.a, p.b));
            h->prof_ms[p.kind] += ms;
            h->prof_n[p.kind] += 1;
        }
        h->prof_pending.clear();
        h->prof_used = 0;
        if (ms1) *ms1 = h->prof_ms[0];
        if (n1) *n1 = h->prof_n[0];
        if (ms2) *ms2 = h->prof_ms[1];
        if (n2) *n2 = h->prof_n[1];
        if (reset) {
            h->prof_ms[0] = h->prof_ms[1] = 0.0;
            h->prof_n[0] = h->prof_n[1] = 0;
        }
    });
}

long long mhdb_launch_count(const mhdb_solver* h)
{
    return h == nullptr ? 0 : h->launches;
}

int mhdb_tile_config_count(int precision)
{
    return precision == MHDB_FP32 ? stage_config_count_mixed() : stage_config_count_f64();
}

int mhdb_tile_config_info(int precision, int config, int* tile_x, int* tile_y, int* threads,
                          int* min_blocks)
{
    if (config < 0 || config >= mhdb_tile_config_count(precision)) {
        return MHDB_INVALID_ARGUMENT;
    }
    const TileConfigInfo t = precision == MHDB_FP32 ? stage_config_info_mixed(config)
                                                    : stage_config_info_f64(config);
    if (tile_x) *tile_x = t.tile_x;
    if (tile_y) *tile_y = t.tile_y;
    if (threads) *threads = t.threads;
    if (min_blocks) *min_blocks = t.min_blocks;
    return MHDB_OK;
}

int mhdb_tile_config_kind(int precision, int config)
{
    if (config < 0 || config >= mhdb_tile_config_count(precision)) {
        return -1;
    }
    return (precision == MHDB_FP32 ? stage_config_info_mixed(config)
                                   : stage_config_info_f64(config)).kind;
}

int mhdb_set_tile_config(mhdb_solver* h, int config)
{
    if (h == nullptr) {
        return MHDB_INVALID_ARGUMENT;
    }
    if (config < -1 || config >= mhdb_tile_config_count(h->precision)) {
        h->last_error = "unknown tile configuration";
        return MHDB_INVALID_ARGUMENT;
    }
    h->tile_config = config;
    return MHDB_OK;
}

int mhdb_debug_stall_copies(mhdb_solver* h, int extra_bytes)
{
    if (h == nullptr) {
        return MHDB_INVALID_ARGUMENT;
    }
    if (extra_bytes < 0 || extra_bytes > 4096) {
        h->last_error = "stall bytes must lie in [0, 4096]";
        return MHDB_INVALID_ARGUMENT;
    }
    h->stall_tx = extra_bytes;
    return MHDB_OK;
}

int mhdb_set_reduce_rows(mhdb_solver* h, int y0, int y1)
{
    return guarded(h, [&] {
        if (y0 < 0 || y1 > h->grid.ny || y0 >= y1) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "reduce rows must satisfy 0 <= y0 < y1 <= ny"};
        }
        if (h->strip) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "a deferred solve is running"};
        }
        h->geom.ry0 = y0;
        h->geom.ry1 = y1;
    });
}

int mhdb_set_cell_size(mhdb_solver* h, double dx, double dy)
{
    return guarded(h, [&] {
        if (!(dx > 0.0) || !(dy > 0.0) || !std::isfinite(dx) || !std::isfinite(dy)) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "cell size must be positive and finite"};
        }
        if (h->strip) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "a deferred solve is running"};
        }
        h->dx = dx;
        h->dy = dy;
    });
}

int mhdb_strip_view(mhdb_solver* h, mhdb_strip_state* out)
{
    return guarded(h, [&] {
        if (out == nullptr) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "out must not be NULL"};
        }
        out->state = h->U;
        out->ch_bits = &h->ctrl->ch_bits;
        out->pitch = h->geom.pitch;
        out->plane = static_cast<long long>(h->geom.plane);
        out->planes = h->precision == MHDB_FP64 ? 9 : 18;
        out->elem_bytes = h->precision == MHDB_FP64 ? 8 : 4;
    });
}

int mhdb_strip_begin(mhdb_solver* h, const mhdb_params* params, int nsteps)
{
    return guarded(h, [&] {
        validate_params(params, nsteps < 0);
        h->strip.reset();
        auto plan = std::make_unique<StepPlan>(make_plan(h, params));
        prepare_solve(h, params);
        h->strip_fixed = nsteps >= 0;
        h->strip_t_end = params->t_end;
        start_solve(h, *plan, nsteps >= 0 ? static_cast<double>(INFINITY) : params->t_end,
                    nsteps >= 0 ? nsteps : params->max_steps, 1);
        h->strip = std::move(plan);
        h->strip_advance = false;
        h->strip_due = true;
    });
}

int mhdb_strip_step(mhdb_solver* h)
{
    return guarded(h, [&] {
        if (!h->strip || h->strip_due) {
            throw ApiError{MHDB_INVALID_ARGUMENT,
                           "strip step: no deferred solve, or its reduction awaits mhdb_strip_finish"};
        }
        launch_step_direct(h, *h->strip);
        MHDB_CHECK(cudaGetLastError());
        h->strip_advance = true;
        h->strip_due = true;
    });
}

int mhdb_strip_finish(mhdb_solver* h)
{
    return guarded(h, [&] {
        if (!h->strip || !h->strip_due) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "strip finish: no reduction awaits it"};
        }
        finish_step_kernel<<<1, 1, 0, h->stream>>>(h->ctrl, h->strip->k, h->strip_advance ? 1 : 0);
        ++h->launches;
        MHDB_CHECK(cudaGetLastError());
        h->strip_due = false;
    });
}

int mhdb_strip_poll(mhdb_solver* h, int* finished, int* steps, double* t)
{
    return guarded(h, [&] {
        if (!h->strip) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "strip poll: no deferred solve"};
        }
        read_ctrl(h);
        if (finished != nullptr) *finished = h->ctrl_host->finished;
        if (steps != nullptr) *steps = h->ctrl_host->steps;
        if (t != nullptr) *t = h->ctrl_host->t;
    });
}

int mhdb_strip_end(mhdb_solver* h, mhdb_result* result)
{
    return guarded(h, [&] {
        if (!h->strip || h->strip_due) {
            throw ApiError{MHDB_INVALID_ARGUMENT,
                           "strip end: no deferred solve, or its reduction awaits mhdb_strip_finish"};
        }
        if (result == nullptr) {
            throw ApiError{MHDB_INVALID_ARGUMENT, "result must not be NULL"};
        }
        read_ctrl(h);
        settle_buffers(h, *h->strip);
        h->strip.reset();
        collect_result(h, !h->strip_fixed, h->strip_t_end, result);
    });
}

} // extern "C"
