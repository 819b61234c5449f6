// Allocation-free variant of the fixed-step FP64 solve (mhdb_solve_steps_noalloc_f64).
//
// Some callers cannot allocate device memory: code running inside another framework's memory
// pool or under a strict memory budget, code that must not synchronise the device the way
// cudaMalloc/cudaFree can, and callers that fix their whole device footprint up front. This entry
// point lets them advance an FP64 state that they own, in device memory they already hold,
// without the library allocating anything. The scratch the stage kernels need (the intermediate
// RK2 stage state U* and the Ctrl block of the FP64 clock and CFL reduction) lives in one
// file-scope __device__ array of fixed size, which every GPU that loads this library holds
// until the process exits.

#include "mhd_b200.h"

#include "stage_select.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

using namespace mhdb;

namespace mhdb {
extern thread_local std::string g_create_error; // solver.cu
}

namespace {

// 16 MiB of stage state plus 256 bytes for the Ctrl block.
constexpr size_t kScratchStateBytes = size_t(16) << 20;
constexpr size_t kCtrlBytes = 256;
constexpr size_t kScratchBytes = kScratchStateBytes + kCtrlBytes;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_scratch_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Most interior cells the scratch holds: 9 FP64 planes of U*.
constexpr size_t kMaxCells = kScratchStateBytes / (9 * sizeof(double));

int fail(int code, const std::string& msg)
{
    mhdb::g_create_error = msg; // reported by mhdb_last_error(NULL)
    return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
    char buf[256];
    std::snprintf(buf, sizeof buf, "CUDA: %s (%s)", cudaGetErrorString(e), what);
    return fail(MHDB_CUDA_ERROR, buf);
}

// Device address of the scratch array on the current device. In host code the array's name is
// only a host-side stand-in, so the address is looked up once per device with that device
// current and cached for the life of the process (a cudaDeviceReset of that device would leave
// the cached address stale).
cudaError_t scratch_address(int device, void** out)
{
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (g_scratch_ptr[device] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            return e;
        }
        g_scratch_ptr[device] = p;
    }
    *out = g_scratch_ptr[device];
    return cudaSuccess;
}

template <int NT>
__global__ void noalloc_cfl_init(const double* __restrict__ u, Geometry g, Consts k, Ctrl* ctrl)
{
    double smax = 0.0;
    const long long ncell = static_cast<long long>(g.nx) * g.ny;
    for (long long c = blockIdx.x * static_cast<long long>(NT) + threadIdx.x; c < ncell;
         c += static_cast<long long>(gridDim.x) * NT) {
        const int x = static_cast<int>(c % g.nx), y = static_cast<int>(c / g.nx);
        double r[9];
        load_cons_f64(u, g, x, y, r);
        smax = vmax(smax, PolicyF64::signal_speed(r, k));
    }
    reduce_signal_speed_and_finish(smax, ctrl, k, gridDim.x, false);
}

} // namespace

extern "C" {

int mhdb_solve_steps_noalloc_f64(const mhdb_grid* grid, int bc_x, int bc_y,
                                 const mhdb_params* params, int nsteps, const double* u_in,
                                 double* u_out, mhdb_result* result, void* stream)
{
    if (grid == nullptr || params == nullptr || result == nullptr || u_in == nullptr ||
        u_out == nullptr) {
        return fail(MHDB_INVALID_ARGUMENT, "grid, params, result and state pointers are required");
    }
    if (grid->nx < 1 || grid->ny < 1 || nsteps < 0) {
        return fail(MHDB_INVALID_ARGUMENT, "grid sizes must be positive and nsteps non-negative");
    }
    const size_t cells = static_cast<size_t>(grid->nx) * static_cast<size_t>(grid->ny);
    if (cells > kMaxCells) {
        char buf[160];
        std::snprintf(buf, sizeof buf,
                      "grid of %zu cells exceeds the %zu-cell limit of the allocation-free solve",
                      cells, kMaxCells);
        return fail(MHDB_INVALID_ARGUMENT, buf);
    }
    if ((bc_x != kPeriodic && bc_x != kOutflow) || (bc_y != kPeriodic && bc_y != kOutflow)) {
        return fail(MHDB_INVALID_ARGUMENT, "boundary types must be periodic or outflow");
    }
    if (params->cfl <= 0.0) {
        return fail(MHDB_INVALID_ARGUMENT, "CFL number must be positive");
    }
    if (params->limiter < kMinmod || params->limiter > kVanLeer) {
        return fail(MHDB_INVALID_ARGUMENT, "unknown slope limiter");
    }
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) {
        return cuda_fail(e, "cudaGetDevice");
    }
    if (device < 0 || device >= kMaxDevices) {
        return fail(MHDB_INVALID_ARGUMENT, "device index out of range");
    }
    void* scratch = nullptr;
    e = scratch_address(device, &scratch);
    if (e != cudaSuccess) {
        return cuda_fail(e, "cudaGetSymbolAddress");
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    Geometry g{};
    g.nx = grid->nx;
    g.ny = grid->ny;
    g.pitch = grid->nx; // dense planes of the caller: nx * ny doubles each
    g.bc_x = bc_x;
    g.bc_y = bc_y;
    g.plane = cells;
    g.ry0 = 0;
    g.ry1 = grid->ny;

    // Per-solve constants, as make_consts in solver.cu.
    Consts k{};
    const double dx = (grid->x_max - grid->x_min) / static_cast<double>(grid->nx);
    const double dy = (grid->y_max - grid->y_min) / static_cast<double>(grid->ny);
    k.gamma = params->gamma;
    k.gm1 = params->gamma - 1.0;
    k.inv_gm1 = 1.0 / (params->gamma - 1.0);
    k.glm_alpha = params->glm_alpha;
    k.inv_dx = 1.0 / dx;
    k.inv_dy = 1.0 / dy;
    k.inv_2dx = 0.5 / dx;
    k.inv_2dy = 0.5 / dy;
    k.h = (dy < dx) ? dy : dx;
    k.cfl = params->cfl;
    double eta = 0.0;
    auto vmx = [](double a, double b) { return (a < b) ? b : a; };
    if (params->ohmic) eta = vmx(eta, std::fabs(params->eta_ohm));
    if (params->hall) eta = vmx(eta, std::fabs(params->eta_hall));
    if (params->ambipolar) eta = vmx(eta, std::fabs(params->eta_ambipolar));
    k.eta_max = eta;
    k.dt_diff = eta > 0.0 ? params->cfl * k.h * k.h / (2.0 * 2.0 * eta) : 0.0;
    k.ni = NonIdealCoef{params->ohmic != 0, params->hall != 0, params->ambipolar != 0,
                        params->eta_ohm, params->eta_hall, params->eta_ambipolar};
    k.ni_any = (params->ohmic && params->eta_ohm != 0.0) ||
               (params->hall && params->eta_hall != 0.0) ||
               (params->ambipolar && params->eta_ambipolar != 0.0);

    const StageKernels sk = select_stage_f64(params->limiter, k.ni_any != 0, false, 0);
    if (sk.threads == 0) {
        return fail(MHDB_INVALID_ARGUMENT, "no stage kernel for this configuration");
    }

    // Scratch layout: [Ctrl | 256-byte pad][U*: 9 dense planes].
    Ctrl* ctrl = static_cast<Ctrl*>(scratch);
    double* ustar = reinterpret_cast<double*>(static_cast<unsigned char*>(scratch) + kCtrlBytes);

    // u_out either is u_in or lies wholly apart from it: a partial overlap would make the copy
    // below overlap itself and the stages read a half-written state.
    const size_t state_bytes = 9 * cells * sizeof(double);
    const uintptr_t in0 = reinterpret_cast<uintptr_t>(u_in);
    const uintptr_t out0 = reinterpret_cast<uintptr_t>(u_out);
    if (u_out != u_in && in0 < out0 + state_bytes && out0 < in0 + state_bytes) {
        return fail(MHDB_INVALID_ARGUMENT, "u_out must equal u_in or not overlap it");
    }
    // The stage-2 kernel updates its state in place, so the caller's output buffer carries the
    // state from the start.
    if (u_out != u_in) {
        e = cudaMemcpyAsync(u_out, u_in, state_bytes, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) {
            return cuda_fail(e, "cudaMemcpyAsync");
        }
    }
    // The scratch keeps the previous call's contents; the Ctrl block must start from zero.
    Ctrl c0{};
    c0.t_end = static_cast<double>(INFINITY);
    c0.max_steps = nsteps;
    e = cudaMemcpyAsync(ctrl, &c0, sizeof(Ctrl), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        return cuda_fail(e, "cudaMemcpyAsync");
    }
    if ((e = cudaFuncSetAttribute(sk.f64_stage1, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(sk.smem))) != cudaSuccess ||
        (e = cudaFuncSetAttribute(sk.f64_stage2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(sk.smem))) != cudaSuccess) {
        return cuda_fail(e, "cudaFuncSetAttribute");
    }
    const long long ncell = static_cast<long long>(cells);
    const int init_blocks =
        static_cast<int>(std::min<long long>((ncell + 255) / 256, 148LL * 8));
    noalloc_cfl_init<256><<<init_blocks, 256, 0, s>>>(u_out, g, k, ctrl);
    const StageArgsF64 a1{u_out, ustar, nullptr, ctrl, g, k, 1};
    const StageArgsF64 a2{ustar, u_out, nullptr, ctrl, g, k, 1};
    const dim3 grid2((grid->nx + sk.tile_x - 1) / sk.tile_x, (grid->ny + sk.tile_y - 1) / sk.tile_y);
    for (int i = 0; i < nsteps; ++i) {
        sk.f64_stage1<<<grid2, sk.threads, sk.smem, s>>>(a1);
        sk.f64_stage2<<<grid2, sk.threads, sk.smem, s>>>(a2);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        return cuda_fail(e, "kernel launch");
    }
    Ctrl c1{};
    e = cudaMemcpyAsync(&c1, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) {
        e = cudaStreamSynchronize(s);
    }
    if (e != cudaSuccess) {
        return cuda_fail(e, "reading the step control");
    }
    if ((c1.status & kStatusBadDt) != 0) {
        return fail(MHDB_BAD_TIMESTEP, "ssp_rk2_step requires positive dt");
    }
    result->t = c1.t;
    result->steps = c1.steps;
    result->c_h = c1.c_h;
    return MHDB_OK;
}

} // extern "C"
