// Batched form: many independent solves of uneven sizes advanced together.
//
// A batch holds solves, each with its own grid, gamma, CFL, limiter, non-ideal coefficients,
// boundary rule, time target and HBM-resident state (U^n and the stage state, stream-ordered
// allocations). Every RK2 step is one persistent launch per stage and per (limiter, non-ideal)
// combination present: each launch walks a block work-list covering all unfinished solves of that
// combination (FP64: the shared-memory tile kernel, batch_stage_kernel in stage_kernel.cuh;
// FP32-mixed: the TMA strip march, batch_march_tma_kernel in march_tma.cuh, with each solve's
// tensor maps in its descriptor). Each solve
// keeps its own Ctrl block (FP64
// clock, dt, c_h, step count) in one slot array, so one device-to-host copy reports every solve.
// Chunks of steps are captured as CUDA graphs and replayed while the set of solves is unchanged.

#include "mhd_b200.h"

#include "kernel_table.cuh"
#include "stage_f64.cuh"
#include "stage_mixed.cuh"
#include "generate.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <tuple>
#include <memory>
#include <string>
#include <utility>
#include <vector>

using namespace mhdb;

namespace mhdb {
extern thread_local std::string g_create_error; // solver.cu
}

namespace {

struct BatchFail {
    int code;
    std::string msg;
};

void check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) {
        char buf[256];
        std::snprintf(buf, sizeof buf, "CUDA: %s (%s)", cudaGetErrorString(e), what);
        throw BatchFail{MHDB_CUDA_ERROR, buf};
    }
}

constexpr int kInitThreads = 256;

__global__ void batch_unpack_f64(const double* __restrict__ stg, double* __restrict__ u, Geometry g,
                                 int ng, int nxt, size_t ntot)
{
    const long long n = static_cast<long long>(g.nx) * g.ny;
    for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(c % g.nx), y = static_cast<int>(c / g.nx);
        const size_t s = static_cast<size_t>(y + ng) * nxt + (x + ng);
        const size_t d = static_cast<size_t>(y) * g.pitch + x;
        for (int k = 0; k < 9; ++k) {
            u[k * g.plane + d] = stg[k * ntot + s];
        }
    }
}

__global__ void batch_unpack_mx(const double* __restrict__ stg, MixedState u, Geometry g, int ng,
                                int nxt, size_t ntot)
{
    const long long n = static_cast<long long>(g.nx) * g.ny;
    for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(c % g.nx), y = static_cast<int>(c / g.nx);
        const size_t s = static_cast<size_t>(y + ng) * nxt + (x + ng);
        const size_t d = static_cast<size_t>(y) * g.pitch + x;
        for (int q = 0; q < 9; ++q) {
            split_store(u, q * g.plane + d, stg[q * ntot + s]);
        }
    }
}

// Ghost fill by the boundary index map on download (no mask in batches).
template <class Load>
__global__ void batch_pack(Load load, double* __restrict__ stg, Geometry g, int ng, int nxt,
                           int nyt, size_t ntot)
{
    const long long n = static_cast<long long>(nxt) * nyt;
    for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(c % nxt), j = static_cast<int>(c / nxt);
        const int sx = map_index(i - ng, g.nx, g.bc_x), sy = map_index(j - ng, g.ny, g.bc_y);
        double v[9];
        load(sx, sy, v);
        for (int q = 0; q < 9; ++q) {
            stg[q * ntot + static_cast<size_t>(c)] = v[q];
        }
    }
}

struct LoadF64 {
    const double* u;
    Geometry g;
    __device__ void operator()(int x, int y, double* v) const { load_cons_f64(u, g, x, y, v); }
};
struct LoadMx {
    MixedState u;
    Geometry g;
    __device__ void operator()(int x, int y, double* v) const { load_cons_mx(u, g, x, y, v); }
};
// State of an increment-form solve: buffer (steps & 1) of its step counter, read on the device
// when the copy runs.
struct LoadMxParity {
    MixedState u0, u1;
    Geometry g;
    const Ctrl* ctrl;
    __device__ void operator()(int x, int y, double* v) const
    {
        load_cons_mx((ctrl->steps & 1) != 0 ? u1 : u0, g, x, y, v);
    }
};

template <int NT, class Load, class Speed>
__global__ void batch_cfl_init(Load load, Speed speed, Geometry g, Consts k, Ctrl* ctrl)
{
    double smax = 0.0;
    const long long ncell = static_cast<long long>(g.nx) * g.ny;
    for (long long c = blockIdx.x * static_cast<long long>(NT) + threadIdx.x; c < ncell;
         c += static_cast<long long>(gridDim.x) * NT) {
        const int x = static_cast<int>(c % g.nx), y = static_cast<int>(c / g.nx);
        double r[9];
        load(x, y, r);
        smax = vmax(smax, speed(r, k));
    }
    reduce_signal_speed_and_finish(smax, ctrl, k, gridDim.x, false);
}

struct SpeedF64 {
    __device__ double operator()(const double* r, const Consts& k) const
    {
        return PolicyF64::signal_speed(r, k);
    }
};
struct SpeedMx {
    __device__ double operator()(const double* r, const Consts& k) const
    {
        return PolicyMixed::signal_speed(r, k);
    }
};

Consts consts_of(const mhdb_grid& grid, const mhdb_params& p)
{
    Consts k{};
    const double dx = (grid.x_max - grid.x_min) / static_cast<double>(grid.nx);
    const double dy = (grid.y_max - grid.y_min) / static_cast<double>(grid.ny);
    k.gamma = p.gamma;
    k.gm1 = p.gamma - 1.0;
    k.inv_gm1 = 1.0 / (p.gamma - 1.0);
    k.glm_alpha = p.glm_alpha;
    k.inv_dx = 1.0 / dx;
    k.inv_dy = 1.0 / dy;
    k.inv_2dx = 0.5 / dx;
    k.inv_2dy = 0.5 / dy;
    k.h = (dy < dx) ? dy : dx;
    k.cfl = p.cfl;
    double eta = 0.0;
    auto vmx = [](double a, double b) { return (a < b) ? b : a; };
    if (p.ohmic) eta = vmx(eta, std::fabs(p.eta_ohm));
    if (p.hall) eta = vmx(eta, std::fabs(p.eta_hall));
    if (p.ambipolar) eta = vmx(eta, std::fabs(p.eta_ambipolar));
    k.eta_max = eta;
    k.dt_diff = eta > 0.0 ? p.cfl * k.h * k.h / (2.0 * 2.0 * eta) : 0.0;
    k.ni = NonIdealCoef{p.ohmic != 0, p.hall != 0, p.ambipolar != 0, p.eta_ohm, p.eta_hall,
                        p.eta_ambipolar};
    k.ni_any = (p.ohmic && p.eta_ohm != 0.0) || (p.hall && p.eta_hall != 0.0) ||
               (p.ambipolar && p.eta_ambipolar != 0.0);
    return k;
}

int blocks_for(long long n, int threads)
{
    return static_cast<int>(std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 16)));
}

// Batch configurations: the kernel variants a solve of a batch can run with (the tile shape, the
// halo staging and the threads per work item), picked per solve (mhdb_batch_set_config; by
// default from the solve's size) and so per size class by the batch autotuner.
struct BatchVariant {
    int tile_x, tile_y, threads, kind; // kind: MHDB_KERNEL_*
};

template <class Policy>
struct BatchKernels;

template <>
struct BatchKernels<PolicyF64> {
    using Cfg = TileCfg<32, 8, 320, 2>;
    using Desc = BatchSolve<PolicyF64>;
    using Fn = void (*)(const Desc*, const int2*, int);
    static constexpr int kVariants = 1;
    static BatchVariant variant(int) { return {Cfg::TX, Cfg::TY, Cfg::NT, MHDB_KERNEL_TILE}; }
    static int default_variant(long long) { return 0; }
    template <int L, bool NI, int STAGE>
    static Fn fn(int)
    {
        return batch_stage_kernel<PolicyF64, L, NI, STAGE, Cfg::TX, Cfg::TY, Cfg::NT, Cfg::MINB>;
    }
    static size_t smem(int, bool ni, int)
    {
        return ni ? stage_smem_bytes<double, Cfg::TX, Cfg::TY, true>()
                  : stage_smem_bytes<double, Cfg::TX, Cfg::TY, false>();
    }
};

// FP32-mixed variants:
//   0: TMA strip march, one warp (28 columns x 32 rows) per item, 16 blocks per SM, stage 1
//      through TMA row stores, stage 2 through plain stores;
//   1: register strip march (rows loaded by the lanes, no shared-memory staging), 4 warps
//      (112 columns x 32 rows) per item, 4 blocks per SM;
//   2: as 0 with 64 rows per item;
//   3: as 0 in the increment form (stage_delta.cuh): stage 1 stores the FP32 increment, stage 2
//      writes U^{n+1} to the other state buffer (per-solve buffer parity from its step counter).
template <>
struct BatchKernels<PolicyMixed> {
    using Desc = BatchSolveTma;
    using Fn = void (*)(const Desc*, const int2*, int);
    static constexpr int kVariants = 4;
    static constexpr int kDeltaVariant = 3;
    static BatchVariant variant(int v)
    {
        if (v == 1) return {4 * kMarchOwned, 32, 128, MHDB_KERNEL_MARCH};
        if (v == 2) return {kMarchOwned, 64, 32, MHDB_KERNEL_MARCH_TMA};
        if (v == 3) return {kMarchOwned, 32, 32, MHDB_KERNEL_MARCH_TMA_DELTA};
        return {kMarchOwned, 32, 32, MHDB_KERNEL_MARCH_TMA};
    }
    // Small solves have too few strips to fill the GPU on their own; their per-item set-up is
    // cheaper in the register march. Larger ones run the increment form.
    static int default_variant(long long cells) { return cells >= 128LL * 128 ? 3 : 1; }
    template <int L, bool NI, int STAGE>
    static Fn fn(int v)
    {
        if (v == 1) return batch_march_kernel<PolicyMixed, L, NI, STAGE, 32, 4, 4, BatchSolveTma>;
        if (v == 2) return batch_march_tma_kernel<L, NI, STAGE, 64, 1, 16, true, (STAGE == 1 ? 1 : 0)>;
        if (v == 3) return batch_march_delta_kernel<L, NI, STAGE, 32, 1, 16, true>;
        return batch_march_tma_kernel<L, NI, STAGE, 32, 1, 16, true, (STAGE == 1 ? 1 : 0)>;
    }
    static size_t smem(int v, bool, int stage)
    {
        if (v == 1) return 0;
        if (v == 3) {
            return stage == 1 ? march_tma_smem_bytes<1, 0, 4, 1>(1)
                              : march_tma_smem_bytes<2, 0, 4, 2>(1);
        }
        return stage == 1 ? march_tma_smem_bytes<1, 1>(1) : march_tma_smem_bytes<2, 0>(1);
    }
};

template <class Policy>
typename BatchKernels<Policy>::Fn batch_fn(int variant, int lim, bool ni, int stage)
{
    using K = BatchKernels<Policy>;
#define MHDB_BF(LL)                                                                                \
    if (ni) return stage == 1 ? K::template fn<LL, true, 1>(variant) : K::template fn<LL, true, 2>(variant); \
    return stage == 1 ? K::template fn<LL, false, 1>(variant) : K::template fn<LL, false, 2>(variant);
    if (lim == kMinmod) {
        MHDB_BF(kMinmod)
    } else if (lim == kMC) {
        MHDB_BF(kMC)
    } else {
        MHDB_BF(kVanLeer)
    }
#undef MHDB_BF
}

struct SolveRec {
    bool live = false;
    mhdb_grid grid{};
    mhdb_params params{};
    Geometry geom{};
    Consts k{};
    int limiter = 0;
    bool ni = false;
    void* U = nullptr;
    void* Us = nullptr;
    size_t bytes = 0;
    int slot = -1;
    int config = -1;  // batch configuration chosen for this solve (-1: from its size)
    int variant = 0;  // configuration in use (set when the work lists are built)
    int tiles_x = 0, tiles_y = 0;
    bool fixed = false;
    Ctrl last{}; // host copy after the last poll
    MarchTmaMaps maps[2]{}; // FP32-mixed: tensor maps of stage 1 and stage 2
    // increment form (FP32-mixed variant 3): the increment planes, the tensor maps of both
    // buffer parities, whether the solve uses it, and whether it has been stepped (after which
    // it can no longer change between the stored and the increment form)
    float* delta = nullptr;
    MarchTmaMaps dmaps[2][2]{};
    bool alternates = false;
    bool stepped = false;
};

} // namespace

struct mhdb_batch {
    int precision = MHDB_FP32;
    int device = 0;
    cudaStream_t stream = nullptr;
    // Downloads of finished solves run here, beside the steps in flight on `stream`.
    cudaStream_t dl_stream = nullptr;
    cudaEvent_t dl_wait = nullptr;
    // Device memory of the batch's states and staging buffers: a pool of its own that keeps
    // freed memory for the next solves instead of returning it to the driver at each
    // synchronisation, so admitting a solve does not map new memory.
    cudaMemPool_t pool = nullptr;
    std::string last_error;
    std::vector<SolveRec> solves; // index = id
    std::vector<int> free_ids;
    Ctrl* ctrl = nullptr;         // device slot array
    Ctrl* ctrl_host = nullptr;    // pinned mirror
    int ctrl_cap = 0;
    std::vector<int> free_slots;
    int next_slot = 0;
    void* descs = nullptr;        // device descriptors (BatchSolve<PolicyF64> or BatchSolveTma)
    size_t descs_cap = 0;         // bytes
    int2* work = nullptr;
    size_t work_cap = 0;          // items
    struct List {
        int variant;
        int limiter;
        bool ni;
        int offset, count;
    };
    std::vector<List> lists;
    bool dirty = true;
    size_t bytes_in_use = 0;
    long long launches = 0;
    int resident_ctas[4][2][2] = {}; // [variant][ni][stage-1] CTAs per SM
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
};

namespace {

template <class F>
int guarded(mhdb_batch* b, F&& f)
{
    if (b == nullptr) {
        mhdb::g_create_error = "batch handle must not be NULL";
        return MHDB_INVALID_ARGUMENT;
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != b->device) {
        cudaSetDevice(b->device);
    }
    int rc = MHDB_OK;
    try {
        f();
    } catch (const BatchFail& e) {
        b->last_error = e.msg;
        rc = e.code;
    } catch (const std::bad_alloc&) {
        b->last_error = "out of host memory";
        rc = MHDB_CUDA_ERROR;
    }
    if (prev >= 0 && prev != b->device) {
        cudaSetDevice(prev);
    }
    return rc;
}

void grow_ctrl(mhdb_batch* b, int need)
{
    if (need <= b->ctrl_cap) {
        return;
    }
    int cap = std::max(64, b->ctrl_cap * 2);
    while (cap < need) cap *= 2;
    Ctrl* d = nullptr;
    Ctrl* hst = nullptr;
    check(cudaMalloc(reinterpret_cast<void**>(&d), sizeof(Ctrl) * cap), "cudaMalloc(ctrl)");
    check(cudaMallocHost(reinterpret_cast<void**>(&hst), sizeof(Ctrl) * cap), "cudaMallocHost(ctrl)");
    check(cudaMemsetAsync(d, 0, sizeof(Ctrl) * cap, b->stream), "cudaMemsetAsync");
    if (b->ctrl != nullptr) {
        check(cudaMemcpyAsync(d, b->ctrl, sizeof(Ctrl) * b->ctrl_cap, cudaMemcpyDeviceToDevice, b->stream),
              "cudaMemcpyAsync(ctrl)");
        check(cudaStreamSynchronize(b->stream), "cudaStreamSynchronize");
        cudaFree(b->ctrl);
        cudaFreeHost(b->ctrl_host);
    }
    b->ctrl = d;
    b->ctrl_host = hst;
    b->ctrl_cap = cap;
    b->dirty = true; // descriptors hold ctrl pointers
}

template <class Policy>
void rebuild(mhdb_batch* b)
{
    using K = BatchKernels<Policy>;
    using Desc = typename K::Desc;
    std::vector<Desc> descs;
    std::map<std::tuple<int, int, int>, std::vector<int2>> items; // (variant, limiter, ni)
    for (size_t id = 0; id < b->solves.size(); ++id) {
        SolveRec& s = b->solves[id];
        if (!s.live || s.last.finished != 0) {
            continue;
        }
        s.variant = (s.config >= 0 && s.config < K::kVariants)
                        ? s.config
                        : K::default_variant(static_cast<long long>(s.grid.nx) * s.grid.ny);
        const BatchVariant bv = K::variant(s.variant);
        s.tiles_x = (s.grid.nx + bv.tile_x - 1) / bv.tile_x;
        s.tiles_y = (s.grid.ny + bv.tile_y - 1) / bv.tile_y;
        Desc d{};
        Ctrl* ctrl = b->ctrl + s.slot;
        if constexpr (sizeof(typename Policy::T) == 8) {
            d.stage[0] = StageArgsF64{static_cast<const double*>(s.U), static_cast<double*>(s.Us),
                                      nullptr, ctrl, s.geom, s.k, 1};
            d.stage[1] = StageArgsF64{static_cast<const double*>(s.Us), static_cast<double*>(s.U),
                                      nullptr, ctrl, s.geom, s.k, 1};
        } else {
            const MixedState u = mixed_view(s.U, s.geom), us = mixed_view(s.Us, s.geom);
            d.stage[0] = StageArgsMx{u, us, nullptr, ctrl, s.geom, s.k, 1};
            d.stage[1] = StageArgsMx{us, u, nullptr, ctrl, s.geom, s.k, 1};
            d.maps[0] = s.maps[0];
            d.maps[1] = s.maps[1];
            const bool alt = s.variant == BatchKernels<PolicyMixed>::kDeltaVariant;
            if (!s.stepped) {
                s.alternates = alt;
            }
            if (s.alternates) {
                if (s.delta == nullptr) {
                    const size_t db = 9 * s.geom.plane * sizeof(float);
                    check(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&s.delta), db, b->pool,
                                                  b->stream), "cudaMallocFromPoolAsync(delta)");
                    b->bytes_in_use += db;
                    s.bytes += db;
                    const MixedState bufs[2] = {u, us};
                    for (int q = 0; q < 2; ++q) {
                        std::string err;
                        if (!encode_march_maps_delta(bufs[q], s.delta, s.geom, &s.dmaps[q][0],
                                                     &s.dmaps[q][1], &err)) {
                            throw BatchFail{MHDB_CUDA_ERROR, err};
                        }
                    }
                }
                const MixedState bufs[2] = {u, us};
                for (int q = 0; q < 2; ++q) {
                    d.dstage[q] = StageArgsDelta{bufs[q], bufs[1 - q], s.delta, nullptr, ctrl,
                                                 s.geom, s.k, 1};
                    d.dmaps[q][0] = s.dmaps[q][0];
                    d.dmaps[q][1] = s.dmaps[q][1];
                }
            }
        }
        d.tiles_x = s.tiles_x;
        d.ntiles = s.tiles_x * s.tiles_y;
        const int di = static_cast<int>(descs.size());
        descs.push_back(d);
        auto& v = items[{s.variant, s.limiter, s.ni ? 1 : 0}];
        for (int t = 0; t < d.ntiles; ++t) {
            v.push_back(make_int2(di, t));
        }
    }
    std::vector<int2> work;
    b->lists.clear();
    for (auto& kv : items) {
        b->lists.push_back({std::get<0>(kv.first), std::get<1>(kv.first),
                            std::get<2>(kv.first) != 0, static_cast<int>(work.size()),
                            static_cast<int>(kv.second.size())});
        work.insert(work.end(), kv.second.begin(), kv.second.end());
    }
    const size_t dbytes = std::max<size_t>(1, descs.size()) * sizeof(Desc);
    if (dbytes > b->descs_cap) {
        if (b->descs) cudaFree(b->descs);
        check(cudaMalloc(&b->descs, dbytes * 2), "cudaMalloc(descs)");
        b->descs_cap = dbytes * 2;
    }
    if (work.size() > b->work_cap || b->work == nullptr) {
        if (b->work) cudaFree(b->work);
        const size_t cap = std::max<size_t>(1024, work.size() * 2);
        check(cudaMalloc(reinterpret_cast<void**>(&b->work), cap * sizeof(int2)), "cudaMalloc(work)");
        b->work_cap = cap;
    }
    if (!descs.empty()) {
        check(cudaMemcpyAsync(b->descs, descs.data(), descs.size() * sizeof(Desc),
                              cudaMemcpyHostToDevice, b->stream), "cudaMemcpyAsync(descs)");
        check(cudaMemcpyAsync(b->work, work.data(), work.size() * sizeof(int2),
                              cudaMemcpyHostToDevice, b->stream), "cudaMemcpyAsync(work)");
        check(cudaStreamSynchronize(b->stream), "cudaStreamSynchronize");
    }
    // CTAs per SM of each kernel family in use (occupancy of the persistent grid).
    for (const auto& l : b->lists) {
        const BatchVariant bv = K::variant(l.variant);
        for (int st = 1; st <= 2; ++st) {
            auto fn = batch_fn<Policy>(l.variant, l.limiter, l.ni, st);
            const size_t sm = K::smem(l.variant, l.ni, st);
            check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm)),
                  "cudaFuncSetAttribute");
            int nb = 0;
            check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, bv.threads, sm), "occupancy");
            b->resident_ctas[l.variant][l.ni ? 1 : 0][st - 1] = std::max(1, nb);
        }
    }
    if (b->graph != nullptr) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    b->dirty = false;
}

// One RK2 step of every work list: per stage, one persistent launch per list, each filling the
// GPU with its kernel's resident CTAs.
template <class Policy>
void launch_step(mhdb_batch* b, int sms)
{
    using K = BatchKernels<Policy>;
    const auto* descs = static_cast<const typename K::Desc*>(b->descs);
    for (int stage = 1; stage <= 2; ++stage) {
        for (const auto& l : b->lists) {
            auto fn = batch_fn<Policy>(l.variant, l.limiter, l.ni, stage);
            const size_t sm = K::smem(l.variant, l.ni, stage);
            const int grid =
                std::min(l.count, sms * b->resident_ctas[l.variant][l.ni ? 1 : 0][stage - 1]);
            fn<<<grid, K::variant(l.variant).threads, sm, b->stream>>>(descs, b->work + l.offset,
                                                                      l.count);
            ++b->launches;
        }
    }
}

template <class Policy>
void run_steps(mhdb_batch* b, int nsteps)
{
    if (b->dirty) {
        rebuild<Policy>(b);
    }
    if (b->lists.empty() || nsteps <= 0) {
        return;
    }
    for (auto& s : b->solves) {
        if (s.live && s.last.finished == 0) {
            s.stepped = true;
        }
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    // One captured graph of `chunk` RK2 steps (each step: the persistent stage launches of every
    // list), replayed; the remainder is launched directly.
    const int chunk = std::min(nsteps, 16);
    if (b->graph == nullptr || b->graph_steps != chunk) {
        if (b->graph != nullptr) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
        cudaGraph_t g = nullptr;
        check(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "capture");
        const long long before = b->launches;
        try {
            for (int i = 0; i < chunk; ++i) {
                launch_step<Policy>(b, sms);
            }
        } catch (...) {
            cudaStreamEndCapture(b->stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        b->launches = before;
        check(cudaStreamEndCapture(b->stream, &g), "cudaStreamEndCapture");
        const cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        check(e, "cudaGraphInstantiate");
        b->graph_steps = chunk;
    }
    const long long per_step = 2LL * static_cast<long long>(b->lists.size());
    int done = 0;
    for (; done + chunk <= nsteps; done += chunk) {
        check(cudaGraphLaunch(b->graph, b->stream), "cudaGraphLaunch");
        b->launches += per_step * chunk;
    }
    for (; done < nsteps; ++done) {
        launch_step<Policy>(b, sms);
    }
    check(cudaGetLastError(), "batch step launch");
}

void poll(mhdb_batch* b)
{
    if (b->next_slot == 0) {
        return;
    }
    check(cudaMemcpyAsync(b->ctrl_host, b->ctrl, sizeof(Ctrl) * b->next_slot, cudaMemcpyDeviceToHost,
                          b->stream), "cudaMemcpyAsync(ctrl)");
    check(cudaStreamSynchronize(b->stream), "cudaStreamSynchronize");
    for (auto& s : b->solves) {
        if (!s.live) {
            continue;
        }
        const bool was = s.last.finished != 0;
        s.last = b->ctrl_host[s.slot];
        if (!was && s.last.finished != 0) {
            b->dirty = true; // drop its tiles from the work lists
        }
    }
}

} // namespace

extern "C" {

int mhdb_batch_create(int precision, mhdb_batch** out)
{
    if (out == nullptr || (precision != MHDB_FP64 && precision != MHDB_FP32)) {
        mhdb::g_create_error = "invalid batch arguments";
        return MHDB_INVALID_ARGUMENT;
    }
    *out = nullptr;
    if (!mhdb_cuda_available()) {
        mhdb::g_create_error = "CUDA: no device available";
        return MHDB_NO_DEVICE;
    }
    auto* b = new (std::nothrow) mhdb_batch();
    if (b == nullptr) {
        mhdb::g_create_error = "out of host memory";
        return MHDB_CUDA_ERROR;
    }
    b->precision = precision;
    if (cudaGetDevice(&b->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete b;
        mhdb::g_create_error = "CUDA: cannot create the batch stream";
        return MHDB_CUDA_ERROR;
    }
    if (cudaStreamCreateWithFlags(&b->dl_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->dl_wait, cudaEventDisableTiming) != cudaSuccess) {
        if (b->dl_stream) cudaStreamDestroy(b->dl_stream);
        cudaStreamDestroy(b->stream);
        delete b;
        mhdb::g_create_error = "CUDA: cannot create the batch download stream";
        return MHDB_CUDA_ERROR;
    }
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = b->device;
    unsigned long long keep = ~0ull;
    if (cudaMemPoolCreate(&b->pool, &props) != cudaSuccess ||
        cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
        if (b->pool) cudaMemPoolDestroy(b->pool);
        cudaEventDestroy(b->dl_wait);
        cudaStreamDestroy(b->dl_stream);
        cudaStreamDestroy(b->stream);
        delete b;
        mhdb::g_create_error = "CUDA: cannot create the batch memory pool";
        return MHDB_CUDA_ERROR;
    }
    *out = b;
    return MHDB_OK;
}

void mhdb_batch_destroy(mhdb_batch* b)
{
    if (b == nullptr) {
        return;
    }
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    for (auto& s : b->solves) {
        if (s.live) {
            cudaFreeAsync(s.U, b->stream);
            cudaFreeAsync(s.Us, b->stream);
            if (s.delta) cudaFreeAsync(s.delta, b->stream);
        }
    }
    cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->ctrl) cudaFree(b->ctrl);
    if (b->ctrl_host) cudaFreeHost(b->ctrl_host);
    if (b->descs) cudaFree(b->descs);
    if (b->work) cudaFree(b->work);
    cudaStreamSynchronize(b->dl_stream);
    cudaStreamDestroy(b->dl_stream);
    cudaEventDestroy(b->dl_wait);
    cudaStreamDestroy(b->stream);
    cudaMemPoolDestroy(b->pool);
    if (prev >= 0) cudaSetDevice(prev);
    delete b;
}

const char* mhdb_batch_last_error(const mhdb_batch* b)
{
    return b == nullptr ? mhdb::g_create_error.c_str() : b->last_error.c_str();
}

} // extern "C"

namespace {

// Shared by mhdb_batch_add (host state uploaded through a staging buffer) and
// mhdb_batch_add_generated (state generated on the device).
void add_solve(mhdb_batch* b, const mhdb_grid* grid, const mhdb_params* params, int bc_x, int bc_y,
               const double* const comps[9], size_t n_tot, const mhdb_init* init, int fixed_steps,
               int* id)
{
    if (grid == nullptr || params == nullptr || id == nullptr || (comps == nullptr && init == nullptr)) {
        throw BatchFail{MHDB_INVALID_ARGUMENT, "grid, params, state and id are required"};
    }
    if (grid->ng < 2 || grid->nx < 1 || grid->ny < 1) {
        throw BatchFail{MHDB_INVALID_ARGUMENT, "CUDA solver requires grid.ng >= 2"};
    }
    if ((bc_x != kPeriodic && bc_x != kOutflow) || (bc_y != kPeriodic && bc_y != kOutflow)) {
        throw BatchFail{MHDB_INVALID_ARGUMENT, "Reflective boundary conditions are not implemented yet"};
    }
    if (!fixed_steps && params->t_end < 0.0) {
        throw BatchFail{MHDB_INVALID_ARGUMENT, "t_end must be non-negative"};
    }
    if (params->cfl <= 0.0) {
        throw BatchFail{MHDB_INVALID_ARGUMENT, "CFL number must be positive"};
    }
    if (params->limiter < kMinmod || params->limiter > kVanLeer) {
        throw BatchFail{MHDB_INVALID_ARGUMENT, "unknown slope limiter"};
    }
    if (init != nullptr && init->kind == MHDB_INIT_FOURIER && (init->coef == nullptr || init->kmax < 1)) {
        throw BatchFail{MHDB_INVALID_ARGUMENT, "Fourier initial state needs kmax >= 1 and coef"};
    }
    const int nxt = grid->nx + 2 * grid->ng, nyt = grid->ny + 2 * grid->ng;
    if (comps != nullptr && n_tot != static_cast<size_t>(nxt) * nyt) {
        throw BatchFail{MHDB_INVALID_ARGUMENT, "StateField size does not match Grid2D"};
    }
    SolveRec s;
    s.grid = *grid;
    s.params = *params;
    s.fixed = fixed_steps != 0;
    s.limiter = params->limiter;
    s.k = consts_of(*grid, *params);
    s.ni = s.k.ni_any != 0;
    s.geom.nx = grid->nx;
    s.geom.ny = grid->ny;
    s.geom.pitch = (grid->nx + 31) / 32 * 32;
    s.geom.bc_x = bc_x;
    s.geom.bc_y = bc_y;
    s.geom.plane = static_cast<size_t>(s.geom.pitch) * grid->ny;
    s.geom.ry0 = 0;
    s.geom.ry1 = grid->ny;
    const size_t bytes = 9 * s.geom.plane * 8;
    check(cudaMallocFromPoolAsync(&s.U, bytes, b->pool, b->stream), "cudaMallocFromPoolAsync(U)");
    const cudaError_t e2 = cudaMallocFromPoolAsync(&s.Us, bytes, b->pool, b->stream);
    if (e2 != cudaSuccess) {
        cudaFreeAsync(s.U, b->stream);
        check(e2, "cudaMallocFromPoolAsync(U*)");
    }
    s.bytes = 2 * bytes;
    if (b->precision != MHDB_FP64) {
        const MixedState u = mixed_view(s.U, s.geom), us = mixed_view(s.Us, s.geom);
        std::string err;
        if (!encode_march_maps(u, us, s.geom, &s.maps[0], &err) ||
            !encode_march_maps(us, u, s.geom, &s.maps[1], &err)) {
            cudaFreeAsync(s.U, b->stream);
            cudaFreeAsync(s.Us, b->stream);
            throw BatchFail{MHDB_CUDA_ERROR, err};
        }
    }
    const long long n = static_cast<long long>(grid->nx) * grid->ny;
    if (comps != nullptr) {
        double* stg = nullptr;
        const cudaError_t e3 = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&stg), 9 * n_tot * sizeof(double), b->pool, b->stream);
        if (e3 != cudaSuccess) {
            cudaFreeAsync(s.U, b->stream);
            cudaFreeAsync(s.Us, b->stream);
            check(e3, "cudaMallocFromPoolAsync(staging)");
        }
        for (int c = 0; c < 9; ++c) {
            check(cudaMemcpyAsync(stg + c * n_tot, comps[c], n_tot * sizeof(double),
                                  cudaMemcpyHostToDevice, b->stream), "cudaMemcpyAsync(state)");
        }
        if (b->precision == MHDB_FP64) {
            batch_unpack_f64<<<blocks_for(n, 256), 256, 0, b->stream>>>(stg, static_cast<double*>(s.U), s.geom, grid->ng, nxt, n_tot);
        } else {
            batch_unpack_mx<<<blocks_for(n, 256), 256, 0, b->stream>>>(stg, mixed_view(s.U, s.geom), s.geom, grid->ng, nxt, n_tot);
        }
        ++b->launches;
        check(cudaGetLastError(), "batch unpack launch");
        check(cudaFreeAsync(stg, b->stream), "cudaFreeAsync(staging)");
    } else {
        GenSpec spec{};
        spec.kind = init->kind;
        spec.kmax = init->kmax;
        spec.gamma = params->gamma;
        std::memcpy(spec.quad, init->quad, sizeof spec.quad);
        spec.x_min = grid->x_min;
        spec.x_max = grid->x_max;
        spec.y_min = grid->y_min;
        spec.y_max = grid->y_max;
        cudaError_t e;
        if (b->precision == MHDB_FP64) {
            e = launch_generate(b->stream, spec, init->coef, s.geom, static_cast<double*>(s.Us),
                                StoreF64{static_cast<double*>(s.U), s.geom.plane});
        } else {
            e = launch_generate(b->stream, spec, init->coef, s.geom, static_cast<double*>(s.Us),
                                StoreMx{mixed_view(s.U, s.geom), s.geom.plane});
        }
        b->launches += init->kind == MHDB_INIT_FOURIER ? 2 : 1;
        check(e, "generate");
        // the spectra were copied from caller memory; wait before returning
        check(cudaStreamSynchronize(b->stream), "cudaStreamSynchronize");
    }
    int slot;
    if (!b->free_slots.empty()) {
        slot = b->free_slots.back();
        b->free_slots.pop_back();
    } else {
        slot = b->next_slot++;
        grow_ctrl(b, b->next_slot);
    }
    s.slot = slot;
    Ctrl c0{};
    c0.t_end = fixed_steps ? static_cast<double>(INFINITY) : params->t_end;
    c0.max_steps = params->max_steps;
    b->ctrl_host[slot] = c0;
    check(cudaMemcpyAsync(b->ctrl + slot, &b->ctrl_host[slot], sizeof(Ctrl), cudaMemcpyHostToDevice,
                          b->stream), "cudaMemcpyAsync(ctrl)");
    const int init_blocks = static_cast<int>(std::min<long long>((n + kInitThreads - 1) / kInitThreads, 148LL * 4));
    if (b->precision == MHDB_FP64) {
        batch_cfl_init<kInitThreads><<<init_blocks, kInitThreads, 0, b->stream>>>(
            LoadF64{static_cast<const double*>(s.U), s.geom}, SpeedF64{}, s.geom, s.k, b->ctrl + slot);
    } else {
        batch_cfl_init<kInitThreads><<<init_blocks, kInitThreads, 0, b->stream>>>(
            LoadMx{mixed_view(s.U, s.geom), s.geom}, SpeedMx{}, s.geom, s.k, b->ctrl + slot);
    }
    ++b->launches;
    check(cudaGetLastError(), "batch cfl launch");
    check(cudaMemcpyAsync(&b->ctrl_host[slot], b->ctrl + slot, sizeof(Ctrl), cudaMemcpyDeviceToHost,
                          b->stream), "cudaMemcpyAsync(ctrl)");
    check(cudaStreamSynchronize(b->stream), "cudaStreamSynchronize");
    s.last = b->ctrl_host[slot];
    s.live = true;
    if (s.last.status & (kStatusBadDt | kStatusWaitTimeout)) {
        s.last.finished = 1;
    }
    int sid;
    if (!b->free_ids.empty()) {
        sid = b->free_ids.back();
        b->free_ids.pop_back();
        b->solves[sid] = s;
    } else {
        sid = static_cast<int>(b->solves.size());
        b->solves.push_back(s);
    }
    b->bytes_in_use += s.bytes;
    b->dirty = true;
    *id = sid;
}

} // namespace

extern "C" {

int mhdb_batch_add(mhdb_batch* b, const mhdb_grid* grid, const mhdb_params* params, int bc_x,
                   int bc_y, const double* const comps[9], size_t n_tot, int fixed_steps, int* id)
{
    return guarded(b, [&] {
        if (comps == nullptr) {
            throw BatchFail{MHDB_INVALID_ARGUMENT, "grid, params, state and id are required"};
        }
        add_solve(b, grid, params, bc_x, bc_y, comps, n_tot, nullptr, fixed_steps, id);
    });
}

int mhdb_batch_add_generated(mhdb_batch* b, const mhdb_grid* grid, const mhdb_params* params,
                             int bc_x, int bc_y, const mhdb_init* init, int fixed_steps, int* id)
{
    return guarded(b, [&] {
        if (init == nullptr || (init->kind != MHDB_INIT_FOURIER && init->kind != MHDB_INIT_QUADRANTS)) {
            throw BatchFail{MHDB_INVALID_ARGUMENT, "unknown initial-state kind"};
        }
        add_solve(b, grid, params, bc_x, bc_y, nullptr, 0, init, fixed_steps, id);
    });
}

int mhdb_batch_remove(mhdb_batch* b, int id)
{
    return guarded(b, [&] {
        if (id < 0 || id >= static_cast<int>(b->solves.size()) || !b->solves[id].live) {
            throw BatchFail{MHDB_INVALID_ARGUMENT, "unknown solve id"};
        }
        SolveRec& s = b->solves[id];
        check(cudaFreeAsync(s.U, b->stream), "cudaFreeAsync(U)");
        check(cudaFreeAsync(s.Us, b->stream), "cudaFreeAsync(U*)");
        if (s.delta) {
            check(cudaFreeAsync(s.delta, b->stream), "cudaFreeAsync(delta)");
        }
        b->bytes_in_use -= s.bytes;
        b->free_slots.push_back(s.slot);
        s = SolveRec{};
        b->free_ids.push_back(id);
        b->dirty = true;
    });
}

int mhdb_batch_step(mhdb_batch* b, int nsteps, int* active)
{
    return guarded(b, [&] {
        if (nsteps < 0) {
            throw BatchFail{MHDB_INVALID_ARGUMENT, "nsteps must be non-negative"};
        }
        if (b->precision == MHDB_FP64) {
            run_steps<PolicyF64>(b, nsteps);
        } else {
            run_steps<PolicyMixed>(b, nsteps);
        }
        poll(b);
        if (active != nullptr) {
            int n = 0;
            for (const auto& s : b->solves) {
                n += (s.live && s.last.finished == 0) ? 1 : 0;
            }
            *active = n;
        }
    });
}

int mhdb_batch_config_count(int precision)
{
    return precision == MHDB_FP64 ? BatchKernels<PolicyF64>::kVariants
                                  : BatchKernels<PolicyMixed>::kVariants;
}

int mhdb_batch_config_info(int precision, int config, int* tile_x, int* tile_y, int* threads,
                           int* kind)
{
    if (config < 0 || config >= mhdb_batch_config_count(precision)) {
        return MHDB_INVALID_ARGUMENT;
    }
    const BatchVariant v = precision == MHDB_FP64 ? BatchKernels<PolicyF64>::variant(config)
                                                  : BatchKernels<PolicyMixed>::variant(config);
    if (tile_x) *tile_x = v.tile_x;
    if (tile_y) *tile_y = v.tile_y;
    if (threads) *threads = v.threads;
    if (kind) *kind = v.kind;
    return MHDB_OK;
}

int mhdb_batch_set_config(mhdb_batch* b, int id, int config)
{
    return guarded(b, [&] {
        if (id < 0 || id >= static_cast<int>(b->solves.size()) || !b->solves[id].live) {
            throw BatchFail{MHDB_INVALID_ARGUMENT, "unknown solve id"};
        }
        if (config < -1 || config >= mhdb_batch_config_count(b->precision)) {
            throw BatchFail{MHDB_INVALID_ARGUMENT, "unknown batch configuration"};
        }
        SolveRec& s = b->solves[id];
        if (b->precision == MHDB_FP32 && s.stepped) {
            using K = BatchKernels<PolicyMixed>;
            const int v = config >= 0 ? config
                                      : K::default_variant(static_cast<long long>(s.grid.nx) * s.grid.ny);
            if ((v == K::kDeltaVariant) != s.alternates) {
                throw BatchFail{MHDB_INVALID_ARGUMENT,
                                "a solve that has been stepped cannot change between the stored "
                                "and the increment form"};
            }
        }
        if (s.config != config) {
            s.config = config;
            b->dirty = true;
        }
    });
}

int mhdb_batch_debug_stall_copies(mhdb_batch* b, int id, int extra_bytes)
{
    return guarded(b, [&] {
        if (id < 0 || id >= static_cast<int>(b->solves.size()) || !b->solves[id].live) {
            throw BatchFail{MHDB_INVALID_ARGUMENT, "unknown solve id"};
        }
        if (extra_bytes < 0 || extra_bytes > 4096) {
            throw BatchFail{MHDB_INVALID_ARGUMENT, "stall bytes must lie in [0, 4096]"};
        }
        SolveRec& s = b->solves[id];
        if (s.k.stall_tx != extra_bytes) {
            s.k.stall_tx = extra_bytes;
            b->dirty = true; // the descriptors carry the constants
        }
    });
}

int mhdb_batch_launch(mhdb_batch* b, int nsteps)
{
    return guarded(b, [&] {
        if (nsteps < 0) {
            throw BatchFail{MHDB_INVALID_ARGUMENT, "nsteps must be non-negative"};
        }
        if (b->precision == MHDB_FP64) {
            run_steps<PolicyF64>(b, nsteps);
        } else {
            run_steps<PolicyMixed>(b, nsteps);
        }
    });
}

int mhdb_batch_poll(mhdb_batch* b, int* active)
{
    return guarded(b, [&] {
        poll(b);
        if (active != nullptr) {
            int n = 0;
            for (const auto& s : b->solves) {
                n += (s.live && s.last.finished == 0) ? 1 : 0;
            }
            *active = n;
        }
    });
}

int mhdb_batch_status(mhdb_batch* b, int id, mhdb_result* result, int* finished)
{
    return guarded(b, [&] {
        if (id < 0 || id >= static_cast<int>(b->solves.size()) || !b->solves[id].live) {
            throw BatchFail{MHDB_INVALID_ARGUMENT, "unknown solve id"};
        }
        const SolveRec& s = b->solves[id];
        if (result != nullptr) {
            result->t = s.last.t;
            result->steps = s.last.steps;
            result->c_h = s.last.c_h;
        }
        if (finished != nullptr) {
            *finished = s.last.finished;
        }
        if (s.last.status & kStatusWaitTimeout) {
            throw BatchFail{MHDB_CUDA_ERROR, "stage kernel: a bulk-copy wait exceeded its limit"};
        }
        if (s.last.status & kStatusBadDt) {
            throw BatchFail{MHDB_BAD_TIMESTEP, "ssp_rk2_step requires positive dt"};
        }
        if (s.last.finished && !s.fixed && s.last.t < s.params.t_end) {
            throw BatchFail{MHDB_MAX_STEPS, "solve: reached max_steps before t_end"};
        }
    });
}

int mhdb_batch_download(mhdb_batch* b, int id, double* const comps[9], size_t n_tot)
{
    return guarded(b, [&] {
        if (id < 0 || id >= static_cast<int>(b->solves.size()) || !b->solves[id].live) {
            throw BatchFail{MHDB_INVALID_ARGUMENT, "unknown solve id"};
        }
        const SolveRec& s = b->solves[id];
        const int nxt = s.grid.nx + 2 * s.grid.ng, nyt = s.grid.ny + 2 * s.grid.ng;
        if (comps == nullptr || n_tot != static_cast<size_t>(nxt) * nyt) {
            throw BatchFail{MHDB_INVALID_ARGUMENT, "StateField size does not match Grid2D"};
        }
        // A solve that the last poll saw finished is final: every write to it completed before
        // that poll returned, and later steps skip it, so its download does not wait for the
        // steps in flight. Any other solve waits for everything issued so far.
        cudaStream_t st = b->dl_stream;
        if (s.last.finished == 0) {
            check(cudaEventRecord(b->dl_wait, b->stream), "cudaEventRecord");
            check(cudaStreamWaitEvent(st, b->dl_wait, 0), "cudaStreamWaitEvent");
        }
        double* stg = nullptr;
        check(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&stg), 9 * n_tot * sizeof(double), b->pool, st),
              "cudaMallocFromPoolAsync(staging)");
        const long long n = static_cast<long long>(n_tot);
        if (b->precision == MHDB_FP64) {
            batch_pack<<<blocks_for(n, 256), 256, 0, st>>>(
                LoadF64{static_cast<const double*>(s.U), s.geom}, stg, s.geom, s.grid.ng, nxt, nyt, n_tot);
        } else if (s.alternates) {
            batch_pack<<<blocks_for(n, 256), 256, 0, st>>>(
                LoadMxParity{mixed_view(s.U, s.geom), mixed_view(s.Us, s.geom), s.geom,
                             b->ctrl + s.slot},
                stg, s.geom, s.grid.ng, nxt, nyt, n_tot);
        } else {
            batch_pack<<<blocks_for(n, 256), 256, 0, st>>>(
                LoadMx{mixed_view(s.U, s.geom), s.geom}, stg, s.geom, s.grid.ng, nxt, nyt, n_tot);
        }
        ++b->launches;
        check(cudaGetLastError(), "batch pack launch");
        for (int c = 0; c < 9; ++c) {
            check(cudaMemcpyAsync(comps[c], stg + c * n_tot, n_tot * sizeof(double),
                                  cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync(download)");
        }
        check(cudaFreeAsync(stg, st), "cudaFreeAsync(staging)");
        check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    });
}

int mhdb_batch_info(const mhdb_batch* b, size_t* bytes_in_use, int* live, long long* launches)
{
    if (b == nullptr) {
        return MHDB_INVALID_ARGUMENT;
    }
    if (bytes_in_use) *bytes_in_use = b->bytes_in_use;
    if (live) {
        int n = 0;
        for (const auto& s : b->solves) n += s.live ? 1 : 0;
        *live = n;
    }
    if (launches) *launches = b->launches;
    return MHDB_OK;
}

void* mhdb_batch_stream(mhdb_batch* b)
{
    return b == nullptr ? nullptr : static_cast<void*>(b->stream);
}

} // extern "C"
