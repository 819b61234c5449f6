// Device-side types shared by the stage kernels and the host runtime.
#pragma once

#include <cstddef>
#include <cstdint>

#include "physics.cuh"

namespace mhdb {

enum BcKind : int { kPeriodic = 0, kReflective = 1, kOutflow = 2 };

// Interior-only padded SoA layout: plane c of the state starts at c * plane; cell (x, y) of an
// interior of nx x ny cells sits at y * pitch + x. pitch is a multiple of 32 elements so every
// row starts on a 256-byte boundary. The fluid mask (when present) uses the same pitch.
struct Geometry {
    int nx, ny;
    int pitch;
    int bc_x, bc_y;
    size_t plane;
    // Rows [ry0, ry1) of the interior whose cells enter the signal-speed reduction and the
    // diagnostics: 0 and ny for a whole grid; the owned rows of one strip of a grid split into
    // strips with overlap rows (the overlap rows are copies of a neighbour's rows).
    int ry0, ry1;
};

__device__ __forceinline__ bool reduce_row(const Geometry& g, int y)
{
    return y >= g.ry0 && y < g.ry1;
}

// Per-solve constants, all computed on the host in FP64 exactly as the reference computes them.
struct Consts {
    double gamma, gm1, inv_gm1, glm_alpha;
    double inv_dx, inv_dy, inv_2dx, inv_2dy, h;
    double cfl, eta_max, dt_diff;
    NonIdealCoef ni;
    int ni_any;
    // Test hook of the bounded bulk-copy waits (zero in every ordinary solve): the TMA strip
    // marches arm the first row copy of the strip at the grid's origin for this many transaction
    // bytes more than its boxes deliver, so that phase never completes and its wait runs out.
    int stall_tx;
};

// kStatusWaitTimeout: a stage kernel gave up waiting for one of its own bulk copies (bounded
// wait); the solve stops and the host reports it as a CUDA error.
enum CtrlStatus : int { kStatusBadDt = 1, kStatusWaitTimeout = 2 };

// Device-resident time control (FP64 clock). Written only by the last CTA of the stage-2 (or
// initial CFL) kernel, read by every CTA of the following launches.
struct Ctrl {
    double t;       // simulation time since the start of this solve
    double dt;      // dt of the step about to run
    double c_h;     // max signal speed of the step about to run (GLM speed)
    double t_end;   // +inf for fixed-step solves
    unsigned long long ch_bits; // running max of the signal speed (IEEE bits, >= 0)
    unsigned int arrived;       // CTAs finished in the current reduction
    int steps;
    int max_steps;
    int finished;
    int status;
    // Nonzero: the reduction's last CTA leaves the running max in ch_bits and does not run
    // finish_step; the host combines ch_bits over the strips of a split grid (max) and then
    // launches finish_step_kernel.
    int defer;
};

// Boundary rule as an index map onto the interior (include/boundary_conditions/
// boundary_conditions.hpp:26-88): periodic wraps modulo n (valid for any offset, also when
// n < 2), outflow clamps to the nearest interior cell. Ghost (i, j) of the reference holds
// interior (map(i), map(j)) because x ghosts are filled first and y ghosts copy whole rows.
__device__ __forceinline__ int map_index(int x, int n, int bc)
{
    if (x >= 0 && x < n) {
        return x;
    }
    if (bc == kPeriodic) {
        int r = x % n;
        return r < 0 ? r + n : r;
    }
    return x < 0 ? 0 : n - 1;
}

// Host/device twin of the CFL step control (include/mhd/cfl.hpp:80-89 and the loop in
// include/mhd/time_integrator.hpp:84-99). Runs in one thread after the reduction is complete.
__device__ __forceinline__ void finish_step(Ctrl* ctrl, const Consts& k, bool advance)
{
    const double c_h = __longlong_as_double(static_cast<long long>(atomicExch(&ctrl->ch_bits, 0ull)));
    ctrl->arrived = 0u;
    if (advance) {
        ctrl->t += ctrl->dt;
        ctrl->steps += 1;
    }
    if (!(ctrl->t < ctrl->t_end) || ctrl->steps >= ctrl->max_steps ||
        (ctrl->status & kStatusWaitTimeout) != 0) {
        ctrl->finished = 1;
        return;
    }
    double dt = (c_h <= 0.0) ? static_cast<double>(INFINITY)
                             : k.cfl / (c_h * k.inv_dx + c_h * k.inv_dy);
    if (k.eta_max > 0.0) {
        dt = vmin(dt, k.dt_diff);
    }
    dt = vmin(dt, ctrl->t_end - ctrl->t);
    if (!(dt > 0.0) || isinf(dt)) {
        ctrl->status |= kStatusBadDt;
        ctrl->finished = 1;
        return;
    }
    ctrl->dt = dt;
    ctrl->c_h = c_h;
}

// CTA max of the per-thread signal speeds, one 64-bit atomic max per CTA (non-negative IEEE
// doubles order like their bit patterns), then the last CTA to arrive runs finish_step.
__device__ __forceinline__ void reduce_signal_speed_and_finish(double v, Ctrl* ctrl,
                                                               const Consts& k,
                                                               unsigned int nblocks,
                                                               bool advance)
{
    __shared__ double warp_max[32];
    __shared__ int is_last;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v = vmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        warp_max[warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        const int nw = (blockDim.x + 31) >> 5;
        for (int w = 0; w < nw; ++w) {
            m = vmax(m, warp_max[w]);
        }
        if (m > 0.0) {
            atomicMax(&ctrl->ch_bits, static_cast<unsigned long long>(__double_as_longlong(m)));
        }
        __threadfence();
        const unsigned int prev = atomicAdd(&ctrl->arrived, 1u);
        is_last = (prev == nblocks - 1u) ? 1 : 0;
    }
    __syncthreads();
    if (is_last != 0 && threadIdx.x == 0) {
        __threadfence();
        if (ctrl->defer == 0) {
            finish_step(ctrl, k, advance);
        } else {
            ctrl->arrived = 0u;
        }
    }
}

} // namespace mhdb
