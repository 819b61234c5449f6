// Device-side seeded initial states, written straight into a solve's HBM state.
//
// Same fields as mhd_gpu_solver_b200/workloads.py (the host generator), evaluated on the device:
//   * Fourier state: five spectra C_q[ky][kx] (q = vx, vy, A_z, f1, f2; ky = -K..K, kx = 0..K)
//     drawn on the host; each field is Re(sum_k C_q[k] exp(i 2 pi (kx x + ky y))) at cell centres,
//     B = curl(A_z z^) from the analytic derivatives, v and B scaled to rms 1, f1 and f2 to rms 1,
//     rho = 1 + clip(0.2 f1, +-0.2), p = 1 + clip(0.1 f2, +-0.2), vz = Bz = psi = 0;
//   * four quadrants: per quadrant rho, p, vx, vy, By, with Bx = 0.75;
// then to_conservative (include/mhd/mhd_physics.hpp:41-57). The rms sums are reduced on the device
// in a fixed order.
#pragma once

#include "runtime_types.cuh"
#include "stage_mixed.cuh"

namespace mhdb {

constexpr int kGenThreads = 256;
constexpr int kGenBlocks = 296;

struct GenSpec {
    int kind; // 0 Fourier, 1 four quadrants
    int kmax;
    double gamma;
    double quad[4][5]; // rho, p, vx, vy, by per quadrant (x<.5,y<.5), (x>=.5,y<.5), (x<.5,y>=.5), (x>=.5,y>=.5)
    double x_min, x_max, y_min, y_max;
};

// Raw Fourier fields into the scratch planes: 0 f1, 1 vx, 2 vy, 4 f2, 5 bx, 6 by (unscaled),
// and per-block partial sums of vx^2+vy^2, bx^2+by^2, f1^2, f2^2.
static __global__ void __launch_bounds__(kGenThreads) gen_fourier_raw(const double2* __restrict__ coef,
                                                              GenSpec s, Geometry g,
                                                              double* __restrict__ scratch,
                                                              double* __restrict__ partial)
{
    const int K = s.kmax;
    const int KX = K + 1, KY = 2 * K + 1, NC = KX * KY;
    const double lx = s.x_max - s.x_min, ly = s.y_max - s.y_min;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const long long n = static_cast<long long>(g.nx) * g.ny;
    for (long long c = blockIdx.x * static_cast<long long>(kGenThreads) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * kGenThreads) {
        const int x = static_cast<int>(c % g.nx), y = static_cast<int>(c / g.nx);
        const double ux = (x + 0.5) / g.nx, uy = (y + 0.5) / g.ny; // (x - x_min)/lx
        double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0}; // vx, vy, bx, by, and (f1, f2 below)
        double f1 = 0.0, f2 = 0.0;
        for (int iy = 0; iy < KY; ++iy) {
            const int ky = iy - K;
            double sy, cy;
            sincospi(2.0 * ky * uy, &sy, &cy);
            for (int kx = 0; kx <= K; ++kx) {
                double sx, cx;
                sincospi(2.0 * kx * ux, &sx, &cx);
                // e = exp(i 2 pi (kx ux + ky uy))
                const double er = cx * cy - sx * sy, ei = sx * cy + cx * sy;
                const int m = iy * KX + kx;
                const double2 cvx = coef[0 * NC + m], cvy = coef[1 * NC + m];
                const double2 caz = coef[2 * NC + m], cf1 = coef[3 * NC + m], cf2 = coef[4 * NC + m];
                v[0] += cvx.x * er - cvx.y * ei;
                v[1] += cvy.x * er - cvy.y * ei;
                // Re(C (i w) e) = -w Im(C e)
                const double im_az = caz.x * ei + caz.y * er;
                v[2] += -(2.0 * M_PI / ly) * ky * im_az;  // bx = dA/dy
                v[3] += (2.0 * M_PI / lx) * kx * im_az;   // by = -dA/dx
                f1 += cf1.x * er - cf1.y * ei;
                f2 += cf2.x * er - cf2.y * ei;
            }
        }
        const size_t o = static_cast<size_t>(y) * g.pitch + x;
        scratch[0 * g.plane + o] = f1;
        scratch[1 * g.plane + o] = v[0];
        scratch[2 * g.plane + o] = v[1];
        scratch[4 * g.plane + o] = f2;
        scratch[5 * g.plane + o] = v[2];
        scratch[6 * g.plane + o] = v[3];
        acc[0] += v[0] * v[0] + v[1] * v[1];
        acc[1] += v[2] * v[2] + v[3] * v[3];
        acc[2] += f1 * f1;
        acc[3] += f2 * f2;
    }
    __shared__ double sh[4][kGenThreads];
    for (int q = 0; q < 4; ++q) {
        sh[q][threadIdx.x] = acc[q];
    }
    __syncthreads();
    for (int st = kGenThreads / 2; st > 0; st >>= 1) {
        if (static_cast<int>(threadIdx.x) < st) {
            for (int q = 0; q < 4; ++q) {
                sh[q][threadIdx.x] += sh[q][threadIdx.x + st];
            }
        }
        __syncthreads();
    }
    if (threadIdx.x < 4) {
        partial[threadIdx.x * gridDim.x + blockIdx.x] = sh[threadIdx.x][0];
    }
}

template <class Store>
__global__ void __launch_bounds__(kGenThreads) gen_finish(Store store, GenSpec s, Geometry g,
                                                         const double* __restrict__ scratch,
                                                         const double* __restrict__ partial,
                                                         int nblocks)
{
    // scale factors from the block partials (summed in block order by every thread)
    double sum[4] = {0.0, 0.0, 0.0, 0.0};
    if (s.kind == 0) {
        for (int b = 0; b < nblocks; ++b) {
            for (int q = 0; q < 4; ++q) {
                sum[q] += partial[q * nblocks + b];
            }
        }
    }
    const double ncell = static_cast<double>(g.nx) * g.ny;
    const double vs = 1.0 / sqrt(sum[0] / ncell), bs = 1.0 / sqrt(sum[1] / ncell);
    const double f1s = sqrt(sum[2] / ncell), f2s = sqrt(sum[3] / ncell);
    const long long n = static_cast<long long>(g.nx) * g.ny;
    for (long long c = blockIdx.x * static_cast<long long>(kGenThreads) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * kGenThreads) {
        const int x = static_cast<int>(c % g.nx), y = static_cast<int>(c / g.nx);
        const size_t o = static_cast<size_t>(y) * g.pitch + x;
        double rho, p, vx, vy, bx, by;
        if (s.kind == 0) {
            vx = scratch[1 * g.plane + o] * vs;
            vy = scratch[2 * g.plane + o] * vs;
            bx = scratch[5 * g.plane + o] * bs;
            by = scratch[6 * g.plane + o] * bs;
            const double f1 = scratch[0 * g.plane + o] / f1s;
            const double f2 = scratch[4 * g.plane + o] / f2s;
            rho = 1.0 + fmin(fmax(0.2 * f1, -0.2), 0.2);
            p = 1.0 + fmin(fmax(0.1 * f2, -0.2), 0.2);
        } else {
            const double xc = s.x_min + (x + 0.5) * ((s.x_max - s.x_min) / g.nx);
            const double yc = s.y_min + (y + 0.5) * ((s.y_max - s.y_min) / g.ny);
            const int qd = (xc < 0.5 ? 0 : 1) + (yc < 0.5 ? 0 : 2);
            rho = s.quad[qd][0];
            p = s.quad[qd][1];
            vx = s.quad[qd][2];
            vy = s.quad[qd][3];
            by = s.quad[qd][4];
            bx = 0.75;
        }
        const double e_kin = 0.5 * rho * (vx * vx + vy * vy);
        const double e_mag = 0.5 * (bx * bx + by * by);
        const double u[9] = {rho, rho * vx, rho * vy, 0.0, p / (s.gamma - 1.0) + e_kin + e_mag,
                             bx, by, 0.0, 0.0};
        store(o, u);
    }
}

struct StoreF64 {
    double* u;
    size_t plane;
    __device__ void operator()(size_t o, const double* v) const
    {
        for (int c = 0; c < 9; ++c) {
            u[c * plane + o] = v[c];
        }
    }
};

struct StoreMx {
    MixedState u;
    size_t plane;
    __device__ void operator()(size_t o, const double* v) const
    {
        for (int c = 0; c < 9; ++c) {
            split_store(u, c * plane + o, v[c]);
        }
    }
};

} // namespace mhdb

namespace mhdb {

// Host side: generate an initial state into `store` using `scratch` (9 double planes of the
// solve's geometry, e.g. its stage buffer). Allocates two small stream-ordered buffers (the
// spectra and the rms partials) and frees them on the stream.
template <class Store>
inline cudaError_t launch_generate(cudaStream_t st, const GenSpec& spec, const double* coef_host,
                                   const Geometry& g, double* scratch, Store store)
{
    double2* coef = nullptr;
    double* partial = nullptr;
    cudaError_t e = cudaSuccess;
    const int nblocks = kGenBlocks;
    if (spec.kind == 0) {
        const size_t nc = static_cast<size_t>(5) * (2 * spec.kmax + 1) * (spec.kmax + 1);
        if ((e = cudaMallocAsync(reinterpret_cast<void**>(&coef), nc * sizeof(double2), st)) != cudaSuccess) {
            return e;
        }
        if ((e = cudaMallocAsync(reinterpret_cast<void**>(&partial), 4 * nblocks * sizeof(double), st)) != cudaSuccess) {
            cudaFreeAsync(coef, st);
            return e;
        }
        e = cudaMemcpyAsync(coef, coef_host, nc * sizeof(double2), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            gen_fourier_raw<<<nblocks, kGenThreads, 0, st>>>(coef, spec, g, scratch, partial);
            gen_finish<<<nblocks, kGenThreads, 0, st>>>(store, spec, g, scratch, partial, nblocks);
            e = cudaGetLastError();
        }
        cudaFreeAsync(coef, st);
        cudaFreeAsync(partial, st);
        return e;
    }
    gen_finish<<<nblocks, kGenThreads, 0, st>>>(store, spec, g, scratch, nullptr, 0);
    return cudaGetLastError();
}

} // namespace mhdb
