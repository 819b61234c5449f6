// Device-side rasterisation of a fluid/solid mask from circles and rectangles.
//
// The rule of the reference's geometry helpers (gui/geometry.py:22-38 contains(), :130-156
// rasterize()): every interior cell starts fluid (1); the shapes are applied in order, each one
// painting the cells whose centre it contains solid (0) or fluid (1), so later shapes overwrite
// earlier ones. Cell centres are x_min + (i + 0.5) dx with dx = (x_max - x_min) / nx (and the same
// in y); a circle contains (x - cx)^2 + (y - cy)^2 <= r^2, a rectangle min(x0, x1) <= x <=
// max(x0, x1) and min(y0, y1) <= y <= max(y0, y1) (both inclusive). Every product and sum is
// rounded on its own (__dmul_rn / __dadd_rn: no fused multiply-adds), in numpy's order, so the mask
// is bit-identical to the host rasterisation of the same shapes.
#pragma once

#include <cstdint>

#include "mhd_b200.h"
#include "runtime_types.cuh"

namespace mhdb {

constexpr int kShapesPerLaunch = 64; // shapes passed by value per launch (2.6 KB of parameters)

struct ShapeList {
    mhdb_shape s[kShapesPerLaunch];
    int count;
    int first; // the first launch of a rasterisation starts every cell fluid
    double x_min, dx, y_min, dy;
};

__device__ __forceinline__ bool shape_contains(const mhdb_shape& s, double x, double y)
{
    if (s.kind == MHDB_SHAPE_CIRCLE) {
        const double ex = __dsub_rn(x, s.a), ey = __dsub_rn(y, s.b);
        return __dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)) <= __dmul_rn(s.c, s.c);
    }
    const double xa = fmin(s.a, s.c), xb = fmax(s.a, s.c);
    const double ya = fmin(s.b, s.d), yb = fmax(s.b, s.d);
    return x >= xa && x <= xb && y >= ya && y <= yb;
}

// One launch paints up to kShapesPerLaunch shapes onto the padded mask (rows of g.pitch bytes);
// *any_solid is set to 1 when a painted cell ends solid. Grid-stride over the interior cells.
__global__ void rasterize_shapes(uint8_t* __restrict__ mask, Geometry g, ShapeList L,
                                 int* __restrict__ any_solid)
{
    int solid_seen = 0;
    const long long n = static_cast<long long>(g.nx) * g.ny;
    for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(c % g.nx), j = static_cast<int>(c / g.nx);
        const double x = __dadd_rn(L.x_min, __dmul_rn(static_cast<double>(i) + 0.5, L.dx));
        const double y = __dadd_rn(L.y_min, __dmul_rn(static_cast<double>(j) + 0.5, L.dy));
        const size_t o = static_cast<size_t>(j) * g.pitch + i;
        uint8_t v = L.first ? uint8_t(1) : mask[o];
        for (int k = 0; k < L.count; ++k) {
            if (shape_contains(L.s[k], x, y)) {
                v = L.s[k].solid ? uint8_t(0) : uint8_t(1);
            }
        }
        mask[o] = v;
        solid_seen |= (v == 0);
    }
    if (__syncthreads_or(solid_seen) && threadIdx.x == 0) {
        *any_solid = 1;
    }
}

} // namespace mhdb
