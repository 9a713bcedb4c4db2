// field.cuh — the render-side thickness field as CUDA: the body splat, the
// decay draw and field_filter, into device buffers (no graphics stack).
#pragma once

#include "common.cuh"

namespace fcu {

// The projection and the splat of one field pass.
struct FieldGeom {
    float cx, cy;     // world x, y at the field's centre
    float ex, ey;     // world half extents the field spans (clip = (p - c) / e)
    float radius;     // splat radius, world units (1.5 h)
    uint32_t w, h;    // texels
    uint32_t lens;    // 0 none, 1 accel lens, 2 pressure lens, 3 density, 4 speed
    float lo, hi;     // the lens's ramp ends
};

// Fixed-point scale of the splat sums (integer atomics, so the sum does not
// depend on the order the particles land in).
constexpr double kFieldScale = 1048576.0;  // 2^20

// field[h][w] (r thickness, g lens-weighted thickness) *= keep; then
// acc[h][w][2] += the splat of every particle; then field += splat * acc,
// acc cleared. Two launches on `s`.
void launch_field_splat(cudaStream_t s, const FieldGeom &g, const float4 *pos, const float4 *vel,
                        const float4 *pvel, const float *density, uint32_t n, float keep, float splat,
                        float2 *field, unsigned long long *acc);
// field_filter: 7-tap separable Gaussian of field.r with clamped edges, then
// (blurred, x difference, y difference, Laplacian) per texel.
void launch_field_filter(cudaStream_t s, const FieldGeom &g, const float2 *field, float4 *out);

}  // namespace fcu
