// field.cu — the render-side thickness field as CUDA kernels.
//
// Reference: the body splat of crates/fluid-core/src/sim_sprites.wgsl
// (`body`, `weight`, `body_quad`, `lens_at`), the decay draw and the field
// pass of render.rs:3233-3282, and `field_filter` of sim_surface.wgsl. The
// reference rasterises one quad per particle into a half-float render
// target and blends; here each particle visits the texels whose centres its
// quad covers and adds the same falloff weight, and the field is a float2
// device buffer (r: thickness, g: thickness weighted by the lens) that the
// host reads or hands on. No graphics stack is involved.
//
// Weights are summed as 2^-20 fixed-point integers, so the field does not
// depend on the order particles land in; the decay and the blend constant
// then apply per texel in FP32 (-fmad=false, as the CPU oracle).
#include "field.cuh"

namespace fcu {

namespace {

constexpr int kFieldTile = 16, kFieldApron = 4;
constexpr int kFieldSpan = kFieldTile + 2 * kFieldApron;  // 24
constexpr int kFieldInner = kFieldTile + 2;               // 18
// sim_surface.wgsl BLUR: a 7-tap Gaussian, centre first.
__constant__ float kBlur[4] = {0.3125f, 0.234375f, 0.09375f, 0.015625f};

__device__ __forceinline__ float lens_value(const FieldGeom &g, float4 v, float4 pv, float rho) {
    float m;
    switch (g.lens) {  // sim_sprites.wgsl lens_at
    case 1u: m = v.w; break;
    case 2u: m = pv.w; break;
    case 3u: m = rho; break;
    default: m = sqrtf((v.x * v.x + v.y * v.y) + v.z * v.z); break;
    }
    return clampf((m - g.lo) / (g.hi - g.lo), 0.0f, 1.0f);
}

__device__ __forceinline__ unsigned long long fixed_w(float w) {
    return (unsigned long long)__double2ll_rn((double)w * kFieldScale);
}

// One thread per particle: its quad, radius 1.5 h around (x, y) projected
// orthographically, over the texels whose centres it covers; weight
// (1 - |corner|^2)^2 / 2 (sim_sprites.wgsl `weight`).
__global__ void __launch_bounds__(256) k_body_splat(FieldGeom g, const float4 *__restrict__ pos,
                                                    const float4 *__restrict__ vel,
                                                    const float4 *__restrict__ pvel,
                                                    const float *__restrict__ density, uint32_t n,
                                                    unsigned long long *acc) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = __ldg(&pos[i]);
    const float px = (p.x - g.cx) / g.ex, py = (p.y - g.cy) / g.ey;
    const float rx = g.radius / g.ex, ry = g.radius / g.ey;
    const float W = (float)g.w, H = (float)g.h;
    // a superset of the covered texels; the weight is zero outside the quad
    int tx0 = (int)floorf((px - rx + 1.0f) * 0.5f * W - 0.5f) - 1;
    int tx1 = (int)ceilf((px + rx + 1.0f) * 0.5f * W - 0.5f) + 1;
    int ty0 = (int)floorf((1.0f - (py + ry)) * 0.5f * H - 0.5f) - 1;
    int ty1 = (int)ceilf((1.0f - (py - ry)) * 0.5f * H - 0.5f) + 1;
    tx0 = tx0 < 0 ? 0 : tx0;
    ty0 = ty0 < 0 ? 0 : ty0;
    tx1 = tx1 > (int)g.w - 1 ? (int)g.w - 1 : tx1;
    ty1 = ty1 > (int)g.h - 1 ? (int)g.h - 1 : ty1;
    const float lv = g.lens ? lens_value(g, __ldg(&vel[i]), __ldg(&pvel[i]), __ldg(&density[i])) : 0.0f;
    for (int ty = ty0; ty <= ty1; ++ty) {
        const float yt = 1.0f - ((float)ty + 0.5f) / H * 2.0f;
        const float cy = (yt - py) / ry;
        for (int tx = tx0; tx <= tx1; ++tx) {
            const float xt = ((float)tx + 0.5f) / W * 2.0f - 1.0f;
            const float cx = (xt - px) / rx;
            const float falloff = fmaxf(1.0f - (cx * cx + cy * cy), 0.0f);
            const float w = falloff * falloff * 0.5f;
            if (w > 0.0f) {
                unsigned long long *a = &acc[2 * ((size_t)ty * g.w + tx)];
                atomicAdd(&a[0], fixed_w(w));
                if (g.lens) atomicAdd(&a[1], fixed_w(w * lv));
            }
        }
    }
}

// The decay draw and the splat's blend (render.rs:3253-3282): field * keep
// + splat * sum, and the sums cleared for the next pass.
__global__ void __launch_bounds__(256) k_field_resolve(float2 *field, unsigned long long *acc, uint32_t texels,
                                                       float keep, float splat) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= texels) return;
    const float r = (float)((double)acc[2 * t] / kFieldScale);
    const float gsum = (float)((double)acc[2 * t + 1] / kFieldScale);
    const float2 f = field[t];
    field[t] = make_float2(f.x * keep + splat * r, f.y * keep + splat * gsum);
    acc[2 * t] = 0ull;
    acc[2 * t + 1] = 0ull;
}

// sim_surface.wgsl field_filter: a 16 x 16 tile with a four-texel apron
// (edge-clamped loads), rows blurred, columns blurred, then the tile's
// centred differences off the blurred neighbours.
__global__ void __launch_bounds__(256) k_field_filter(FieldGeom g, const float2 *__restrict__ field,
                                                      float4 *out) {
    __shared__ float raw[kFieldSpan * kFieldSpan];
    __shared__ float rows[kFieldSpan * kFieldInner];
    const int lx = threadIdx.x, ly = threadIdx.y;
    const int lin = ly * kFieldTile + lx;
    const int ox = (int)blockIdx.x * kFieldTile - kFieldApron, oy = (int)blockIdx.y * kFieldTile - kFieldApron;
    for (int i = lin; i < kFieldSpan * kFieldSpan; i += kFieldTile * kFieldTile) {
        int cx = ox + i % kFieldSpan, cy = oy + i / kFieldSpan;
        cx = cx < 0 ? 0 : (cx > (int)g.w - 1 ? (int)g.w - 1 : cx);
        cy = cy < 0 ? 0 : (cy > (int)g.h - 1 ? (int)g.h - 1 : cy);
        raw[i] = field[(size_t)cy * g.w + cx].x;
    }
    __syncthreads();
    for (int i = lin; i < kFieldSpan * kFieldInner; i += kFieldTile * kFieldTile) {
        const int base = (i / kFieldInner) * kFieldSpan + i % kFieldInner + 3;
        float a = raw[base] * kBlur[0];
        for (int k = 1; k <= 3; ++k) a += (raw[base + k] + raw[base - k]) * kBlur[k];
        rows[i] = a;
    }
    __syncthreads();
    for (int i = lin; i < kFieldInner * kFieldInner; i += kFieldTile * kFieldTile) {
        const int base = i + 3 * kFieldInner;
        float a = rows[base] * kBlur[0];
        for (int k = 1; k <= 3; ++k) a += (rows[base + k * kFieldInner] + rows[base - k * kFieldInner]) * kBlur[k];
        raw[i] = a;
    }
    __syncthreads();
    const int centre = (ly + 1) * kFieldInner + lx + 1;
    const float d = raw[centre];
    const float xp = raw[centre + 1], xm = raw[centre - 1];
    const float yp = raw[centre + kFieldInner], ym = raw[centre - kFieldInner];
    const int tx = (int)blockIdx.x * kFieldTile + lx, ty = (int)blockIdx.y * kFieldTile + ly;
    if (tx < (int)g.w && ty < (int)g.h) {
        const float sx = 2.0f * g.ex / (float)g.w, sy = 2.0f * g.ey / (float)g.h;
        const float aspect = (sx * sx) / (sy * sy);
        const float lap = (xp + xm - 2.0f * d) + (yp + ym - 2.0f * d) * aspect;
        out[(size_t)ty * g.w + tx] = make_float4(d, xp - xm, ym - yp, lap);
    }
}

}  // namespace

void launch_field_splat(cudaStream_t s, const FieldGeom &g, const float4 *pos, const float4 *vel,
                        const float4 *pvel, const float *density, uint32_t n, float keep, float splat,
                        float2 *field, unsigned long long *acc) {
    if (n) k_body_splat<<<(n + 255) / 256, 256, 0, s>>>(g, pos, vel, pvel, density, n, acc);
    const uint32_t texels = g.w * g.h;
    k_field_resolve<<<(texels + 255) / 256, 256, 0, s>>>(field, acc, texels, keep, splat);
}

void launch_field_filter(cudaStream_t s, const FieldGeom &g, const float2 *field, float4 *out) {
    const dim3 grid((g.w + kFieldTile - 1) / kFieldTile, (g.h + kFieldTile - 1) / kFieldTile);
    k_field_filter<<<grid, dim3(kFieldTile, kFieldTile), 0, s>>>(g, field, out);
}

}  // namespace fcu
