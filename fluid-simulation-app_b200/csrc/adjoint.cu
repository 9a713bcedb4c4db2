// adjoint.cu — the differentiable DFSPH model and its hand-written adjoint,
// behind fluid_adjoint_*.
//
// The model is the substep of solve.cu (sim_solve.wgsl: density_div,
// the divergence Jacobi loop, forces_eval, forces_den_apply, the density
// Jacobi loop, integrate) written once over a real type T (float or
// double), with the particles kept in a fixed order (no reorder between
// substeps) and each particle's neighbour list built afresh every substep
// from the neighbour grid. It carries what moves the fluid: positions,
// velocities and the previous pressure (the warm start). Temperature, the
// acceleration and pressure lenses, fingers and frame rotation do not
// influence the motion and are left out.
//
// Differentiation holds three things fixed, as the controls move:
//   * each substep's neighbour lists (the kernel and its gradient vanish at
//     the support radius, so a pair entering or leaving adds nothing to
//     first order);
//   * each substep's divergence and density iteration counts, decided once
//     by the tolerance rule (FP64 residuals) on the first forward run and
//     frozen (fluid_adjoint_get/set_schedule carry them between handles);
//   * the branch of every clamp (speed ceiling, wall clamp, max(., 0)).
//
// The backward pass is reverse mode over the substeps. Every sweep has an
// adjoint kernel, one thread per particle: the particle's own terms are
// accumulated directly, its neighbours' shares go out by atomic adds. Pair
// terms use the analytic derivatives of the cubic spline (gradient and
// Hessian: d(gs x)/dx = gs I + (gs'/r) x x^T); the wall polynomials are
// differentiated by a three-slot forward-mode dual over the particle's
// position. The state is checkpointed every `checkpoint_every` frames and
// each segment is recomputed (storing its substeps' tapes) before it is
// reversed.
//
// The reference has no adjoint; nothing here replaces a reference call.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "grid.cuh"

namespace fcu {
int32_t report_error(int32_t code, const std::string &msg);
bool host_valid_config(const FluidSimConfig *c, std::string &why);
void host_params(const FluidSimConfig &c, uint32_t count, DevParams &P);
void host_seed(const FluidSimConfig &c, std::vector<float> &pos);
}  // namespace fcu

using namespace fcu;

#define AK(expr)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (expr);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return report_error(e_ == cudaErrorMemoryAllocation ? FLUID_ERR_OOM : FLUID_ERR_CUDA, \
                                std::string(#expr) + ": " + cudaGetErrorString(e_));              \
    } while (0)

#define DEV __device__ __forceinline__

namespace {

constexpr int kAdjThreads = 128;
constexpr uint32_t kModelCap = 128;  // neighbours a particle may have in the model
// The model's grid keys are cell * kAdjSlabs + the x slab, as a simulation's:
// each cell's particles in slab order, so the density sweep can skip the
// stencil cells and x slabs beyond the support (ADJ_CULL).
constexpr uint32_t kAdjSlabs = kSimSlabs;
#ifndef ADJ_CULL
#define ADJ_CULL 1
#endif

// ---- small vector and dual types --------------------------------------------
template <class T>
struct V3 {
    T x, y, z;
};
template <class T> DEV V3<T> mk(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T> DEV V3<T> operator+(V3<T> a, V3<T> b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T> DEV V3<T> operator-(V3<T> a, V3<T> b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T> DEV V3<T> operator-(V3<T> a) { return mk(-a.x, -a.y, -a.z); }
template <class T> DEV V3<T> operator*(T s, V3<T> a) { return mk(s * a.x, s * a.y, s * a.z); }
template <class T> DEV V3<T> operator*(V3<T> a, T s) { return mk(a.x * s, a.y * s, a.z * s); }
template <class T> DEV V3<T> operator/(V3<T> a, T s) { return mk(a.x / s, a.y / s, a.z / s); }
template <class T> DEV T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> DEV V3<T> zero3() { return mk(T(0), T(0), T(0)); }
template <class T> DEV T comp(V3<T> a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

// Fixed-order sums: each block adds its threads' four values by xor-shuffle
// trees in every warp, then thread q adds the warps' totals in warp order
// into part[4 * block + q]; k_sum_parts adds the blocks' partials in a fixed
// order. No floating-point atomics, so the sums are the same bits on every
// run (for a given launch shape).
DEV void block_sums4(double (&v)[4], double *part) {
    __shared__ double s[32][4];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    }
    if (lane == 0)
        for (int q = 0; q < 4; ++q) s[warp][q] = v[q];
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (uint32_t w = 0; w < nw; ++w) t += s[w][threadIdx.x];
        part[4 * (size_t)blockIdx.x + threadIdx.x] = t;
    }
}

// Where the four sums of k_sum_parts go (null: dropped); `add` adds them to
// what is there instead of overwriting it.
struct Sum4Out {
    double *dst[4];
    int add;
};

__global__ void __launch_bounds__(256) k_sum_parts(const double *__restrict__ part, uint32_t nb, Sum4Out o) {
    __shared__ double s[256];
    for (int q = 0; q < 4; ++q) {
        if (!o.dst[q]) continue;
        double t = 0.0;
        for (uint32_t b = threadIdx.x; b < nb; b += 256) t += part[4 * (size_t)b + q];
        s[threadIdx.x] = t;
        __syncthreads();
        for (uint32_t w = 128; w > 0; w >>= 1) {
            if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) *o.dst[q] = (o.add ? *o.dst[q] : 0.0) + s[0];
        __syncthreads();
    }
}

// Value and three partial derivatives (forward mode over a position).
template <class T>
struct D3 {
    T v, d0, d1, d2;
};
template <class T> DEV D3<T> dc(T c) { return D3<T>{c, T(0), T(0), T(0)}; }
template <class T> DEV D3<T> operator+(D3<T> a, D3<T> b) { return {a.v + b.v, a.d0 + b.d0, a.d1 + b.d1, a.d2 + b.d2}; }
template <class T> DEV D3<T> operator-(D3<T> a, D3<T> b) { return {a.v - b.v, a.d0 - b.d0, a.d1 - b.d1, a.d2 - b.d2}; }
template <class T> DEV D3<T> operator-(D3<T> a) { return {-a.v, -a.d0, -a.d1, -a.d2}; }
template <class T> DEV D3<T> operator*(D3<T> a, D3<T> b) {
    return {a.v * b.v, a.d0 * b.v + a.v * b.d0, a.d1 * b.v + a.v * b.d1, a.d2 * b.v + a.v * b.d2};
}
template <class T> DEV D3<T> operator/(D3<T> a, D3<T> b) {
    const T q = a.v / b.v;
    return {q, (a.d0 - q * b.d0) / b.v, (a.d1 - q * b.d1) / b.v, (a.d2 - q * b.d2) / b.v};
}
template <class T, class U, class = typename std::enable_if<std::is_arithmetic<U>::value>::type>
DEV D3<T> operator+(D3<T> a, U s) { return {a.v + T(s), a.d0, a.d1, a.d2}; }
template <class T, class U, class = typename std::enable_if<std::is_arithmetic<U>::value>::type>
DEV D3<T> operator+(U s, D3<T> a) { return {T(s) + a.v, a.d0, a.d1, a.d2}; }
template <class T, class U, class = typename std::enable_if<std::is_arithmetic<U>::value>::type>
DEV D3<T> operator-(D3<T> a, U s) { return {a.v - T(s), a.d0, a.d1, a.d2}; }
template <class T, class U, class = typename std::enable_if<std::is_arithmetic<U>::value>::type>
DEV D3<T> operator-(U s, D3<T> a) { return {T(s) - a.v, -a.d0, -a.d1, -a.d2}; }
template <class T, class U, class = typename std::enable_if<std::is_arithmetic<U>::value>::type>
DEV D3<T> operator*(D3<T> a, U s) { return {a.v * T(s), a.d0 * T(s), a.d1 * T(s), a.d2 * T(s)}; }
template <class T, class U, class = typename std::enable_if<std::is_arithmetic<U>::value>::type>
DEV D3<T> operator*(U s, D3<T> a) { return {T(s) * a.v, T(s) * a.d0, T(s) * a.d1, T(s) * a.d2}; }
template <class T, class U, class = typename std::enable_if<std::is_arithmetic<U>::value>::type>
DEV D3<T> operator/(D3<T> a, U s) { return {a.v / T(s), a.d0 / T(s), a.d1 / T(s), a.d2 / T(s)}; }
template <class T, class U, class = typename std::enable_if<std::is_arithmetic<U>::value>::type>
DEV D3<T> operator/(U s, D3<T> a) { return dc<T>(T(s)) / a; }
template <class T, class U> DEV bool operator<(D3<T> a, U s) { return a.v < T(s); }
template <class T, class U> DEV bool operator>(D3<T> a, U s) { return a.v > T(s); }
template <class T, class U> DEV bool operator>=(D3<T> a, U s) { return a.v >= T(s); }

template <class S> DEV S cst(float c) { return S(c); }
template <> DEV D3<float> cst<D3<float>>(float c) { return dc<float>(c); }
template <> DEV D3<double> cst<D3<double>>(float c) { return dc<double>((double)c); }
template <class S> DEV S sclamp(S v, float lo, float hi) {
    if (v < lo) return cst<S>(lo);
    if (v > hi) return cst<S>(hi);
    return v;
}

// ---- model constants ---------------------------------------------------------
// The model's constants are the FP32 values of solve.cu, promoted to T.
template <class T>
struct MP {
    T h, inv_h, sigma, sigma_h, sup2, m, rho0, rho0_half, eps;
    T lo[3], hi[3];
    T coh_c, coh_k, coh_near, gamma, beta, visc_k, k_near;
    float box_min[3], cell;
    uint32_t dims[3];
};

template <class T>
MP<T> model_params(const DevParams &P) {
    MP<T> p;
    p.h = P.h;
    p.inv_h = P.inv_h;
    p.sigma = P.sigma;
    p.sigma_h = P.sigma_h;
    p.sup2 = P.support_sq;
    p.m = P.mass;
    p.rho0 = P.rho0;
    p.rho0_half = 0.5f * P.rho0;
    p.eps = 0.01f * P.h * P.h;
    for (int a = 0; a < 3; ++a) {
        p.lo[a] = P.wall_lo[a];
        p.hi[a] = P.wall_hi[a];
        p.box_min[a] = P.box_min[a];
        p.dims[a] = P.dims[a];
    }
    p.cell = P.cell;
    // forces_eval's constants, in FP32 as the sweep computes them
    const float coh_c = 2.0f * P.h;
    const float c3 = coh_c * coh_c * coh_c;
    p.coh_c = coh_c;
    p.coh_k = 32.0f / (3.14159265f * c3 * c3 * c3);
    p.coh_near = c3 * c3 / 64.0f;
    const float c = 2.0f * P.h;
    p.gamma = SIGMA_WATER * 7040.0f / (21.0f * LATTICE_SIGMA * P.rho0 * P.rho0 * c * c);
    p.beta = SIGMA_WATER * (1.0f + COS_CONTACT) * 1558.4f / (LATTICE_SIGMA * P.rho0 * P.rho0 * c * c);
    p.visc_k = 2.0f * DYNAMIC_VISCOSITY;
    p.k_near = K_NEAR;
    return p;
}

// ---- wall terms over S = T or D3<T> (sim_solve.wgsl:213-361) -------------------
template <class S> DEV S w_density(S t) {
    if (t >= 2.0f) return cst<S>(0.0f);
    const S t3 = t * t * t;
    if (t < 1.0f) return 0.5f - 0.7f * t + t3 * (1.0f / 3.0f + t * t * (-0.15f + 0.05f * t));
    return 8.0f / 15.0f - 0.8f * t + t3 * (2.0f / 3.0f + t * (-0.5f + t * (0.15f - t / 60.0f)));
}
template <class S> DEV S w_gradient(S t) {
    if (t >= 2.0f) return cst<S>(0.0f);
    const S t2 = t * t;
    if (t < 1.0f) return 0.7f + t2 * (-1.0f + t2 * (0.75f - t * 0.3f));
    return 0.8f + t2 * (-2.0f + t * (2.0f + t * (-0.75f + t * 0.1f)));
}
template <class S> DEV S w_wedge(S t1, S t2) {
    if (t1 * t1 + t2 * t2 >= 4.0f) return cst<S>(0.0f);
    return (2.5005807e-01f +
            t2 * (-3.4681153e-01f +
                  t2 * (-4.0986882e-02f +
                        t2 * (3.0301620e-01f +
                              t2 * (-1.9202736e-01f + t2 * (4.6947582e-02f + t2 * (-3.8543515e-03f))))))) +
           t1 * ((-3.4681153e-01f +
                  t2 * (4.8587248e-01f +
                        t2 * (1.0092180e-02f +
                              t2 * (-2.9978363e-01f + t2 * (1.5320335e-01f + t2 * (-2.2544282e-02f)))))) +
                 t1 * ((-4.0986882e-02f +
                        t2 * (1.0092180e-02f +
                              t2 * (-5.4145610e-02f + t2 * (7.9597369e-02f + t2 * (-2.3350373e-02f))))) +
                       t1 * ((3.0301620e-01f +
                              t2 * (-2.9978363e-01f + t2 * (7.9597369e-02f + t2 * (-8.2431946e-03f)))) +
                             t1 * ((-1.9202736e-01f + t2 * (1.5320335e-01f + t2 * (-2.3350373e-02f))) +
                                   t1 * ((4.6947582e-02f + t2 * (-2.2544282e-02f)) +
                                         t1 * (-3.8543515e-03f))))));
}
template <class S> DEV S w_wedge_d(S t1, S t2) {
    if (t1 * t1 + t2 * t2 >= 4.0f) return cst<S>(0.0f);
    return (-3.4611994e-01f +
            t2 * (4.4757673e-01f +
                  t2 * (1.1932939e-01f +
                        t2 * (-4.6460101e-01f +
                              t2 * (2.7637253e-01f + t2 * (-6.2846025e-02f + t2 * (4.3871652e-03f))))))) +
           t1 * ((-6.3622823e-02f +
                  t2 * (2.0521006e-01f +
                        t2 * (-3.7311339e-01f +
                              t2 * (3.7508155e-01f + t2 * (-1.6629713e-01f + t2 * (2.5030129e-02f)))))) +
                 t1 * ((7.8352497e-01f +
                        t2 * (-1.2658344e+00f +
                              t2 * (5.8898945e-01f + t2 * (-1.0772903e-01f + t2 * (1.3535777e-02f))))) +
                       t1 * ((-4.9470084e-01f +
                              t2 * (9.1302071e-01f + t2 * (-3.4330355e-01f + t2 * (2.4034609e-02f)))) +
                             t1 * ((-2.5605481e-02f + t2 * (-2.0067981e-01f + t2 * (5.9854468e-02f))) +
                                   t1 * ((8.8898623e-02f + t2 * (3.9914838e-03f)) +
                                         t1 * (-1.7788321e-02f))))));
}
template <class S> DEV S w_adhesion(S t) {
    const S u = sclamp(2.0f - t, 0.0f, 2.0f);
    return u * u *
           (1.7847015e-3f +
            u * (3.3392196e-3f + u * (-4.3394677e-3f + u * (1.6711868e-3f + u * (-2.1788750e-4f)))));
}

// The fill of the truncated kernel by the six walls, minus the edge wedges.
template <class T, class S> DEV S w_fill(const MP<T> &p, S x, S y, S z) {
    const S tlx = (x - p.lo[0]) * p.inv_h, tly = (y - p.lo[1]) * p.inv_h, tlz = (z - p.lo[2]) * p.inv_h;
    const S thx = (p.hi[0] - x) * p.inv_h, thy = (p.hi[1] - y) * p.inv_h, thz = (p.hi[2] - z) * p.inv_h;
    S f = cst<S>(0.0f);
    f = f + (w_density(tlx) + w_density(thx));
    f = f + (w_density(tly) + w_density(thy));
    f = f + (w_density(tlz) + w_density(thz));
    S w = w_wedge(tlx, tly) + w_wedge(tlx, thy) + w_wedge(thx, tly) + w_wedge(thx, thy);
    w = w + (w_wedge(tlx, tlz) + w_wedge(tlx, thz) + w_wedge(thx, tlz) + w_wedge(thx, thz));
    w = w + (w_wedge(tly, tlz) + w_wedge(tly, thz) + w_wedge(thy, tlz) + w_wedge(thy, thz));
    return f - w;
}

template <class S> DEV S w_dsum(S t, S a, S b, S c, S d) {
    return w_wedge_d(t, a) + w_wedge_d(t, b) + w_wedge_d(t, c) + w_wedge_d(t, d);
}

// wall_grad_sum (sim_solve.wgsl:310-328)
template <class T, class S> DEV void w_grad(const MP<T> &p, S x, S y, S z, S &gx, S &gy, S &gz) {
    const T inv_h = T(1) / p.h;
    const S tlx = (x - p.lo[0]) * inv_h, tly = (y - p.lo[1]) * inv_h, tlz = (z - p.lo[2]) * inv_h;
    const S thx = (p.hi[0] - x) * inv_h, thy = (p.hi[1] - y) * inv_h, thz = (p.hi[2] - z) * inv_h;
    const T scale = p.rho0 * inv_h;
    gx = cst<S>(0.0f) - scale * (w_gradient(tlx) + w_dsum(tlx, tly, thy, tlz, thz));
    gx = gx + scale * (w_gradient(thx) + w_dsum(thx, tly, thy, tlz, thz));
    gy = cst<S>(0.0f) - scale * (w_gradient(tly) + w_dsum(tly, tlx, thx, tlz, thz));
    gy = gy + scale * (w_gradient(thy) + w_dsum(thy, tlx, thx, tlz, thz));
    gz = cst<S>(0.0f) - scale * (w_gradient(tlz) + w_dsum(tlz, tlx, thx, tly, thy));
    gz = gz + scale * (w_gradient(thz) + w_dsum(thz, tlx, thx, tly, thy));
}

// wall_adh_sum (sim_solve.wgsl:349-361)
template <class T, class S> DEV void w_adh(const MP<T> &p, S x, S y, S z, S &ax, S &ay, S &az) {
    const T inv_h = T(1) / p.h;
    ax = cst<S>(0.0f) - w_adhesion((x - p.lo[0]) * inv_h) + w_adhesion((p.hi[0] - x) * inv_h);
    ay = cst<S>(0.0f) - w_adhesion((y - p.lo[1]) * inv_h) + w_adhesion((p.hi[1] - y) * inv_h);
    az = cst<S>(0.0f) - w_adhesion((z - p.lo[2]) * inv_h) + w_adhesion((p.hi[2] - z) * inv_h);
}

template <class T> DEV V3<T> wall_grad(const MP<T> &p, V3<T> x) {
    V3<T> g;
    w_grad<T, T>(p, x.x, x.y, x.z, g.x, g.y, g.z);
    return g;
}

// J^T u for the Jacobian of a wall vector field at x (rows = components).
template <class T> struct J3 {
    T a[3][3];  // a[row][col] = d field_row / d x_col
};
template <class T> DEV V3<T> jt_mul(const J3<T> &J, V3<T> u) {
    return mk(J.a[0][0] * u.x + J.a[1][0] * u.y + J.a[2][0] * u.z,
              J.a[0][1] * u.x + J.a[1][1] * u.y + J.a[2][1] * u.z,
              J.a[0][2] * u.x + J.a[1][2] * u.y + J.a[2][2] * u.z);
}
template <class T> DEV void seed(V3<T> x, D3<T> &dx, D3<T> &dy, D3<T> &dz) {
    dx = D3<T>{x.x, T(1), T(0), T(0)};
    dy = D3<T>{x.y, T(0), T(1), T(0)};
    dz = D3<T>{x.z, T(0), T(0), T(1)};
}
template <class T> DEV void rows(J3<T> &J, D3<T> gx, D3<T> gy, D3<T> gz) {
    J.a[0][0] = gx.d0; J.a[0][1] = gx.d1; J.a[0][2] = gx.d2;
    J.a[1][0] = gy.d0; J.a[1][1] = gy.d1; J.a[1][2] = gy.d2;
    J.a[2][0] = gz.d0; J.a[2][1] = gz.d1; J.a[2][2] = gz.d2;
}
template <class T> DEV J3<T> wall_grad_jac(const MP<T> &p, V3<T> x) {
    D3<T> dx, dy, dz, gx, gy, gz;
    seed(x, dx, dy, dz);
    w_grad<T, D3<T>>(p, dx, dy, dz, gx, gy, gz);
    J3<T> J;
    rows(J, gx, gy, gz);
    return J;
}
template <class T> DEV J3<T> wall_adh_jac(const MP<T> &p, V3<T> x) {
    D3<T> dx, dy, dz, gx, gy, gz;
    seed(x, dx, dy, dz);
    w_adh<T, D3<T>>(p, dx, dy, dz, gx, gy, gz);
    J3<T> J;
    rows(J, gx, gy, gz);
    return J;
}
template <class T> DEV V3<T> fill_grad(const MP<T> &p, V3<T> x) {
    D3<T> dx, dy, dz;
    seed(x, dx, dy, dz);
    const D3<T> f = w_fill<T, D3<T>>(p, dx, dy, dz);
    return mk(f.d0, f.d1, f.d2);
}

// ---- the cubic spline and its radial derivatives (sim_solve.wgsl:176-196) -----
// W(r), dW/dr, gs = (dW/dr) / r (the gradient is gs x), and gs'(r).
template <class T>
struct Radial {
    T r, q, W, dW, gs, dgs;
};
template <class T> DEV Radial<T> radial(const MP<T> &p, T r2) {
    Radial<T> o;
    o.r = sqrt(r2);
    o.q = o.r * p.inv_h;
    const T q = o.q;
    T d2W;
    if (q < T(1)) {
        o.W = p.sigma * (T(1) - T(1.5f) * q * q * (T(1) - T(0.5f) * q));
        o.dW = p.sigma_h * (T(-3) * q + T(2.25f) * q * q);
        d2W = p.sigma_h * p.inv_h * (T(-3) + T(4.5f) * q);
    } else {
        const T t = T(2) - q;
        o.W = p.sigma * T(0.25f) * t * t * t;
        o.dW = p.sigma_h * (T(-0.75f) * t * t);
        d2W = p.sigma_h * p.inv_h * (T(1.5f) * t);
    }
    if (o.r < T(1e-9f)) {
        o.gs = T(0);
        o.dgs = T(0);
    } else {
        o.gs = o.dW / o.r;
        o.dgs = (d2W - o.gs) / o.r;
    }
    return o;
}
// H u, H = d(gs x)/dx = gs I + (gs'/r) x x^T
template <class T> DEV V3<T> hess(const Radial<T> &R, V3<T> x, V3<T> u) {
    if (R.r < T(1e-9f)) return zero3<T>();
    return R.gs * u + (R.dgs / R.r * dot(x, u)) * x;
}

// ---- forward kernels -----------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_m_pos4(const V3<T> *__restrict__ x, float4 *pos4, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pos4[i] = make_float4((float)x[i].x, (float)x[i].y, (float)x[i].z, 0.0f);
}

// Neighbour list of every particle (stencil order, grid order inside a
// cell) with each pair's gradient scale gs (into gsl when given), density,
// near density, alpha and the wall gradient. With `perm`
// null the particles are in the grid's cell order (slot k is particle k);
// otherwise slot k holds particle perm[k].
template <class T>
__global__ void __launch_bounds__(kAdjThreads) k_m_density(MP<T> p, uint32_t n, const V3<T> *__restrict__ x,
                                                           const float4 *__restrict__ pos4,
                                                           const uint32_t *__restrict__ starts,
                                                           const uint32_t *__restrict__ perm, uint32_t *nbr,
                                                           T *gsl, uint32_t *nbr_n, T *rho, T *rhon, T *alpha,
                                                           V3<T> *wg, uint32_t *over) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V3<T> xi = x[i];
    const float4 pf = make_float4((float)xi.x, (float)xi.y, (float)xi.z, 0.0f);
    const int bx = (int)axis_cell(pf.x, p.box_min[0], p.cell, p.dims[0]);
    const int by = (int)axis_cell(pf.y, p.box_min[1], p.cell, p.dims[1]);
    const int bz = (int)axis_cell(pf.z, p.box_min[2], p.cell, p.dims[2]);
    T w_sum = p.sigma, near = T(0), gsq = T(0);
    V3<T> gsum = zero3<T>();
    uint32_t cnt = 0;
#if ADJ_CULL
    // Stencil cells and x slabs beyond the support skipped, as in the
    // simulation's density sweep: on the float position the grid was built
    // from, the distances to the own cell's faces shrunk by a margin far
    // above both its rounding and the float / T difference of positions.
    const float cellf = p.cell, sup2f = (float)p.sup2;
    const float margin = 1e-3f * cellf + 1e-6f * (fabsf(pf.x) + fabsf(pf.y) + fabsf(pf.z));
    const float fx = pf.x - (p.box_min[0] + (float)bx * cellf);
    const float fy = pf.y - (p.box_min[1] + (float)by * cellf);
    const float fz = pf.z - (p.box_min[2] + (float)bz * cellf);
    const float xl = fmaxf(fx - margin, 0.0f), xh = fmaxf(cellf - fx - margin, 0.0f);
    const float yl = fmaxf(fy - margin, 0.0f), yh = fmaxf(cellf - fy - margin, 0.0f);
    const float zl = fmaxf(fz - margin, 0.0f), zh = fmaxf(cellf - fz - margin, 0.0f);
#endif
    for (int oz = -1; oz <= 1; ++oz)
        for (int oy = -1; oy <= 1; ++oy) {
            const int cz = bz + oz, cy = by + oy;
            if (cz < 0 || cz >= (int)p.dims[2] || cy < 0 || cy >= (int)p.dims[1]) continue;
            const uint32_t row = ((uint32_t)cz * p.dims[1] + (uint32_t)cy) * p.dims[0];
#if ADJ_CULL
            const float dperp = (oz < 0 ? zl * zl : (oz > 0 ? zh * zh : 0.0f)) +
                                (oy < 0 ? yl * yl : (oy > 0 ? yh * yh : 0.0f));
            if (dperp >= sup2f) continue;
            const int cx0 = (bx > 0 && dperp + xl * xl < sup2f) ? bx - 1 : bx;
            const int cx1 = (bx + 1 < (int)p.dims[0] && dperp + xh * xh < sup2f) ? bx + 1 : bx;
            const float w = sqrtf(sup2f - dperp) * 1.001f + margin;
            const float xa = pf.x - w, xb = pf.x + w;
            const uint32_t ca = axis_cell(xa, p.box_min[0], cellf, p.dims[0]);
            const uint32_t cb = axis_cell(xb, p.box_min[0], cellf, p.dims[0]);
            const uint32_t klo = max(ca * kAdjSlabs + axis_slab(xa, p.box_min[0], cellf, ca, kAdjSlabs),
                                     (uint32_t)cx0 * kAdjSlabs);
            const uint32_t khi = min(cb * kAdjSlabs + axis_slab(xb, p.box_min[0], cellf, cb, kAdjSlabs),
                                     (uint32_t)cx1 * kAdjSlabs + (kAdjSlabs - 1));
            uint32_t s = starts[row * kAdjSlabs + klo], e = starts[row * kAdjSlabs + khi + 1];
            if (s > e) s = e;
#else
            const int cx0 = bx > 0 ? bx - 1 : bx;
            const int cx1 = bx + 1 < (int)p.dims[0] ? bx + 1 : bx;
            uint32_t s = starts[(row + cx0) * kAdjSlabs], e = starts[(row + cx1 + 1) * kAdjSlabs];
#endif
            if (e > n) e = n;
            // candidates four at a time: their positions load together
            for (uint32_t k0 = s; k0 < e; k0 += 4) {
                uint32_t jj[4];
                V3<T> xj[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const uint32_t k = k0 + u;
                    const uint32_t jr = k < e ? (perm ? perm[k] : k) : i;
                    jj[u] = jr;
                    xj[u] = x[jr < n ? jr : i];
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                const uint32_t j = jj[u];
                if (k0 + u >= e || j == i || j >= n) continue;
                const V3<T> xij = xi - xj[u];
                const T r2 = dot(xij, xij);
                if (r2 >= p.sup2) continue;
                const Radial<T> R = radial(p, r2);
                w_sum += R.W;
                const T wn = R.q < T(1) ? T(1) - R.q : T(0);
                near += wn * wn * wn;
                const V3<T> gw = R.gs * xij;
                gsum = gsum + gw;
                gsq += dot(gw, gw);
                if (cnt < kModelCap) {
                    nbr[(size_t)cnt * n + i] = j;
                    if (gsl) gsl[(size_t)cnt * n + i] = R.gs;
                }
                cnt++;
                }
            }
        }
    nbr_n[i] = cnt < kModelCap ? cnt : kModelCap;
    if (cnt > kModelCap) atomicAdd(over, 1u);
    const T fill = w_fill<T, T>(p, xi.x, xi.y, xi.z);
    const T r = p.m * w_sum + p.rho0 * fill;
    const V3<T> g = wall_grad(p, xi);
    wg[i] = g;
    const V3<T> G = p.m * gsum + g;
    T den = dot(G, G) + p.m * p.m * gsq;
    if (den < T(1e-4f)) den = T(1e-4f);
    rho[i] = r;
    rhon[i] = near;
    alpha[i] = r / den;
}

// The substep's state in the grid's cell order: slot k takes particle
// perm[k] (positions, velocities, previous pressure, id).
template <class T>
__global__ void __launch_bounds__(256) k_m_gather(uint32_t n, const uint32_t *__restrict__ perm,
                                                  const V3<T> *__restrict__ x, const V3<T> *__restrict__ v,
                                                  const T *__restrict__ pp, const uint32_t *__restrict__ id,
                                                  V3<T> *xw, V3<T> *vw, T *ppw, uint32_t *idw, uint32_t *perm_out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint32_t j = perm[k];
    if (j >= n) j = k;  // only after a grid build that gave up
    xw[k] = x[j];
    vw[k] = v[j];
    ppw[k] = pp[j];
    idw[k] = id[j];
    perm_out[k] = j;
}

// Walks this lane's share of particle i's list in order, kMB entries at a
// time: the entries and their gradient scales, then the neighbours' records
// (load(j)), and only then use(gs, record) for each, so a batch's loads
// overlap.
constexpr int kMB = 4;
constexpr int kRB = 2;  // the reverse sweeps with wide records
// Each particle's list is shared by kLanes adjacent lanes of a warp: lane l
// takes entries l, l + kLanes, ... and the lanes' partial sums are folded by
// lane_sum (the model fixes its own summation order; at 64k particles one
// lane per particle leaves most of the GPU's warp slots empty).
#ifndef ADJ_LANES
#define ADJ_LANES 4
#endif
constexpr int kLanes = ADJ_LANES;
static_assert(32 % kLanes == 0 && kAdjThreads % kLanes == 0, "lanes of a particle share a warp");
template <class T>
DEV T lane_sum(T v) {
#pragma unroll
    for (int o = 1; o < kLanes; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <class T>
DEV V3<T> lane_sum(V3<T> v) {
    return mk(lane_sum(v.x), lane_sum(v.y), lane_sum(v.z));
}
// The particle and lane of a thread of a lane-split sweep; `live` is false
// for the launch's tail past n, whose lanes take part in the folds with an
// empty list and write nothing.
struct LaneOf {
    uint32_t i, lane;
    bool live;
};
DEV LaneOf lane_of(uint32_t n) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = t / kLanes;
    return LaneOf{i < n ? i : n - 1, t % kLanes, i < n};
}
template <class T, class R, class Load, class Use>
DEV void mwalk(const uint32_t *__restrict__ nbr, const T *__restrict__ gsl, uint32_t n, uint32_t i,
               uint32_t cnt, uint32_t lane, Load load, Use use) {
    for (uint32_t k = lane; k < cnt; k += kLanes * kMB) {
        uint32_t j[kMB];
        T g[kMB];
#pragma unroll
        for (int u = 0; u < kMB; ++u) {
            const uint32_t kk = k + u * kLanes;
            const bool ok = kk < cnt;
            j[u] = ok ? nbr[(size_t)kk * n + i] : i;
            g[u] = ok ? gsl[(size_t)kk * n + i] : T(0);
        }
        R r[kMB];
#pragma unroll
        for (int u = 0; u < kMB; ++u) r[u] = load(j[u]);
#pragma unroll
        for (int u = 0; u < kMB; ++u)
            if (k + u * kLanes < cnt) use(g[u], r[u]);
    }
}
template <class T> struct XV {
    V3<T> x, v;
};
template <class T> struct XK {
    V3<T> x;
    T kd;
};

// mwalk for the reverse sweeps, which keep no gradient scales: kB entries,
// then their records, then use(j, record) for each, in the lane's order.
template <int kB, class R, class Load, class Use>
DEV void rwalk(const uint32_t *__restrict__ nbr, uint32_t n, uint32_t i, uint32_t cnt, uint32_t lane, Load load,
               Use use) {
    for (uint32_t k = lane; k < cnt; k += kLanes * kB) {
        uint32_t j[kB];
#pragma unroll
        for (int u = 0; u < kB; ++u) j[u] = k + u * kLanes < cnt ? nbr[(size_t)(k + u * kLanes) * n + i] : i;
        R r[kB];
#pragma unroll
        for (int u = 0; u < kB; ++u) r[u] = load(j[u]);
#pragma unroll
        for (int u = 0; u < kB; ++u)
            if (k + u * kLanes < cnt) use(j[u], r[u]);
    }
}
template <class T> struct XVK {
    V3<T> x, v;
    T k;
};

// d_i = m sum (v_i - v_j).grad W_ij + v_i.wg_i
template <class T>
DEV T div_of(const MP<T> &p, uint32_t n, uint32_t i, const V3<T> *__restrict__ x, const V3<T> *__restrict__ v,
             const uint32_t *__restrict__ nbr, const T *__restrict__ gsl, uint32_t cnt, V3<T> wgi,
             uint32_t lane) {
    const V3<T> xi = x[i], vi = v[i];
    T d = T(0);
    mwalk<T, XV<T>>(
        nbr, gsl, n, i, cnt, lane, [&](uint32_t j) { return XV<T>{x[j], v[j]}; },
        [&](T gs, const XV<T> &q) { d += dot(vi - q.v, gs * (xi - q.x)); });
    return p.m * lane_sum(d) + dot(vi, wgi);
}

// div_of with each pair's gradient scale recomputed (the reverse sweeps,
// which keep no scales): the same values, so the same sum.
template <class T>
DEV T div_of_radial(const MP<T> &p, uint32_t n, uint32_t i, const V3<T> *__restrict__ x,
                    const V3<T> *__restrict__ v, const uint32_t *__restrict__ nbr, uint32_t cnt, V3<T> wgi,
                    uint32_t lane) {
    const V3<T> xi = x[i], vi = v[i];
    T d = T(0);
    rwalk<kMB, XV<T>>(
        nbr, n, i, cnt, lane, [&](uint32_t j) { return XV<T>{x[j], v[j]}; },
        [&](uint32_t, const XV<T> &q) {
            const V3<T> xij = xi - q.x;
            const Radial<T> R = radial(p, dot(xij, xij));
            d += dot(vi - q.v, R.gs * xij);
        });
    return p.m * lane_sum(d) + dot(vi, wgi);
}

// sum (kd_i + kd_j) grad W_ij
template <class T>
DEV V3<T> kappa_of(uint32_t n, uint32_t i, V3<T> xi, T kdi, const V3<T> *__restrict__ x,
                   const T *__restrict__ kd, const uint32_t *__restrict__ nbr, const T *__restrict__ gsl,
                   uint32_t cnt, uint32_t lane) {
    V3<T> s = zero3<T>();
    mwalk<T, XK<T>>(
        nbr, gsl, n, i, cnt, lane, [&](uint32_t j) { return XK<T>{x[j], kd[j]}; },
        [&](T gs, const XK<T> &q) { s = s + (kdi + q.kd) * (gs * (xi - q.x)); });
    return lane_sum(s);
}

// Divergence (den = 0) or density (den = 1) prediction; the residual term
// sums into *res (FP64).
template <class T>
__global__ void __launch_bounds__(kAdjThreads) k_m_kappa(MP<T> p, uint32_t n, int den, T dt,
                                                         const V3<T> *__restrict__ x, const V3<T> *__restrict__ v,
                                                         const uint32_t *__restrict__ nbr, const T *__restrict__ gsl,
                                                         const uint32_t *__restrict__ nbr_n, const T *__restrict__ rho,
                                                         const T *__restrict__ alpha, const V3<T> *__restrict__ wg,
                                                         T *kd, T *pinc, unsigned long long *res) {
    const LaneOf L = lane_of(n);
    const uint32_t i = L.i;
    double term = 0.0;
    const T d = div_of(p, n, i, x, v, nbr, gsl, L.live ? nbr_n[i] : 0u, wg[i], L.lane);
    if (L.live && L.lane == 0) {
        const T r = rho[i], a = alpha[i];
        if (!den) {
            const T dp = d > T(0) ? d : T(0);
            kd[i] = dp * a / dt / r;
            term = (double)dp * (double)dt / (double)p.rho0;
        } else {
            const T rs = r + dt * d;
            const T e = rs - p.rho0;
            const T kk = (e > T(0) ? e : T(0)) * a / (dt * dt);
            kd[i] = kk / r;
            pinc[i] = kk * r;
            const double t = (double)rs / (double)p.rho0 - 1.0;
            term = t > 0.0 ? t : 0.0;
        }
    }
    if (res) {
        // the production solve's exact sum: 2^-28 units added as integers
        const unsigned long long q = warp_sum_u64(fixed_term(term));
        if ((threadIdx.x & 31) == 0 && q) atomicAdd(res, q);
    }
}

// v_out = v_in - dt (m sum (kd_i + kd_j) grad W_ij + kd_i wg_i); pressure += pinc
template <class T>
__global__ void __launch_bounds__(kAdjThreads) k_m_apply(MP<T> p, uint32_t n, T dt, const V3<T> *__restrict__ x,
                                                         const V3<T> *v_in, V3<T> *v_out,
                                                         const uint32_t *__restrict__ nbr, const T *__restrict__ gsl,
                                                         const uint32_t *__restrict__ nbr_n, const T *__restrict__ kd,
                                                         const V3<T> *__restrict__ wg, const T *__restrict__ pinc,
                                                         T *pressure) {
    const LaneOf L = lane_of(n);
    const uint32_t i = L.i;
    const V3<T> xi = x[i];
    const T kdi = kd[i];
    const V3<T> s = kappa_of(n, i, xi, kdi, x, kd, nbr, gsl, L.live ? nbr_n[i] : 0u, L.lane);
    if (!L.live || L.lane != 0) return;
    const V3<T> dv = p.m * s + kdi * wg[i];
    v_out[i] = v_in[i] - dt * dv;
    if (pinc) pressure[i] += pinc[i];
}

// forces_eval without the heat terms (sim_solve.wgsl:524-592)
template <class T>
__global__ void __launch_bounds__(kAdjThreads) k_m_forces_eval(MP<T> p, uint32_t n, const V3<T> *__restrict__ x,
                                                               const V3<T> *__restrict__ v,
                                                               const uint32_t *__restrict__ nbr,
                                                               const uint32_t *__restrict__ nbr_n,
                                                               const T *__restrict__ rho, const T *__restrict__ rhon,
                                                               const T *__restrict__ pp, V3<T> *accel, V3<T> *blend,
                                                               T *kd, T *pressure) {
    const LaneOf L = lane_of(n);
    const uint32_t i = L.i;
    const V3<T> xi = x[i], vi = v[i];
    const T rho_i = rho[i], near_i = rhon[i];
    const uint32_t cnt = L.live ? nbr_n[i] : 0u;
    V3<T> visc = zero3<T>(), bl = zero3<T>(), near = zero3<T>(), ten = zero3<T>();
    struct Rec {
        V3<T> x, v;
        T rho, near;
    };
    rwalk<kRB, Rec>(nbr, n, i, cnt, L.lane, [&](uint32_t j) { return Rec{x[j], v[j], rho[j], rhon[j]}; },
                    [&](uint32_t, const Rec &q) {
        const V3<T> xij = xi - q.x;
        const T r2 = dot(xij, xij);
        const Radial<T> R = radial(p, r2);
        const T rho_j = q.rho;
        const T f = R.gs * r2 / (r2 + p.eps);
        const T pair = p.m / (rho_i * rho_j) * f;
        const V3<T> dv = vi - q.v;
        const T wn = R.q < T(1) ? T(1) - R.q : T(0);
        const T rr = R.r > T(1e-5f) ? R.r : T(1e-5f);
        near = near + ((near_i + q.near) * wn * wn / rr) * xij;
        visc = visc + (p.visc_k * pair) * dv;
        bl = bl - (p.m / rho_j * R.W) * dv;
        T C = T(0);
        if (R.r < p.coh_c && R.r >= T(1e-9f)) {
            const T cr = p.coh_c - R.r;
            const T a = cr * cr * cr * R.r * R.r * R.r;
            C = T(2) * R.r > p.coh_c ? p.coh_k * a : p.coh_k * (T(2) * a - p.coh_near);
        }
        const T corr = T(2) * p.rho0 / (rho_i + rho_j);
        const T rt = R.r > T(1e-9f) ? R.r : T(1e-9f);
        ten = ten - (corr * p.m * C / rt) * xij;
    });
    visc = lane_sum(visc);
    bl = lane_sum(bl);
    near = lane_sum(near);
    ten = lane_sum(ten);
    if (!L.live || L.lane != 0) return;
    V3<T> ad;
    w_adh<T, T>(p, xi.x, xi.y, xi.z, ad.x, ad.y, ad.z);
    accel[i] = visc + p.k_near * near + p.gamma * ten + (p.beta * p.rho0) * ad;
    blend[i] = bl;
    const T half = T(0.5f) * pp[i];
    kd[i] = half / (rho_i * rho_i);
    pressure[i] = half;
}

// v_out = v + dt (f + accel) + c blend - dt (m sum (kd_i + kd_j) grad W + kd_i wg)
template <class T>
__global__ void __launch_bounds__(kAdjThreads) k_m_forces_apply(MP<T> p, uint32_t n, T dt, V3<T> f, T c,
                                                                const V3<T> *__restrict__ x, const V3<T> *v_in,
                                                                V3<T> *v_out, const V3<T> *__restrict__ accel,
                                                                const V3<T> *__restrict__ blend,
                                                                const uint32_t *__restrict__ nbr,
                                                                const T *__restrict__ gsl,
                                                                const uint32_t *__restrict__ nbr_n,
                                                                const T *__restrict__ kd, const V3<T> *__restrict__ wg) {
    const LaneOf L = lane_of(n);
    const uint32_t i = L.i;
    const V3<T> xi = x[i];
    const T kdi = kd[i];
    const V3<T> s = kappa_of(n, i, xi, kdi, x, kd, nbr, gsl, L.live ? nbr_n[i] : 0u, L.lane);
    if (!L.live || L.lane != 0) return;
    const V3<T> forced = v_in[i] + dt * (f + accel[i]) + c * blend[i];
    v_out[i] = forced - dt * (p.m * s + kdi * wg[i]);
}

// integrate without the lenses and temperature (sim_solve.wgsl:709-756)
template <class T>
__global__ void __launch_bounds__(256) k_m_integrate(MP<T> p, uint32_t n, T dt, T vclamp, const V3<T> *x_in,
                                                     V3<T> *x_out, const V3<T> *__restrict__ v_in, V3<T> *v_out,
                                                     const T *__restrict__ pressure, T *pp, const T *__restrict__ rho) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3<T> v = v_in[i];
    const T speed = sqrt(dot(v, v));
    const T ceiling = rho[i] < p.rho0_half ? T(3) * vclamp : vclamp;
    if (speed > ceiling) v = v * (ceiling / speed);
    const V3<T> xi = x_in[i];
    V3<T> o;
    T pa[3] = {xi.x + v.x * dt, xi.y + v.y * dt, xi.z + v.z * dt};
    T va[3] = {v.x, v.y, v.z};
    T oa[3];
    for (int a = 0; a < 3; ++a) {
        T c = pa[a] < p.lo[a] ? p.lo[a] : pa[a];
        c = c > p.hi[a] ? p.hi[a] : c;
        if (c != pa[a]) va[a] = T(0);
        oa[a] = c;
    }
    o = mk(oa[0], oa[1], oa[2]);
    x_out[i] = o;
    v_out[i] = mk(va[0], va[1], va[2]);
    pp[i] = pressure[i];
}

// The loss sums: centre of mass and squared density deviation.
template <class T>
__global__ void __launch_bounds__(256) k_m_loss(MP<T> p, uint32_t n, const V3<T> *__restrict__ x,
                                                const T *__restrict__ rho, double *part) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    if (i < n) {
        s[0] = (double)x[i].x;
        s[1] = (double)x[i].y;
        s[2] = (double)x[i].z;
        const double d = (double)rho[i] / (double)p.rho0 - 1.0;
        s[3] = d * d;
    }
    block_sums4(s, part);
}

// ---- reverse kernels -------------------------------------------------------------

// integrate: x' = clamp(x + v_c dt), v' = v_c zeroed where clamped, v_c the
// speed-clamped v. In place: xbar, vbar hold the adjoints of x', v' on entry
// and of x, v on exit.
template <class T>
__global__ void __launch_bounds__(256) k_r_integrate(MP<T> p, uint32_t n, T dt, T vclamp,
                                                     const V3<T> *__restrict__ x, const V3<T> *__restrict__ v_pre,
                                                     const T *__restrict__ rho, V3<T> *xbar, V3<T> *vbar) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3<T> v = v_pre[i];
    const T speed = sqrt(dot(v, v));
    const T ceiling = rho[i] < p.rho0_half ? T(3) * vclamp : vclamp;
    const bool sc = speed > ceiling;
    const V3<T> vc = sc ? v * (ceiling / speed) : v;
    const V3<T> xi = x[i];
    const V3<T> xb = xbar[i], vb = vbar[i];
    T xo[3], vco[3];
    for (int a = 0; a < 3; ++a) {
        const T pa = comp(xi, a) + comp(vc, a) * dt;
        T c = pa < p.lo[a] ? p.lo[a] : pa;
        c = c > p.hi[a] ? p.hi[a] : c;
        if (c != pa) {
            xo[a] = T(0);
            vco[a] = T(0);
        } else {
            xo[a] = comp(xb, a);
            vco[a] = dt * comp(xb, a) + comp(vb, a);
        }
    }
    V3<T> vcb = mk(vco[0], vco[1], vco[2]);
    if (sc) {
        const V3<T> u = v / speed;
        vcb = (ceiling / speed) * (vcb - dot(u, vcb) * u);
    }
    xbar[i] = mk(xo[0], xo[1], xo[2]);
    vbar[i] = vcb;
}

// ---- reverse sweeps, gathered ------------------------------------------------
// The neighbour lists are symmetric: j lists i exactly when i lists j (both
// test the same squared distance, x_i - x_j and x_j - x_i differ only in
// sign). So the share that a pair (i, j) adds to particle j's adjoints through
// particle i's equation can be formed by j itself, from i's stored adjoints.
// Every reverse sweep below writes only its own particle's entries, with no
// atomics; the pair terms are evaluated once from each end.

// apply (v_out = v_in - dt (m sum (kd_i + kd_j) grad W_ij + kd_i wg_i)):
// given vbar (the adjoint of v_out, and of v_in), write the adjoint of kd and
// add the adjoint of x.
template <class T>
__global__ void __launch_bounds__(kAdjThreads) k_r_apply(MP<T> p, uint32_t n, T dt, const V3<T> *__restrict__ x,
                                                         const uint32_t *__restrict__ nbr,
                                                         const uint32_t *__restrict__ nbr_n, const T *__restrict__ kd,
                                                         const V3<T> *__restrict__ wg, const V3<T> *__restrict__ vbar,
                                                         T *kdbar, V3<T> *xbar) {
    const LaneOf L = lane_of(n);
    const uint32_t i = L.i;
    const V3<T> xi = x[i], vb = vbar[i];
    const T kdi = kd[i];
    const T c = -dt * p.m;
    const uint32_t cnt = L.live ? nbr_n[i] : 0u;
    T s = T(0);
    V3<T> xs = zero3<T>();
    rwalk<kMB, XVK<T>>(
        nbr, n, i, cnt, L.lane, [&](uint32_t j) { return XVK<T>{x[j], vbar[j], kd[j]}; },
        [&](uint32_t, const XVK<T> &q) {
            const V3<T> xij = xi - q.x;
            const Radial<T> R = radial(p, dot(xij, xij));
            const V3<T> dvb = vb - q.v;
            s += dot(R.gs * xij, dvb);
            xs = xs + (c * (kdi + q.k)) * hess(R, xij, dvb);
        });
    s = lane_sum(s);
    xs = lane_sum(xs);
    if (!L.live || L.lane != 0) return;
    const V3<T> wgi = wg[i];
    kdbar[i] = -dt * (p.m * s + dot(wgi, vb));
    const J3<T> J = wall_grad_jac(p, xi);
    xbar[i] = xbar[i] + xs + (-dt * kdi) * jt_mul(J, vb);
}

// kappa, first pass (div: kd = max(d,0) a / dt / rho; den: kk = max(rho +
// dt d - rho0, 0) a / dt^2, kd = kk / rho, pinc = kk rho): from kdbar and
// pbar (the pressure's adjoint), the adjoint of the divergence d (dbar) and
// the particle's own shares of the adjoints of rho and alpha.
template <class T>
__global__ void __launch_bounds__(kAdjThreads) k_r_kappa_a(MP<T> p, uint32_t n, int den, T dt,
                                                           const V3<T> *__restrict__ x, const V3<T> *__restrict__ v,
                                                           const uint32_t *__restrict__ nbr,
                                                           const uint32_t *__restrict__ nbr_n,
                                                           const T *__restrict__ rho, const T *__restrict__ alpha,
                                                           const V3<T> *__restrict__ wg, const T *__restrict__ kdbar,
                                                           const T *__restrict__ pbar, T *dbar, T *rhobar,
                                                           T *alphabar) {
    const LaneOf L = lane_of(n);
    const uint32_t i = L.i;
    const T d = div_of_radial(p, n, i, x, v, nbr, L.live ? nbr_n[i] : 0u, wg[i], L.lane);
    if (!L.live || L.lane != 0) return;
    const T r = rho[i], a = alpha[i], kb = kdbar[i];
    T db = T(0), rb = T(0), ab = T(0);
    if (!den) {
        if (d > T(0)) {
            db = kb * a / (dt * r);
            ab = kb * d / (dt * r);
            rb = -kb * d * a / (dt * r * r);
        }
    } else {
        const T e = r + dt * d - p.rho0;
        const T kk = (e > T(0) ? e : T(0)) * a / (dt * dt);
        const T pb = pbar[i];
        const T kkb = kb / r + pb * r;
        rb = -kb * kk / (r * r) + pb * kk;
        if (e > T(0)) {
            ab = kkb * e / (dt * dt);
            const T eb = kkb * a / (dt * dt);
            rb += eb;
            db = eb * dt;
        }
    }
    dbar[i] = db;
    rhobar[i] += rb;
    alphabar[i] += ab;
}

// kappa, second pass: d_i = m sum (v_i - v_j).grad W_ij + v_i.wg_i, so
// vbar_i += m sum (dbar_i + dbar_j) grad W_ij + dbar_i wg_i and
// xbar_i += m sum (dbar_i + dbar_j) H_ij (v_i - v_j) + dbar_i Jwg^T v_i.
template <class T>
__global__ void __launch_bounds__(kAdjThreads) k_r_kappa_b(MP<T> p, uint32_t n, const V3<T> *__restrict__ x,
                                                           const V3<T> *__restrict__ v,
                                                           const uint32_t *__restrict__ nbr,
                                                           const uint32_t *__restrict__ nbr_n,
                                                           const V3<T> *__restrict__ wg, const T *__restrict__ dbar,
                                                           V3<T> *vbar, V3<T> *xbar) {
    const LaneOf L = lane_of(n);
    const uint32_t i = L.i;
    const V3<T> xi = x[i], vi = v[i];
    const T di = dbar[i];
    const uint32_t cnt = L.live ? nbr_n[i] : 0u;
    V3<T> vs = zero3<T>(), xs = zero3<T>();
    rwalk<kMB, XVK<T>>(
        nbr, n, i, cnt, L.lane, [&](uint32_t j) { return XVK<T>{x[j], v[j], dbar[j]}; },
        [&](uint32_t, const XVK<T> &q) {
            const T c = p.m * (di + q.k);
            if (c == T(0)) return;
            const V3<T> xij = xi - q.x;
            const Radial<T> R = radial(p, dot(xij, xij));
            vs = vs + (c * R.gs) * xij;
            xs = xs + c * hess(R, xij, vi - q.v);
        });
    vs = lane_sum(vs);
    xs = lane_sum(xs);
    if (!L.live || L.lane != 0) return;
    vbar[i] = vbar[i] + vs + di * wg[i];
    if (di != T(0)) {
        const J3<T> J = wall_grad_jac(p, xi);
        xs = xs + di * jt_mul(J, vi);
    }
    xbar[i] = xbar[i] + xs;
}

// forces_apply: given vbar (adjoint of v_out; the same for v_in), store the
// adjoints of accel (dt vbar) and blend (c vbar), write the adjoint of the
// warm-start kd, add those of the force, of the XSPH coefficient and of x.
template <class T>
__global__ void __launch_bounds__(kAdjThreads) k_r_forces_apply(MP<T> p, uint32_t n, T dt, T c,
                                                                const V3<T> *__restrict__ x,
                                                                const V3<T> *__restrict__ blend,
                                                                const uint32_t *__restrict__ nbr,
                                                                const uint32_t *__restrict__ nbr_n,
                                                                const T *__restrict__ kd, const V3<T> *__restrict__ wg,
                                                                const V3<T> *__restrict__ vbar, V3<T> *abar, V3<T> *bbar,
                                                                T *kdbar, V3<T> *xbar, double *part) {
    const LaneOf L = lane_of(n);
    const uint32_t i = L.i;
    double red[4] = {0.0, 0.0, 0.0, 0.0};
    const V3<T> xi = x[i], vb = vbar[i];
    const T kdi = kd[i];
    const T cc = -dt * p.m;
    const uint32_t cnt = L.live ? nbr_n[i] : 0u;
    T s = T(0);
    V3<T> xs = zero3<T>();
    rwalk<kMB, XVK<T>>(
        nbr, n, i, cnt, L.lane, [&](uint32_t j) { return XVK<T>{x[j], vbar[j], kd[j]}; },
        [&](uint32_t, const XVK<T> &q) {
            const V3<T> xij = xi - q.x;
            const Radial<T> R = radial(p, dot(xij, xij));
            const V3<T> dvb = vb - q.v;
            s += dot(R.gs * xij, dvb);
            xs = xs + (cc * (kdi + q.k)) * hess(R, xij, dvb);
        });
    s = lane_sum(s);
    xs = lane_sum(xs);
    if (L.live && L.lane == 0) {
        abar[i] = dt * vb;
        bbar[i] = c * vb;
        red[0] = (double)dt * (double)vb.x;
        red[1] = (double)dt * (double)vb.y;
        red[2] = (double)dt * (double)vb.z;
        red[3] = (double)dot(blend[i], vb);
        const V3<T> wgi = wg[i];
        kdbar[i] = -dt * (p.m * s + dot(wgi, vb));
        const J3<T> J = wall_grad_jac(p, xi);
        xbar[i] = xbar[i] + xs + (-dt * kdi) * jt_mul(J, vb);
    }
    block_sums4(red, part);
}

// One pair's share of forces_eval in particle a's equation (neighbour b,
// x_ab = x_a - x_b, dv = v_a - v_b), reversed: given a's accel and blend
// adjoints, the adjoints of x_ab, dv, rho_a, rho_b and of (near_a + near_b).
template <class T>
struct PairBar {
    V3<T> gx, gdv;
    T rb_a, rb_b, nb;
};
template <class T>
DEV PairBar<T> forces_pair_bar(const MP<T> &p, V3<T> xab, T r2, const Radial<T> &R, V3<T> dv, T rho_a, T rho_b,
                               T near_a, T near_b, V3<T> ab, V3<T> bb) {
    PairBar<T> o;
    o.gx = zero3<T>();
    o.gdv = zero3<T>();
    o.rb_a = T(0);
    o.rb_b = T(0);
    const T r = R.r;
    const V3<T> ab_near = p.k_near * ab, ab_ten = p.gamma * ab;
    // viscosity: visc_k m / (rho_a rho_b) phi(r) dv, phi = gs r^2 / (r^2 + eps)
    {
        const T den = r2 + p.eps;
        const T phi = R.gs * r2 / den;
        const T s = p.visc_k * p.m / (rho_a * rho_b) * phi;
        o.gdv = o.gdv + s * ab;
        const T sb = dot(ab, dv);
        o.rb_a += -sb * s / rho_a;
        o.rb_b += -sb * s / rho_b;
        if (r >= T(1e-9f)) {
            // dphi/dr = (gs' r^2 + 2 gs r) / den - gs r^2 2 r / den^2
            const T dphi = (R.dgs * r2 + T(2) * R.gs * r) / den - R.gs * r2 * T(2) * r / (den * den);
            const T phib = sb * p.visc_k * p.m / (rho_a * rho_b);
            o.gx = o.gx + (phib * dphi / r) * xab;
        }
    }
    // near pressure: (near_a + near_b) psi(r) x, psi = wn^2 / max(r, 1e-5)
    {
        const T wn = R.q < T(1) ? T(1) - R.q : T(0);
        const T rr = r > T(1e-5f) ? r : T(1e-5f);
        const T psi = wn * wn / rr;
        const T sn = near_a + near_b;
        const T xa = dot(xab, ab_near);
        o.nb = psi * xa;
        T dpsi = T(0);
        if (wn > T(0)) {
            dpsi = T(2) * wn * (-p.inv_h) / rr;
            if (r > T(1e-5f)) dpsi -= wn * wn / (r * r);
        }
        o.gx = o.gx + (sn * psi) * ab_near;
        if (r >= T(1e-9f)) o.gx = o.gx + (sn * dpsi / r * xa) * xab;
    }
    // XSPH blend: -(m / rho_b) W dv
    {
        const T s = p.m / rho_b * R.W;
        o.gdv = o.gdv - s * bb;
        const T bdv = dot(bb, dv);
        o.rb_b += s / rho_b * bdv;
        if (r >= T(1e-9f)) o.gx = o.gx + (-(p.m / rho_b) * bdv * R.dW / r) * xab;
    }
    // surface tension: -corr m chi(r) x, chi = C(r) / max(r, 1e-9)
    {
        T C = T(0), dC = T(0);
        if (r < p.coh_c && r >= T(1e-9f)) {
            const T cr = p.coh_c - r;
            const T a = cr * cr * cr * r * r * r;
            const T da = T(-3) * cr * cr * r * r * r + T(3) * cr * cr * cr * r * r;
            if (T(2) * r > p.coh_c) {
                C = p.coh_k * a;
                dC = p.coh_k * da;
            } else {
                C = p.coh_k * (T(2) * a - p.coh_near);
                dC = p.coh_k * T(2) * da;
            }
        }
        const T rt = r > T(1e-9f) ? r : T(1e-9f);
        const T chi = C / rt;
        const T dchi = r > T(1e-9f) ? dC / r - C / (r * r) : T(0);
        const T sr = rho_a + rho_b;
        const T corr = T(2) * p.rho0 / sr;
        const T xa = dot(xab, ab_ten);
        const T corrb = -p.m * chi * xa;
        const T srb = -corrb * T(2) * p.rho0 / (sr * sr);
        o.rb_a += srb;
        o.rb_b += srb;
        o.gx = o.gx - (corr * p.m * chi) * ab_ten;
        if (r >= T(1e-9f)) o.gx = o.gx - (corr * p.m * dchi / r * xa) * xab;
    }
    return o;
}

// forces_eval: given abar, bbar (adjoints of accel and blend), kdbar (of the
// warm-start kd = pp / (2 rho^2)) and pbar (of pressure = pp / 2), add the
// adjoints of x, v, rho and near density, and write that of the previous
// pressure. Each pair is reversed in the particle's own equation and in the
// neighbour's.
template <class T>
__global__ void __launch_bounds__(kAdjThreads) k_r_forces_eval(MP<T> p, uint32_t n, const V3<T> *__restrict__ x,
                                                               const V3<T> *__restrict__ v,
                                                               const uint32_t *__restrict__ nbr,
                                                               const uint32_t *__restrict__ nbr_n,
                                                               const T *__restrict__ rho, const T *__restrict__ rhon,
                                                               const T *__restrict__ pp, const V3<T> *__restrict__ abar,
                                                               const V3<T> *__restrict__ bbar,
                                                               const T *__restrict__ kdbar, const T *__restrict__ pbar,
                                                               V3<T> *xbar, V3<T> *vbar, T *rhobar, T *rhonbar,
                                                               T *ppbar) {
    const LaneOf L = lane_of(n);
    const uint32_t i = L.i;
    const V3<T> xi = x[i], vi = v[i];
    const T rho_i = rho[i], near_i = rhon[i];
    const V3<T> ab = abar[i], bb = bbar[i];
    T rb_i = T(0);
    T nb_i = T(0);
    V3<T> xs = zero3<T>(), vs = zero3<T>();
    const uint32_t cnt = L.live ? nbr_n[i] : 0u;
    struct Rec {
        V3<T> x, v, ab, bb;
        T rho, near;
    };
    rwalk<kRB, Rec>(
        nbr, n, i, cnt, L.lane, [&](uint32_t j) { return Rec{x[j], v[j], abar[j], bbar[j], rho[j], rhon[j]}; },
        [&](uint32_t, const Rec &q) {
            const V3<T> xij = xi - q.x;
            const T r2 = dot(xij, xij);
            const Radial<T> R = radial(p, r2);
            const V3<T> dv = vi - q.v;
            const PairBar<T> own = forces_pair_bar(p, xij, r2, R, dv, rho_i, q.rho, near_i, q.near, ab, bb);
            const PairBar<T> oth = forces_pair_bar(p, -xij, r2, R, -dv, q.rho, rho_i, q.near, near_i, q.ab, q.bb);
            xs = xs + own.gx - oth.gx;
            vs = vs + own.gdv - oth.gdv;
            rb_i += own.rb_a + oth.rb_b;
            nb_i += own.nb + oth.nb;
        });
    xs = lane_sum(xs);
    vs = lane_sum(vs);
    rb_i = lane_sum(rb_i);
    nb_i = lane_sum(nb_i);
    if (!L.live || L.lane != 0) return;
    // own terms: kd = half / rho^2, pressure = half, half = pp / 2
    const T kb = kdbar[i];
    ppbar[i] = T(0.5f) * kb / (rho_i * rho_i) + T(0.5f) * pbar[i];
    rb_i += -kb * pp[i] / (rho_i * rho_i * rho_i);
    const J3<T> Ja = wall_adh_jac(p, xi);
    xs = xs + (p.beta * p.rho0) * jt_mul(Ja, ab);
    xbar[i] = xbar[i] + xs;
    vbar[i] = vbar[i] + vs;
    rhobar[i] += rb_i;
    rhonbar[i] += nb_i;
}

// density, first pass: with rhobar, alphabar complete, the total adjoint of
// rho (through rho itself and alpha = rho / max(|G|^2 + S, 1e-4)) and those
// of G = m sum grad W + wg(x) and S = m^2 sum |grad W|^2.
template <class T>
__global__ void __launch_bounds__(kAdjThreads) k_r_density_a(MP<T> p, uint32_t n, const V3<T> *__restrict__ x,
                                                             const uint32_t *__restrict__ nbr,
                                                             const uint32_t *__restrict__ nbr_n,
                                                             const T *__restrict__ rho, const T *__restrict__ rhobar,
                                                             const T *__restrict__ alphabar, T *rbt, V3<T> *gbar,
                                                             T *sbar) {
    const LaneOf L = lane_of(n);
    const uint32_t i = L.i;
    const V3<T> xi = x[i];
    const uint32_t cnt = L.live ? nbr_n[i] : 0u;
    V3<T> gsum = zero3<T>();
    T gsq = T(0);
    rwalk<kMB, V3<T>>(
        nbr, n, i, cnt, L.lane, [&](uint32_t j) { return x[j]; },
        [&](uint32_t, const V3<T> &xj) {
            const V3<T> xij = xi - xj;
            const Radial<T> R = radial(p, dot(xij, xij));
            const V3<T> gw = R.gs * xij;
            gsum = gsum + gw;
            gsq += dot(gw, gw);
        });
    gsum = lane_sum(gsum);
    gsq = lane_sum(gsq);
    if (!L.live || L.lane != 0) return;
    const V3<T> G = p.m * gsum + wall_grad(p, xi);
    const T den = dot(G, G) + p.m * p.m * gsq;
    const T r = rho[i];
    const T ab = alphabar[i];
    T rb = rhobar[i];
    V3<T> Gb = zero3<T>();
    T Sb = T(0);
    if (den > T(1e-4f)) {
        rb += ab / den;
        const T c = -ab * r / (den * den);
        Gb = (T(2) * c) * G;
        Sb = c;
    } else {
        rb += ab / T(1e-4f);
    }
    rbt[i] = rb;
    gbar[i] = Gb;
    sbar[i] = Sb;
}

// The gradient, with respect to x_ab, of particle a's density-pass terms
// weighted by its adjoints: rho (rb m grad W), G (m H Gb), S (2 Sb m^2 H
// grad W) and near density (nb 3 wn^2 d wn / d x).
template <class T>
DEV V3<T> density_pair_bar(const MP<T> &p, V3<T> xab, const Radial<T> &R, T rb, V3<T> Gb, T Sb, T nb) {
    const V3<T> gw = R.gs * xab;
    V3<T> g = (rb * p.m) * gw;
    g = g + p.m * hess(R, xab, Gb);
    g = g + (Sb * p.m * p.m * T(2)) * hess(R, xab, gw);
    if (R.q < T(1) && R.r >= T(1e-9f)) {
        const T wn = T(1) - R.q;
        g = g + (nb * T(3) * wn * wn * (-p.inv_h) / R.r) * xab;
    }
    return g;
}

// density, second pass: add the adjoint of x from every pair, reversed in
// the particle's own terms and in the neighbour's, and from the walls.
template <class T>
__global__ void __launch_bounds__(kAdjThreads) k_r_density_b(MP<T> p, uint32_t n, const V3<T> *__restrict__ x,
                                                             const uint32_t *__restrict__ nbr,
                                                             const uint32_t *__restrict__ nbr_n,
                                                             const T *__restrict__ rbt, const V3<T> *__restrict__ gbar,
                                                             const T *__restrict__ sbar,
                                                             const T *__restrict__ rhonbar, V3<T> *xbar) {
    const LaneOf L = lane_of(n);
    const uint32_t i = L.i;
    const V3<T> xi = x[i];
    const T rb = rbt[i], Sb = sbar[i], nb = rhonbar[i];
    const V3<T> Gb = gbar[i];
    const uint32_t cnt = L.live ? nbr_n[i] : 0u;
    V3<T> xs = zero3<T>();
    struct Rec {
        V3<T> x, gb;
        T rb, sb, nb;
    };
    rwalk<kRB, Rec>(
        nbr, n, i, cnt, L.lane, [&](uint32_t j) { return Rec{x[j], gbar[j], rbt[j], sbar[j], rhonbar[j]}; },
        [&](uint32_t, const Rec &q) {
            const V3<T> xij = xi - q.x;
            const Radial<T> R = radial(p, dot(xij, xij));
            xs = xs + density_pair_bar(p, xij, R, rb, Gb, Sb, nb) - density_pair_bar(p, -xij, R, q.rb, q.gb, q.sb, q.nb);
        });
    xs = lane_sum(xs);
    if (!L.live || L.lane != 0) return;
    const J3<T> J = wall_grad_jac(p, xi);
    xs = xs + jt_mul(J, Gb) + (rb * p.rho0) * fill_grad(p, xi);
    xbar[i] = xbar[i] + xs;
}

// The gather's adjoint: the adjoints of the cell-ordered inputs go back to
// the order the substep started from (a permutation, so no sums).
template <class T>
__global__ void __launch_bounds__(256) k_r_unpermute(uint32_t n, const uint32_t *__restrict__ perm,
                                                     const V3<T> *__restrict__ xb, const V3<T> *__restrict__ vb,
                                                     const T *__restrict__ ppb, V3<T> *xo, V3<T> *vo, T *ppo) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t j = perm[k];
    xo[j] = xb[k];
    vo[j] = vb[k];
    ppo[j] = ppb[k];
}

// The loss's own adjoints: xbar = 2 (com - target) / n, rhobar =
// 2 (rho / rho0 - 1) / (rho0 n); the rest zero.
template <class T>
__global__ void __launch_bounds__(256) k_r_loss(MP<T> p, uint32_t n, const T *__restrict__ rho, V3<T> gcom,
                                                V3<T> *xbar, V3<T> *vbar, T *rhobar, T *rhonbar, T *alphabar,
                                                T *ppbar) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    xbar[i] = gcom;
    vbar[i] = zero3<T>();
    rhobar[i] = T(2) * (rho[i] / p.rho0 - T(1)) / (p.rho0 * T(n));
    rhonbar[i] = T(0);
    alphabar[i] = T(0);
    ppbar[i] = T(0);
}

inline uint32_t nblk(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

}  // namespace

// ---- host ----------------------------------------------------------------------

struct AdjBase {
    virtual ~AdjBase() {}
    virtual int32_t forward(const double *forces, double xsph, const double target[3], double *loss) = 0;
    virtual int32_t backward(double *grad_forces, double *grad_xsph) = 0;
    virtual int32_t final_state(double *pos3, double *vel3) = 0;
    uint32_t n = 0, frames = 0, spf = 0, ce = 1;
    std::vector<uint32_t> div_it, den_it;
    bool frozen = false, have_forward = false;
    float last_forward_ms = 0.0f, last_backward_ms = 0.0f;
};

namespace {

// One substep's buffers; the tape of the backward keeps one per substep of
// a segment, the forward reuses one.
template <class T>
struct Tape {
    V3<T> *x = nullptr;
    T *pp = nullptr;
    uint32_t *nbr = nullptr, *nbr_n = nullptr;
    T *rho = nullptr, *rhon = nullptr, *alpha = nullptr;
    V3<T> *wg = nullptr, *blend = nullptr, *accel = nullptr;
    std::vector<V3<T> *> vdiv, vden;  // velocities before each apply, and after the loop
    std::vector<T *> kddiv, kdden;
    T *kdf = nullptr;  // warm-start kd
    uint32_t *perm = nullptr;  // slot k of the substep held particle perm[k] of the state before it
};

template <class T>
struct AdjImpl : AdjBase {
    FluidSimConfig cfg{};
    DevParams P{};
    MP<T> mp{};
    int device = 0;
    uint32_t cells = 0;
    T dt = T(0), vclamp = T(0);
    float div_tol = 0.01f, den_tol = 0.001f;
    uint32_t max_iters = 100;
    cudaStream_t stream = nullptr;
    std::vector<void *> allocs;
    // grid
    GridWork gw{};
    void *grid_ws = nullptr;
    float4 *pos4 = nullptr;
    uint32_t *keys = nullptr, *starts = nullptr, *perm = nullptr, *over = nullptr;
    // state and its checkpoints
    V3<T> *x = nullptr, *v = nullptr;
    T *pp = nullptr;
    uint32_t *id = nullptr, *id2 = nullptr;  // particle ids of the state's order
    std::vector<float> x0;
    std::vector<V3<T> *> ck_x, ck_v;
    std::vector<T *> ck_pp;
    std::vector<uint32_t *> ck_id;
    // forward scratch (one substep) and the backward's segment tapes
    Tape<T> work;
    std::vector<Tape<T>> seg;
    uint32_t seg_div_cap = 0, seg_den_cap = 0;
    Tape<T> fin;  // the final density pass of the loss
    T *kd = nullptr, *pinc = nullptr, *pressure = nullptr;
    T *gsl = nullptr;  // the substep's gradient scales beside its list (forward sweeps only)
    double *acc = nullptr;  // loss sums (4)
    unsigned long long *res_acc = nullptr;  // a loop's residual, 2^-28 fixed point
    double *part = nullptr;  // per-block partial sums of the fixed-order reductions
    // controls of the last forward
    std::vector<double> forces;
    double xsph = 0.0, target[3] = {0, 0, 0}, com[3] = {0, 0, 0};
    // adjoints
    V3<T> *xbar = nullptr, *vbar = nullptr, *abar = nullptr, *bbar = nullptr, *xbar2 = nullptr, *vbar2 = nullptr;
    T *rhobar = nullptr, *rhonbar = nullptr, *alphabar = nullptr, *kdbar = nullptr, *pbar = nullptr,
      *ppbar = nullptr, *ppbar_next = nullptr, *dbar = nullptr, *rbt = nullptr, *sbar = nullptr;
    V3<T> *gbar = nullptr;
    double *fbar = nullptr, *cbar = nullptr;

    template <class U>
    cudaError_t alloc(U **p, size_t cnt) {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, (cnt ? cnt : 1) * sizeof(U));
        if (e == cudaSuccess) {
            allocs.push_back(q);
            *p = (U *)q;
        }
        return e;
    }
    ~AdjImpl() override {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        for (void *p : allocs) cudaFree(p);
        if (grid_ws) cudaFree(grid_ws);
        if (stream) cudaStreamDestroy(stream);
    }

    int32_t alloc_tape(Tape<T> &t, uint32_t ndiv, uint32_t nden, bool with_x) {
        const size_t N = n;
        if (with_x) {
            AK(alloc(&t.x, N));
            AK(alloc(&t.pp, N));
            AK(alloc(&t.perm, N));
        }
        AK(alloc(&t.nbr, N * kModelCap));
        AK(alloc(&t.nbr_n, N));
        AK(alloc(&t.rho, N));
        AK(alloc(&t.rhon, N));
        AK(alloc(&t.alpha, N));
        AK(alloc(&t.wg, N));
        AK(alloc(&t.blend, N));
        AK(alloc(&t.accel, N));
        AK(alloc(&t.kdf, N));
        t.vdiv.assign(ndiv + 1, nullptr);
        t.vden.assign(nden + 1, nullptr);
        t.kddiv.assign(ndiv, nullptr);
        t.kdden.assign(nden, nullptr);
        for (auto &p : t.vdiv) AK(alloc(&p, N));
        for (auto &p : t.vden) AK(alloc(&p, N));
        for (auto &p : t.kddiv) AK(alloc(&p, N));
        for (auto &p : t.kdden) AK(alloc(&p, N));
        return FLUID_OK;
    }

    int32_t create(const FluidSimConfig &c, uint32_t frames_, uint32_t spf_, float frame_dt, float vclamp_,
                   uint32_t ce_) {
        cfg = c;
        device = c.device;
        frames = frames_;
        spf = spf_;
        ce = ce_;
        div_tol = c.div_tol;
        den_tol = c.den_tol;
        max_iters = c.max_iters;
        AK(cudaSetDevice(device));
        host_seed(c, x0);
        const uint64_t n64 = x0.size() / 4;
        if (n64 == 0 || n64 > (1u << 26)) return report_error(FLUID_ERR_ARG, "adjoint: 1..2^26 particles");
        n = (uint32_t)n64;
        host_params(c, n, P);
        mp = model_params<T>(P);
        const float dts = frame_dt / (float)spf;
        dt = T(dts);
        vclamp = T(vclamp_);
        const uint64_t c64 = (uint64_t)P.dims[0] * P.dims[1] * P.dims[2];
        if (c64 * kAdjSlabs >= 0xffffffffull) return report_error(FLUID_ERR_ARG, "adjoint: grid has too many cells");
        cells = (uint32_t)(c64 * kAdjSlabs);  // grid keys: cell * slabs + x slab
        AK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        const size_t N = n;
        AK(alloc(&pos4, N));
        AK(alloc(&keys, N));
        AK(alloc(&starts, (size_t)cells + 1));
        AK(alloc(&perm, N));
        AK(alloc(&over, 1));
        AK(cudaMalloc(&grid_ws, grid_work_bytes(n, cells)));
        gw = grid_work_carve(grid_ws, n, cells, nullptr);
        AK(alloc(&x, N));
        AK(alloc(&v, N));
        AK(alloc(&pp, N));
        AK(alloc(&id, N));
        AK(alloc(&id2, N));
        const uint32_t nck = (frames + ce - 1) / ce + 1;
        ck_x.assign(nck, nullptr);
        ck_v.assign(nck, nullptr);
        ck_pp.assign(nck, nullptr);
        ck_id.assign(nck, nullptr);
        for (uint32_t k = 0; k < nck; ++k) {
            AK(alloc(&ck_x[k], N));
            AK(alloc(&ck_v[k], N));
            AK(alloc(&ck_pp[k], N));
            AK(alloc(&ck_id[k], N));
        }
        // the forward's scratch substep holds the longest schedule any substep may take
        int32_t rc = alloc_tape(work, kMaxIters + 1, kMaxIters + 1, true);
        if (rc != FLUID_OK) return rc;
        rc = alloc_tape(fin, 0, 0, false);
        if (rc != FLUID_OK) return rc;
        AK(alloc(&kd, N));
        AK(alloc(&gsl, N * kModelCap));
        AK(alloc(&pinc, N));
        AK(alloc(&pressure, N));
        AK(alloc(&acc, 8));
        AK(alloc(&res_acc, 1));
        AK(alloc(&part, 4 * (size_t)std::max(nblk(n * kLanes, kAdjThreads), nblk(n, 256))));
        AK(alloc(&xbar, N));
        AK(alloc(&vbar, N));
        AK(alloc(&xbar2, N));
        AK(alloc(&vbar2, N));
        AK(alloc(&abar, N));
        AK(alloc(&bbar, N));
        AK(alloc(&rhobar, N));
        AK(alloc(&rhonbar, N));
        AK(alloc(&alphabar, N));
        AK(alloc(&kdbar, N));
        AK(alloc(&dbar, N));
        AK(alloc(&rbt, N));
        AK(alloc(&sbar, N));
        AK(alloc(&gbar, N));
        AK(alloc(&pbar, N));
        AK(alloc(&ppbar, N));
        AK(alloc(&ppbar_next, N));
        AK(alloc(&fbar, (size_t)frames * spf * 3));
        AK(alloc(&cbar, 1));
        return FLUID_OK;
    }

    int32_t load_initial() {
        std::vector<V3<T>> xs(n), zs(n);
        std::vector<uint32_t> ids(n);
        for (uint32_t i = 0; i < n; ++i) {
            xs[i] = V3<T>{T(x0[4 * i]), T(x0[4 * i + 1]), T(x0[4 * i + 2])};
            zs[i] = V3<T>{T(0), T(0), T(0)};
            ids[i] = i;
        }
        AK(cudaMemcpyAsync(id, ids.data(), 4ull * n, cudaMemcpyHostToDevice, stream));
        AK(cudaMemcpyAsync(x, xs.data(), sizeof(V3<T>) * n, cudaMemcpyHostToDevice, stream));
        AK(cudaMemcpyAsync(v, zs.data(), sizeof(V3<T>) * n, cudaMemcpyHostToDevice, stream));
        AK(cudaMemsetAsync(pp, 0, sizeof(T) * n, stream));
        AK(cudaStreamSynchronize(stream));
        return FLUID_OK;
    }

    // Neighbour grid of positions xs (the state's order): starts and perm.
    int32_t grid(const V3<T> *xs) {
        k_m_pos4<T><<<nblk(n, 256), 256, 0, stream>>>(xs, pos4, n);
        GridGeom g;
        for (int a = 0; a < 3; ++a) {
            g.min[a] = P.box_min[a];
            g.dims[a] = P.dims[a];
        }
        g.cell = P.cell;
        g.slabs = kAdjSlabs;
        AK(cudaMemsetAsync(gw.err, 0, 4, stream));
        AK(grid_build_enqueue(stream, pos4, n, g, keys, starts, perm, gw, nullptr, nullptr, nullptr, 1));
        return FLUID_OK;
    }

    // Neighbour grid of positions xs, then lists and densities into t (the
    // loss's pass over the final state, which is not in its own cell order).
    int32_t density(const V3<T> *xs, Tape<T> &t) {
        const int32_t rc = grid(xs);
        if (rc != FLUID_OK) return rc;
        k_m_density<T><<<nblk(n, kAdjThreads), kAdjThreads, 0, stream>>>(
            mp, n, xs, pos4, starts, perm, t.nbr, nullptr, t.nbr_n, t.rho, t.rhon, t.alpha, t.wg, over);
        AK(cudaGetLastError());
        return FLUID_OK;
    }

    int32_t read_residual(double *r) {
        unsigned long long q = 0;
        AK(cudaMemcpyAsync(&q, res_acc, 8, cudaMemcpyDeviceToHost, stream));
        AK(cudaStreamSynchronize(stream));
        *r = (double)q / kFixedScale / (double)n;
        return FLUID_OK;
    }

    // One substep of the model from the state (x, v, pp) to the state. With
    // `record`, t is a segment tape sized for this substep's iterations and
    // the substep runs its frozen schedule; otherwise t is the work tape and,
    // unless the schedule is frozen, the tolerance rule decides it.
    int32_t substep(uint32_t k, V3<T> f, T c, Tape<T> &t, bool record) {
        const bool decide = !frozen && !record;
        // the state in cell order, then lists and densities over slots
        int32_t rc = grid(x);
        if (rc != FLUID_OK) return rc;
        k_m_gather<T><<<nblk(n, 256), 256, 0, stream>>>(n, perm, x, v, pp, id, t.x, t.vdiv[0], t.pp, id2, t.perm);
        std::swap(id, id2);
        const uint32_t B = nblk(n, kAdjThreads), BL = nblk(n * kLanes, kAdjThreads);
        k_m_density<T><<<B, kAdjThreads, 0, stream>>>(mp, n, t.x, pos4, starts, nullptr, t.nbr, gsl, t.nbr_n,
                                                      t.rho, t.rhon, t.alpha, t.wg, over);
        // divergence loop
        uint32_t nd = decide ? 0u : div_it[k];
        if (decide) AK(cudaMemsetAsync(res_acc, 0, 8, stream));
        unsigned long long *res = decide ? res_acc : nullptr;
        k_m_kappa<T><<<BL, kAdjThreads, 0, stream>>>(mp, n, 0, dt, t.x, t.vdiv[0], t.nbr, gsl, t.nbr_n, t.rho, t.alpha,
                                                    t.wg, t.kddiv.empty() ? kd : t.kddiv[0], nullptr, res);
        uint32_t it = 0;
        for (;;) {
            if (decide) {
                double r;
                rc = read_residual(&r);
                if (rc != FLUID_OK) return rc;
                const bool go = it < max_iters && (r > (double)div_tol || it < 1u);
                if (!go) break;
            } else if (it >= nd) {
                break;
            }
            T *kd_t = t.kddiv[it];
            k_m_apply<T><<<BL, kAdjThreads, 0, stream>>>(mp, n, dt, t.x, t.vdiv[it], t.vdiv[it + 1], t.nbr, gsl, t.nbr_n,
                                                        kd_t, t.wg, nullptr, nullptr);
            ++it;
            if (decide || it < nd) {
                if (decide) AK(cudaMemsetAsync(res_acc, 0, 8, stream));
                k_m_kappa<T><<<BL, kAdjThreads, 0, stream>>>(mp, n, 0, dt, t.x, t.vdiv[it], t.nbr, gsl, t.nbr_n, t.rho,
                                                            t.alpha, t.wg, t.kddiv[it], nullptr, res);
            }
        }
        nd = it;
        // forces
        k_m_forces_eval<T><<<BL, kAdjThreads, 0, stream>>>(mp, n, t.x, t.vdiv[nd], t.nbr, t.nbr_n, t.rho, t.rhon,
                                                          t.pp, t.accel, t.blend, t.kdf, pressure);
        k_m_forces_apply<T><<<BL, kAdjThreads, 0, stream>>>(mp, n, dt, f, c, t.x, t.vdiv[nd], t.vden[0], t.accel,
                                                           t.blend, t.nbr, gsl, t.nbr_n, t.kdf, t.wg);
        // density loop
        const uint32_t ne = decide ? 0u : den_it[k];
        it = 0;
        for (;;) {
            if (!decide && it >= ne) break;
            if (decide) AK(cudaMemsetAsync(res_acc, 0, 8, stream));
            k_m_kappa<T><<<BL, kAdjThreads, 0, stream>>>(mp, n, 1, dt, t.x, t.vden[it], t.nbr, gsl, t.nbr_n, t.rho,
                                                        t.alpha, t.wg, t.kdden[it], pinc, res);
            if (decide) {
                double r;
                rc = read_residual(&r);
                if (rc != FLUID_OK) return rc;
                if (!(it < max_iters && r > (double)den_tol)) break;
            }
            k_m_apply<T><<<BL, kAdjThreads, 0, stream>>>(mp, n, dt, t.x, t.vden[it], t.vden[it + 1], t.nbr, gsl, t.nbr_n,
                                                        t.kdden[it], t.wg, pinc, pressure);
            ++it;
        }
        if (decide) {
            div_it[k] = nd;
            den_it[k] = it;
        }
        k_m_integrate<T><<<nblk(n, 256), 256, 0, stream>>>(mp, n, dt, vclamp, t.x, x, t.vden[it], v, pressure, pp,
                                                           t.rho);
        AK(cudaGetLastError());
        return FLUID_OK;
    }

    void set_controls(const double *f, double c, const double tg[3]) {
        forces.assign(f, f + 3 * (size_t)frames);
        xsph = c;
        for (int a = 0; a < 3; ++a) target[a] = tg[a];
    }
    V3<T> force_of(uint32_t k) const {
        const size_t fr = k / spf;
        return V3<T>{T(forces[3 * fr]), T(forces[3 * fr + 1]), T(forces[3 * fr + 2])};
    }

    int32_t check_overflow() {
        uint32_t o = 0;
        AK(cudaMemcpyAsync(&o, over, 4, cudaMemcpyDeviceToHost, stream));
        AK(cudaStreamSynchronize(stream));
        if (o) return report_error(FLUID_ERR_STATE, "adjoint: a particle has more than 128 neighbours");
        return FLUID_OK;
    }

    int32_t forward(const double *f, double c, const double tg[3], double *loss) override {
        AK(cudaSetDevice(device));
        set_controls(f, c, tg);
        const uint32_t S = frames * spf;
        if (!frozen) {
            div_it.assign(S, 0);
            den_it.assign(S, 0);
        }
        cudaEvent_t e0, e1;
        AK(cudaEventCreate(&e0));
        AK(cudaEventCreate(&e1));
        int32_t rc = load_initial();
        if (rc != FLUID_OK) return rc;
        AK(cudaMemsetAsync(over, 0, 4, stream));
        AK(cudaEventRecord(e0, stream));
        for (uint32_t fr = 0; fr < frames; ++fr) {
            if (fr % ce == 0) {
                const uint32_t q = fr / ce;
                AK(cudaMemcpyAsync(ck_x[q], x, sizeof(V3<T>) * n, cudaMemcpyDeviceToDevice, stream));
                AK(cudaMemcpyAsync(ck_v[q], v, sizeof(V3<T>) * n, cudaMemcpyDeviceToDevice, stream));
                AK(cudaMemcpyAsync(ck_pp[q], pp, sizeof(T) * n, cudaMemcpyDeviceToDevice, stream));
                AK(cudaMemcpyAsync(ck_id[q], id, 4ull * n, cudaMemcpyDeviceToDevice, stream));
            }
            for (uint32_t s = 0; s < spf; ++s) {
                const uint32_t k = fr * spf + s;
                rc = substep(k, force_of(k), T(xsph), work, false);
                if (rc != FLUID_OK) return rc;
            }
        }
        rc = density(x, fin);
        if (rc != FLUID_OK) return rc;
        k_m_loss<T><<<nblk(n, 256), 256, 0, stream>>>(mp, n, x, fin.rho, part);
        k_sum_parts<<<1, 256, 0, stream>>>(part, nblk(n, 256), Sum4Out{{acc + 1, acc + 2, acc + 3, acc + 4}, 0});
        AK(cudaEventRecord(e1, stream));
        double sums[4];
        AK(cudaMemcpyAsync(sums, acc + 1, 32, cudaMemcpyDeviceToHost, stream));
        AK(cudaStreamSynchronize(stream));
        AK(cudaEventElapsedTime(&last_forward_ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        rc = check_overflow();
        if (rc != FLUID_OK) return rc;
        double l = 0.0;
        for (int a = 0; a < 3; ++a) {
            com[a] = sums[a] / (double)n;
            l += (com[a] - target[a]) * (com[a] - target[a]);
        }
        l += sums[3] / (double)n;
        *loss = l;
        frozen = true;
        have_forward = true;
        return FLUID_OK;
    }

    int32_t ensure_segment_tapes() {
        uint32_t md = 0, me = 0;
        for (uint32_t k = 0; k < div_it.size(); ++k) {
            md = div_it[k] > md ? div_it[k] : md;
            me = den_it[k] > me ? den_it[k] : me;
        }
        const uint32_t len = ce * spf;
        if (seg.size() == len && md <= seg_div_cap && me <= seg_den_cap) return FLUID_OK;
        seg.assign(len, Tape<T>());
        for (auto &t : seg) {
            int32_t rc = alloc_tape(t, md, me, true);
            if (rc != FLUID_OK) return rc;
        }
        seg_div_cap = md;
        seg_den_cap = me;
        return FLUID_OK;
    }

    // The density pass reversed: total rho, G and S adjoints, then x.
    void reverse_density(const V3<T> *xs, const uint32_t *nb, const uint32_t *nbn, const T *rho) {
        const uint32_t B = nblk(n * kLanes, kAdjThreads);
        k_r_density_a<T><<<B, kAdjThreads, 0, stream>>>(mp, n, xs, nb, nbn, rho, rhobar, alphabar, rbt, gbar, sbar);
        k_r_density_b<T><<<B, kAdjThreads, 0, stream>>>(mp, n, xs, nb, nbn, rbt, gbar, sbar, rhonbar, xbar);
    }

    void reverse_substep(uint32_t k, const Tape<T> &t) {
        const uint32_t B = nblk(n * kLanes, kAdjThreads), B2 = nblk(n, 256);
        const uint32_t nd = div_it[k], ne = den_it[k];
        const size_t N = n;
        k_r_integrate<T><<<B2, 256, 0, stream>>>(mp, n, dt, vclamp, t.x, t.vden[ne], t.rho, xbar, vbar);
        cudaMemcpyAsync(pbar, ppbar_next, sizeof(T) * N, cudaMemcpyDeviceToDevice, stream);
        cudaMemsetAsync(rhobar, 0, sizeof(T) * N, stream);
        cudaMemsetAsync(rhonbar, 0, sizeof(T) * N, stream);
        cudaMemsetAsync(alphabar, 0, sizeof(T) * N, stream);
        for (uint32_t q = ne; q-- > 0;) {
            k_r_apply<T><<<B, kAdjThreads, 0, stream>>>(mp, n, dt, t.x, t.nbr, t.nbr_n, t.kdden[q], t.wg, vbar,
                                                        kdbar, xbar);
            k_r_kappa_a<T><<<B, kAdjThreads, 0, stream>>>(mp, n, 1, dt, t.x, t.vden[q], t.nbr, t.nbr_n, t.rho,
                                                          t.alpha, t.wg, kdbar, pbar, dbar, rhobar, alphabar);
            k_r_kappa_b<T><<<B, kAdjThreads, 0, stream>>>(mp, n, t.x, t.vden[q], t.nbr, t.nbr_n, t.wg, dbar, vbar,
                                                          xbar);
        }
        k_r_forces_apply<T><<<B, kAdjThreads, 0, stream>>>(mp, n, dt, T(xsph), t.x, t.blend, t.nbr, t.nbr_n, t.kdf,
                                                           t.wg, vbar, abar, bbar, kdbar, xbar, part);
        double *fk = fbar + 3 * (size_t)k;
        k_sum_parts<<<1, 256, 0, stream>>>(part, B, Sum4Out{{fk, fk + 1, fk + 2, cbar}, 1});
        k_r_forces_eval<T><<<B, kAdjThreads, 0, stream>>>(mp, n, t.x, t.vdiv[nd], t.nbr, t.nbr_n, t.rho, t.rhon,
                                                          t.pp, abar, bbar, kdbar, pbar, xbar, vbar, rhobar, rhonbar,
                                                          ppbar);
        for (uint32_t q = nd; q-- > 0;) {
            k_r_apply<T><<<B, kAdjThreads, 0, stream>>>(mp, n, dt, t.x, t.nbr, t.nbr_n, t.kddiv[q], t.wg, vbar,
                                                        kdbar, xbar);
            k_r_kappa_a<T><<<B, kAdjThreads, 0, stream>>>(mp, n, 0, dt, t.x, t.vdiv[q], t.nbr, t.nbr_n, t.rho,
                                                          t.alpha, t.wg, kdbar, nullptr, dbar, rhobar, alphabar);
            k_r_kappa_b<T><<<B, kAdjThreads, 0, stream>>>(mp, n, t.x, t.vdiv[q], t.nbr, t.nbr_n, t.wg, dbar, vbar,
                                                          xbar);
        }
        reverse_density(t.x, t.nbr, t.nbr_n, t.rho);
        // back to the order the substep started from
        k_r_unpermute<T><<<B2, 256, 0, stream>>>(n, t.perm, xbar, vbar, ppbar, xbar2, vbar2, ppbar_next);
        std::swap(xbar, xbar2);
        std::swap(vbar, vbar2);
    }

    int32_t backward(double *grad_forces, double *grad_xsph) override {
        if (!have_forward) return report_error(FLUID_ERR_STATE, "adjoint: backward needs a forward first");
        AK(cudaSetDevice(device));
        int32_t rc = ensure_segment_tapes();
        if (rc != FLUID_OK) return rc;
        cudaEvent_t e0, e1;
        AK(cudaEventCreate(&e0));
        AK(cudaEventCreate(&e1));
        AK(cudaEventRecord(e0, stream));
        const uint32_t S = frames * spf;
        AK(cudaMemsetAsync(fbar, 0, sizeof(double) * 3 * S, stream));
        AK(cudaMemsetAsync(cbar, 0, sizeof(double), stream));
        // the loss: x is the final state, fin its density pass
        const V3<T> gcom = V3<T>{T(2.0 * (com[0] - target[0]) / n), T(2.0 * (com[1] - target[1]) / n),
                                 T(2.0 * (com[2] - target[2]) / n)};
        k_r_loss<T><<<nblk(n, 256), 256, 0, stream>>>(mp, n, fin.rho, gcom, xbar, vbar, rhobar, rhonbar, alphabar,
                                                      ppbar_next);
        reverse_density(x, fin.nbr, fin.nbr_n, fin.rho);
        AK(cudaGetLastError());
        const uint32_t nseg = (frames + ce - 1) / ce;
        for (uint32_t q = nseg; q-- > 0;) {
            const uint32_t f0 = q * ce, f1 = (f0 + ce < frames) ? f0 + ce : frames;
            // recompute the segment from its checkpoint, keeping every substep's tape
            AK(cudaMemcpyAsync(x, ck_x[q], sizeof(V3<T>) * n, cudaMemcpyDeviceToDevice, stream));
            AK(cudaMemcpyAsync(v, ck_v[q], sizeof(V3<T>) * n, cudaMemcpyDeviceToDevice, stream));
            AK(cudaMemcpyAsync(pp, ck_pp[q], sizeof(T) * n, cudaMemcpyDeviceToDevice, stream));
            AK(cudaMemcpyAsync(id, ck_id[q], 4ull * n, cudaMemcpyDeviceToDevice, stream));
            for (uint32_t k = f0 * spf; k < f1 * spf; ++k) {
                rc = substep(k, force_of(k), T(xsph), seg[k - f0 * spf], true);
                if (rc != FLUID_OK) return rc;
            }
            for (uint32_t k = f1 * spf; k-- > f0 * spf;) reverse_substep(k, seg[k - f0 * spf]);
            AK(cudaGetLastError());
        }
        AK(cudaEventRecord(e1, stream));
        std::vector<double> fb(3 * (size_t)S);
        double cb = 0.0;
        AK(cudaMemcpyAsync(fb.data(), fbar, sizeof(double) * 3 * S, cudaMemcpyDeviceToHost, stream));
        AK(cudaMemcpyAsync(&cb, cbar, sizeof(double), cudaMemcpyDeviceToHost, stream));
        AK(cudaStreamSynchronize(stream));
        AK(cudaEventElapsedTime(&last_backward_ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        // the state is back at the last segment's end: restore the final state
        // by re-running nothing; the final positions are still in the loss pass
        if (grad_forces) {
            for (uint32_t fr = 0; fr < frames; ++fr)
                for (int a = 0; a < 3; ++a) {
                    double s = 0.0;
                    for (uint32_t j = 0; j < spf; ++j) s += fb[3 * ((size_t)fr * spf + j) + a];
                    grad_forces[3 * (size_t)fr + a] = s;
                }
        }
        if (grad_xsph) *grad_xsph = cb;
        have_forward = false;  // the state was overwritten by the recomputation
        return FLUID_OK;
    }

    int32_t final_state(double *pos3, double *vel3) override {
        if (!have_forward) return report_error(FLUID_ERR_STATE, "adjoint: no forward state to read");
        AK(cudaSetDevice(device));
        std::vector<V3<T>> a(n), b(n);
        std::vector<uint32_t> ids(n);
        AK(cudaMemcpyAsync(a.data(), x, sizeof(V3<T>) * n, cudaMemcpyDeviceToHost, stream));
        AK(cudaMemcpyAsync(b.data(), v, sizeof(V3<T>) * n, cudaMemcpyDeviceToHost, stream));
        AK(cudaMemcpyAsync(ids.data(), id, 4ull * n, cudaMemcpyDeviceToHost, stream));
        AK(cudaStreamSynchronize(stream));
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t i = ids[k] < n ? ids[k] : k;
            if (pos3) {
                pos3[3 * i] = (double)a[k].x;
                pos3[3 * i + 1] = (double)a[k].y;
                pos3[3 * i + 2] = (double)a[k].z;
            }
            if (vel3) {
                vel3[3 * i] = (double)b[k].x;
                vel3[3 * i + 1] = (double)b[k].y;
                vel3[3 * i + 2] = (double)b[k].z;
            }
        }
        return FLUID_OK;
    }
};

}  // namespace

struct FluidAdjoint {
    AdjBase *impl = nullptr;
    uint32_t precision = 32;
};

extern "C" {

FluidAdjoint *fluid_adjoint_create(const FluidSimConfig *cfg, uint32_t frames, uint32_t substeps_per_frame,
                                   float frame_dt, float v_clamp, uint32_t checkpoint_every,
                                   uint32_t precision) {
    std::string why;
    if (!host_valid_config(cfg, why)) {
        report_error(FLUID_ERR_ARG, "adjoint: " + why);
        return nullptr;
    }
    if (frames == 0 || substeps_per_frame == 0 || checkpoint_every == 0 || !(frame_dt > 0.0f) ||
        !(v_clamp > 0.0f) || (precision != 32 && precision != 64)) {
        report_error(FLUID_ERR_ARG, "adjoint: frames, substeps, checkpoint interval, dt and v_clamp must be "
                                    "positive; precision 32 or 64");
        return nullptr;
    }
    FluidAdjoint *a = new FluidAdjoint();
    a->precision = precision;
    int32_t rc;
    if (precision == 64) {
        auto *m = new AdjImpl<double>();
        a->impl = m;
        rc = m->create(*cfg, frames, substeps_per_frame, frame_dt, v_clamp, checkpoint_every);
    } else {
        auto *m = new AdjImpl<float>();
        a->impl = m;
        rc = m->create(*cfg, frames, substeps_per_frame, frame_dt, v_clamp, checkpoint_every);
    }
    if (rc != FLUID_OK) {
        delete a->impl;
        delete a;
        return nullptr;
    }
    return a;
}

void fluid_adjoint_destroy(FluidAdjoint *a) {
    if (!a) return;
    delete a->impl;
    delete a;
}

uint32_t fluid_adjoint_count(const FluidAdjoint *a) { return a ? a->impl->n : 0u; }

int32_t fluid_adjoint_forward(FluidAdjoint *a, const double *forces, double xsph, const double target[3],
                              double *loss) {
    if (!a || !forces || !target || !loss) return report_error(FLUID_ERR_ARG, "adjoint: null argument");
    return a->impl->forward(forces, xsph, target, loss);
}

int32_t fluid_adjoint_backward(FluidAdjoint *a, double *grad_forces, double *grad_xsph) {
    if (!a) return report_error(FLUID_ERR_ARG, "adjoint: null handle");
    return a->impl->backward(grad_forces, grad_xsph);
}

int32_t fluid_adjoint_get_schedule(const FluidAdjoint *a, uint32_t *div_iters, uint32_t *den_iters) {
    if (!a || !div_iters || !den_iters) return report_error(FLUID_ERR_ARG, "adjoint: null argument");
    if (!a->impl->frozen) return report_error(FLUID_ERR_STATE, "adjoint: no schedule yet (run a forward)");
    std::memcpy(div_iters, a->impl->div_it.data(), 4 * a->impl->div_it.size());
    std::memcpy(den_iters, a->impl->den_it.data(), 4 * a->impl->den_it.size());
    return FLUID_OK;
}

int32_t fluid_adjoint_set_schedule(FluidAdjoint *a, const uint32_t *div_iters, const uint32_t *den_iters) {
    if (!a || !div_iters || !den_iters) return report_error(FLUID_ERR_ARG, "adjoint: null argument");
    const size_t S = (size_t)a->impl->frames * a->impl->spf;
    for (size_t k = 0; k < S; ++k)
        if (div_iters[k] > kMaxIters || den_iters[k] > kMaxIters)
            return report_error(FLUID_ERR_ARG, "adjoint: iteration counts are capped at 126");
    a->impl->div_it.assign(div_iters, div_iters + S);
    a->impl->den_it.assign(den_iters, den_iters + S);
    a->impl->frozen = true;
    a->impl->have_forward = false;
    return FLUID_OK;
}

int32_t fluid_adjoint_final_state(FluidAdjoint *a, double *pos3, double *vel3) {
    if (!a) return report_error(FLUID_ERR_ARG, "adjoint: null handle");
    return a->impl->final_state(pos3, vel3);
}

int32_t fluid_adjoint_timing(const FluidAdjoint *a, float *forward_ms, float *backward_ms) {
    if (!a) return report_error(FLUID_ERR_ARG, "adjoint: null handle");
    if (forward_ms) *forward_ms = a->impl->last_forward_ms;
    if (backward_ms) *backward_ms = a->impl->last_backward_ms;
    return FLUID_OK;
}

}  // extern "C"
