// Device-side views of the C-ABI descriptors, B-spline stencil evaluation
// and small helpers shared by every transfer kernel.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "../../include/picasso_b200.h"

namespace pb {

// ---------------------------------------------------------------------------
// error plumbing (host)
// ---------------------------------------------------------------------------
void set_last_cuda_error(cudaError_t e);
picasso_status check_launch();  // reads cudaGetLastError after a launch

#define PB_CUDA_TRY(expr)                                   \
    do {                                                    \
        cudaError_t e_ = (expr);                            \
        if (e_ != cudaSuccess) {                            \
            ::pb::set_last_cuda_error(e_);                  \
            return PICASSO_ERR_CUDA;                        \
        }                                                   \
    } while (0)

inline cudaStream_t stream_of(const picasso_exec* ex)
{
    return ex ? static_cast<cudaStream_t>(ex->stream) : nullptr;
}

// Grid of at most max_blocks blocks of `threads` for n work items.
inline unsigned grid_for(int64_t n, int threads, int64_t max_blocks = 148LL * 64)
{
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > max_blocks) b = max_blocks;
    return static_cast<unsigned>(b);
}

// ---------------------------------------------------------------------------
// particle members
// ---------------------------------------------------------------------------
struct PField {
    char* data;
    int32_t shift;       // clamp(vector_shift, 0, 63)
    int64_t mask;        // AoSoA lane mask (all ones for plain arrays)
    int64_t tile_stride;
    int64_t comp_stride;

    __host__ __device__ __forceinline__ int64_t index(int64_t p, int c) const
    {
        return (p >> shift) * tile_stride + (p & mask) + (int64_t)c * comp_stride;
    }
    template <class T>
    __device__ __forceinline__ T get(int64_t p, int c) const
    {
        return reinterpret_cast<const T*>(data)[index(p, c)];
    }
    template <class T>
    __device__ __forceinline__ void set(int64_t p, int c, T v) const
    {
        reinterpret_cast<T*>(data)[index(p, c)] = v;
    }
};

inline PField make_pfield(const picasso_particle_field& f)
{
    PField r;
    r.data = static_cast<char*>(f.data);
    if (f.vector_shift >= 62) {
        r.shift = 63;
        r.mask = -1;
        r.tile_stride = 0;
    } else {
        r.shift = f.vector_shift;
        r.mask = (int64_t(1) << f.vector_shift) - 1;
        r.tile_stride = f.tile_stride;
    }
    r.comp_stride = f.comp_stride;
    return r;
}

// ---------------------------------------------------------------------------
// grid arrays
// ---------------------------------------------------------------------------
struct GField {
    char* data;
    int64_t s[4];
    int32_t fixed_bits;
    int32_t* overflow;  // optional counter of fixed-point values out of range

    __device__ __forceinline__ int64_t index(int i, int j, int k, int c) const
    {
        return (int64_t)i * s[0] + (int64_t)j * s[1] + (int64_t)k * s[2] + (int64_t)c * s[3];
    }
    template <class T>
    __device__ __forceinline__ T* ptr(int i, int j, int k, int c) const
    {
        return reinterpret_cast<T*>(data) + index(i, j, k, c);
    }
};

inline GField make_gfield(const picasso_grid_field& f)
{
    GField g;
    g.data = static_cast<char*>(f.data);
    for (int d = 0; d < 4; ++d) g.s[d] = f.stride[d];
    g.fixed_bits = f.fixed_bits;
    g.overflow = nullptr;
    return g;
}

// Fixed-point headroom: a value whose magnitude times 2^fixed_bits reaches
// 2^62 leaves no room for the sums it enters (a 64-bit sum wraps at 2^63).
constexpr float kFixedLimitF = 4.611686018427387904e18f;  // 2^62
constexpr double kFixedLimitD = 4.611686018427387904e18;

// Rounds a scaled value to fixed point; counts it in g.overflow (when given)
// if it is out of range (the conversion saturates, so the sum is wrong).
__device__ __forceinline__ long long to_fixed(const GField& g, float scaled)
{
    if (!(fabsf(scaled) < kFixedLimitF) && g.overflow) atomicAdd(g.overflow, 1);
    return __float2ll_rn(scaled);
}
__device__ __forceinline__ long long to_fixed(const GField& g, double scaled)
{
    if (!(fabs(scaled) < kFixedLimitD) && g.overflow) atomicAdd(g.overflow, 1);
    return __double2ll_rn(scaled);
}

// ---------------------------------------------------------------------------
// mesh + spline parameters
// ---------------------------------------------------------------------------
struct MeshP {
    int ext[3];
    int own_lo[3];
    int own_n[3];
    int periodic[3];
    double lo[3];   // coordinate of entity index 0 along each dimension
    double dx[3];   // coord(1) - coord(0)
    double rdx[3];  // 1 / dx
};

inline void entity_offset(int loc, double off[3])
{
    for (int d = 0; d < 3; ++d) off[d] = 0.0;
    if (loc == PICASSO_CELL) {
        off[0] = off[1] = off[2] = 0.5;
    } else if (loc >= PICASSO_FACE_I && loc <= PICASSO_FACE_K) {
        for (int d = 0; d < 3; ++d) off[d] = (d == loc - PICASSO_FACE_I) ? 0.0 : 0.5;
    } else if (loc >= PICASSO_EDGE_I && loc <= PICASSO_EDGE_K) {
        for (int d = 0; d < 3; ++d) off[d] = (d == loc - PICASSO_EDGE_I) ? 0.5 : 0.0;
    }
}

inline int staggered_dim(int loc)
{
    if (loc >= PICASSO_FACE_I && loc <= PICASSO_FACE_K) return loc - PICASSO_FACE_I;
    if (loc >= PICASSO_EDGE_I && loc <= PICASSO_EDGE_K) return loc - PICASSO_EDGE_I;
    return -1;
}

// Validates the mesh / location / order and fills the device parameters.
picasso_status make_mesh(const picasso_spline* sd, MeshP* mp);
picasso_status validate_mesh(const picasso_mesh* m);
// A member of n particles; null data is accepted when n == 0.
picasso_status validate_pfield(int64_t n, const picasso_particle_field& f, int dtype_a,
                               int dtype_b = -1);
picasso_status validate_gfield(const picasso_grid_field& f, int dtype_a, int dtype_b = -1);

// Knots per dimension and offset of the first knot from floor(x0).
template <int ORDER>
struct SplineTraits;
template <>
struct SplineTraits<1> {
    static constexpr int K = 2;
    static constexpr int first = 0;
    static constexpr double shift = 0.0;
};
template <>
struct SplineTraits<2> {
    static constexpr int K = 3;
    static constexpr int first = -1;
    static constexpr double shift = 0.5;
};
template <>
struct SplineTraits<3> {
    static constexpr int K = 4;
    static constexpr int first = -1;
    static constexpr double shift = 0.0;
};

// One dimension of the spline: first stencil index, weights, physical
// distances (entity - particle) and, for order 1, weight gradients.
template <int ORDER, class R>
struct Spline1D {
    int s0;  // first stencil index (unwrapped)
    R w[SplineTraits<ORDER>::K];
    R d[SplineTraits<ORDER>::K];
    R g[SplineTraits<ORDER>::K];
};

// Logical position of a particle in the entity index space, rounded step by
// step (no fused multiply-add) so that the stencil start -- and with it the
// particle's sort bin -- is bit-identical in every kernel and in the oracle.
__device__ __forceinline__ double logical_coord(double x, double lo, double rdx, double shift)
{
    return __dadd_rn(__dmul_rn(__dsub_rn(x, lo), rdx), shift);
}

// FP64 evaluation that follows the oracle's expression order (used by the
// plain FP64 kernels so that they agree with the oracle to rounding of the
// accumulation order only).
template <int ORDER>
__device__ __forceinline__ void spline_eval_f64(double x, double lo, double dx, double rdx,
                                                Spline1D<ORDER, double>& sp)
{
    double x0 = logical_coord(x, lo, rdx, SplineTraits<ORDER>::shift);
    double fl = floor(x0);
    int s0 = (int)fl;
    double t = x0 - fl;
    sp.s0 = s0 + SplineTraits<ORDER>::first;
    if (ORDER == 1) {
        sp.w[0] = 1.0 - t;
        sp.w[1] = t;
        sp.g[0] = -rdx;
        sp.g[1] = rdx;
    } else if (ORDER == 2) {
        double xn = t - 0.5;
        sp.w[0] = 0.5 * xn * xn - 0.5 * xn + 0.125;
        sp.w[1] = 0.75 - xn * xn;
        sp.w[2] = 0.5 * xn * xn + 0.5 * xn + 0.125;
        sp.g[0] = (xn - 0.5) * rdx;
        sp.g[1] = -2.0 * xn * rdx;
        sp.g[2] = (xn + 0.5) * rdx;
    } else {
        double u = 1.0 - t;
        sp.w[0] = u * u * u / 6.0;
        sp.w[1] = 2.0 / 3.0 - t * t + 0.5 * t * t * t;
        sp.w[2] = 2.0 / 3.0 - u * u + 0.5 * u * u * u;
        sp.w[3] = t * t * t / 6.0;
        sp.g[0] = -0.5 * u * u * rdx;
        sp.g[1] = (-2.0 * t + 1.5 * t * t) * rdx;
        sp.g[2] = (2.0 * u - 1.5 * u * u) * rdx;
        sp.g[3] = 0.5 * t * t * rdx;
    }
#pragma unroll
    for (int n = 0; n < SplineTraits<ORDER>::K; ++n)
        sp.d[n] = lo + (double)(sp.s0 + n) * dx - x;
}

// Weights, gradients and distances of one dimension from the in-cell
// fraction t of the logical position (t = x0 - floor(x0)), in R; h = dx.
template <int ORDER, class R>
__device__ __forceinline__ void spline_from_frac(R t, R h, double rdx, Spline1D<ORDER, R>& sp)
{
    if (ORDER == 1) {
        sp.w[0] = R(1) - t;
        sp.w[1] = t;
        sp.g[0] = (R)(-rdx);
        sp.g[1] = (R)rdx;
    } else if (ORDER == 2) {
        R xn = t - R(0.5);
        sp.w[0] = R(0.5) * (R(0.5) - xn) * (R(0.5) - xn);
        sp.w[1] = R(0.75) - xn * xn;
        sp.w[2] = R(0.5) * (R(0.5) + xn) * (R(0.5) + xn);
        sp.g[0] = (xn - R(0.5)) * (R)rdx;
        sp.g[1] = R(-2) * xn * (R)rdx;
        sp.g[2] = (xn + R(0.5)) * (R)rdx;
    } else {
        R u = R(1) - t;
        sp.w[0] = u * u * u * R(1.0 / 6.0);
        sp.w[1] = R(2.0 / 3.0) - t * t * (R(1) - R(0.5) * t);
        sp.w[2] = R(2.0 / 3.0) - u * u * (R(1) - R(0.5) * u);
        sp.w[3] = t * t * t * R(1.0 / 6.0);
        sp.g[0] = R(-0.5) * u * u * (R)rdx;
        sp.g[1] = (R(-2) * t + R(1.5) * t * t) * (R)rdx;
        sp.g[2] = (R(2) * u - R(1.5) * u * u) * (R)rdx;
        sp.g[3] = R(0.5) * t * t * (R)rdx;
    }
    // entity n sits at logical offset (first + n) from floor(x0); the
    // particle at t - shift
#pragma unroll
    for (int n = 0; n < SplineTraits<ORDER>::K; ++n)
        sp.d[n] = (R(SplineTraits<ORDER>::first + n + SplineTraits<ORDER>::shift) - t) * h;
}

// In-cell fraction of the logical position of x and the stencil start, the
// logical position and its integer part formed in FP64 (step by step, as in
// every kernel, so the stencil start is bit-identical everywhere).
template <int ORDER>
__device__ __forceinline__ float logical_frac(double x, double lo, double rdx, int& s0)
{
    const double x0 = logical_coord(x, lo, rdx, SplineTraits<ORDER>::shift);
    const double fl = floor(x0);
    s0 = (int)fl + SplineTraits<ORDER>::first;
    return (float)(x0 - fl);
}

// Reduced-precision evaluation: the logical position and its integer part
// are formed in FP64 from the FP64 position; the in-cell fraction, weights
// and distances are then formed in R from the fraction, so no large
// coordinates are cancelled in R.
template <int ORDER, class R>
__device__ __forceinline__ void spline_eval_frac(double x, double lo, double dx, double rdx,
                                                 Spline1D<ORDER, R>& sp)
{
    double x0 = logical_coord(x, lo, rdx, SplineTraits<ORDER>::shift);
    double fl = floor(x0);
    int s0 = (int)fl;
    R t = (R)(x0 - fl);
    sp.s0 = s0 + SplineTraits<ORDER>::first;
    spline_from_frac<ORDER, R>(t, (R)dx, rdx, sp);
}

// Periodic wrap / bounds check of a stencil start: fills the K resolved
// indices; returns false if the stencil leaves a non-periodic mesh.
template <int K>
__device__ __forceinline__ bool resolve_stencil(const MeshP& mp, int d, int s0, int idx[K])
{
    if (mp.periodic[d]) {
        int n = mp.own_n[d];
        int r = (s0 - mp.own_lo[d]) % n;
        if (r < 0) r += n;
#pragma unroll
        for (int q = 0; q < K; ++q) {
            idx[q] = mp.own_lo[d] + r;
            r = (r + 1 == n) ? 0 : r + 1;
        }
        return true;
    }
    // written so that no sum can overflow for non-finite positions
    if (s0 < 0 || s0 > mp.ext[d] - K) return false;
#pragma unroll
    for (int q = 0; q < K; ++q) idx[q] = s0 + q;
    return true;
}

// ---------------------------------------------------------------------------
// accumulation into grid arrays
// ---------------------------------------------------------------------------
// FP64 grid: hardware FP64 atomic add.  I64 fixed-point grid: the value is
// rounded to the nearest multiple of 2^-bits and added as a 64-bit integer,
// which makes the sum independent of the order of contributions.
struct AccF64 {
    __device__ __forceinline__ static void add(const GField& g, int i, int j, int k, int c,
                                               double v, double /*scale*/)
    {
        atomicAdd(g.ptr<double>(i, j, k, c), v);
    }
};
struct AccFixed {
    __device__ __forceinline__ static void add(const GField& g, int i, int j, int k, int c,
                                               double v, double scale)
    {
        long long q = to_fixed(g, v * scale);
        atomicAdd(reinterpret_cast<unsigned long long*>(g.ptr<long long>(i, j, k, c)),
                  (unsigned long long)q);
    }
    __device__ __forceinline__ static void add(const GField& g, int i, int j, int k, int c,
                                               float v, float scale)
    {
        long long q = to_fixed(g, v * scale);
        atomicAdd(reinterpret_cast<unsigned long long*>(g.ptr<long long>(i, j, k, c)),
                  (unsigned long long)q);
    }
};

}  // namespace pb
