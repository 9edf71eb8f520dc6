// PolyPIC particle-to-grid and grid-to-particle transfers, one thread per
// particle.  Linear (8 modes) follows Picasso_PolyPIC.hpp; quadratic (27
// modes) has no reference implementation and is the 3-D tensor-product
// extension of the reference's 2-D derivation (doc/polypic/
// polypic_2d_quadratic.nb): per dimension the weight-orthogonal modes
//   s0 = 1, s1 = r, s2 = r^2 - h^2/4 - alpha r,
//   alpha = p (h^2 - 4 p^2) / h^2, p = particle offset from the centre knot,
// and the G2P coefficients are the weighted least-squares projections
//   c_r = sum_i w_i s_r(r_i) u_i / sum_i w_i s_r(r_i)^2
// (for linear splines these reduce to w and dw/dx, PolyPIC.hpp:269-284).
#include "common.cuh"
#include "transfer.cuh"

namespace pb {

// Mode r <-> per-dimension degree.  Modes 0..7 are the reference's linear
// modes {1, x, y, z, xy, xz, yz, xyz} (PolyPIC.hpp:109-116); 8..26 the
// remaining degree <= 2 tensor products, lexicographic in (a, b, c).  The
// degrees of dimension d are packed two bits per mode so that the lookup
// folds to a constant inside unrolled loops.
__host__ __device__ __forceinline__ constexpr int mode_deg(int r, int d)
{
    return (int)(((d == 0 ? 0x2aaaa554004504ull : d == 1 ? 0x2a540a92a45110ull
                                                         : 0x2492492a4a5440ull) >>
                  (2 * r)) & 3ull);
}

// Inverse of mode_deg: the mode with degrees (a, b, c) (all below D).
__host__ __device__ __forceinline__ constexpr int mode_of(int a, int b, int c)
{
    int r = 0;
    while (!(mode_deg(r, 0) == a && mode_deg(r, 1) == b && mode_deg(r, 2) == c)) ++r;
    return r;
}

// a[i] for a register array and a run-time i (a select chain, no local memory).
template <int K, class T>
__device__ __forceinline__ T pick(const T (&a)[K], int i)
{
    T v = a[0];
#pragma unroll
    for (int q = 1; q < K; ++q) v = (i == q) ? a[q] : v;
    return v;
}

template <class R>
__device__ __forceinline__ R quad_alpha(R p, R h)
{
    return p * (h * h - R(4) * p * p) / (h * h);
}

template <class R>
__device__ __forceinline__ R mode1d(int deg, R r, R h, R alpha)
{
    return deg == 0 ? R(1) : (deg == 1 ? r : r * r - R(0.25) * h * h - alpha * r);
}

// 3x3 inverse by cofactors times 1/det (BatchedLinearAlgebra.hpp:4337-4350,
// 4626-4686); row-major.
template <class R>
__device__ __forceinline__ void inverse3(const R a[9], R inv[9])
{
    const R det = a[0] * a[4] * a[8] + a[1] * a[5] * a[6] + a[2] * a[3] * a[7] -
                  a[2] * a[4] * a[6] - a[1] * a[3] * a[8] - a[0] * a[5] * a[7];
    const R r = R(1) / det;
    inv[0] = (a[4] * a[8] - a[5] * a[7]) * r;
    inv[1] = (a[2] * a[7] - a[1] * a[8]) * r;
    inv[2] = (a[1] * a[5] - a[2] * a[4]) * r;
    inv[3] = (a[5] * a[6] - a[3] * a[8]) * r;
    inv[4] = (a[0] * a[8] - a[2] * a[6]) * r;
    inv[5] = (a[2] * a[3] - a[0] * a[5]) * r;
    inv[6] = (a[3] * a[7] - a[4] * a[6]) * r;
    inv[7] = (a[1] * a[6] - a[0] * a[7]) * r;
    inv[8] = (a[0] * a[4] - a[1] * a[3]) * r;
}

// ---------------------------------------------------------------------------
// P2G: PolyPIC.hpp:41-130 (collocated) and :140-229 (staggered)
// ---------------------------------------------------------------------------
template <int ORDER, int NC, bool STAG, class PT, class R, class ACC>
__global__ void __launch_bounds__(128)
polypic_p2g_kernel(MeshP mp, int64_t n, PField x, PField m, PField u, PField c, GField gmu,
                   GField gm, R dt, int col, R scale_mu, R scale_m, int* err)
{
    constexpr int K = SplineTraits<ORDER>::K;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        Spline1D<ORDER, R> sp[3];
        int idx[3][K];
        bool ok = true;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            eval_spline<ORDER>(x.get<double>(p, d), mp.lo[d], mp.dx[d], mp.rdx[d], sp[d]);
            ok = ok && resolve_stencil<K>(mp, d, sp[d].s0, idx[d]);
        }
        if (!ok) {
            if (err) atomicAdd(err, 1);
            continue;
        }
        const R mass = (R)m.get<PT>(p, 0);
        // affine material motion operator and its inverse (PolyPIC.hpp:81-87)
        R am[9], ai[9];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const R v = dt * (R)u.get<PT>(p, (1 + a) * 3 + b);
                am[3 * a + b] = (a == b) ? R(1) + v : v;
            }
        inverse3(am, ai);
        R alpha[3] = {R(0), R(0), R(0)};
        R h[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            h[d] = (R)mp.dx[d];
            if (ORDER == 2) alpha[d] = quad_alpha(-sp[d].d[1], h[d]);
        }
        // modes of the transferred field: all NC columns, or column `col`
        constexpr int NCU = STAG ? 1 : NC;
        constexpr int D = ORDER + 1;  // modes per dimension: degrees 0 .. ORDER
        const int ncp = STAG ? (col >= 0 ? NC : 1) : NC;
        // The components are transferred in passes of CB (27 FP64 modes: one
        // at a time, so that a pass holds 27 mode values rather than 81 in
        // registers).
        // The basis sum sum_r c_r b_r(xi) is contracted one dimension at a
        // time: sum_a f0_a sum_b f1_b sum_c f2_c c_(abc).
        constexpr int CB = (sizeof(R) == 8 && ORDER == 2) ? 1 : NCU;
#pragma unroll 1
        for (int d0 = 0; d0 < NCU; d0 += CB) {
            R cp[D][D][D][CB];
#pragma unroll
            for (int a = 0; a < D; ++a)
#pragma unroll
                for (int b = 0; b < D; ++b)
#pragma unroll
                    for (int cc = 0; cc < D; ++cc)
#pragma unroll
                        for (int e = 0; e < CB; ++e)
                            cp[a][b][cc][e] = (R)c.get<PT>(
                                p, mode_of(a, b, cc) * ncp + (STAG ? col : d0 + e));
            // 27 FP64 modes: i-planes one after the other (not unrolled: bounds
            // the live range of the 9-node plane bodies, which would spill)
#pragma unroll(sizeof(R) == 8 && ORDER == 2 ? 1 : K)
            for (int i = 0; i < K; ++i) {
                const R wxi = pick<K>(sp[0].w, i), dxi = pick<K>(sp[0].d, i);
                const int gi = pick<K>(idx[0], i);
#pragma unroll
                for (int j = 0; j < K; ++j)
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const R wm = mass * wxi * sp[1].w[j] * sp[2].w[k];
                        const R dist[3] = {dxi, sp[1].d[j], sp[2].d[k]};
                        // backtracked distance xi = A^-1 d (PolyPIC.hpp:90-106)
                        R map[3];
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            R t = R(0);
#pragma unroll
                            for (int v = 0; v < 3; ++v) t += ai[3 * q + v] * dist[v];
                            map[q] = t;
                        }
                        R f[3][D];
#pragma unroll
                        for (int q = 0; q < 3; ++q)
#pragma unroll
                            for (int g = 0; g < D; ++g)
                                f[q][g] = (ORDER == 1) ? (g == 0 ? R(1) : map[q])
                                                       : mode1d(g, map[q], h[q], alpha[q]);
#pragma unroll
                        for (int e = 0; e < CB; ++e) {
                            R sa = R(0);
#pragma unroll
                            for (int a = 0; a < D; ++a) {
                                R sb = R(0);
#pragma unroll
                                for (int b = 0; b < D; ++b) {
                                    R sc = R(0);
#pragma unroll
                                    for (int cc = 0; cc < D; ++cc) sc += f[2][cc] * cp[a][b][cc][e];
                                    sb += f[1][b] * sc;
                                }
                                sa += f[0][a] * sb;
                            }
                            ACC::add(gmu, gi, idx[1][j], idx[2][k], d0 + e, wm * sa, scale_mu);
                        }
                        if (d0 == 0) ACC::add(gm, gi, idx[1][j], idx[2][k], 0, wm, scale_m);
                    }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// G2P: PolyPIC.hpp:236-293 (collocated) and :300-358 (staggered)
// ---------------------------------------------------------------------------
template <int ORDER, int NC, bool STAG, class GT, class PT, class R>
__global__ void __launch_bounds__(128)
polypic_g2p_kernel(MeshP mp, int64_t n, PField x, GField u, PField c, int col, int* err)
{
    constexpr int K = SplineTraits<ORDER>::K;
    constexpr int NCU = STAG ? 1 : NC;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        Spline1D<ORDER, R> sp[3];
        int idx[3][K];
        bool ok = true;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            eval_spline<ORDER>(x.get<double>(p, d), mp.lo[d], mp.dx[d], mp.rdx[d], sp[d]);
            ok = ok && resolve_stencil<K>(mp, d, sp[d].s0, idx[d]);
        }
        if (!ok) {
            if (err) atomicAdd(err, 1);
            continue;
        }
        // per-dimension factors G[d][degree][knot]
        R G[3][3][K];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
#pragma unroll
            for (int q = 0; q < K; ++q) {
                G[d][0][q] = sp[d].w[q];
                G[d][1][q] = sp[d].g[q];
                G[d][2][q] = R(0);
            }
            if (ORDER == 2) {
                // closed forms of w s_g(r) / sum_n w s_g(r)^2: G1 = 4 w r / h^2,
                // G2 = {1/(2h^2), -1/h^2, 1/(2h^2)} (the degree-2 quotient is
                // a 0/0 limit at cell faces)
                const R h = (R)mp.dx[d];
                const R rh2 = R(1) / (h * h);
#pragma unroll
                for (int q = 0; q < K; ++q) G[d][1][q] = R(4) * sp[d].w[q] * sp[d].d[q] * rh2;
                G[d][2][0] = R(0.5) * rh2;
                G[d][2][1] = -rh2;
                G[d][2][2] = R(0.5) * rh2;
            }
        }
        // c_(abc) = sum_i G0[a][i] sum_j G1[b][j] sum_k G2[c][k] u_ijk, one
        // i-plane at a time, the components in passes of CB (27 FP64 modes:
        // one component per pass)
        constexpr int D = ORDER + 1;
        constexpr int CB = (sizeof(R) == 8 && ORDER == 2) ? 1 : NCU;
        const int ncp = STAG ? (col >= 0 ? NC : 1) : NC;
#pragma unroll
        for (int d0 = 0; d0 < NCU; d0 += CB) {
            R cp[D][D][D][CB];
#pragma unroll
            for (int a = 0; a < D; ++a)
#pragma unroll
                for (int b = 0; b < D; ++b)
#pragma unroll
                    for (int cc = 0; cc < D; ++cc)
#pragma unroll
                        for (int e = 0; e < CB; ++e) cp[a][b][cc][e] = R(0);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                R t2[D][D][CB];  // [b][c] of this i-plane
#pragma unroll
                for (int b = 0; b < D; ++b)
#pragma unroll
                    for (int cc = 0; cc < D; ++cc)
#pragma unroll
                        for (int e = 0; e < CB; ++e) t2[b][cc][e] = R(0);
#pragma unroll
                for (int j = 0; j < K; ++j) {
                    R ue[K][CB];
#pragma unroll
                    for (int k = 0; k < K; ++k)
#pragma unroll
                        for (int e = 0; e < CB; ++e)
                            ue[k][e] = (R)__ldg(u.ptr<GT>(idx[0][i], idx[1][j], idx[2][k], d0 + e));
#pragma unroll
                    for (int cc = 0; cc < D; ++cc)
#pragma unroll
                        for (int e = 0; e < CB; ++e) {
                            R t1 = R(0);
#pragma unroll
                            for (int k = 0; k < K; ++k) t1 += G[2][cc][k] * ue[k][e];
#pragma unroll
                            for (int b = 0; b < D; ++b) t2[b][cc][e] += G[1][b][j] * t1;
                        }
                }
#pragma unroll
                for (int a = 0; a < D; ++a)
#pragma unroll
                    for (int b = 0; b < D; ++b)
#pragma unroll
                        for (int cc = 0; cc < D; ++cc)
#pragma unroll
                            for (int e = 0; e < CB; ++e)
                                cp[a][b][cc][e] += G[0][a][i] * t2[b][cc][e];
            }
#pragma unroll
            for (int a = 0; a < D; ++a)
#pragma unroll
                for (int b = 0; b < D; ++b)
#pragma unroll
                    for (int cc = 0; cc < D; ++cc)
#pragma unroll
                        for (int e = 0; e < CB; ++e)
                            c.set<PT>(p, mode_of(a, b, cc) * ncp + (STAG ? col : d0 + e),
                                      (PT)cp[a][b][cc][e]);
        }
    }
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
template <int ORDER, int NC, bool STAG>
static void launch_pp_p2g(int form, const MeshP& mp, int64_t n, const PField& x, const PField& m,
                          const PField& u, const PField& c, const GField& gmu, const GField& gm,
                          double dt, int col, int* err, cudaStream_t st)
{
    const int threads = 128;
    const unsigned blocks = grid_for(n, threads, 148LL * 128);
    if (form == 0)
        polypic_p2g_kernel<ORDER, NC, STAG, double, double, AccF64><<<blocks, threads, 0, st>>>(
            mp, n, x, m, u, c, gmu, gm, dt, col, 0.0, 0.0, err);
    else if (form == 1)
        polypic_p2g_kernel<ORDER, NC, STAG, float, float, AccFixed><<<blocks, threads, 0, st>>>(
            mp, n, x, m, u, c, gmu, gm, (float)dt, col, ldexpf(1.0f, gmu.fixed_bits),
            ldexpf(1.0f, gm.fixed_bits), err);
    else
        polypic_p2g_kernel<ORDER, NC, STAG, double, double, AccFixed><<<blocks, threads, 0, st>>>(
            mp, n, x, m, u, c, gmu, gm, dt, col, ldexp(1.0, gmu.fixed_bits),
            ldexp(1.0, gm.fixed_bits), err);
}

template <int ORDER, int NC, bool STAG>
static void launch_pp_g2p(bool f32, const MeshP& mp, int64_t n, const PField& x, const GField& u,
                          const PField& c, int col, int* err, cudaStream_t st)
{
    const int threads = 128;
    const unsigned blocks = grid_for(n, threads, 148LL * 128);
    if (f32)
        polypic_g2p_kernel<ORDER, NC, STAG, float, float, float><<<blocks, threads, 0, st>>>(
            mp, n, x, u, c, col, err);
    else
        polypic_g2p_kernel<ORDER, NC, STAG, double, double, double><<<blocks, threads, 0, st>>>(
            mp, n, x, u, c, col, err);
}

#define PB_PP_NC_SWITCH(ncomp, ...)                                   \
    switch (ncomp) {                                                  \
        case 1: { constexpr int NC_ = 1; __VA_ARGS__; } break;        \
        case 2: { constexpr int NC_ = 2; __VA_ARGS__; } break;        \
        default: { constexpr int NC_ = 3; __VA_ARGS__; } break;       \
    }

}  // namespace pb

using namespace pb;

static picasso_status polypic_common(const picasso_spline* sd, int64_t n, int32_t ncomp,
                                     MeshP* mp, int* stag, int* col)
{
    picasso_status st = make_mesh(sd, mp);
    if (st) return st;
    if (n < 0 || ncomp < 1 || ncomp > 3) return PICASSO_ERR_INVALID_ARGUMENT;
    if (sd->order == 3) return PICASSO_ERR_UNSUPPORTED;
    *stag = staggered_dim(sd->location);
    if (*stag >= 0 && sd->order != 1) return PICASSO_ERR_UNSUPPORTED;
    // staggered: a 3-component field works on column `dim`, a scalar field
    // on column 0 (PolyPIC.hpp:181, :325)
    *col = (*stag >= 0) ? (ncomp == 3 ? *stag : 0) : -1;
    return PICASSO_OK;
}

extern "C" picasso_status picasso_polypic_p2g(const picasso_spline* sd, int64_t num_particles,
                                              int32_t ncomp, picasso_particle_field x_p,
                                              picasso_particle_field m_p,
                                              picasso_particle_field u_p,
                                              picasso_particle_field c_p,
                                              picasso_grid_field mu_i, picasso_grid_field m_i,
                                              double dt, const picasso_exec* exec)
{
    MeshP mp;
    int stag, col;
    picasso_status st = polypic_common(sd, num_particles, ncomp, &mp, &stag, &col);
    if (st) return st;
    if ((st = validate_pfield(num_particles, x_p, PICASSO_F64))) return st;
    if ((st = validate_pfield(num_particles, m_p, PICASSO_F64, PICASSO_F32))) return st;
    if ((st = validate_pfield(num_particles, u_p, m_p.dtype))) return st;
    if ((st = validate_pfield(num_particles, c_p, m_p.dtype))) return st;
    if ((st = validate_gfield(m_i, PICASSO_F64, PICASSO_I64_FIXED))) return st;
    if ((st = validate_gfield(mu_i, m_i.dtype))) return st;
    int form;
    if (m_p.dtype == PICASSO_F64 && m_i.dtype == PICASSO_F64) form = 0;
    else if (m_p.dtype == PICASSO_F32 && m_i.dtype == PICASSO_I64_FIXED) form = 1;
    else if (m_p.dtype == PICASSO_F64 && m_i.dtype == PICASSO_I64_FIXED) form = 2;
    else return PICASSO_ERR_UNSUPPORTED;
    if (num_particles == 0) return PICASSO_OK;
    cudaStream_t s = stream_of(exec);
    int* err = exec ? exec->error_count : nullptr;
    PField x = make_pfield(x_p), m = make_pfield(m_p), u = make_pfield(u_p), c = make_pfield(c_p);
    GField gmu = make_gfield(mu_i), gm = make_gfield(m_i);
    if (sd->order == 1) {
        if (stag >= 0) {
            PB_PP_NC_SWITCH(ncomp, launch_pp_p2g<1, NC_, true>(form, mp, num_particles, x, m, u, c,
                                                                gmu, gm, dt, col, err, s));
        } else {
            PB_PP_NC_SWITCH(ncomp, launch_pp_p2g<1, NC_, false>(form, mp, num_particles, x, m, u, c,
                                                                 gmu, gm, dt, col, err, s));
        }
    } else {
        PB_PP_NC_SWITCH(ncomp, launch_pp_p2g<2, NC_, false>(form, mp, num_particles, x, m, u, c,
                                                             gmu, gm, dt, col, err, s));
    }
    return check_launch();
}

extern "C" picasso_status picasso_polypic_g2p(const picasso_spline* sd, int64_t num_particles,
                                              int32_t ncomp, picasso_particle_field x_p,
                                              picasso_grid_field u_i, picasso_particle_field c_p,
                                              const picasso_exec* exec)
{
    MeshP mp;
    int stag, col;
    picasso_status st = polypic_common(sd, num_particles, ncomp, &mp, &stag, &col);
    if (st) return st;
    if ((st = validate_pfield(num_particles, x_p, PICASSO_F64))) return st;
    if ((st = validate_gfield(u_i, PICASSO_F64, PICASSO_F32))) return st;
    if ((st = validate_pfield(num_particles, c_p, u_i.dtype))) return st;
    if (num_particles == 0) return PICASSO_OK;
    const bool f32 = u_i.dtype == PICASSO_F32;
    cudaStream_t s = stream_of(exec);
    int* err = exec ? exec->error_count : nullptr;
    PField x = make_pfield(x_p), c = make_pfield(c_p);
    GField u = make_gfield(u_i);
    if (sd->order == 1) {
        if (stag >= 0) {
            PB_PP_NC_SWITCH(ncomp, launch_pp_g2p<1, NC_, true>(f32, mp, num_particles, x, u, c, col,
                                                                err, s));
        } else {
            PB_PP_NC_SWITCH(ncomp, launch_pp_g2p<1, NC_, false>(f32, mp, num_particles, x, u, c, col,
                                                                 err, s));
        }
    } else {
        PB_PP_NC_SWITCH(ncomp, launch_pp_g2p<2, NC_, false>(f32, mp, num_particles, x, u, c, col,
                                                             err, s));
    }
    return check_launch();
}
