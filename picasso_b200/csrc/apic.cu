// APIC particle-to-grid and grid-to-particle transfers, one thread per
// particle, accumulating straight into HBM with atomics.  This is the plain
// form of Picasso_APIC.hpp (and the path taken for unsorted particles); the
// shared-memory tiled kernels for binned particles live in tiled.cu.
#include "common.cuh"
#include "transfer.cuh"

namespace pb {

// ---------------------------------------------------------------------------
// P2G
// ---------------------------------------------------------------------------
// NC: field components (collocated); STAG: staggered (Face/Edge) location,
// scattering c_p column `stag` of a 3-component matrix into component 0.
// PT: particle storage type of m_p / c_p; R: arithmetic type; ACC: grid
// accumulation policy (FP64 atomics or 64-bit fixed point).
template <int ORDER, int NC, bool STAG, class PT, class R, class ACC>
__global__ void __launch_bounds__(256)
apic_p2g_kernel(MeshP mp, int64_t n, PField x, PField m, PField c, GField gm, GField gmu,
                int stag, R scale_m, R scale_mu, int* err)
{
    constexpr int K = SplineTraits<ORDER>::K;
    constexpr int NCI = STAG ? 3 : NC;  // columns of c_p
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
        R cp[4][NCI];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int d = 0; d < NCI; ++d) cp[r][d] = (R)c.get<PT>(p, r * NCI + d);

        if (ORDER >= 2) {
            // APIC.hpp:94-139 (collocated) and :190-231 (staggered)
            const R D = inertial_scaling<ORDER, R>(mp.dx[0]);
            R DB[NCI][3];
#pragma unroll
            for (int d = 0; d < NCI; ++d)
#pragma unroll
                for (int a = 0; a < 3; ++a) DB[d][a] = D * cp[1 + a][d];
            // staggered: row `stag` of D*B and c_p(0, stag)
            R c0s = R(0), DBs[3] = {R(0), R(0), R(0)};
            if (STAG) {
                c0s = select<NCI>(cp[0], stag);
#pragma unroll
                for (int a = 0; a < 3; ++a) DBs[a] = D * select<NCI>(cp[1 + a], stag);
            }
#pragma unroll
            for (int i = 0; i < K; ++i)
#pragma unroll
                for (int j = 0; j < K; ++j)
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const R wm = sp[0].w[i] * sp[1].w[j] * sp[2].w[k] * mass;
                        const R dist[3] = {sp[0].d[i], sp[1].d[j], sp[2].d[k]};
                        if (!STAG) {
#pragma unroll
                            for (int d = 0; d < NC; ++d) {
                                R dbd = R(0);
#pragma unroll
                                for (int a = 0; a < 3; ++a) dbd += DB[d][a] * dist[a];
                                ACC::add(gmu, idx[0][i], idx[1][j], idx[2][k], d,
                                         wm * (cp[0][d] + dbd), scale_mu);
                            }
                        } else {
                            R bd = R(0);
#pragma unroll
                            for (int a = 0; a < 3; ++a) bd += DBs[a] * dist[a];
                            ACC::add(gmu, idx[0][i], idx[1][j], idx[2][k], 0,
                                     wm * (c0s + bd), scale_mu);
                        }
                        ACC::add(gm, idx[0][i], idx[1][j], idx[2][k], 0, wm, scale_m);
                    }
        } else {
            // order 1, gradient form: APIC.hpp:276-318 and :363-401
            R c0s = R(0), Bs[3] = {R(0), R(0), R(0)};
            if (STAG) {
                c0s = select<NCI>(cp[0], stag);
#pragma unroll
                for (int a = 0; a < 3; ++a) Bs[a] = select<NCI>(cp[1 + a], stag);
            }
#pragma unroll
            for (int i = 0; i < K; ++i)
#pragma unroll
                for (int j = 0; j < K; ++j)
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const R wm = sp[0].w[i] * sp[1].w[j] * sp[2].w[k] * mass;
                        R gm3[3];
                        gm3[0] = sp[0].g[i] * sp[1].w[j] * sp[2].w[k] * mass;
                        gm3[1] = sp[0].w[i] * sp[1].g[j] * sp[2].w[k] * mass;
                        gm3[2] = sp[0].w[i] * sp[1].w[j] * sp[2].g[k] * mass;
                        if (!STAG) {
#pragma unroll
                            for (int d = 0; d < NC; ++d) {
                                R bg = R(0);
#pragma unroll
                                for (int a = 0; a < 3; ++a) bg += cp[1 + a][d] * gm3[a];
                                ACC::add(gmu, idx[0][i], idx[1][j], idx[2][k], d,
                                         wm * cp[0][d] + bg, scale_mu);
                            }
                        } else {
                            R bg = R(0);
#pragma unroll
                            for (int a = 0; a < 3; ++a) bg += Bs[a] * gm3[a];
                            ACC::add(gmu, idx[0][i], idx[1][j], idx[2][k], 0,
                                     wm * c0s + bg, scale_mu);
                        }
                        ACC::add(gm, idx[0][i], idx[1][j], idx[2][k], 0, wm, scale_m);
                    }
        }
    }
}

// ---------------------------------------------------------------------------
// G2P
// ---------------------------------------------------------------------------
// GT: grid storage type of u_i; PT: particle storage type of c_p.
template <int ORDER, int NC, bool STAG, class GT, class PT, class R>
__global__ void __launch_bounds__(256)
apic_g2p_kernel(MeshP mp, int64_t n, PField x, GField u, PField c, int stag, int* err)
{
    constexpr int K = SplineTraits<ORDER>::K;
    constexpr int NCO = STAG ? 3 : NC;
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
        R up[NCO];
        R B[NCO][3];
#pragma unroll
        for (int d = 0; d < NCO; ++d) {
            up[d] = R(0);
#pragma unroll
            for (int a = 0; a < 3; ++a) B[d][a] = R(0);
        }
        // APIC.hpp:439-461 (collocated) and :512-533 (staggered)
#pragma unroll
        for (int i = 0; i < K; ++i)
#pragma unroll
            for (int j = 0; j < K; ++j)
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const R w = sp[0].w[i] * sp[1].w[j] * sp[2].w[k];
                    const R dist[3] = {sp[0].d[i], sp[1].d[j], sp[2].d[k]};
                    if (!STAG) {
                        R ue[NC];
#pragma unroll
                        for (int d = 0; d < NC; ++d)
                            ue[d] = (R)__ldg(u.ptr<GT>(idx[0][i], idx[1][j], idx[2][k], d));
#pragma unroll
                        for (int d = 0; d < NC; ++d) {
                            up[d] = up[d] + w * ue[d];
                            const R wu = w * ue[d];
#pragma unroll
                            for (int a = 0; a < 3; ++a) B[d][a] += wu * dist[a];
                        }
                    } else {
                        const R ue = (R)__ldg(u.ptr<GT>(idx[0][i], idx[1][j], idx[2][k], 0));
                        const R wu = w * ue;
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            if (d == stag) {
                                up[d] += wu;
#pragma unroll
                                for (int a = 0; a < 3; ++a) B[d][a] += wu * dist[a];
                            }
                        }
                    }
                }
        // c_p(0,d) = u_p(d); c_p(1+a,d) = B_p(d,a)  (APIC.hpp:464-471)
#pragma unroll
        for (int d = 0; d < NCO; ++d) {
            c.set<PT>(p, 0 * NCO + d, (PT)up[d]);
#pragma unroll
            for (int a = 0; a < 3; ++a) c.set<PT>(p, (1 + a) * NCO + d, (PT)B[d][a]);
        }
    }
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
template <int ORDER, int NC, bool STAG>
static void launch_p2g(Form form, const MeshP& mp, int64_t n, const PField& x, const PField& m,
                       const PField& c, const GField& gm, const GField& gmu, int stag, int* err,
                       cudaStream_t st)
{
    const int threads = 256;
    const unsigned blocks = grid_for(n, threads);
    if (form == Form::F64) {
        apic_p2g_kernel<ORDER, NC, STAG, double, double, AccF64><<<blocks, threads, 0, st>>>(
            mp, n, x, m, c, gm, gmu, stag, 0.0, 0.0, err);
    } else if (form == Form::F32Fixed) {
        apic_p2g_kernel<ORDER, NC, STAG, float, float, AccFixed><<<blocks, threads, 0, st>>>(
            mp, n, x, m, c, gm, gmu, stag, ldexpf(1.0f, gm.fixed_bits),
            ldexpf(1.0f, gmu.fixed_bits), err);
    } else {
        apic_p2g_kernel<ORDER, NC, STAG, double, double, AccFixed><<<blocks, threads, 0, st>>>(
            mp, n, x, m, c, gm, gmu, stag, ldexp(1.0, gm.fixed_bits),
            ldexp(1.0, gmu.fixed_bits), err);
    }
}

template <int ORDER, int NC, bool STAG>
static void launch_g2p(bool f32, const MeshP& mp, int64_t n, const PField& x, const GField& u,
                       const PField& c, int stag, int* err, cudaStream_t st)
{
    const int threads = 256;
    const unsigned blocks = grid_for(n, threads);
    if (f32)
        apic_g2p_kernel<ORDER, NC, STAG, float, float, float><<<blocks, threads, 0, st>>>(
            mp, n, x, u, c, stag, err);
    else
        apic_g2p_kernel<ORDER, NC, STAG, double, double, double><<<blocks, threads, 0, st>>>(
            mp, n, x, u, c, stag, err);
}

#define PB_ORDER_SWITCH(order, ...)               \
    switch (order) {                              \
        case 1: { constexpr int O_ = 1; __VA_ARGS__; } break; \
        case 2: { constexpr int O_ = 2; __VA_ARGS__; } break; \
        default: { constexpr int O_ = 3; __VA_ARGS__; } break; \
    }

picasso_status apic_p2g_plain(const MeshP& mp, int order, int stag, int ncomp, Form form,
                              int64_t n, const PField& x, const PField& m, const PField& c,
                              const GField& gm, const GField& gmu, int* err, cudaStream_t st)
{
    if (stag >= 0) {
        PB_ORDER_SWITCH(order, launch_p2g<O_, 3, true>(form, mp, n, x, m, c, gm, gmu, stag, err, st));
    } else if (ncomp == 1) {
        PB_ORDER_SWITCH(order, launch_p2g<O_, 1, false>(form, mp, n, x, m, c, gm, gmu, -1, err, st));
    } else if (ncomp == 2) {
        PB_ORDER_SWITCH(order, launch_p2g<O_, 2, false>(form, mp, n, x, m, c, gm, gmu, -1, err, st));
    } else {
        PB_ORDER_SWITCH(order, launch_p2g<O_, 3, false>(form, mp, n, x, m, c, gm, gmu, -1, err, st));
    }
    return check_launch();
}

picasso_status apic_g2p_plain(const MeshP& mp, int order, int stag, int ncomp, bool f32,
                              int64_t n, const PField& x, const GField& u, const PField& c,
                              int* err, cudaStream_t st)
{
    if (stag >= 0) {
        PB_ORDER_SWITCH(order, launch_g2p<O_, 3, true>(f32, mp, n, x, u, c, stag, err, st));
    } else if (ncomp == 1) {
        PB_ORDER_SWITCH(order, launch_g2p<O_, 1, false>(f32, mp, n, x, u, c, -1, err, st));
    } else if (ncomp == 2) {
        PB_ORDER_SWITCH(order, launch_g2p<O_, 2, false>(f32, mp, n, x, u, c, -1, err, st));
    } else {
        PB_ORDER_SWITCH(order, launch_g2p<O_, 3, false>(f32, mp, n, x, u, c, -1, err, st));
    }
    return check_launch();
}

// Tiled kernels for binned particles (tiled.cu).
picasso_status apic_p2g_tiled(const MeshP& mp, int order, int ncomp, Form form, int64_t n,
                              const PField& x, const PField& m, const PField& c, const GField& gm,
                              const GField& gmu, const picasso_bins& bins, int* err,
                              cudaStream_t st, bool* handled);
picasso_status apic_g2p_tiled(const MeshP& mp, int order, int ncomp, bool f32, int64_t n,
                              const PField& x, const GField& u, const PField& c,
                              const picasso_bins& bins, int* err, cudaStream_t st, bool* handled);

}  // namespace pb

using namespace pb;

extern "C" picasso_status picasso_apic_p2g(const picasso_spline* sd, int64_t num_particles,
                                           int32_t ncomp, picasso_particle_field x_p,
                                           picasso_particle_field m_p, picasso_particle_field c_p,
                                           picasso_grid_field m_i, picasso_grid_field mu_i,
                                           const picasso_exec* exec)
{
    MeshP mp;
    picasso_status st = make_mesh(sd, &mp);
    if (st) return st;
    if (num_particles < 0) return PICASSO_ERR_INVALID_ARGUMENT;
    const int stag = staggered_dim(sd->location);
    if (stag >= 0 ? ncomp != 3 : (ncomp < 1 || ncomp > 3)) return PICASSO_ERR_INVALID_ARGUMENT;
    if ((st = validate_pfield(x_p, PICASSO_F64))) return st;
    if ((st = validate_pfield(m_p, PICASSO_F64, PICASSO_F32))) return st;
    if ((st = validate_pfield(c_p, m_p.dtype))) return st;
    if ((st = validate_gfield(m_i, PICASSO_F64, PICASSO_I64_FIXED))) return st;
    if ((st = validate_gfield(mu_i, m_i.dtype))) return st;
    Form form;
    if (m_p.dtype == PICASSO_F64 && m_i.dtype == PICASSO_F64) form = Form::F64;
    else if (m_p.dtype == PICASSO_F32 && m_i.dtype == PICASSO_I64_FIXED) form = Form::F32Fixed;
    else if (m_p.dtype == PICASSO_F64 && m_i.dtype == PICASSO_I64_FIXED) form = Form::F64Fixed;
    else return PICASSO_ERR_UNSUPPORTED;
    if (num_particles == 0) return PICASSO_OK;
    cudaStream_t s = stream_of(exec);
    int* err = exec ? exec->error_count : nullptr;
    PField x = make_pfield(x_p), m = make_pfield(m_p), c = make_pfield(c_p);
    GField gm = make_gfield(m_i), gmu = make_gfield(mu_i);
    if (exec && exec->bins) {
        // bins describe particles sorted for this spline
        if (exec->bins->order != sd->order || exec->bins->location != sd->location)
            return PICASSO_ERR_INVALID_ARGUMENT;
        bool handled = false;
        if (stag < 0) {
            st = apic_p2g_tiled(mp, sd->order, ncomp, form, num_particles, x, m, c, gm, gmu,
                                *exec->bins, err, s, &handled);
            if (st || handled) return st;
        }
    }
    return apic_p2g_plain(mp, sd->order, stag, ncomp, form, num_particles, x, m, c, gm, gmu,
                          err, s);
}

extern "C" picasso_status picasso_apic_g2p(const picasso_spline* sd, int64_t num_particles,
                                           int32_t ncomp, picasso_particle_field x_p,
                                           picasso_grid_field u_i, picasso_particle_field c_p,
                                           const picasso_exec* exec)
{
    MeshP mp;
    picasso_status st = make_mesh(sd, &mp);
    if (st) return st;
    if (num_particles < 0) return PICASSO_ERR_INVALID_ARGUMENT;
    const int stag = staggered_dim(sd->location);
    if (stag >= 0 ? ncomp != 3 : (ncomp < 1 || ncomp > 3)) return PICASSO_ERR_INVALID_ARGUMENT;
    if ((st = validate_pfield(x_p, PICASSO_F64))) return st;
    if ((st = validate_gfield(u_i, PICASSO_F64, PICASSO_F32))) return st;
    if ((st = validate_pfield(c_p, u_i.dtype))) return st;
    if (num_particles == 0) return PICASSO_OK;
    const bool f32 = u_i.dtype == PICASSO_F32;
    cudaStream_t s = stream_of(exec);
    int* err = exec ? exec->error_count : nullptr;
    PField x = make_pfield(x_p), c = make_pfield(c_p);
    GField u = make_gfield(u_i);
    if (exec && exec->bins) {
        if (exec->bins->order != sd->order || exec->bins->location != sd->location)
            return PICASSO_ERR_INVALID_ARGUMENT;
        bool handled = false;
        if (stag < 0) {
            st = apic_g2p_tiled(mp, sd->order, ncomp, f32, num_particles, x, u, c, *exec->bins,
                                err, s, &handled);
            if (st || handled) return st;
        }
    }
    return apic_g2p_plain(mp, sd->order, stag, ncomp, f32, num_particles, x, u, c, err, s);
}
