// Grid-side operations between P2G and G2P: fill (the GridOperator's zeroing
// of scatter fields), the FP64 momentum-to-velocity update with the
// near-empty-node threshold, and the FP64 particle position update.
#include <cmath>

#include "gridops.cuh"

namespace pb {

template <class T>
__global__ void fill_kernel(Box b, GField f, int ncomp, T v)
{
    const int64_t total = b.count() * ncomp;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        b.at(e / ncomp, i, j, k);
        *f.ptr<T>(i, j, k, (int)(e % ncomp)) = v;
    }
}

template <class MT, class UT, int NC>
__global__ void velocity_kernel(Box b, GField gm, GField gmu, GField gu, GField gu64,
                                double thr, double inv_m, double inv_mu)
{
    const int64_t total = b.count();
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        b.at(e, i, j, k);
        velocity_node<MT, UT, NC>(gm, gmu, gu, gu64, i, j, k, thr, inv_m, inv_mu);
    }
}

template <class MT, class UT>
static void launch_velocity(int ncomp, Box b, GField gm, GField gmu, GField gu, GField gu64,
                            double thr, double inv_m, double inv_mu, cudaStream_t st)
{
    const unsigned blocks = grid_for(b.count(), 256, 148LL * 32);
    if (ncomp == 1)
        velocity_kernel<MT, UT, 1><<<blocks, 256, 0, st>>>(b, gm, gmu, gu, gu64, thr, inv_m, inv_mu);
    else if (ncomp == 2)
        velocity_kernel<MT, UT, 2><<<blocks, 256, 0, st>>>(b, gm, gmu, gu, gu64, thr, inv_m, inv_mu);
    else
        velocity_kernel<MT, UT, 3><<<blocks, 256, 0, st>>>(b, gm, gmu, gu, gu64, thr, inv_m, inv_mu);
}

template <class MT, class FT, class UT>
__global__ void update_kernel(Box b, GridUpdate P, GField gm, GField gmu, GField gf, GField gu,
                              GField gu64)
{
    const int64_t total = b.count();
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        b.at(e, i, j, k);
        update_node<MT, FT, UT>(P, gm, gmu, gf, gu, gu64, i, j, k);
    }
}

template <class CT>
__global__ void advect_kernel(int64_t n, PField x, PField c, Advect a)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int d = 0; d < 3; ++d)
            x.set<double>(p, d, advect_coord(a, d, x.get<double>(p, d), (double)c.get<CT>(p, d)));
    }
}

}  // namespace pb

using namespace pb;

// Fill of a contiguous element range: 16-byte stores (the array start is
// element-aligned; a scalar head and tail handle the unaligned ends).
template <class T>
__global__ void fill_contiguous_kernel(T* data, int64_t n, T v)
{
    constexpr int V = 16 / sizeof(T);
    const uintptr_t addr = reinterpret_cast<uintptr_t>(data);
    const int64_t h0 = (int64_t)(((16 - addr % 16) % 16) / sizeof(T));
    const int64_t head = n < h0 ? n : h0;
    const int64_t nvec = (n - head) / V;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t0 < head) data[t0] = v;
    struct alignas(16) Vec {
        T e[V];
    };
    Vec w;
#pragma unroll
    for (int q = 0; q < V; ++q) w.e[q] = v;
    Vec* vd = reinterpret_cast<Vec*>(data + head);
    for (int64_t i = t0; i < nvec; i += stride) vd[i] = w;
    const int64_t tail = head + nvec * V;
    if (t0 < n - tail) data[tail + t0] = v;
}

// True when the box of ncomp components is one contiguous element range of f
// (Cabana LayoutRight over the whole local grid).
static bool contiguous(const Box& b, const GField& f, int ncomp)
{
    return (ncomp == 1 || f.s[3] == 1) && f.s[2] == ncomp && f.s[1] == (int64_t)b.n[2] * ncomp &&
           f.s[0] == (int64_t)b.n[1] * b.n[2] * ncomp && b.lo[0] == 0 && b.lo[1] == 0 &&
           b.lo[2] == 0;
}

extern "C" picasso_status picasso_grid_fill(const picasso_mesh* mesh, int32_t ncomp,
                                            picasso_grid_field f, double value,
                                            const picasso_exec* exec)
{
    picasso_status st = validate_mesh(mesh);
    if (st) return st;
    if (ncomp < 1) return PICASSO_ERR_INVALID_ARGUMENT;
    if ((st = validate_gfield(f, PICASSO_F64, PICASSO_F32)) &&
        (st = validate_gfield(f, PICASSO_I64_FIXED)))
        return st;
    Box b = full_box(*mesh);
    GField g = make_gfield(f);
    cudaStream_t s = stream_of(exec);
    if (contiguous(b, g, ncomp)) {
        const int64_t n = b.count() * ncomp;
        const unsigned blocks = grid_for(n / 2, 256, 148LL * 16);
        if (f.dtype == PICASSO_F64) {
            if (value == 0.0) PB_CUDA_TRY(cudaMemsetAsync(f.data, 0, n * sizeof(double), s));
            else fill_contiguous_kernel<double><<<blocks, 256, 0, s>>>((double*)f.data, n, value);
        } else if (f.dtype == PICASSO_F32) {
            if (value == 0.0) PB_CUDA_TRY(cudaMemsetAsync(f.data, 0, n * sizeof(float), s));
            else
                fill_contiguous_kernel<float><<<blocks, 256, 0, s>>>((float*)f.data, n,
                                                                     (float)value);
        } else {
            const long long q = llrint(ldexp(value, f.fixed_bits));
            if (q == 0) PB_CUDA_TRY(cudaMemsetAsync(f.data, 0, n * sizeof(long long), s));
            else
                fill_contiguous_kernel<long long><<<blocks, 256, 0, s>>>((long long*)f.data,
                                                                         n, q);
        }
        return check_launch();
    }
    const unsigned blocks = grid_for(b.count() * ncomp, 256, 148LL * 32);
    if (f.dtype == PICASSO_F64)
        fill_kernel<double><<<blocks, 256, 0, s>>>(b, g, ncomp, value);
    else if (f.dtype == PICASSO_F32)
        fill_kernel<float><<<blocks, 256, 0, s>>>(b, g, ncomp, (float)value);
    else
        fill_kernel<long long><<<blocks, 256, 0, s>>>(b, g, ncomp,
                                                      llrint(ldexp(value, f.fixed_bits)));
    return check_launch();
}

extern "C" picasso_status picasso_grid_velocity(const picasso_mesh* mesh, int32_t ncomp,
                                                picasso_grid_field m_i, picasso_grid_field mu_i,
                                                double mass_threshold, picasso_grid_field u_i,
                                                picasso_grid_field u64_i,
                                                const picasso_exec* exec)
{
    picasso_status st = validate_mesh(mesh);
    if (st) return st;
    if (ncomp < 1 || ncomp > 3) return PICASSO_ERR_INVALID_ARGUMENT;
    if ((st = validate_gfield(m_i, PICASSO_F64, PICASSO_I64_FIXED))) return st;
    if ((st = validate_gfield(mu_i, m_i.dtype))) return st;
    if ((st = validate_gfield(u_i, PICASSO_F64, PICASSO_F32))) return st;
    if (u64_i.data && (st = validate_gfield(u64_i, PICASSO_F64))) return st;
    Box b = owned_box(*mesh);
    GField gm = make_gfield(m_i), gmu = make_gfield(mu_i), gu = make_gfield(u_i);
    GField gu64 = make_gfield(u64_i);
    gm.overflow = exec ? exec->overflow_count : nullptr;
    cudaStream_t s = stream_of(exec);
    const bool fixed = m_i.dtype == PICASSO_I64_FIXED;
    const double inv_m = fixed ? ldexp(1.0, -m_i.fixed_bits) : 1.0;
    const double inv_mu = fixed ? ldexp(1.0, -mu_i.fixed_bits) : 1.0;
    if (fixed) {
        if (u_i.dtype == PICASSO_F32)
            launch_velocity<long long, float>(ncomp, b, gm, gmu, gu, gu64, mass_threshold, inv_m,
                                              inv_mu, s);
        else
            launch_velocity<long long, double>(ncomp, b, gm, gmu, gu, gu64, mass_threshold,
                                               inv_m, inv_mu, s);
    } else {
        if (u_i.dtype == PICASSO_F32)
            launch_velocity<double, float>(ncomp, b, gm, gmu, gu, gu64, mass_threshold, inv_m,
                                           inv_mu, s);
        else
            launch_velocity<double, double>(ncomp, b, gm, gmu, gu, gu64, mass_threshold, inv_m,
                                            inv_mu, s);
    }
    return check_launch();
}

picasso_status pb::make_grid_update(const picasso_mesh* mesh, const picasso_grid_update_params* prm,
                                const picasso_grid_field& m_i, const picasso_grid_field& mu_i,
                                const picasso_grid_field& f_i, GridUpdate* P)
{
    if (!mesh || !prm || prm->wall_width < 0) return PICASSO_ERR_INVALID_ARGUMENT;
    for (int d = 0; d < 3; ++d)
        for (int s = 0; s < 2; ++s)
            if (prm->wall[d][s] < PICASSO_WALL_NONE || prm->wall[d][s] > PICASSO_WALL_FREE_SLIP)
                return PICASSO_ERR_INVALID_ARGUMENT;
    const bool force = f_i.data != nullptr;
    P->dt = prm->dt;
    P->thr = prm->mass_threshold;
    const bool fixed = m_i.dtype == PICASSO_I64_FIXED;
    P->inv_m = fixed ? ldexp(1.0, -m_i.fixed_bits) : 1.0;
    P->inv_mu = fixed ? ldexp(1.0, -mu_i.fixed_bits) : 1.0;
    P->inv_f = (force && f_i.dtype == PICASSO_I64_FIXED) ? ldexp(1.0, -f_i.fixed_bits) : 1.0;
    P->force = force;
    for (int d = 0; d < 3; ++d) {
        P->g[d] = prm->gravity[d];
        const bool walls = !mesh->periodic[d];
        P->wall[d][0] = walls ? prm->wall[d][0] : PICASSO_WALL_NONE;
        P->wall[d][1] = walls ? prm->wall[d][1] : PICASSO_WALL_NONE;
        P->lo_wall[d] = mesh->own_begin[d] + prm->wall_width;
        P->hi_wall[d] = mesh->own_begin[d] + mesh->own_extent[d] - prm->wall_width;
    }
    return PICASSO_OK;
}

extern "C" picasso_status picasso_grid_update(const picasso_mesh* mesh, picasso_grid_field m_i,
                                              picasso_grid_field mu_i, picasso_grid_field f_i,
                                              const picasso_grid_update_params* prm,
                                              picasso_grid_field u_i, picasso_grid_field u64_i,
                                              const picasso_exec* exec)
{
    picasso_status st = validate_mesh(mesh);
    if (st) return st;
    if (!prm || prm->wall_width < 0) return PICASSO_ERR_INVALID_ARGUMENT;
    for (int d = 0; d < 3; ++d)
        for (int s = 0; s < 2; ++s)
            if (prm->wall[d][s] < PICASSO_WALL_NONE || prm->wall[d][s] > PICASSO_WALL_FREE_SLIP)
                return PICASSO_ERR_INVALID_ARGUMENT;
    if ((st = validate_gfield(m_i, PICASSO_F64, PICASSO_I64_FIXED))) return st;
    if ((st = validate_gfield(mu_i, m_i.dtype))) return st;
    const bool force = f_i.data != nullptr;
    if (force && (st = validate_gfield(f_i, PICASSO_F64, mu_i.dtype))) return st;
    if ((st = validate_gfield(u_i, PICASSO_F64, PICASSO_F32))) return st;
    if (u64_i.data && (st = validate_gfield(u64_i, PICASSO_F64))) return st;
    GridUpdate P;
    if ((st = make_grid_update(mesh, prm, m_i, mu_i, f_i, &P))) return st;
    const bool fixed = m_i.dtype == PICASSO_I64_FIXED;
    Box b = owned_box(*mesh);
    GField gm = make_gfield(m_i), gmu = make_gfield(mu_i), gf = make_gfield(f_i);
    GField gu = make_gfield(u_i), gu64 = make_gfield(u64_i);
    gm.overflow = exec ? exec->overflow_count : nullptr;
    cudaStream_t s = stream_of(exec);
    const unsigned blocks = grid_for(b.count(), 256, 148LL * 32);
    const bool f64f = !force || f_i.dtype == PICASSO_F64;
    const bool u32 = u_i.dtype == PICASSO_F32;
#define PB_UPD(MT, FT, UT) \
    update_kernel<MT, FT, UT><<<blocks, 256, 0, s>>>(b, P, gm, gmu, gf, gu, gu64)
    if (fixed) {
        if (f64f) { if (u32) PB_UPD(long long, double, float); else PB_UPD(long long, double, double); }
        else { if (u32) PB_UPD(long long, long long, float); else PB_UPD(long long, long long, double); }
    } else {
        if (u32) PB_UPD(double, double, float);
        else PB_UPD(double, double, double);
    }
#undef PB_UPD
    return check_launch();
}

extern "C" picasso_status picasso_advect(const picasso_mesh* mesh, int64_t num_particles,
                                         double dt, picasso_particle_field x_p,
                                         picasso_particle_field c_p, const picasso_exec* exec)
{
    picasso_status st = validate_mesh(mesh);
    if (st) return st;
    if (num_particles < 0) return PICASSO_ERR_INVALID_ARGUMENT;
    if ((st = validate_pfield(num_particles, x_p, PICASSO_F64))) return st;
    if ((st = validate_pfield(num_particles, c_p, PICASSO_F64, PICASSO_F32))) return st;
    if (num_particles == 0) return PICASSO_OK;
    PField x = make_pfield(x_p), c = make_pfield(c_p);
    const Advect a = make_advect(*mesh, dt);
    cudaStream_t s = stream_of(exec);
    const unsigned blocks = grid_for(num_particles, 256);
    if (c_p.dtype == PICASSO_F64)
        advect_kernel<double><<<blocks, 256, 0, s>>>(num_particles, x, c, a);
    else
        advect_kernel<float><<<blocks, 256, 0, s>>>(num_particles, x, c, a);
    return check_launch();
}
