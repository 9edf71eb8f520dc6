// APIC particle-to-grid and grid-to-particle transfers, one thread per
// particle, accumulating straight into HBM with atomics.  This is the plain
// form of Picasso_APIC.hpp (and the path taken for unsorted particles); the
// per-particle bodies are in plain.cuh, the shared-memory tiled kernels for
// binned particles in tiled.cu.
#include "plain.cuh"

namespace pb {

// ---------------------------------------------------------------------------
// kernels: one thread per particle, grid-stride
// ---------------------------------------------------------------------------
template <int ORDER, int NC, bool STAG, class PT, class R, class ACC>
__global__ void __launch_bounds__(256)
apic_p2g_kernel(MeshP mp, int64_t n, PField x, PField m, PField c, GField gm, GField gmu,
                int stag, R scale_m, R scale_mu, int* err)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride)
        apic_p2g_particle<ORDER, NC, STAG, PT, R, ACC>(mp, p, x, m, c, gm, gmu, stag, scale_m,
                                                       scale_mu, err);
}

template <int ORDER, int NC, bool STAG, class GT, class PT, class R, bool ADV>
__global__ void __launch_bounds__(256)
apic_g2p_kernel(MeshP mp, int64_t n, PField x, GField u, PField c, int stag, int* err, Advect adv)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride)
        apic_g2p_particle<ORDER, NC, STAG, GT, PT, R, false, ADV>(mp, p, x, u, c, stag, err,
                                                                   &adv);
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

// adv != nullptr (collocated, 3 components only): G2P then the position update.
template <int ORDER, int NC, bool STAG>
static void launch_g2p(bool f32, const MeshP& mp, int64_t n, const PField& x, const GField& u,
                       const PField& c, int stag, int* err, const Advect* adv, cudaStream_t st)
{
    const int threads = 256;
    const unsigned blocks = grid_for(n, threads);
    const Advect a = adv ? *adv : Advect{};
    if constexpr (NC == 3 && !STAG) {
        if (adv) {
            if (f32)
                apic_g2p_kernel<ORDER, NC, STAG, float, float, float, true>
                    <<<blocks, threads, 0, st>>>(mp, n, x, u, c, stag, err, a);
            else
                apic_g2p_kernel<ORDER, NC, STAG, double, double, double, true>
                    <<<blocks, threads, 0, st>>>(mp, n, x, u, c, stag, err, a);
            return;
        }
    }
    if (f32)
        apic_g2p_kernel<ORDER, NC, STAG, float, float, float, false><<<blocks, threads, 0, st>>>(
            mp, n, x, u, c, stag, err, a);
    else
        apic_g2p_kernel<ORDER, NC, STAG, double, double, double, false>
            <<<blocks, threads, 0, st>>>(mp, n, x, u, c, stag, err, a);
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
                              int* err, const Advect* adv, cudaStream_t st)
{
    if (stag >= 0) {
        PB_ORDER_SWITCH(order, launch_g2p<O_, 3, true>(f32, mp, n, x, u, c, stag, err, nullptr, st));
    } else if (ncomp == 1) {
        PB_ORDER_SWITCH(order, launch_g2p<O_, 1, false>(f32, mp, n, x, u, c, -1, err, nullptr, st));
    } else if (ncomp == 2) {
        PB_ORDER_SWITCH(order, launch_g2p<O_, 2, false>(f32, mp, n, x, u, c, -1, err, nullptr, st));
    } else {
        PB_ORDER_SWITCH(order, launch_g2p<O_, 3, false>(f32, mp, n, x, u, c, -1, err, adv, st));
    }
    return check_launch();
}

// Tiled kernels for binned particles (tiled.cu).
struct FusedUpdate;
struct HaloPeers;
picasso_status apic_p2g_tiled(const MeshP& mp, int order, int ncomp, Form form, int64_t n,
                              const PField& x, const PField& m, const PField& c, const GField& gm,
                              const GField& gmu, const picasso_bins& bins, int* err,
                              cudaStream_t st, bool* handled, const FusedUpdate* fu = nullptr,
                              int stag = -1, const HaloPeers* hp = nullptr);
picasso_status apic_g2p_tiled(const MeshP& mp, int order, int ncomp, bool f32, int64_t n,
                              const PField& x, const GField& u, const PField& c,
                              const picasso_bins& bins, int* err, const Advect* adv,
                              cudaStream_t st, bool* handled, int stag = -1,
                              const HaloPeers* hp = nullptr);

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
    if ((st = validate_pfield(num_particles, x_p, PICASSO_F64))) return st;
    if ((st = validate_pfield(num_particles, m_p, PICASSO_F64, PICASSO_F32))) return st;
    if ((st = validate_pfield(num_particles, c_p, m_p.dtype))) return st;
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
    gm.overflow = gmu.overflow = exec ? exec->overflow_count : nullptr;
    if (exec && exec->bins) {
        // bins describe particles sorted for this spline
        if (exec->bins->order != sd->order || exec->bins->location != sd->location)
            return PICASSO_ERR_INVALID_ARGUMENT;
        bool handled = false;
        st = apic_p2g_tiled(mp, sd->order, ncomp, form, num_particles, x, m, c, gm, gmu,
                            *exec->bins, err, s, &handled, nullptr, stag);
        if (st || handled) return st;
    }
    return apic_p2g_plain(mp, sd->order, stag, ncomp, form, num_particles, x, m, c, gm, gmu,
                          err, s);
}

// G2P, and with dt != nullptr the position update x += dt u_p after it.
// dt != nullptr: G2P with advection; key_out != nullptr: it also writes the
// sort key of every moved particle for bins of the given tile shape.
static picasso_status apic_g2p_entry(const picasso_spline* sd, int64_t num_particles,
                                     int32_t ncomp, picasso_particle_field x_p,
                                     picasso_grid_field u_i, picasso_particle_field c_p,
                                     const double* dt, const picasso_exec* exec,
                                     const int32_t* key_tile = nullptr,
                                     uint32_t* key_out = nullptr)
{
    MeshP mp;
    picasso_status st = make_mesh(sd, &mp);
    if (st) return st;
    if (num_particles < 0) return PICASSO_ERR_INVALID_ARGUMENT;
    const int stag = staggered_dim(sd->location);
    if (stag >= 0 ? ncomp != 3 : (ncomp < 1 || ncomp > 3)) return PICASSO_ERR_INVALID_ARGUMENT;
    if (dt && (stag >= 0 || ncomp != 3)) return PICASSO_ERR_INVALID_ARGUMENT;
    if ((st = validate_pfield(num_particles, x_p, PICASSO_F64))) return st;
    if ((st = validate_gfield(u_i, PICASSO_F64, PICASSO_F32))) return st;
    if ((st = validate_pfield(num_particles, c_p, u_i.dtype))) return st;
    BinP bins;
    if (key_tile) {
        int64_t ntiles = 0;
        if ((st = make_binp(sd, key_tile, &bins, &ntiles))) return st;
        if (num_particles > 0 && !key_out) return PICASSO_ERR_INVALID_ARGUMENT;
    }
    if (num_particles == 0) return PICASSO_OK;
    const bool f32 = u_i.dtype == PICASSO_F32;
    cudaStream_t s = stream_of(exec);
    int* err = exec ? exec->error_count : nullptr;
    PField x = make_pfield(x_p), c = make_pfield(c_p);
    GField u = make_gfield(u_i);
    Advect adv;
    if (dt) adv = make_advect(sd->mesh, *dt);
    if (dt && key_tile) {
        adv.key_out = key_out;
        adv.bins = bins;
    }
    const Advect* ap = dt ? &adv : nullptr;
    if (exec && exec->bins) {
        if (exec->bins->order != sd->order || exec->bins->location != sd->location)
            return PICASSO_ERR_INVALID_ARGUMENT;
        bool handled = false;
        st = apic_g2p_tiled(mp, sd->order, ncomp, f32, num_particles, x, u, c, *exec->bins, err,
                            ap, s, &handled, stag);
        if (st || handled) return st;
    }
    return apic_g2p_plain(mp, sd->order, stag, ncomp, f32, num_particles, x, u, c, err, ap, s);
}

extern "C" picasso_status picasso_apic_g2p(const picasso_spline* sd, int64_t num_particles,
                                           int32_t ncomp, picasso_particle_field x_p,
                                           picasso_grid_field u_i, picasso_particle_field c_p,
                                           const picasso_exec* exec)
{
    return apic_g2p_entry(sd, num_particles, ncomp, x_p, u_i, c_p, nullptr, exec);
}

extern "C" picasso_status picasso_apic_g2p_advect(const picasso_spline* sd,
                                                  int64_t num_particles,
                                                  picasso_particle_field x_p,
                                                  picasso_grid_field u_i,
                                                  picasso_particle_field c_p, double dt,
                                                  const picasso_exec* exec)
{
    return apic_g2p_entry(sd, num_particles, 3, x_p, u_i, c_p, &dt, exec);
}

extern "C" picasso_status picasso_apic_g2p_advect_keys(const picasso_spline* sd,
                                                       int64_t num_particles,
                                                       picasso_particle_field x_p,
                                                       picasso_grid_field u_i,
                                                       picasso_particle_field c_p, double dt,
                                                       const int32_t tile[3], uint32_t* key_out,
                                                       const picasso_exec* exec)
{
    if (!tile) return PICASSO_ERR_INVALID_ARGUMENT;
    return apic_g2p_entry(sd, num_particles, 3, x_p, u_i, c_p, &dt, exec, tile, key_out);
}
