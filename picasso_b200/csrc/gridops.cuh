// Per-node bodies of the grid operations between P2G and G2P: the node box
// iterated by the grid kernels (grid.cu, batch.cu) and the FP64
// momentum-to-velocity update with the near-empty-node threshold.
#pragma once

#include "binkey.cuh"
#include "common.cuh"

namespace pb {

struct Box {
    int lo[3];
    int n[3];
    __host__ __device__ int64_t count() const { return (int64_t)n[0] * n[1] * n[2]; }
    __device__ __forceinline__ void at(int64_t e, int& i, int& j, int& k) const
    {
        k = lo[2] + (int)(e % n[2]);
        e /= n[2];
        j = lo[1] + (int)(e % n[1]);
        i = lo[0] + (int)(e / n[1]);
    }
};

// All entities of the local grid (the fill range).
inline Box full_box(const picasso_mesh& m)
{
    Box b;
    for (int d = 0; d < 3; ++d) {
        b.lo[d] = 0;
        b.n[d] = m.extent[d];
    }
    return b;
}

// Nodes a periodic mesh owns (non-periodic: all entities); the velocity range.
inline Box owned_box(const picasso_mesh& m)
{
    Box b;
    for (int d = 0; d < 3; ++d) {
        b.lo[d] = m.periodic[d] ? m.own_begin[d] : 0;
        b.n[d] = m.periodic[d] ? m.own_extent[d] : m.extent[d];
    }
    return b;
}

// A fixed-point node mass is a sum of non-negative contributions: a negative
// sum has wrapped past 2^63 (too many fraction bits for the mass at that
// node).  Counted in gm.overflow when the caller asked for it.
template <class MT>
__device__ __forceinline__ void count_wrapped_mass(const GField& gm, MT raw)
{
    if constexpr (std::is_same<MT, long long>::value)
        if (raw < 0 && gm.overflow) atomicAdd(gm.overflow, 1);
}

// u = mu / m where m > threshold else 0; all arithmetic in FP64.  CG loads
// the accumulators through L2 only (grids written earlier in the same launch).
template <class MT, class UT, int NC, bool CG = false>
__device__ __forceinline__ void velocity_node(const GField& gm, const GField& gmu,
                                              const GField& gu, const GField& gu64, int i, int j,
                                              int k, double thr, double inv_m, double inv_mu)
{
    auto load = [](const MT* a) { return CG ? __ldcg(a) : *a; };
    const MT raw = load(gm.ptr<MT>(i, j, k, 0));
    count_wrapped_mass(gm, raw);
    const double m = (double)raw * inv_m;
    const bool keep = m > thr;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const double v = keep ? (double)load(gmu.ptr<MT>(i, j, k, c)) * inv_mu / m : 0.0;
        *gu.ptr<UT>(i, j, k, c) = (UT)v;
        if (gu64.data) *gu64.ptr<double>(i, j, k, c) = v;
    }
}

// Grid update of one node: u = (mu + dt f) / m + dt g where m > thr (else 0),
// then the wall conditions; FP64 rounded step by step.
struct GridUpdate {
    double dt, g[3], thr, inv_m, inv_mu, inv_f;
    int wall[3][2];
    int lo_wall[3];  // nodes with index < lo_wall[d] are on the low wall
    int hi_wall[3];  // nodes with index >= hi_wall[d] are on the high wall
    bool force;
};

// CG: the accumulators are read through L2 only (written by other blocks of
// the same launch).
template <class MT, class FT, class UT, bool CG = false>
__device__ __forceinline__ void update_node(const GridUpdate& P, const GField& gm,
                                            const GField& gmu, const GField& gf, const GField& gu,
                                            const GField& gu64, int i, int j, int k)
{
    auto load = [](const MT* a) { return CG ? __ldcg(a) : *a; };
    const MT raw = load(gm.ptr<MT>(i, j, k, 0));
    count_wrapped_mass(gm, raw);
    const double m = __dmul_rn((double)raw, P.inv_m);
    const bool keep = m > P.thr;
    double u[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double p = __dmul_rn((double)load(gmu.ptr<MT>(i, j, k, c)), P.inv_mu);
        if (P.force) p = __dadd_rn(p, __dmul_rn(P.dt, __dmul_rn((double)*gf.ptr<FT>(i, j, k, c), P.inv_f)));
        u[c] = keep ? __dadd_rn(__ddiv_rn(p, m), __dmul_rn(P.dt, P.g[c])) : 0.0;
    }
    const int idx[3] = {i, j, k};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int side = idx[d] < P.lo_wall[d] ? 0 : (idx[d] >= P.hi_wall[d] ? 1 : -1);
        if (side < 0) continue;
        const int w = P.wall[d][side];
        if (w == PICASSO_WALL_NO_SLIP) u[0] = u[1] = u[2] = 0.0;
        else if (w == PICASSO_WALL_FREE_SLIP) u[d] = 0.0;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        *gu.ptr<UT>(i, j, k, c) = (UT)u[c];
        if (gu64.data) *gu64.ptr<double>(i, j, k, c) = u[c];
    }
}

// Parameters of the grid update for a mesh, update settings and the grids'
// types; PICASSO_ERR_INVALID_ARGUMENT for bad settings (grid.cu).
picasso_status make_grid_update(const picasso_mesh* mesh, const picasso_grid_update_params* prm,
                                const picasso_grid_field& m_i, const picasso_grid_field& mu_i,
                                const picasso_grid_field& f_i, GridUpdate* P);

// Position update x += dt v with periodic wrap into the owned box, FP64,
// rounded step by step as x + (dt * v) (no FMA, so every path that advects
// gives the same bits).
struct Advect {
    double dt;
    int periodic[3];
    double lo[3];   // coordinate of the owned box's low face
    double len[3];  // owned box length
    // optional: key_out[p] = sort key (bins) of the moved particle p, the key
    // the cell sort would compute from the new position
    uint32_t* key_out;
    BinP bins;
};

inline Advect make_advect(const picasso_mesh& m, double dt)
{
    Advect a{};
    a.dt = dt;
    a.key_out = nullptr;
    for (int d = 0; d < 3; ++d) {
        a.periodic[d] = m.periodic[d] != 0;
        a.lo[d] = m.low_corner[d] + m.own_begin[d] * m.cell_size[d];
        a.len[d] = m.own_extent[d] * m.cell_size[d];
    }
    return a;
}

__device__ __forceinline__ double advect_coord(const Advect& a, int d, double x, double v)
{
    double xn = __dadd_rn(x, __dmul_rn(a.dt, v));
    if (a.periodic[d]) {
        if (xn < a.lo[d]) xn += a.len[d];
        else if (xn >= a.lo[d] + a.len[d]) xn -= a.len[d];
    }
    return xn;
}

// Moves particle p (x_p += dt u_p, wrapped) and emits its new sort key when
// asked for; xp: the old position, u: the stored velocity.
template <class XStore>
__device__ __forceinline__ void advect_particle(const Advect& a, int64_t p, const double xp[3],
                                                const double u[3], XStore&& store)
{
    double xn[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        xn[d] = advect_coord(a, d, xp[d], u[d]);
        store(d, xn[d]);
    }
    if (a.key_out) a.key_out[p] = particle_key(a.bins, xn);
}

}  // namespace pb
