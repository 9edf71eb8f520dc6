// Per-particle bodies of the plain APIC transfers: one thread handles one
// particle and accumulates straight into HBM with atomics (the form of
// Picasso_APIC.hpp applied per particle by GridOperator::apply).  Used by the
// plain kernels (apic.cu) and by the batched kernel (batch.cu).
#pragma once

#include "common.cuh"
#include "gridops.cuh"
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
__device__ __forceinline__ void apic_p2g_particle(const MeshP& mp, int64_t p, const PField& x,
                                                  const PField& m, const PField& c,
                                                  const GField& gm, const GField& gmu, int stag,
                                                  R scale_m, R scale_mu, int* err)
{
    constexpr int K = SplineTraits<ORDER>::K;
    constexpr int NCI = STAG ? 3 : NC;  // columns of c_p
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
        return;
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

// ---------------------------------------------------------------------------
// G2P
// ---------------------------------------------------------------------------
// GT: grid storage type of u_i; PT: particle storage type of c_p.
// CG: load u_i through L2 only (for grids written earlier in the same launch).
// ADV (collocated, 3 components): then moves the particle, x += dt u_p with
// the stored (PT-rounded) u_p, exactly as picasso_advect would afterwards.
template <int ORDER, int NC, bool STAG, class GT, class PT, class R, bool CG = false,
          bool ADV = false>
__device__ __forceinline__ void apic_g2p_particle(const MeshP& mp, int64_t p, const PField& x,
                                                  const GField& u, const PField& c, int stag,
                                                  int* err, const Advect* adv = nullptr)
{
    constexpr int K = SplineTraits<ORDER>::K;
    constexpr int NCO = STAG ? 3 : NC;
    auto load = [](const GT* a) { return CG ? __ldcg(a) : __ldg(a); };
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
        return;
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
                        ue[d] = (R)load(u.ptr<GT>(idx[0][i], idx[1][j], idx[2][k], d));
#pragma unroll
                    for (int d = 0; d < NC; ++d) {
                        up[d] = up[d] + w * ue[d];
                        const R wu = w * ue[d];
#pragma unroll
                        for (int a = 0; a < 3; ++a) B[d][a] += wu * dist[a];
                    }
                } else {
                    const R ue = (R)load(u.ptr<GT>(idx[0][i], idx[1][j], idx[2][k], 0));
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
    if constexpr (ADV) {
        static_assert(!STAG && NC == 3, "advection needs the 3-component collocated velocity");
        const double xo[3] = {x.get<double>(p, 0), x.get<double>(p, 1), x.get<double>(p, 2)};
        const double uo[3] = {(double)(PT)up[0], (double)(PT)up[1], (double)(PT)up[2]};
        advect_particle(*adv, p, xo, uo, [&](int d, double v) { x.set<double>(p, d, v); });
    }
}

}  // namespace pb
