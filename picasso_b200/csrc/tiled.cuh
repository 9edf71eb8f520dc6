// Work items of the shared-memory tiled APIC transfers (FP32 precision form)
// on cell-sorted particles in packed storage: x_p (N,3) FP64, m_p (N) FP32,
// c_p (N,4,3) FP32.  Used by the single-call kernels (tiled.cu) and by the
// persistent batched kernel (batch.cu).
//
// Work items are chunks of at most `chunk` particles of one tile (the sort
// writes the per-tile item prefix).
//
// P2G item (one warp): particles are processed in runs -- contiguous ranges
// of the sorted item, so consecutive particles of a run mostly share a
// stencil -- and each run is handled by LPP lanes (1, 2 or 4) that split the
// four grid fields (mass, 3 momentum components) between them.  A lane keeps
// the K^3 sums of its fields for the run's current bin in registers.
// Particle records arrive through a cp.async ring in shared memory a few
// particles ahead of use.  When a run's bin changes its lanes stage their
// partial sums and the warp adds the staged partials into its FP32 node tile
// ((T + K - 1)^3 nodes) one staged lane after the other: a fixed order without
// atomics, so the tile sums are reproducible.  At the end of the item the
// touched box of the tile is rounded to 64-bit fixed point and added to HBM
// with integer reductions, whose result does not depend on their order; P2G
// is deterministic for a given particle order.
//
// G2P item (one warp or one CTA): the item's node velocities are staged once
// in a shared float4 tile and every thread gathers its particles' stencils
// from there, contracting the stencil one dimension at a time.
//
// Both read either the FP64 positions or, when the bins carry them, spline
// records (in-cell fractions as FP32 + sort key, written by
// picasso_spline_records from the same FP64 arithmetic): same splines and
// bins, 16 instead of 24 bytes per particle, no FP64 instruction.  Staggered
// locations (Face / Edge) accumulate two grid fields (mass and the entity's
// momentum component) instead of four.  The P2G can also apply the grid
// update to the nodes whose sums are complete (fused_update_arrive).
#pragma once

#include "common.cuh"
#include "gridops.cuh"
#include "transfer.cuh"

namespace pb {

constexpr int kStageLanes = 8;   // lanes staged per full merge round
constexpr int kStageBases = 32;  // stage_base entries (k-plane merges stage every lane at once)
constexpr unsigned kFull = 0xFFFFFFFFu;

// Element type of the P2G node tile that sums the lanes' FP32 partials.
#ifndef PB_P2G_TILE_F64
#define PB_P2G_TILE_F64 0
#endif
using TileVal = std::conditional<PB_P2G_TILE_F64 != 0, double, float>::type;
constexpr int kTileWords = sizeof(TileVal) / sizeof(float);

struct TileP {
    int T[3];    // bins per tile
    int nt[3];   // tiles per dimension
    int nb[3];   // bins per dimension
    int NT[3];   // nodes per tile dimension (T + K - 1)
    int nodes;   // NT0 * NT1 * NT2
    int SJ, SI;  // P2G node-tile strides along j and i (k stride 1), padded so
    int P;       // that a merge's stencil nodes hit distinct banks; P = stride
                 // between the 4 field planes
    int chunk;
    int tsh[3];      // log2(T[d]) when T[d] is a power of two, else -1
    uint32_t tsize;  // bins per tile (sort keys of tile t start at t * tsize)
    int64_t ntiles;
    const int64_t* off;     // tile particle offsets (ntiles + 1)
    const uint32_t* items;  // tile work-item prefix (ntiles + 1)
};

// Neighbour grids of a slab decomposition along x: the local x-planes below
// lo_end are the lower neighbour's planes (index + lo_shift there), those
// from hi_begin on the upper neighbour's (index + hi_shift); the neighbours'
// grids have the local strides.  P2G adds the sums of those nodes into the
// neighbour's grid (lo[0] / hi[0]: mass, [1]: momentum) and G2P reads their
// velocities from it ([0]): the halo exchange happens inside the transfers,
// through peer memory when the neighbour is another GPU.
struct HaloPeers {
    int on;
    int lo_end, hi_begin;
    int lo_shift, hi_shift;
    char* lo[2];
    char* hi[2];
};

// Grid base holding local x-plane gi (own, or a neighbour's field f) and the
// plane's index there.
__device__ __forceinline__ char* halo_route(const HaloPeers& hp, int f, char* own, int gi, int& gx)
{
    gx = gi;
    if (hp.on) {
        if (gi < hp.lo_end) {
            gx = gi + hp.lo_shift;
            return hp.lo[f];
        }
        if (gi >= hp.hi_begin) {
            gx = gi + hp.hi_shift;
            return hp.hi[f];
        }
    }
    return own;
}

// Per-call (per-instance) arguments of the tiled kernels.
struct P2GArgs {
    MeshP mp;
    TileP tp;
    int stag;          // staggered location: the entity's dimension (else -1)
    const double* x;
    const float* rec;  // spline records (4 floats per particle) or null
    const float* m;
    const float* c;
    GField gm;
    GField gmu;
    float scale_m;
    float scale_mu;
    int* err;
    // gm and gmu are one packed accumulator (a node's mass and momentum are 4
    // consecutive 64-bit words, 16-byte aligned): the item's flush adds whole
    // k-rows with bulk reductions (flush_rows_bulk)
    int bulk_flush;
    HaloPeers hp;
};

struct G2PArgs {
    MeshP mp;
    TileP tp;
    int stag;           // staggered location: the entity's dimension (else -1)
    const double* x;
    const float4* rec;  // spline records or null
    GField u;
    float* c;
    int* err;
    double* x_out;  // G2P with advection: positions updated in place (= x)
    Advect adv;
    HaloPeers hp;
};

__device__ __forceinline__ int bin_of(const MeshP& mp, const TileP& tp, int d, int s0)
{
    if (mp.periodic[d]) {
        const int nb = tp.nb[d];
        int r = s0 - mp.own_lo[d];
        if (r < 0) r += nb;          // one period covers every particle inside or
        else if (r >= nb) r -= nb;   // next to the owned box
        if ((unsigned)r >= (unsigned)nb) {
            r %= nb;
            if (r < 0) r += nb;
        }
        return r;
    }
    return s0;
}

__device__ __forceinline__ int node_global(const MeshP& mp, const TileP& tp, int d, int ob,
                                           int local)
{
    int g = ob + local;
    if (mp.periodic[d]) {
        if (g >= tp.nb[d]) g -= tp.nb[d];
        return mp.own_lo[d] + g;
    }
    return g;
}

// Work item w -> tile t and particle range [a, b).  False past the last item.
__device__ __forceinline__ bool item_range(const TileP& tp, int64_t w, int64_t& t, int64_t& a,
                                           int64_t& b)
{
    if (w >= (int64_t)__ldg(tp.items + tp.ntiles)) return false;
    int64_t lo = 0, hi = tp.ntiles - 1;  // last t with items[t] <= w
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if ((int64_t)__ldg(tp.items + mid) <= w) lo = mid;
        else hi = mid - 1;
    }
    t = lo;
    a = __ldg(tp.off + t) + (w - (int64_t)__ldg(tp.items + t)) * tp.chunk;
    b = min(a + (int64_t)tp.chunk, (int64_t)__ldg(tp.off + t + 1));
    return a < b;
}

__device__ __forceinline__ void tile_origin(const TileP& tp, int64_t t, int ob[3])
{
    ob[2] = (int)(t % tp.nt[2]) * tp.T[2];
    ob[1] = (int)((t / tp.nt[2]) % tp.nt[1]) * tp.T[1];
    ob[0] = (int)(t / ((int64_t)tp.nt[1] * tp.nt[2])) * tp.T[0];
}

// Spline of a particle at x and its bin inside the tile with bin origin ob;
// false if the particle is not in this tile (or not in the mesh).
template <int ORDER>
__device__ __forceinline__ bool locate(const MeshP& mp, const TileP& tp, const double xp[3],
                                       const int ob[3], Spline1D<ORDER, float> sp[3], int lb[3])
{
    constexpr int K = SplineTraits<ORDER>::K;
    bool ok = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        eval_spline<ORDER>(xp[d], mp.lo[d], mp.dx[d], mp.rdx[d], sp[d]);
        if (!mp.periodic[d] && (sp[d].s0 < 0 || sp[d].s0 > mp.ext[d] - K)) ok = false;
        lb[d] = bin_of(mp, tp, d, sp[d].s0) - ob[d];
        if (lb[d] < 0 || lb[d] >= tp.T[d]) ok = false;
    }
    return ok;
}

// ---------------------------------------------------------------------------
// cp.async (asynchronous global -> shared copies)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_addr(const void* p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src)
{
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst)),
                     "l"(src));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(smem_addr(dst)),
                     "l"(src), "n"(BYTES));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// ---------------------------------------------------------------------------
// bulk reductions (shared -> global through the tensor memory accelerator;
// both addresses 16-byte aligned, size a multiple of 16 bytes)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void bulk_add_u64(long long* dst, const long long* src, int bytes)
{
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.u64 [%0], [%1], %2;\n"
                 ::"l"(dst), "r"(smem_addr(src)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// the shared-memory sources of this thread's committed bulk operations have
// been read (the buffer may be rewritten)
__device__ __forceinline__ void bulk_wait_read()
{
    asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
}
// shared-memory writes of this thread become visible to the bulk operations
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// P2G
// ---------------------------------------------------------------------------
// Shared-memory layout of one P2G warp: particle-record ring, staging area,
// node tile.  Field g of a node n = (a, b, c) of a bin receives
//   w_n m (e_d + sum_q G_dq (n_q - n0))                     (order 2 / 3)
//   m * (c0 www + cx gww + cy wgw + cz wwg)                  (order 1)
// for the momentum components d = g - 1 and w_n m for the mass (g = 0), with
// n0 the stencil's centre knot, e_d = v_d + D sum_q B_dq dist_q(n0) and
// G_dq = D dx B_dq: the affine term D B dist (APIC.hpp:110-139) written
// relative to the centre knot, where dist_q(n) - dist_q(n0) = (n_q - n0) dx,
// so the nodes next to the centre need one addition and the centre none.
// Order 1: APIC.hpp:287-318 with D = 1.
//
// REC: the particle's position arrives as a spline record (in-cell fraction
// of the logical position along each dimension in FP32, and the sort key
// of its bin) instead of the FP64 position.
// STAG: a staggered location (Face<D> / Edge<D>, APIC.hpp:148-232): two
// grid fields, the mass and the one momentum component of the entity's
// dimension, which comes from column `stag` of c_p.
template <int ORDER, int LPP, bool REC = false, bool STAG = false>
struct P2GCfg {
    static constexpr int K = SplineTraits<ORDER>::K;
    static constexpr int NF = STAG ? 2 : 4;  // grid fields
    static constexpr int KKK = K * K * K;
    static constexpr int N0 = 1;  // centre knot of the quadratic and cubic stencils
    // Cubic stencils with 4 lanes per particle split the stencil by its
    // i-planes (lane h sums all four fields of the 16 nodes (h, j, k)); the
    // other splits are by field (lane h sums fields h F .. h F + F - 1 of all
    // K^3 nodes).  The plane split needs one x-weight per lane and shares the
    // affine products of a (j, k) node between the three momentum fields.
    static constexpr bool ISPLIT = ORDER == 3 && LPP == 4;
    static constexpr int NL = ISPLIT ? K * K : KKK;  // nodes per lane
    static constexpr int ROWS = NL / K;              // k-rows per lane
    static constexpr int FS = (NL + 3) & ~3;         // staged floats per field
    static constexpr int F = ISPLIT ? NF : NF / LPP;  // fields per lane
    static constexpr int RUNS = 32 / LPP;            // runs per warp
    static constexpr int SV = F * FS;                // staged values per lane
    // staging stride: a multiple of 4 floats whose quarter is odd keeps the
    // float4 stores of 8 staged lanes on distinct banks
    static constexpr int SS = ((SV / 4) % 2 == 0) ? SV + 4 : SV;
    static constexpr int R = (SV + 31) / 32;  // merge rounds per staged lane
    // k-plane merges (a lane's bin advanced by one along k): the K^2 nodes of
    // the stencil's first k-plane, F fields, packed
    static constexpr int PV = F * ROWS;
    static constexpr int PV4 = (PV + 3) & ~3;
    static constexpr int PS = ((PV4 / 4) % 2 == 0) ? PV4 + 4 : PV4;
    static constexpr int RP = (PV + 31) / 32;
    static_assert(PS <= SS, "a plane stages inside a full stage slot");
    // ring per stage: position (6 floats: 3 doubles; REC: one 16-byte
    // record) | c (12 floats) | m (1 float) per run
    static constexpr int XS = REC ? 4 : 6;
    static constexpr int RING_X = 0, RING_C = XS * RUNS, RING_M = (XS + 12) * RUNS;
    static constexpr int RING =
        (XS + 13) * RUNS + (((XS + 13) * RUNS) % 4 ? 4 - ((XS + 13) * RUNS) % 4 : 0);
    // ring depth: records of DEPTH - 1 particles are in flight per run; the
    // warps with fewer runs (more lanes per particle) need more to keep the
    // same bytes in flight.  Deeper rings cost shared memory, which costs
    // warps (measured: depth 4 fastest for one lane per particle, and for
    // cubic stencils, whose ~600 instructions per lane and particle hide the
    // loads: 256^3 8 ppc, tile (4, 4, 8): depth 4 14.6 ms, 6 14.7, 10 15.7).
    static constexpr int DEPTH = LPP == 1 ? 4 : (LPP == 2 ? 8 : (ORDER == 3 ? 4 : 10));
    static constexpr int STAGE_OFF = DEPTH * RING;
    // staging area: kStageLanes full stencils, or the first k-plane of every
    // lane (used one after the other)
    static constexpr int STAGE_FLOATS = 32 * PS > kStageLanes * SS ? 32 * PS : kStageLanes * SS;
    static constexpr int TILE_OFF = STAGE_OFF + STAGE_FLOATS;
    // plane split with records, collocated: the lanes of a run evaluate the
    // splines and affine form of the run's next LPP particles once (one
    // particle each) and share them through a table after the node tile
    // (p2g_item)
    static constexpr bool SHARE = ISPLIT && REC && !STAG;
    static constexpr int ENTRY = 28;  // floats of one particle's table entry
    // entries of sub-step q start 8 q floats later (bank skew, p2g_item)
    static constexpr int TABLE = SHARE ? 32 * ENTRY + 8 * (LPP - 1) : 0;
    static_assert(LPP == 1 || LPP == 2 || LPP == 4, "1, 2 or 4 lanes per particle");
    static_assert(F >= 1, "at least one field per lane");
};

// Single-warp CTAs per SM the P2G register budget is sized for: 1 lane per
// particle holds 4 x K^3 accumulators (~255 registers), 2 and 4 lanes a half
// and a quarter of them; cubic 4-lane items also hold a 64-node stencil.
template <int ORDER, int LPP>
struct P2GOccupancy {
    static constexpr int value = LPP == 1 ? 8 : (LPP == 2 ? 12 : (ORDER == 3 ? 12 : 16));
};

template <int ORDER, int LPP, bool REC = false, bool STAG = false>
__host__ __device__ constexpr int p2g_warp_floats(int P)
{
    return P2GCfg<ORDER, LPP, REC, STAG>::TILE_OFF +
           P2GCfg<ORDER, LPP, REC, STAG>::NF * P * kTileWords +
           P2GCfg<ORDER, LPP, REC, STAG>::TABLE;
}

// p + s g for a small integer s (s = 0: p exactly).  Called with unrolled
// loop indices, so the branch folds at compile time.
__device__ __forceinline__ float add_steps(int s, float p, float g)
{
    if (s == 0) return p;
    if (s == 1) return p + g;
    if (s == -1) return p - g;
    return fmaf((float)s, g, p);
}

template <int ORDER, int LPP, bool STAG = false>
struct P2GAcc {
    using C = P2GCfg<ORDER, LPP, false, STAG>;
    float acc[C::F][C::NL];

    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int f = 0; f < C::F; ++f)
#pragma unroll
            for (int n = 0; n < C::NL; ++n) acc[f][n] = 0.f;
    }

    // Orders 2 / 3.  E[f], G[f][q]: the centre-knot form of field f of the
    // lane (mass: E = 1, G = 0); h: the lane's share of the particle (its
    // i-plane when C::ISPLIT).  `mass_first`: field 0 of the lane is the
    // mass (known at compile time for one lane per particle and for the
    // plane split).
    __device__ __forceinline__ void add(const Spline1D<ORDER, float> sp[3], float mass,
                                        const float E[C::F], const float G[C::F][3], int h)
    {
        constexpr int K = C::K;
        constexpr int N0 = C::N0;
        constexpr bool MASS0 = C::ISPLIT || LPP == 1;
        if constexpr (C::ISPLIT) {
            float wx = 0.f;
#pragma unroll
            for (int i = 0; i < K; ++i)
                if (i == h) wx = sp[0].w[i];
            add_isplit(wx, sp[1].w, sp[2].w, mass, E, G, h);
        } else {
#pragma unroll
            for (int i = 0; i < K; ++i) {
                const float wi = sp[0].w[i] * mass;
                float pi[C::F];
#pragma unroll
                for (int f = 0; f < C::F; ++f) pi[f] = add_steps(i - N0, E[f], G[f][0]);
#pragma unroll
                for (int j = 0; j < K; ++j) {
                    const float wij = wi * sp[1].w[j];
                    float pij[C::F];
#pragma unroll
                    for (int f = 0; f < C::F; ++f) pij[f] = add_steps(j - N0, pi[f], G[f][1]);
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const int n = (i * K + j) * K + k;
                        const float w = wij * sp[2].w[k];
#pragma unroll
                        for (int f = 0; f < C::F; ++f) {
                            if (MASS0 && f == 0) acc[f][n] += w;
                            else
                                acc[f][n] =
                                    fmaf(w, add_steps(k - N0, pij[f], G[f][2]), acc[f][n]);
                        }
                    }
                }
            }
        }
    }

    // Plane split: the lane's i-plane h, x-weight wx = w_x[h]; node (h, j, k)
    // receives w = wx m wy_j wz_k.
    __device__ __forceinline__ void add_isplit(float wx, const float* wy, const float* wz,
                                               float mass, const float E[C::F],
                                               const float G[C::F][3], int h)
    {
        constexpr int K = C::K;
        constexpr int N0 = C::N0;
        const float wxm = wx * mass;
        const float hs = (float)(h - N0);
        float pi[C::F];
#pragma unroll
        for (int f = 1; f < C::F; ++f) pi[f] = fmaf(hs, G[f][0], E[f]);
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const float wij = wxm * wy[j];
            float pij[C::F];
#pragma unroll
            for (int f = 1; f < C::F; ++f) pij[f] = add_steps(j - N0, pi[f], G[f][1]);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int n = j * K + k;
                const float w = wij * wz[k];
                acc[0][n] += w;
#pragma unroll
                for (int f = 1; f < C::F; ++f)
                    acc[f][n] = fmaf(w, add_steps(k - N0, pij[f], G[f][2]), acc[f][n]);
            }
        }
    }

    // Order 1 (gradient form); co[f] = (c0, cx, cy, cz) of field f.
    __device__ __forceinline__ void add_linear(const Spline1D<ORDER, float> sp[3], float mass,
                                               const float co[C::F][4])
    {
        constexpr int K = C::K;
#pragma unroll
        for (int i = 0; i < K; ++i)
#pragma unroll
            for (int j = 0; j < K; ++j)
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const int n = (i * K + j) * K + k;
                    const float www = sp[0].w[i] * sp[1].w[j] * sp[2].w[k] * mass;
                    const float gww = sp[0].g[i] * sp[1].w[j] * sp[2].w[k] * mass;
                    const float wgw = sp[0].w[i] * sp[1].g[j] * sp[2].w[k] * mass;
                    const float wwg = sp[0].w[i] * sp[1].w[j] * sp[2].g[k] * mass;
#pragma unroll
                    for (int f = 0; f < C::F; ++f) {
                        if (LPP == 1 && f == 0) acc[f][n] += www;  // mass
                        else
                            acc[f][n] += co[f][0] * www + co[f][1] * gww + co[f][2] * wgw +
                                         co[f][3] * wwg;
                    }
                }
    }

    // st[f * FS + n] <- acc[f][n] with 16-byte stores.
    __device__ __forceinline__ void stage(float* st) const
    {
#pragma unroll
        for (int f = 0; f < C::F; ++f)
#pragma unroll
            for (int q = 0; q < C::FS / 4; ++q) {
                float4 v;
                v.x = (4 * q + 0 < C::NL) ? acc[f][4 * q + 0] : 0.f;
                v.y = (4 * q + 1 < C::NL) ? acc[f][4 * q + 1] : 0.f;
                v.z = (4 * q + 2 < C::NL) ? acc[f][4 * q + 2] : 0.f;
                v.w = (4 * q + 3 < C::NL) ? acc[f][4 * q + 3] : 0.f;
                *reinterpret_cast<float4*>(st + f * C::FS + 4 * q) = v;
            }
    }

    // value v of the first k-plane: field v / ROWS, k-row v % ROWS (the row
    // (i, j) with i * K + j = v % ROWS, or (h, j) with j = v % ROWS for the
    // plane split), its node k = 0
    __device__ __forceinline__ float plane_value(int v) const
    {
        return acc[v / C::ROWS][(v % C::ROWS) * C::K];
    }

    // st[v] <- plane_value(v) with 16-byte stores.
    __device__ __forceinline__ void stage_plane(float* st) const
    {
#pragma unroll
        for (int q = 0; q < C::PV4 / 4; ++q) {
            float4 v;
            v.x = (4 * q + 0 < C::PV) ? plane_value(4 * q + 0) : 0.f;
            v.y = (4 * q + 1 < C::PV) ? plane_value(4 * q + 1) : 0.f;
            v.z = (4 * q + 2 < C::PV) ? plane_value(4 * q + 2) : 0.f;
            v.w = (4 * q + 3 < C::PV) ? plane_value(4 * q + 3) : 0.f;
            *reinterpret_cast<float4*>(st + 4 * q) = v;
        }
    }

    // Moves the sums one node down along k (the stencil moved up by one):
    // planes 1 .. K-1 become 0 .. K-2, the last plane starts at zero.
    __device__ __forceinline__ void shift_k()
    {
        constexpr int K = C::K;
#pragma unroll
        for (int f = 0; f < C::F; ++f)
#pragma unroll
            for (int ij = 0; ij < C::ROWS; ++ij) {
#pragma unroll
                for (int k = 0; k + 1 < K; ++k) acc[f][ij * K + k] = acc[f][ij * K + k + 1];
                acc[f][ij * K + K - 1] = 0.f;
            }
    }
};

// Merge plan of one lane: staged value v = lane + 32 r of a staged lane that
// handles fields hh F .. hh F + F - 1 (plane split: i-plane hh) lands at tile
// offset moff[r] + hh * fstride from the stencil start.
template <int ORDER, int LPP, bool STAG = false>
struct MergePlan {
    using C = P2GCfg<ORDER, LPP, false, STAG>;
    int moff[C::R];
    int poff[C::RP];  // the same for the values of a k-plane stage
    int fstride;      // F * P (plane split: SI)
    unsigned valid;   // bit r: value lane + 32 r exists
    unsigned pvalid;
    __device__ __forceinline__ void init(const TileP& tp, int lane)
    {
        constexpr int K = C::K;
        valid = 0;
        // the plane split offsets a staged lane's values by its i-plane
        fstride = C::ISPLIT ? tp.SI : C::F * tp.P;
#pragma unroll
        for (int r = 0; r < C::R; ++r) {
            const int v = lane + 32 * r;
            const int fs = v / C::FS, nn = v - (v / C::FS) * C::FS;
            moff[r] = 0;
            if (v < C::SV && nn < C::NL) {
                const int a = nn / (K * K), b = (nn / K) % K, c = nn % K;
                moff[r] = fs * tp.P + a * tp.SI + b * tp.SJ + c;
                valid |= 1u << r;
            }
        }
        pvalid = 0;
#pragma unroll
        for (int r = 0; r < C::RP; ++r) {
            const int v = lane + 32 * r;
            poff[r] = 0;
            if (v < C::PV) {
                const int fs = v / C::ROWS, ij = v % C::ROWS;
                poff[r] = fs * tp.P + (ij / K) * tp.SI + (ij % K) * tp.SJ;
                pvalid |= 1u << r;
            }
        }
    }
};

// The warp adds staged values into the node tile: lane l adds value l + 32 r
// of each staged slot at tile offset base + off[r], slot after slot in a
// fixed order (so the tile sums are reproducible): slots 0 .. n - 1 (LANES
// false, n = `slots`) or the set bits of `slots`, lowest first (LANES true,
// not empty).  The next slot's base and values are read before this slot's
// tile updates, so only the tile read-add-write is on the dependency chain.
template <int NR, int SLOT, int LPP, bool LANES>
__device__ __forceinline__ void add_staged(unsigned slots, const float* stage,
                                           const int* stage_base, const int (&off)[NR],
                                           unsigned valid, int fstride, TileVal* tile, int lane)
{
    int q = LANES ? __ffs(slots) - 1 : 0;
    unsigned rest = LANES ? slots & (slots - 1u) : slots - 1u;  // LANES false: slots left
    int sb = stage_base[q];
    float v[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r)
        v[r] = ((valid >> r) & 1u) ? stage[q * SLOT + lane + 32 * r] : 0.f;
    for (;;) {
        const int qn = rest ? (LANES ? __ffs(rest) - 1 : q + 1) : q;
        const int sbn = stage_base[qn];
        float vn[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r)
            vn[r] = ((valid >> r) & 1u) ? stage[qn * SLOT + lane + 32 * r] : 0.f;
        const int base = (sb & 0x0FFFFFFF) + (LPP > 1 ? (sb >> 28) * fstride : 0);
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if ((valid >> r) & 1u) tile[base + off[r]] += v[r];
        __syncwarp();
        if (!rest) break;
        rest = LANES ? rest & (rest - 1u) : rest - 1u;
        q = qn;
        sb = sbn;
#pragma unroll
        for (int r = 0; r < NR; ++r) v[r] = vn[r];
    }
}

// Lanes in `mask` hand their partial sums to the warp's node tile in lane
// order (rounds of at most kStageLanes lanes); their accumulators are zeroed.
template <int ORDER, int LPP, bool STAG>
__device__ __forceinline__ void merge_partials(unsigned mask, P2GAcc<ORDER, LPP, STAG>& acc,
                                               int cur_base,
                                               const MergePlan<ORDER, LPP, STAG>& plan,
                                               TileVal* tile, float* stage, int* stage_base,
                                               int lane)
{
    using C = P2GCfg<ORDER, LPP, false, STAG>;
    while (mask) {
        unsigned batch = mask;
        if (__popc(mask) > kStageLanes) {  // the lowest kStageLanes lanes
            batch = 0;
            unsigned mm = mask;
#pragma unroll
            for (int q = 0; q < kStageLanes; ++q) {
                batch |= mm & (~mm + 1u);
                mm &= mm - 1u;
            }
        }
        mask &= ~batch;
        if ((batch >> lane) & 1u) {
            const int slot = __popc(batch & ((1u << lane) - 1u));
            acc.stage(stage + slot * C::SS);
            stage_base[slot] = cur_base | ((lane % LPP) << 28);
            acc.zero();
        }
        __syncwarp();
        add_staged<C::R, C::SS, LPP, false>(__popc(batch), stage, stage_base, plan.moff,
                                            plan.valid, plan.fstride, tile, lane);
    }
}

// Lanes in `mask` (whose bin moved one step along k) hand the first k-plane
// of their sums to the node tile and shift the rest down: every lane of the
// mask stages its plane in its own slot and shifts (one pass for the warp),
// then the warp adds the planes in lane order.
template <int ORDER, int LPP, bool STAG>
__device__ __forceinline__ void merge_plane(unsigned mask, P2GAcc<ORDER, LPP, STAG>& acc,
                                            int cur_base, const MergePlan<ORDER, LPP, STAG>& plan,
                                            TileVal* tile, float* stage, int* stage_base, int lane)
{
    using C = P2GCfg<ORDER, LPP, false, STAG>;
    if ((mask >> lane) & 1u) {
        acc.stage_plane(stage + lane * C::PS);
        acc.shift_k();
    }
    stage_base[lane] = cur_base | ((lane % LPP) << 28);
    __syncwarp();
    add_staged<C::RP, C::PS, LPP, true>(mask, stage, stage_base, plan.poff, plan.pvalid,
                                        plan.fstride, tile, lane);
}

// Bin inside tile t of a particle from its sort key; false if the key is
// not one of the tile's bins (another tile, or outside the mesh).
__device__ __forceinline__ bool bin_of_key(const TileP& tp, int64_t t, uint32_t key, int lb[3])
{
    const uint32_t ll = key - (uint32_t)t * tp.tsize;
    uint32_t r;
    if (tp.tsh[2] >= 0) {
        lb[2] = (int)(ll & (uint32_t)(tp.T[2] - 1));
        r = ll >> tp.tsh[2];
    } else {
        r = ll / (uint32_t)tp.T[2];
        lb[2] = (int)(ll - r * (uint32_t)tp.T[2]);
    }
    if (tp.tsh[1] >= 0) {
        lb[1] = (int)(r & (uint32_t)(tp.T[1] - 1));
        lb[0] = (int)(r >> tp.tsh[1]);
    } else {
        const uint32_t r2 = r / (uint32_t)tp.T[1];
        lb[1] = (int)(r - r2 * (uint32_t)tp.T[1]);
        lb[0] = (int)r2;
    }
    return ll < tp.tsize;
}

// Spline of a particle from its record (in-cell fractions, key) and its bin
// inside tile t; false if the particle is not in this tile.
template <int ORDER>
__device__ __forceinline__ bool locate_record(const MeshP& mp, const TileP& tp, int64_t t,
                                              float4 r, Spline1D<ORDER, float> sp[3], int lb[3])
{
    const bool ok = bin_of_key(tp, t, __float_as_uint(r.w), lb);
    spline_from_frac<ORDER, float>(r.x, (float)mp.dx[0], mp.rdx[0], sp[0]);
    spline_from_frac<ORDER, float>(r.y, (float)mp.dx[1], mp.rdx[1], sp[1]);
    spline_from_frac<ORDER, float>(r.z, (float)mp.dx[2], mp.rdx[2], sp[2]);
    return ok;
}

// Flush of a P2G item's node box (bin rows [i_lo, i_hi] plus the halo, the
// whole tile along j and k) into a packed accumulator: the box's k-rows are
// rounded to fixed point into `buf` (room for buf_nodes nodes of 4 words, a
// group of rows at a time) and each row is added to HBM by one bulk
// reduction (two where it wraps around a periodic boundary; rows and nodes
// past a non-periodic mesh end are left out -- no stencil reaches them).
// The integer sums do not depend on the order of the reductions.
template <int ORDER>
__device__ __forceinline__ void flush_rows_bulk(const P2GArgs& A, const TileVal* tile, int i_lo,
                                                int i_hi, const int ob[3], float* buf_f,
                                                int buf_nodes, int lane)
{
    constexpr int K = SplineTraits<ORDER>::K;
    const MeshP& mp = A.mp;
    const TileP& tp = A.tp;
    long long* buf = reinterpret_cast<long long*>(buf_f);
    const int e1 = tp.NT[1], e2 = tp.NT[2];
    const int rows = (i_hi - i_lo + K) * e1;
    const int per = buf_nodes / e2;  // rows per group (>= 1, checked by the host)
    // nodes of a row before the periodic wrap or the mesh end along k
    const int gk0 = node_global(mp, tp, 2, ob[2], 0);
    const int n0 = mp.periodic[2] ? min(e2, tp.nb[2] - ob[2]) : min(e2, mp.ext[2] - gk0);
    const bool wraps = mp.periodic[2] && n0 < e2;
    const int gk1 = wraps ? node_global(mp, tp, 2, ob[2], n0) : 0;
    for (int r0 = 0; r0 < rows; r0 += per) {
        const int nr = min(per, rows - r0);
        if (r0 > 0) {  // the previous group's rows have been read
            bulk_wait_read();
            __syncwarp();
        }
        for (int node = lane; node < nr * e2; node += 32) {  // node of the group
            const int q = node / e2;
            const int k = node - q * e2;
            const int row = r0 + q;
            const int i = i_lo + row / e1, j = row - (row / e1) * e1;
            const int idx = i * tp.SI + j * tp.SJ + k;
            long long w[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                const TileVal x = tile[f * tp.P + idx];
                w[f] = x != TileVal(0)
                           ? to_fixed(f == 0 ? A.gm : A.gmu,
                                      x * (TileVal)(f == 0 ? A.scale_m : A.scale_mu))
                           : 0LL;
            }
            longlong2* d = reinterpret_cast<longlong2*>(buf + 4 * node);
            d[0] = make_longlong2(w[0], w[1]);
            d[1] = make_longlong2(w[2], w[3]);
        }
        fence_proxy_async_smem();
        __syncwarp();
        for (int q = lane; q < nr; q += 32) {
            const int row = r0 + q;
            const int i = i_lo + row / e1, j = row - (row / e1) * e1;
            const int gi = node_global(mp, tp, 0, ob[0], i);
            const int gj = node_global(mp, tp, 1, ob[1], j);
            if ((!mp.periodic[0] && gi >= mp.ext[0]) || (!mp.periodic[1] && gj >= mp.ext[1]))
                continue;
            const long long* src = buf + (size_t)q * e2 * 4;
            if (n0 > 0) bulk_add_u64(A.gm.ptr<long long>(gi, gj, gk0, 0), src, n0 * 32);
            if (wraps)
                bulk_add_u64(A.gm.ptr<long long>(gi, gj, gk1, 0), src + 4 * n0, (e2 - n0) * 32);
        }
        bulk_commit();
    }
    bulk_wait_read();  // the buffer is the next item's ring
    __syncwarp();
}

// One P2G work item (tile t, particles [a, b)) by the calling warp.  `warp_smem`
// holds p2g_warp_floats<ORDER, LPP, REC>(P) floats (16-byte aligned),
// `stage_base` kStageLanes ints of shared memory.
template <int ORDER, int LPP, bool REC = false, bool STAG = false>
__device__ void p2g_item(const P2GArgs& A, int64_t t, int64_t a, int64_t b, float* warp_smem,
                         int* stage_base)
{
    using C = P2GCfg<ORDER, LPP, REC, STAG>;
    using Acc = P2GAcc<ORDER, LPP, STAG>;
    static_assert(C::SV == P2GCfg<ORDER, LPP, false, STAG>::SV &&
                      C::SS == P2GCfg<ORDER, LPP, false, STAG>::SS,
                  "the record form changes only the ring");
    constexpr int K = C::K;
    const MeshP& mp = A.mp;
    const TileP& tp = A.tp;
    const int lane = threadIdx.x & 31;
    const int run = lane / LPP, h = lane % LPP;
    float* ring = warp_smem;
    float* stage = warp_smem + C::STAGE_OFF;
    TileVal* tile = reinterpret_cast<TileVal*>(warp_smem + C::TILE_OFF);

    int ob[3];
    tile_origin(tp, t, ob);
    const int U = (int)((b - a + C::RUNS - 1) / C::RUNS);
    const int64_t my0 = a + (int64_t)run * U;
    const int cnt = (int)max((int64_t)0, min(my0 + U, b) - my0);
    // bin rows spanned by the item (keys are i-major within a tile): the
    // first and last particle bound them; the item's node box is these rows
    // plus the halo, over the whole tile along j and k
    int i_lo = 0, i_hi = tp.T[0] - 1;
    {
        int la[3], lz[3];
        bool oka, okb;
        if constexpr (REC) {
            oka = bin_of_key(tp, t, __float_as_uint(__ldg(A.rec + 4 * a + 3)), la);
            okb = bin_of_key(tp, t, __float_as_uint(__ldg(A.rec + 4 * (b - 1) + 3)), lz);
        } else {
            Spline1D<ORDER, float> sp[3];
            const double xa[3] = {A.x[3 * a], A.x[3 * a + 1], A.x[3 * a + 2]};
            const double xb[3] = {A.x[3 * (b - 1)], A.x[3 * (b - 1) + 1], A.x[3 * (b - 1) + 2]};
            oka = locate<ORDER>(mp, tp, xa, ob, sp, la);
            okb = locate<ORDER>(mp, tp, xb, ob, sp, lz);
        }
        if (oka && okb && lz[0] >= la[0]) {
            i_lo = la[0];
            i_hi = lz[0];
        }
    }

    for (int i = lane; i < C::NF * tp.P; i += 32) tile[i] = TileVal(0);
    MergePlan<ORDER, LPP, STAG> plan;
    plan.init(tp, lane);
    const float D = (ORDER >= 2) ? inertial_scaling<ORDER, float>(mp.dx[0]) : 1.f;
    const float Dh = D * (float)mp.dx[0];

    auto slot = [&](int q) { return ring + (q % C::DEPTH) * C::RING; };
    // the copies of a particle record are spread over the run's lanes: copy
    // j is issued by lane h == j % LPP (position: 3 x 8 bytes or one 16-byte
    // record, c: 3 x 16 bytes, m: 4 bytes)
    constexpr int NX = REC ? 1 : 3;
    auto issue = [&](int q) {
        if (q < cnt) {
            const int64_t p = my0 + q;
            float* s = slot(q);
            float* sx = s + C::RING_X + run * C::XS;
            float* sc = s + C::RING_C + run * 12;
#pragma unroll
            for (int j = 0; j < NX + 4; ++j) {
                if (j % LPP != h) continue;
                if (j < NX) {
                    if constexpr (REC) cp_async<16>(sx, A.rec + 4 * p);
                    else cp_async<8>(sx + 2 * j, A.x + 3 * p + j);
                } else if (j < NX + 3) {
                    cp_async<16>(sc + 4 * (j - NX), A.c + 12 * p + 4 * (j - NX));
                } else {
                    cp_async<4>(s + C::RING_M + run, A.m + p);
                }
            }
        }
        cp_async_commit();
    };
#pragma unroll
    for (int q = 0; q < C::DEPTH - 1; ++q) issue(q);

    // Spline and bin of one particle, and its mass and coefficients, read
    // from its ring slot.
    struct Part {
        Spline1D<ORDER, float> sp[3];
        int lb[3];
        bool ok;
    };
    auto locate_slot = [&](int q, Part& P) {
        P.ok = false;
        P.lb[0] = P.lb[1] = P.lb[2] = 0;
        if (q >= cnt) return;
        if constexpr (REC) {
            const float4 r = *reinterpret_cast<const float4*>(slot(q) + C::RING_X + run * 4);
            P.ok = locate_record<ORDER>(mp, tp, t, r, P.sp, P.lb);
        } else {
            const double* sx = reinterpret_cast<const double*>(slot(q) + C::RING_X + run * 6);
            const double xp[3] = {sx[0], sx[1], sx[2]};
            P.ok = locate<ORDER>(mp, tp, xp, ob, P.sp, P.lb);
        }
        // a particle out of the item's rows (the particles are not sorted)
        // is skipped like one of another tile
        P.ok = P.ok && P.lb[0] >= i_lo && P.lb[0] <= i_hi;
        if (!P.ok && A.err && h == 0) atomicAdd(A.err, 1);
    };
    auto read_c = [&](int q, float cp[12], float& mass) {
        const float* sl = slot(q);
        const float* sc = sl + C::RING_C + run * 12;
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const float4 w = *reinterpret_cast<const float4*>(sc + 4 * v);
            cp[4 * v] = w.x;
            cp[4 * v + 1] = w.y;
            cp[4 * v + 2] = w.z;
            cp[4 * v + 3] = w.w;
        }
        mass = sl[C::RING_M + run];
    };
    // cp[r * 3 + d] = c_p(r, d); field g of the lane: mass (g = 0) or
    // momentum d = g - 1 (staggered: d = the entity's dimension)
    auto centre_form = [&](const float cp[12], const Spline1D<ORDER, float> sp[3],
                           float E[C::F], float G[C::F][3]) {
#pragma unroll
        for (int f = 0; f < C::F; ++f) {
            const int g = C::ISPLIT ? f : h * C::F + f;
            if (g == 0) {
                E[f] = 1.f;
                G[f][0] = G[f][1] = G[f][2] = 0.f;
            } else {
                const int d = STAG ? A.stag : g - 1;
                const float bx = d == 0 ? cp[3] : (d == 1 ? cp[4] : cp[5]);
                const float by = d == 0 ? cp[6] : (d == 1 ? cp[7] : cp[8]);
                const float bz = d == 0 ? cp[9] : (d == 1 ? cp[10] : cp[11]);
                const float v = d == 0 ? cp[0] : (d == 1 ? cp[1] : cp[2]);
                const float bd = fmaf(bz, sp[2].d[C::N0],
                                      fmaf(by, sp[1].d[C::N0], bx * sp[0].d[C::N0]));
                E[f] = fmaf(D, bd, v);
                G[f][0] = Dh * bx;
                G[f][1] = Dh * by;
                G[f][2] = Dh * bz;
            }
        }
    };
    auto linear_form = [&](const float cp[12], float co[C::F][4]) {
#pragma unroll
        for (int f = 0; f < C::F; ++f) {
            const int g = h * C::F + f;
            if (g == 0) {
                co[f][0] = 1.f;
                co[f][1] = co[f][2] = co[f][3] = 0.f;
            } else {
                const int d = STAG ? A.stag : g - 1;
                co[f][0] = d == 0 ? cp[0] : (d == 1 ? cp[1] : cp[2]);
                co[f][1] = d == 0 ? cp[3] : (d == 1 ? cp[4] : cp[5]);
                co[f][2] = d == 0 ? cp[6] : (d == 1 ? cp[7] : cp[8]);
                co[f][3] = d == 0 ? cp[9] : (d == 1 ? cp[10] : cp[11]);
            }
        }
    };

    Acc acc;
    acc.zero();
    int cur = -1, cur_base = 0;
    if constexpr (C::SHARE) {
        // Groups of LPP steps: lane h of a run evaluates particle s0 + h of
        // the run (record, splines, bin, affine form) and writes it to the
        // table; in sub-step q the run's lanes read entry (q, run).  Entries
        // are sub-step-major so that the 8 runs' entries of one sub-step fall
        // on different banks, and the entries of sub-step q are shifted by 8 q
        // floats so that the 8 lanes of a quarter warp (2 runs x 4 sub-steps)
        // write to different banks too (ENTRY * 8 is a multiple of 32).  The
        // ring holds one group (DEPTH == LPP): the
        // next group's records are issued once the entries are written and
        // arrive during the sub-steps.  Same arithmetic as the loop below.
        static_assert(C::DEPTH == LPP, "one group in the ring");
        float* table = warp_smem + C::TILE_OFF + C::NF * tp.P * kTileWords;
        issue(C::DEPTH - 1);  // steps 0 .. DEPTH - 2 are in flight
        for (int s0 = 0; s0 < U; s0 += LPP) {
            cp_async_wait<0>();  // the group's records have landed
            __syncwarp();        // ... for every lane of each run
            {
                const int q = s0 + h;
                Spline1D<ORDER, float> sp[3];
                int lb[3] = {0, 0, 0};
                bool ok = false;
                float cp[12], mass = 0.f;
#pragma unroll
                for (int v = 0; v < 12; ++v) cp[v] = 0.f;
#pragma unroll
                for (int d = 0; d < 3; ++d)
#pragma unroll
                    for (int n = 0; n < K; ++n) sp[d].w[n] = sp[d].d[n] = 0.f;
                if (q < cnt) {
                    const float4 r = *reinterpret_cast<const float4*>(slot(q) + C::RING_X + run * 4);
                    ok = locate_record<ORDER>(mp, tp, t, r, sp, lb);
                    // a particle out of the item's rows is skipped like one of
                    // another tile
                    ok = ok && lb[0] >= i_lo && lb[0] <= i_hi;
                    if (!ok && A.err) atomicAdd(A.err, 1);
                    read_c(q, cp, mass);
                }
                float E[C::F], G[C::F][3];
                centre_form(cp, sp, E, G);
                float4* e =
                    reinterpret_cast<float4*>(table + (h * C::RUNS + run) * C::ENTRY + 8 * h);
                e[0] = make_float4(sp[0].w[0], sp[0].w[1], sp[0].w[2], sp[0].w[3]);
                e[1] = make_float4(sp[1].w[0], sp[1].w[1], sp[1].w[2], sp[1].w[3]);
                e[2] = make_float4(sp[2].w[0], sp[2].w[1], sp[2].w[2], sp[2].w[3]);
                e[3] = make_float4(mass, E[1], E[2], E[3]);
                e[4] = make_float4(G[1][0], G[1][1], G[1][2], G[2][0]);
                e[5] = make_float4(G[2][1], G[2][2], G[3][0], G[3][1]);
                const int lbin = ok ? (lb[0] * tp.T[1] + lb[1]) * tp.T[2] + lb[2] : -1;
                e[6] = make_float4(G[3][2], __int_as_float(lbin),
                                   __int_as_float(lb[0] * tp.SI + lb[1] * tp.SJ + lb[2]),
                                   __int_as_float(lb[2]));
            }
            __syncwarp();  // entries written, the group's ring slots read
#pragma unroll
            for (int q = 0; q < LPP; ++q) issue(s0 + LPP + q);
            for (int q = 0; q < LPP; ++q) {
                const float* ef = table + (q * C::RUNS + run) * C::ENTRY + 8 * q;
                const float4* e = reinterpret_cast<const float4*>(ef);
                const float wx = ef[h];
                const float4 wy4 = e[1], wz4 = e[2], me = e[3], g0 = e[4], g1 = e[5], g2 = e[6];
                const int lbin = __float_as_int(g2.y);
                const bool ok = lbin >= 0;
                const bool chg = ok && cur >= 0 && lbin != cur;
                const bool kstep = chg && lbin == cur + 1 && __float_as_int(g2.w) != 0;
                const unsigned pm = __ballot_sync(kFull, kstep);
                const unsigned fm = __ballot_sync(kFull, chg && !kstep);
                if (pm) merge_plane(pm, acc, cur_base, plan, tile, stage, stage_base, lane);
                if (fm) merge_partials(fm, acc, cur_base, plan, tile, stage, stage_base, lane);
                if (ok) {
                    if (lbin != cur) {
                        cur = lbin;
                        cur_base = __float_as_int(g2.z);
                    }
                    const float wy[4] = {wy4.x, wy4.y, wy4.z, wy4.w};
                    const float wz[4] = {wz4.x, wz4.y, wz4.z, wz4.w};
                    const float E[C::F] = {1.f, me.y, me.z, me.w};
                    const float G[C::F][3] = {{0.f, 0.f, 0.f},
                                              {g0.x, g0.y, g0.z},
                                              {g0.w, g1.x, g1.y},
                                              {g1.z, g1.w, g2.x}};
                    acc.add_isplit(wx, wy, wz, me.x, E, G, h);
                }
            }
        }
    } else
    for (int s = 0; s < U; ++s) {
        __syncwarp();  // no lane still reads the slot refilled next
        issue(s + C::DEPTH - 1);
        cp_async_wait<C::DEPTH - 1>();  // record s has landed
        __syncwarp();                   // ... for every lane of its run
        Part P;
        locate_slot(s, P);
        const bool ok = P.ok;
        const int* lb = P.lb;
        const int lbin = ok ? (lb[0] * tp.T[1] + lb[1]) * tp.T[2] + lb[2] : -1;
        // a bin change to the next bin along k (same i, j) keeps two thirds
        // of the stencil: only the finished k-plane is merged
        const bool chg = ok && cur >= 0 && lbin != cur;
        const bool kstep = chg && lbin == cur + 1 && lb[2] != 0;
        const unsigned pm = __ballot_sync(kFull, kstep);
        const unsigned fm = __ballot_sync(kFull, chg && !kstep);
        if (pm) merge_plane(pm, acc, cur_base, plan, tile, stage, stage_base, lane);
        if (fm) merge_partials(fm, acc, cur_base, plan, tile, stage, stage_base, lane);
        if (ok) {
            if (lbin != cur) {
                cur = lbin;
                cur_base = lb[0] * tp.SI + lb[1] * tp.SJ + lb[2];
            }
            float cp[12], mass;
            read_c(s, cp, mass);
            if constexpr (ORDER >= 2) {
                float E[C::F], G[C::F][3];
                centre_form(cp, P.sp, E, G);
                acc.add(P.sp, mass, E, G, h);
            } else {
                float co[C::F][4];
                linear_form(cp, co);
                acc.add_linear(P.sp, mass, co);
            }
        }
    }
    cp_async_wait<0>();
    const unsigned fm = __ballot_sync(kFull, cur >= 0);
    if (fm) merge_partials(fm, acc, cur_base, plan, tile, stage, stage_base, lane);
    // the item's node box, rounded to fixed point and added to HBM: by bulk
    // reductions of whole k-rows into a packed accumulator (the ring and the
    // staging area hold the rounded rows), else node by node (nodes that
    // received nothing are skipped)
    if (!STAG && A.bulk_flush && __any_sync(kFull, cur >= 0)) {
        flush_rows_bulk<ORDER>(A, tile, i_lo, i_hi, ob, warp_smem, C::TILE_OFF / 8, lane);
    } else if (__any_sync(kFull, cur >= 0)) {
        const int e1 = tp.NT[1], e2 = tp.NT[2];
        const int total = (i_hi - i_lo + K) * e1 * e2;
        for (int e = lane; e < total; e += 32) {
            const int k = e % e2;
            const int j = (e / e2) % e1;
            const int i = i_lo + e / (e1 * e2);
            const int idx = i * tp.SI + j * tp.SJ + k;
            const int gi = node_global(mp, tp, 0, ob[0], i);
            const int gj = node_global(mp, tp, 1, ob[1], j);
            const int gk = node_global(mp, tp, 2, ob[2], k);
            // this rank's grids, or the neighbour's that owns plane gi
            int gx_m, gx_mu;
            char* bm = halo_route(A.hp, 0, A.gm.data, gi, gx_m);
            char* bmu = halo_route(A.hp, 1, A.gmu.data, gi, gx_mu);
#pragma unroll
            for (int f = 0; f < C::NF; ++f) {
                const TileVal v = tile[f * tp.P + idx];
                if (v != TileVal(0)) {
                    const long long q = to_fixed(
                        f == 0 ? A.gm : A.gmu, v * (TileVal)(f == 0 ? A.scale_m : A.scale_mu));
                    unsigned long long* dst =
                        f == 0 ? reinterpret_cast<unsigned long long*>(bm) +
                                     A.gm.index(gx_m, gj, gk, 0)
                               : reinterpret_cast<unsigned long long*>(bmu) +
                                     A.gmu.index(gx_mu, gj, gk, STAG ? 0 : f - 1);
                    atomicAdd(dst, (unsigned long long)q);
                }
            }
        }
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// P2G with the grid update in its flush
// ---------------------------------------------------------------------------
// A node's value is final once every work item that can touch it has added
// its tile box.  Every node belongs to the tile of the bin with its index
// (for a non-periodic mesh the last tile along a dimension also takes the
// K - 1 nodes past the last bin), and a tile's nodes form 8 regions by
// whether each local index is below K - 1: those nodes are also touched by
// the items of the previous tile along that dimension, the others only by
// the tile's own items (tiles of at least K - 1 bins).  An item that has
// flushed counts its arrival at every region it can touch (27: the tile and
// its successors along each dimension, their low parts); the item whose
// arrival completes a region's count (the items of the up to 8 tiles that
// touch it) converts the region's nodes with the grid update.  The
// accumulators are exact integer sums, so the conversion sees the same
// values as a separate update pass after P2G: results are bit-identical.
struct FusedUpdate {
    GridUpdate P;
    GField gf, gu, gu64;  // force (optional, FP64), velocity, FP64 velocity (optional)
    uint32_t* count;      // 8 arrival counters per tile, zero at launch
};

// Local node range [lo, hi) of the region part `low` of tile q along d.
__device__ __forceinline__ void region_range(const MeshP& mp, const TileP& tp, int d, int q,
                                             int low, int K, int& lo, int& hi)
{
    const int teff = min(tp.T[d], tp.nb[d] - q * tp.T[d]);
    if (low) {
        lo = 0;
        hi = K - 1;
    } else {
        lo = K - 1;
        hi = teff + ((!mp.periodic[d] && q == tp.nt[d] - 1) ? K - 1 : 0);
    }
}

__device__ __forceinline__ uint32_t tile_items_of(const TileP& tp, int64_t s)
{
    return __ldg(tp.items + s + 1) - __ldg(tp.items + s);
}

// Items of the tiles that touch region `reg` of tile (q0, q1, q2).
__device__ __forceinline__ uint32_t region_items(const MeshP& mp, const TileP& tp, const int q[3],
                                                 int reg)
{
    uint32_t expected = 0;
    for (int mm = 0; mm < 8; ++mm) {
        if (mm & ~reg) continue;
        int pp[3];
        bool ok = true;
        for (int d = 0; d < 3; ++d) {
            pp[d] = q[d] - ((mm >> d) & 1);
            if (pp[d] < 0) {
                if (mp.periodic[d]) pp[d] += tp.nt[d];
                else ok = false;
            }
        }
        if (ok) expected += tile_items_of(tp, ((int64_t)pp[0] * tp.nt[1] + pp[1]) * tp.nt[2] + pp[2]);
    }
    return expected;
}

// Global node of local index g[d] in tile q along d.
__device__ __forceinline__ void region_node(const MeshP& mp, const TileP& tp, const int q[3],
                                            int g[3])
{
    for (int d = 0; d < 3; ++d) {
        g[d] += q[d] * tp.T[d];
        if (mp.periodic[d]) g[d] += mp.own_lo[d];
    }
}

// Called by the whole warp after p2g_item(A, t, ...) has flushed its box.
template <int ORDER>
__device__ void fused_update_arrive(const P2GArgs& A, const FusedUpdate& F, int64_t t)
{
    constexpr int K = SplineTraits<ORDER>::K;
    const MeshP& mp = A.mp;
    const TileP& tp = A.tp;
    const int lane = threadIdx.x & 31;
    __threadfence();  // this lane's reductions are visible before its item counts
    __syncwarp();
    const int q[3] = {(int)(t / ((int64_t)tp.nt[1] * tp.nt[2])),
                      (int)((t / tp.nt[2]) % tp.nt[1]), (int)(t % tp.nt[2])};
    bool last = false;
    int64_t tt = 0;
    int reg = 0;
    if (lane < 27) {
        // per dimension: 0 = this tile, high part; 1 = this tile, low part;
        // 2 = the next tile, low part
        const int o[3] = {lane / 9, (lane / 3) % 3, lane % 3};
        int qq[3];
        bool exists = true;
        for (int d = 0; d < 3; ++d) {
            qq[d] = q[d] + (o[d] == 2);
            if (qq[d] >= tp.nt[d]) {
                if (mp.periodic[d]) qq[d] = 0;
                else exists = false;
            }
            reg |= (o[d] >= 1) << d;
        }
        if (exists) {
            tt = ((int64_t)qq[0] * tp.nt[1] + qq[1]) * tp.nt[2] + qq[2];
            // the items of the tiles that touch the region: qq and, along
            // the region's low dimensions, the previous tile
            const uint32_t expected = region_items(mp, tp, qq, reg);
            const uint32_t old = atomicAdd(F.count + tt * 8 + reg, 1u);
            last = old + 1 == expected;
        }
    }
    unsigned lm = __ballot_sync(kFull, last);
    while (lm) {
        const int src = __ffs(lm) - 1;
        lm &= lm - 1;
        const int64_t ct = __shfl_sync(kFull, tt, src);
        const int cr = __shfl_sync(kFull, reg, src);
        __threadfence();  // every arrival counted: their reductions are visible
        const int cq[3] = {(int)(ct / ((int64_t)tp.nt[1] * tp.nt[2])),
                           (int)((ct / tp.nt[2]) % tp.nt[1]), (int)(ct % tp.nt[2])};
        int lo[3], hi[3];
        for (int d = 0; d < 3; ++d) region_range(mp, tp, d, cq[d], (cr >> d) & 1, K, lo[d], hi[d]);
        const int n1 = hi[1] - lo[1], n2 = hi[2] - lo[2];
        const int total = (hi[0] - lo[0]) * n1 * n2;
        for (int e = lane; e < total; e += 32) {
            int g[3] = {lo[0] + e / (n1 * n2), lo[1] + (e / n2) % n1, lo[2] + e % n2};
            region_node(mp, tp, cq, g);
            update_node<long long, double, float, true>(F.P, A.gm, A.gmu, F.gf, F.gu, F.gu64,
                                                        g[0], g[1], g[2]);
        }
    }
}

// Regions no work item touches are converted by no item: one thread per
// (tile, region) writes them the update of an empty node, 0.
template <int ORDER>
__global__ void zero_untouched_regions_kernel(MeshP mp, TileP tp, FusedUpdate F)
{
    constexpr int K = SplineTraits<ORDER>::K;
    const int64_t total = tp.ntiles * 8;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < total;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = r / 8;
        const int reg = (int)(r % 8);
        const int q[3] = {(int)(t / ((int64_t)tp.nt[1] * tp.nt[2])),
                          (int)((t / tp.nt[2]) % tp.nt[1]), (int)(t % tp.nt[2])};
        if (region_items(mp, tp, q, reg) != 0) continue;
        int lo[3], hi[3];
        for (int d = 0; d < 3; ++d) region_range(mp, tp, d, q[d], (reg >> d) & 1, K, lo[d], hi[d]);
        for (int i = lo[0]; i < hi[0]; ++i)
            for (int j = lo[1]; j < hi[1]; ++j)
                for (int k = lo[2]; k < hi[2]; ++k) {
                    int g[3] = {i, j, k};
                    region_node(mp, tp, q, g);
                    for (int c = 0; c < 3; ++c) {
                        *F.gu.ptr<float>(g[0], g[1], g[2], c) = 0.f;
                        if (F.gu64.data) *F.gu64.ptr<double>(g[0], g[1], g[2], c) = 0.0;
                    }
                }
    }
}

// ---------------------------------------------------------------------------
// G2P
// ---------------------------------------------------------------------------
// One G2P work item by NTHR threads (a warp or a CTA) sharing `tile`
// (tp.nodes float4).  Threads are numbered tid in [0, NTHR).
// ADV: each particle is then moved, x += dt u_p (FP64, as picasso_advect).
// The positions of the item's first and last particle are read before the
// tile barrier, so no thread reads a position another thread has moved.
// REC: the particles' splines come from their records (not with ADV).
// STAG: a staggered location (APIC.hpp:477-544): the grid field is the scalar
// velocity component of the entity's dimension, which lands in column `stag`
// of c_p (the other columns are written as zero, as the plain kernel does).
template <int ORDER, int NTHR, bool ADV = false, bool REC = false, bool STAG = false>
__device__ void g2p_item(const G2PArgs& A, int64_t t, int64_t a, int64_t b, float4* tile,
                         int tid)
{
    static_assert(!(ADV && REC), "the advection reads the FP64 positions");
    static_assert(!(ADV && STAG), "the advection moves by the 3-component velocity");
    constexpr int NU = STAG ? 1 : 3;  // velocity components gathered
    constexpr int K = SplineTraits<ORDER>::K;
    constexpr int N0 = ORDER == 1 ? 0 : 1;  // centre knot of the stencil
    const MeshP& mp = A.mp;
    const TileP& tp = A.tp;
    auto sync = [] {
        if (NTHR == 32) __syncwarp();
        else __syncthreads();
    };
    int ob[3];
    tile_origin(tp, t, ob);
    // bin rows spanned by the item: the first and last particle bound the
    // slowest tile dimension (keys are i-major within a tile)
    int i_lo = 0, i_hi = tp.T[0] - 1;
    if constexpr (REC) {
        int la[3], lz[3];
        const bool oka = bin_of_key(tp, t, __float_as_uint(__ldg(&A.rec[a].w)), la);
        const bool okb = bin_of_key(tp, t, __float_as_uint(__ldg(&A.rec[b - 1].w)), lz);
        if (oka && okb && lz[0] >= la[0]) {
            i_lo = la[0];
            i_hi = lz[0];
        }
    } else {
        Spline1D<ORDER, float> sp[3];
        int lb[3];
        const double xa[3] = {A.x[3 * a], A.x[3 * a + 1], A.x[3 * a + 2]};
        const double xb[3] = {A.x[3 * (b - 1)], A.x[3 * (b - 1) + 1], A.x[3 * (b - 1) + 2]};
        const bool oka = locate<ORDER>(mp, tp, xa, ob, sp, lb);
        const int la = lb[0];
        const bool okb = locate<ORDER>(mp, tp, xb, ob, sp, lb);
        if (oka && okb && lb[0] >= la) {
            i_lo = la;
            i_hi = lb[0];
        }
    }
    const int plane = tp.NT[1] * tp.NT[2];
    const int total = (i_hi - i_lo + K) * plane;
    sync();  // the previous item's threads are done with the tile
    for (int e = tid; e < total; e += NTHR) {
        const int k = e % tp.NT[2];
        const int j = (e / tp.NT[2]) % tp.NT[1];
        const int i = i_lo + e / plane;
        const int gi = node_global(mp, tp, 0, ob[0], i);
        const int gj = node_global(mp, tp, 1, ob[1], j);
        const int gk = node_global(mp, tp, 2, ob[2], k);
        const bool inside = (mp.periodic[0] || gi < mp.ext[0]) &&
                            (mp.periodic[1] || gj < mp.ext[1]) &&
                            (mp.periodic[2] || gk < mp.ext[2]);
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (inside) {  // through L2: the batched kernel writes u_i in the same launch
            int gx;
            const float* ub =
                reinterpret_cast<const float*>(halo_route(A.hp, 0, A.u.data, gi, gx));
            v.x = __ldcg(ub + A.u.index(gx, gj, gk, 0));
            if (!STAG) {
                v.y = __ldcg(ub + A.u.index(gx, gj, gk, 1));
                v.z = __ldcg(ub + A.u.index(gx, gj, gk, 2));
            }
        }
        tile[(i * tp.NT[1] + j) * tp.NT[2] + k] = v;
    }
    sync();
    // positions (records) are prefetched one particle ahead
    double xn[3] = {0.0, 0.0, 0.0};
    float4 rn = make_float4(0.f, 0.f, 0.f, 0.f);
    if (a + tid < b) {
        const int64_t p0 = a + tid;
        if constexpr (REC) {
            rn = __ldg(A.rec + p0);
        } else {
            xn[0] = A.x[3 * p0];
            xn[1] = A.x[3 * p0 + 1];
            xn[2] = A.x[3 * p0 + 2];
        }
    }
    for (int64_t p = a + tid; p < b; p += NTHR) {
        const double xp[3] = {xn[0], xn[1], xn[2]};
        const float4 rp = rn;
        const int64_t pn = p + NTHR;
        if (pn < b) {
            if constexpr (REC) {
                rn = __ldg(A.rec + pn);
            } else {
                xn[0] = A.x[3 * pn];
                xn[1] = A.x[3 * pn + 1];
                xn[2] = A.x[3 * pn + 2];
            }
        }
        Spline1D<ORDER, float> sp[3];
        int lb[3];
        bool ok;
        if constexpr (REC) ok = locate_record<ORDER>(mp, tp, t, rp, sp, lb);
        else ok = locate<ORDER>(mp, tp, xp, ob, sp, lb);
        if (!ok || lb[0] < i_lo || lb[0] > i_hi) {
            if (A.err) atomicAdd(A.err, 1);
            continue;
        }
        const int base = (lb[0] * tp.NT[1] + lb[1]) * tp.NT[2] + lb[2];
        // APIC.hpp:439-461, contracted one dimension at a time, with the
        // distances relative to the centre knot n0 (dist_q(n) = dist_q(n0)
        // + (n_q - n0) dx):
        //   u_p      = sum_i wx_i sum_j wy_j sum_k wz_k u_ijk
        //   M_q      = sum_ijk w_ijk u_ijk (n_q - n0)
        //   B_p(:,q) = dx M_q + dist_q(n0) u_p
        float up[3] = {0.f, 0.f, 0.f};
        float M[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
#pragma unroll
        for (int i = 0; i < K; ++i) {
            float A0[3] = {0.f, 0.f, 0.f}, A1[3] = {0.f, 0.f, 0.f}, A2[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int j = 0; j < K; ++j) {
                const float4* row = tile + base + (i * tp.NT[1] + j) * tp.NT[2];
                float S0[3] = {0.f, 0.f, 0.f}, S1[3] = {0.f, 0.f, 0.f};
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const float4 ue = row[k];
                    const float uk[3] = {ue.x, ue.y, ue.z};
#pragma unroll
                    for (int d = 0; d < NU; ++d) {
                        const float wu = sp[2].w[k] * uk[d];
                        S0[d] += wu;
                        S1[d] = add_steps(k - N0, S1[d], wu);
                    }
                }
                const float wy = sp[1].w[j];
#pragma unroll
                for (int d = 0; d < NU; ++d) {
                    const float wS0 = wy * S0[d];
                    A0[d] += wS0;
                    A1[d] = add_steps(j - N0, A1[d], wS0);
                    A2[d] = fmaf(wy, S1[d], A2[d]);
                }
            }
            const float wx = sp[0].w[i];
#pragma unroll
            for (int d = 0; d < NU; ++d) {
                const float wA0 = wx * A0[d];
                up[d] += wA0;
                M[d][0] = add_steps(i - N0, M[d][0], wA0);
                M[d][1] = fmaf(wx, A1[d], M[d][1]);
                M[d][2] = fmaf(wx, A2[d], M[d][2]);
            }
        }
        float B[3][3];
#pragma unroll
        for (int d = 0; d < NU; ++d)
#pragma unroll
            for (int q = 0; q < 3; ++q)
                B[d][q] = fmaf((float)mp.dx[q], M[d][q], sp[q].d[N0] * up[d]);
        if constexpr (STAG) {
            // the gathered component belongs to column stag; the others are 0
            const float u0 = up[0], b0[3] = {B[0][0], B[0][1], B[0][2]};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const bool mine = d == A.stag;
                up[d] = mine ? u0 : 0.f;
#pragma unroll
                for (int q = 0; q < 3; ++q) B[d][q] = mine ? b0[q] : 0.f;
            }
        }
        // c_p(0, d) = u_p(d); c_p(1 + q, d) = B_p(d, q)  (APIC.hpp:464-471)
        float4* out = reinterpret_cast<float4*>(A.c + 12 * p);
        out[0] = make_float4(up[0], up[1], up[2], B[0][0]);
        out[1] = make_float4(B[1][0], B[2][0], B[0][1], B[1][1]);
        out[2] = make_float4(B[2][1], B[0][2], B[1][2], B[2][2]);
        if constexpr (ADV) {
            const double uo[3] = {(double)up[0], (double)up[1], (double)up[2]};
            advect_particle(A.adv, p, xp, uo, [&](int d, double v) { A.x_out[3 * p + d] = v; });
        }
    }
}

// host helpers (tiled.cu)
bool fused_update_fits(const TileP& tp, int order);
bool make_tilep(const MeshP& mp, int order, const picasso_bins& bins, TileP* tp, int lpp = 0,
                int nf = 4);
int device_smem_optin();
bool packed_x(const PField& x);
bool packed_m(const PField& m);
bool packed_c(const PField& c);
int default_lpp(int order);
bool valid_lpp(int order, int lpp, bool stag = false);
size_t p2g_warp_bytes(int order, int lpp, int P, bool rec = false, bool stag = false);

}  // namespace pb
