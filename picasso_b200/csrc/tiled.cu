// Shared-memory tiled APIC P2G / G2P (FP32 precision form) for particles
// sorted by picasso_cell_sort, on packed particle storage: x_p (N,3) FP64,
// m_p (N) FP32, c_p (N,4,3) FP32.
//
// Work items are chunks of at most `chunk` particles of one tile (the sort
// writes the per-tile item prefix).
//
// P2G (one single-warp CTA per item): every lane sweeps its own contiguous run of the
// item's particles -- sorted by bin, so consecutive particles mostly share a
// stencil -- and accumulates the 4 x K^3 mass / momentum contributions of its
// current bin in registers.  Particle records arrive through a per-lane
// cp.async ring in shared memory, a few particles ahead of use.  When a
// lane's bin changes it stages its partial sums and the warp adds the staged
// partials into the warp's node tile ((T + K - 1)^3 nodes, FP32) one lane
// after the other: a fixed order without atomics, so the tile sums are
// reproducible.  At the end of the item the touched part of the tile is
// rounded to 64-bit fixed point and added to HBM with integer reductions,
// whose result does not depend on their order.  P2G is therefore
// deterministic for a given particle order.
//
// G2P (one CTA per item): the item's node velocities are staged once in a
// CTA-shared tile (float4 per node) and every thread gathers its particles'
// stencils from there.
#include "common.cuh"
#include "transfer.cuh"

namespace pb {

constexpr int kWarps = 4;          // warps per CTA
constexpr int kStageLanes = 8;     // lanes staged per merge round
constexpr int kStageStride = 116;  // floats per staged lane (4 fields x 28 + pad;
                                   // 116 mod 32 = 20 keeps 8 float4 stores apart)
constexpr int kRing = 3;           // particles in flight per lane
// ring of particle records, one slot per lane and stage, in three arrays so
// that every access pattern is free of bank conflicts: x (3 doubles, 6-word
// lane stride), c (12 floats, 12-word stride), m (1 float)
constexpr int kRingX = 6, kRingC = 12;
constexpr int kRingFloats = 32 * (kRingX + kRingC + 1);
constexpr unsigned kFull = 0xFFFFFFFFu;

struct TileP {
    int T[3];    // bins per tile
    int nt[3];   // tiles per dimension
    int nb[3];   // bins per dimension
    int NT[3];   // nodes per tile dimension (T + K - 1)
    int nodes;   // NT0 * NT1 * NT2
    int SJ, SI;  // P2G node-tile strides along j and i (k stride 1), padded so
    int P;       // the 27 (64) stencil nodes of a merge hit distinct banks;
                 // P = stride between the 4 field planes
    int chunk;
    int64_t ntiles;
    const int64_t* off;     // tile particle offsets (ntiles + 1)
    const uint32_t* items;  // tile work-item prefix (ntiles + 1)
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
// cp.async helpers (Ampere-style asynchronous global -> shared copies)
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
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// ---------------------------------------------------------------------------
// P2G
// ---------------------------------------------------------------------------
template <int ORDER>
struct P2GAcc {
    static constexpr int K = SplineTraits<ORDER>::K;
    static constexpr int KKK = K * K * K;
    static constexpr int FS = (KKK + 3) & ~3;  // staged floats per field
    float am[KKK];
    float ap[KKK][3];

    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int n = 0; n < KKK; ++n) {
            am[n] = 0.f;
            ap[n][0] = ap[n][1] = ap[n][2] = 0.f;
        }
    }

    // One particle: APIC.hpp:110-139 (order 2/3) and :287-318 (order 1).
    __device__ __forceinline__ void add(const Spline1D<ORDER, float> sp[3], float mass,
                                        const float cp[12], float D)
    {
        // cp[r * 3 + d] = c_p(r, d)
        if (ORDER >= 2) {
            float DB[3][3];
#pragma unroll
            for (int d = 0; d < 3; ++d)
#pragma unroll
                for (int a = 0; a < 3; ++a) DB[d][a] = D * cp[(1 + a) * 3 + d];
#pragma unroll
            for (int i = 0; i < K; ++i)
#pragma unroll
                for (int j = 0; j < K; ++j) {
                    const float wij = sp[0].w[i] * sp[1].w[j] * mass;
                    float pij[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        pij[d] = cp[d] + DB[d][0] * sp[0].d[i] + DB[d][1] * sp[1].d[j];
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const int n = (i * K + j) * K + k;
                        const float w = wij * sp[2].w[k];
                        am[n] += w;
#pragma unroll
                        for (int d = 0; d < 3; ++d)
                            ap[n][d] += w * (pij[d] + DB[d][2] * sp[2].d[k]);
                    }
                }
        } else {
#pragma unroll
            for (int i = 0; i < K; ++i)
#pragma unroll
                for (int j = 0; j < K; ++j)
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const int n = (i * K + j) * K + k;
                        const float wm = sp[0].w[i] * sp[1].w[j] * sp[2].w[k] * mass;
                        const float g0 = sp[0].g[i] * sp[1].w[j] * sp[2].w[k] * mass;
                        const float g1 = sp[0].w[i] * sp[1].g[j] * sp[2].w[k] * mass;
                        const float g2 = sp[0].w[i] * sp[1].w[j] * sp[2].g[k] * mass;
                        am[n] += wm;
#pragma unroll
                        for (int d = 0; d < 3; ++d)
                            ap[n][d] += wm * cp[d] + cp[3 + d] * g0 + cp[6 + d] * g1 +
                                        cp[9 + d] * g2;
                    }
        }
    }

    __device__ __forceinline__ float field(int f, int n) const
    {
        return f == 0 ? am[n] : ap[n][f - 1];
    }

    __device__ __forceinline__ void stage(float* st) const
    {
#pragma unroll
        for (int f = 0; f < 4; ++f)
#pragma unroll
            for (int q = 0; q < FS / 4; ++q) {
                float4 v;
                v.x = (4 * q + 0 < KKK) ? field(f, 4 * q + 0) : 0.f;
                v.y = (4 * q + 1 < KKK) ? field(f, 4 * q + 1) : 0.f;
                v.z = (4 * q + 2 < KKK) ? field(f, 4 * q + 2) : 0.f;
                v.w = (4 * q + 3 < KKK) ? field(f, 4 * q + 3) : 0.f;
                *reinterpret_cast<float4*>(st + f * FS + 4 * q) = v;
            }
    }
};

// Merge plan of one lane: staged value v = lane + 32 r lands at tile offset
// moff[r] relative to the stencil start (or nowhere if the bit is clear).
template <int ORDER>
struct MergePlan {
    int moff[4];
    unsigned valid;
    __device__ __forceinline__ void init(const TileP& tp, int lane)
    {
        using A = P2GAcc<ORDER>;
        constexpr int K = A::K;
        valid = 0;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int v = lane + 32 * r;
            const int f = v / A::FS, nn = v - (v / A::FS) * A::FS;
            moff[r] = 0;
            if (v < 4 * A::FS && nn < A::KKK) {
                const int a = nn / (K * K), b = (nn / K) % K, c = nn % K;
                moff[r] = f * tp.P + a * tp.SI + b * tp.SJ + c;
                valid |= 1u << r;
            }
        }
    }
};

// Lanes in `mask` hand their partial sums to the warp's node tile in lane
// order; their accumulators are zeroed.
template <int ORDER>
__device__ __forceinline__ void merge_partials(unsigned mask, P2GAcc<ORDER>& acc, int cur_base,
                                               const MergePlan<ORDER>& plan, float* tile,
                                               float* stage, int* stage_base, int lane)
{
    while (mask) {
        unsigned batch = mask;
        if (__popc(mask) > kStageLanes) {  // lowest kStageLanes lanes
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
            acc.stage(stage + slot * kStageStride);
            stage_base[slot] = cur_base;
            acc.zero();
        }
        __syncwarp();
        const int nstage = __popc(batch);
        for (int q = 0; q < nstage; ++q) {
            const float* st = stage + q * kStageStride;
            const int base = stage_base[q];
#pragma unroll
            for (int r = 0; r < 4; ++r)
                if ((plan.valid >> r) & 1u) tile[base + plan.moff[r]] += st[lane + 32 * r];
            __syncwarp();
        }
    }
}

template <int ORDER>
__global__ void __launch_bounds__(32, 8)
p2g_tiled_kernel(MeshP mp, TileP tp, int64_t n, const double* __restrict__ xg,
                 const float* __restrict__ mg, const float* __restrict__ cg, GField gm, GField gmu,
                 float scale_m, float scale_mu, int* err)
{
    using A = P2GAcc<ORDER>;
    constexpr int K = A::K;
    // one warp per CTA: warps finish their items independently
    extern __shared__ __align__(16) float smem[];
    __shared__ int stage_base[kStageLanes];
    const int lane = threadIdx.x;
    float* ring = smem;  // [kRing][x: 32*6 | c: 32*12 | m: 32]
    float* stage = ring + kRing * kRingFloats;
    float* tile = stage + kStageLanes * kStageStride;

    if (blockIdx.x == 0 && threadIdx.x == 0 && err) {
        const int64_t n_valid = __ldg(tp.off + tp.ntiles);
        if (n > n_valid) atomicAdd(err, (int)(n - n_valid));
    }
    int64_t t, a, b;
    if (!item_range(tp, blockIdx.x, t, a, b)) return;
    int ob[3];
    tile_origin(tp, t, ob);
    const int U = (int)((b - a + 31) / 32);
    const int64_t my0 = a + (int64_t)lane * U;
    const int cnt = (int)max((int64_t)0, min(my0 + U, b) - my0);

    for (int i = lane; i < 4 * tp.P; i += 32) tile[i] = 0.f;
    MergePlan<ORDER> plan;
    plan.init(tp, lane);
    const float D = (ORDER >= 2) ? inertial_scaling<ORDER, float>(mp.dx[0]) : 0.f;

    auto slot_x = [&](int q) { return ring + (q % kRing) * kRingFloats + lane * kRingX; };
    auto slot_c = [&](int q) {
        return ring + (q % kRing) * kRingFloats + 32 * kRingX + lane * kRingC;
    };
    auto slot_m = [&](int q) {
        return ring + (q % kRing) * kRingFloats + 32 * (kRingX + kRingC) + lane;
    };
    auto issue = [&](int q) {
        if (q < cnt) {
            const int64_t p = my0 + q;
            float* sx = slot_x(q);
            float* sc = slot_c(q);
            cp_async<8>(sx + 0, xg + 3 * p + 0);
            cp_async<8>(sx + 2, xg + 3 * p + 1);
            cp_async<8>(sx + 4, xg + 3 * p + 2);
            cp_async<16>(sc + 0, cg + 12 * p + 0);
            cp_async<16>(sc + 4, cg + 12 * p + 4);
            cp_async<16>(sc + 8, cg + 12 * p + 8);
            cp_async<4>(slot_m(q), mg + p);
        }
        cp_async_commit();
    };
#pragma unroll
    for (int q = 0; q < kRing - 1; ++q) issue(q);
    __syncwarp();

    A acc;
    acc.zero();
    int cur = -1, cur_base = 0;
    int bmin[3] = {1 << 30, 1 << 30, 1 << 30}, bmax[3] = {-1, -1, -1};
    for (int s = 0; s < U; ++s) {
        __syncwarp();  // no lane still reads the slot refilled next
        issue(s + kRing - 1);
        cp_async_wait<kRing - 1>();
        const bool valid = s < cnt;
        Spline1D<ORDER, float> sp[3];
        int lb[3] = {0, 0, 0};
        bool ok = false;
        float cp[12], mass = 0.f;
        if (valid) {
            const double* sx = reinterpret_cast<const double*>(slot_x(s));
            const double xp[3] = {sx[0], sx[1], sx[2]};
            ok = locate<ORDER>(mp, tp, xp, ob, sp, lb);
            if (!ok && err) atomicAdd(err, 1);
            const float* sc = slot_c(s);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const float4 v = *reinterpret_cast<const float4*>(sc + 4 * q);
                cp[4 * q] = v.x;
                cp[4 * q + 1] = v.y;
                cp[4 * q + 2] = v.z;
                cp[4 * q + 3] = v.w;
            }
            mass = *slot_m(s);
        }
        const int lbin = ok ? (lb[0] * tp.T[1] + lb[1]) * tp.T[2] + lb[2] : -1;
        const unsigned fm = __ballot_sync(kFull, ok && cur >= 0 && lbin != cur);
        if (fm) merge_partials<ORDER>(fm, acc, cur_base, plan, tile, stage, stage_base, lane);
        if (ok) {
            if (lbin != cur) {
                cur = lbin;
                cur_base = lb[0] * tp.SI + lb[1] * tp.SJ + lb[2];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    bmin[d] = min(bmin[d], lb[d]);
                    bmax[d] = max(bmax[d], lb[d]);
                }
            }
            acc.add(sp, mass, cp, D);
        }
    }
    cp_async_wait<0>();
    const unsigned fm = __ballot_sync(kFull, cur >= 0);
    if (fm) merge_partials<ORDER>(fm, acc, cur_base, plan, tile, stage, stage_base, lane);
    // touched node box, rounded to fixed point and added to HBM
#pragma unroll
    for (int d = 0; d < 3; ++d) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            bmin[d] = min(bmin[d], __shfl_xor_sync(kFull, bmin[d], o));
            bmax[d] = max(bmax[d], __shfl_xor_sync(kFull, bmax[d], o));
        }
    }
    if (bmax[0] < 0) return;
    const int e0 = bmax[0] - bmin[0] + K, e1 = bmax[1] - bmin[1] + K, e2 = bmax[2] - bmin[2] + K;
    const int total = e0 * e1 * e2;
    for (int e = lane; e < total; e += 32) {
        const int k = bmin[2] + e % e2;
        const int j = bmin[1] + (e / e2) % e1;
        const int i = bmin[0] + e / (e1 * e2);
        const int idx = i * tp.SI + j * tp.SJ + k;
        const int gi = node_global(mp, tp, 0, ob[0], i);
        const int gj = node_global(mp, tp, 1, ob[1], j);
        const int gk = node_global(mp, tp, 2, ob[2], k);
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const float v = tile[f * tp.P + idx];
            if (v != 0.f) {
                const long long q = __float2ll_rn(v * (f == 0 ? scale_m : scale_mu));
                unsigned long long* dst = reinterpret_cast<unsigned long long*>(
                    f == 0 ? gm.ptr<long long>(gi, gj, gk, 0)
                           : gmu.ptr<long long>(gi, gj, gk, f - 1));
                atomicAdd(dst, (unsigned long long)q);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// G2P
// ---------------------------------------------------------------------------
template <int ORDER>
__global__ void __launch_bounds__(kWarps * 32)
g2p_tiled_kernel(MeshP mp, TileP tp, int64_t n, const double* __restrict__ xg, GField u,
                 float* __restrict__ cg, int* err)
{
    constexpr int K = SplineTraits<ORDER>::K;
    extern __shared__ __align__(16) float smem[];
    float4* tile = reinterpret_cast<float4*>(smem);

    if (blockIdx.x == 0 && threadIdx.x == 0 && err) {
        const int64_t n_valid = __ldg(tp.off + tp.ntiles);
        if (n > n_valid) atomicAdd(err, (int)(n - n_valid));
    }
    int64_t t, a, b;
    if (!item_range(tp, blockIdx.x, t, a, b)) return;  // CTA-uniform
    int ob[3];
    tile_origin(tp, t, ob);
    // bin rows spanned by the item: the first and last particle bound the
    // slowest tile dimension (keys are i-major within a tile)
    int i_lo = 0, i_hi = tp.T[0] - 1;
    {
        Spline1D<ORDER, float> sp[3];
        int lb[3];
        const double xa[3] = {xg[3 * a], xg[3 * a + 1], xg[3 * a + 2]};
        const double xb[3] = {xg[3 * (b - 1)], xg[3 * (b - 1) + 1], xg[3 * (b - 1) + 2]};
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
    for (int e = threadIdx.x; e < total; e += kWarps * 32) {
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
        if (inside) {
            v.x = __ldg(u.ptr<float>(gi, gj, gk, 0));
            v.y = __ldg(u.ptr<float>(gi, gj, gk, 1));
            v.z = __ldg(u.ptr<float>(gi, gj, gk, 2));
        }
        tile[(i * tp.NT[1] + j) * tp.NT[2] + k] = v;
    }
    __syncthreads();
    // positions are prefetched one particle ahead
    double xn[3] = {0.0, 0.0, 0.0};
    if (a + threadIdx.x < b) {
        const int64_t p0 = a + threadIdx.x;
        xn[0] = xg[3 * p0];
        xn[1] = xg[3 * p0 + 1];
        xn[2] = xg[3 * p0 + 2];
    }
    for (int64_t p = a + threadIdx.x; p < b; p += kWarps * 32) {
        const double xp[3] = {xn[0], xn[1], xn[2]};
        const int64_t pn = p + kWarps * 32;
        if (pn < b) {
            xn[0] = xg[3 * pn];
            xn[1] = xg[3 * pn + 1];
            xn[2] = xg[3 * pn + 2];
        }
        Spline1D<ORDER, float> sp[3];
        int lb[3];
        if (!locate<ORDER>(mp, tp, xp, ob, sp, lb) || lb[0] < i_lo || lb[0] > i_hi) {
            if (err) atomicAdd(err, 1);
            continue;
        }
        const int base = (lb[0] * tp.NT[1] + lb[1]) * tp.NT[2] + lb[2];
        // APIC.hpp:439-461, contracted one dimension at a time:
        //   u_p    = sum_i wx_i sum_j wy_j sum_k wz_k u_ijk
        //   B_p(:,q) = sum_ijk w_ijk u_ijk dist_q  (dist_q along x, y or z)
        float up[3] = {0.f, 0.f, 0.f};
        float B[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
        float wzdz[K];
#pragma unroll
        for (int k = 0; k < K; ++k) wzdz[k] = sp[2].w[k] * sp[2].d[k];
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
                    for (int d = 0; d < 3; ++d) {
                        S0[d] += sp[2].w[k] * uk[d];
                        S1[d] += wzdz[k] * uk[d];
                    }
                }
                const float wy = sp[1].w[j], wydy = wy * sp[1].d[j];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    A0[d] += wy * S0[d];
                    A1[d] += wydy * S0[d];
                    A2[d] += wy * S1[d];
                }
            }
            const float wx = sp[0].w[i], wxdx = wx * sp[0].d[i];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                up[d] += wx * A0[d];
                B[d][0] += wxdx * A0[d];
                B[d][1] += wx * A1[d];
                B[d][2] += wx * A2[d];
            }
        }
        // c_p(0, d) = u_p(d); c_p(1 + q, d) = B_p(d, q)  (APIC.hpp:464-471)
        float4* out = reinterpret_cast<float4*>(cg + 12 * p);
        out[0] = make_float4(up[0], up[1], up[2], B[0][0]);
        out[1] = make_float4(B[1][0], B[2][0], B[0][1], B[1][1]);
        out[2] = make_float4(B[2][1], B[0][2], B[1][2], B[2][2]);
    }
}

// ---------------------------------------------------------------------------
// host dispatch
// ---------------------------------------------------------------------------
// Padded node-tile strides for the P2G merge: value v = lane + 32 r of a
// staged lane (field v / FS, stencil node v % FS) lands at
// f * P + a * SI + b * SJ + c; pick the smallest padding that maximises the
// number of distinct banks per merge instruction.  Cached per tile shape.
static void choose_strides(const int NT[3], int K, int* SJ, int* SI, int* P)
{
    static thread_local int cache_key[5] = {-1, -1, -1, -1, -1};
    static thread_local int cache_val[3];
    if (cache_key[0] == NT[0] && cache_key[1] == NT[1] && cache_key[2] == NT[2] &&
        cache_key[3] == K) {
        *SJ = cache_val[0];
        *SI = cache_val[1];
        *P = cache_val[2];
        return;
    }
    const int KKK = K * K * K, FS = (KKK + 3) & ~3;
    int best = -1, bsj = NT[2], bsi = NT[1] * NT[2], bp = NT[0] * NT[1] * NT[2];
    long best_size = 0;
    for (int sj = NT[2]; sj < NT[2] + 8; ++sj)
        for (int si = NT[1] * sj; si < NT[1] * sj + 16; ++si)
            for (int pp = NT[0] * si; pp < NT[0] * si + 16; ++pp) {
                int distinct = 0;
                for (int r = 0; r < 4; ++r) {
                    unsigned banks = 0;
                    for (int lane = 0; lane < 32; ++lane) {
                        const int v = lane + 32 * r, f = v / FS, nn = v % FS;
                        if (v >= 4 * FS || nn >= KKK) continue;
                        const int a = nn / (K * K), b = (nn / K) % K, c = nn % K;
                        const int off = f * pp + a * si + b * sj + c;
                        const unsigned bit = 1u << (off & 31);
                        if (!(banks & bit)) ++distinct;
                        banks |= bit;
                    }
                }
                const long size = 4L * pp;
                if (distinct > best || (distinct == best && size < best_size)) {
                    best = distinct;
                    best_size = size;
                    bsj = sj;
                    bsi = si;
                    bp = pp;
                }
            }
    *SJ = bsj;
    *SI = bsi;
    *P = bp;
    cache_key[0] = NT[0];
    cache_key[1] = NT[1];
    cache_key[2] = NT[2];
    cache_key[3] = K;
    cache_val[0] = bsj;
    cache_val[1] = bsi;
    cache_val[2] = bp;
}

static bool make_tilep(const MeshP& mp, int order, const picasso_bins& bins, TileP* tp)
{
    const int K = order + 1;
    int64_t nt = 1;
    for (int d = 0; d < 3; ++d) {
        const int nb = mp.periodic[d] ? mp.own_n[d] : mp.ext[d];
        if (bins.bin_extent[d] != nb || bins.tile[d] < 1) return false;
        if (bins.num_tiles[d] != (nb + bins.tile[d] - 1) / bins.tile[d]) return false;
        tp->T[d] = bins.tile[d];
        tp->nt[d] = bins.num_tiles[d];
        tp->nb[d] = nb;
        tp->NT[d] = bins.tile[d] + K - 1;
        nt *= bins.num_tiles[d];
    }
    tp->nodes = tp->NT[0] * tp->NT[1] * tp->NT[2];
    choose_strides(tp->NT, K, &tp->SJ, &tp->SI, &tp->P);
    tp->ntiles = nt;
    tp->off = bins.tile_offset;
    tp->items = bins.tile_items;
    tp->chunk = bins.chunk;
    return bins.tile_offset && bins.tile_items && bins.chunk >= 32;
}

static int device_smem_optin()
{
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

// Packed storage the tiled kernels read: x (N,3) FP64, m (N) FP32, c (N,12)
// FP32 with 16-byte aligned rows.
static bool packed_x(const PField& x)
{
    return x.shift == 0 && x.tile_stride == 3 && x.comp_stride == 1 &&
           (reinterpret_cast<uintptr_t>(x.data) % 8) == 0;
}
static bool packed_m(const PField& m)
{
    return (m.shift == 0 && m.tile_stride == 1) || m.shift == 63;
}
static bool packed_c(const PField& c)
{
    return c.shift == 0 && c.tile_stride == 12 && c.comp_stride == 1 &&
           (reinterpret_cast<uintptr_t>(c.data) % 16) == 0;
}

static int64_t item_bound(const TileP& tp, int64_t n)
{
    return tp.ntiles + (n + tp.chunk - 1) / tp.chunk;
}

template <int ORDER>
static size_t p2g_smem(const TileP& tp)
{
    return sizeof(float) *
           ((size_t)kRing * kRingFloats + kStageLanes * kStageStride + 4 * (size_t)tp.P);
}

template <int ORDER>
static picasso_status launch_p2g_tiled(const MeshP& mp, const TileP& tp, int64_t n,
                                       const PField& x, const PField& m, const PField& c,
                                       const GField& gm, const GField& gmu, int* err,
                                       cudaStream_t st)
{
    const size_t smem = p2g_smem<ORDER>(tp);
    PB_CUDA_TRY(cudaFuncSetAttribute(p2g_tiled_kernel<ORDER>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t items = item_bound(tp, n);
    p2g_tiled_kernel<ORDER><<<(unsigned)(items ? items : 1), 32, smem, st>>>(
        mp, tp, n, reinterpret_cast<const double*>(x.data), reinterpret_cast<const float*>(m.data),
        reinterpret_cast<const float*>(c.data), gm, gmu, ldexpf(1.f, gm.fixed_bits),
        ldexpf(1.f, gmu.fixed_bits), err);
    return check_launch();
}

template <int ORDER>
static picasso_status launch_g2p_tiled(const MeshP& mp, const TileP& tp, int64_t n,
                                       const PField& x, const GField& u, const PField& c,
                                       int* err, cudaStream_t st)
{
    const size_t smem = sizeof(float4) * (size_t)tp.nodes;
    PB_CUDA_TRY(cudaFuncSetAttribute(g2p_tiled_kernel<ORDER>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t items = item_bound(tp, n);
    g2p_tiled_kernel<ORDER><<<(unsigned)(items ? items : 1), kWarps * 32, smem, st>>>(
        mp, tp, n, reinterpret_cast<const double*>(x.data), u, reinterpret_cast<float*>(c.data),
        err);
    return check_launch();
}

picasso_status apic_p2g_tiled(const MeshP& mp, int order, int ncomp, Form form, int64_t n,
                              const PField& x, const PField& m, const PField& c, const GField& gm,
                              const GField& gmu, const picasso_bins& bins, int* err,
                              cudaStream_t st, bool* handled)
{
    *handled = false;
    if (form != Form::F32Fixed || ncomp != 3 || order > 2 || !packed_x(x) || !packed_m(m) ||
        !packed_c(c))
        return PICASSO_OK;
    TileP tp;
    if (!make_tilep(mp, order, bins, &tp)) return PICASSO_ERR_INVALID_ARGUMENT;
    const size_t smem = order == 1 ? p2g_smem<1>(tp) : p2g_smem<2>(tp);
    if ((int64_t)smem > device_smem_optin()) return PICASSO_OK;  // tile too large: plain path
    *handled = true;
    if (order == 1) return launch_p2g_tiled<1>(mp, tp, n, x, m, c, gm, gmu, err, st);
    return launch_p2g_tiled<2>(mp, tp, n, x, m, c, gm, gmu, err, st);
}

picasso_status apic_g2p_tiled(const MeshP& mp, int order, int ncomp, bool f32, int64_t n,
                              const PField& x, const GField& u, const PField& c,
                              const picasso_bins& bins, int* err, cudaStream_t st, bool* handled)
{
    *handled = false;
    if (!f32 || ncomp != 3 || !packed_x(x) || !packed_c(c)) return PICASSO_OK;
    TileP tp;
    if (!make_tilep(mp, order, bins, &tp)) return PICASSO_ERR_INVALID_ARGUMENT;
    const size_t smem = sizeof(float4) * (size_t)tp.nodes;
    if ((int64_t)smem > device_smem_optin()) return PICASSO_OK;
    *handled = true;
    if (order == 1) return launch_g2p_tiled<1>(mp, tp, n, x, u, c, err, st);
    if (order == 2) return launch_g2p_tiled<2>(mp, tp, n, x, u, c, err, st);
    return launch_g2p_tiled<3>(mp, tp, n, x, u, c, err, st);
}

}  // namespace pb
