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
#include "tiled.cuh"
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
// Spline and stencil indices of a particle on the whole local mesh (periodic
// wrap, bounds check): the placement of the plain kernels.
template <int ORDER, class R>
struct MeshPlace {
    const MeshP& mp;
    __device__ __forceinline__ bool operator()(const double xp[3], Spline1D<ORDER, R> sp[3],
                                               int idx[3][SplineTraits<ORDER>::K]) const
    {
        bool ok = true;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            eval_spline<ORDER>(xp[d], mp.lo[d], mp.dx[d], mp.rdx[d], sp[d]);
            ok = ok && resolve_stencil<SplineTraits<ORDER>::K>(mp, d, sp[d].s0, idx[d]);
        }
        return ok;
    }
};

// One particle.  place(xp, sp, idx) evaluates the spline and the stencil's
// grid indices (false: skip the particle); acc(f, i, j, k, v) adds v to grid
// field f (0 mass, 1 + d momentum component d); mode(v) returns c_p value v
// (element v of the particle's record).
template <int ORDER, int NC, bool STAG, class PT, class R, class Place, class Acc, class Mode>
__device__ __forceinline__ void polypic_p2g_particle(const MeshP& mp, int64_t p, const PField& x,
                                                     const PField& m, const PField& u, R dt,
                                                     int col, int* err, Place&& place, Acc&& acc,
                                                     Mode&& mode)
{
    constexpr int K = SplineTraits<ORDER>::K;
    {
        Spline1D<ORDER, R> sp[3];
        int idx[3][K];
        const double xp[3] = {x.get<double>(p, 0), x.get<double>(p, 1), x.get<double>(p, 2)};
        if (!place(xp, sp, idx)) {
            if (err) atomicAdd(err, 1);
            return;
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
            // loop over the modes: their degrees fold to constants
#pragma unroll
            for (int r = 0; r < D * D * D; ++r)
#pragma unroll
                for (int e = 0; e < CB; ++e)
                    cp[mode_deg(r, 0)][mode_deg(r, 1)][mode_deg(r, 2)][e] =
                        (R)mode(r * ncp + (STAG ? col : d0 + e));
            // quadratic: i-planes one after the other, not unrolled (bounds the
            // live range of the 9-node plane bodies, which spill in FP64, and
            // the code size, whose instruction-cache misses stalled the FP32
            // kernel: 6.55 -> 5.50 ms at 128^3 8 ppc)
#pragma unroll(ORDER == 2 ? 1 : K)
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
                            acc(1 + d0 + e, gi, idx[1][j], idx[2][k], wm * sa);
                        }
                        if (d0 == 0) acc(0, gi, idx[1][j], idx[2][k], wm);
                    }
            }
        }
    }
}

// Modes per particle record (c_p rows): 8 linear, 27 quadratic.
template <int ORDER>
struct PPModes {
    static constexpr int value = ORDER == 1 ? 8 : 27;
};

// Shared-memory records of a warp's 32 consecutive particles (packed c_p of
// NV values each, at an odd stride so that the 32 lanes' records start on
// distinct banks): the warp writes every particle's record with coalesced
// stores instead of NV strided stores per thread.
template <class PT, int NV>
struct WarpRecords {
    static constexpr int NVP = NV | 1;
    PT* buf;
    static constexpr size_t kBytesPerWarp = sizeof(PT) * 32 * NVP;
    __device__ __forceinline__ PT& at(int lane, int v) const { return buf[lane * NVP + v]; }
    // records of the particles in `mask` (bit q: particle p0 + q) to packed
    // storage
    __device__ __forceinline__ void store(PT* dst, int cnt, unsigned mask, int lane) const
    {
        __syncwarp();
        for (int e = lane; e < cnt * NV; e += 32) {
            const int q = e / NV;
            if ((mask >> q) & 1u) dst[e] = buf[q * NVP + (e - q * NV)];
        }
        __syncwarp();
    }
};

template <int ORDER, int NC, bool STAG, class PT, class R, class ACC>
__global__ void __launch_bounds__(128)
polypic_p2g_kernel(MeshP mp, int64_t n, PField x, PField m, PField u, PField c, GField gmu,
                   GField gm, R dt, int col, R scale_mu, R scale_m, int* err)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const MeshPlace<ORDER, R> place{mp};
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride)
        polypic_p2g_particle<ORDER, NC, STAG, PT, R>(
            mp, p, x, m, u, dt, col, err, place,
            [&](int f, int i, int j, int k, R v) {
                if (f == 0) ACC::add(gm, i, j, k, 0, v, scale_m);
                else ACC::add(gmu, i, j, k, f - 1, v, scale_mu);
            },
            [&](int v) { return c.get<PT>(p, v); });
}

// ---------------------------------------------------------------------------
// G2P: PolyPIC.hpp:236-293 (collocated) and :300-358 (staggered)
// ---------------------------------------------------------------------------
// One particle; emit(v, value) receives c_p value v (element v of the
// particle's record).  False if the particle was skipped (stencil outside a
// non-periodic mesh): then nothing is emitted.
// place: as for polypic_p2g_particle; grid(i, j, k, c) returns component c
// of u at stencil indices (i, j, k).
template <int ORDER, int NC, bool STAG, class PT, class R, class Place, class Grid, class Emit>
__device__ __forceinline__ bool polypic_g2p_particle(const MeshP& mp, int64_t p, const PField& x,
                                                     int col, int* err, Place&& place,
                                                     Grid&& grid, Emit&& emit)
{
    constexpr int K = SplineTraits<ORDER>::K;
    constexpr int NCU = STAG ? 1 : NC;
    {
        Spline1D<ORDER, R> sp[3];
        int idx[3][K];
        const double xp[3] = {x.get<double>(p, 0), x.get<double>(p, 1), x.get<double>(p, 2)};
        if (!place(xp, sp, idx)) {
            if (err) atomicAdd(err, 1);
            return false;
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
                            ue[k][e] = grid(idx[0][i], idx[1][j], idx[2][k], d0 + e);
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
            for (int r = 0; r < D * D * D; ++r)
#pragma unroll
                for (int e = 0; e < CB; ++e)
                    emit(r * ncp + (STAG ? col : d0 + e),
                         (PT)cp[mode_deg(r, 0)][mode_deg(r, 1)][mode_deg(r, 2)][e]);
        }
    }
    return true;
}

// WS: c_p is packed (the record of particle p at element p * NV) and written
// through WarpRecords; the lanes of a warp take consecutive particles and
// iterate together.
template <int ORDER, int NC, bool STAG, class GT, class PT, class R, bool WS>
__global__ void __launch_bounds__(128)
polypic_g2p_kernel(MeshP mp, int64_t n, PField x, GField u, PField c, int col, int* err)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const MeshPlace<ORDER, R> place{mp};
    auto grid = [&](int i, int j, int k, int cc) { return (R)__ldg(u.ptr<GT>(i, j, k, cc)); };
    if constexpr (!WS) {
        for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride)
            polypic_g2p_particle<ORDER, NC, STAG, PT, R>(
                mp, p, x, col, err, place, grid, [&](int v, PT val) { c.set<PT>(p, v, val); });
    } else {
        constexpr int NV = PPModes<ORDER>::value * NC;
        extern __shared__ __align__(16) unsigned char pp_smem[];
        const int lane = threadIdx.x & 31;
        const WarpRecords<PT, NV> rec{reinterpret_cast<PT*>(pp_smem) +
                                      (threadIdx.x >> 5) * 32 * WarpRecords<PT, NV>::NVP};
        PT* cbase = reinterpret_cast<PT*>(c.data);
        for (int64_t p0 = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); p0 < n;
             p0 += stride) {
            const int cnt = (int)min((int64_t)32, n - p0);
            bool wrote = false;
            if (lane < cnt)
                wrote = polypic_g2p_particle<ORDER, NC, STAG, PT, R>(
                    mp, p0 + lane, x, col, err, place, grid,
                    [&](int v, PT val) { rec.at(lane, v) = val; });
            rec.store(cbase + p0 * NV, cnt, __ballot_sync(0xFFFFFFFFu, wrote), lane);
        }
    }
}

// c_p stored packed: the record of particle p (all modes and components) at
// element p * NV, 16-byte aligned.
template <int ORDER, int NC, class PT>
static bool packed_record(const PField& c)
{
    constexpr int NV = PPModes<ORDER>::value * NC;
    return c.shift == 0 && c.tile_stride == NV && c.comp_stride == 1 &&
           reinterpret_cast<uintptr_t>(c.data) % 16 == 0;
}

// ---------------------------------------------------------------------------
// Tiled FP32-form kernels (cell-sorted particles, one 128-thread CTA per work
// item of the bins)
// ---------------------------------------------------------------------------
// Placement inside a tile: the spline of the plain FP32 form and the stencil
// in tile-local node indices; false if the particle is not in this tile.
template <int ORDER>
struct TilePlace {
    const MeshP& mp;
    const TileP& tp;
    const int* ob;
    __device__ __forceinline__ bool operator()(const double xp[3], Spline1D<ORDER, float> sp[3],
                                               int idx[3][SplineTraits<ORDER>::K]) const
    {
        int lb[3];
        if (!locate<ORDER>(mp, tp, xp, ob, sp, lb)) return false;
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int q = 0; q < SplineTraits<ORDER>::K; ++q) idx[d][q] = lb[d] + q;
        return true;
    }
};

__device__ __forceinline__ void count_unsorted(const TileP& tp, int64_t n, int* err)
{
    // particles sorted past the last tile (outside the mesh) belong to no item
    if (blockIdx.x == 0 && threadIdx.x == 0 && err) {
        const int64_t n_valid = __ldg(tp.off + tp.ntiles);
        if (n > n_valid) atomicAdd(err, (int)(n - n_valid));
    }
}

// P2G: the item's contributions are rounded to 64-bit fixed point exactly as
// the plain kernel rounds them and summed in a shared-memory node tile with
// 32-bit integer atomics, either on three slices of each value (q = hi 2^32 +
// mid 2^16 + lo with mid, lo in [0, 2^16): the lo and mid sums of at most
// 65536 contributions are exact, the hi sum is exact modulo 2^32) or on two
// words (the low word's carries, read from the atomics' old values, added to
// the high word), so the recombined 64-bit total equals the sum of the q
// modulo 2^64; then the tile is added to the grid.  Integer sums do not
// depend on their order: the grid is bit-identical to the plain kernel's
// (which adds every contribution to the grid), with one grid atomic per
// touched node and field per item instead of per particle and node.
// Quadratic: 3 CTAs per SM (168 registers, 44 bytes of spills) instead of 2 at
// 255 registers: 27 modes at 128^3 8 ppc 6.24 -> 5.85 ms.
template <int ORDER, int NC>
__global__ void __launch_bounds__(128, ORDER == 2 ? 3 : 1)
polypic_p2g_tiled_kernel(MeshP mp, TileP tp, int64_t n, PField x, PField m, PField u, PField c,
                         GField gmu, GField gm, float dt, float scale_mu, float scale_m, int* err)
{
    extern __shared__ __align__(16) unsigned int pp_tacc[];  // 3 slices x (1 + NC) x nodes
    count_unsorted(tp, n, err);
    int64_t t, a, b;
    if (!item_range(tp, blockIdx.x, t, a, b)) return;  // CTA-uniform
    // linear stencils (consecutive particles per warp): two words per value,
    // the low word's carry found from the atomic's old value and added to
    // the high word (2.11 -> 1.52 ms at 128^3 8 ppc); quadratic stencils (a
    // run per thread): three slices without returned values (the returning
    // atomic measured 6.20 -> 7.27 ms there)
    constexpr bool TWO = ORDER == 1;
    const int nodes = tp.nodes, slice = (1 + NC) * nodes;
    for (int e = threadIdx.x; e < (TWO ? 2 : 3) * slice; e += blockDim.x) pp_tacc[e] = 0u;
    __syncthreads();
    int ob[3];
    tile_origin(tp, t, ob);
    const TilePlace<ORDER> place{mp, tp, ob};
    // Quadratic: each thread sweeps its own contiguous run of the item, so
    // that the lanes of a warp sit in different cells and their tile atomics
    // rarely hit the same node (128^3 8 ppc: 6.5 ms instead of 9.1 ms with
    // consecutive particles per warp).  Linear (8 nodes, little arithmetic)
    // keeps consecutive particles per warp for coalesced loads (2.1 vs 2.5 ms).
    const int64_t U = ORDER == 2 ? (b - a + blockDim.x - 1) / blockDim.x : 1;
    const int64_t r0 = ORDER == 2 ? a + (int64_t)threadIdx.x * U : a + threadIdx.x;
    const int64_t r1 = ORDER == 2 ? min(r0 + U, b) : b;
    const int64_t step = ORDER == 2 ? 1 : blockDim.x;
    for (int64_t p = r0; p < r1; p += step)
        polypic_p2g_particle<ORDER, NC, false, float, float>(
            mp, p, x, m, u, dt, -1, err, place,
            [&](int f, int i, int j, int k, float v) {
                const long long q = to_fixed(f == 0 ? gm : gmu, v * (f == 0 ? scale_m : scale_mu));
                const int e = f * nodes + (i * tp.NT[1] + j) * tp.NT[2] + k;
                if constexpr (TWO) {
                    const unsigned long long uq = (unsigned long long)q;
                    const unsigned lo = (unsigned)uq;
                    const unsigned old = atomicAdd(&pp_tacc[e], lo);
                    const unsigned hi = (unsigned)(uq >> 32) + (old + lo < old ? 1u : 0u);
                    if (hi) atomicAdd(&pp_tacc[slice + e], hi);
                } else {
                    atomicAdd(&pp_tacc[e], (unsigned int)(q & 0xFFFF));
                    atomicAdd(&pp_tacc[slice + e], (unsigned int)((q >> 16) & 0xFFFF));
                    atomicAdd(&pp_tacc[2 * slice + e], (unsigned int)(q >> 32));
                }
            },
            [&](int v) { return c.get<float>(p, v); });
    __syncthreads();
    for (int e = threadIdx.x; e < nodes; e += blockDim.x) {
        const int k = e % tp.NT[2], j = (e / tp.NT[2]) % tp.NT[1], i = e / (tp.NT[1] * tp.NT[2]);
        const int gi = node_global(mp, tp, 0, ob[0], i);
        const int gj = node_global(mp, tp, 1, ob[1], j);
        const int gk = node_global(mp, tp, 2, ob[2], k);
#pragma unroll
        for (int f = 0; f <= NC; ++f) {
            const int q = f * nodes + e;
            const unsigned long long v =
                TWO ? ((unsigned long long)pp_tacc[slice + q] << 32) + (unsigned long long)pp_tacc[q]
                    : ((unsigned long long)pp_tacc[2 * slice + q] << 32) +
                          ((unsigned long long)pp_tacc[slice + q] << 16) +
                          (unsigned long long)pp_tacc[q];
            if (v)
                atomicAdd(reinterpret_cast<unsigned long long*>(
                              f == 0 ? gm.ptr<long long>(gi, gj, gk, 0)
                                     : gmu.ptr<long long>(gi, gj, gk, f - 1)),
                          v);
        }
    }
}

// G2P: the tile's node velocities are staged once per item in shared memory;
// packed c_p records leave through WarpRecords.
template <int ORDER, int NC, bool WS>
__global__ void __launch_bounds__(128)
polypic_g2p_tiled_kernel(MeshP mp, TileP tp, int64_t n, PField x, GField u, PField c, int* err)
{
    extern __shared__ __align__(16) unsigned char pp_smem[];
    float4* tile = reinterpret_cast<float4*>(pp_smem);
    count_unsorted(tp, n, err);
    int64_t t, a, b;
    if (!item_range(tp, blockIdx.x, t, a, b)) return;  // CTA-uniform
    int ob[3];
    tile_origin(tp, t, ob);
    for (int e = threadIdx.x; e < tp.nodes; e += blockDim.x) {
        const int k = e % tp.NT[2], j = (e / tp.NT[2]) % tp.NT[1], i = e / (tp.NT[1] * tp.NT[2]);
        const int gi = node_global(mp, tp, 0, ob[0], i);
        const int gj = node_global(mp, tp, 1, ob[1], j);
        const int gk = node_global(mp, tp, 2, ob[2], k);
        const bool inside = (mp.periodic[0] || gi < mp.ext[0]) &&
                            (mp.periodic[1] || gj < mp.ext[1]) &&
                            (mp.periodic[2] || gk < mp.ext[2]);
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (inside) {
            v.x = __ldg(u.ptr<float>(gi, gj, gk, 0));
            if (NC > 1) v.y = __ldg(u.ptr<float>(gi, gj, gk, 1));
            if (NC > 2) v.z = __ldg(u.ptr<float>(gi, gj, gk, 2));
        }
        tile[e] = v;
    }
    __syncthreads();
    const TilePlace<ORDER> place{mp, tp, ob};
    auto grid = [&](int i, int j, int k, int cc) {
        const float4 v = tile[(i * tp.NT[1] + j) * tp.NT[2] + k];
        return cc == 0 ? v.x : (cc == 1 ? v.y : v.z);
    };
    if constexpr (!WS) {
        for (int64_t p = a + threadIdx.x; p < b; p += blockDim.x)
            polypic_g2p_particle<ORDER, NC, false, float, float>(
                mp, p, x, -1, err, place, grid, [&](int v, float val) { c.set<float>(p, v, val); });
    } else {
        constexpr int NV = PPModes<ORDER>::value * NC;
        const int lane = threadIdx.x & 31;
        const WarpRecords<float, NV> rec{
            reinterpret_cast<float*>(pp_smem + ((sizeof(float4) * tp.nodes + 15) & ~size_t(15))) +
            (threadIdx.x >> 5) * 32 * WarpRecords<float, NV>::NVP};
        float* cbase = reinterpret_cast<float*>(c.data);
        for (int64_t p0 = a + (threadIdx.x & ~31); p0 < b; p0 += blockDim.x) {
            const int cnt = (int)min((int64_t)32, b - p0);
            bool wrote = false;
            if (lane < cnt)
                wrote = polypic_g2p_particle<ORDER, NC, false, float, float>(
                    mp, p0 + lane, x, -1, err, place, grid,
                    [&](int v, float val) { rec.at(lane, v) = val; });
            rec.store(cbase + p0 * NV, cnt, __ballot_sync(0xFFFFFFFFu, wrote), lane);
        }
    }
}

template <int ORDER, int NC>
static picasso_status launch_pp_p2g_tiled(const MeshP& mp, const TileP& tp, int64_t n,
                                          const PField& x, const PField& m, const PField& u,
                                          const PField& c, const GField& gmu, const GField& gm,
                                          double dt, int* err, cudaStream_t st)
{
    const size_t smem = 3 * sizeof(unsigned int) * (1 + NC) * (size_t)tp.nodes;
    auto kern = polypic_p2g_tiled_kernel<ORDER, NC>;
    PB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t items = tp.ntiles + (n + tp.chunk - 1) / tp.chunk;
    kern<<<(unsigned)items, 128, smem, st>>>(mp, tp, n, x, m, u, c, gmu, gm, (float)dt,
                                             ldexpf(1.f, gmu.fixed_bits), ldexpf(1.f, gm.fixed_bits),
                                             err);
    return check_launch();
}

template <int ORDER, int NC>
static picasso_status launch_pp_g2p_tiled(const MeshP& mp, const TileP& tp, int64_t n,
                                          const PField& x, const GField& u, const PField& c,
                                          int* err, cudaStream_t st)
{
    constexpr int NV = PPModes<ORDER>::value * NC;
    const bool ws = packed_record<ORDER, NC, float>(c);
    const size_t smem = ((sizeof(float4) * tp.nodes + 15) & ~size_t(15)) +
                        (ws ? 4 * WarpRecords<float, NV>::kBytesPerWarp : 0);
    const int64_t items = tp.ntiles + (n + tp.chunk - 1) / tp.chunk;
    if (ws) {
        auto kern = polypic_g2p_tiled_kernel<ORDER, NC, true>;
        PB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<(unsigned)items, 128, smem, st>>>(mp, tp, n, x, u, c, err);
    } else {
        auto kern = polypic_g2p_tiled_kernel<ORDER, NC, false>;
        PB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<(unsigned)items, 128, smem, st>>>(mp, tp, n, x, u, c, err);
    }
    return check_launch();
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
// Launches `kernel` with warp-staged records (dynamic shared memory of four
// warps' records) or without.
template <class PT, int NV, class Kern, class... Args>
static void launch_staged(Kern kernel, bool ws, unsigned blocks, cudaStream_t st, Args... args)
{
    const size_t smem = ws ? 4 * WarpRecords<PT, NV>::kBytesPerWarp : 0;
    if (ws) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kernel<<<blocks, 128, smem, st>>>(args...);
}

template <int ORDER, int NC, bool STAG, class PT, class R, class ACC>
static void launch_pp_p2g_form(const MeshP& mp, int64_t n, const PField& x, const PField& m,
                               const PField& u, const PField& c, const GField& gmu,
                               const GField& gm, R dt, int col, R smu, R sm, int* err,
                               cudaStream_t st)
{
    const unsigned blocks = grid_for(n, 128, 148LL * 128);
    polypic_p2g_kernel<ORDER, NC, STAG, PT, R, ACC><<<blocks, 128, 0, st>>>(
        mp, n, x, m, u, c, gmu, gm, dt, col, smu, sm, err);
}

template <int ORDER, int NC, bool STAG>
static void launch_pp_p2g(int form, const MeshP& mp, int64_t n, const PField& x, const PField& m,
                          const PField& u, const PField& c, const GField& gmu, const GField& gm,
                          double dt, int col, int* err, cudaStream_t st)
{
    if (form == 0)
        launch_pp_p2g_form<ORDER, NC, STAG, double, double, AccF64>(
            mp, n, x, m, u, c, gmu, gm, dt, col, 0.0, 0.0, err, st);
    else if (form == 1)
        launch_pp_p2g_form<ORDER, NC, STAG, float, float, AccFixed>(
            mp, n, x, m, u, c, gmu, gm, (float)dt, col, ldexpf(1.0f, gmu.fixed_bits),
            ldexpf(1.0f, gm.fixed_bits), err, st);
    else
        launch_pp_p2g_form<ORDER, NC, STAG, double, double, AccFixed>(
            mp, n, x, m, u, c, gmu, gm, dt, col, ldexp(1.0, gmu.fixed_bits),
            ldexp(1.0, gm.fixed_bits), err, st);
}

template <int ORDER, int NC, bool STAG, class T>
static void launch_pp_g2p_form(const MeshP& mp, int64_t n, const PField& x, const GField& u,
                               const PField& c, int col, int* err, cudaStream_t st)
{
    constexpr int NV = PPModes<ORDER>::value * NC;
    const unsigned blocks = grid_for(n, 128, 148LL * 128);
    if (!STAG && packed_record<ORDER, NC, T>(c))
        launch_staged<T, NV>(polypic_g2p_kernel<ORDER, NC, STAG, T, T, T, true>, true, blocks, st,
                             mp, n, x, u, c, col, err);
    else
        launch_staged<T, NV>(polypic_g2p_kernel<ORDER, NC, STAG, T, T, T, false>, false, blocks,
                             st, mp, n, x, u, c, col, err);
}

template <int ORDER, int NC, bool STAG>
static void launch_pp_g2p(bool f32, const MeshP& mp, int64_t n, const PField& x, const GField& u,
                          const PField& c, int col, int* err, cudaStream_t st)
{
    if (f32) launch_pp_g2p_form<ORDER, NC, STAG, float>(mp, n, x, u, c, col, err, st);
    else launch_pp_g2p_form<ORDER, NC, STAG, double>(mp, n, x, u, c, col, err, st);
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

// Tiled path for sorted particles (picasso_exec.bins): FP32 form, collocated
// locations; the bins must match the spline.  *tiled stays false (plain
// kernels) when not eligible or when the node tile of `node_bytes` per node
// does not fit in shared memory.
static picasso_status polypic_tiles(const picasso_spline* sd, const picasso_exec* exec,
                                    bool eligible, const MeshP& mp, int node_bytes, bool* tiled,
                                    TileP* tp)
{
    *tiled = false;
    if (!exec || !exec->bins) return PICASSO_OK;
    if (exec->bins->order != sd->order || exec->bins->location != sd->location)
        return PICASSO_ERR_INVALID_ARGUMENT;
    if (!eligible) return PICASSO_OK;
    if (!make_tilep(mp, sd->order, *exec->bins, tp)) return PICASSO_ERR_INVALID_ARGUMENT;
    // records of four warps on top of the node tile in the G2P (at most)
    const int64_t extra = 4 * 32 * 82 * 4;
    if ((int64_t)node_bytes * tp->nodes + extra > device_smem_optin()) return PICASSO_OK;
    *tiled = true;
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
    gmu.overflow = gm.overflow = exec ? exec->overflow_count : nullptr;
    bool tiled = false;
    TileP tp;
    // (the tile's 32-bit slice sums are exact for work items of at most
    // 65536 particles)
    const bool p2g_ok = form == 1 && stag < 0 && exec && exec->bins && exec->bins->chunk <= 65536;
    if ((st = polypic_tiles(sd, exec, p2g_ok, mp, 12 * (1 + ncomp), &tiled, &tp))) return st;
    if (tiled) {
        if (sd->order == 1) {
            PB_PP_NC_SWITCH(ncomp, return launch_pp_p2g_tiled<1, NC_>(mp, tp, num_particles, x, m,
                                                                      u, c, gmu, gm, dt, err, s));
        } else {
            PB_PP_NC_SWITCH(ncomp, return launch_pp_p2g_tiled<2, NC_>(mp, tp, num_particles, x, m,
                                                                      u, c, gmu, gm, dt, err, s));
        }
    }
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
    bool tiled = false;
    TileP tp;
    if ((st = polypic_tiles(sd, exec, f32 && stag < 0, mp, 16, &tiled, &tp))) return st;
    if (tiled) {
        if (sd->order == 1) {
            PB_PP_NC_SWITCH(ncomp, return launch_pp_g2p_tiled<1, NC_>(mp, tp, num_particles, x, u,
                                                                      c, err, s));
        } else {
            PB_PP_NC_SWITCH(ncomp, return launch_pp_g2p_tiled<2, NC_>(mp, tp, num_particles, x, u,
                                                                      c, err, s));
        }
    }
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
