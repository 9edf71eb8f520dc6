// Particle cell-sort: key = (tile, bin in tile) of the particle's stencil
// start, then a stable LSD radix sort of (key, particle index) pairs, then
// per-tile particle offsets.  Also the member gather used to apply the
// permutation to particle storage.
//
// Radix pass (digit width <= 9 bits): a histogram kernel counts the digits
// of each 2048-element block, a device-wide exclusive scan turns the
// digit-major [digit][block] count table into output offsets, and the
// scatter kernel ranks each element among equal digits of its block in
// original order (warp __match_any_sync + a per-warp running count, then a
// prefix over the block's warps), so every pass is stable.
#include <cmath>

#include "binkey.cuh"

namespace pb {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // elements per block
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kMaxDigitBits = 9;
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void key_kernel(BinP bp, int64_t n, PField x, uint32_t* __restrict__ keys,
                           uint32_t* __restrict__ vals)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const double xs[3] = {x.get<double>(p, 0), x.get<double>(p, 1), x.get<double>(p, 2)};
        keys[p] = particle_key(bp, xs);
        vals[p] = (uint32_t)p;
    }
}

__global__ void __launch_bounds__(kSortThreads)
radix_hist_kernel(const uint32_t* __restrict__ keys, int64_t n, int shift, int bits,
                  uint32_t* __restrict__ hist, int64_t nblk, uint32_t kmax)
{
    __shared__ uint32_t cnt[1 << kMaxDigitBits];
    const int nd = 1 << bits;
    const uint32_t mask = (uint32_t)nd - 1;
    for (int i = threadIdx.x; i < nd; i += kSortThreads) cnt[i] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const int64_t e = base + (int64_t)r * kSortThreads + threadIdx.x;
        const bool valid = e < n;
        const uint32_t dig = valid ? (min(__ldg(keys + e), kmax) >> shift) & mask : 0xFFFFFFFFu;
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, dig);
        if (valid && lane == __ffs(peers) - 1) atomicAdd(&cnt[dig], (uint32_t)__popc(peers));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nd; i += kSortThreads) hist[(int64_t)i * nblk + blockIdx.x] = cnt[i];
}

__global__ void __launch_bounds__(kSortThreads)
radix_scatter_kernel(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                     uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, int64_t n,
                     int shift, int bits, const uint32_t* __restrict__ offs, int64_t nblk,
                     uint32_t kmax)
{
    __shared__ uint32_t wcnt[kSortWarps][1 << kMaxDigitBits];
    const int nd = 1 << bits;
    const uint32_t mask = (uint32_t)nd - 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < kSortWarps * (1 << kMaxDigitBits); i += kSortThreads)
        (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile + (int64_t)warp * 32 * kSortItems;
    const unsigned lt_mask = (1u << lane) - 1u;
    uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const int64_t e = base + r * 32 + lane;
        const bool valid = e < n;
        key[r] = valid ? min(__ldg(kin + e), kmax) : 0u;
        val[r] = valid ? (vin ? __ldg(vin + e) : (uint32_t)e) : 0u;  // no vin: the index
        const uint32_t dig = valid ? (key[r] >> shift) & mask : 0xFFFFFFFFu;
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, dig);
        uint32_t cur = 0;
        if (valid) cur = wcnt[warp][dig];
        __syncwarp();
        rank[r] = cur + (uint32_t)__popc(peers & lt_mask);
        if (valid && lane == 31 - __clz(peers)) wcnt[warp][dig] = cur + (uint32_t)__popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: block offset from the scanned table, then exclusive prefix
    // over the warps in warp order
    for (int d = threadIdx.x; d < nd; d += kSortThreads) {
        uint32_t run = offs[(int64_t)d * nblk + blockIdx.x];
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t t = wcnt[w][d];
            wcnt[w][d] = run;
            run += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const int64_t e = base + r * 32 + lane;
        if (e < n) {
            const uint32_t pos = wcnt[warp][(key[r] >> shift) & mask] + rank[r];
            kout[pos] = key[r];
            vout[pos] = val[r];
        }
    }
}

// ---------------------------------------------------------------------------
// exclusive scan of a uint32 array (three phases)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_sums,
                                                         uint32_t* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        uint32_t s = lane < nw ? warp_sums[lane] : 0u;
        uint32_t si = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, si, o);
            if (lane >= o) si += t;
        }
        if (lane < nw) warp_sums[lane] = si - s;
        if (lane == 31) *total = si;
    }
    __syncthreads();
    const uint32_t r = warp_sums[warp] + inc - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanThreads)
scan_reduce_kernel(const uint32_t* __restrict__ in, int64_t m, uint32_t* __restrict__ sums)
{
    __shared__ uint32_t red[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q)
        if (base + q < m) s += in[base + q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t t = red[threadIdx.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xFFFFFFFFu, t, o);
        if (threadIdx.x == 0) sums[blockIdx.x] = t;
    }
}

// Single block: exclusive scan of the block sums in place.
__global__ void __launch_bounds__(kScanThreads) scan_sums_kernel(uint32_t* sums, int64_t nb)
{
    __shared__ uint32_t ws[32];
    __shared__ uint32_t total;
    uint32_t carry = 0;
    for (int64_t base = 0; base < nb; base += kScanThreads) {
        const int64_t e = base + threadIdx.x;
        const uint32_t v = e < nb ? sums[e] : 0u;
        const uint32_t ex = block_exclusive_scan(v, ws, &total);
        if (e < nb) sums[e] = carry + ex;
        carry += total;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kScanThreads)
scan_apply_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int64_t m,
                  const uint32_t* __restrict__ sums)
{
    __shared__ uint32_t ws[32];
    __shared__ uint32_t total;
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        v[q] = (base + q < m) ? in[base + q] : 0u;
        s += v[q];
    }
    uint32_t run = block_exclusive_scan(s, ws, &total) + sums[blockIdx.x];
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        if (base + q < m) out[base + q] = run;
        run += v[q];
    }
}

__global__ void tile_offset_kernel(const uint32_t* __restrict__ keys, int64_t n, int64_t ntiles,
                                   uint32_t tsize, int64_t* __restrict__ tile_offset)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= ntiles;
         t += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t target = (uint64_t)t * tsize;
        int64_t lo = 0, hi = n;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if ((uint64_t)keys[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        tile_offset[t] = lo;
    }
}

__global__ void tile_items_kernel(const int64_t* __restrict__ tile_offset, int64_t ntiles,
                                  int chunk, uint32_t* __restrict__ items)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= ntiles;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t cnt = t < ntiles ? tile_offset[t + 1] - tile_offset[t] : 0;
        items[t] = (uint32_t)((cnt + chunk - 1) / chunk);
    }
}

template <class T>
__global__ void permute_kernel(int64_t n, int ncomp, const uint32_t* __restrict__ perm, PField src,
                               PField dst)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = perm[p];
        for (int c = 0; c < ncomp; ++c) dst.set<T>(p, c, src.get<T>(q, c));
    }
}

// Packed rows (array of structures): one thread per (particle, word) with the
// widest word that divides the row and both base addresses, so that the
// stores of a warp are contiguous and a row is read in whole words.
template <class W>
__global__ void permute_rows_kernel(int64_t n, int words, const uint32_t* __restrict__ perm,
                                    const W* __restrict__ src, W* __restrict__ dst)
{
    const int64_t total = n * words;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = e / words;
        const int w = (int)(e - p * words);
        dst[e] = src[(int64_t)__ldg(perm + p) * words + w];
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct SortPlan {
    BinP bp;
    int64_t ntiles;
    int bits, passes, width;
    int64_t nblk, hist_len, scan_blocks;
    int64_t off_keys, off_vals, off_hist, off_scan, off_sums, bytes;
};

static int64_t align256(int64_t v) { return (v + 255) & ~int64_t(255); }

picasso_status make_binp(const picasso_spline* sd, const int32_t tile[3], BinP* bp,
                         int64_t* ntiles)
{
    picasso_status st = make_mesh(sd, &bp->mp);
    if (st) return st;
    if (!tile) return PICASSO_ERR_INVALID_ARGUMENT;
    bp->order = sd->order;
    int64_t nt_total = 1, tsize = 1;
    for (int d = 0; d < 3; ++d) {
        if (tile[d] < 1) return PICASSO_ERR_INVALID_ARGUMENT;
        bp->tile[d] = tile[d];
        bp->tshift[d] = -1;
        for (int sh = 0; sh < 31; ++sh)
            if ((1 << sh) == tile[d]) bp->tshift[d] = sh;
        bp->nb[d] = sd->mesh.periodic[d] ? sd->mesh.own_extent[d] : sd->mesh.extent[d];
        bp->nt[d] = (bp->nb[d] + tile[d] - 1) / tile[d];
        nt_total *= bp->nt[d];
        tsize *= tile[d];
    }
    const int64_t nkeys = nt_total * tsize;
    if (nkeys >= 0xFFFFFFFFLL) return PICASSO_ERR_OUT_OF_RANGE;
    bp->tsize = (uint32_t)tsize;
    bp->nkeys = (uint32_t)nkeys;
    *ntiles = nt_total;
    return PICASSO_OK;
}

static picasso_status make_plan(const picasso_spline* sd, int64_t n, const int32_t tile[3],
                                SortPlan* pl)
{
    if (!sd || !tile || n < 0 || n > 0xFFFFFFFELL) return PICASSO_ERR_INVALID_ARGUMENT;
    picasso_status st = make_binp(sd, tile, &pl->bp, &pl->ntiles);
    if (st) return st;
    const int64_t nkeys = pl->bp.nkeys;
    int bits = 1;
    while ((int64_t(1) << bits) <= nkeys) ++bits;  // keys are in [0, nkeys]
    pl->bits = bits;
    pl->passes = (bits + kMaxDigitBits - 1) / kMaxDigitBits;
    pl->width = (bits + pl->passes - 1) / pl->passes;
    pl->nblk = (n + kSortTile - 1) / kSortTile;
    if (pl->nblk < 1) pl->nblk = 1;
    // the digit table is also reused for the per-tile work-item counts
    pl->hist_len = (int64_t(1) << pl->width) * pl->nblk;
    if (pl->hist_len < pl->ntiles + 1) pl->hist_len = pl->ntiles + 1;
    pl->scan_blocks = (pl->hist_len + kScanTile - 1) / kScanTile;
    int64_t o = 0;
    pl->off_keys = o;
    o = align256(o + 4 * (n > 0 ? n : 1));
    pl->off_vals = o;
    o = align256(o + 4 * (n > 0 ? n : 1));
    pl->off_hist = o;
    o = align256(o + 4 * pl->hist_len);
    pl->off_scan = o;
    o = align256(o + 4 * pl->hist_len);
    pl->off_sums = o;
    o = align256(o + 4 * pl->scan_blocks);
    pl->bytes = o;
    return PICASSO_OK;
}

}  // namespace pb

using namespace pb;

extern "C" picasso_status picasso_cell_sort_workspace(const picasso_spline* sd,
                                                      int64_t num_particles,
                                                      const int32_t tile[3], int64_t* bytes)
{
    if (!bytes) return PICASSO_ERR_INVALID_ARGUMENT;
    SortPlan pl;
    picasso_status st = make_plan(sd, num_particles, tile, &pl);
    if (st) return st;
    *bytes = pl.bytes;
    return PICASSO_OK;
}

// The sort proper.  key_src == nullptr: keys from the positions x_p;
// otherwise the first radix pass reads the caller's keys (clamped to nkeys)
// and takes the particle index as its value.
static picasso_status cell_sort_impl(const picasso_spline* sd, int64_t num_particles,
                                     const picasso_particle_field* x_p, const uint32_t* key_src,
                                     const int32_t tile[3], int32_t chunk, uint32_t* key,
                                     uint32_t* perm, int64_t* tile_offset, uint32_t* tile_items,
                                     void* workspace, int64_t workspace_bytes,
                                     picasso_bins* bins_out, const picasso_exec* exec)
{
    SortPlan pl;
    picasso_status st = make_plan(sd, num_particles, tile, &pl);
    if (st) return st;
    if (x_p && (st = validate_pfield(num_particles, *x_p, PICASSO_F64))) return st;
    if ((num_particles > 0 && (!key || !perm)) || !tile_offset || !tile_items || !workspace ||
        workspace_bytes < pl.bytes || chunk < 32)
        return PICASSO_ERR_INVALID_ARGUMENT;
    if (!x_p && num_particles > 0 && (!key_src || key_src == key || key_src == perm))
        return PICASSO_ERR_INVALID_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(workspace) % 256) return PICASSO_ERR_INVALID_ARGUMENT;
    const int64_t n = num_particles;
    const uint32_t kmax = pl.bp.nkeys;
    cudaStream_t s = stream_of(exec);
    char* ws = static_cast<char*>(workspace);
    uint32_t* wk = reinterpret_cast<uint32_t*>(ws + pl.off_keys);
    uint32_t* wv = reinterpret_cast<uint32_t*>(ws + pl.off_vals);
    uint32_t* hist = reinterpret_cast<uint32_t*>(ws + pl.off_hist);
    uint32_t* scan = reinterpret_cast<uint32_t*>(ws + pl.off_scan);
    uint32_t* sums = reinterpret_cast<uint32_t*>(ws + pl.off_sums);
    // ping-pong so that the last pass writes the caller's arrays
    uint32_t *ka = wk, *va = wv, *kb = key, *vb = perm;
    if (pl.passes % 2 == 0) {
        ka = key;
        va = perm;
        kb = wk;
        vb = wv;
    }
    if (n > 0) {
        const uint32_t* kin = ka;
        const uint32_t* vin = va;
        if (x_p) {
            key_kernel<<<grid_for(n, 256), 256, 0, s>>>(pl.bp, n, make_pfield(*x_p), ka, va);
        } else {
            kin = key_src;
            vin = nullptr;
        }
        for (int pass = 0; pass < pl.passes; ++pass) {
            const int shift = pass * pl.width;
            const int bits = (shift + pl.width <= pl.bits) ? pl.width : pl.bits - shift;
            radix_hist_kernel<<<(unsigned)pl.nblk, kSortThreads, 0, s>>>(kin, n, shift, bits, hist,
                                                                          pl.nblk, kmax);
            const int64_t m = (int64_t(1) << bits) * pl.nblk;
            const int64_t sb = (m + kScanTile - 1) / kScanTile;
            scan_reduce_kernel<<<(unsigned)sb, kScanThreads, 0, s>>>(hist, m, sums);
            scan_sums_kernel<<<1, kScanThreads, 0, s>>>(sums, sb);
            scan_apply_kernel<<<(unsigned)sb, kScanThreads, 0, s>>>(hist, scan, m, sums);
            radix_scatter_kernel<<<(unsigned)pl.nblk, kSortThreads, 0, s>>>(
                kin, vin, kb, vb, n, shift, bits, scan, pl.nblk, kmax);
            uint32_t* t = ka;
            ka = kb;
            kb = t;
            t = va;
            va = vb;
            vb = t;
            kin = ka;
            vin = va;
        }
    }
    tile_offset_kernel<<<grid_for(pl.ntiles + 1, 256), 256, 0, s>>>(key, n, pl.ntiles, pl.bp.tsize,
                                                                     tile_offset);
    // work items: exclusive prefix of ceil(count / chunk) per tile
    {
        const int64_t m = pl.ntiles + 1;
        const int64_t sb = (m + kScanTile - 1) / kScanTile;
        tile_items_kernel<<<grid_for(m, 256), 256, 0, s>>>(tile_offset, pl.ntiles, chunk, hist);
        scan_reduce_kernel<<<(unsigned)sb, kScanThreads, 0, s>>>(hist, m, sums);
        scan_sums_kernel<<<1, kScanThreads, 0, s>>>(sums, sb);
        scan_apply_kernel<<<(unsigned)sb, kScanThreads, 0, s>>>(hist, tile_items, m, sums);
    }
    if ((st = check_launch())) return st;
    if (bins_out) {
        for (int d = 0; d < 3; ++d) {
            bins_out->tile[d] = pl.bp.tile[d];
            bins_out->num_tiles[d] = pl.bp.nt[d];
            bins_out->bin_extent[d] = pl.bp.nb[d];
        }
        bins_out->order = sd->order;
        bins_out->location = sd->location;
        bins_out->chunk = chunk;
        bins_out->p2g_lanes = 0;
        bins_out->tile_offset = tile_offset;
        bins_out->tile_items = tile_items;
        bins_out->records = nullptr;
    }
    return PICASSO_OK;
}

extern "C" picasso_status picasso_cell_sort(const picasso_spline* sd, int64_t num_particles,
                                            picasso_particle_field x_p, const int32_t tile[3],
                                            int32_t chunk, uint32_t* key, uint32_t* perm,
                                            int64_t* tile_offset, uint32_t* tile_items,
                                            void* workspace, int64_t workspace_bytes,
                                            picasso_bins* bins_out, const picasso_exec* exec)
{
    return cell_sort_impl(sd, num_particles, &x_p, nullptr, tile, chunk, key, perm, tile_offset,
                          tile_items, workspace, workspace_bytes, bins_out, exec);
}

extern "C" picasso_status picasso_cell_sort_keys(const picasso_spline* sd, int64_t num_particles,
                                                 const uint32_t* key_in, const int32_t tile[3],
                                                 int32_t chunk, uint32_t* key, uint32_t* perm,
                                                 int64_t* tile_offset, uint32_t* tile_items,
                                                 void* workspace, int64_t workspace_bytes,
                                                 picasso_bins* bins_out,
                                                 const picasso_exec* exec)
{
    return cell_sort_impl(sd, num_particles, nullptr, key_in, tile, chunk, key, perm, tile_offset,
                          tile_items, workspace, workspace_bytes, bins_out, exec);
}

extern "C" picasso_status picasso_permute(int64_t num_particles, int32_t ncomp,
                                          const uint32_t* perm, picasso_particle_field src,
                                          picasso_particle_field dst, const picasso_exec* exec)
{
    if (num_particles < 0 || ncomp < 1 || (num_particles > 0 && !perm))
        return PICASSO_ERR_INVALID_ARGUMENT;
    picasso_status st;
    if ((st = validate_pfield(num_particles, src, PICASSO_F64, PICASSO_F32))) return st;
    if ((st = validate_pfield(num_particles, dst, src.dtype))) return st;
    if (num_particles > 0 && src.data == dst.data) return PICASSO_ERR_INVALID_ARGUMENT;
    if (num_particles == 0) return PICASSO_OK;
    cudaStream_t s = stream_of(exec);
    const int64_t esize = src.dtype == PICASSO_F64 ? 8 : 4;
    auto packed = [&](const picasso_particle_field& f) {
        return (f.vector_shift == 0 && f.tile_stride == ncomp && (f.comp_stride == 1 || ncomp == 1)) ||
               (ncomp == 1 && f.vector_shift >= 62);
    };
    if (packed(src) && packed(dst)) {
        const int64_t row = esize * ncomp;
        const uintptr_t al = reinterpret_cast<uintptr_t>(src.data) | reinterpret_cast<uintptr_t>(dst.data);
        const int64_t word = (row % 16 == 0 && al % 16 == 0) ? 16 : ((row % 8 == 0 && al % 8 == 0) ? 8 : 4);
        const int words = (int)(row / word);
        const unsigned blocks = grid_for(num_particles * words, 256);
        if (word == 16)
            permute_rows_kernel<uint4><<<blocks, 256, 0, s>>>(num_particles, words, perm,
                                                              (const uint4*)src.data, (uint4*)dst.data);
        else if (word == 8)
            permute_rows_kernel<uint2><<<blocks, 256, 0, s>>>(num_particles, words, perm,
                                                              (const uint2*)src.data, (uint2*)dst.data);
        else
            permute_rows_kernel<uint32_t><<<blocks, 256, 0, s>>>(num_particles, words, perm,
                                                                 (const uint32_t*)src.data,
                                                                 (uint32_t*)dst.data);
        return check_launch();
    }
    const unsigned blocks = grid_for(num_particles, 256);
    if (src.dtype == PICASSO_F64)
        permute_kernel<double><<<blocks, 256, 0, s>>>(num_particles, ncomp, perm, make_pfield(src),
                                                      make_pfield(dst));
    else
        permute_kernel<float><<<blocks, 256, 0, s>>>(num_particles, ncomp, perm, make_pfield(src),
                                                     make_pfield(dst));
    return check_launch();
}

// ---------------------------------------------------------------------------
// Spline records
// ---------------------------------------------------------------------------
// rec[p] = (t_x, t_y, t_z, key): the in-cell fraction of the particle's
// logical position along each dimension (FP32, rounded from the FP64
// position exactly as the transfer kernels round it) and its sort key for
// the bins' tile shape (the cell sort's key, stencil starts from the same
// FP64 arithmetic), so a transfer that reads the record builds the same
// spline and bin as one that reads the position.
namespace pb {

template <int ORDER>
__global__ void records_kernel(BinP bp, int64_t n, PField x, float4* rec)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        int s[3];
        float t[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            t[d] = logical_frac<ORDER>(x.get<double>(p, d), bp.mp.lo[d], bp.mp.rdx[d], s[d]);
        rec[p] = make_float4(t[0], t[1], t[2], __uint_as_float(key_from_starts(bp, s)));
    }
}

}  // namespace pb

extern "C" picasso_status picasso_spline_records(const picasso_spline* sd, int64_t num_particles,
                                                 picasso_particle_field x_p,
                                                 const picasso_bins* bins, void* records,
                                                 const picasso_exec* exec)
{
    if (!sd || !bins || num_particles < 0) return PICASSO_ERR_INVALID_ARGUMENT;
    if (bins->order != sd->order || bins->location != sd->location)
        return PICASSO_ERR_INVALID_ARGUMENT;
    BinP bp;
    int64_t ntiles = 0;
    picasso_status st = make_binp(sd, bins->tile, &bp, &ntiles);
    if (st) return st;
    for (int d = 0; d < 3; ++d)
        if (bins->num_tiles[d] != bp.nt[d] || bins->bin_extent[d] != bp.nb[d])
            return PICASSO_ERR_INVALID_ARGUMENT;
    if ((st = validate_pfield(num_particles, x_p, PICASSO_F64))) return st;
    if (num_particles == 0) return PICASSO_OK;
    if (!records || reinterpret_cast<uintptr_t>(records) % 16) return PICASSO_ERR_INVALID_ARGUMENT;
    cudaStream_t s = stream_of(exec);
    const PField x = make_pfield(x_p);
    float4* rec = static_cast<float4*>(records);
    const unsigned blocks = grid_for(num_particles, 256);
    if (sd->order == 1) records_kernel<1><<<blocks, 256, 0, s>>>(bp, num_particles, x, rec);
    else if (sd->order == 2) records_kernel<2><<<blocks, 256, 0, s>>>(bp, num_particles, x, rec);
    else records_kernel<3><<<blocks, 256, 0, s>>>(bp, num_particles, x, rec);
    return check_launch();
}

// ---------------------------------------------------------------------------
// Cell sort without allocation
// ---------------------------------------------------------------------------
// Callers that cannot allocate device memory when they sort -- an application
// that hands all of the GPU's memory to its own pool at start-up, a plugin
// hosted by such an application, or a time-critical loop that must never hit
// the allocator's latency or out-of-memory path -- get a sort whose scratch
// is a fixed array compiled into this library.  The array is
// kStaticSortScratchBytes large; every device on which the library's kernels
// are loaded holds it until the process exits.
namespace pb {

constexpr int64_t kStaticSortScratchBytes = 32LL << 20;  // 32 MiB
static __device__ __align__(256) unsigned char g_sort_scratch[kStaticSortScratchBytes];

// Device address of g_sort_scratch in the current context.  It is looked up
// on every call: the host-side name of a __device__ array is not a device
// address, and a cached address would go stale when the application resets
// the device or its primary context (the module is then loaded again and the
// array may move).  The lookup costs microseconds, small next to the sort's
// launches.
static picasso_status static_sort_scratch(void** out)
{
    void* p = nullptr;
    PB_CUDA_TRY(cudaGetSymbolAddress(&p, g_sort_scratch));
    *out = p;
    return PICASSO_OK;
}

}  // namespace pb

extern "C" picasso_status picasso_cell_sort_static(const picasso_spline* sd,
                                                   int64_t num_particles,
                                                   picasso_particle_field x_p,
                                                   const int32_t tile[3], int32_t chunk,
                                                   uint32_t* key, uint32_t* perm,
                                                   int64_t* tile_offset, uint32_t* tile_items,
                                                   picasso_bins* bins_out,
                                                   const picasso_exec* exec)
{
    SortPlan pl;
    picasso_status st = make_plan(sd, num_particles, tile, &pl);
    if (st) return st;
    if (pl.bytes > kStaticSortScratchBytes) return PICASSO_ERR_OUT_OF_RANGE;
    void* ws = nullptr;
    if ((st = static_sort_scratch(&ws))) return st;
    // Every scratch word the sort reads is written earlier in the same call,
    // so nothing needs clearing between calls.
    return picasso_cell_sort(sd, num_particles, x_p, tile, chunk, key, perm, tile_offset,
                             tile_items, ws, kStaticSortScratchBytes, bins_out, exec);
}
