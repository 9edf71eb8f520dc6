// Single-call tiled APIC P2G / G2P kernels (FP32 precision form) for
// particles sorted by picasso_cell_sort: one CTA per work item, the item
// bodies are in tiled.cuh.
//
// P2G runs single-warp CTAs (warps finish their items independently; a
// 4-warp CTA would wait for its slowest warp) with LPP lanes per particle.
// G2P runs 128-thread CTAs sharing one node tile.
#include <mutex>

#include "tiled.cuh"

namespace pb {

// Threads of a tiled G2P CTA (one work item each).  Measured at 256^3
// 8 ppc: quadratic 2.92 ms with 128 threads, 2.79 with 64, 2.94 with 32;
// cubic 5.09 / 4.73 / 4.54 ms; linear 1.87 with 64, 2.28 with 32.
template <int ORDER>
struct G2PThreads {
    static constexpr int value = ORDER == 3 ? 32 : 64;
};

template <int ORDER, int LPP, bool REC, bool FUSED, bool STAG>
__global__ void __launch_bounds__(32, (P2GOccupancy<ORDER, LPP>::value))
p2g_tiled_kernel(P2GArgs A, FusedUpdate F, int64_t n)
{
    extern __shared__ __align__(16) float smem[];
    __shared__ int stage_base[kStageBases];
    if (blockIdx.x == 0 && threadIdx.x == 0 && A.err) {
        const int64_t n_valid = __ldg(A.tp.off + A.tp.ntiles);
        if (n > n_valid) atomicAdd(A.err, (int)(n - n_valid));
    }
    int64_t t, a, b;
    if (!item_range(A.tp, blockIdx.x, t, a, b)) return;
    p2g_item<ORDER, LPP, REC, STAG>(A, t, a, b, smem, stage_base);
    if constexpr (FUSED) fused_update_arrive<ORDER>(A, F, t);
}

template <int ORDER, bool ADV, bool REC, bool STAG>
__global__ void __launch_bounds__(G2PThreads<ORDER>::value) g2p_tiled_kernel(G2PArgs A, int64_t n)
{
    extern __shared__ __align__(16) float smem[];
    if (blockIdx.x == 0 && threadIdx.x == 0 && A.err) {
        const int64_t n_valid = __ldg(A.tp.off + A.tp.ntiles);
        if (n > n_valid) atomicAdd(A.err, (int)(n - n_valid));
    }
    int64_t t, a, b;
    if (!item_range(A.tp, blockIdx.x, t, a, b)) return;  // CTA-uniform
    g2p_item<ORDER, G2PThreads<ORDER>::value, ADV, REC, STAG>(A, t, a, b,
                                                       reinterpret_cast<float4*>(smem),
                                                       threadIdx.x);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// Padded node-tile strides for the P2G merge: value v = lane + 32 r of a
// staged lane (field v / FS of its F fields, stencil node v % FS) lands at
// f * P + a * SI + b * SJ + c; pick the smallest padding that maximises the
// number of distinct banks per merge instruction.  The search takes a fraction
// of a millisecond, so results are cached per (tile nodes, K, F) for callers
// that alternate between tile shapes (batches of meshes).
struct StrideKey {
    int NT[3], K, F, split;
    bool operator==(const StrideKey& o) const
    {
        return NT[0] == o.NT[0] && NT[1] == o.NT[1] && NT[2] == o.NT[2] && K == o.K &&
               F == o.F && split == o.split;
    }
};

// Tile strides (SJ, SI, P) that spread the tile offsets of one merge round
// (32 staged values added by 32 lanes) over as many shared-memory banks as
// possible; the smallest tile among equals.  `split`: the staging of the
// i-plane split (F fields of K^2 nodes per lane, whose k-plane merges are
// counted as well).
static void search_strides(const StrideKey& key, int* SJ, int* SI, int* P)
{
    const int* NT = key.NT;
    const int K = key.K, F = key.F;
    const int NL = key.split ? K * K : K * K * K, FS = (NL + 3) & ~3, SV = F * FS;
    const int R = (SV + 31) / 32;
    const int ROWS = NL / K, PV = F * ROWS, RP = key.split ? (PV + 31) / 32 : 0;
    int best = -1, bsj = NT[2], bsi = NT[1] * NT[2], bp = NT[0] * NT[1] * NT[2];
    long best_size = 0;
    for (int sj = NT[2]; sj < NT[2] + 8; ++sj)
        for (int si = NT[1] * sj; si < NT[1] * sj + 16; ++si)
            for (int pp = NT[0] * si; pp < NT[0] * si + 16; ++pp) {
                int distinct = 0;
                for (int r = 0; r < R; ++r) {
                    unsigned banks = 0;
                    for (int lane = 0; lane < 32; ++lane) {
                        const int v = lane + 32 * r, f = v / FS, nn = v % FS;
                        if (v >= SV || nn >= NL) continue;
                        const int a = nn / (K * K), b = (nn / K) % K, c = nn % K;
                        const int off = f * pp + a * si + b * sj + c;
                        // 8-byte tile words: a half warp per bank cycle
                        const unsigned bit = kTileWords == 2
                                                 ? (1u << ((off & 15) + 16 * (lane >> 4)))
                                                 : (1u << (off & 31));
                        if (!(banks & bit)) ++distinct;
                        banks |= bit;
                    }
                }
                for (int r = 0; r < RP; ++r) {
                    unsigned banks = 0;
                    for (int lane = 0; lane < 32; ++lane) {
                        const int v = lane + 32 * r;
                        if (v >= PV) continue;
                        const int ij = v % ROWS;
                        const int off = (v / ROWS) * pp + (ij / K) * si + (ij % K) * sj;
                        const unsigned bit = kTileWords == 2
                                                 ? (1u << ((off & 15) + 16 * (lane >> 4)))
                                                 : (1u << (off & 31));
                        if (!(banks & bit)) ++distinct;
                        banks |= bit;
                    }
                }
                const long size = 4L * pp * kTileWords;
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
}

static void choose_strides(const int NT[3], int K, int F, int split, int* SJ, int* SI, int* P)
{
    constexpr int kSlots = 64;
    static std::mutex mu;
    static StrideKey keys[kSlots];
    static int vals[kSlots][3];
    static int used = 0, next = 0;
    const StrideKey key{{NT[0], NT[1], NT[2]}, K, F, split};
    {
        std::lock_guard<std::mutex> lock(mu);
        for (int i = 0; i < used; ++i)
            if (keys[i] == key) {
                *SJ = vals[i][0];
                *SI = vals[i][1];
                *P = vals[i][2];
                return;
            }
    }
    search_strides(key, SJ, SI, P);
    std::lock_guard<std::mutex> lock(mu);
    const int slot = used < kSlots ? used++ : (next++ % kSlots);
    keys[slot] = key;
    vals[slot][0] = *SJ;
    vals[slot][1] = *SI;
    vals[slot][2] = *P;
}

static_assert(P2GCfg<3, 4>::ISPLIT && !P2GCfg<2, 4>::ISPLIT && !P2GCfg<1, 4>::ISPLIT &&
                  !P2GCfg<1, 2>::ISPLIT,
              "make_tilep's stride choice follows the accumulator split");

int default_lpp(int order) { return order == 3 ? 4 : 1; }

// Orders 1 and 2 take 1, 2 or 4 lanes per particle (staggered locations, with
// two grid fields: 1 or 2); order 3 (4 x 64 accumulators) takes 4.
bool valid_lpp(int order, int lpp, bool stag)
{
    if (order == 3) return lpp == 4;
    return lpp == 1 || lpp == 2 || (lpp == 4 && !stag);
}

// Tile geometry for the bins; lpp > 0 also picks the P2G tile strides for nf
// grid fields.
bool make_tilep(const MeshP& mp, int order, const picasso_bins& bins, TileP* tp, int lpp, int nf)
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
        tp->tsh[d] = -1;
        for (int sh = 0; sh < 31; ++sh)
            if ((1 << sh) == bins.tile[d]) tp->tsh[d] = sh;
        nt *= bins.num_tiles[d];
    }
    tp->tsize = (uint32_t)bins.tile[0] * (uint32_t)bins.tile[1] * (uint32_t)bins.tile[2];
    tp->nodes = tp->NT[0] * tp->NT[1] * tp->NT[2];
    if (lpp > 0) {
        // the accumulator split of p2g_item (P2GCfg::ISPLIT, F)
        const int split = order == 3 && lpp == 4;
        choose_strides(tp->NT, K, split ? nf : nf / lpp, split, &tp->SJ, &tp->SI, &tp->P);
    } else {
        tp->SJ = tp->NT[2];
        tp->SI = tp->NT[1] * tp->NT[2];
        tp->P = tp->nodes;
    }
    tp->ntiles = nt;
    tp->off = bins.tile_offset;
    tp->items = bins.tile_items;
    tp->chunk = bins.chunk;
    return bins.tile_offset && bins.tile_items && bins.chunk >= 32;
}

// The fused update needs every tile (the last one included) to hold at least
// K - 1 bins along each dimension, so that a node is touched by the items of
// its own tile and of the previous one only.
bool fused_update_fits(const TileP& tp, int order)
{
    const int K = order + 1;
    for (int d = 0; d < 3; ++d) {
        const int last = tp.nb[d] - (tp.nt[d] - 1) * tp.T[d];
        if (tp.T[d] < K - 1 || last < K - 1) return false;
    }
    return true;
}

int device_smem_optin()
{
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

// Packed storage the tiled kernels read: x (N,3) FP64, m (N) FP32, c (N,12)
// FP32 with 16-byte aligned rows.
bool packed_x(const PField& x)
{
    return x.shift == 0 && x.tile_stride == 3 && x.comp_stride == 1 &&
           (reinterpret_cast<uintptr_t>(x.data) % 8) == 0;
}
bool packed_m(const PField& m) { return (m.shift == 0 && m.tile_stride == 1) || m.shift == 63; }
bool packed_c(const PField& c)
{
    return c.shift == 0 && c.tile_stride == 12 && c.comp_stride == 1 &&
           (reinterpret_cast<uintptr_t>(c.data) % 16) == 0;
}

size_t p2g_warp_bytes(int order, int lpp, int P, bool rec, bool stag)
{
#define PB_CASE(O, L, S)                                                                \
    if (order == O && lpp == L && stag == S)                                            \
        return sizeof(float) * (size_t)(rec ? p2g_warp_floats<O, L, true, S>(P)         \
                                            : p2g_warp_floats<O, L, false, S>(P));
    PB_CASE(1, 1, false) PB_CASE(1, 2, false) PB_CASE(1, 4, false)
    PB_CASE(2, 1, false) PB_CASE(2, 2, false) PB_CASE(2, 4, false)
    PB_CASE(3, 4, false)
    PB_CASE(1, 1, true) PB_CASE(1, 2, true) PB_CASE(2, 1, true) PB_CASE(2, 2, true)
    PB_CASE(3, 4, true)
#undef PB_CASE
    return 0;
}

static int64_t item_bound(const TileP& tp, int64_t n)
{
    return tp.ntiles + (n + tp.chunk - 1) / tp.chunk;
}

template <int ORDER, int LPP, bool REC, bool STAG>
static picasso_status launch_p2g_tiled(const P2GArgs& args, const FusedUpdate* fu, int64_t n,
                                       cudaStream_t st)
{
    P2GArgs A = args;
    // the bulk flush rounds rows into the ring and staging area: one k-row
    // at least must fit
    if (P2GCfg<ORDER, LPP, REC, STAG>::TILE_OFF / 8 < A.tp.NT[2]) A.bulk_flush = 0;
    const size_t smem = p2g_warp_bytes(ORDER, LPP, A.tp.P, REC, STAG);
    const int64_t items = item_bound(A.tp, n);
    if constexpr (!STAG) {
        if (fu) {
            PB_CUDA_TRY(cudaFuncSetAttribute(p2g_tiled_kernel<ORDER, LPP, REC, true, false>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem));
            p2g_tiled_kernel<ORDER, LPP, REC, true, false>
                <<<(unsigned)(items ? items : 1), 32, smem, st>>>(A, *fu, n);
            return check_launch();
        }
    } else if (fu) {
        return PICASSO_ERR_UNSUPPORTED;  // the fused update is collocated
    }
    PB_CUDA_TRY(cudaFuncSetAttribute(p2g_tiled_kernel<ORDER, LPP, REC, false, STAG>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    p2g_tiled_kernel<ORDER, LPP, REC, false, STAG>
        <<<(unsigned)(items ? items : 1), 32, smem, st>>>(A, FusedUpdate{}, n);
    return check_launch();
}

template <int ORDER, bool ADV, bool REC, bool STAG>
static picasso_status launch_g2p_tiled(const G2PArgs& A, int64_t n, cudaStream_t st)
{
    const size_t smem = sizeof(float4) * (size_t)A.tp.nodes;
    PB_CUDA_TRY(cudaFuncSetAttribute(g2p_tiled_kernel<ORDER, ADV, REC, STAG>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t items = item_bound(A.tp, n);
    g2p_tiled_kernel<ORDER, ADV, REC, STAG>
        <<<(unsigned)(items ? items : 1), G2PThreads<ORDER>::value, smem, st>>>(A, n);
    return check_launch();
}

// gm and gmu are views of one (..., 4) 64-bit accumulator: a node's mass and
// momentum are 4 consecutive words, nodes 16-byte aligned, a k-row of nodes
// contiguous.
static bool packed_accumulator(const GField& gm, const GField& gmu)
{
    return gmu.data == gm.data + sizeof(long long) && gm.s[2] == 4 && gmu.s[2] == 4 &&
           gm.s[0] == gmu.s[0] && gm.s[1] == gmu.s[1] && gmu.s[3] == 1 && gm.s[0] % 2 == 0 &&
           gm.s[1] % 2 == 0 && reinterpret_cast<uintptr_t>(gm.data) % 16 == 0;
}

// Spline records the tiled kernels may read instead of the positions: a
// 16-byte aligned array, when the bins carry one.
static const float* bins_records(const picasso_bins& bins)
{
    const uintptr_t r = reinterpret_cast<uintptr_t>(bins.records);
    return (r && r % 16 == 0) ? static_cast<const float*>(bins.records) : nullptr;
}

// stag: the entity's dimension of a staggered location (its grid fields are
// the mass and one momentum component: c_p column stag), else -1.
picasso_status apic_p2g_tiled(const MeshP& mp, int order, int ncomp, Form form, int64_t n,
                              const PField& x, const PField& m, const PField& c, const GField& gm,
                              const GField& gmu, const picasso_bins& bins, int* err,
                              cudaStream_t st, bool* handled, const FusedUpdate* fu, int stag,
                              const HaloPeers* hp)
{
    *handled = false;
    if (form != Form::F32Fixed || ncomp != 3 || !packed_x(x) || !packed_m(m) || !packed_c(c))
        return PICASSO_OK;
    const bool sg = stag >= 0;
    const int lpp = bins.p2g_lanes ? bins.p2g_lanes : default_lpp(order);
    if (!valid_lpp(order, lpp, sg)) return PICASSO_ERR_INVALID_ARGUMENT;
    P2GArgs A;
    if (!make_tilep(mp, order, bins, &A.tp, lpp, sg ? 2 : 4)) return PICASSO_ERR_INVALID_ARGUMENT;
    A.rec = bins_records(bins);
    const bool rec = A.rec != nullptr;
    const size_t smem = p2g_warp_bytes(order, lpp, A.tp.P, rec, sg);
    if ((int64_t)smem > device_smem_optin()) return PICASSO_OK;  // tile too large: plain path
    *handled = true;
    A.mp = mp;
    A.stag = stag;
    A.x = reinterpret_cast<const double*>(x.data);
    A.m = reinterpret_cast<const float*>(m.data);
    A.c = reinterpret_cast<const float*>(c.data);
    A.gm = gm;
    A.gmu = gmu;
    A.scale_m = ldexpf(1.f, gm.fixed_bits);
    A.scale_mu = ldexpf(1.f, gmu.fixed_bits);
    A.err = err;
    A.hp = hp ? *hp : HaloPeers{};
    // the fused update counts its arrivals after element-wise reductions; a
    // neighbour's rows take element-wise reductions too
    A.bulk_flush = !sg && !fu && !A.hp.on && packed_accumulator(gm, gmu);
#define PB_CASE(O, L, S)                                                                \
    if (order == O && lpp == L && sg == S)                                              \
        return rec ? launch_p2g_tiled<O, L, true, S>(A, fu, n, st)                      \
                   : launch_p2g_tiled<O, L, false, S>(A, fu, n, st);
    PB_CASE(1, 1, false) PB_CASE(1, 2, false) PB_CASE(1, 4, false)
    PB_CASE(2, 1, false) PB_CASE(2, 2, false) PB_CASE(2, 4, false)
    PB_CASE(3, 4, false)
    PB_CASE(1, 1, true) PB_CASE(1, 2, true) PB_CASE(2, 1, true) PB_CASE(2, 2, true)
    PB_CASE(3, 4, true)
#undef PB_CASE
    return PICASSO_ERR_INVALID_ARGUMENT;
}

template <int ORDER>
static picasso_status launch_g2p_order(const G2PArgs& A, int64_t n, cudaStream_t st, bool adv,
                                       bool stag)
{
    if (adv) return launch_g2p_tiled<ORDER, true, false, false>(A, n, st);
    if (stag) {
        if (A.rec) return launch_g2p_tiled<ORDER, false, true, true>(A, n, st);
        return launch_g2p_tiled<ORDER, false, false, true>(A, n, st);
    }
    if (A.rec) return launch_g2p_tiled<ORDER, false, true, false>(A, n, st);
    return launch_g2p_tiled<ORDER, false, false, false>(A, n, st);
}

picasso_status apic_g2p_tiled(const MeshP& mp, int order, int ncomp, bool f32, int64_t n,
                              const PField& x, const GField& u, const PField& c,
                              const picasso_bins& bins, int* err, const Advect* adv,
                              cudaStream_t st, bool* handled, int stag, const HaloPeers* hp)
{
    *handled = false;
    if (!f32 || ncomp != 3 || !packed_x(x) || !packed_c(c)) return PICASSO_OK;
    if (adv && stag >= 0) return PICASSO_OK;
    G2PArgs A;
    if (!make_tilep(mp, order, bins, &A.tp)) return PICASSO_ERR_INVALID_ARGUMENT;
    const size_t smem = sizeof(float4) * (size_t)A.tp.nodes;
    if ((int64_t)smem > device_smem_optin()) return PICASSO_OK;
    *handled = true;
    A.mp = mp;
    A.stag = stag;
    A.x = reinterpret_cast<const double*>(x.data);
    A.u = u;
    A.c = reinterpret_cast<float*>(c.data);
    A.err = err;
    A.x_out = adv ? reinterpret_cast<double*>(x.data) : nullptr;
    A.adv = adv ? *adv : Advect{};
    A.hp = hp ? *hp : HaloPeers{};
    // the advection needs the positions; without it the records replace them
    A.rec = adv ? nullptr : reinterpret_cast<const float4*>(bins_records(bins));
    if (order == 1) return launch_g2p_order<1>(A, n, st, adv != nullptr, stag >= 0);
    if (order == 2) return launch_g2p_order<2>(A, n, st, adv != nullptr, stag >= 0);
    return launch_g2p_order<3>(A, n, st, adv != nullptr, stag >= 0);
}

}  // namespace pb

using namespace pb;

// Arrival counters of the fused update: 8 per tile.
extern "C" picasso_status picasso_apic_p2g_update_workspace(const picasso_bins* bins,
                                                            int64_t* bytes)
{
    if (!bins || !bytes) return PICASSO_ERR_INVALID_ARGUMENT;
    int64_t nt = 1;
    for (int d = 0; d < 3; ++d) {
        if (bins->num_tiles[d] < 1) return PICASSO_ERR_INVALID_ARGUMENT;
        nt *= bins->num_tiles[d];
    }
    *bytes = nt * 8 * (int64_t)sizeof(uint32_t);
    return PICASSO_OK;
}

// Halo peers of the ABI in the kernels' form; false if they do not describe
// neighbour slabs of this (x-non-periodic) mesh.
static bool make_halo_peers(const picasso_halo_peers* p, const MeshP& mp, int nfields,
                            HaloPeers* hp)
{
    if (!p || mp.periodic[0]) return false;
    if (p->lo_end < 0 || p->hi_begin > mp.ext[0] || p->lo_end > p->hi_begin) return false;
    *hp = HaloPeers{};
    hp->on = 1;
    hp->lo_end = p->lo_end;
    hp->hi_begin = p->hi_begin;
    hp->lo_shift = p->lo_shift;
    hp->hi_shift = p->hi_shift;
    for (int f = 0; f < nfields; ++f) {
        if ((p->lo_end > 0 && !p->lo[f]) || (p->hi_begin < mp.ext[0] && !p->hi[f])) return false;
        hp->lo[f] = static_cast<char*>(p->lo[f]);
        hp->hi[f] = static_cast<char*>(p->hi[f]);
    }
    return true;
}

extern "C" picasso_status picasso_apic_p2g_halo(const picasso_spline* sd, int64_t num_particles,
                                                picasso_particle_field x_p,
                                                picasso_particle_field m_p,
                                                picasso_particle_field c_p,
                                                picasso_grid_field m_i, picasso_grid_field mu_i,
                                                const picasso_halo_peers* peers,
                                                const picasso_exec* exec)
{
    MeshP mp;
    picasso_status st = make_mesh(sd, &mp);
    if (st) return st;
    if (num_particles < 0 || !peers) return PICASSO_ERR_INVALID_ARGUMENT;
    if ((st = validate_pfield(num_particles, x_p, PICASSO_F64))) return st;
    if ((st = validate_pfield(num_particles, m_p, PICASSO_F64, PICASSO_F32))) return st;
    if ((st = validate_pfield(num_particles, c_p, m_p.dtype))) return st;
    if ((st = validate_gfield(m_i, PICASSO_F64, PICASSO_I64_FIXED))) return st;
    if ((st = validate_gfield(mu_i, m_i.dtype))) return st;
    if (sd->location != PICASSO_NODE || m_p.dtype != PICASSO_F32 ||
        m_i.dtype != PICASSO_I64_FIXED || !exec || !exec->bins)
        return PICASSO_ERR_UNSUPPORTED;
    if (exec->bins->order != sd->order || exec->bins->location != sd->location)
        return PICASSO_ERR_INVALID_ARGUMENT;
    HaloPeers hp;
    if (!make_halo_peers(peers, mp, 2, &hp)) return PICASSO_ERR_INVALID_ARGUMENT;
    if (num_particles == 0) return PICASSO_OK;
    const PField x = make_pfield(x_p), m = make_pfield(m_p), c = make_pfield(c_p);
    GField gm = make_gfield(m_i), gmu = make_gfield(mu_i);
    gm.overflow = gmu.overflow = exec->overflow_count;
    bool handled = false;
    st = apic_p2g_tiled(mp, sd->order, 3, Form::F32Fixed, num_particles, x, m, c, gm, gmu,
                        *exec->bins, exec->error_count, stream_of(exec), &handled, nullptr, -1,
                        &hp);
    if (st) return st;
    return handled ? PICASSO_OK : PICASSO_ERR_UNSUPPORTED;
}

extern "C" picasso_status picasso_apic_g2p_halo(const picasso_spline* sd, int64_t num_particles,
                                                picasso_particle_field x_p,
                                                picasso_grid_field u_i,
                                                picasso_particle_field c_p,
                                                const picasso_halo_peers* peers,
                                                const picasso_exec* exec)
{
    MeshP mp;
    picasso_status st = make_mesh(sd, &mp);
    if (st) return st;
    if (num_particles < 0 || !peers) return PICASSO_ERR_INVALID_ARGUMENT;
    if ((st = validate_pfield(num_particles, x_p, PICASSO_F64))) return st;
    if ((st = validate_gfield(u_i, PICASSO_F64, PICASSO_F32))) return st;
    if ((st = validate_pfield(num_particles, c_p, u_i.dtype))) return st;
    if (sd->location != PICASSO_NODE || u_i.dtype != PICASSO_F32 || !exec || !exec->bins)
        return PICASSO_ERR_UNSUPPORTED;
    if (exec->bins->order != sd->order || exec->bins->location != sd->location)
        return PICASSO_ERR_INVALID_ARGUMENT;
    HaloPeers hp;
    if (!make_halo_peers(peers, mp, 1, &hp)) return PICASSO_ERR_INVALID_ARGUMENT;
    if (num_particles == 0) return PICASSO_OK;
    const PField x = make_pfield(x_p), c = make_pfield(c_p);
    const GField u = make_gfield(u_i);
    bool handled = false;
    st = apic_g2p_tiled(mp, sd->order, 3, true, num_particles, x, u, c, *exec->bins,
                        exec->error_count, nullptr, stream_of(exec), &handled, -1, &hp);
    if (st) return st;
    return handled ? PICASSO_OK : PICASSO_ERR_UNSUPPORTED;
}

extern "C" picasso_status picasso_apic_p2g_update(
    const picasso_spline* sd, int64_t num_particles, picasso_particle_field x_p,
    picasso_particle_field m_p, picasso_particle_field c_p, picasso_grid_field m_i,
    picasso_grid_field mu_i, picasso_grid_field f_i, const picasso_grid_update_params* prm,
    picasso_grid_field u_i, picasso_grid_field u64_i, void* workspace, int64_t workspace_bytes,
    const picasso_exec* exec)
{
    MeshP mp;
    picasso_status st = make_mesh(sd, &mp);
    if (st) return st;
    if (num_particles < 0 || !prm) return PICASSO_ERR_INVALID_ARGUMENT;
    // the separate calls: same results, two passes (validation included)
    auto separate = [&]() {
        picasso_status s2 = picasso_apic_p2g(sd, num_particles, 3, x_p, m_p, c_p, m_i, mu_i, exec);
        if (s2) return s2;
        return picasso_grid_update(&sd->mesh, m_i, mu_i, f_i, prm, u_i, u64_i, exec);
    };
    const picasso_bins* bins = exec ? exec->bins : nullptr;
    const bool eligible = bins && staggered_dim(sd->location) < 0 && num_particles > 0 &&
                          m_p.dtype == PICASSO_F32 && m_i.dtype == PICASSO_I64_FIXED &&
                          mu_i.dtype == PICASSO_I64_FIXED && u_i.dtype == PICASSO_F32 &&
                          (!f_i.data || f_i.dtype == PICASSO_F64) &&
                          (!u64_i.data || u64_i.dtype == PICASSO_F64) &&
                          bins->order == sd->order && bins->location == sd->location;
    if (!eligible) return separate();
    if ((st = validate_pfield(num_particles, x_p, PICASSO_F64))) return st;
    if ((st = validate_pfield(num_particles, m_p, PICASSO_F32))) return st;
    if ((st = validate_pfield(num_particles, c_p, PICASSO_F32))) return st;
    if ((st = validate_gfield(m_i, PICASSO_I64_FIXED))) return st;
    if ((st = validate_gfield(mu_i, PICASSO_I64_FIXED))) return st;
    if ((st = validate_gfield(u_i, PICASSO_F32))) return st;
    if (f_i.data && (st = validate_gfield(f_i, PICASSO_F64))) return st;
    if (u64_i.data && (st = validate_gfield(u64_i, PICASSO_F64))) return st;
    TileP tp;
    if (!make_tilep(mp, sd->order, *bins, &tp)) return PICASSO_ERR_INVALID_ARGUMENT;
    int64_t need = 0;
    if ((st = picasso_apic_p2g_update_workspace(bins, &need))) return st;
    if (!fused_update_fits(tp, sd->order)) return separate();
    if (!workspace || workspace_bytes < need || reinterpret_cast<uintptr_t>(workspace) % 4)
        return PICASSO_ERR_INVALID_ARGUMENT;
    FusedUpdate F;
    if ((st = make_grid_update(&sd->mesh, prm, m_i, mu_i, f_i, &F.P))) return st;
    F.gf = make_gfield(f_i);
    F.gu = make_gfield(u_i);
    F.gu64 = make_gfield(u64_i);
    F.count = static_cast<uint32_t*>(workspace);
    cudaStream_t s = stream_of(exec);
    PB_CUDA_TRY(cudaMemsetAsync(workspace, 0, (size_t)need, s));
    // nodes of regions that no work item touches get the update of an
    // empty node, 0
    {
        const unsigned blocks = grid_for(tp.ntiles * 8, 256, 148LL * 16);
        if (sd->order == 1) zero_untouched_regions_kernel<1><<<blocks, 256, 0, s>>>(mp, tp, F);
        else if (sd->order == 2) zero_untouched_regions_kernel<2><<<blocks, 256, 0, s>>>(mp, tp, F);
        else zero_untouched_regions_kernel<3><<<blocks, 256, 0, s>>>(mp, tp, F);
        if ((st = check_launch())) return st;
    }
    const PField x = make_pfield(x_p), m = make_pfield(m_p), c = make_pfield(c_p);
    GField gm = make_gfield(m_i), gmu = make_gfield(mu_i);
    gm.overflow = gmu.overflow = exec->overflow_count;
    bool handled = false;
    st = apic_p2g_tiled(mp, sd->order, 3, Form::F32Fixed, num_particles, x, m, c, gm, gmu, *bins,
                        exec->error_count, s, &handled, &F, -1, nullptr);
    if (st || handled) return st;
    // the tiled kernel does not take these particles (layout, tile size):
    // the fill of u above is overwritten by the separate update
    return separate();
}
