// Batched independent APIC problems in persistent launches.
//
// Every instance contributes work items to one queue, phase-major:
//   phase 0  fill      zero m_i and mu_i            (kNodeItem nodes per item)
//   phase 1  P2G       one sorted work item of the instance's bins
//   phase 2  velocity  u = mu / m, FP64 division    (kNodeItem nodes per item)
//   phase 3  G2P       one sorted work item
// and, inside a phase, instances in decreasing particle count (largest first,
// so the tail of a phase is made of small items).  Persistent single-warp
// CTAs take items from the queue with an atomic counter.
//
// FUSED mode runs the whole step in one launch.  An item of phase p > 0 of
// instance i first waits until every item of phase p - 1 of instance i has
// finished (per-instance completion counters).  This cannot deadlock: items
// leave the queue in order and all items an item depends on left it earlier,
// so they are held by warps that are already running and that only wait for
// items that left the queue before theirs.  Each wait is bounded all the same
// (kWaitPolls polls); a wait that runs out sets the batch's status word and
// every later wait returns at once, so the launch always ends.
// PHASED mode runs one launch per phase (no waits, each launch with the
// registers of its own phase only).
//
// Work items reuse the single-call bodies: tiled P2G / G2P (tiled.cuh) for the
// precision form, the per-particle plain transfers (plain.cuh) on sorted
// particles for FP64, the per-node velocity update (gridops.cuh).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "gridops.cuh"
#include "plain.cuh"
#include "tiled.cuh"

namespace pb {

constexpr int kPhases = 4;
// P2G variants: the phased step runs one P2G kernel per variant, each with the
// registers of that variant alone.  Precision form: (order, lanes per
// particle); FP64: order.
constexpr int kVariants = 7;
constexpr int kVarOrder[kVariants] = {1, 1, 1, 2, 2, 2, 3};
constexpr int kVarLanes[kVariants] = {1, 2, 4, 1, 2, 4, 4};

__host__ __device__ constexpr int p2g_variant(bool f32, int order, int lpp)
{
    return f32 ? (order == 3 ? 6 : (order - 1) * 3 + (lpp == 1 ? 0 : (lpp == 2 ? 1 : 2)))
               : order - 1;
}
constexpr int kNodeItem = 4096;           // nodes per fill / velocity item
constexpr unsigned kWaitPolls = 1u << 22;  // default bound: ~1-2 s of polling

struct BInst {
    P2GArgs p2g;  // tiled P2G arguments (precision form)
    G2PArgs g2p;  // tiled G2P arguments (precision form)
    PField x, m, c;
    GField gm, gmu, gu;
    Box full, owned;
    double thr, inv_m, inv_mu;
    int64_t n;
    int order, lpp;
    uint32_t nitems[kPhases];
};

struct BatchDev {
    const BInst* inst;
    const uint32_t* qbegin;  // kPhases * count + 1 queue offsets, phase-major
    const int32_t* rank;     // kPhases * count: instance at rank r of phase p
    uint32_t* done;          // kPhases * count completion counters
    uint32_t* head;          // queue heads: one per phase launch, then one per P2G
                             // variant launch (fused mode uses head[0])
    int* status;             // bit 0: a dependency wait ran out; bit 1: cancelled
    unsigned wait_polls;     // polls before a dependency wait gives up
    int count;
};

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Lane 0 polls until *counter reaches target; false if the wait ran out (or an
// earlier one did).
__device__ bool wait_for(const BatchDev& B, const uint32_t* counter, uint32_t target, int lane)
{
    int ok = 1;
    if (lane == 0) {
        unsigned polls = 0;
        while (ld_acquire(counter) < target) {
            if (*(volatile int*)B.status != 0 || ++polls > B.wait_polls) {
                atomicOr(B.status, 1);
                ok = 0;
                break;
            }
            __nanosleep(256);
        }
    }
    ok = __shfl_sync(kFull, ok, 0);
    __threadfence();  // the other lanes read what the producers wrote
    return ok != 0;
}

// Item bodies.  `tid` in [0, NT) numbers the NT threads that share an item
// (one warp, or the CTA when NT > 32).
template <bool F32, int NT>
__device__ void fill_item(const BInst& I, uint32_t local, int tid)
{
    using T = typename std::conditional<F32, long long, double>::type;
    const int64_t total = I.full.count();
    const int64_t e0 = (int64_t)local * kNodeItem, e1 = min(e0 + kNodeItem, total);
    for (int64_t e = e0 + tid; e < e1; e += NT) {
        int i, j, k;
        I.full.at(e, i, j, k);
        *I.gm.ptr<T>(i, j, k, 0) = T(0);
#pragma unroll
        for (int c = 0; c < 3; ++c) *I.gmu.ptr<T>(i, j, k, c) = T(0);
    }
    if (local == 0 && tid == 0 && I.p2g.err) {  // particles the sort left out of every tile
        const int64_t n_valid = __ldg(I.p2g.tp.off + I.p2g.tp.ntiles);
        if (I.n > n_valid) atomicAdd(I.p2g.err, (int)(I.n - n_valid));
    }
}

template <bool F32, int NT>
__device__ void velocity_item(const BInst& I, uint32_t local, int tid)
{
    using MT = typename std::conditional<F32, long long, double>::type;
    using UT = typename std::conditional<F32, float, double>::type;
    const int64_t total = I.owned.count();
    const int64_t e0 = (int64_t)local * kNodeItem, e1 = min(e0 + kNodeItem, total);
    GField none;
    none.data = nullptr;
    for (int64_t e = e0 + tid; e < e1; e += NT) {
        int i, j, k;
        I.owned.at(e, i, j, k);
        velocity_node<MT, UT, 3, true>(I.gm, I.gmu, I.gu, none, i, j, k, I.thr, I.inv_m,
                                       I.inv_mu);
    }
}

// Item bodies called out of line: each variant gets its own register
// allocation instead of one allocation for the union of all inlined variants.
template <int ORDER, int LPP>
__device__ __noinline__ void p2g_item_call(const P2GArgs& A, int64_t t, int64_t a, int64_t b,
                                           float* smem, int* stage_base)
{
    p2g_item<ORDER, LPP>(A, t, a, b, smem, stage_base);
}

template <int ORDER, int NT>
__device__ __noinline__ void g2p_item_call(const G2PArgs& A, int64_t t, int64_t a, int64_t b,
                                           float4* tile, int tid)
{
    g2p_item<ORDER, NT>(A, t, a, b, tile, tid);
}

template <int ORDER, int NT>
__device__ __noinline__ void plain_p2g_call(const BInst& I, int64_t a, int64_t b, int tid)
{
    for (int64_t p = a + tid; p < b; p += NT)
        apic_p2g_particle<ORDER, 3, false, double, double, AccF64>(
            I.p2g.mp, p, I.x, I.m, I.c, I.gm, I.gmu, -1, 0.0, 0.0, I.p2g.err);
}

template <int ORDER, int NT>
__device__ __noinline__ void plain_g2p_call(const BInst& I, int64_t a, int64_t b, int tid)
{
    for (int64_t p = a + tid; p < b; p += NT)
        apic_g2p_particle<ORDER, 3, false, double, double, double, true>(I.g2p.mp, p, I.x, I.gu,
                                                                         I.c, -1, I.g2p.err);
}

// Copies an argument block into shared memory with the NT threads of the
// item: the item bodies then read the instance's mesh and tile parameters
// from shared memory instead of global memory on every particle.
template <class T, int NT>
__device__ __forceinline__ const T& stage_args(const T& src, T* dst, int tid)
{
    static_assert(sizeof(T) % 4 == 0, "argument blocks are word-sized");
    const uint32_t* s = reinterpret_cast<const uint32_t*>(&src);
    uint32_t* d = reinterpret_cast<uint32_t*>(dst);
    for (int w = tid; w < (int)(sizeof(T) / 4); w += NT) d[w] = __ldg(s + w);
    if (NT == 32) __syncwarp();
    else __syncthreads();
    return *dst;
}

// Precision-form P2G items are single-warp (NT = 32); FP64 items any NT.
// VAR >= 0: every item of this kernel is of P2G variant VAR (inlined body);
// VAR < 0: any variant (out-of-line bodies).
template <bool F32, int NT, int VAR>
__device__ void p2g_batch_item(const BInst& I, uint32_t local, float* smem, int* stage_base,
                               P2GArgs* args, int tid)
{
    int64_t t, a, b;
    if (!item_range(I.p2g.tp, local, t, a, b)) return;
    if constexpr (VAR >= 0) {
        constexpr int O = F32 ? kVarOrder[VAR] : VAR + 1;
        if constexpr (F32) {
            static_assert(NT == 32, "tiled P2G items are single-warp");
            const P2GArgs& A = stage_args<P2GArgs, NT>(I.p2g, args, tid);
            p2g_item<O, kVarLanes[VAR]>(A, t, a, b, smem, stage_base);
        } else {
            for (int64_t p = a + tid; p < b; p += NT)
                apic_p2g_particle<O, 3, false, double, double, AccF64>(
                    I.p2g.mp, p, I.x, I.m, I.c, I.gm, I.gmu, -1, 0.0, 0.0, I.p2g.err);
        }
    } else if constexpr (F32) {
        static_assert(!F32 || NT == 32, "tiled P2G items are single-warp");
        const int key = I.order * 8 + I.lpp;
        const P2GArgs& A = stage_args<P2GArgs, NT>(I.p2g, args, tid);
        switch (key) {
            case 1 * 8 + 1: p2g_item_call<1, 1>(A, t, a, b, smem, stage_base); break;
            case 1 * 8 + 2: p2g_item_call<1, 2>(A, t, a, b, smem, stage_base); break;
            case 1 * 8 + 4: p2g_item_call<1, 4>(A, t, a, b, smem, stage_base); break;
            case 2 * 8 + 1: p2g_item_call<2, 1>(A, t, a, b, smem, stage_base); break;
            case 2 * 8 + 2: p2g_item_call<2, 2>(A, t, a, b, smem, stage_base); break;
            case 2 * 8 + 4: p2g_item_call<2, 4>(A, t, a, b, smem, stage_base); break;
            default: p2g_item_call<3, 4>(A, t, a, b, smem, stage_base); break;
        }
    } else {
        if (I.order == 1) plain_p2g_call<1, NT>(I, a, b, tid);
        else if (I.order == 2) plain_p2g_call<2, NT>(I, a, b, tid);
        else plain_p2g_call<3, NT>(I, a, b, tid);
    }
}

template <bool F32, int NT>
__device__ void g2p_batch_item(const BInst& I, uint32_t local, float* smem, G2PArgs* args,
                               int tid)
{
    int64_t t, a, b;
    if (!item_range(I.g2p.tp, local, t, a, b)) return;  // uniform over the NT threads
    if constexpr (F32) {
        float4* tile = reinterpret_cast<float4*>(smem);
        const int order = I.order;
        const G2PArgs& A = stage_args<G2PArgs, NT>(I.g2p, args, tid);
        if (order == 1) g2p_item_call<1, NT>(A, t, a, b, tile, tid);
        else if (order == 2) g2p_item_call<2, NT>(A, t, a, b, tile, tid);
        else g2p_item_call<3, NT>(A, t, a, b, tile, tid);
        if (NT == 32) __syncwarp();  // the next item rewrites args
        else __syncthreads();
    } else {
        if (I.order == 1) plain_g2p_call<1, NT>(I, a, b, tid);
        else if (I.order == 2) plain_g2p_call<2, NT>(I, a, b, tid);
        else plain_g2p_call<3, NT>(I, a, b, tid);
    }
}

// Launch shape of each kernel variant.  PMASK: phases it runs (0xF = fused).
// Fused and precision-form P2G kernels are single-warp CTAs (items are
// per-warp); fill and velocity take 256 threads per item, the other phases
// 128.
template <bool F32, int PMASK, int VAR = -1>
struct BatchShape {
    static constexpr int threads = (PMASK == 0xF || (F32 && PMASK == 0x2)) ? 32
                                   : (PMASK == 0x1 || PMASK == 0x4)       ? 256
                                                                          : 128;
    // a single-variant precision-form P2G kernel gets the occupancy of the
    // single-call kernel of that variant
    static constexpr int min_blocks =
        threads == 32 ? ((VAR >= 0 && F32) ? P2GOccupancy<kVarOrder[VAR >= 0 ? VAR : 0],
                                                          kVarLanes[VAR >= 0 ? VAR : 0]>::value
                                           : 8)
                      : (!F32 && threads == 128 ? 3 : 4);
};

template <bool F32, int PMASK, int VAR = -1>
__global__ void __launch_bounds__(BatchShape<F32, PMASK, VAR>::threads,
                                  BatchShape<F32, PMASK, VAR>::min_blocks)
batch_kernel(BatchDev B, uint32_t qlo, uint32_t qhi, int slot)
{
    constexpr int NT = BatchShape<F32, PMASK, VAR>::threads;
    extern __shared__ __align__(16) float smem[];
    __shared__ int stage_base[kStageBases];
    __shared__ uint32_t s_item;
    __shared__ __align__(16) P2GArgs s_p2g;
    __shared__ __align__(16) G2PArgs s_g2p;
    const int tid = threadIdx.x;
    const int nk = kPhases * B.count;
    for (;;) {
        uint32_t w = 0;
        if (NT == 32) {
            if (tid == 0) w = qlo + atomicAdd(B.head + slot, 1u);
            w = __shfl_sync(kFull, w, 0);
        } else {
            if (tid == 0) s_item = qlo + atomicAdd(B.head + slot, 1u);
            __syncthreads();
            w = s_item;
            __syncthreads();  // every thread has read s_item before it is rewritten
        }
        if (w >= qhi) break;
        int lo = 0, hi = nk - 1;  // the queue range holding w
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(B.qbegin + mid) <= w) lo = mid;
            else hi = mid - 1;
        }
        const int ph = lo / B.count;
        const int i = __ldg(B.rank + lo);
        const uint32_t local = w - __ldg(B.qbegin + lo);
        const BInst& I = B.inst[i];
        bool run = true;
        if (PMASK == 0xF && ph > 0)
            run = wait_for(B, B.done + (ph - 1) * B.count + i, I.nitems[ph - 1], tid);
        if (run) {
            if constexpr ((PMASK & 0x1) != 0)
                if (ph == 0) fill_item<F32, NT>(I, local, tid);
            if constexpr ((PMASK & 0x2) != 0)
                if (ph == 1)
                    p2g_batch_item<F32, NT, VAR>(I, local, smem, stage_base, &s_p2g, tid);
            if constexpr ((PMASK & 0x4) != 0)
                if (ph == 2) velocity_item<F32, NT>(I, local, tid);
            if constexpr ((PMASK & 0x8) != 0)
                if (ph == 3) g2p_batch_item<F32, NT>(I, local, smem, &s_g2p, tid);
        }
        if (PMASK == 0xF) {
            __threadfence();  // this item's writes before its completion count
            __syncwarp();
            if (tid == 0) atomicAdd(B.done + ph * B.count + i, 1u);
        }
    }
}

}  // namespace pb

using namespace pb;

struct picasso_batch {
    int count = 0;
    bool f32 = false;
    int mode = 0;
    int device = 0;
    int smem[kPhases + 1] = {0, 0, 0, 0, 0};    // per phase, [kPhases] = fused
    int blocks[kPhases + 1] = {0, 0, 0, 0, 0};
    // phased P2G: one launch per variant over queue slots [var_lo, var_hi)
    int var_smem[kVariants] = {};
    int var_blocks[kVariants] = {};
    uint32_t var_lo[kVariants] = {}, var_hi[kVariants] = {};
    std::vector<uint32_t> qbegin;
    std::vector<picasso_batch_instance> inst;
    int64_t particles = 0;
    void* dmem = nullptr;
    BatchDev dev{};
    size_t counter_bytes = 0;  // done + head, cleared before every step
    cudaStream_t capture = nullptr;
    cudaGraphExec_t graph = nullptr;
};

namespace {

using pb::BInst;

template <bool F32, int PMASK, int VAR = -1>
picasso_status configure_kernel(int smem, int items, int* blocks)
{
    auto k = batch_kernel<F32, PMASK, VAR>;
    PB_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0, dev = 0, sms = 0;
    PB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, k, BatchShape<F32, PMASK, VAR>::threads, smem));
    PB_CUDA_TRY(cudaGetDevice(&dev));
    PB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (per_sm < 1) return PICASSO_ERR_UNSUPPORTED;
    *blocks = std::max(1, std::min(per_sm * sms, items));
    return PICASSO_OK;
}

// FP64 has variants 0..2 (orders 1..3) only.
template <bool F32, int VAR>
picasso_status configure_variant(picasso_batch* b)
{
    if constexpr (F32 || VAR < 3) {
        const int n = (int)(b->var_hi[VAR] - b->var_lo[VAR]);
        if (n) return configure_kernel<F32, 0x2, VAR>(b->var_smem[VAR], n, &b->var_blocks[VAR]);
    }
    return PICASSO_OK;
}

template <bool F32>
picasso_status configure(picasso_batch* b)
{
    picasso_status st;
    const int total = (int)b->qbegin.back();
    if ((st = configure_kernel<F32, 0xF>(b->smem[kPhases], total, &b->blocks[kPhases])))
        return st;
    int items[kPhases];
    for (int p = 0; p < kPhases; ++p)
        items[p] = (int)(b->qbegin[(p + 1) * b->count] - b->qbegin[p * b->count]);
    if ((st = configure_kernel<F32, 0x1>(b->smem[0], items[0], &b->blocks[0]))) return st;
    if ((st = configure_kernel<F32, 0x2>(b->smem[1], items[1], &b->blocks[1]))) return st;
    if ((st = configure_kernel<F32, 0x4>(b->smem[2], items[2], &b->blocks[2]))) return st;
    if ((st = configure_kernel<F32, 0x8>(b->smem[3], items[3], &b->blocks[3]))) return st;
    if ((st = configure_variant<F32, 0>(b))) return st;
    if ((st = configure_variant<F32, 1>(b))) return st;
    if ((st = configure_variant<F32, 2>(b))) return st;
    if ((st = configure_variant<F32, 3>(b))) return st;
    if ((st = configure_variant<F32, 4>(b))) return st;
    if ((st = configure_variant<F32, 5>(b))) return st;
    return configure_variant<F32, 6>(b);
}

template <bool F32, int VAR>
void launch_p2g_variant(const picasso_batch* b, cudaStream_t s)
{
    if constexpr (F32 || VAR < 3) {
        const uint32_t lo = b->var_lo[VAR], hi = b->var_hi[VAR];
        if (lo == hi) return;
        batch_kernel<F32, 0x2, VAR>
            <<<b->var_blocks[VAR], BatchShape<F32, 0x2, VAR>::threads, b->var_smem[VAR], s>>>(
                b->dev, lo, hi, kPhases + VAR);
    }
}

template <bool F32>
void launch_phase(const picasso_batch* b, int p, cudaStream_t s)
{
    const uint32_t lo = b->qbegin[p * b->count], hi = b->qbegin[(p + 1) * b->count];
    if (lo == hi) return;
    if (p == 1) {  // one launch per P2G variant, each with its own queue head
        launch_p2g_variant<F32, 0>(b, s);
        launch_p2g_variant<F32, 1>(b, s);
        launch_p2g_variant<F32, 2>(b, s);
        launch_p2g_variant<F32, 3>(b, s);
        launch_p2g_variant<F32, 4>(b, s);
        launch_p2g_variant<F32, 5>(b, s);
        launch_p2g_variant<F32, 6>(b, s);
        return;
    }
#define PB_PHASE(P, M)                                                                  \
    batch_kernel<F32, M><<<b->blocks[P], BatchShape<F32, M>::threads, b->smem[P], s>>>(    \
        b->dev, lo, hi, P)
    switch (p) {
        case 0: PB_PHASE(0, 0x1); break;
        case 1: PB_PHASE(1, 0x2); break;
        case 2: PB_PHASE(2, 0x4); break;
        default: PB_PHASE(3, 0x8); break;
    }
#undef PB_PHASE
}

picasso_status enqueue_step(const picasso_batch* b, cudaStream_t s)
{
    PB_CUDA_TRY(cudaMemsetAsync(b->dev.done, 0, b->counter_bytes, s));
    const uint32_t total = b->qbegin.back();
    if (b->mode == PICASSO_BATCH_FUSED) {
        if (b->f32)
            batch_kernel<true, 0xF><<<b->blocks[kPhases], 32, b->smem[kPhases], s>>>(b->dev, 0,
                                                                                   total, 0);
        else
            batch_kernel<false, 0xF><<<b->blocks[kPhases], 32, b->smem[kPhases], s>>>(b->dev, 0,
                                                                                    total, 0);
    } else {
        for (int p = 0; p < kPhases; ++p) {
            if (b->f32) launch_phase<true>(b, p, s);
            else launch_phase<false>(b, p, s);
        }
    }
    return check_launch();
}

// Validates one instance and fills its device descriptor; raises *smem to
// the instance's shared-memory need.
picasso_status make_instance(const picasso_batch_instance& in, bool f32, BInst* I,
                             int* smem_p2g, int* smem_g2p)
{
    picasso_status st;
    MeshP mp;
    if ((st = make_mesh(&in.spline, &mp))) return st;
    if (in.spline.location != PICASSO_NODE || in.num_particles < 0)
        return PICASSO_ERR_INVALID_ARGUMENT;
    const int pt = f32 ? PICASSO_F32 : PICASSO_F64;
    const int gt = f32 ? PICASSO_I64_FIXED : PICASSO_F64;
    if ((st = validate_pfield(in.num_particles, in.x_p, PICASSO_F64))) return st;
    if ((st = validate_pfield(in.num_particles, in.m_p, pt))) return st;
    if ((st = validate_pfield(in.num_particles, in.c_p, pt))) return st;
    if ((st = validate_gfield(in.m_i, gt))) return st;
    if ((st = validate_gfield(in.mu_i, gt))) return st;
    if ((st = validate_gfield(in.u_i, pt))) return st;
    const PField x = make_pfield(in.x_p), m = make_pfield(in.m_p), c = make_pfield(in.c_p);
    if (!packed_x(x) || !packed_m(m) || !packed_c(c)) return PICASSO_ERR_INVALID_ARGUMENT;
    const picasso_bins& bins = in.bins;
    if (bins.order != in.spline.order || bins.location != in.spline.location)
        return PICASSO_ERR_INVALID_ARGUMENT;
    const int order = in.spline.order;
    const int lpp = bins.p2g_lanes ? bins.p2g_lanes : default_lpp(order);
    if (f32 && !valid_lpp(order, lpp)) return PICASSO_ERR_INVALID_ARGUMENT;
    TileP tp;
    if (!make_tilep(mp, order, bins, &tp, f32 ? lpp : 0)) return PICASSO_ERR_INVALID_ARGUMENT;

    std::memset(static_cast<void*>(I), 0, sizeof(BInst));
    I->p2g.mp = mp;
    I->p2g.tp = tp;
    I->p2g.x = reinterpret_cast<const double*>(in.x_p.data);
    I->p2g.m = reinterpret_cast<const float*>(in.m_p.data);
    I->p2g.c = reinterpret_cast<const float*>(in.c_p.data);
    I->p2g.gm = make_gfield(in.m_i);
    I->p2g.gmu = make_gfield(in.mu_i);
    I->p2g.scale_m = f32 ? ldexpf(1.f, in.m_i.fixed_bits) : 0.f;
    I->p2g.scale_mu = f32 ? ldexpf(1.f, in.mu_i.fixed_bits) : 0.f;
    I->p2g.err = in.error_count;
    I->p2g.stag = -1;
    // element-wise flush: in the fused launch the next phase's items read the
    // accumulators once the P2G items have counted themselves done
    I->p2g.bulk_flush = 0;
    I->p2g.hp = HaloPeers{};
    I->g2p.hp = HaloPeers{};
    I->g2p.mp = mp;
    I->g2p.tp = tp;
    I->g2p.x = I->p2g.x;
    I->g2p.u = make_gfield(in.u_i);
    I->g2p.c = reinterpret_cast<float*>(in.c_p.data);
    I->g2p.err = in.error_count;
    I->g2p.stag = -1;
    I->x = x;
    I->m = m;
    I->c = c;
    I->gm = I->p2g.gm;
    I->gmu = I->p2g.gmu;
    I->gu = I->g2p.u;
    I->full = full_box(in.spline.mesh);
    I->owned = owned_box(in.spline.mesh);
    I->thr = in.mass_threshold;
    I->inv_m = f32 ? ldexp(1.0, -in.m_i.fixed_bits) : 1.0;
    I->inv_mu = f32 ? ldexp(1.0, -in.mu_i.fixed_bits) : 1.0;
    I->n = in.num_particles;
    I->order = order;
    I->lpp = lpp;
    const int64_t work = in.num_particles ? tp.ntiles + (in.num_particles + tp.chunk - 1) / tp.chunk
                                          : 0;
    const int64_t fill = (I->full.count() + kNodeItem - 1) / kNodeItem;
    const int64_t vel = (I->owned.count() + kNodeItem - 1) / kNodeItem;
    if (work > (1LL << 30) || fill > (1LL << 30)) return PICASSO_ERR_OUT_OF_RANGE;
    I->nitems[0] = (uint32_t)fill;
    I->nitems[1] = (uint32_t)work;
    I->nitems[2] = (uint32_t)vel;
    I->nitems[3] = (uint32_t)work;
    if (f32) {
        *smem_p2g = std::max(*smem_p2g, (int)p2g_warp_bytes(order, lpp, tp.P));
        *smem_g2p = std::max(*smem_g2p, (int)(sizeof(float4) * (size_t)tp.nodes));
    }
    return PICASSO_OK;
}

}  // namespace

extern "C" picasso_status picasso_batch_create(const picasso_batch_instance* instances,
                                               int32_t count, int32_t mode, picasso_batch** out)
{
    if (!out) return PICASSO_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!instances) return PICASSO_ERR_INVALID_ARGUMENT;
    if (count < 1 || (mode != PICASSO_BATCH_FUSED && mode != PICASSO_BATCH_PHASED))
        return PICASSO_ERR_INVALID_ARGUMENT;
    const bool f32 = instances[0].m_p.dtype == PICASSO_F32;
    std::vector<BInst> hinst(count);
    int smem_p2g = 0, smem_g2p = 0;
    for (int i = 0; i < count; ++i) {
        picasso_status st = make_instance(instances[i], f32, &hinst[i], &smem_p2g, &smem_g2p);
        if (st) return st;
    }
    if (std::max(smem_p2g, smem_g2p) > device_smem_optin()) return PICASSO_ERR_UNSUPPORTED;

    picasso_batch* b = new (std::nothrow) picasso_batch();
    if (!b) return PICASSO_ERR_OUT_OF_RANGE;
    b->count = count;
    b->f32 = f32;
    b->mode = mode;
    b->smem[1] = smem_p2g;
    b->smem[3] = smem_g2p;
    b->smem[kPhases] = std::max(smem_p2g, smem_g2p);
    b->inst.assign(instances, instances + count);
    // queue: phase-major, instances by decreasing particle count; in the P2G
    // phase grouped by variant first (one phased launch per variant)
    std::vector<int> var(count);
    for (int i = 0; i < count; ++i) var[i] = p2g_variant(f32, hinst[i].order, hinst[i].lpp);
    std::vector<int32_t> by_size(count);
    std::iota(by_size.begin(), by_size.end(), 0);
    std::stable_sort(by_size.begin(), by_size.end(), [&](int a, int c) {
        return instances[a].num_particles > instances[c].num_particles;
    });
    std::vector<int32_t> by_var(by_size);
    std::stable_sort(by_var.begin(), by_var.end(), [&](int a, int c) { return var[a] < var[c]; });
    std::vector<int32_t> rank((size_t)kPhases * count);
    for (int p = 0; p < kPhases; ++p) {
        const std::vector<int32_t>& order = p == 1 ? by_var : by_size;
        std::copy(order.begin(), order.end(), rank.begin() + (size_t)p * count);
    }
    b->qbegin.assign((size_t)kPhases * count + 1, 0);
    uint64_t q = 0;
    for (int p = 0; p < kPhases; ++p)
        for (int r = 0; r < count; ++r) {
            const int i = rank[(size_t)p * count + r];
            b->qbegin[(size_t)p * count + r] = (uint32_t)q;
            if (p == 1 && hinst[i].nitems[p]) {
                const int v = var[i];
                if (b->var_lo[v] == b->var_hi[v]) b->var_lo[v] = (uint32_t)q;
                b->var_hi[v] = (uint32_t)(q + hinst[i].nitems[p]);
                if (f32)
                    b->var_smem[v] = std::max(b->var_smem[v],
                                              (int)p2g_warp_bytes(hinst[i].order, hinst[i].lpp,
                                                                  hinst[i].p2g.tp.P));
            }
            q += hinst[i].nitems[p];
        }
    for (int i = 0; i < count; ++i) b->particles += instances[i].num_particles;
    if (q >= (1ULL << 31)) {
        delete b;
        return PICASSO_ERR_OUT_OF_RANGE;
    }
    b->qbegin.back() = (uint32_t)q;

    // device tables: instances | qbegin | rank | done + heads | status
    auto align = [](size_t v) { return (v + 255) & ~size_t(255); };
    const size_t o_inst = 0;
    const size_t o_q = align(o_inst + sizeof(BInst) * count);
    const size_t o_rank = align(o_q + sizeof(uint32_t) * b->qbegin.size());
    const size_t o_done = align(o_rank + sizeof(int32_t) * rank.size());
    b->counter_bytes = sizeof(uint32_t) * ((size_t)kPhases * count + kPhases + kVariants);
    const size_t o_status = align(o_done + b->counter_bytes);
    const size_t bytes = o_status + 256;
    auto fail = [&](cudaError_t e) {
        set_last_cuda_error(e);
        if (b->dmem) cudaFree(b->dmem);
        delete b;
        return PICASSO_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaGetDevice(&b->device)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&b->dmem, bytes)) != cudaSuccess) return fail(e);
    char* base = static_cast<char*>(b->dmem);
    if ((e = cudaMemcpy(base + o_inst, hinst.data(), sizeof(BInst) * count,
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(base + o_q, b->qbegin.data(), sizeof(uint32_t) * b->qbegin.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(base + o_rank, rank.data(), sizeof(int32_t) * rank.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(base + o_done, 0, b->counter_bytes)) != cudaSuccess ||
        (e = cudaMemset(base + o_status, 0, 256)) != cudaSuccess)
        return fail(e);
    b->dev.inst = reinterpret_cast<const BInst*>(base + o_inst);
    b->dev.qbegin = reinterpret_cast<const uint32_t*>(base + o_q);
    b->dev.rank = reinterpret_cast<const int32_t*>(base + o_rank);
    b->dev.done = reinterpret_cast<uint32_t*>(base + o_done);
    b->dev.head = b->dev.done + (size_t)kPhases * count;
    b->dev.status = reinterpret_cast<int*>(base + o_status);
    b->dev.wait_polls = kWaitPolls;
    b->dev.count = count;
    picasso_status st = f32 ? configure<true>(b) : configure<false>(b);
    if (st) {
        cudaFree(b->dmem);
        delete b;
        return st;
    }
    *out = b;
    return PICASSO_OK;
}

extern "C" picasso_status picasso_batch_step(picasso_batch* b, void* stream, int32_t use_graph)
{
    if (!b) return PICASSO_ERR_INVALID_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!use_graph) return enqueue_step(b, s);
    if (!b->graph) {
        if (!b->capture) PB_CUDA_TRY(cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking));
        PB_CUDA_TRY(cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal));
        picasso_status st = enqueue_step(b, b->capture);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->capture, &g);
        if (st) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        PB_CUDA_TRY(e);
        const cudaError_t ei = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        PB_CUDA_TRY(ei);
    }
    PB_CUDA_TRY(cudaGraphLaunch(b->graph, s));
    return PICASSO_OK;
}

extern "C" picasso_status picasso_batch_step_sequential(picasso_batch* b, void* stream)
{
    if (!b) return PICASSO_ERR_INVALID_ARGUMENT;
    for (const picasso_batch_instance& in : b->inst) {
        picasso_exec ex{stream, in.error_count, &in.bins};
        picasso_exec ex_nobins{stream, nullptr, nullptr};
        picasso_status st;
        if ((st = picasso_grid_fill(&in.spline.mesh, 1, in.m_i, 0.0, &ex_nobins))) return st;
        if ((st = picasso_grid_fill(&in.spline.mesh, 3, in.mu_i, 0.0, &ex_nobins))) return st;
        if ((st = picasso_apic_p2g(&in.spline, in.num_particles, 3, in.x_p, in.m_p, in.c_p,
                                   in.m_i, in.mu_i, &ex)))
            return st;
        picasso_grid_field none{};
        if ((st = picasso_grid_velocity(&in.spline.mesh, 3, in.m_i, in.mu_i, in.mass_threshold,
                                        in.u_i, none, &ex_nobins)))
            return st;
        if ((st = picasso_apic_g2p(&in.spline, in.num_particles, 3, in.x_p, in.u_i, in.c_p,
                                   &ex)))
            return st;
    }
    return PICASSO_OK;
}

extern "C" picasso_status picasso_batch_status(picasso_batch* b, void* stream)
{
    if (!b) return PICASSO_ERR_INVALID_ARGUMENT;
    PB_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    int flag = 0;
    PB_CUDA_TRY(cudaMemcpy(&flag, b->dev.status, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        PB_CUDA_TRY(cudaMemset(b->dev.status, 0, sizeof(int)));
        return PICASSO_ERR_TIMEOUT;
    }
    return PICASSO_OK;
}

extern "C" picasso_status picasso_batch_set_wait_limit(picasso_batch* b, uint32_t polls)
{
    if (!b) return PICASSO_ERR_INVALID_ARGUMENT;
    b->dev.wait_polls = polls;
    if (b->graph) {  // the captured launches hold the old limit
        int prev = 0;
        PB_CUDA_TRY(cudaGetDevice(&prev));
        PB_CUDA_TRY(cudaSetDevice(b->device));
        const cudaError_t e = cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        cudaSetDevice(prev);
        PB_CUDA_TRY(e);
    }
    return PICASSO_OK;
}

extern "C" picasso_status picasso_batch_cancel(picasso_batch* b, void* stream)
{
    if (!b) return PICASSO_ERR_INVALID_ARGUMENT;
    // one byte of the status word: bit 1 (cancelled); bit 0 keeps its meaning
    PB_CUDA_TRY(cudaMemsetAsync(b->dev.status, 2, 1, static_cast<cudaStream_t>(stream)));
    return PICASSO_OK;
}

extern "C" picasso_status picasso_batch_get_info(const picasso_batch* b, picasso_batch_info* info)
{
    if (!b || !info) return PICASSO_ERR_INVALID_ARGUMENT;
    info->count = b->count;
    info->precision_form = b->f32 ? 1 : 0;
    const int k = b->mode == PICASSO_BATCH_FUSED ? kPhases : 1;
    info->grid_blocks = b->blocks[k];
    info->smem_bytes = b->smem[k];
    for (int p = 0; p < kPhases; ++p)
        info->items[p] = (int64_t)b->qbegin[(size_t)(p + 1) * b->count] -
                         (int64_t)b->qbegin[(size_t)p * b->count];
    info->particles = b->particles;
    return PICASSO_OK;
}

extern "C" picasso_status picasso_batch_destroy(picasso_batch* b)
{
    if (!b) return PICASSO_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->capture) cudaStreamDestroy(b->capture);
    if (b->dmem) cudaFree(b->dmem);
    cudaSetDevice(prev);
    delete b;
    return PICASSO_OK;
}
