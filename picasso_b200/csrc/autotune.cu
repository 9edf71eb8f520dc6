// Native autotuner of the sorted (tiled) transfer step: for one instance's
// own particles it measures fill -> P2G -> velocity -> G2P for every
// candidate tile shape, work-item size and P2G lanes-per-particle, and
// returns the fastest.  A host-side composition of the public entry points
// (cell sort, permute, grid fill, APIC P2G, grid velocity, APIC G2P) on
// sorted copies of the particles, timed with CUDA events on the caller's
// stream.  Candidates: tiles (4,4,4) (4,4,8) (4,8,8) (8,8,8), work items of
// 1024 and 4096 particles, 1 or 2 lanes per particle (orders 1-2), 4 (order 3).
#include <vector>

#include "common.cuh"

namespace {

// Device buffers of one tuning run, released on every exit path.
struct Scratch {
    std::vector<void*> ptrs;
    ~Scratch()
    {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t get(T** out, size_t bytes)
    {
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes < 256 ? 256 : bytes);
        if (e == cudaSuccess) ptrs.push_back(p);
        *out = static_cast<T*>(p);
        return e;
    }
};

picasso_particle_field packed_member(void* data, int32_t dtype, int64_t row)
{
    picasso_particle_field f{};
    f.data = data;
    f.dtype = dtype;
    f.vector_shift = 0;
    f.tile_stride = row;
    f.comp_stride = 1;
    return f;
}

}  // namespace

using namespace pb;

extern "C" picasso_status picasso_autotune(const picasso_spline* sd, int64_t num_particles,
                                           picasso_particle_field x_p, picasso_particle_field m_p,
                                           picasso_particle_field c_p, picasso_grid_field m_i,
                                           picasso_grid_field mu_i, picasso_grid_field u_i,
                                           double mass_threshold, int32_t trials,
                                           picasso_tune_result* best, const picasso_exec* exec)
{
    MeshP mp;
    picasso_status st = make_mesh(sd, &mp);
    if (st) return st;
    if (!best || num_particles < 1 || trials < 1) return PICASSO_ERR_INVALID_ARGUMENT;
    if (staggered_dim(sd->location) >= 0) return PICASSO_ERR_UNSUPPORTED;
    if ((st = validate_pfield(num_particles, x_p, PICASSO_F64))) return st;
    if ((st = validate_pfield(num_particles, m_p, PICASSO_F32))) return st;
    if ((st = validate_pfield(num_particles, c_p, PICASSO_F32))) return st;
    if ((st = validate_gfield(m_i, PICASSO_I64_FIXED))) return st;
    if ((st = validate_gfield(mu_i, PICASSO_I64_FIXED))) return st;
    if ((st = validate_gfield(u_i, PICASSO_F32))) return st;
    const int64_t n = num_particles;
    cudaStream_t s = stream_of(exec);
    picasso_exec ex{};
    ex.stream = s;

    // sorted copies of the members in the packed layout of the tiled kernels
    Scratch mem;
    double* xs;
    float *ms, *cs;
    uint32_t *key, *perm;
    PB_CUDA_TRY(mem.get(&xs, sizeof(double) * 3 * n));
    PB_CUDA_TRY(mem.get(&ms, sizeof(float) * n));
    PB_CUDA_TRY(mem.get(&cs, sizeof(float) * 12 * n));
    PB_CUDA_TRY(mem.get(&key, sizeof(uint32_t) * n));
    PB_CUDA_TRY(mem.get(&perm, sizeof(uint32_t) * n));
    const picasso_particle_field xf = packed_member(xs, PICASSO_F64, 3);
    const picasso_particle_field mf = packed_member(ms, PICASSO_F32, 1);
    const picasso_particle_field cf = packed_member(cs, PICASSO_F32, 12);
    cudaEvent_t e0, e1;
    PB_CUDA_TRY(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return PICASSO_ERR_CUDA;
    }
    struct Events {
        cudaEvent_t a, b;
        ~Events()
        {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } evs{e0, e1};

    const int32_t tiles[4][3] = {{4, 4, 4}, {4, 4, 8}, {4, 8, 8}, {8, 8, 8}};
    const int32_t chunks[2] = {1024, 4096};
    const int32_t lanes_lo[2] = {1, 2}, lanes_cubic[1] = {4};
    const int32_t* lanes = sd->order == 3 ? lanes_cubic : lanes_lo;
    const int nlanes = sd->order == 3 ? 1 : 2;
    float best_ms = -1.f;

    for (const auto& tile : tiles) {
        int64_t ntiles = 1;
        for (int d = 0; d < 3; ++d) {
            const int64_t nb = sd->mesh.periodic[d] ? sd->mesh.own_extent[d] : sd->mesh.extent[d];
            ntiles *= (nb + tile[d] - 1) / tile[d];
        }
        int64_t ws_bytes = 0;
        if ((st = picasso_cell_sort_workspace(sd, n, tile, &ws_bytes))) return st;
        Scratch tmem;
        int64_t* toff;
        uint32_t* titems;
        void* ws;
        PB_CUDA_TRY(tmem.get(&toff, sizeof(int64_t) * (ntiles + 1)));
        PB_CUDA_TRY(tmem.get(&titems, sizeof(uint32_t) * (ntiles + 1)));
        PB_CUDA_TRY(tmem.get(&ws, (size_t)ws_bytes));
        for (int32_t chunk : chunks) {
            picasso_bins bins{};
            if ((st = picasso_cell_sort(sd, n, x_p, tile, chunk, key, perm, toff, titems, ws,
                                        ws_bytes, &bins, &ex)))
                return st;
            if ((st = picasso_permute(n, 3, perm, x_p, xf, &ex))) return st;
            if ((st = picasso_permute(n, 1, perm, m_p, mf, &ex))) return st;
            for (int li = 0; li < nlanes; ++li) {
                bins.p2g_lanes = lanes[li];
                picasso_exec bex = ex;
                bex.bins = &bins;
                // c_p is re-gathered before each candidate: G2P overwrites it
                auto step = [&]() -> picasso_status {
                    picasso_status r;
                    if ((r = picasso_grid_fill(&sd->mesh, 1, m_i, 0.0, &ex))) return r;
                    if ((r = picasso_grid_fill(&sd->mesh, 3, mu_i, 0.0, &ex))) return r;
                    if ((r = picasso_apic_p2g(sd, n, 3, xf, mf, cf, m_i, mu_i, &bex))) return r;
                    picasso_grid_field none{};
                    if ((r = picasso_grid_velocity(&sd->mesh, 3, m_i, mu_i, mass_threshold, u_i,
                                                   none, &ex)))
                        return r;
                    return picasso_apic_g2p(sd, n, 3, xf, u_i, cf, &bex);
                };
                if ((st = picasso_permute(n, 12, perm, c_p, cf, &ex))) return st;
                if ((st = step())) return st;  // warm-up
                PB_CUDA_TRY(cudaEventRecord(e0, s));
                for (int t = 0; t < trials; ++t)
                    if ((st = step())) return st;
                PB_CUDA_TRY(cudaEventRecord(e1, s));
                PB_CUDA_TRY(cudaEventSynchronize(e1));
                float ms_total = 0.f;
                PB_CUDA_TRY(cudaEventElapsedTime(&ms_total, e0, e1));
                const float per = ms_total / trials;
                if (best_ms < 0.f || per < best_ms) {
                    best_ms = per;
                    for (int d = 0; d < 3; ++d) best->tile[d] = tile[d];
                    best->chunk = chunk;
                    best->p2g_lanes = lanes[li];
                    best->step_ms = per;
                }
            }
        }
        PB_CUDA_TRY(cudaStreamSynchronize(s));  // before the tile's buffers are freed
    }
    return PICASSO_OK;
}
