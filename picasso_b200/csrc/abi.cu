// Library-level C-ABI entry points (version, status strings) and the host
// validation of the descriptors shared by every transfer entry point.
#include <cmath>

#include "common.cuh"

namespace pb {

static thread_local cudaError_t g_last_cuda_error = cudaSuccess;

void set_last_cuda_error(cudaError_t e) { g_last_cuda_error = e; }

picasso_status check_launch()
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_cuda_error(e);
        return PICASSO_ERR_CUDA;
    }
    return PICASSO_OK;
}

picasso_status validate_mesh(const picasso_mesh* m)
{
    if (!m) return PICASSO_ERR_INVALID_ARGUMENT;
    for (int d = 0; d < 3; ++d) {
        if (m->extent[d] <= 0) return PICASSO_ERR_INVALID_ARGUMENT;
        if (!(m->cell_size[d] > 0.0) || !std::isfinite(m->cell_size[d]))
            return PICASSO_ERR_INVALID_ARGUMENT;
        if (!std::isfinite(m->low_corner[d])) return PICASSO_ERR_INVALID_ARGUMENT;
        if (m->periodic[d]) {
            if (m->own_extent[d] <= 0 || m->own_begin[d] < 0 ||
                m->own_begin[d] + m->own_extent[d] > m->extent[d])
                return PICASSO_ERR_INVALID_ARGUMENT;
        }
    }
    return PICASSO_OK;
}

picasso_status make_mesh(const picasso_spline* sd, MeshP* mp)
{
    if (!sd) return PICASSO_ERR_INVALID_ARGUMENT;
    picasso_status st = validate_mesh(&sd->mesh);
    if (st) return st;
    if (sd->order < 1 || sd->order > 3) return PICASSO_ERR_INVALID_ARGUMENT;
    if (sd->location < PICASSO_NODE || sd->location > PICASSO_EDGE_K)
        return PICASSO_ERR_INVALID_ARGUMENT;
    double off[3];
    entity_offset(sd->location, off);
    for (int d = 0; d < 3; ++d) {
        const double cs = sd->mesh.cell_size[d];
        const double lo = sd->mesh.low_corner[d] + (0.0 + off[d]) * cs;
        const double lo1 = sd->mesh.low_corner[d] + (1.0 + off[d]) * cs;
        mp->ext[d] = sd->mesh.extent[d];
        mp->own_lo[d] = sd->mesh.own_begin[d];
        mp->own_n[d] = sd->mesh.own_extent[d];
        mp->periodic[d] = sd->mesh.periodic[d] ? 1 : 0;
        mp->lo[d] = lo;
        mp->dx[d] = lo1 - lo;
        mp->rdx[d] = 1.0 / mp->dx[d];
    }
    return PICASSO_OK;
}

picasso_status validate_pfield(int64_t n, const picasso_particle_field& f, int dtype_a,
                               int dtype_b)
{
    if (!f.data && n > 0) return PICASSO_ERR_INVALID_ARGUMENT;
    if (f.dtype != dtype_a && f.dtype != dtype_b) return PICASSO_ERR_INVALID_ARGUMENT;
    if (f.vector_shift < 0) return PICASSO_ERR_INVALID_ARGUMENT;
    if (f.vector_shift < 62 && f.tile_stride < 0) return PICASSO_ERR_INVALID_ARGUMENT;
    if (f.comp_stride < 0) return PICASSO_ERR_INVALID_ARGUMENT;
    return PICASSO_OK;
}

picasso_status validate_gfield(const picasso_grid_field& f, int dtype_a, int dtype_b)
{
    if (!f.data) return PICASSO_ERR_INVALID_ARGUMENT;
    if (f.dtype != dtype_a && f.dtype != dtype_b) return PICASSO_ERR_INVALID_ARGUMENT;
    if (f.dtype == PICASSO_I64_FIXED && (f.fixed_bits < 0 || f.fixed_bits > 62))
        return PICASSO_ERR_INVALID_ARGUMENT;
    for (int d = 0; d < 4; ++d)
        if (f.stride[d] < 0) return PICASSO_ERR_INVALID_ARGUMENT;
    return PICASSO_OK;
}

}  // namespace pb

extern "C" {

const char* picasso_version(void) { return "picasso_b200 0.1.0 (sm_100a)"; }

const char* picasso_status_string(picasso_status s)
{
    switch (s) {
        case PICASSO_OK: return "ok";
        case PICASSO_ERR_INVALID_ARGUMENT: return "invalid argument";
        case PICASSO_ERR_UNSUPPORTED: return "unsupported combination";
        case PICASSO_ERR_CUDA: return "CUDA error";
        case PICASSO_ERR_OUT_OF_RANGE: return "out of range";
        case PICASSO_ERR_TIMEOUT: return "device wait timed out";
        case PICASSO_ERR_NO_DEVICE: return "no usable device";
    }
    return "unknown status";
}

const char* picasso_last_cuda_error(void)
{
    return pb::g_last_cuda_error == cudaSuccess ? "" : cudaGetErrorString(pb::g_last_cuda_error);
}

}  // extern "C"
