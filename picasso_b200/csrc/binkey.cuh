// Sort key of a particle: the (tile, bin-in-tile) of its stencil start, as
// the cell sort orders particles.  Shared by the sort and by the kernels that
// emit the key of a particle they have just moved (G2P with advection).
#pragma once

#include "common.cuh"

namespace pb {

struct BinP {  // bins of one mesh / spline / tile shape
    MeshP mp;
    int order;
    int tile[3];
    int tshift[3];  // log2(tile[d]) when tile[d] is a power of two, else -1
    int nt[3];
    int nb[3];
    uint32_t tsize;
    uint32_t nkeys;  // valid keys are < nkeys; out-of-mesh particles get nkeys
};

// Key of a particle from the (unwrapped) stencil starts s[d] of its spline.
__device__ __forceinline__ uint32_t key_from_starts(const BinP& bp, const int s[3])
{
    const int K = bp.order + 1;
    int q[3], r[3];  // tile index and bin inside the tile
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        int b;
        if (bp.mp.periodic[d]) {
            // (s - own_lo) mod nb; one period covers every particle inside or
            // next to the owned box, the remainder the rest
            const int nb = bp.nb[d];
            b = s[d] - bp.mp.own_lo[d];
            if (b < 0) b += nb;
            else if (b >= nb) b -= nb;
            if ((unsigned)b >= (unsigned)nb) {
                b %= nb;
                if (b < 0) b += nb;
            }
        } else {
            if (s[d] < 0 || s[d] > bp.mp.ext[d] - K) return bp.nkeys;
            b = s[d];
        }
        if (bp.tshift[d] >= 0) {
            q[d] = b >> bp.tshift[d];
            r[d] = b & (bp.tile[d] - 1);
        } else {
            q[d] = b / bp.tile[d];
            r[d] = b - q[d] * bp.tile[d];
        }
    }
    const uint32_t tl = ((uint32_t)q[0] * bp.nt[1] + (uint32_t)q[1]) * bp.nt[2] + (uint32_t)q[2];
    const uint32_t ll = ((uint32_t)r[0] * bp.tile[1] + (uint32_t)r[1]) * bp.tile[2] + (uint32_t)r[2];
    return tl * bp.tsize + ll;
}

__device__ __forceinline__ uint32_t particle_key(const BinP& bp, const double xs[3])
{
    const int first = (bp.order == 1) ? 0 : -1;
    const double shift = (bp.order == 2) ? 0.5 : 0.0;
    int s[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double x0 = logical_coord(xs[d], bp.mp.lo[d], bp.mp.rdx[d], shift);
        s[d] = (int)floor(x0) + first;
    }
    return key_from_starts(bp, s);
}

// BinP of a spline (mesh, order, location) and tile shape; *ntiles = the
// number of tiles.  PICASSO_ERR_OUT_OF_RANGE when the keys do not fit 32 bits.
picasso_status make_binp(const picasso_spline* sd, const int32_t tile[3], BinP* bp,
                         int64_t* ntiles);

}  // namespace pb
