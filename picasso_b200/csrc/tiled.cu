// Shared-memory tiled P2G / G2P for particles sorted by picasso_cell_sort.
#include "common.cuh"
#include "transfer.cuh"

namespace pb {

picasso_status apic_p2g_tiled(const MeshP&, int, int, Form, int64_t, const PField&,
                              const PField&, const PField&, const GField&, const GField&,
                              const picasso_bins&, int*, cudaStream_t, bool* handled)
{
    *handled = false;
    return PICASSO_OK;
}

picasso_status apic_g2p_tiled(const MeshP&, int, int, bool, int64_t, const PField&,
                              const GField&, const PField&, const picasso_bins&, int*,
                              cudaStream_t, bool* handled)
{
    *handled = false;
    return PICASSO_OK;
}

}  // namespace pb
