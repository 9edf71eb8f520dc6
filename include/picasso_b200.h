/*
 * picasso_b200.h -- C ABI of the B200 particle/grid transfer library.
 *
 * The library re-implements the particle-to-grid (P2G) and grid-to-particle
 * (G2P) transfers of Picasso (APIC and PolyPIC) on the uniform Cartesian mesh,
 * the B-spline stencil evaluation they use, the particle cell-sort that feeds
 * the tiled kernels, the grid velocity update between P2G and G2P, and the
 * batched 3x3 linear algebra used by PolyPIC.
 *
 * Every entry point takes plain pointers, sizes and POD descriptors; device
 * pointers are CUDA device memory on the current device.  Calls over zero
 * particles are valid no-ops (their particle pointers may then be NULL).  All launches are
 * asynchronous on the stream in picasso_exec; a returned PICASSO_OK means the
 * arguments were valid and the work was enqueued.  No exceptions cross the ABI.
 *
 * Reference interfaces replaced (paths inside the Picasso source tree):
 *   Picasso::APIC::p2g / g2p          src/Picasso_APIC.hpp:55-544
 *   Picasso::PolyPIC::p2g / g2p       src/Picasso_PolyPIC.hpp:39-359
 *   Picasso::createSpline             src/Picasso_ParticleInterpolation.hpp:88-105
 *   GridOperator::apply over particles (particle loop + ScatterView zero /
 *     contribute)                     src/Picasso_GridOperator.hpp:403-429,521-591,612-642
 *   LinearAlgebra::operator! / inverse (3x3)
 *                                     src/Picasso_BatchedLinearAlgebra.hpp:4337-4350,4626-4686
 */
#ifndef PICASSO_B200_H
#define PICASSO_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define PICASSO_API __attribute__((visibility("default")))
#else
#define PICASSO_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                             */
/* ------------------------------------------------------------------------ */
typedef enum picasso_status {
    PICASSO_OK = 0,
    PICASSO_ERR_INVALID_ARGUMENT = 1, /* bad descriptor, size, dtype combination */
    PICASSO_ERR_UNSUPPORTED = 2,      /* valid but not implemented combination */
    PICASSO_ERR_CUDA = 3,             /* a CUDA runtime call failed */
    PICASSO_ERR_OUT_OF_RANGE = 4,     /* key / index range exceeds the format */
    PICASSO_ERR_TIMEOUT = 5,          /* a bounded device wait gave up */
    PICASSO_ERR_NO_DEVICE = 6         /* no usable sm_100 device */
} picasso_status;

/* Element types of particle and grid arrays. */
typedef enum picasso_dtype {
    PICASSO_F64 = 0,
    PICASSO_F32 = 1,
    PICASSO_I64_FIXED = 2 /* signed 64-bit fixed point: value = raw * 2^-fixed_bits */
} picasso_dtype;

/* Mesh entity the spline is defined on (Picasso FieldLocation / Cabana::Grid
 * entity types).  Face<D>: on nodes along D, on cell centres along the other
 * two dimensions.  Edge<D>: on cell centres along D, on nodes elsewhere. */
typedef enum picasso_location {
    PICASSO_NODE = 0,
    PICASSO_CELL = 1,
    PICASSO_FACE_I = 2,
    PICASSO_FACE_J = 3,
    PICASSO_FACE_K = 4,
    PICASSO_EDGE_I = 5,
    PICASSO_EDGE_J = 6,
    PICASSO_EDGE_K = 7
} picasso_location;

/* ------------------------------------------------------------------------ */
/* Descriptors                                                              */
/* ------------------------------------------------------------------------ */

/* Local uniform mesh.  Index space of the grid arrays passed to a call: entity
 * (i,j,k) with 0 <= i < extent[0] etc. (ghost layers included, as in a
 * Cabana::Grid local array).  Physical coordinate of entity (i,j,k) along d:
 *     low_corner[d] + (index[d] + offset_d(location)) * cell_size[d]
 * with offset 0 (node-aligned) or 0.5 (cell-centre-aligned).
 * periodic[d] != 0: stencil indices are wrapped into
 *     [own_begin[d], own_begin[d] + own_extent[d])
 * so that all periodic images accumulate into the owned entity (what the
 * reference's halo Sum scatter does after P2G and its halo gather provides
 * before G2P).  Non-periodic: a particle whose stencil leaves
 * [0, extent[d]) is skipped and counted in picasso_exec.error_count. */
typedef struct picasso_mesh {
    int32_t extent[3];
    int32_t own_begin[3];
    int32_t own_extent[3];
    int32_t periodic[3];
    double low_corner[3];
    double cell_size[3];
} picasso_mesh;

/* Equivalent of createSpline(Location, InterpolationOrder<order>, mesh, x):
 * the spline is evaluated inside the kernels from each particle position. */
typedef struct picasso_spline {
    picasso_mesh mesh;
    int32_t location; /* picasso_location */
    int32_t order;    /* 1 (linear), 2 (quadratic), 3 (cubic) */
} picasso_spline;

/* Particle member.  Element (p, c) of a member with C components lives at
 *   data + ((p >> vector_shift) * tile_stride + c * comp_stride
 *           + (p & ((1 << vector_shift) - 1)))        [in elements]
 * which covers plain structure-of-arrays (vector_shift >= 62, comp_stride =
 * number of particles), array-of-structures (vector_shift = 0, tile_stride =
 * C, comp_stride = 1) and Cabana AoSoA storage (vector_shift = log2 of the
 * vector length, tile_stride = elements per SoA, comp_stride = vector length,
 * data = the member's first element).  Matrix members c_p(r, d) use component
 * index c = r * ncomp + d, which is Cabana's row-major matrix member layout. */
typedef struct picasso_particle_field {
    void* data;
    int32_t dtype;        /* picasso_dtype (F64 or F32) */
    int32_t vector_shift; /* log2 of the AoSoA vector length; >= 62 for SoA */
    int64_t tile_stride;
    int64_t comp_stride;
} picasso_particle_field;

/* Grid array: element (i, j, k, comp) at data + i*stride[0] + j*stride[1] +
 * k*stride[2] + comp*stride[3] (elements).  A Cabana::Grid array (Kokkos
 * LayoutRight) has stride = {ny*nz*nc, nz*nc, nc, 1}. */
typedef struct picasso_grid_field {
    void* data;
    int32_t dtype;      /* picasso_dtype */
    int32_t fixed_bits; /* PICASSO_I64_FIXED only: fraction bits (0..62) */
    int64_t stride[4];
} picasso_grid_field;

/* Particles sorted by stencil bin in tiles (output of picasso_cell_sort after
 * the particle arrays were permuted with picasso_permute).  With it the P2G
 * and G2P entry points use the shared-memory tiled kernels (FP32 precision
 * form, collocated 3-component fields, packed storage: x_p (N,3) FP64,
 * m_p (N) FP32, c_p (N,4,3) FP32 contiguous; other calls take the plain
 * path).  Work items are chunks of at most `chunk` particles of one tile. */
typedef struct picasso_bins {
    int32_t tile[3];             /* bins per tile along i, j, k */
    int32_t num_tiles[3];        /* tiles along i, j, k */
    int32_t bin_extent[3];       /* bins along i, j, k */
    int32_t order;               /* spline order the bins were built for */
    int32_t location;            /* picasso_location the bins were built for */
    int32_t chunk;               /* particles per work item */
    int32_t p2g_lanes;           /* lanes per particle of the tiled P2G: 1, 2 or
                                    4 for orders 1-2 (the 4 grid fields are
                                    split between them), 4 for order 3 (one
                                    stencil i-plane each); 0 = the library's
                                    choice; set to 0 by the sort */
    const int64_t* tile_offset;  /* device, num_tiles_total + 1 particle offsets */
    const uint32_t* tile_items;  /* device, num_tiles_total + 1: first work item
                                    of each tile (exclusive prefix of
                                    ceil(count / chunk)) */
    const void* records;         /* optional device, 16-byte aligned: the spline
                                    record of every (sorted) particle as
                                    picasso_spline_records writes it for these
                                    bins; the tiled P2G and G2P (not the one
                                    with advection) then read it instead of the
                                    positions.  Set by the caller after the
                                    permutation; the sort sets it to NULL.  It
                                    must be rewritten whenever a position
                                    changes. */
} picasso_bins;

/* Execution context of one call. */
typedef struct picasso_exec {
    void* stream;           /* cudaStream_t; NULL = legacy default stream */
    int32_t* error_count;   /* optional device int32: particles skipped because
                               their stencil left a non-periodic mesh */
    const picasso_bins* bins; /* optional: particles are tile-sorted (see above) */
    int32_t* overflow_count;  /* optional device int32, I64_FIXED grids only: P2G
                                 counts contributions (and tile sums) whose
                                 |value| * 2^fixed_bits reached 2^62, the grid
                                 velocity / update passes count nodes whose
                                 mass sum wrapped negative; nonzero means the
                                 fixed-point grid is unreliable (choose fewer
                                 fraction bits) */
} picasso_exec;

/* ------------------------------------------------------------------------ */
/* Library                                                                  */
/* ------------------------------------------------------------------------ */
PICASSO_API const char* picasso_version(void);
PICASSO_API const char* picasso_status_string(picasso_status s);
/* Name of the last CUDA error seen by this host thread (or ""). */
PICASSO_API const char* picasso_last_cuda_error(void);

/* ------------------------------------------------------------------------ */
/* APIC (Picasso::APIC, src/Picasso_APIC.hpp)                               */
/* ------------------------------------------------------------------------ */

/* APIC::p2g(m_p, c_p, m_i, mu_i, sd) over num_particles particles.
 * Replaces Picasso_APIC.hpp:55-140 (collocated, order 2/3), :148-232
 * (staggered Face/Edge, order 2/3), :240-319 (collocated, order 1) and
 * :327-402 (staggered, order 1), looped as GridOperator.hpp:612-642 does.
 * c_p is the 4 x ncomp particle matrix (row 0 = field value, rows 1..3 =
 * transposed affine matrix).  Collocated locations scatter ncomp components
 * into mu_i; Face/Edge locations scatter the location's dimension of a
 * 3-component c_p into component 0 of mu_i.  Results are ADDED to m_i / mu_i
 * (the reference's ScatterView contribution); zero them first with
 * picasso_grid_fill to get the GridOperator semantics.
 * dtypes: plain form: x_p, m_p, c_p, m_i, mu_i all F64 (global FP64 atomics).
 *         precision form: x_p F64; m_p, c_p F32; m_i, mu_i I64_FIXED
 *         (deterministic: every contribution is rounded to fixed point).
 *         F64 particles with I64_FIXED grid is also accepted. */
PICASSO_API picasso_status picasso_apic_p2g(const picasso_spline* sd, int64_t num_particles,
                                int32_t ncomp, picasso_particle_field x_p,
                                picasso_particle_field m_p, picasso_particle_field c_p,
                                picasso_grid_field m_i, picasso_grid_field mu_i,
                                const picasso_exec* exec);

/* APIC::g2p(u_i, c_p, sd).  Replaces Picasso_APIC.hpp:407-472 (collocated)
 * and :477-544 (staggered: writes row `dim` of u_p / B_p, zero elsewhere, as
 * the reference does).  c_p is overwritten.
 * dtypes: x_p F64; u_i F64 with c_p F64, or u_i F32 with c_p F32. */
PICASSO_API picasso_status picasso_apic_g2p(const picasso_spline* sd, int64_t num_particles,
                                int32_t ncomp, picasso_particle_field x_p,
                                picasso_grid_field u_i, picasso_particle_field c_p,
                                const picasso_exec* exec);

/* ------------------------------------------------------------------------ */
/* PolyPIC (Picasso::PolyPIC, src/Picasso_PolyPIC.hpp)                      */
/* ------------------------------------------------------------------------ */

/* PolyPIC::p2g(m_p, u_p, c_p, mu_i, m_i, dt, sd) -- note field before mass,
 * as in the reference.  Linear (order 1, 8 modes) replaces
 * Picasso_PolyPIC.hpp:39-130 (collocated) and :138-229 (staggered).
 * Quadratic (order 2, 27 modes) has no reference implementation; see the
 * library documentation for its definition.  u_p is the 8 (27) x 3 velocity
 * mode matrix defining the affine material motion, c_p the 8 (27) x ncomp
 * field modes (u_p == c_p when the field is the velocity).  Adds into mu_i
 * and m_i. */
PICASSO_API picasso_status picasso_polypic_p2g(const picasso_spline* sd, int64_t num_particles,
                                   int32_t ncomp, picasso_particle_field x_p,
                                   picasso_particle_field m_p, picasso_particle_field u_p,
                                   picasso_particle_field c_p, picasso_grid_field mu_i,
                                   picasso_grid_field m_i, double dt,
                                   const picasso_exec* exec);

/* PolyPIC::g2p(u_i, c_p, sd).  Replaces Picasso_PolyPIC.hpp:235-293
 * (collocated, c_p overwritten) and :299-358 (staggered: only column `dim`
 * of c_p is overwritten). */
PICASSO_API picasso_status picasso_polypic_g2p(const picasso_spline* sd, int64_t num_particles,
                                   int32_t ncomp, picasso_particle_field x_p,
                                   picasso_grid_field u_i, picasso_particle_field c_p,
                                   const picasso_exec* exec);

/* ------------------------------------------------------------------------ */
/* Grid-side helpers between P2G and G2P                                    */
/* ------------------------------------------------------------------------ */

/* Set components [0, ncomp) of every entity of the extent[0..2] box of mesh
 * to `value` (GridOperator.hpp:532-533 zeroes scatter fields this way). */
PICASSO_API picasso_status picasso_grid_fill(const picasso_mesh* mesh, int32_t ncomp,
                                 picasso_grid_field f, double value,
                                 const picasso_exec* exec);

/* Grid velocity update u_i = mu_i / m_i where m_i > mass_threshold, else 0,
 * on the owned entities (all entities along non-periodic dimensions).  The
 * division and threshold run in FP64 whatever the storage types; u_i may be
 * F64 or F32, m_i / mu_i F64 or I64_FIXED.  Optional u64_i (F64, may have
 * data == NULL) receives the FP64 velocity as well.  No reference
 * counterpart (the reference leaves the grid update to applications). */
PICASSO_API picasso_status picasso_grid_velocity(const picasso_mesh* mesh, int32_t ncomp,
                                     picasso_grid_field m_i, picasso_grid_field mu_i,
                                     double mass_threshold, picasso_grid_field u_i,
                                     picasso_grid_field u64_i, const picasso_exec* exec);

/* Grid update ("field solve" of the reference's explicit APIC time step,
 * doc/basic/explict_nearly_incompressible_flow.md:20-21):
 *   u_i = (mu_i + dt f_i) / m_i + dt g   where m_i > mass_threshold, else 0,
 * then the wall conditions below, on the owned entities (all entities along
 * non-periodic dimensions).  3 components.  FP64 arithmetic rounded step by
 * step (no FMA), so results are reproducible bit for bit.  f_i (F64 or the
 * type of mu_i) is optional (data == NULL: no force).  Walls apply along
 * non-periodic dimensions to the nodes within wall_width of the owned range's
 * first / last node (and to the ghost nodes beyond): NO_SLIP sets u = 0,
 * FREE_SLIP sets the wall-normal component to 0. */
typedef enum picasso_wall {
    PICASSO_WALL_NONE = 0,
    PICASSO_WALL_NO_SLIP = 1,
    PICASSO_WALL_FREE_SLIP = 2
} picasso_wall;

typedef struct picasso_grid_update_params {
    double dt;
    double gravity[3];
    double mass_threshold;
    int32_t wall[3][2];  /* picasso_wall per dimension, low and high side */
    int32_t wall_width;  /* nodes from the wall the condition covers (>= 0) */
} picasso_grid_update_params;

PICASSO_API picasso_status picasso_grid_update(const picasso_mesh* mesh, picasso_grid_field m_i,
                                               picasso_grid_field mu_i, picasso_grid_field f_i,
                                               const picasso_grid_update_params* params,
                                               picasso_grid_field u_i, picasso_grid_field u64_i,
                                               const picasso_exec* exec);

/* APIC::p2g (collocated, 3 components) followed by the grid update, in one
 * launch for cell-sorted particles in the precision form: the work items of
 * the tiled P2G count their arrival at the node regions they touch, and the
 * item that completes a region converts its nodes with the update of
 * picasso_grid_update (u = (mu + dt f) / m + dt g, threshold, walls) while
 * they are still in L2.  Results are bit-identical to picasso_apic_p2g then
 * picasso_grid_update, which is also what runs when the fused form does not
 * apply (no bins, FP64 form, staggered location, tiles of fewer than K - 1
 * bins, F32 velocity not requested).  m_i / mu_i receive the P2G sums as in
 * picasso_apic_p2g (zero them first); f_i: optional FP64 force; u_i: FP32;
 * u64_i optional FP64 copy.  `workspace`: device memory of the size
 * picasso_apic_p2g_update_workspace reports (8 counters per tile), cleared by
 * the call.  No counterpart in the reference, which leaves the step between
 * P2G and G2P to the application (doc/basic/explict_nearly_incompressible_flow.md:20-21). */
PICASSO_API picasso_status picasso_apic_p2g_update_workspace(const picasso_bins* bins,
                                                             int64_t* bytes);
PICASSO_API picasso_status picasso_apic_p2g_update(
    const picasso_spline* sd, int64_t num_particles, picasso_particle_field x_p,
    picasso_particle_field m_p, picasso_particle_field c_p, picasso_grid_field m_i,
    picasso_grid_field mu_i, picasso_grid_field f_i, const picasso_grid_update_params* params,
    picasso_grid_field u_i, picasso_grid_field u64_i, void* workspace, int64_t workspace_bytes,
    const picasso_exec* exec);

/* Particle advection x_p += dt * c_p(0, :) in FP64, then periodic wrap of the
 * position into the owned box along periodic dimensions. */
PICASSO_API picasso_status picasso_advect(const picasso_mesh* mesh, int64_t num_particles,
                              double dt, picasso_particle_field x_p,
                              picasso_particle_field c_p, const picasso_exec* exec);

/* picasso_apic_g2p (collocated, 3 components) followed by picasso_advect on
 * the same particles, in one pass: each particle's new velocity is written
 * to c_p and its position moved by dt times that velocity (as stored in
 * c_p's type) before the next particle.  Same results, bit for bit, as the
 * two calls; saves re-reading x_p and c_p.  The G2P half replaces
 * APIC.hpp:407-472; the position update is application code in the
 * reference (doc/basic/explict_nearly_incompressible_flow.md). */
PICASSO_API picasso_status picasso_apic_g2p_advect(const picasso_spline* sd,
                                                   int64_t num_particles,
                                                   picasso_particle_field x_p,
                                                   picasso_grid_field u_i,
                                                   picasso_particle_field c_p, double dt,
                                                   const picasso_exec* exec);

/* picasso_apic_g2p_advect that also writes, for every moved particle p,
 * key_out[p] = its sort key for bins of the given tile shape (the key
 * picasso_cell_sort defines, computed from the new position with the same
 * arithmetic), so that the next step's sort can start from the keys
 * (picasso_cell_sort_keys) instead of re-reading the positions.  key_out is
 * indexed like the particles (device, num_particles entries).  No reference
 * counterpart (Picasso has no sort). */
PICASSO_API picasso_status picasso_apic_g2p_advect_keys(const picasso_spline* sd,
                                                        int64_t num_particles,
                                                        picasso_particle_field x_p,
                                                        picasso_grid_field u_i,
                                                        picasso_particle_field c_p, double dt,
                                                        const int32_t tile[3], uint32_t* key_out,
                                                        const picasso_exec* exec);

/* ------------------------------------------------------------------------ */
/* Halo exchange inside the transfers (slab decomposition along x)          */
/* ------------------------------------------------------------------------ */

/* Neighbour grids of a rank whose local mesh is a slab of x-planes with
 * ghost planes on either side.  Local x-planes p < lo_end belong to the lower
 * neighbour (its plane p + lo_shift), planes p >= hi_begin to the upper one
 * (its plane p + hi_shift).  The neighbour grids have this rank's strides and
 * dtypes and must be addressable from this device (the same device, or a
 * peer GPU's memory mapped here, e.g. by CUDA IPC with peer access).
 * P2G: lo[0] / hi[0] are the neighbours' m_i, lo[1] / hi[1] their mu_i.
 * G2P: lo[0] / hi[0] are the neighbours' u_i. */
typedef struct picasso_halo_peers {
    int32_t lo_end;
    int32_t hi_begin;
    int32_t lo_shift;
    int32_t hi_shift;
    void* lo[2];
    void* hi[2];
} picasso_halo_peers;

/* picasso_apic_p2g whose contributions to ghost-plane nodes are added
 * directly into the neighbour that owns them (64-bit integer reductions, over
 * NVLink for a peer GPU): once every rank's call has completed, each rank's
 * owned planes hold the complete sums and its ghost planes are untouched.
 * This is the reference's P2G followed by the halo scatter with Sum
 * (Picasso_FieldManager.hpp:157-164) in one pass.  Tiled FP32 form only
 * (exec->bins, F32 particle fields, I64_FIXED grids, collocated Node
 * location, packed particle storage); anything else returns
 * PICASSO_ERR_UNSUPPORTED. */
PICASSO_API picasso_status picasso_apic_p2g_halo(const picasso_spline* sd, int64_t num_particles,
                                                 picasso_particle_field x_p,
                                                 picasso_particle_field m_p,
                                                 picasso_particle_field c_p,
                                                 picasso_grid_field m_i, picasso_grid_field mu_i,
                                                 const picasso_halo_peers* peers,
                                                 const picasso_exec* exec);
/* picasso_apic_g2p reading the ghost-plane velocities from the neighbours'
 * u_i (their owned planes) instead of this rank's ghost planes: the halo
 * gather (Picasso_FieldManager.hpp:174-181) folded into the G2P's staging of
 * node velocities.  Tiled FP32 form only (exec->bins, F32 u_i and c_p). */
PICASSO_API picasso_status picasso_apic_g2p_halo(const picasso_spline* sd, int64_t num_particles,
                                                 picasso_particle_field x_p,
                                                 picasso_grid_field u_i,
                                                 picasso_particle_field c_p,
                                                 const picasso_halo_peers* peers,
                                                 const picasso_exec* exec);

/* ------------------------------------------------------------------------ */
/* Particle cell-sort                                                       */
/* ------------------------------------------------------------------------ */

/* Bytes of device workspace picasso_cell_sort needs for num_particles
 * particles and the given spline / tile shape. */
PICASSO_API picasso_status picasso_cell_sort_workspace(const picasso_spline* sd, int64_t num_particles,
                                           const int32_t tile[3], int64_t* bytes);

/* Stable sort of the particles by stencil bin in tiles.  The bin of a
 * particle is the first index of its spline stencil along each dimension
 * (wrapped into the owned range along periodic dimensions); the key is
 *   key = tile_linear * (tile[0]*tile[1]*tile[2]) + bin_in_tile_linear
 * (i slowest, k fastest in both).  A particle whose stencil leaves a
 * non-periodic mesh gets key = num_tiles * tile volume and sorts last.
 * Outputs (device): key[num_particles] (sorted keys), perm[num_particles]
 * (perm[r] = original index of the particle of rank r; ties keep the
 * original order) and tile_offset[num_tiles + 1] (first rank of each tile;
 * the last entry counts the particles inside the mesh).  bins_out (host) is
 * filled for picasso_exec.bins.  tile_items[num_tiles + 1] receives the
 * work-item prefix for chunks of `chunk` particles (chunk >= 32).
 * workspace: device memory of at least the size picasso_cell_sort_workspace
 * reports, 256-byte aligned.
 * No reference counterpart: Picasso has no particle sort. */
PICASSO_API picasso_status picasso_cell_sort(const picasso_spline* sd, int64_t num_particles,
                                 picasso_particle_field x_p, const int32_t tile[3],
                                 int32_t chunk, uint32_t* key, uint32_t* perm,
                                 int64_t* tile_offset, uint32_t* tile_items,
                                 void* workspace, int64_t workspace_bytes,
                                 picasso_bins* bins_out, const picasso_exec* exec);

/* picasso_cell_sort from keys the caller already has: key_in[p] (device) is
 * the sort key of particle p as picasso_cell_sort defines it, e.g. written by
 * picasso_apic_g2p_advect_keys for the same spline and tile shape.  Keys
 * above num_tiles * tile volume count as that value (outside the mesh).
 * Same outputs as picasso_cell_sort on the positions the keys came from.
 * key_in must not overlap key, perm or the workspace; it is not modified.
 * No reference counterpart. */
PICASSO_API picasso_status picasso_cell_sort_keys(const picasso_spline* sd, int64_t num_particles,
                                                  const uint32_t* key_in, const int32_t tile[3],
                                                  int32_t chunk, uint32_t* key, uint32_t* perm,
                                                  int64_t* tile_offset, uint32_t* tile_items,
                                                  void* workspace, int64_t workspace_bytes,
                                                  picasso_bins* bins_out,
                                                  const picasso_exec* exec);

/* Spline records of sorted particles for the tiled transfers: records[p]
 * (16 bytes, device, 16-byte aligned) = the in-cell fractions (t_x, t_y, t_z)
 * of particle p's logical position as FP32 and, in the fourth word, its sort
 * key (uint32) for `bins`.  Both are formed from the FP64 position with the
 * arithmetic every kernel uses, so P2G / G2P that read the records (set
 * bins->records) build the same splines and bins as from the positions, while
 * reading 16 instead of 24 bytes per particle and no FP64 arithmetic.  Call it
 * after picasso_permute (x_p in sorted order) and after every position
 * change.  No counterpart in the reference (its splines are evaluated from
 * the positions in every transfer, ParticleInterpolation.hpp:88-105). */
PICASSO_API picasso_status picasso_spline_records(const picasso_spline* sd,
                                                  int64_t num_particles,
                                                  picasso_particle_field x_p,
                                                  const picasso_bins* bins, void* records,
                                                  const picasso_exec* exec);

/* picasso_cell_sort for callers that cannot allocate device memory when they
 * sort (an application that gives all GPU memory to its own pool at start-up,
 * a plugin hosted by one, a loop that must not meet the allocator's latency
 * or out-of-memory path).  Same arguments and results as picasso_cell_sort
 * minus the workspace: the scratch is a 32 MiB array compiled into the
 * library, held by every device that loads the library's kernels until the
 * process exits.  Returns PICASSO_ERR_OUT_OF_RANGE, before any launch, when
 * the sort needs more than 32 MiB (picasso_cell_sort_workspace reports the
 * need; about 8 bytes per particle plus the digit tables, i.e. up to roughly
 * 3 million particles).  Every call looks up the array's device address in
 * the current context (cudaGetSymbolAddress), so a device or context reset in
 * between is harmless; the first call on a device may load the module, so
 * make it before any stream capture.  All calls share the array: calls whose
 * work overlaps on the GPU (other streams, other host threads) race, so order
 * them.  No counterpart in the reference. */
PICASSO_API picasso_status picasso_cell_sort_static(const picasso_spline* sd,
                                                    int64_t num_particles,
                                                    picasso_particle_field x_p,
                                                    const int32_t tile[3], int32_t chunk,
                                                    uint32_t* key, uint32_t* perm,
                                                    int64_t* tile_offset, uint32_t* tile_items,
                                                    picasso_bins* bins_out,
                                                    const picasso_exec* exec);

/* Fastest launch knobs of the sorted (tiled) step for one instance. */
typedef struct picasso_tune_result {
    int32_t tile[3];   /* bins per tile for picasso_cell_sort */
    int32_t chunk;     /* particles per work item */
    int32_t p2g_lanes; /* picasso_bins.p2g_lanes */
    float step_ms;     /* measured fill + P2G + velocity + G2P, milliseconds */
} picasso_tune_result;

/* Autotuner of the precision-form tiled step (FP32 m_p / c_p, 64-bit
 * fixed-point m_i / mu_i, FP32 u_i; collocated, 3 components) on the
 * caller's own particles: for tiles (4,4,4) (4,4,8) (4,8,8) (8,8,8), work items
 * of 1024 and 4096 particles and 1 or 2 P2G lanes per particle (4 for cubic)
 * it sorts and permutes copies of the particles and times `trials` steps of
 * grid fill -> P2G -> grid velocity -> G2P with CUDA events on the stream,
 * and writes the fastest candidate to *best.  The particle members are not
 * modified; m_i, mu_i and u_i serve as the step's grids and hold the last
 * candidate's values afterwards.  Allocates and frees device memory (about
 * 84 bytes per particle plus the sort workspace) and waits for the stream:
 * a set-up call, not one for a time step.  The candidates' grid results
 * agree to FP32 rounding (the tiled P2G sums a work item in FP32 before its
 * fixed-point flush, so the tiling sets the rounding; each choice is itself
 * deterministic).  Returns PICASSO_ERR_UNSUPPORTED for staggered locations.  No reference
 * counterpart (Picasso has no tiled path to tune). */
PICASSO_API picasso_status picasso_autotune(const picasso_spline* sd, int64_t num_particles,
                                            picasso_particle_field x_p, picasso_particle_field m_p,
                                            picasso_particle_field c_p, picasso_grid_field m_i,
                                            picasso_grid_field mu_i, picasso_grid_field u_i,
                                            double mass_threshold, int32_t trials,
                                            picasso_tune_result* best, const picasso_exec* exec);

/* Gather a particle member: dst(p, c) = src(perm[p], c) for c < ncomp.
 * src and dst must not overlap. */
PICASSO_API picasso_status picasso_permute(int64_t num_particles, int32_t ncomp, const uint32_t* perm,
                               picasso_particle_field src, picasso_particle_field dst,
                               const picasso_exec* exec);

/* ------------------------------------------------------------------------ */
/* Batched 3x3 linear algebra (LinearAlgebra, BatchedLinearAlgebra.hpp)     */
/* ------------------------------------------------------------------------ */

/* For each of n row-major 3x3 FP64 matrices a[9*b..]: det[b] = !a
 * (Picasso_BatchedLinearAlgebra.hpp:4337-4350) and, when a_inv != NULL,
 * a_inv = inverse(a) by cofactors times 1/det (:4626-4686).  When x != NULL
 * and y != NULL also y = a_inv * x (3-vectors). */
PICASSO_API picasso_status picasso_mat3_inverse(int64_t n, const double* a, double* a_inv, double* det,
                                    const double* x, double* y, const picasso_exec* exec);

/* ------------------------------------------------------------------------ */
/* Batched independent APIC problems                                        */
/* ------------------------------------------------------------------------ */
/* No counterpart in the reference, which runs one mesh per rank and one
 * kernel per GridOperator::apply.  A batch holds many independent APIC
 * problems (meshes of any size, any particle count, order 1-3 each) and runs
 * one APIC step over all of them -- fill of the scatter fields, P2G, grid
 * velocity, G2P, i.e. GridOperator.hpp:532 zeroing + APIC.hpp:55-140 +
 * v = p / m + APIC.hpp:407-471 per instance -- in persistent kernel launches
 * that take work items of every instance from one queue. */

typedef struct picasso_batch_instance {
    picasso_spline spline;          /* collocated NODE location, order 1..3 */
    int64_t num_particles;
    picasso_particle_field x_p;     /* packed (n,3) F64 */
    picasso_particle_field m_p;     /* packed (n): F32 (precision form) or F64 */
    picasso_particle_field c_p;     /* packed (n,4,3), 16-byte aligned, type of m_p */
    picasso_grid_field m_i;         /* node mass: I64_FIXED (precision form) or F64 */
    picasso_grid_field mu_i;        /* node momentum (3 components), type of m_i */
    picasso_grid_field u_i;         /* node velocity (3 components): F32 or F64 */
    double mass_threshold;          /* u = mu / m where m > threshold, else 0 */
    picasso_bins bins;              /* bins of the sorted particles (picasso_cell_sort) */
    int32_t* error_count;           /* optional device counter (skipped particles) */
} picasso_batch_instance;

typedef enum picasso_batch_mode {
    /* one persistent launch per step; an instance's items wait for the
       instance's previous phase (bounded spin on device counters) */
    PICASSO_BATCH_FUSED = 0,
    /* one persistent launch per phase (4 per step), no waits */
    PICASSO_BATCH_PHASED = 1
} picasso_batch_mode;

typedef struct picasso_batch_info {
    int32_t count;            /* instances */
    int32_t precision_form;   /* 1 = FP32 particles + fixed-point grid, 0 = FP64 */
    int32_t grid_blocks;      /* persistent CTAs (one warp each) */
    int32_t smem_bytes;       /* dynamic shared memory per CTA */
    int64_t items[4];         /* work items per phase: fill, p2g, velocity, g2p */
    int64_t particles;        /* total particles */
} picasso_batch_info;

typedef struct picasso_batch picasso_batch;  /* opaque */

/* Validates the instances, copies their descriptors to the device (the
 * pointed-to arrays are not copied: they must stay valid, and the bins must
 * keep describing the particles, for the life of the batch) and sizes the
 * persistent launch.  All instances use the same form: precision form
 * (F32 m_p, c_p; I64_FIXED m_i, mu_i; F32 u_i) or FP64 (all F64).  Allocates
 * its device tables here and nowhere else. */
PICASSO_API picasso_status picasso_batch_create(const picasso_batch_instance* instances,
                                                int32_t count, int32_t mode,
                                                picasso_batch** out);
/* One APIC step of every instance on `stream`.  use_graph != 0 replays a
 * CUDA graph captured at the first such call (one memset node + the
 * persistent launches).  Returns PICASSO_ERR_CUDA for launch errors; a wait
 * that ran out (which the queue order rules out at the default limit) is
 * reported by picasso_batch_status.  Steps of one batch must not overlap on the GPU (they
 * share the queue counters). */
PICASSO_API picasso_status picasso_batch_step(picasso_batch* batch, void* stream,
                                              int32_t use_graph);
/* The same step issued as single launches, instance after instance
 * (picasso_grid_fill x 2, picasso_apic_p2g, picasso_grid_velocity,
 * picasso_apic_g2p): the comparison for the batched launch. */
PICASSO_API picasso_status picasso_batch_step_sequential(picasso_batch* batch, void* stream);
/* Synchronises `stream` and returns PICASSO_ERR_TIMEOUT if a dependency wait
 * of an earlier step ran out of polls or gave up after picasso_batch_cancel
 * (and clears the flag), else PICASSO_OK.  Items whose wait gave up skip
 * their work, so that step's results are incomplete. */
PICASSO_API picasso_status picasso_batch_status(picasso_batch* batch, void* stream);
/* Bound of every dependency wait of the fused step, in polls of ~0.25 us
 * (default 2^22, about a second).  Takes effect from the next step (a
 * captured graph is released and captured again).  0 makes a wait give up at
 * its first unmet check.  No counterpart in the reference. */
PICASSO_API picasso_status picasso_batch_set_wait_limit(picasso_batch* batch, uint32_t polls);
/* Enqueues on `stream` a write of the batch's status word: every dependency
 * wait of a fused step that runs after it gives up at once (its item is
 * skipped) until picasso_batch_status reads and clears the flag.  The host's
 * way to end a fused step early, e.g. when another rank has failed.  No
 * counterpart in the reference. */
PICASSO_API picasso_status picasso_batch_cancel(picasso_batch* batch, void* stream);
PICASSO_API picasso_status picasso_batch_get_info(const picasso_batch* batch,
                                                  picasso_batch_info* info);
PICASSO_API picasso_status picasso_batch_destroy(picasso_batch* batch);

#ifdef __cplusplus
}
#endif

#endif /* PICASSO_B200_H */
