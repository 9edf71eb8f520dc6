"""Host-side interface mirroring Picasso's transfer API on top of the C ABI.

Reference interfaces (paths inside the Picasso source tree):
  UniformMesh geometry           src/Picasso_UniformMesh.hpp:73-196
  FieldLocation / entity types   src/Picasso_FieldTypes.hpp:125-168
  InterpolationOrder, createSpline
                                 src/Picasso_ParticleInterpolation.hpp:27-105
  APIC::p2g / APIC::g2p          src/Picasso_APIC.hpp:55-544
  PolyPIC::p2g / PolyPIC::g2p    src/Picasso_PolyPIC.hpp:39-359
  GridOperator scatter zeroing   src/Picasso_GridOperator.hpp:532-533

Particle members are torch CUDA tensors shaped (N,), (N, C) or (N, R, C) with
any strides whose inner (R, C) block is row-major contiguous; grid arrays are
torch CUDA tensors shaped (nx, ny, nz) or (nx, ny, nz, C).  A fixed-point grid
accumulator is a :class:`FixedGrid` (an int64 tensor plus its fraction bits).
Every call enqueues on the current torch CUDA stream unless ``stream`` is
given; there is no CPU path.
"""

import ctypes as C
import math

import torch

from . import _abi
from ._abi import check

# ---------------------------------------------------------------------------
# field locations and orders
# ---------------------------------------------------------------------------


class FieldLocation:
    """Mesh entity types (Picasso FieldLocation)."""

    Node = _abi.NODE
    Cell = _abi.CELL

    @staticmethod
    def Face(dim):
        if dim not in (0, 1, 2):
            raise ValueError("Face dimension out of bounds")
        return _abi.FACE_I + dim

    @staticmethod
    def Edge(dim):
        if dim not in (0, 1, 2):
            raise ValueError("Edge dimension out of bounds")
        return _abi.EDGE_I + dim


def staggered_dim(location):
    if _abi.FACE_I <= location <= _abi.FACE_K:
        return location - _abi.FACE_I
    if _abi.EDGE_I <= location <= _abi.EDGE_K:
        return location - _abi.EDGE_I
    return -1


def _node_aligned(location, d):
    """True if the entity sits on nodes along dimension d."""
    if location == _abi.NODE:
        return True
    if location == _abi.CELL:
        return False
    s = staggered_dim(location)
    if location <= _abi.FACE_K:
        return d == s
    return d != s


class InterpolationOrder(int):
    """InterpolationOrder<N>: 1 linear, 2 quadratic, 3 cubic."""

    def __new__(cls, n):
        if n not in (1, 2, 3):
            raise ValueError("interpolation order must be 1, 2 or 3")
        return int.__new__(cls, n)


# ---------------------------------------------------------------------------
# mesh
# ---------------------------------------------------------------------------


class UniformMesh:
    """Single-rank uniform mesh with the geometry conventions of
    Picasso::UniformMesh: cells from a cell size (or a cell count) over a
    bounding box, non-periodic dimensions padded by the minimum halo width,
    a local grid with ``halo_cell_width`` ghost layers on every side whose
    node (0,0,0) sits at ``low_corner``."""

    def __init__(self, global_bounding_box, cell_size=None, global_num_cell=None,
                 periodic=(False, False, False), halo_cell_width=0,
                 minimum_halo_cell_width=0):
        box = [float(v) for v in global_bounding_box]
        if len(box) != 6:
            raise ValueError("bounding box needs 6 entries")
        if cell_size is not None:
            cs = float(cell_size)
            ncell = [int(round((box[d + 3] - box[d]) / cs)) for d in range(3)]
        elif global_num_cell is not None:
            ncell = [int(v) for v in global_num_cell]
            if len(ncell) != 3:
                raise ValueError("3 entries required for mesh.global_num_cell")
            cs = (box[3] - box[0]) / ncell[0]
        else:
            raise ValueError("Invalid uniform mesh size parameters")
        for d in range(3):
            if abs(ncell[d] * cs - (box[d + 3] - box[d])) > 1.1920929e-07:
                raise ValueError("Extent not evenly divisible by uniform cell size")
        periodic = [bool(p) for p in periodic]
        if len(periodic) != 3:
            raise ValueError("3 entries required for mesh.periodic")
        low = box[:3]
        for d in range(3):
            if not periodic[d]:
                ncell[d] += 2 * minimum_halo_cell_width
                low[d] -= cs * minimum_halo_cell_width
        self.cell_size = cs
        self.global_num_cell = ncell
        self.periodic = periodic
        self.halo_cell_width = max(int(minimum_halo_cell_width), int(halo_cell_width))
        h = self.halo_cell_width
        self.global_low_corner = low
        self.low_corner = [low[d] - h * cs for d in range(3)]

    def owned_extent(self, location, d):
        n = self.global_num_cell[d]
        if _node_aligned(location, d) and not self.periodic[d]:
            return n + 1
        return n

    def extent(self, location):
        """Local (ghosted) index extent of the entity arrays of a location."""
        h = self.halo_cell_width
        return tuple(self.owned_extent(location, d) + 2 * h for d in range(3))

    def descriptor(self, location):
        m = _abi.Mesh()
        ext = self.extent(location)
        for d in range(3):
            m.extent[d] = ext[d]
            m.own_begin[d] = self.halo_cell_width
            m.own_extent[d] = self.owned_extent(location, d)
            m.periodic[d] = 1 if self.periodic[d] else 0
            m.low_corner[d] = self.low_corner[d]
            m.cell_size[d] = self.cell_size
        return m

    def zeros(self, location, ncomp=None, dtype=torch.float64, device="cuda"):
        shape = self.extent(location) + ((ncomp,) if ncomp else ())
        return torch.zeros(shape, dtype=dtype, device=device)


class Spline:
    """createSpline(Location, InterpolationOrder<N>, mesh, x): the stencil is
    evaluated inside the transfer kernels from the particle positions."""

    def __init__(self, location, order, mesh, x):
        self.location = int(location)
        self.order = int(InterpolationOrder(int(order)))
        self.mesh = mesh
        self.x = x
        self.desc = _abi.Spline()
        self.desc.mesh = mesh.descriptor(self.location)
        self.desc.location = self.location
        self.desc.order = self.order

    @property
    def num_particles(self):
        return self.x.shape[0]


def create_spline(location, order, mesh, x, *members):
    """Mirror of Picasso::createSpline; spline members (SplineValue, ...) are
    accepted and ignored because every member is computed on the fly."""
    return Spline(location, order, mesh, x)


# ---------------------------------------------------------------------------
# descriptors from tensors
# ---------------------------------------------------------------------------

_DT = {torch.float64: _abi.F64, torch.float32: _abi.F32}


class FixedGrid:
    """A 64-bit fixed-point grid accumulator: value = raw * 2**-bits."""

    def __init__(self, raw, bits):
        if raw.dtype != torch.int64:
            raise TypeError("fixed-point grid must be int64")
        self.raw = raw
        self.bits = int(bits)

    def to_float(self, dtype=torch.float64):
        return self.raw.to(dtype) * (2.0 ** -self.bits)


def particle_field(t):
    """Descriptor of a particle member tensor (N,), (N, C) or (N, R, C)."""
    if t.dtype not in _DT:
        raise TypeError("particle members must be float64 or float32")
    if not t.is_cuda:
        raise ValueError("particle members must be CUDA tensors")
    f = _abi.ParticleField()
    f.data = t.data_ptr()
    f.dtype = _DT[t.dtype]
    f.vector_shift = 0
    f.tile_stride = t.stride(0) if t.dim() >= 1 else 1
    if t.dim() == 1:
        f.comp_stride = 0
    elif t.dim() == 2:
        f.comp_stride = t.stride(1)
    elif t.dim() == 3:
        if t.shape[2] > 1 and t.stride(1) != t.shape[2] * t.stride(2):
            raise ValueError("matrix members need a row-major (R, C) block")
        f.comp_stride = t.stride(2) if t.shape[2] > 1 else t.stride(1)
    else:
        raise ValueError("particle members are (N,), (N, C) or (N, R, C)")
    return f


def grid_field(t):
    """Descriptor of a grid tensor (nx, ny, nz[, C]) or a FixedGrid."""
    g = _abi.GridField()
    if isinstance(t, FixedGrid):
        raw = t.raw
        g.dtype = _abi.I64_FIXED
        g.fixed_bits = t.bits
    else:
        raw = t
        if raw.dtype not in _DT:
            raise TypeError("grid arrays must be float64, float32 or a FixedGrid")
        g.dtype = _DT[raw.dtype]
        g.fixed_bits = 0
    if not raw.is_cuda:
        raise ValueError("grid arrays must be CUDA tensors")
    if raw.dim() not in (3, 4):
        raise ValueError("grid arrays are (nx, ny, nz) or (nx, ny, nz, C)")
    g.data = raw.data_ptr()
    for d in range(3):
        g.stride[d] = raw.stride(d)
    g.stride[3] = raw.stride(3) if raw.dim() == 4 else 0
    return g


def _grid_tensor(t):
    return t.raw if isinstance(t, FixedGrid) else t


def _ncomp_of_grid(t):
    r = _grid_tensor(t)
    return r.shape[3] if r.dim() == 4 else 1


def _check_grid_extent(t, mesh_desc):
    r = _grid_tensor(t)
    for d in range(3):
        if r.shape[d] < mesh_desc.extent[d]:
            raise ValueError("grid array smaller than the mesh extent along %d" % d)


class Exec:
    """Execution context: stream, optional skipped-particle counter, bins,
    optional fixed-point overflow counter (int32 CUDA tensors)."""

    def __init__(self, stream=None, error_count=None, bins=None, overflow_count=None):
        self.desc = _abi.Exec()
        s = stream if stream is not None else torch.cuda.current_stream()
        self.desc.stream = s.cuda_stream if hasattr(s, "cuda_stream") else s
        self._err = error_count
        self.desc.error_count = error_count.data_ptr() if error_count is not None else None
        self._bins = bins
        self.desc.bins = C.pointer(bins.desc) if bins is not None else None
        self._ovf = overflow_count
        self.desc.overflow_count = (overflow_count.data_ptr() if overflow_count is not None
                                    else None)


def _exec(stream, error_count, bins, overflow_count=None):
    return Exec(stream, error_count, bins, overflow_count)


def _lib():
    return _abi.load_library()


# ---------------------------------------------------------------------------
# APIC
# ---------------------------------------------------------------------------


class APIC:
    """Picasso::APIC transfers over all particles of the spline."""

    @staticmethod
    def p2g(m_p, c_p, m_i, mu_i, sd, stream=None, error_count=None, bins=None,
            overflow_count=None, peers=None):
        """APIC::p2g(m_p, c_p, m_i, mu_i, sd): adds mass and momentum into the
        grid (zero them first for the GridOperator semantics).
        `overflow_count` (int32 CUDA tensor): fixed-point grids add the
        number of contributions out of the 64-bit range to it.
        `peers` (HaloPeers, e.g. SlabDecomposition.halo_peers): contributions
        to ghost-plane nodes go straight into the neighbours' grids
        (picasso_apic_p2g_halo; tiled precision form only)."""
        ncomp = c_p.shape[2]
        _check_grid_extent(m_i, sd.desc.mesh)
        _check_grid_extent(mu_i, sd.desc.mesh)
        ex = _exec(stream, error_count, bins, overflow_count)
        if peers is not None:
            check(_lib().picasso_apic_p2g_halo(C.byref(sd.desc), sd.num_particles,
                                               particle_field(sd.x), particle_field(m_p),
                                               particle_field(c_p), grid_field(m_i),
                                               grid_field(mu_i), C.byref(peers),
                                               C.byref(ex.desc)), "APIC::p2g (halo)")
            return
        check(_lib().picasso_apic_p2g(C.byref(sd.desc), sd.num_particles, ncomp,
                                      particle_field(sd.x), particle_field(m_p),
                                      particle_field(c_p), grid_field(m_i), grid_field(mu_i),
                                      C.byref(ex.desc)), "APIC::p2g")

    @staticmethod
    def p2g_update(m_p, c_p, m_i, mu_i, u_i, sd, dt=0.0, gravity=(0.0, 0.0, 0.0), f_i=None,
                   mass_threshold=1e-12, walls=None, wall_width=1, u64_i=None, workspace=None,
                   stream=None, error_count=None, bins=None, overflow_count=None):
        """APIC::p2g followed by the grid update of grid_update (same
        arguments), fused into one launch for cell-sorted particles in the
        precision form (picasso_apic_p2g_update; the two separate calls
        otherwise, with bit-identical results).  `workspace`: a uint8 CUDA
        tensor of p2g_update_workspace(bins) bytes, allocated if not given."""
        _check_grid_extent(m_i, sd.desc.mesh)
        _check_grid_extent(mu_i, sd.desc.mesh)
        _check_grid_extent(u_i, sd.desc.mesh)
        if workspace is None and bins is not None:
            workspace = torch.empty(max(p2g_update_workspace(bins), 1), dtype=torch.uint8,
                                    device=sd.x.device)
        prm = _update_params(dt, gravity, mass_threshold, walls, wall_width)
        ex = _exec(stream, error_count, bins, overflow_count)
        none = _abi.GridField()
        check(_lib().picasso_apic_p2g_update(
            C.byref(sd.desc), sd.num_particles, particle_field(sd.x), particle_field(m_p),
            particle_field(c_p), grid_field(m_i), grid_field(mu_i),
            grid_field(f_i) if f_i is not None else none, C.byref(prm), grid_field(u_i),
            grid_field(u64_i) if u64_i is not None else none,
            workspace.data_ptr() if workspace is not None else None,
            workspace.numel() if workspace is not None else 0, C.byref(ex.desc)),
            "APIC::p2g_update")

    @staticmethod
    def g2p(u_i, c_p, sd, stream=None, error_count=None, bins=None, peers=None):
        """APIC::g2p(u_i, c_p, sd): overwrites c_p (4 x ncomp per particle).
        `peers`: ghost-plane velocities are read from the neighbours' u_i
        (picasso_apic_g2p_halo; tiled precision form only)."""
        ncomp = c_p.shape[2]
        _check_grid_extent(u_i, sd.desc.mesh)
        ex = _exec(stream, error_count, bins)
        if peers is not None:
            check(_lib().picasso_apic_g2p_halo(C.byref(sd.desc), sd.num_particles,
                                               particle_field(sd.x), grid_field(u_i),
                                               particle_field(c_p), C.byref(peers),
                                               C.byref(ex.desc)), "APIC::g2p (halo)")
            return
        check(_lib().picasso_apic_g2p(C.byref(sd.desc), sd.num_particles, ncomp,
                                      particle_field(sd.x), grid_field(u_i), particle_field(c_p),
                                      C.byref(ex.desc)), "APIC::g2p")

    @staticmethod
    def g2p_advect(u_i, c_p, sd, dt, stream=None, error_count=None, bins=None, key_tile=None,
                   keys_out=None):
        """APIC::g2p followed by the position update x_p += dt * c_p(0, :)
        (FP64, periodic wrap) in one pass; collocated, 3 components.  The
        spline's positions sd.x are updated in place.  With key_tile (a tile
        shape) it also returns the sort key of every moved particle (int32
        tensor of uint32 values, written into keys_out if given), the input of
        cell_sort(..., keys=...) for the next step."""
        _check_grid_extent(u_i, sd.desc.mesh)
        ex = _exec(stream, error_count, bins)
        if key_tile is None:
            check(_lib().picasso_apic_g2p_advect(C.byref(sd.desc), sd.num_particles,
                                                 particle_field(sd.x), grid_field(u_i),
                                                 particle_field(c_p), float(dt),
                                                 C.byref(ex.desc)), "APIC::g2p_advect")
            return None
        n = sd.num_particles
        if keys_out is None:
            keys_out = torch.empty(max(n, 1), dtype=torch.int32, device=sd.x.device)
        elif keys_out.dtype != torch.int32 or keys_out.numel() < n or not keys_out.is_contiguous():
            raise ValueError("keys_out: contiguous int32 tensor of at least %d entries" % n)
        t3 = (C.c_int32 * 3)(*key_tile)
        check(_lib().picasso_apic_g2p_advect_keys(C.byref(sd.desc), n, particle_field(sd.x),
                                                  grid_field(u_i), particle_field(c_p),
                                                  float(dt), t3, keys_out.data_ptr(),
                                                  C.byref(ex.desc)), "APIC::g2p_advect")
        return keys_out[:n]


class PolyPIC:
    """Picasso::PolyPIC transfers (linear 8 modes; quadratic 27 modes)."""

    @staticmethod
    def p2g(m_p, u_p, c_p, mu_i, m_i, dt, sd, stream=None, error_count=None, bins=None,
            overflow_count=None):
        """PolyPIC::p2g(m_p, u_p, c_p, mu_i, m_i, dt, sd) -- field before mass.
        With bins (cell-sorted particles) the FP32 form runs the tiled kernel
        (bit-identical grid)."""
        ncomp = c_p.shape[2]
        _check_grid_extent(m_i, sd.desc.mesh)
        _check_grid_extent(mu_i, sd.desc.mesh)
        ex = _exec(stream, error_count, bins, overflow_count)
        check(_lib().picasso_polypic_p2g(C.byref(sd.desc), sd.num_particles, ncomp,
                                         particle_field(sd.x), particle_field(m_p),
                                         particle_field(u_p), particle_field(c_p),
                                         grid_field(mu_i), grid_field(m_i), float(dt),
                                         C.byref(ex.desc)), "PolyPIC::p2g")

    @staticmethod
    def g2p(u_i, c_p, sd, stream=None, error_count=None, bins=None):
        """PolyPIC::g2p(u_i, c_p, sd).  With bins the FP32 form runs the tiled
        kernel (bit-identical c_p)."""
        ncomp = c_p.shape[2]
        _check_grid_extent(u_i, sd.desc.mesh)
        ex = _exec(stream, error_count, bins)
        check(_lib().picasso_polypic_g2p(C.byref(sd.desc), sd.num_particles, ncomp,
                                         particle_field(sd.x), grid_field(u_i),
                                         particle_field(c_p), C.byref(ex.desc)),
              "PolyPIC::g2p")


# ---------------------------------------------------------------------------
# grid helpers
# ---------------------------------------------------------------------------


def grid_fill(mesh_desc, f, value=0.0, ncomp=None, stream=None):
    ex = _exec(stream, None, None)
    nc = ncomp or _ncomp_of_grid(f)
    check(_lib().picasso_grid_fill(C.byref(mesh_desc), nc, grid_field(f), float(value),
                                   C.byref(ex.desc)), "grid_fill")


def grid_velocity(mesh_desc, m_i, mu_i, u_i, mass_threshold=1e-12, u64_i=None, stream=None,
                  overflow_count=None):
    """u_i = mu_i / m_i (FP64 arithmetic) where m_i > threshold, else 0.
    `overflow_count`: fixed-point masses that wrapped negative are counted."""
    ex = _exec(stream, None, None, overflow_count)
    g64 = grid_field(u64_i) if u64_i is not None else _abi.GridField()
    check(_lib().picasso_grid_velocity(C.byref(mesh_desc), _ncomp_of_grid(mu_i), grid_field(m_i),
                                       grid_field(mu_i), float(mass_threshold), grid_field(u_i),
                                       g64, C.byref(ex.desc)), "grid_velocity")


def _update_params(dt, gravity, mass_threshold, walls, wall_width):
    kinds = {"none": _abi.WALL_NONE, "no_slip": _abi.WALL_NO_SLIP,
             "free_slip": _abi.WALL_FREE_SLIP}
    prm = _abi.GridUpdateParams()
    prm.dt = float(dt)
    for d in range(3):
        prm.gravity[d] = float(gravity[d])
        for side in range(2):
            prm.wall[d][side] = kinds[walls[d][side]] if walls else _abi.WALL_NONE
    prm.mass_threshold = float(mass_threshold)
    prm.wall_width = int(wall_width)
    return prm


def grid_update(mesh_desc, m_i, mu_i, u_i, dt, gravity=(0.0, 0.0, 0.0), f_i=None,
                mass_threshold=1e-12, walls=None, wall_width=1, u64_i=None, stream=None,
                overflow_count=None):
    """u_i = (mu_i + dt f_i) / m_i + dt g where m_i > threshold (else 0), then
    wall conditions along non-periodic dimensions: ``walls[d] = (low, high)``
    with "none", "no_slip" or "free_slip"."""
    prm = _update_params(dt, gravity, mass_threshold, walls, wall_width)
    ex = _exec(stream, None, None, overflow_count)
    none = _abi.GridField()
    check(_lib().picasso_grid_update(C.byref(mesh_desc), grid_field(m_i), grid_field(mu_i),
                                     grid_field(f_i) if f_i is not None else none,
                                     C.byref(prm), grid_field(u_i),
                                     grid_field(u64_i) if u64_i is not None else none,
                                     C.byref(ex.desc)), "grid_update")


def advect(mesh_desc, x_p, c_p, dt, stream=None):
    """x_p += dt * c_p(0, :) in FP64 with periodic wrap."""
    ex = _exec(stream, None, None)
    v = c_p[:, 0, :] if c_p.dim() == 3 else c_p
    check(_lib().picasso_advect(C.byref(mesh_desc), x_p.shape[0], float(dt), particle_field(x_p),
                                particle_field(v), C.byref(ex.desc)), "advect")


# ---------------------------------------------------------------------------
# cell sort
# ---------------------------------------------------------------------------


class Bins:
    """Result of cell_sort: the C descriptor plus the tensors it points to
    (and the spline records attached with spline_records, if any)."""

    def __init__(self, desc, tile_offset, tile_items):
        self.desc = desc
        self.tile_offset = tile_offset
        self.tile_items = tile_items
        self.records = None

    def attach_records(self, records):
        """Let the tiled transfers read these spline records (an (N, 4)
        float32 CUDA tensor from spline_records) instead of the positions;
        None detaches them."""
        self.records = records
        self.desc.records = records.data_ptr() if records is not None else None

    @property
    def num_tiles(self):
        return self.desc.num_tiles[0] * self.desc.num_tiles[1] * self.desc.num_tiles[2]


def num_tiles(sd, tile):
    """Tiles of the spline's mesh for a tile shape (bins per tile)."""
    nt = 1
    m = sd.desc.mesh
    for d in range(3):
        nb = m.own_extent[d] if m.periodic[d] else m.extent[d]
        nt *= -(-nb // tile[d])
    return nt


class SortBuffers:
    """Outputs of cell_sort kept across the steps of a time loop (key,
    perm, tile offsets, tile work items and the workspace), so that its
    sorts allocate nothing."""

    def __init__(self, sd, tile=(4, 8, 8)):
        dev = sd.x.device
        n = max(sd.num_particles, 1)
        nt = num_tiles(sd, tile)
        self.tile = tuple(tile)
        self.key = torch.empty(n, dtype=torch.int32, device=dev)
        self.perm = torch.empty(n, dtype=torch.int32, device=dev)
        self.tile_offset = torch.empty(nt + 1, dtype=torch.int64, device=dev)
        self.tile_items = torch.empty(nt + 1, dtype=torch.int32, device=dev)
        self.workspace = sort_workspace(sd, tile)


def cell_sort(sd, tile=(4, 8, 8), chunk=4096, stream=None, workspace=None, p2g_lanes=0,
              keys=None, out=None):
    """Stable sort of the spline's particles by (tile, bin).  Returns
    (key, perm, bins): keys and permutation as int32 tensors holding uint32
    values, and the Bins to pass to the transfers once the particle members
    have been permuted (see permute / permute_members).  `p2g_lanes` (1, 2, 4;
    0 = library choice) is the tiled P2G's lanes per particle.  `keys`: the
    particles' keys for this tile shape as APIC.g2p_advect(key_tile=tile)
    returned them; the sort then starts from them instead of the positions.
    `out`: a SortBuffers for this spline and tile shape whose tensors receive
    the results (nothing is allocated); the returned Bins then point into
    them, so they stay valid until the next sort into the same buffers."""
    lib = _lib()
    n = sd.num_particles
    t3 = (C.c_int32 * 3)(*tile)
    dev = sd.x.device
    nt = num_tiles(sd, tile)
    if out is not None:
        if (out.tile != tuple(tile) or out.key.numel() < n or out.perm.numel() < n
                or out.tile_offset.numel() != nt + 1):
            raise ValueError("SortBuffers made for another particle count or tile shape")
        key, perm, tile_offset, tile_items = out.key, out.perm, out.tile_offset, out.tile_items
        workspace = out.workspace
    else:
        nbytes = C.c_int64()
        check(lib.picasso_cell_sort_workspace(C.byref(sd.desc), n, t3, C.byref(nbytes)),
              "cell_sort_workspace")
        if workspace is None or workspace.numel() < nbytes.value:
            workspace = torch.empty(max(nbytes.value, 1), dtype=torch.uint8, device=dev)
        key = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
        perm = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
        tile_offset = torch.empty(nt + 1, dtype=torch.int64, device=dev)
        tile_items = torch.empty(nt + 1, dtype=torch.int32, device=dev)
    bins = _abi.Bins()
    ex = _exec(stream, None, None)
    if keys is not None:
        if keys.dtype != torch.int32 or keys.numel() < n or not keys.is_contiguous():
            raise ValueError("keys: contiguous int32 tensor of at least %d entries" % n)
        check(lib.picasso_cell_sort_keys(C.byref(sd.desc), n, keys.data_ptr(), t3, int(chunk),
                                         key.data_ptr(), perm.data_ptr(), tile_offset.data_ptr(),
                                         tile_items.data_ptr(), workspace.data_ptr(),
                                         workspace.numel(), C.byref(bins), C.byref(ex.desc)),
              "cell_sort")
    else:
        check(lib.picasso_cell_sort(C.byref(sd.desc), n, particle_field(sd.x), t3, int(chunk),
                                    key.data_ptr(), perm.data_ptr(), tile_offset.data_ptr(),
                                    tile_items.data_ptr(), workspace.data_ptr(),
                                    workspace.numel(), C.byref(bins), C.byref(ex.desc)),
              "cell_sort")
    bins.p2g_lanes = int(p2g_lanes)
    return key[:n], perm[:n], Bins(bins, tile_offset, tile_items)


def spline_records(sd, bins, out=None, attach=True, stream=None):
    """picasso_spline_records: the (N, 4) float32 tensor of the sorted
    particles' spline records (in-cell fractions and sort key) for `bins`;
    with attach=True the bins then carry them, so that the tiled P2G / G2P
    read them instead of the positions.  Call again after the positions
    change."""
    n = sd.num_particles
    if out is None:
        out = torch.empty((max(n, 1), 4), dtype=torch.float32, device=sd.x.device)
    elif (out.dtype != torch.float32 or out.shape[0] < n or out.shape[1:] != (4,)
          or not out.is_contiguous()):
        raise ValueError("out: contiguous (N, 4) float32 tensor")
    ex = _exec(stream, None, None)
    check(_lib().picasso_spline_records(C.byref(sd.desc), n, particle_field(sd.x),
                                        C.byref(bins.desc), out.data_ptr(), C.byref(ex.desc)),
          "spline_records")
    if attach:
        bins.attach_records(out)
    return out


def p2g_update_workspace(bins):
    """Bytes of device workspace APIC.p2g_update needs for these bins."""
    nbytes = C.c_int64()
    check(_lib().picasso_apic_p2g_update_workspace(C.byref(bins.desc), C.byref(nbytes)),
          "p2g_update_workspace")
    return nbytes.value


def sort_workspace(sd, tile=(4, 8, 8)):
    """Device workspace for cell_sort(sd, tile, workspace=...), to keep one
    across steps instead of allocating it in every call."""
    t3 = (C.c_int32 * 3)(*tile)
    nbytes = C.c_int64()
    check(_lib().picasso_cell_sort_workspace(C.byref(sd.desc), sd.num_particles, t3,
                                             C.byref(nbytes)), "cell_sort_workspace")
    return torch.empty(max(nbytes.value, 1), dtype=torch.uint8, device=sd.x.device)


def permute(perm, src, dst=None, stream=None):
    """dst[p] = src[perm[p]] for a particle member tensor."""
    if dst is None:
        dst = torch.empty_like(src)
    ncomp = 1
    for s in src.shape[1:]:
        ncomp *= s
    ex = _exec(stream, None, None)
    check(_lib().picasso_permute(src.shape[0], ncomp, perm.data_ptr(), particle_field(src),
                                 particle_field(dst), C.byref(ex.desc)), "permute")
    return dst


def permute_members(perm, *members, stream=None):
    return tuple(permute(perm, m, stream=stream) for m in members)


def tune_tiled_step(sd, m_p, c_p, m_i, mu_i, u_i, mass_threshold=1e-12, trials=3, stream=None):
    """Launch knobs of the precision-form tiled step measured on these
    particles (picasso_autotune): returns {"tile", "chunk", "p2g_lanes",
    "step_ms"}.  The particle tensors are not modified; m_i, mu_i (FixedGrid)
    and u_i (FP32) serve as the step's grids.  Allocates device memory and
    waits for the stream: call it at set-up, then pass tile / chunk to
    cell_sort and p2g_lanes to it (or to the bins)."""
    res = _abi.TuneResult()
    ex = _exec(stream, None, None)
    check(_lib().picasso_autotune(C.byref(sd.desc), sd.num_particles, particle_field(sd.x),
                                  particle_field(m_p), particle_field(c_p), grid_field(m_i),
                                  grid_field(mu_i), grid_field(u_i), float(mass_threshold),
                                  int(trials), C.byref(res), C.byref(ex.desc)), "autotune")
    return {"tile": tuple(res.tile), "chunk": res.chunk, "p2g_lanes": res.p2g_lanes,
            "step_ms": res.step_ms}


# ---------------------------------------------------------------------------
# 3x3 linear algebra
# ---------------------------------------------------------------------------


def mat3_inverse(a, x=None, stream=None):
    """Batched (n, 3, 3) FP64 determinant and cofactor inverse; with x (n, 3)
    also returns inverse(a) @ x."""
    a = a.contiguous()
    n = a.shape[0]
    inv = torch.empty_like(a)
    det = torch.empty(n, dtype=a.dtype, device=a.device)
    y = torch.empty_like(x) if x is not None else None
    ex = _exec(stream, None, None)
    check(_lib().picasso_mat3_inverse(n, a.data_ptr(), inv.data_ptr(), det.data_ptr(),
                                      x.contiguous().data_ptr() if x is not None else None,
                                      y.data_ptr() if y is not None else None, C.byref(ex.desc)),
          "mat3_inverse")
    return (inv, det, y) if x is not None else (inv, det)


# ---------------------------------------------------------------------------
# batched independent instances
# ---------------------------------------------------------------------------


class BatchInstance:
    """One APIC problem of a :class:`Batch`: its spline (collocated Node
    mesh and order), packed particle members sorted with :func:`cell_sort`
    (x (N, 3) FP64, m (N), c (N, 4, 3)), its grid arrays and its bins.
    Precision form: m, c float32, m_i / mu_i FixedGrid, u_i float32; FP64
    form: all float64."""

    def __init__(self, sd, m_p, c_p, m_i, mu_i, u_i, bins, mass_threshold=1e-12,
                 error_count=None):
        d = _abi.BatchInstance()
        d.spline = sd.desc
        d.num_particles = sd.num_particles
        d.x_p = particle_field(sd.x)
        d.m_p = particle_field(m_p)
        d.c_p = particle_field(c_p)
        d.m_i = grid_field(m_i)
        d.mu_i = grid_field(mu_i)
        d.u_i = grid_field(u_i)
        d.mass_threshold = float(mass_threshold)
        d.bins = bins.desc
        d.error_count = error_count.data_ptr() if error_count is not None else None
        self.desc = d
        # the batch reads these arrays at every step
        self._keep = (sd, m_p, c_p, m_i, mu_i, u_i, bins, error_count)


class Batch:
    """Many independent APIC problems stepped together: fill, P2G, grid
    velocity and G2P of every instance in persistent launches fed by one
    work queue (``mode="fused"``: one launch per step; ``"phased"``: one
    launch per phase).  ``step(graph=True)`` replays a captured CUDA graph.
    ``step_sequential`` issues the same work as single calls, instance after
    instance."""

    MODES = {"fused": _abi.BATCH_FUSED, "phased": _abi.BATCH_PHASED}

    def __init__(self, instances, mode="fused"):
        self.instances = list(instances)
        arr = (_abi.BatchInstance * len(self.instances))(*[i.desc for i in self.instances])
        h = C.c_void_p()
        check(_lib().picasso_batch_create(arr, len(self.instances), self.MODES[mode],
                                          C.byref(h)), "batch_create")
        self._h = h
        self.mode = mode

    def _stream(self, stream):
        s = stream if stream is not None else torch.cuda.current_stream()
        return s.cuda_stream

    def step(self, stream=None, graph=True):
        check(_lib().picasso_batch_step(self._h, self._stream(stream), int(bool(graph))),
              "batch_step")

    def step_sequential(self, stream=None):
        check(_lib().picasso_batch_step_sequential(self._h, self._stream(stream)),
              "batch_step_sequential")

    def status(self, stream=None):
        """Synchronises the stream; raises if a dependency wait ran out."""
        check(_lib().picasso_batch_status(self._h, self._stream(stream)), "batch_status")

    def set_wait_limit(self, polls):
        """Bound of the fused step's dependency waits (polls of ~0.25 us)."""
        check(_lib().picasso_batch_set_wait_limit(self._h, int(polls)), "batch_set_wait_limit")

    def cancel(self, stream=None):
        """Makes every dependency wait of the following fused steps give up
        until status() has reported it."""
        check(_lib().picasso_batch_cancel(self._h, self._stream(stream)), "batch_cancel")

    def info(self):
        inf = _abi.BatchInfo()
        check(_lib().picasso_batch_get_info(self._h, C.byref(inf)), "batch_get_info")
        return {"count": inf.count, "precision_form": bool(inf.precision_form),
                "grid_blocks": inf.grid_blocks, "smem_bytes": inf.smem_bytes,
                "items": list(inf.items), "particles": inf.particles}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib().picasso_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fixed_bits_for(max_abs):
    """Largest fraction bit count whose 64-bit fixed point still holds
    +-max_abs with a factor 4 of headroom."""
    if max_abs <= 0:
        return 40
    return max(0, min(62, 60 - int(math.ceil(math.log2(max_abs)))))
