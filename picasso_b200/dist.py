"""Domain decomposition of a periodic uniform mesh over ranks: slabs along x,
the halo exchange around the transfers, and the particle hand-off after the
particles move.

This is the multi-GPU form of the reference's FieldManager halo operations
(src/Picasso_FieldManager.hpp:157-164 scatter with Sum after P2G,
:174-181 gather before G2P) over Cabana::Grid halos, restated for one process
per GPU with torch.distributed (NCCL between GPUs, gloo on the CPU):

* Each rank owns ``own`` x-planes of nodes (cells) ``[x0, x0 + own)`` of the
  global periodic mesh and holds ``halo`` ghost planes on each side along x
  (y and z stay periodic and whole).  Its local mesh is non-periodic along x,
  so a stencil of one of its particles writes ghost planes instead of
  wrapping.  ``halo = 2`` covers quadratic and cubic stencils (a stencil
  reaches one plane below and two above the owned range).
* ``scatter_sum`` (after P2G): the ghost planes are sent to the neighbour
  that owns them and added into its owned planes, then cleared.  The grid
  arrays are (x, y, z[, comp]) row-major, so a block of x-planes is one
  contiguous range: no packing.  With the fixed-point accumulators of the
  precision form the sums are integers and do not depend on the order in
  which ghost planes arrive (the per-particle FP32 contributions can differ
  from a single-domain run in the last bit, because each rank measures
  logical coordinates from its own low corner).
* ``gather`` (before G2P): the owned boundary planes are copied into the
  neighbours' ghost planes.
* ``migrate`` (after the positions moved, by less than one slab): particles
  whose x left the owned range go to the neighbour that owns them; x is
  wrapped into the global box.
* ``halo_peers`` / ``map_peer_grids``: the device form of the two exchanges.
  With the neighbours' grids mapped into this process (CUDA IPC with peer
  access between GPUs), the tiled P2G adds its ghost-plane sums straight into
  the neighbour's owned planes and the tiled G2P reads its ghost velocities
  from the neighbour's owned planes (picasso_apic_p2g_halo /
  picasso_apic_g2p_halo): no ghost planes are sent, and the only host step
  left is a barrier after each transfer.

Every rank takes the same collective steps in the same order.  Two phases per
exchange (towards +x, then towards -x) keep the messages of two ranks that
are each other's upper and lower neighbour (2 ranks) unambiguous.
"""

import torch
import torch.distributed as tdist

from . import _abi
from .api import FieldLocation


class SlabDecomposition:
    """Slab ``rank`` of ``world`` of a periodic mesh of ``cells`` (nx, ny, nz)
    cells of size ``cell_size`` with low corner ``low``."""

    def __init__(self, cells, cell_size, world, rank, halo=2, low=(0.0, 0.0, 0.0), group=None):
        self.cells = [int(c) for c in cells]
        self.cell_size = float(cell_size)
        self.world = int(world)
        self.rank = int(rank)
        self.halo = int(halo) if world > 1 else 0
        self.low = [float(v) for v in low]
        self.group = group
        nx = self.cells[0]
        if nx < world * max(self.halo, 1):
            raise ValueError("each slab needs at least `halo` planes")
        base, extra = divmod(nx, world)
        self.sizes = [base + (1 if r < extra else 0) for r in range(world)]
        self.starts = [sum(self.sizes[:r]) for r in range(world)]
        self.x0 = self.starts[rank]
        self.own = self.sizes[rank]
        self.lower = (rank - 1) % world
        self.upper = (rank + 1) % world
        self.length = [self.cells[d] * self.cell_size for d in range(3)]

    # -- mesh -----------------------------------------------------------------
    def extent(self, location=FieldLocation.Node):
        if location != FieldLocation.Node:
            raise ValueError("the slab decomposition is defined for node fields")
        return (self.own + 2 * self.halo, self.cells[1], self.cells[2])

    def descriptor(self, location=FieldLocation.Node):
        """Local mesh of this rank: ghosted along x, periodic along y and z
        (and along x too on a single rank)."""
        m = _abi.Mesh()
        ext = self.extent(location)
        for d in range(3):
            m.extent[d] = ext[d]
            m.own_begin[d] = self.halo if d == 0 else 0
            m.own_extent[d] = self.own if d == 0 else self.cells[d]
            m.periodic[d] = 0 if (d == 0 and self.world > 1) else 1
            m.low_corner[d] = self.low[d] + ((self.x0 - self.halo) * self.cell_size if d == 0
                                             else 0.0)
            m.cell_size[d] = self.cell_size
        return m

    def global_descriptor(self, location=FieldLocation.Node):
        """The whole periodic mesh (for the position update's wrap)."""
        m = _abi.Mesh()
        for d in range(3):
            m.extent[d] = self.cells[d]
            m.own_begin[d] = 0
            m.own_extent[d] = self.cells[d]
            m.periodic[d] = 1
            m.low_corner[d] = self.low[d]
            m.cell_size[d] = self.cell_size
        return m

    def zeros(self, location=FieldLocation.Node, ncomp=None, dtype=torch.float64, device="cuda"):
        shape = self.extent(location) + ((ncomp,) if ncomp else ())
        return torch.zeros(shape, dtype=dtype, device=device)

    def owned(self, grid):
        """View of the owned x-planes of a local grid array."""
        return grid[self.halo:self.halo + self.own]

    # -- particles ------------------------------------------------------------
    def owner(self, x):
        """Rank owning each position (x wrapped into the global box)."""
        plane = torch.floor((x[:, 0] - self.low[0]) / self.cell_size).to(torch.int64)
        plane = torch.remainder(plane, self.cells[0])
        starts = torch.tensor(self.starts[1:], dtype=torch.int64, device=x.device)
        return torch.bucketize(plane, starts, right=True)

    def wrap(self, x):
        """Positions wrapped into the global periodic box (in place)."""
        for d in range(3):
            lo, ln = self.low[d], self.length[d]
            x[:, d] = lo + torch.remainder(x[:, d] - lo, ln)
        return x

    # -- exchanges inside the transfers ----------------------------------------
    def halo_peers(self, lower, upper):
        """HaloPeers for APIC.p2g / APIC.g2p(peers=...): `lower` and `upper`
        are the neighbours' grids of the same shapes as this rank's -- (m_i,
        mu_i) for P2G, u_i for G2P -- as tensors (or FixedGrid) addressable
        from this device: the neighbouring slabs' arrays on this GPU, or the
        ones map_peer_grids returns.  Local plane p < halo is the lower
        neighbour's plane p + own(lower), plane p >= halo + own the upper
        neighbour's plane p - own."""
        if self.world == 1:
            raise ValueError("a single slab is periodic along x and has no neighbours")

        def ptrs(g):
            gs = g if isinstance(g, (tuple, list)) else (g,)
            return [(x.raw if hasattr(x, "raw") else x).data_ptr() for x in gs] + [None]

        p = _abi.HaloPeers()
        p.lo_end = self.halo
        p.hi_begin = self.halo + self.own
        p.lo_shift = self.sizes[self.lower]
        p.hi_shift = -self.own
        lo, hi = ptrs(lower), ptrs(upper)
        for f in range(2):
            p.lo[f] = lo[f]
            p.hi[f] = hi[f]
        return p

    def map_peer_grids(self, *grids):
        """Maps the neighbours' copies of `grids` into this process: every rank
        calls it with its own grids (same shapes and order; FixedGrid or
        tensors) and gets (lower, upper), lists of tensors over the lower and
        upper neighbours' memory (CUDA IPC handles exchanged through the
        process group; peer access between GPUs).  The grids must stay
        allocated while the mapping is used."""
        from torch.multiprocessing.reductions import reduce_tensor
        raws = [g.raw if hasattr(g, "raw") else g for g in grids]
        # per grid: the IPC handle of its storage and the view's geometry
        mine = [reduce_tensor(r) for r in raws]
        everyone = [None] * self.world
        tdist.all_gather_object(everyone, mine, group=self.group)

        def load(r):
            return [fn(*args) for fn, args in everyone[r]]
        return load(self.lower), load(self.upper)

    # -- exchanges ------------------------------------------------------------
    def _shift(self, send, to, recv, frm):
        """One phase: send `send` to rank `to` while receiving `recv` from rank
        `frm`; empty tensors are not sent (both sides know the sizes)."""
        ops = []
        if send.numel():
            ops.append(tdist.P2POp(tdist.isend, send.contiguous(), to, self.group))
        if recv.numel():
            ops.append(tdist.P2POp(tdist.irecv, recv, frm, self.group))
        if ops:
            for r in tdist.batch_isend_irecv(ops):
                r.wait()

    def _exchange(self, send_up, send_down, like_lower=None, like_upper=None):
        """Sends send_up to the upper neighbour and send_down to the lower one;
        returns (from_lower, from_upper), shaped like send_up / send_down
        unless given.  Same steps on every rank: +x first, then -x."""
        from_lower = torch.empty_like(send_up) if like_lower is None else like_lower
        from_upper = torch.empty_like(send_down) if like_upper is None else like_upper
        self._shift(send_up, self.upper, from_lower, self.lower)
        self._shift(send_down, self.lower, from_upper, self.upper)
        return from_lower, from_upper

    def scatter_sum(self, *grids):
        """After P2G: add every ghost plane into its owner's owned plane and
        clear the ghosts (FieldManager halo scatter with Sum)."""
        if self.world == 1:
            return
        h, o = self.halo, self.own
        for g in grids:
            raw = g.raw if hasattr(g, "raw") else g
            up = raw[h + o:2 * h + o].clone()    # my upper ghosts = upper's first owned
            down = raw[0:h].clone()              # my lower ghosts = lower's last owned
            from_lower, from_upper = self._exchange(up, down)
            raw[h:2 * h] += from_lower          # lower's upper ghosts -> my first planes
            raw[o:o + h] += from_upper          # upper's lower ghosts -> my last planes
            raw[0:h] = 0
            raw[h + o:2 * h + o] = 0

    def gather(self, *grids):
        """Before G2P: fill the ghost planes with the neighbours' owned planes
        (FieldManager halo gather)."""
        if self.world == 1:
            return
        h, o = self.halo, self.own
        for g in grids:
            raw = g.raw if hasattr(g, "raw") else g
            up = raw[o:o + h].clone()            # my last owned -> upper's lower ghosts
            down = raw[h:2 * h].clone()          # my first owned -> lower's upper ghosts
            from_lower, from_upper = self._exchange(up, down)
            raw[0:h] = from_lower
            raw[h + o:2 * h + o] = from_upper

    def migrate(self, x, *members):
        """After the positions moved: wrap x into the global box and hand the
        particles that left this slab to the neighbour that owns them (a
        particle may move at most one slab per call).  Returns the new
        (x, *members) of this rank, own particles first in their old order,
        then those from the lower and from the upper neighbour."""
        self.wrap(x)
        if self.world == 1:
            return (x,) + members
        own = self.owner(x)
        keep = own == self.rank
        to_up = own == self.upper
        to_down = (own == self.lower) & ~to_up
        if bool(((~keep) & (~to_up) & (~to_down)).any()):
            raise RuntimeError("a particle moved further than one slab")
        arrays = (x,) + members
        # counts first, so that every rank can size its receive buffers
        counts = torch.tensor([int(to_up.sum()), int(to_down.sum())], dtype=torch.int64,
                              device=x.device)
        c_lower, c_upper = self._exchange(counts[:1].clone(), counts[1:].clone())
        out = []
        for a in arrays:
            tail = tuple(a.shape[1:])
            recv_lower = torch.empty((int(c_lower.item()),) + tail, dtype=a.dtype, device=a.device)
            recv_upper = torch.empty((int(c_upper.item()),) + tail, dtype=a.dtype, device=a.device)
            self._exchange(a[to_up], a[to_down], recv_lower, recv_upper)
            out.append(torch.cat([a[keep], recv_lower, recv_upper]))
        return tuple(out)
