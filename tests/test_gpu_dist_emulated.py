"""The GPU kernels on the ghosted local meshes of a slab decomposition, all
slabs in one process on one GPU (the exchange between them done by tensor
adds, as SlabDecomposition.scatter_sum / gather would do between ranks).

Checked against the single-domain tiled kernels: the owned planes of every
slab after the halo sum, and c_p of every particle after G2P on its slab with
the ghosts filled.  Each slab measures logical coordinates from its own low
corner, so a particle's FP32 weights can differ from the single-domain ones
in the last bit: the tolerance is 1e-6 (normwise relative), well below the
1e-5 the precision form is held to against the FP64 oracle.
"""

import numpy as np
import pytest
import torch

from particles import clustered_particles, periodic_mesh, rel_err
from picasso_b200 import (APIC, FieldLocation, FixedGrid, cell_sort, create_spline,
                          permute_members)
from picasso_b200.dist import SlabDecomposition

pytestmark = pytest.mark.gpu
N = 24
BITS = 36


class _Slab:
    """Minimal mesh object for create_spline on a slab's local mesh."""

    def __init__(self, dec):
        self.dec = dec

    def descriptor(self, location):
        return self.dec.descriptor(location)


def _p2g(mesh_obj, ext, order, x, m, c, tile):
    sd0 = create_spline(FieldLocation.Node, order, mesh_obj, x)
    _, perm, bins = cell_sort(sd0, tile)
    xs, ms, cs = permute_members(perm, x, m, c)
    sd = create_spline(FieldLocation.Node, order, mesh_obj, xs)
    acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    APIC.p2g(ms, cs, FixedGrid(acc[..., 0], BITS), FixedGrid(acc[..., 1:], BITS), sd, bins=bins,
             error_count=err)
    return acc, sd, cs, bins, perm, int(err.item())


@pytest.mark.parametrize("world,order", [(3, 2), (2, 3)])
def test_slabs_reproduce_single_domain(cuda, world, order):
    mesh = periodic_mesh(N, halo=0)
    x, m, c = clustered_particles(mesh, N ** 3 * 4, nblob=4, sigma_cells=2.0, frac=0.6, seed=610)
    xd = torch.as_tensor(x, device="cuda")
    md = torch.as_tensor(m, dtype=torch.float32, device="cuda")
    cd = torch.as_tensor(c, dtype=torch.float32, device="cuda").contiguous()
    ext = mesh.extent(FieldLocation.Node)
    acc_g, sd_g, cs_g, bins_g, perm_g, err = _p2g(mesh, ext, order, xd, md, cd, (4, 8, 8))
    assert err == 0
    decs = [SlabDecomposition((N, N, N), 1.0 / N, world, r) for r in range(world)]
    parts = []
    for dec in decs:
        mine = dec.owner(xd) == dec.rank
        acc, sd, cs, bins, perm, err = _p2g(_Slab(dec), dec.extent(), order, xd[mine], md[mine],
                                            cd[mine], (4, 8, 8))
        assert err == 0
        parts.append((dec, acc, sd, cs, bins, mine))
    # halo sum between slabs (what scatter_sum does between ranks)
    accs = [p[1] for p in parts]
    sums = [a.clone() for a in accs]
    for r, dec in enumerate(decs):
        h, o = dec.halo, dec.own
        sums[dec.upper][h:2 * h] += accs[r][h + o:2 * h + o]
        sums[dec.lower][decs[dec.lower].own:decs[dec.lower].own + h] += accs[r][0:h]
    for dec, s in zip(decs, sums):
        got = dec.owned(s).double().cpu().numpy()
        ref = acc_g[dec.x0:dec.x0 + dec.own].double().cpu().numpy()
        assert rel_err(got[..., 0], ref[..., 0]) <= 1e-6
        assert rel_err(got[..., 1:], ref[..., 1:]) <= 1e-6
    # G2P: single domain, then each slab with its ghosts filled from the
    # global velocity (what gather provides)
    u = torch.randn(ext + (3,), generator=torch.Generator(device="cuda").manual_seed(611),
                    device="cuda", dtype=torch.float32)
    c_g = torch.zeros_like(cs_g)
    APIC.g2p(u, c_g, sd_g, bins=bins_g)
    c_full = torch.empty_like(c_g)
    c_full[perm_g.long()] = c_g  # back to the input order
    for dec, _, sd, cs, bins, mine in parts:
        planes = torch.tensor([(dec.x0 - dec.halo + i) % N for i in range(dec.extent()[0])],
                              device="cuda")
        ul = u[planes].contiguous()
        cl = torch.zeros_like(cs)
        APIC.g2p(ul, cl, sd, bins=bins)
        # the slab's particles in the order of its sort
        sd0 = create_spline(FieldLocation.Node, order, _Slab(dec), xd[mine])
        _, perm, _ = cell_sort(sd0, (4, 8, 8))
        expect = c_full[mine][perm.long()]
        assert rel_err(cl.double().cpu().numpy(), expect.double().cpu().numpy()) <= 1e-6
