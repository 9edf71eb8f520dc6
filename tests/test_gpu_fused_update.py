"""P2G with the grid update fused into its flush (picasso_apic_p2g_update).

The work items of the tiled P2G count their arrival at the node regions they
touch and the last one converts the region's nodes with the grid update.
Checked here, bit for bit, against picasso_apic_p2g followed by
picasso_grid_update on the same particles: grid mass and momentum, FP32 and
FP64 velocity, for every order, periodic meshes whose size is not a multiple
of the tile, records and positions, and a non-periodic mesh with walls,
gravity and a force field.  Tiles too small for the fused form (fewer than
K - 1 bins) take the two separate passes, with the same results.
"""

import numpy as np
import pytest
import torch

from particles import clustered_particles, periodic_mesh, uniform_particles
from picasso_b200 import (APIC, FieldLocation, FixedGrid, UniformMesh, cell_sort, create_spline,
                          grid_update, p2g_update_workspace, permute_members, spline_records)

pytestmark = pytest.mark.gpu
BITS = 36


def _dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _prepare(mesh, order, x, m, c, tile, records):
    loc = FieldLocation.Node
    xd = _dev(x)
    md, cd = _dev(m, torch.float32), _dev(c, torch.float32)
    sd = create_spline(loc, order, mesh, xd)
    _, perm, bins = cell_sort(sd, tile, chunk=512)
    xd, md, cd = permute_members(perm, xd, md, cd)
    sd = create_spline(loc, order, mesh, xd)
    if records:
        spline_records(sd, bins)
    return sd, md, cd, bins


def _grids(mesh):
    ext = mesh.extent(FieldLocation.Node)
    acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
    u = torch.full(ext + (3,), 7.0, dtype=torch.float32, device="cuda")  # overwritten
    u64 = torch.full(ext + (3,), 7.0, dtype=torch.float64, device="cuda")
    return acc, FixedGrid(acc[..., 0], BITS), FixedGrid(acc[..., 1:], BITS), u, u64


def _compare(mesh, order, x, m, c, tile, records, **upd):
    sd, md, cd, bins = _prepare(mesh, order, x, m, c, tile, records)
    desc = sd.desc.mesh
    a0, gm0, gmu0, u0, w0 = _grids(mesh)
    a1, gm1, gmu1, u1, w1 = _grids(mesh)
    err0 = torch.zeros(1, dtype=torch.int32, device="cuda")
    err1 = torch.zeros(1, dtype=torch.int32, device="cuda")
    # reference: the two separate passes; the grid update writes the owned
    # nodes only, so both velocity grids start from the same values
    APIC.p2g(md, cd, gm0, gmu0, sd, bins=bins, error_count=err0)
    grid_update(desc, gm0, gmu0, u0, u64_i=w0, **upd)
    ws = torch.empty(p2g_update_workspace(bins), dtype=torch.uint8, device="cuda")
    ws.fill_(0xAB)  # the call clears its counters
    APIC.p2g_update(md, cd, gm1, gmu1, u1, sd, u64_i=w1, workspace=ws, bins=bins,
                    error_count=err1, **upd)
    torch.cuda.synchronize()
    assert int(err0.item()) == int(err1.item())
    assert torch.equal(a0, a1)
    own = [slice(desc.own_begin[d], desc.own_begin[d] + desc.own_extent[d])
           if desc.periodic[d] else slice(None) for d in range(3)]
    assert torch.equal(u0[own[0], own[1], own[2]], u1[own[0], own[1], own[2]])
    assert torch.equal(w0[own[0], own[1], own[2]], w1[own[0], own[1], own[2]])
    return u1


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("tile", [(4, 8, 8), (4, 4, 4), (3, 5, 6)])
@pytest.mark.parametrize("kind", ["uniform", "clustered"])
def test_fused_update_bit_identical_periodic(cuda, order, tile, kind):
    mesh = periodic_mesh(22, halo=1)  # 22 is not a multiple of the tiles
    if kind == "uniform":
        x, m, c = uniform_particles(mesh, 5, seed=90 + order)
    else:
        x, m, c = clustered_particles(mesh, 22 ** 3 * 5, nblob=3, sigma_cells=1.5, frac=0.7,
                                      seed=95 + order)
    _compare(mesh, order, x, m, c, tile, records=(kind == "clustered"), dt=1e-3,
             gravity=(0.0, -9.81, 0.0))


def test_fused_update_walls_gravity_force(cuda):
    mesh = UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1 / 12, periodic=(True, False, False),
                       halo_cell_width=2)
    rng = np.random.default_rng(97)
    x = rng.uniform(0.02, 0.98, (12 ** 3 * 4, 3))
    m = rng.uniform(0.5, 1.5, x.shape[0])
    c = np.concatenate([rng.standard_normal((x.shape[0], 1, 3)),
                        0.1 * rng.standard_normal((x.shape[0], 3, 3))], axis=1)
    ext = mesh.extent(FieldLocation.Node)
    f = torch.as_tensor(rng.standard_normal(ext + (3,)), device="cuda")
    walls = [("none", "none"), ("no_slip", "free_slip"), ("free_slip", "no_slip")]
    _compare(mesh, 2, x, m, c, (4, 4, 4), records=True, dt=2e-3, gravity=(0.0, 0.0, -9.81),
             f_i=f, walls=walls, wall_width=2)


@pytest.mark.parametrize("order,tile", [(3, (1, 4, 4)), (2, (4, 4, 1))])
def test_small_tiles_take_separate_passes(cuda, order, tile):
    """Tiles of fewer than K - 1 bins: the call runs P2G and the update as
    two passes (no fused launch), same results."""
    mesh = periodic_mesh(12, halo=0)
    x, m, c = uniform_particles(mesh, 4, seed=99)
    _compare(mesh, order, x, m, c, tile, records=False, dt=1e-3)


def test_untouched_nodes_get_zero_velocity(cuda):
    """Regions that no work item touches (an empty part of the mesh) are
    not converted by any item: their velocity is the empty node's, 0."""
    mesh = periodic_mesh(24, halo=0)
    rng = np.random.default_rng(100)
    x = rng.uniform(0.0, 0.25, (4000, 3))  # particles in one corner only
    m = rng.uniform(0.5, 1.5, 4000)
    c = np.concatenate([rng.standard_normal((4000, 1, 3)),
                        0.1 * rng.standard_normal((4000, 3, 3))], axis=1)
    u = _compare(mesh, 2, x, m, c, (4, 4, 4), records=False, dt=1e-3)
    # the stencils reach nodes 23 (wrapped) .. 7 along each dimension
    assert float(u[9:22, 9:22, 9:22].abs().max()) == 0.0
    assert float(u[:7, :7, :7].abs().max()) > 0.0
