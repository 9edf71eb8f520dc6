"""Bulk flush of the tiled P2G (cp.reduce.async.bulk .add.u64).

When the mass and momentum grids are views of one (..., 4) 64-bit
accumulator, the tiled P2G adds its node box to HBM with one bulk reduction
per k-row instead of one reduction per node and field.  The accumulators
hold integer sums, so the result must equal, bit for bit, the element-wise
flush into separate mass and momentum arrays (the layout the bulk form does
not take).  Checked for every order and lane split, periodic meshes whose
size is not a multiple of the tile (rows that wrap), meshes with halos,
non-periodic meshes (rows that end at the mesh), records and positions, and
the overflow count.
"""

import numpy as np
import pytest
import torch

from particles import clustered_particles, periodic_mesh, uniform_particles
from picasso_b200 import (APIC, FieldLocation, FixedGrid, UniformMesh, cell_sort, create_spline,
                          permute_members, spline_records)

pytestmark = pytest.mark.gpu
BITS = 36


def _dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _sorted(mesh, loc, order, x, m, c, tile, lanes, records):
    xd = _dev(x)
    md, cd = _dev(m, torch.float32), _dev(c, torch.float32)
    sd = create_spline(loc, order, mesh, xd)
    _, perm, bins = cell_sort(sd, tile, chunk=512, p2g_lanes=lanes)
    xd, md, cd = permute_members(perm, xd, md, cd)
    sd = create_spline(loc, order, mesh, xd)
    if records:
        spline_records(sd, bins)
    return sd, md, cd, bins


def _both(mesh, order, x, m, c, tile=(4, 4, 8), lanes=0, records=False, bits=BITS,
          loc=FieldLocation.Node):
    """P2G into a packed (..., 4) accumulator (bulk flush) and into separate
    mass / momentum arrays (element-wise flush); returns both as (..., 4)
    int64 arrays, the error counts and the overflow counts."""
    sd, md, cd, bins = _sorted(mesh, loc, order, x, m, c, tile, lanes, records)
    ext = mesh.extent(loc)
    acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
    sep_m = torch.zeros(ext, dtype=torch.int64, device="cuda")
    sep_mu = torch.zeros(ext + (3,), dtype=torch.int64, device="cuda")
    errs, ovfs = [], []
    for gm, gmu in ((FixedGrid(acc[..., 0], bits), FixedGrid(acc[..., 1:], bits)),
                    (FixedGrid(sep_m, bits), FixedGrid(sep_mu, bits))):
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        ovf = torch.zeros(1, dtype=torch.int32, device="cuda")
        APIC.p2g(md, cd, gm, gmu, sd, bins=bins, error_count=err, overflow_count=ovf)
        errs.append(err)
        ovfs.append(ovf)
    torch.cuda.synchronize()
    sep = torch.cat([sep_m[..., None], sep_mu], dim=-1)
    return acc, sep, [int(e.item()) for e in errs], [int(o.item()) for o in ovfs]


@pytest.mark.parametrize("order,lanes", [(1, 1), (1, 4), (2, 1), (2, 2), (2, 4), (3, 4)])
@pytest.mark.parametrize("kind", ["uniform", "clustered"])
def test_bulk_flush_equals_elementwise(cuda, order, lanes, kind):
    mesh = periodic_mesh(22, halo=1)  # 22: rows wrap around the periodic end
    if kind == "uniform":
        x, m, c = uniform_particles(mesh, 5, seed=110 + order)
    else:
        x, m, c = clustered_particles(mesh, 22 ** 3 * 5, nblob=3, sigma_cells=1.5, frac=0.7,
                                      seed=120 + order)
    acc, sep, errs, ovfs = _both(mesh, order, x, m, c, lanes=lanes,
                                 records=(kind == "clustered"))
    assert errs == [0, 0] and ovfs == [0, 0]
    assert int((sep != 0).sum().item()) > 0
    assert torch.equal(acc, sep)


@pytest.mark.parametrize("tile", [(4, 8, 8), (3, 5, 7), (8, 8, 16)])
def test_bulk_flush_tile_shapes(cuda, tile):
    mesh = periodic_mesh(24, halo=0)
    x, m, c = clustered_particles(mesh, 24 ** 3 * 6, nblob=4, sigma_cells=2.0, frac=0.7, seed=130)
    acc, sep, errs, _ = _both(mesh, 2, x, m, c, tile=tile, records=True)
    assert errs == [0, 0]
    assert torch.equal(acc, sep)


@pytest.mark.parametrize("loc", [FieldLocation.Node, FieldLocation.Cell])
def test_bulk_flush_non_periodic_mesh(cuda, loc):
    """Rows that reach past the mesh end are cut there; particles outside
    the mesh are skipped and counted the same way."""
    mesh = UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1 / 18, periodic=(False, True, False),
                       halo_cell_width=2)
    rng = np.random.default_rng(131)
    x = rng.uniform(-0.3, 1.3, (18 ** 3 * 5, 3))
    m = rng.uniform(0.5, 1.5, x.shape[0])
    c = np.concatenate([rng.standard_normal((x.shape[0], 1, 3)),
                        0.1 * rng.standard_normal((x.shape[0], 3, 3))], axis=1)
    acc, sep, errs, _ = _both(mesh, 2, x, m, c, tile=(4, 4, 8), loc=loc)
    assert errs[0] == errs[1] and errs[0] > 0
    assert torch.equal(acc, sep)


def test_bulk_flush_counts_overflow(cuda):
    mesh = periodic_mesh(12, halo=0)
    x, m, c = uniform_particles(mesh, 4, seed=132, jitter_mass=False)
    acc, sep, errs, ovfs = _both(mesh, 2, x, m * 100.0, c, bits=60)
    assert ovfs[0] == ovfs[1] and ovfs[0] > 0
    assert torch.equal(acc, sep)
