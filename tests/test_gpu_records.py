"""Spline records (picasso_spline_records) and the tiled transfers that read
them instead of the positions.

A record is (t_x, t_y, t_z, key): the in-cell fraction of the particle's
logical position per dimension in FP32 and its sort key.  Checked here:
  * the key is the cell sort's key of the sorted particle, bit for bit, and
    the fractions are the FP64 fraction rounded to FP32 (restated in numpy
    from the logical-position rule of every kernel);
  * the tiled P2G and G2P give bit-identical results from records and from
    positions (same splines, same bins), for every order and P2G lane split;
  * particles outside a non-periodic mesh and particles of the wrong tile
    are skipped and counted as with positions.
"""

import numpy as np
import pytest
import torch

from particles import clustered_particles, periodic_mesh, uniform_particles
from picasso_b200 import (APIC, FieldLocation, FixedGrid, UniformMesh, cell_sort, create_spline,
                          grid_velocity, permute_members, spline_records)

pytestmark = pytest.mark.gpu
BITS = 36
SHIFT = {1: 0.0, 2: 0.5, 3: 0.0}


def _dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _fractions(mesh, loc, order, x):
    """FP64 logical position (x - lo) / dx + shift, rounded step by step,
    its in-cell fraction rounded to FP32."""
    d = mesh.descriptor(loc)
    lo = np.array([d.low_corner[i] for i in range(3)])
    rdx = 1.0 / np.array([d.cell_size[i] for i in range(3)])
    off = {FieldLocation.Node: 0.0, FieldLocation.Cell: 0.5}[loc]
    x0 = (x - (lo + off / rdx)) * rdx + SHIFT[order]
    return (x0 - np.floor(x0)).astype(np.float32)


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("tile", [(4, 8, 8), (3, 4, 5)])
def test_records_are_sort_keys_and_fractions(cuda, order, tile):
    mesh = periodic_mesh(24, halo=1)
    x, _, _ = clustered_particles(mesh, 24 ** 3 * 4, nblob=3, sigma_cells=1.5, frac=0.6,
                                  seed=40 + order)
    loc = FieldLocation.Node
    sd = create_spline(loc, order, mesh, _dev(x))
    key, perm, bins = cell_sort(sd, tile)
    (xs,) = permute_members(perm, sd.x)
    rec = spline_records(create_spline(loc, order, mesh, xs), bins)
    torch.cuda.synchronize()
    r = rec.cpu().numpy()
    assert np.array_equal(r[:, 3].view(np.uint32), key.cpu().numpy().view(np.uint32))
    t = _fractions(mesh, loc, order, xs.cpu().numpy())
    # the fraction is exact to the FP32 rounding of the same FP64 value
    assert np.array_equal(r[:, :3], t)
    assert bins.desc.records == rec.data_ptr()


def _tiled_step(mesh, order, x, m, c, tile, lanes, records):
    loc = FieldLocation.Node
    xd = _dev(x)
    md, cd = _dev(m, torch.float32), _dev(c, torch.float32)
    sd = create_spline(loc, order, mesh, xd)
    _, perm, bins = cell_sort(sd, tile, chunk=512, p2g_lanes=lanes)
    xd, md, cd = permute_members(perm, xd, md, cd)
    sd = create_spline(loc, order, mesh, xd)
    if records:
        spline_records(sd, bins)
    ext = mesh.extent(loc)
    acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
    gm, gmu = FixedGrid(acc[..., 0], BITS), FixedGrid(acc[..., 1:], BITS)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    APIC.p2g(md, cd, gm, gmu, sd, bins=bins, error_count=err)
    u = torch.zeros(ext + (3,), dtype=torch.float32, device="cuda")
    grid_velocity(sd.desc.mesh, gm, gmu, u, 1e-12)
    out = torch.zeros_like(cd)
    APIC.g2p(u, out, sd, bins=bins, error_count=err)
    torch.cuda.synchronize()
    return acc, out, int(err.item())


@pytest.mark.parametrize("order,lanes", [(1, 1), (1, 2), (1, 4), (2, 1), (2, 2), (2, 4), (3, 4)])
@pytest.mark.parametrize("kind", ["uniform", "clustered"])
def test_record_path_is_bit_identical_to_positions(cuda, order, lanes, kind):
    mesh = periodic_mesh(20, halo=0)
    if kind == "uniform":
        x, m, c = uniform_particles(mesh, 6, seed=60 + order)
    else:
        x, m, c = clustered_particles(mesh, 20 ** 3 * 6, nblob=3, sigma_cells=1.5, frac=0.7,
                                      seed=70 + order)
    tile = (4, 4, 8)
    a0, c0, e0 = _tiled_step(mesh, order, x, m, c, tile, lanes, records=False)
    a1, c1, e1 = _tiled_step(mesh, order, x, m, c, tile, lanes, records=True)
    assert e0 == 0 and e1 == 0
    assert torch.equal(a0, a1)
    assert torch.equal(c0, c1)


def test_records_outside_non_periodic_mesh_are_counted(cuda):
    mesh = UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1 / 8, periodic=(False, False, False),
                       halo_cell_width=1)
    rng = np.random.default_rng(8)
    x = rng.uniform(-0.3, 1.3, (6000, 3))
    m = rng.uniform(0.5, 1.5, 6000)
    c = rng.standard_normal((6000, 4, 3)) * 0.1
    a0, c0, e0 = _tiled_step(mesh, 2, x, m, c, (4, 4, 4), 1, records=False)
    a1, c1, e1 = _tiled_step(mesh, 2, x, m, c, (4, 4, 4), 1, records=True)
    assert e0 > 0 and e0 == e1
    assert torch.equal(a0, a1)
    assert torch.equal(c0, c1)


def test_stale_records_of_another_tile_are_skipped(cuda):
    """Records whose key names another tile (positions moved without new
    records) are skipped and counted, never written outside their tile."""
    mesh = periodic_mesh(16, halo=0)
    x, m, c = uniform_particles(mesh, 4, seed=81)
    loc = FieldLocation.Node
    xd = _dev(x)
    md, cd = _dev(m, torch.float32), _dev(c, torch.float32)
    sd = create_spline(loc, 2, mesh, xd)
    _, perm, bins = cell_sort(sd, (4, 4, 4), chunk=256)
    xd, md, cd = permute_members(perm, xd, md, cd)
    sd = create_spline(loc, 2, mesh, xd)
    rec = spline_records(sd, bins)
    # keys of the first 100 particles point to the last tile instead
    rec[:100, 3] = torch.tensor(np.full(100, (bins.num_tiles - 1) * 64, np.uint32).view(np.float32),
                                device="cuda")
    ext = mesh.extent(loc)
    acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
    gm, gmu = FixedGrid(acc[..., 0], BITS), FixedGrid(acc[..., 1:], BITS)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    APIC.p2g(md, cd, gm, gmu, sd, bins=bins, error_count=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 100
    total = float(gm.to_float().sum())
    assert abs(total - float(md.double()[100:].sum())) < 1e-6 * total
