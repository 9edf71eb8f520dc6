"""Edge cases through the C ABI: empty particle sets, single particles,
particles exactly on cell faces and on the periodic box faces, tiles that do
not divide the mesh, tiles too large for shared memory (plain-path fallback),
and work items that split one tile many times."""

import numpy as np
import pytest
import torch

import oracle
from particles import periodic_mesh, rel_err, uniform_particles
from picasso_b200 import (APIC, FieldLocation, FixedGrid, PolyPIC, advect, cell_sort,
                          create_spline, grid_velocity, permute, permute_members)

pytestmark = pytest.mark.gpu
BITS = 36


def _dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def test_empty_particle_sets_are_no_ops(cuda):
    mesh = periodic_mesh(8, halo=0)
    loc = FieldLocation.Node
    ext = mesh.extent(loc)
    x = torch.zeros((0, 3), dtype=torch.float64, device="cuda")
    m = torch.zeros((0,), dtype=torch.float32, device="cuda")
    c = torch.zeros((0, 4, 3), dtype=torch.float32, device="cuda")
    sd = create_spline(loc, 2, mesh, x)
    key, perm, bins = cell_sort(sd, (4, 4, 4))
    torch.cuda.synchronize()
    assert key.numel() == 0 and perm.numel() == 0
    assert int(bins.tile_offset.abs().sum()) == 0 and int(bins.tile_items.abs().sum()) == 0
    acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
    gm, gmu = FixedGrid(acc[..., 0], BITS), FixedGrid(acc[..., 1:], BITS)
    APIC.p2g(m, c, gm, gmu, sd, bins=bins)
    APIC.p2g(m, c, gm, gmu, sd)
    u = torch.zeros(ext + (3,), dtype=torch.float32, device="cuda")
    APIC.g2p(u, c, sd, bins=bins)
    APIC.g2p_advect(u, c, sd, 0.1, bins=bins)
    advect(sd.desc.mesh, x, c, 0.1)
    assert permute(perm, c).numel() == 0
    mu = torch.zeros((0, 8, 3), dtype=torch.float64, device="cuda")
    g64 = torch.zeros(ext + (4,), dtype=torch.float64, device="cuda")
    sd1 = create_spline(loc, 1, mesh, x)
    PolyPIC.p2g(m.double(), mu, mu, g64[..., 1:], g64[..., 0], 0.01, sd1)
    PolyPIC.g2p(g64[..., 1:], mu, sd1)
    torch.cuda.synchronize()
    assert int(acc.abs().sum()) == 0 and float(g64.abs().sum()) == 0.0


def _step_vs_oracle(mesh, order, x, m, c, tile, chunk):
    loc = FieldLocation.Node
    ext = mesh.extent(loc)
    sdo = create_spline(loc, order, mesh, None).desc
    gm_o, gmu_o, gu_o = np.zeros(ext), np.zeros(ext + (3,)), np.zeros(ext + (3,))
    oracle.apic_p2g(sdo, x, m, c, gm_o, gmu_o)
    oracle.grid_velocity(sdo.mesh, gm_o, gmu_o, gu_o, 1e-12)
    c_o = np.zeros_like(c)
    oracle.apic_g2p(sdo, x, gu_o, c_o)
    xd = _dev(x)
    md, cd = _dev(m, torch.float32), _dev(c, torch.float32)
    sd0 = create_spline(loc, order, mesh, xd)
    _, perm, bins = cell_sort(sd0, tile, chunk=chunk)
    xd, md, cd = permute_members(perm, xd, md, cd)
    sd = create_spline(loc, order, mesh, xd)
    acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
    gm, gmu = FixedGrid(acc[..., 0], BITS), FixedGrid(acc[..., 1:], BITS)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    APIC.p2g(md, cd, gm, gmu, sd, bins=bins, error_count=err)
    u32 = torch.zeros(ext + (3,), dtype=torch.float32, device="cuda")
    grid_velocity(sd.desc.mesh, gm, gmu, u32, 1e-12)
    out = torch.zeros_like(cd)
    APIC.g2p(u32, out, sd, bins=bins, error_count=err)
    torch.cuda.synchronize()
    inv = torch.empty_like(perm.long())
    inv[perm.long()] = torch.arange(perm.numel(), device="cuda")
    a = acc.double().cpu().numpy() * 2.0 ** -BITS
    return (int(err.item()), rel_err(a[..., 0], gm_o), rel_err(a[..., 1:], gmu_o),
            rel_err(out[inv].double().cpu().numpy(), c_o))


@pytest.mark.parametrize("order", [1, 2, 3])
def test_single_particle_tiled(cuda, order):
    mesh = periodic_mesh(12, halo=0)
    x = np.array([[0.37, 0.912, 0.0413]])
    m = np.array([1.25])
    c = np.random.default_rng(800).standard_normal((1, 4, 3)) * 0.5
    m, c = m.astype(np.float32).astype(np.float64), c.astype(np.float32).astype(np.float64)
    err, e_m, e_mu, e_c = _step_vs_oracle(mesh, order, x, m, c, (4, 4, 4), 256)
    assert err == 0 and e_m <= 1e-5 and e_mu <= 1e-5 and e_c <= 1e-5


@pytest.mark.parametrize("order", [1, 2, 3])
def test_particles_on_faces_and_box_edges(cuda, order):
    """Positions exactly on cell faces (node-aligned and half-cell) and on the
    low face of the periodic box and just below its high face."""
    n = 16
    mesh = periodic_mesh(n, halo=0)
    h = 1.0 / n
    rng = np.random.default_rng(801)
    faces = np.array([k * h for k in range(n)] + [(k + 0.5) * h for k in range(n)])
    x = np.stack([rng.choice(faces, 3000), rng.choice(faces, 3000),
                  rng.uniform(0, 1, 3000)], axis=1)
    x[:50] = 0.0
    x[50:100] = np.nextafter(1.0, 0.0)
    m = rng.uniform(0.5, 1.5, x.shape[0]).astype(np.float32).astype(np.float64)
    c = (rng.standard_normal((x.shape[0], 4, 3)) * 0.3).astype(np.float32).astype(np.float64)
    err, e_m, e_mu, e_c = _step_vs_oracle(mesh, order, x, m, c, (4, 8, 8), 512)
    assert err == 0 and e_m <= 1e-5 and e_mu <= 1e-5 and e_c <= 1e-5


@pytest.mark.parametrize("tile,chunk", [((3, 5, 7), 64), ((1, 1, 1), 32), ((20, 20, 20), 4096),
                                        ((32, 32, 32), 1 << 20)])
def test_ragged_tiles_small_items_and_oversized_tiles(cuda, tile, chunk):
    """Tiles that do not divide the 20^3 mesh, one-bin tiles with 32-particle
    items, one tile for the whole mesh, and a tile whose node tile exceeds
    the shared memory of a CTA (the calls fall back to the plain kernels)."""
    mesh = periodic_mesh(20, halo=0)
    x, m, c = uniform_particles(mesh, 5, seed=802)
    m, c = m.astype(np.float32).astype(np.float64), c.astype(np.float32).astype(np.float64)
    err, e_m, e_mu, e_c = _step_vs_oracle(mesh, 2, x, m, c, tile, chunk)
    assert err == 0 and e_m <= 1e-5 and e_mu <= 1e-5 and e_c <= 1e-5
