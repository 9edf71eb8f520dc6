"""G2P + advection that emits the next sort's keys, and the sort that starts
from them (picasso_apic_g2p_advect_keys, picasso_cell_sort_keys).

* The emitted key of every particle equals the oracle's key of its new
  position (the oracle's stable counting sort of the moved positions, read
  back through its permutation): bit-exact.
* cell_sort from the emitted keys gives the same sorted keys, permutation,
  tile offsets and work items as cell_sort from the moved positions.
* Positions and c_p are the bits picasso_apic_g2p_advect gives.
Covered: FP32 tiled (sorted, with bins) and FP64 plain paths, orders 1-3, a
periodic mesh with a key tile different from the bins' tile, and a
non-periodic mesh where particles leave the mesh (key = num_tiles x tile
volume, sorted last).
"""

import numpy as np
import pytest
import torch

import oracle
from particles import clustered_particles, periodic_mesh
from picasso_b200 import (APIC, FieldLocation, PicassoError, UniformMesh, cell_sort,
                          create_spline, permute_members)

pytestmark = pytest.mark.gpu


def _u(mesh, loc, f32, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    u = torch.randn(mesh.extent(loc) + (3,), generator=g, device="cuda", dtype=torch.float64)
    return u.float() if f32 else u


def _oracle_keys(sd, x, tile):
    """Per-particle keys of the oracle's sort (in the particles' order)."""
    skey, sperm, off = oracle.cell_sort(sd.desc, x, tile)
    keys = np.empty(x.shape[0], dtype=np.uint32)
    keys[sperm.astype(np.int64)] = skey
    return keys, skey, sperm, off


def _check(sd_new, keys, tile, chunk):
    """keys vs the oracle, and the sort from keys vs the sort from positions."""
    x_new = sd_new.x.cpu().numpy()
    k_ref, skey, sperm, off = _oracle_keys(sd_new, x_new, tile)
    got = keys.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, k_ref)
    a_key, a_perm, a_bins = cell_sort(sd_new, tile, chunk=chunk)
    b_key, b_perm, b_bins = cell_sort(sd_new, tile, chunk=chunk, keys=keys)
    torch.cuda.synchronize()
    assert torch.equal(a_key, b_key) and torch.equal(a_perm, b_perm)
    assert torch.equal(a_bins.tile_offset, b_bins.tile_offset)
    assert torch.equal(a_bins.tile_items, b_bins.tile_items)
    assert np.array_equal(b_key.cpu().numpy().view(np.uint32), skey)
    assert np.array_equal(b_perm.cpu().numpy().view(np.uint32), sperm)
    assert np.array_equal(b_bins.tile_offset.cpu().numpy(), off)
    return skey


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("form", ["fp64", "fp32_tiled"])
def test_emitted_keys_feed_the_next_sort(cuda, order, form):
    mesh = periodic_mesh(16, halo=0)
    loc = FieldLocation.Node
    x, m, c = clustered_particles(mesh, 16 ** 3 * 6, nblob=3, sigma_cells=1.5, frac=0.6,
                                  seed=700 + order)
    f32 = form != "fp64"
    dtype = torch.float32 if f32 else torch.float64
    xd = torch.as_tensor(x, device="cuda")
    md = torch.as_tensor(m, device="cuda", dtype=dtype)
    cd = torch.as_tensor(c, device="cuda", dtype=dtype).contiguous()
    u = _u(mesh, loc, f32, 701)
    bins = None
    if f32:
        sd0 = create_spline(loc, order, mesh, xd)
        _, perm, bins = cell_sort(sd0, (4, 8, 8), chunk=256)
        xd, md, cd = permute_members(perm, xd, md, cd)
    dt = 0.1 / 16 * 3.0  # many particles change cells and wrap
    x1, c1, x2, c2 = xd.clone(), cd.clone(), xd.clone(), cd.clone()
    sd1, sd2 = create_spline(loc, order, mesh, x1), create_spline(loc, order, mesh, x2)
    APIC.g2p_advect(u, c1, sd1, dt, bins=bins)
    key_tile = (2, 4, 8)  # the next sort may use another tile shape
    keys = APIC.g2p_advect(u, c2, sd2, dt, bins=bins, key_tile=key_tile)
    torch.cuda.synchronize()
    assert torch.equal(x1, x2) and torch.equal(c1, c2)
    _check(sd2, keys, key_tile, 512)


def test_keys_outside_a_non_periodic_mesh_sort_last(cuda):
    mesh = UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1 / 12, periodic=(False, False, False),
                       halo_cell_width=2)
    loc = FieldLocation.Node
    rng = np.random.default_rng(702)
    x = rng.uniform(0.02, 0.98, (12 ** 3 * 4, 3))
    c = rng.standard_normal((x.shape[0], 4, 3))
    xd = torch.as_tensor(x, device="cuda")
    cd = torch.as_tensor(c, device="cuda").contiguous()
    u = _u(mesh, loc, False, 703) * 40.0  # dt * u reaches past the ghosts for some
    sd = create_spline(loc, 2, mesh, xd)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    keys = APIC.g2p_advect(u, cd, sd, 0.01, key_tile=(4, 4, 4), error_count=err)
    torch.cuda.synchronize()
    skey = _check(sd, keys, (4, 4, 4), 64)
    ext = mesh.extent(loc)
    nt = 1
    for d in range(3):
        nt *= -(-ext[d] // 4)
    outside = int((skey == nt * 64).sum())
    assert outside > 0 and bool((skey[-outside:] == nt * 64).all())


def test_keys_argument_checks(cuda):
    mesh = periodic_mesh(8, halo=0)
    x = torch.rand(64, 3, dtype=torch.float64, device="cuda")
    c = torch.zeros(64, 4, 3, dtype=torch.float64, device="cuda")
    u = torch.zeros(mesh.extent(FieldLocation.Node) + (3,), dtype=torch.float64, device="cuda")
    sd = create_spline(FieldLocation.Node, 2, mesh, x)
    with pytest.raises(PicassoError):
        APIC.g2p_advect(u, c, sd, 0.1, key_tile=(0, 4, 4))
    keys = APIC.g2p_advect(u, c, sd, 0.1, key_tile=(4, 4, 4))
    with pytest.raises(ValueError):
        cell_sort(sd, (4, 4, 4), keys=keys.long())
