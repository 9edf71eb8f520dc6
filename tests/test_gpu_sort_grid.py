"""Cell sort (bit-exact permutation vs the oracle's stable counting sort),
permutation gather, grid velocity update, advection and batched 3x3
inverse on the GPU through the C ABI."""

import numpy as np
import pytest
import torch

import oracle
from particles import clustered_particles, periodic_mesh, rel_err, uniform_particles
from picasso_b200 import (FieldLocation, UniformMesh, advect, cell_sort, create_spline,
                          grid_velocity, mat3_inverse, permute)

pytestmark = pytest.mark.gpu


def _dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("tile", [(4, 4, 4), (8, 4, 2), (1, 1, 1)])
def test_cell_sort_matches_oracle(cuda, order, tile):
    mesh = periodic_mesh(16, halo=1)
    x, _, _ = clustered_particles(mesh, 16 ** 3 * 6, nblob=3, sigma_cells=1.5, frac=0.6,
                                  seed=order)
    sdo = create_spline(FieldLocation.Node, order, mesh, None).desc
    key_o, perm_o, off_o = oracle.cell_sort(sdo, x, tile)
    sd = create_spline(FieldLocation.Node, order, mesh, _dev(x))
    key, perm, bins = cell_sort(sd, tile)
    assert np.array_equal(key.cpu().numpy().view(np.uint32), key_o)
    assert np.array_equal(perm.cpu().numpy().view(np.uint32), perm_o)
    assert np.array_equal(bins.tile_offset.cpu().numpy(), off_o)


def test_cell_sort_non_periodic_out_of_mesh_last(cuda):
    mesh = UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1 / 8, periodic=(False, False, False),
                       halo_cell_width=1)
    rng = np.random.default_rng(5)
    x = rng.uniform(-0.3, 1.3, (5000, 3))
    sdo = create_spline(FieldLocation.Cell, 2, mesh, None).desc
    key_o, perm_o, off_o = oracle.cell_sort(sdo, x, (4, 4, 4))
    key, perm, bins = cell_sort(create_spline(FieldLocation.Cell, 2, mesh, _dev(x)), (4, 4, 4))
    assert np.array_equal(perm.cpu().numpy().view(np.uint32), perm_o)
    assert np.array_equal(bins.tile_offset.cpu().numpy(), off_o)
    assert off_o[-1] < x.shape[0]  # some particles are outside and sort last


def test_cell_sort_large_is_stable_and_sorted(cuda):
    """Size-independent properties at a larger size: keys ascending, the
    permutation is a bijection and ties keep the original order."""
    mesh = periodic_mesh(64, halo=0)
    x, _, _ = clustered_particles(mesh, 64 ** 3 * 8, nblob=32, sigma_cells=2.0, frac=0.7, seed=9)
    sd = create_spline(FieldLocation.Node, 2, mesh, _dev(x))
    key, perm, bins = cell_sort(sd, (8, 8, 8))
    k = key.to(torch.int64) & 0xFFFFFFFF
    p = perm.to(torch.int64) & 0xFFFFFFFF
    assert bool((k[1:] >= k[:-1]).all())
    same = k[1:] == k[:-1]
    assert bool((p[1:][same] > p[:-1][same]).all())
    assert torch.equal(torch.sort(p).values, torch.arange(x.shape[0], device="cuda"))


def test_permute(cuda):
    rng = np.random.default_rng(2)
    src = _dev(rng.standard_normal((1000, 4, 3)))
    perm = torch.as_tensor(rng.permutation(1000).astype(np.int32), device="cuda")
    dst = permute(perm, src)
    assert torch.equal(dst, src[perm.long()])
    s32 = src.float()
    assert torch.equal(permute(perm, s32), s32[perm.long()])
    # packed rows of 24 B (8-byte words), 4 B and 8 B scalars, and a strided
    # view (element-wise path)
    x = _dev(rng.standard_normal((1000, 3)))
    assert torch.equal(permute(perm, x), x[perm.long()])
    m32 = s32[:, 0, 0].contiguous()
    assert torch.equal(permute(perm, m32), m32[perm.long()])
    m64 = src[:, 0, 0].contiguous()
    assert torch.equal(permute(perm, m64), m64[perm.long()])
    strided = src[:, 1:3, :]
    assert torch.equal(permute(perm, strided), strided[perm.long()])


def test_grid_velocity_vs_oracle(cuda):
    mesh = periodic_mesh(12, halo=1)
    ext = mesh.extent(FieldLocation.Node)
    rng = np.random.default_rng(4)
    gm = rng.uniform(0, 2, ext)
    gm[rng.random(ext) < 0.2] = 0.0
    gmu = rng.standard_normal(ext + (3,))
    desc = mesh.descriptor(FieldLocation.Node)
    gu_o = np.zeros_like(gmu)
    oracle.grid_velocity(desc, gm, gmu, gu_o, 1e-12)
    gu = torch.zeros(ext + (3,), dtype=torch.float64, device="cuda")
    grid_velocity(desc, _dev(gm), _dev(gmu), gu, 1e-12)
    assert np.array_equal(gu.cpu().numpy(), gu_o)


def test_advect_vs_oracle(cuda):
    mesh = periodic_mesh(8, halo=0)
    x, _, c = uniform_particles(mesh, 2, seed=6)
    c[:, 0] *= 5.0
    desc = mesh.descriptor(FieldLocation.Node)
    xo = x.copy()
    v = np.ascontiguousarray(c[:, 0])
    oracle.advect(desc, xo, v, 0.02)
    xd = _dev(x)
    advect(desc, xd, _dev(c), 0.02)
    got = xd.cpu().numpy()
    assert np.array_equal(got, xo)
    assert got.min() >= 0.0 and got.max() < 1.0


def test_mat3_inverse(cuda):
    rng = np.random.default_rng(3923423)
    n = 1000
    a = rng.uniform(-1, 1, (n, 3, 3))
    x0 = rng.uniform(-1, 1, (n, 3))
    # the reference's kernel test builds op = 0.75 (A + 0.5 A^T) and solves
    # op x1 = op x0 (tstBatchedLinearAlgebra.hpp:1769-1789); here with the
    # cofactor inverse, same tolerance 1e-11
    op = 0.75 * (a + 0.5 * np.transpose(a, (0, 2, 1)))
    b = np.einsum("nij,nj->ni", op, x0)
    inv, det, y = mat3_inverse(_dev(op), _dev(b))
    inv_o, det_o, y_o = oracle.mat3_inverse(op, b)
    assert rel_err(det.cpu().numpy(), det_o) <= 1e-14
    assert rel_err(inv.cpu().numpy(), inv_o) <= 1e-12
    cond_ok = np.abs(det_o) > 1e-3
    np.testing.assert_allclose(y.cpu().numpy()[cond_ok], x0[cond_ok], rtol=0, atol=1e-11)


@pytest.mark.parametrize("kind", ["f64", "f32", "fixed"])
@pytest.mark.parametrize("value", [0.0, 1.25])
def test_grid_fill_contiguous_and_strided(cuda, kind, value):
    """Fill of a whole (nx, ny, nz, c) array (one contiguous range: memset or
    vector stores, odd element counts and an offset start included) and of a
    strided component view (element by element)."""
    from picasso_b200 import FixedGrid, grid_fill
    mesh = periodic_mesh(7, halo=1)
    desc = mesh.descriptor(FieldLocation.Node)
    ext = mesh.extent(FieldLocation.Node)
    dt = {"f64": torch.float64, "f32": torch.float32, "fixed": torch.int64}[kind]
    raw = torch.full((1,) + ext + (3,), 7, dtype=dt, device="cuda")
    whole = raw[0] if kind != "fixed" else FixedGrid(raw[0], 20)
    grid_fill(desc, whole, value, ncomp=3)
    part = torch.full(ext + (3,), 7, dtype=dt, device="cuda")
    comp = part[..., 1] if kind != "fixed" else FixedGrid(part[..., 1], 20)
    grid_fill(desc, comp, value, ncomp=1)
    torch.cuda.synchronize()
    expect = value if kind != "fixed" else int(round(value * 2 ** 20))
    assert bool((raw == expect).all())
    assert bool((part[..., 1] == expect).all())
    assert bool((part[..., 0] == 7).all()) and bool((part[..., 2] == 7).all())
    # an odd-sized contiguous range that starts off a 16-byte boundary
    buf = torch.full((1 + 5 * 5 * 5 * 1,), 7, dtype=dt, device="cuda")
    small = UniformMesh([0, 0, 0, 1, 1, 1], cell_size=0.2, periodic=(True,) * 3)
    view = buf[1:].view(5, 5, 5)
    grid_fill(small.descriptor(FieldLocation.Node),
              view if kind != "fixed" else FixedGrid(view, 20), value, ncomp=1)
    torch.cuda.synchronize()
    assert int(buf[0]) == 7 and bool((buf[1:] == expect).all())


@pytest.mark.parametrize("storage", ["f64", "fixed"])
@pytest.mark.parametrize("walls", [None, (("no_slip", "free_slip"), ("free_slip", "none"),
                                          ("none", "no_slip"))])
def test_grid_update_vs_oracle(cuda, storage, walls):
    """Field solve u = (mu + dt f) / m + dt g (m > 1e-12) with wall conditions
    on a non-periodic Node mesh, against the oracle: bit-identical FP64."""
    from picasso_b200 import FixedGrid, grid_update
    mesh = UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1 / 10, periodic=(False, True, False),
                       halo_cell_width=2)
    loc = FieldLocation.Node
    ext = mesh.extent(loc)
    rng = np.random.default_rng(700)
    m = rng.uniform(0.0, 2.0, ext)
    m[rng.random(ext) < 0.2] = 0.0  # empty nodes
    mu = rng.standard_normal(ext + (3,))
    f = rng.standard_normal(ext + (3,))
    bits = 30
    if storage == "fixed":  # values representable in the fixed-point format
        m = np.round(m * 2 ** bits) / 2 ** bits
        mu = np.round(mu * 2 ** bits) / 2 ** bits
    dt, g = 0.01, (0.0, -9.81, 0.5)
    code = {"none": 0, "no_slip": 1, "free_slip": 2}
    wcodes = [[code[w] for w in pair] for pair in walls] if walls else None
    desc = mesh.descriptor(loc)
    u_o = np.full(ext + (3,), 5.0)  # entries outside the owned box stay as they were
    oracle.grid_update(desc, m, mu, u_o, dt, g, f_i=f, thr=1e-12, walls=wcodes, width=2)
    if storage == "fixed":
        gm = FixedGrid(torch.as_tensor(np.round(m * 2 ** bits).astype(np.int64), device="cuda"),
                       bits)
        gmu = FixedGrid(torch.as_tensor(np.round(mu * 2 ** bits).astype(np.int64),
                                        device="cuda"), bits)
    else:
        gm, gmu = torch.as_tensor(m, device="cuda"), torch.as_tensor(mu, device="cuda")
    u = torch.full(ext + (3,), 5.0, dtype=torch.float64, device="cuda")
    u32 = torch.full(ext + (3,), 5.0, dtype=torch.float32, device="cuda")
    grid_update(desc, gm, gmu, u32, dt, g, f_i=torch.as_tensor(f, device="cuda"),
                walls=walls, wall_width=2, u64_i=u)
    torch.cuda.synchronize()
    assert np.array_equal(u.cpu().numpy(), u_o)
    assert np.array_equal(u32.cpu().numpy(), u_o.astype(np.float32))
    if walls:
        un = u.cpu().numpy()
        own_y = slice(2, 12)  # y is periodic: its ghost entries are not written
        assert (un[:3, own_y] == 0).all()            # x low: no-slip (width 2 + ghosts)
        assert (un[-3:, own_y, :, 0] == 0).all()     # x high: free-slip, normal component
