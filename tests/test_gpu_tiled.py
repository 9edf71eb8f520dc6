"""Tiled (cell-sorted, shared-memory) FP32-form APIC kernels through the C
ABI: error against the FP64 oracle (normwise relative <= 1e-5 for grid and
particle fields), bit-reproducibility, and safety when the particles passed
with bins are not actually sorted."""

import numpy as np
import pytest
import torch

import oracle
from particles import clustered_particles, periodic_mesh, rel_err, uniform_particles
from picasso_b200 import (APIC, FieldLocation, FixedGrid, UniformMesh, cell_sort, create_spline,
                          grid_velocity, permute_members)

pytestmark = pytest.mark.gpu
TOL = 1e-5
BITS = 36


def _dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _oracle_step(mesh, loc, order, x, m, c):
    ext = mesh.extent(loc)
    sdo = create_spline(loc, order, mesh, None).desc
    gm, gmu, gu = np.zeros(ext), np.zeros(ext + (3,)), np.zeros(ext + (3,))
    oracle.apic_p2g(sdo, x, m, c, gm, gmu)
    oracle.grid_velocity(sdo.mesh, gm, gmu, gu, 1e-12)
    co = np.zeros_like(c)
    oracle.apic_g2p(sdo, x, gu, co)
    return gm, gmu, gu, co


def _gpu_step(mesh, loc, order, x, m, c, tile, sort=True, lanes=0):
    xd = _dev(x)
    md, cd = _dev(m, torch.float32), _dev(c, torch.float32)
    sd = create_spline(loc, order, mesh, xd)
    key, perm, bins = cell_sort(sd, tile, p2g_lanes=lanes)
    if sort:
        xd, md, cd = permute_members(perm, xd, md, cd)
        sd = create_spline(loc, order, mesh, xd)
    ext = mesh.extent(loc)
    acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
    gm, gmu = FixedGrid(acc[..., 0], BITS), FixedGrid(acc[..., 1:], BITS)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    APIC.p2g(md, cd, gm, gmu, sd, bins=bins, error_count=err)
    u32 = torch.zeros(ext + (3,), dtype=torch.float32, device="cuda")
    u64 = torch.zeros(ext + (3,), dtype=torch.float64, device="cuda")
    grid_velocity(sd.desc.mesh, gm, gmu, u32, 1e-12, u64_i=u64)
    c_out = torch.zeros_like(cd)
    APIC.g2p(u32, c_out, sd, bins=bins, error_count=err)
    torch.cuda.synchronize()
    inv = torch.empty_like(perm.long())
    inv[perm.long()] = torch.arange(perm.numel(), device="cuda")
    c_out = c_out[inv] if sort else c_out  # back to the input order
    return acc, u64, c_out, int(err.item())


# (particles, order, bins per tile, P2G lanes per particle; 0 = default)
CASES = [
    ("uniform", 2, (8, 8, 8), 0),
    ("clustered", 2, (8, 8, 8), 0),
    ("clustered", 2, (4, 8, 16), 0),
    ("uniform", 2, (8, 8, 8), 2),
    ("clustered", 2, (4, 8, 8), 4),
    ("uniform", 1, (8, 8, 8), 0),
    ("clustered", 1, (4, 8, 8), 2),
    ("uniform", 1, (4, 4, 8), 4),
    ("clustered", 3, (8, 8, 8), 0),
    ("uniform", 3, (4, 8, 8), 4),
]


@pytest.mark.parametrize("kind,order,tile,lanes", CASES)
def test_tiled_vs_oracle(cuda, kind, order, tile, lanes):
    mesh = periodic_mesh(24, halo=0)
    if kind == "uniform":
        x, m, c = uniform_particles(mesh, 8, seed=51)
    else:
        x, m, c = clustered_particles(mesh, 24 ** 3 * 8, nblob=6, sigma_cells=2.0, frac=0.7,
                                      seed=52)
    m = m.astype(np.float32).astype(np.float64)
    c = c.astype(np.float32).astype(np.float64)
    loc = FieldLocation.Node
    gm_o, gmu_o, gu_o, c_o = _oracle_step(mesh, loc, order, x, m, c)
    acc, u64, c_g, nerr = _gpu_step(mesh, loc, order, x, m, c, tile, lanes=lanes)
    assert nerr == 0
    a = acc.double().cpu().numpy() * 2.0 ** -BITS
    assert rel_err(a[..., 0], gm_o) <= TOL
    assert rel_err(a[..., 1:], gmu_o) <= TOL
    assert rel_err(u64.cpu().numpy(), gu_o) <= TOL
    cg = c_g.double().cpu().numpy()
    assert rel_err(cg[:, 0], c_o[:, 0]) <= TOL
    assert rel_err(cg[:, 1:], c_o[:, 1:]) <= TOL


@pytest.mark.parametrize("order,lanes", [(2, 1), (2, 4), (3, 4)])
def test_tiled_is_bit_reproducible(cuda, order, lanes):
    mesh = periodic_mesh(32, halo=0)
    x, m, c = clustered_particles(mesh, 32 ** 3 * 8, nblob=8, sigma_cells=2.0, frac=0.7, seed=53)
    runs = [_gpu_step(mesh, FieldLocation.Node, order, x, m, c, (8, 8, 8), lanes=lanes)
            for _ in range(3)]
    for r in runs[1:]:
        assert torch.equal(r[0], runs[0][0])
        assert torch.equal(r[1], runs[0][1])
        assert torch.equal(r[2], runs[0][2])


def test_tiled_non_periodic_cell_mesh(cuda):
    mesh = UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1 / 20, periodic=(False, False, False),
                       halo_cell_width=2)
    rng = np.random.default_rng(54)
    x = rng.uniform(0.0, 1.0, (20 ** 3 * 6, 3))
    m = rng.uniform(0.5, 1.5, x.shape[0]).astype(np.float32).astype(np.float64)
    c = (0.3 * rng.standard_normal((x.shape[0], 4, 3))).astype(np.float32).astype(np.float64)
    loc = FieldLocation.Cell
    gm_o, gmu_o, gu_o, c_o = _oracle_step(mesh, loc, 2, x, m, c)
    acc, u64, c_g, nerr = _gpu_step(mesh, loc, 2, x, m, c, (8, 8, 8))
    assert nerr == 0
    a = acc.double().cpu().numpy() * 2.0 ** -BITS
    assert rel_err(a[..., 0], gm_o) <= TOL
    assert rel_err(a[..., 1:], gmu_o) <= TOL
    assert rel_err(c_g.double().cpu().numpy(), c_o) <= TOL


def test_unsorted_particles_with_bins_are_flagged(cuda):
    """Passing bins for particles that were not permuted must not touch
    memory outside the tiles: mismatching particles are skipped and
    counted."""
    mesh = periodic_mesh(16, halo=0)
    x, m, c = uniform_particles(mesh, 4, seed=55)
    _, _, _, nerr = _gpu_step(mesh, FieldLocation.Node, 2, x, m, c, (8, 8, 8), sort=False)
    assert nerr > 0


@pytest.mark.parametrize("order,lanes", [(3, 1), (3, 2), (2, 3)])
def test_unsupported_p2g_lanes_are_refused(cuda, order, lanes):
    from picasso_b200._abi import ERR_INVALID_ARGUMENT, PicassoError
    mesh = periodic_mesh(16, halo=0)
    x, m, c = uniform_particles(mesh, 2, seed=56)
    with pytest.raises(PicassoError) as e:
        _gpu_step(mesh, FieldLocation.Node, order, x, m, c, (8, 8, 8), lanes=lanes)
    assert e.value.status == ERR_INVALID_ARGUMENT
