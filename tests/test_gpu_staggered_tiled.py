"""Tiled (cell-sorted, shared-memory) FP32-form APIC transfers on staggered
locations (Face<D>, Edge<D>: APIC.hpp:148-232 P2G, :477-544 G2P).

The grid fields of a staggered location are the mass and the one velocity
component of the entity's dimension (scalar arrays); the particles are
sorted with the staggered spline.  Checked: P2G (mass, momentum) and G2P
(c_p, whose other columns are zero) against the FP64 oracle, normwise
relative <= 1e-5 as every FP32-form tiled test; against the plain fixed-point
kernel on the same particles; and the record path bit-identical to the
position path.
"""

import numpy as np
import pytest
import torch

import oracle
from particles import clustered_particles, periodic_mesh, rel_err, uniform_particles
from picasso_b200 import (APIC, FieldLocation, FixedGrid, cell_sort, create_spline,
                          permute_members, spline_records)

pytestmark = pytest.mark.gpu
TOL = 1e-5
BITS = 36
LOCS = [("face0", FieldLocation.Face(0)), ("face1", FieldLocation.Face(1)),
        ("face2", FieldLocation.Face(2)), ("edge1", FieldLocation.Edge(1))]


def _dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _gpu(mesh, loc, order, x, m, c, u, tiled, lanes=0, records=False):
    """Staggered P2G into fixed-point scalar grids and G2P from u (FP32):
    tiled on sorted particles, or the plain kernel; results in input order."""
    xd = _dev(x)
    md, cd = _dev(m, torch.float32), _dev(c, torch.float32)
    sd = create_spline(loc, order, mesh, xd)
    bins, perm = None, None
    if tiled:
        _, perm, bins = cell_sort(sd, (4, 4, 8), chunk=512, p2g_lanes=lanes)
        xd, md, cd = permute_members(perm, xd, md, cd)
        sd = create_spline(loc, order, mesh, xd)
        if records:
            spline_records(sd, bins)
    ext = mesh.extent(loc)
    gm = FixedGrid(torch.zeros(ext, dtype=torch.int64, device="cuda"), BITS)
    gmu = FixedGrid(torch.zeros(ext, dtype=torch.int64, device="cuda"), BITS)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    APIC.p2g(md, cd, gm, gmu, sd, bins=bins, error_count=err)
    cg = torch.full_like(cd, 5.0)  # every entry is written
    APIC.g2p(_dev(u, torch.float32), cg, sd, bins=bins, error_count=err)
    torch.cuda.synchronize()
    if tiled:
        back = torch.empty_like(cg)
        back[perm.long()] = cg
        cg = back
    return gm.to_float().cpu().numpy(), gmu.to_float().cpu().numpy(), cg, int(err.item())


CASES = [(1, 1), (1, 2), (2, 1), (2, 2), (3, 4)]


@pytest.mark.parametrize("order,lanes", CASES)
@pytest.mark.parametrize("locname,loc", LOCS)
def test_tiled_staggered_vs_oracle_and_plain(cuda, order, lanes, locname, loc):
    mesh = periodic_mesh(16, halo=1)
    if locname.startswith("face"):
        x, m, c = uniform_particles(mesh, 6, seed=20 + order)
    else:
        x, m, c = clustered_particles(mesh, 16 ** 3 * 6, nblob=3, sigma_cells=1.5, frac=0.7,
                                      seed=30 + order)
    ext = mesh.extent(loc)
    sdo = create_spline(loc, order, mesh, None).desc
    gm_o, gmu_o = np.zeros(ext), np.zeros(ext)
    assert oracle.apic_p2g(sdo, x, m, c, gm_o, gmu_o) == 0
    u = np.random.default_rng(order).standard_normal(ext)
    u32 = u.astype(np.float32).astype(np.float64)  # the grid the GPU reads
    c_o = np.zeros_like(c)
    assert oracle.apic_g2p(sdo, x, u32, c_o) == 0
    gm, gmu, cg, e = _gpu(mesh, loc, order, x, m, c, u, tiled=True, lanes=lanes)
    assert e == 0
    assert rel_err(gm, gm_o) <= TOL
    assert rel_err(gmu, gmu_o) <= TOL
    cgn = cg.double().cpu().numpy()
    assert rel_err(cgn, c_o) <= TOL
    # the other columns of c_p are written as zero, as the plain kernel does
    from picasso_b200.api import staggered_dim
    dim = staggered_dim(loc)
    others = [d for d in range(3) if d != dim]
    assert np.abs(cgn[:, :, others]).max() == 0.0
    pm, pmu, pc, pe = _gpu(mesh, loc, order, x, m, c, u, tiled=False)
    assert pe == 0
    assert rel_err(gmu, pmu) <= TOL and rel_err(gm, pm) <= TOL
    assert rel_err(cgn, pc.double().cpu().numpy()) <= TOL


@pytest.mark.parametrize("order,lanes", CASES)
def test_tiled_staggered_records_bit_identical(cuda, order, lanes):
    mesh = periodic_mesh(16, halo=0)
    loc = FieldLocation.Face(2)
    x, m, c = clustered_particles(mesh, 16 ** 3 * 6, nblob=3, sigma_cells=1.5, frac=0.7,
                                  seed=40 + order)
    u = np.random.default_rng(9).standard_normal(mesh.extent(loc))
    a = _gpu(mesh, loc, order, x, m, c, u, tiled=True, lanes=lanes, records=False)
    b = _gpu(mesh, loc, order, x, m, c, u, tiled=True, lanes=lanes, records=True)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert torch.equal(a[2], b[2])
