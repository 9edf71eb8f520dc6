"""Fused G2P + position update (picasso_apic_g2p_advect) through the C ABI.

The fused call must give the same bits as picasso_apic_g2p followed by
picasso_advect on the same inputs: c_p from the G2P, x_p moved by dt times the
stored velocity and wrapped into the periodic box.  Covered: FP64 plain,
FP32 plain and FP32 tiled (sorted, with bins) paths, orders 1-3, a periodic
and a non-periodic mesh, and the refusal of staggered locations.
"""

import numpy as np
import pytest
import torch

from particles import clustered_particles, periodic_mesh, uniform_particles
from picasso_b200 import (APIC, FieldLocation, PicassoError, UniformMesh, advect, cell_sort,
                          create_spline, permute_members)

pytestmark = pytest.mark.gpu


def _state(mesh, loc, x, c, f32, seed):
    dt_ = torch.float32 if f32 else torch.float64
    ext = mesh.extent(loc)
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    u = torch.randn(ext + (3,), generator=g, device="cuda", dtype=torch.float64).to(dt_)
    xd = torch.as_tensor(np.ascontiguousarray(x), device="cuda")
    cd = torch.as_tensor(c, dtype=dt_, device="cuda").contiguous()
    return xd, cd, u


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("form", ["fp64", "fp32", "fp32_tiled"])
def test_fused_equals_g2p_then_advect(cuda, order, form):
    mesh = periodic_mesh(16, halo=0)
    loc = FieldLocation.Node
    x, m, c = clustered_particles(mesh, 16 ** 3 * 6, nblob=3, sigma_cells=1.5, frac=0.6,
                                  seed=400 + order)
    f32 = form != "fp64"
    xd, cd, u = _state(mesh, loc, x, c, f32, 401)
    bins = None
    md = torch.as_tensor(m, device="cuda", dtype=cd.dtype)
    if form == "fp32_tiled":
        sd0 = create_spline(loc, order, mesh, xd)
        _, perm, bins = cell_sort(sd0, (4, 8, 8), chunk=256)
        xd, md, cd = permute_members(perm, xd, md, cd)
    dt = 0.1 / 16 * 3.0  # large enough that many particles change cells and wrap
    # reference sequence
    x1, c1 = xd.clone(), cd.clone()
    sd1 = create_spline(loc, order, mesh, x1)
    APIC.g2p(u, c1, sd1, bins=bins)
    advect(sd1.desc.mesh, x1, c1, dt)
    # fused
    x2, c2 = xd.clone(), cd.clone()
    sd2 = create_spline(loc, order, mesh, x2)
    APIC.g2p_advect(u, c2, sd2, dt, bins=bins)
    torch.cuda.synchronize()
    assert torch.equal(c1, c2)
    assert torch.equal(x1, x2)
    assert not torch.equal(x2, xd)
    lo, hi = 0.0, 1.0
    assert float(x2.min()) >= lo and float(x2.max()) < hi


def test_fused_non_periodic_cell_mesh(cuda):
    mesh = UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1 / 12, periodic=(False, False, False),
                       halo_cell_width=2)
    loc = FieldLocation.Cell
    rng = np.random.default_rng(402)
    x = rng.uniform(0.1, 0.9, (12 ** 3 * 4, 3))
    c = rng.standard_normal((x.shape[0], 4, 3))
    xd, cd, u = _state(mesh, loc, x, c, False, 403)
    x1, c1, x2, c2 = xd.clone(), cd.clone(), xd.clone(), cd.clone()
    sd1, sd2 = create_spline(loc, 2, mesh, x1), create_spline(loc, 2, mesh, x2)
    APIC.g2p(u, c1, sd1)
    advect(sd1.desc.mesh, x1, c1, 0.01)
    APIC.g2p_advect(u, c2, sd2, 0.01)
    torch.cuda.synchronize()
    assert torch.equal(c1, c2) and torch.equal(x1, x2)


def test_fused_refuses_staggered(cuda):
    mesh = periodic_mesh(8, halo=0)
    x, m, c = uniform_particles(mesh, 2, seed=404)
    loc = FieldLocation.Face(1)
    xd, cd, u = _state(mesh, loc, x, c, False, 405)
    sd = create_spline(loc, 2, mesh, xd)
    with pytest.raises(PicassoError):
        APIC.g2p_advect(u[..., :1].contiguous(), cd, sd, 0.01)
