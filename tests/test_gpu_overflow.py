"""Fixed-point range checks of the precision form (picasso_exec.overflow_count).

A 64-bit fixed-point grid with b fraction bits holds node values up to
2^(63-b) in magnitude.  P2G counts every contribution (plain kernels) or tile
sum (tiled kernels) whose magnitude times 2^b reaches 2^62, and the grid
velocity / update passes count nodes whose fixed-point mass -- a sum of
non-negative contributions -- has wrapped negative.  With the benchmark's 36
bits the range is +-1.3e8 per node and nothing is counted; with 60 or 61 bits
and unit masses it overflows and the counters say so.
"""

import numpy as np
import pytest
import torch

from particles import periodic_mesh, uniform_particles
from picasso_b200 import (APIC, FieldLocation, FixedGrid, cell_sort, create_spline, grid_update,
                          grid_velocity, permute_members)

pytestmark = pytest.mark.gpu


def _p2g(bits, mass_scale, ppc, tiled, c_scale=1.0):
    mesh = periodic_mesh(12, halo=0)
    x, m, c = uniform_particles(mesh, ppc, seed=91, jitter_mass=False)
    c = c * c_scale
    xd = torch.as_tensor(x, device="cuda")
    md = torch.as_tensor(m * mass_scale, dtype=torch.float32, device="cuda")
    cd = torch.as_tensor(c, dtype=torch.float32, device="cuda").contiguous()
    sd = create_spline(FieldLocation.Node, 2, mesh, xd)
    bins = None
    if tiled:
        _, perm, bins = cell_sort(sd, (4, 4, 4), chunk=256)
        xd, md, cd = permute_members(perm, xd, md, cd)
        sd = create_spline(FieldLocation.Node, 2, mesh, xd)
    ext = mesh.extent(FieldLocation.Node)
    acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
    gm, gmu = FixedGrid(acc[..., 0], bits), FixedGrid(acc[..., 1:], bits)
    ovf = torch.zeros(1, dtype=torch.int32, device="cuda")
    APIC.p2g(md, cd, gm, gmu, sd, bins=bins, overflow_count=ovf)
    torch.cuda.synchronize()
    return mesh, gm, gmu, int(ovf.item())


@pytest.mark.parametrize("tiled", [False, True])
def test_in_range_grid_counts_nothing(cuda, tiled):
    mesh, gm, gmu, n = _p2g(36, 1.0, 8, tiled)
    assert n == 0
    u = torch.zeros(mesh.extent(FieldLocation.Node) + (3,), dtype=torch.float32, device="cuda")
    ovf = torch.zeros(1, dtype=torch.int32, device="cuda")
    grid_velocity(mesh.descriptor(FieldLocation.Node), gm, gmu, u, 1e-12, overflow_count=ovf)
    torch.cuda.synchronize()
    assert int(ovf.item()) == 0


@pytest.mark.parametrize("tiled", [False, True])
def test_contributions_beyond_range_are_counted(cuda, tiled):
    # masses of 100 with 60 fraction bits: w m 2^60 >= 2^62 for w m >= 4
    _, _, _, n = _p2g(60, 100.0, 4, tiled)
    assert n > 0


@pytest.mark.parametrize("update", [False, True])
def test_wrapped_mass_sums_are_counted(cuda, update):
    # unit masses and small velocities, 61 bits: every contribution is in
    # range (|value| < 2: w <= 0.42, momenta scaled down), but a node's mass
    # (about 6 at 6 particles per cell) is above 2^(63-61) = 4, so its 64-bit
    # sum wraps negative
    mesh, gm, gmu, n = _p2g(61, 1.0, 6, tiled=False, c_scale=0.01)
    assert n == 0
    assert int((gm.raw < 0).sum().item()) > 0
    desc = mesh.descriptor(FieldLocation.Node)
    u = torch.zeros(mesh.extent(FieldLocation.Node) + (3,), dtype=torch.float32, device="cuda")
    ovf = torch.zeros(1, dtype=torch.int32, device="cuda")
    if update:
        grid_update(desc, gm, gmu, u, 1e-3, overflow_count=ovf)
    else:
        grid_velocity(desc, gm, gmu, u, 1e-12, overflow_count=ovf)
    torch.cuda.synchronize()
    assert int(ovf.item()) == int((gm.raw < 0).sum().item())
    # without a counter the passes run as before
    grid_velocity(desc, gm, gmu, u, 1e-12)
    torch.cuda.synchronize()
    assert np.isfinite(u.cpu().numpy()).all()
