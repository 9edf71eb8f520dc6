"""Native autotuner (picasso_autotune) through the C ABI: it returns one of
its candidate launch knobs, leaves the particles untouched, and the tiled
P2G with the chosen knobs gives the grid of the default knobs to FP32
rounding (a work item is summed in FP32 before its fixed-point flush, so the
tiling sets the rounding: normwise 1e-6) and the same bits when repeated."""

import numpy as np
import pytest
import torch

from particles import clustered_particles, periodic_mesh
from picasso_b200 import (APIC, FieldLocation, FixedGrid, cell_sort, create_spline,
                          permute_members, tune_tiled_step)

pytestmark = pytest.mark.gpu
N = 16
BITS = 36
TILES = {(4, 4, 4), (4, 4, 8), (4, 8, 8), (8, 8, 8)}


def _grids(ext):
    acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
    u = torch.zeros(ext + (3,), dtype=torch.float32, device="cuda")
    return acc, FixedGrid(acc[..., 0], BITS), FixedGrid(acc[..., 1:], BITS), u


def _p2g_grid(mesh, order, x, m, c, tile, chunk, lanes):
    sd0 = create_spline(FieldLocation.Node, order, mesh, x)
    _, perm, bins = cell_sort(sd0, tile, chunk=chunk, p2g_lanes=lanes)
    xs, ms, cs = permute_members(perm, x, m, c)
    sd = create_spline(FieldLocation.Node, order, mesh, xs)
    acc, gm, gmu, _ = _grids(mesh.extent(FieldLocation.Node))
    APIC.p2g(ms, cs, gm, gmu, sd, bins=bins)
    torch.cuda.synchronize()
    return acc


@pytest.mark.parametrize("order", [2, 3])
def test_autotune_choice_is_a_candidate_and_exact(cuda, order):
    mesh = periodic_mesh(N, halo=0)
    x, m, c = clustered_particles(mesh, N ** 3 * 4, nblob=3, sigma_cells=1.5, frac=0.6,
                                  seed=800 + order)
    xd = torch.as_tensor(x, device="cuda")
    md = torch.as_tensor(m, dtype=torch.float32, device="cuda")
    cd = torch.as_tensor(c, dtype=torch.float32, device="cuda").contiguous()
    x0, m0, c0 = xd.clone(), md.clone(), cd.clone()
    sd = create_spline(FieldLocation.Node, order, mesh, xd)
    _, gm, gmu, u = _grids(mesh.extent(FieldLocation.Node))
    r = tune_tiled_step(sd, md, cd, gm, gmu, u, trials=2)
    assert r["tile"] in TILES and r["chunk"] in (1024, 4096)
    assert r["p2g_lanes"] in ((4,) if order == 3 else (1, 2))
    assert r["step_ms"] > 0.0
    assert torch.equal(xd, x0) and torch.equal(md, m0) and torch.equal(cd, c0)
    ref = _p2g_grid(mesh, order, xd, md, cd, (4, 8, 8), 4096, 0).double()
    got = _p2g_grid(mesh, order, xd, md, cd, r["tile"], r["chunk"], r["p2g_lanes"])
    again = _p2g_grid(mesh, order, xd, md, cd, r["tile"], r["chunk"], r["p2g_lanes"])
    assert bool((ref != 0).any()) and torch.equal(got, again)
    for f in range(4):
        err = float((got[..., f].double() - ref[..., f]).abs().max() / ref[..., f].abs().max())
        assert err <= 1e-6, (f, err)
