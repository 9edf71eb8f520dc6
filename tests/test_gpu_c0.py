"""The CPU-runnable benchmark configuration at full size against the oracle:
64^3 periodic grid, dx = 1/64, 8 particles per cell uniform in each cell
(2,097,152 particles), v ~ N(0, 1), m ~ U[0.5, 1.5], C ~ N(0, 0.1),
quadratic B-spline on nodes; one P2G (mass, momentum), grid velocity
v = p / m where m > 1e-12, one G2P.

Two error measures for every field, both stated in the assertions:
  * normwise:  max |a - b| / max |b| over the whole field;
  * per entry: for every grid node with m > 1e-12 (or every particle), the
    max-norm of a - b over its components divided by the max-norm of b.
FP64 plain form (unsorted particles, FP64 atomics): <= 1e-12 in both
measures (only the order of the atomic additions differs; the reference's
own known-answer tolerance is 1e-11, tstAPIC.hpp:540).  FP32 precision form,
every field <= 1e-5 normwise, and per node:
  * plain fixed-point kernel (each FP32 contribution rounded to fixed point
    and summed exactly): grid velocity <= 1e-5 per node (measured 5.6e-6);
  * tiled kernels on cell-sorted particles: each lane sums a bin's
    contributions in FP32 registers before they reach the exact integer
    grid.  At the nodes where the affine contributions (about 25 times the
    velocity at dx = 1/64) cancel to a small velocity, that FP32 partial sum
    sets the error: worst node 1.5e-5 (measured; an FP64 node tile changes
    it only to 1.2e-5, so the register sums dominate).  Asserted: <= 2e-5 at
    every node, and above 1e-5 at no more than 1e-4 of the nodes.
"""

import os

import numpy as np
import pytest
import torch

import oracle
from particles import node_rel_err, rel_err
from picasso_b200 import (APIC, FieldLocation, FixedGrid, UniformMesh, cell_sort, create_spline,
                          grid_velocity, permute_members, workloads)

pytestmark = pytest.mark.gpu
N = 64
PPC = 8
BITS = 36
THR = 1e-12


@pytest.fixture(scope="module")
def c0():
    mesh = UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1.0 / N, periodic=(True, True, True))
    x = workloads.positions("uniform", N, PPC, seed=1000)
    m, c = workloads.particle_state(x.shape[0], seed=1000)
    xh, mh, ch = x.cpu().numpy(), m.cpu().numpy(), np.ascontiguousarray(c.cpu().numpy())
    sdo = create_spline(FieldLocation.Node, 2, mesh, None).desc
    co = ch.copy()
    gm, gmu, gu = oracle.apic_step_omp(sdo, xh, mh, co, os.cpu_count() or 1, THR)
    return {"mesh": mesh, "x": x, "m": m, "c": c, "gm": gm, "gmu": gmu, "gu": gu, "c_out": co}


def _check(name, got, ref, tol, mask=None):
    nw = rel_err(got, ref)
    pe = node_rel_err(got, ref, mask)
    print("%s: normwise %.3e, per entry %.3e" % (name, nw, pe))
    return nw, pe


def test_c0_fp64_plain_vs_oracle(cuda, c0):
    mesh = c0["mesh"]
    loc = FieldLocation.Node
    sd = create_spline(loc, 2, mesh, c0["x"])
    gm, gmu, gu = mesh.zeros(loc), mesh.zeros(loc, 3), mesh.zeros(loc, 3)
    APIC.p2g(c0["m"], c0["c"], gm, gmu, sd)
    grid_velocity(sd.desc.mesh, gm, gmu, gu, THR)
    cg = torch.zeros_like(c0["c"])
    APIC.g2p(gu, cg, sd)
    torch.cuda.synchronize()
    heavy = c0["gm"] > THR
    tol = 1e-12
    for name, got, ref, mask in (("grid mass", gm, c0["gm"], heavy),
                                 ("grid momentum", gmu, c0["gmu"], heavy),
                                 ("grid velocity", gu, c0["gu"], heavy),
                                 ("particle c_p", cg, c0["c_out"], None)):
        nw, pe = _check(name, got.cpu().numpy(), ref, tol, mask)
        assert nw <= tol, (name, nw)
        assert pe <= tol, (name, pe)


@pytest.mark.parametrize("tiled", [False, True])
def test_c0_fp32_form_vs_oracle(cuda, c0, tiled):
    mesh = c0["mesh"]
    loc = FieldLocation.Node
    x, m, c = c0["x"], c0["m"].float(), c0["c"].float().contiguous()
    sd = create_spline(loc, 2, mesh, x)
    bins, perm = None, None
    if tiled:
        _, perm, bins = cell_sort(sd, (4, 8, 8), chunk=4096)
        x, m, c = permute_members(perm, x, m, c)
        sd = create_spline(loc, 2, mesh, x)
    ext = mesh.extent(loc)
    acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
    gm, gmu = FixedGrid(acc[..., 0], BITS), FixedGrid(acc[..., 1:], BITS)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ovf = torch.zeros(1, dtype=torch.int32, device="cuda")
    APIC.p2g(m, c, gm, gmu, sd, bins=bins, error_count=err, overflow_count=ovf)
    u = torch.zeros(ext + (3,), dtype=torch.float32, device="cuda")
    grid_velocity(sd.desc.mesh, gm, gmu, u, THR, overflow_count=ovf)
    cg = torch.zeros_like(c)
    APIC.g2p(u, cg, sd, bins=bins, error_count=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0 and int(ovf.item()) == 0
    if tiled:  # back to the generation order of the oracle's particles
        back = torch.empty_like(cg)
        back[perm.long()] = cg
        cg = back
    heavy = c0["gm"] > THR
    tol = 1e-5
    ug = u.cpu().numpy()
    nw, pe = _check("fp32 grid velocity", ug, c0["gu"], tol, heavy)
    assert nw <= tol, nw
    if not tiled:
        assert pe <= tol, pe
    else:
        assert pe <= 2 * tol, pe
        num = np.abs(ug - c0["gu"]).max(axis=-1)
        den = np.abs(c0["gu"]).max(axis=-1)
        sel = heavy & (den > 0)
        above = int(np.count_nonzero(num[sel] / den[sel] > tol))
        print("fp32 tiled: %d of %d nodes above %.0e per node" % (above, int(sel.sum()), tol))
        assert above <= 1e-4 * sel.sum(), above
    for name, got, ref in (("fp32 grid mass", gm.to_float().cpu().numpy(), c0["gm"]),
                           ("fp32 grid momentum", gmu.to_float().cpu().numpy(), c0["gmu"]),
                           ("fp32 particle velocity", cg[:, 0].cpu().numpy(), c0["c_out"][:, 0]),
                           ("fp32 particle affine", cg[:, 1:].cpu().numpy(), c0["c_out"][:, 1:])):
        nw, _ = _check(name, got, ref, tol)
        assert nw <= tol, (name, nw)
