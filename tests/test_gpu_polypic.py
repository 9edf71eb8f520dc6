"""PolyPIC parity on the GPU through the C ABI: linear (8 modes) against the
reference's known answers and the oracle; quadratic (27 modes, no reference
implementation) against the oracle and the exact-recovery property."""

import numpy as np
import pytest
import torch

import oracle
from helpers import golden, poly_fill, reference_mesh, staggered_box_polypic, stencil_range
from particles import clustered_particles, periodic_mesh, rel_err, uniform_particles
from picasso_b200 import (FieldLocation, FixedGrid, PolyPIC, UniformMesh, cell_sort, create_spline,
                          permute_members)

pytestmark = pytest.mark.gpu

G = golden()
BOX = [-50.0, -50.0, -50.0, 50.0, 50.0, 50.0]


def _dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _window(shape, dims, c, width=5):
    arr = np.zeros(tuple(shape) + (len(dims),))
    hi = [min(shape[d], c[d] + width) for d in range(3)]
    lo = [c[d] - width for d in range(3)]
    full = poly_fill(hi, dims)
    arr[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = full[lo[0]:, lo[1]:, lo[2]:]
    return arr


def test_golden_linear_collocated(cuda):
    fx = G["polypic"]["fixture"]
    ck = G["polypic"]["checks"]["1"]
    mesh = reference_mesh(BOX)
    loc = FieldLocation.Node
    c = (fx["cx"], fx["cy"], fx["cz"])
    u = _dev(_window(mesh.extent(loc), [0, 1, 2], c))
    x = _dev([[fx["px"], fx["py"], fx["pz"]]])
    m = _dev([fx["pm"]])
    sd = create_spline(loc, 1, mesh, x)
    modes = torch.zeros((1, 8, 3), dtype=torch.float64, device="cuda")
    PolyPIC.g2p(u, modes, sd)
    np.testing.assert_allclose(modes.cpu().numpy()[0], ck["checkParticleVelocity"]["mathematica"],
                               rtol=0, atol=1e-11)
    gm, gmu = mesh.zeros(loc), mesh.zeros(loc, 3)
    PolyPIC.p2g(m, modes, modes, gmu, gm, fx["dt"], sd)
    gm, gmu = gm.cpu().numpy(), gmu.cpu().numpy()
    mom = np.array(ck["checkGridMomentum"]["mathematica"])
    mass = np.array(ck["checkGridMass"]["mathematica"])
    nodes = [(i, j, k) for i in stencil_range(1, c[0]) for j in stencil_range(1, c[1])
             for k in stencil_range(1, c[2])]
    for n, (i, j, k) in enumerate(nodes):
        np.testing.assert_allclose(gmu[i, j, k], mom[n], rtol=0, atol=1e-11)
        assert abs(gm[i, j, k] - mass[n]) < 1e-11


def test_golden_linear_staggered(cuda):
    fx = G["polypic"]["fixture"]
    ck = G["polypic"]["checks"]["1"]
    c = (fx["cx"], fx["cy"], fx["cz"])
    for dim in range(3):
        mesh = reference_mesh(staggered_box_polypic("edge", dim))
        loc = FieldLocation.Edge(dim)
        u = _dev(_window(mesh.extent(loc), [dim], c)[..., 0])
        x = _dev([[fx["px"], fx["py"], fx["pz"]]])
        m = _dev([fx["pm"]])
        sd = create_spline(loc, 1, mesh, x)
        modes = torch.zeros((1, 8, 3), dtype=torch.float64, device="cuda")
        PolyPIC.g2p(u, modes, sd)
        gold = np.array(ck["checkParticleVelocity"]["mathematica"])
        np.testing.assert_allclose(modes.cpu().numpy()[0][:, dim], gold[:, dim], rtol=0,
                                   atol=1e-11)
        modes = _dev(np.array(ck["setParticleVelocity"]["mathematica"])[None])
        gm, gs = mesh.zeros(loc), mesh.zeros(loc)
        PolyPIC.p2g(m, modes, modes, gs, gm, fx["dt"], sd)
        gm, gs = gm.cpu().numpy(), gs.cpu().numpy()
        mom = np.array(ck["checkGridMomentum"]["mathematica"])
        mass = np.array(ck["checkGridMass"]["mathematica"])
        nodes = [(i, j, k) for i in stencil_range(1, c[0]) for j in stencil_range(1, c[1])
                 for k in stencil_range(1, c[2])]
        for n, (i, j, k) in enumerate(nodes):
            assert abs(gs[i, j, k] - mom[n][dim]) < 1e-11
            assert abs(gm[i, j, k] - mass[n]) < 1e-11


def _modes(rng, n, nm, ncomp):
    u = np.empty((n, nm, ncomp))
    u[:, 0] = rng.standard_normal((n, ncomp))
    u[:, 1:] = 0.05 * rng.standard_normal((n, nm - 1, ncomp))
    return u


@pytest.mark.parametrize("order", [1, 2])
def test_fp64_vs_oracle(cuda, order):
    mesh = periodic_mesh(10, halo=1)
    x, m, _ = uniform_particles(mesh, 4, seed=31)
    nm = 8 if order == 1 else 27
    rng = np.random.default_rng(4)
    u = _modes(rng, x.shape[0], nm, 3)
    loc = FieldLocation.Node
    ext = mesh.extent(loc)
    dt = 0.1 * mesh.cell_size
    sdo = create_spline(loc, order, mesh, None).desc
    gm_o, gmu_o = np.zeros(ext), np.zeros(ext + (3,))
    oracle.polypic_p2g(sdo, x, m, u, u, gmu_o, gm_o, dt)
    sd = create_spline(loc, order, mesh, _dev(x))
    gm, gmu = mesh.zeros(loc), mesh.zeros(loc, 3)
    PolyPIC.p2g(_dev(m), _dev(u), _dev(u), gmu, gm, dt, sd)
    assert rel_err(gm.cpu().numpy(), gm_o) <= 1e-12
    assert rel_err(gmu.cpu().numpy(), gmu_o) <= 1e-12
    ug = np.random.default_rng(5).standard_normal(ext + (3,))
    c_o = np.zeros_like(u)
    oracle.polypic_g2p(sdo, x, ug, c_o)
    c_g = torch.zeros_like(_dev(u))
    PolyPIC.g2p(_dev(ug), c_g, sd)
    assert rel_err(c_g.cpu().numpy(), c_o) <= 1e-12


@pytest.mark.parametrize("order", [1, 2])
def test_fp32_form_per_mode_error(cuda, order):
    mesh = periodic_mesh(10, halo=0)
    x, m, _ = uniform_particles(mesh, 8, seed=41)
    nm = 8 if order == 1 else 27
    u = _modes(np.random.default_rng(8), x.shape[0], nm, 3).astype(np.float32).astype(np.float64)
    m = m.astype(np.float32).astype(np.float64)
    loc = FieldLocation.Node
    ext = mesh.extent(loc)
    dt = 0.1 * mesh.cell_size
    sdo = create_spline(loc, order, mesh, None).desc
    gm_o, gmu_o = np.zeros(ext), np.zeros(ext + (3,))
    oracle.polypic_p2g(sdo, x, m, u, u, gmu_o, gm_o, dt)
    sd = create_spline(loc, order, mesh, _dev(x))
    gm = FixedGrid(torch.zeros(ext, dtype=torch.int64, device="cuda"), 36)
    gmu = FixedGrid(torch.zeros(ext + (3,), dtype=torch.int64, device="cuda"), 36)
    u32 = _dev(u, torch.float32)
    PolyPIC.p2g(_dev(m, torch.float32), u32, u32, gmu, gm, dt, sd)
    assert rel_err(gm.to_float().cpu().numpy(), gm_o) <= 1e-5
    assert rel_err(gmu.to_float().cpu().numpy(), gmu_o) <= 1e-5
    ug = np.random.default_rng(6).standard_normal(ext + (3,)).astype(np.float32)
    c_o = np.zeros_like(u)
    oracle.polypic_g2p(sdo, x, ug.astype(np.float64), c_o)
    c32 = torch.zeros(u.shape, dtype=torch.float32, device="cuda")
    PolyPIC.g2p(_dev(ug, torch.float32), c32, sd)
    got = c32.cpu().numpy()
    for r in range(nm):  # per-mode error against the FP64 oracle
        assert rel_err(got[:, r], c_o[:, r]) <= 2e-5, r


@pytest.mark.parametrize("order", [1, 2])
def test_exact_recovery_single_particle(cuda, order):
    """With dt = 0 and one particle, P2G(G2P(u)) = m w_i u_i on the stencil:
    the 8 (27) modes span the 8 (27) stencil values."""
    mesh = periodic_mesh(8, halo=0)
    rng = np.random.default_rng(12)
    x = (np.array([[3.3, 4.71, 2.05]]) + 0.0) * mesh.cell_size
    ext = mesh.extent(FieldLocation.Node)
    ug = rng.standard_normal(ext + (3,))
    sd = create_spline(FieldLocation.Node, order, mesh, _dev(x))
    nm = 8 if order == 1 else 27
    modes = torch.zeros((1, nm, 3), dtype=torch.float64, device="cuda")
    PolyPIC.g2p(_dev(ug), modes, sd)
    gm, gmu = mesh.zeros(FieldLocation.Node), mesh.zeros(FieldLocation.Node, 3)
    PolyPIC.p2g(_dev([2.0]), modes, modes, gmu, gm, 0.0, sd)
    gm, gmu = gm.cpu().numpy(), gmu.cpu().numpy()
    sel = gm > 0
    np.testing.assert_allclose(gmu[sel], gm[sel][:, None] * ug[sel], rtol=1e-10, atol=1e-12)
    assert sel.sum() == (order + 1) ** 3


@pytest.mark.parametrize("order,layout,periodic", [(1, "packed", True), (2, "packed", True),
                                                   (2, "strided", True), (2, "packed", False)])
def test_tiled_fp32_form_equals_plain(cuda, order, layout, periodic):
    """Cell-sorted particles with bins take the tiled FP32 kernels: the grid
    (integer sums) and c_p must be the plain kernels' bits.  'strided': c_p
    rows are not packed (the G2P writes records directly)."""
    if periodic:
        mesh = periodic_mesh(12, halo=0)
        x, m, _ = clustered_particles(mesh, 12 ** 3 * 6, nblob=3, sigma_cells=1.5, frac=0.6,
                                      seed=50 + order)
    else:
        mesh = UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1 / 12, periodic=(False,) * 3,
                           halo_cell_width=2)
        x = np.random.default_rng(52).uniform(0.05, 0.95, (12 ** 3 * 6, 3))
        m = np.random.default_rng(53).uniform(0.5, 1.5, x.shape[0])
    nm = 8 if order == 1 else 27
    u = _modes(np.random.default_rng(9), x.shape[0], nm, 3)
    loc = FieldLocation.Node
    ext = mesh.extent(loc)
    dt = 0.1 * mesh.cell_size
    f32 = torch.float32
    xd, md, ud = _dev(x), _dev(m, f32), _dev(u, f32)
    sd0 = create_spline(loc, order, mesh, xd)
    _, perm, bins = cell_sort(sd0, (4, 4, 4), chunk=256)
    xs, ms, us = permute_members(perm, xd, md, ud)
    sd = create_spline(loc, order, mesh, xs)

    def p2g(b):
        gm = FixedGrid(torch.zeros(ext, dtype=torch.int64, device="cuda"), 36)
        gmu = FixedGrid(torch.zeros(ext + (3,), dtype=torch.int64, device="cuda"), 36)
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        PolyPIC.p2g(ms, us, us, gmu, gm, dt, sd, bins=b, error_count=err)
        torch.cuda.synchronize()
        return gm.raw, gmu.raw, int(err.item())

    gm_p, gmu_p, e_p = p2g(None)
    gm_t, gmu_t, e_t = p2g(bins)
    assert e_p == 0 and e_t == 0
    assert bool((gm_t != 0).any())
    assert torch.equal(gm_p, gm_t) and torch.equal(gmu_p, gmu_t)
    g = torch.Generator(device="cuda").manual_seed(54)
    ug = torch.randn(ext + (3,), generator=g, device="cuda", dtype=f32)

    def g2p(b):
        if layout == "packed":
            c = torch.full((x.shape[0], nm, 3), 7.0, dtype=f32, device="cuda")
        else:
            c = torch.full((x.shape[0], nm + 1, 3), 7.0, dtype=f32, device="cuda")[:, :nm, :]
        PolyPIC.g2p(ug, c, sd, bins=b)
        torch.cuda.synchronize()
        return c.clone()

    c_p, c_t = g2p(None), g2p(bins)
    assert not bool((c_t == 7.0).all())
    assert torch.equal(c_p, c_t)
