"""APIC parity on the GPU through the C ABI.

- the reference's single-particle known answers (1e-11 absolute);
- many-particle FP64 plain form vs the oracle: normwise relative error
  <= 1e-12 per field (the slack covers the order of FP64 atomic adds);
- FP32 precision form (FP32 particle state, 64-bit fixed-point grid) vs the
  FP64 oracle: grid velocity relative error <= 1e-5 (normwise), particle
  fields <= 1e-5, and bit-identical results for a shuffled particle order.
"""

import numpy as np
import pytest
import torch

import oracle
from helpers import (COLLOCATED_APIC, STAGGERED_APIC_KIND, golden, poly_fill, reference_mesh,
                     staggered_box_apic, stencil_range)
from particles import clustered_particles, periodic_mesh, rel_err, uniform_particles
from picasso_b200 import (APIC, FieldLocation, FixedGrid, create_spline, grid_velocity)

pytestmark = pytest.mark.gpu

G = golden()
BOX = [-50.0, -50.0, -50.0, 50.0, 50.0, 50.0]
TOL_F64 = 1e-12
TOL_F32 = 1e-5


def _dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _fill_window(shape, dims, c, width=6):
    arr = np.zeros(tuple(shape) + (len(dims),))
    lo = [max(0, c[d] - width) for d in range(3)]
    hi = [min(shape[d], c[d] + width) for d in range(3)]
    full = poly_fill(hi, dims)
    arr[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = full[lo[0]:, lo[1]:, lo[2]:]
    return arr


@pytest.mark.parametrize("order", [1, 2, 3])
def test_golden_collocated(cuda, order):
    fx = G["apic"]["fixture"]
    ck = G["apic"]["checks"][str(order)]
    loc = COLLOCATED_APIC[order]
    mesh = reference_mesh(BOX)
    c = (fx["cx"], fx["cy"], fx["cz"])
    ext = mesh.extent(loc)
    u = _dev(_fill_window(ext, [0, 1, 2], c))
    x = _dev([[fx["px"], fx["py"], fx["pz"]]])
    m = _dev([fx["pm"]])
    cp = torch.zeros((1, 4, 3), dtype=torch.float64, device="cuda")
    sd = create_spline(loc, order, mesh, x)
    APIC.g2p(u, cp, sd)
    pu = ck["checkParticleVelocity"]
    h = cp.cpu().numpy()[0]
    np.testing.assert_allclose(h[0], pu["mathematica_u"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(h[1:].T, pu["mathematica_b"], rtol=0, atol=1e-11)
    gm = mesh.zeros(loc)
    gmu = mesh.zeros(loc, 3)
    APIC.p2g(m, cp, gm, gmu, sd)
    gm, gmu = gm.cpu().numpy(), gmu.cpu().numpy()
    mom = np.array(ck["checkGridMomentum"]["mathematica"])
    mass = np.array(ck["checkGridMass"]["mathematica"])
    nodes = [(i, j, k) for i in stencil_range(order, c[0]) for j in stencil_range(order, c[1])
             for k in stencil_range(order, c[2])]
    for n, (i, j, k) in enumerate(nodes):
        np.testing.assert_allclose(gmu[i, j, k], mom[n], rtol=0, atol=1e-11)
        assert abs(gm[i, j, k] - mass[n]) < 1e-11
    assert np.count_nonzero(gm) == len(nodes)


@pytest.mark.parametrize("order", [1, 2, 3])
def test_golden_staggered(cuda, order):
    fx = G["apic"]["fixture"]
    ck = G["apic"]["checks"][str(order)]
    c = (fx["cx"], fx["cy"], fx["cz"])
    for dim in range(3):
        mesh = reference_mesh(staggered_box_apic(STAGGERED_APIC_KIND[order], dim))
        loc = FieldLocation.Face(dim)
        ext = mesh.extent(loc)
        u = _dev(_fill_window(ext, [dim], c)[..., 0])
        x = _dev([[fx["px"], fx["py"], fx["pz"]]])
        m = _dev([fx["pm"]])
        sd = create_spline(loc, order, mesh, x)
        cp = torch.zeros((1, 4, 3), dtype=torch.float64, device="cuda")
        APIC.g2p(u, cp, sd)
        h = cp.cpu().numpy()[0]
        pu = ck["checkParticleVelocity"]
        assert abs(h[0, dim] - pu["mathematica_u"][dim]) < 1e-11
        np.testing.assert_allclose(h[1:, dim], pu["mathematica_b"][dim], rtol=0, atol=1e-11)
        gm = mesh.zeros(loc)
        gs = mesh.zeros(loc)
        APIC.p2g(m, cp, gm, gs, sd)
        gm, gs = gm.cpu().numpy(), gs.cpu().numpy()
        mom = np.array(ck["checkGridMomentum"]["mathematica"])
        mass = np.array(ck["checkGridMass"]["mathematica"])
        nodes = [(i, j, k) for i in stencil_range(order, c[0])
                 for j in stencil_range(order, c[1]) for k in stencil_range(order, c[2])]
        for n, (i, j, k) in enumerate(nodes):
            assert abs(gs[i, j, k] - mom[n][dim]) < 1e-11
            assert abs(gm[i, j, k] - mass[n]) < 1e-11


LOCS = [("node", FieldLocation.Node), ("cell", FieldLocation.Cell),
        ("face1", FieldLocation.Face(1)), ("edge2", FieldLocation.Edge(2))]


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("locname,loc", LOCS)
def test_fp64_plain_vs_oracle(cuda, order, locname, loc):
    mesh = periodic_mesh(12, halo=1)
    x, m, c = uniform_particles(mesh, 4, seed=11 + order)
    from picasso_b200.api import staggered_dim
    stag = staggered_dim(loc) >= 0
    ext = mesh.extent(loc)
    # oracle
    sdo = create_spline(loc, order, mesh, None).desc
    gm_o = np.zeros(ext)
    gmu_o = np.zeros(ext) if stag else np.zeros(ext + (3,))
    assert oracle.apic_p2g(sdo, x, m, c, gm_o, gmu_o) == 0
    # GPU
    xd = _dev(x)
    sd = create_spline(loc, order, mesh, xd)
    gm = mesh.zeros(loc)
    gmu = mesh.zeros(loc) if stag else mesh.zeros(loc, 3)
    APIC.p2g(_dev(m), _dev(c), gm, gmu, sd)
    assert rel_err(gm.cpu().numpy(), gm_o) <= TOL_F64
    assert rel_err(gmu.cpu().numpy(), gmu_o) <= TOL_F64
    # G2P from a random grid field
    rng = np.random.default_rng(7)
    u = rng.standard_normal(gmu_o.shape)
    c_o = np.zeros_like(c)
    assert oracle.apic_g2p(sdo, x, u, c_o) == 0
    c_g = torch.zeros_like(_dev(c))
    APIC.g2p(_dev(u), c_g, sd)
    assert rel_err(c_g.cpu().numpy(), c_o) <= TOL_F64


@pytest.mark.parametrize("ncomp", [1, 2])
def test_fp64_ncomp(cuda, ncomp):
    mesh = periodic_mesh(10, halo=0)
    x, m, c = uniform_particles(mesh, 3, seed=5, ncomp=ncomp)
    loc = FieldLocation.Node
    ext = mesh.extent(loc)
    sdo = create_spline(loc, 2, mesh, None).desc
    gm_o, gmu_o = np.zeros(ext), np.zeros(ext + (ncomp,))
    oracle.apic_p2g(sdo, x, m, c, gm_o, gmu_o)
    sd = create_spline(loc, 2, mesh, _dev(x))
    gm, gmu = mesh.zeros(loc), mesh.zeros(loc, ncomp)
    APIC.p2g(_dev(m), _dev(c), gm, gmu, sd)
    assert rel_err(gmu.cpu().numpy(), gmu_o) <= TOL_F64
    u = np.random.default_rng(3).standard_normal(gmu_o.shape)
    c_o = np.zeros_like(c)
    oracle.apic_g2p(sdo, x, u, c_o)
    c_g = torch.zeros_like(_dev(c))
    APIC.g2p(_dev(u), c_g, sd)
    assert rel_err(c_g.cpu().numpy(), c_o) <= TOL_F64


def _fp32_step(mesh, loc, order, x, m, c, bits=36):
    xd = _dev(x)
    sd = create_spline(loc, order, mesh, xd)
    gm = FixedGrid(torch.zeros(mesh.extent(loc), dtype=torch.int64, device="cuda"), bits)
    gmu = FixedGrid(torch.zeros(mesh.extent(loc) + (3,), dtype=torch.int64, device="cuda"), bits)
    APIC.p2g(_dev(m, torch.float32), _dev(c, torch.float32), gm, gmu, sd)
    u32 = torch.zeros(mesh.extent(loc) + (3,), dtype=torch.float32, device="cuda")
    u64 = torch.zeros(mesh.extent(loc) + (3,), dtype=torch.float64, device="cuda")
    grid_velocity(sd.desc.mesh, gm, gmu, u32, 1e-12, u64_i=u64)
    c32 = torch.zeros(c.shape, dtype=torch.float32, device="cuda")
    APIC.g2p(u32, c32, sd)
    return gm, gmu, u64, c32


@pytest.mark.parametrize("order", [2, 3])
@pytest.mark.parametrize("clustered", [False, True])
def test_fp32_form_error_and_determinism(cuda, order, clustered):
    mesh = periodic_mesh(16, halo=0)
    if clustered:
        x, m, c = clustered_particles(mesh, 16 ** 3 * 8, nblob=4, sigma_cells=2.0, frac=0.7,
                                      seed=21)
    else:
        x, m, c = uniform_particles(mesh, 8, seed=22)
    # the FP32 form reads FP32 masses / affine fields: feed the oracle the
    # same (rounded) values so that only the arithmetic differs
    m = m.astype(np.float32).astype(np.float64)
    c = c.astype(np.float32).astype(np.float64)
    loc = FieldLocation.Node
    ext = mesh.extent(loc)
    sdo = create_spline(loc, order, mesh, None).desc
    gm_o, gmu_o, gu_o = np.zeros(ext), np.zeros(ext + (3,)), np.zeros(ext + (3,))
    oracle.apic_p2g(sdo, x, m, c, gm_o, gmu_o)
    oracle.grid_velocity(sdo.mesh, gm_o, gmu_o, gu_o, 1e-12)
    c_o = np.zeros_like(c)
    oracle.apic_g2p(sdo, x, gu_o, c_o)

    gm, gmu, u64, c32 = _fp32_step(mesh, loc, order, x, m, c)
    assert rel_err(gm.to_float().cpu().numpy(), gm_o) <= TOL_F32
    assert rel_err(gmu.to_float().cpu().numpy(), gmu_o) <= TOL_F32
    assert rel_err(u64.cpu().numpy(), gu_o) <= TOL_F32
    assert rel_err(c32.cpu().numpy()[:, 0], c_o[:, 0]) <= TOL_F32
    assert rel_err(c32.cpu().numpy()[:, 1:], c_o[:, 1:]) <= TOL_F32

    # determinism: a shuffled particle order gives bit-identical grids
    perm = np.random.default_rng(99).permutation(x.shape[0])
    gm2, gmu2, u642, _ = _fp32_step(mesh, loc, order, x[perm], m[perm], c[perm])
    assert torch.equal(gm.raw, gm2.raw)
    assert torch.equal(gmu.raw, gmu2.raw)
    assert torch.equal(u64, u642)


def test_out_of_mesh_particles_are_counted(cuda):
    mesh = reference_mesh(BOX)
    loc = FieldLocation.Node
    x = _dev([[9.31, -8.28, -3.34], [-51.2, 0.0, 0.0], [49.9, 49.9, 51.9], [0.1, 0.2, 0.3]])
    m = _dev([1.0, 1.0, 1.0, 1.0])
    c = torch.zeros((4, 4, 3), dtype=torch.float64, device="cuda")
    c[:, 0, :] = 1.0
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    sd = create_spline(loc, 2, mesh, x)
    gm, gmu = mesh.zeros(loc), mesh.zeros(loc, 3)
    APIC.p2g(m, c, gm, gmu, sd, error_count=err)
    assert int(err.item()) == 2
    assert abs(float(gm.sum()) - 2.0) < 1e-12


def test_aosoa_layout_matches_soa(cuda):
    """Cabana AoSoA storage (vector length 16) gives the same result as SoA."""
    import ctypes as C
    from picasso_b200 import _abi
    from picasso_b200.api import grid_field
    mesh = periodic_mesh(8, halo=0)
    x, m, c = uniform_particles(mesh, 4, seed=3)
    n = x.shape[0]
    VL = 16
    ns = -(-n // VL)
    # one AoSoA with members x(3), m(1), c(4x3): 16 doubles per particle
    soa = np.zeros((ns, 16, VL))
    for p in range(n):
        s, a = divmod(p, VL)
        soa[s, 0:3, a] = x[p]
        soa[s, 3, a] = m[p]
        soa[s, 4:16, a] = c[p].ravel()
    buf = _dev(soa)
    base = buf.data_ptr()

    def member(off):
        f = _abi.ParticleField()
        f.data = base + 8 * off * VL
        f.dtype = _abi.F64
        f.vector_shift = 4
        f.tile_stride = 16 * VL
        f.comp_stride = VL
        return f

    loc = FieldLocation.Node
    sd = create_spline(loc, 2, mesh, _dev(x))
    gm_a, gmu_a = mesh.zeros(loc), mesh.zeros(loc, 3)
    ex = _abi.Exec()
    lib = _abi.load_library()
    st = lib.picasso_apic_p2g(C.byref(sd.desc), n, 3, member(0), member(3), member(4),
                              grid_field(gm_a), grid_field(gmu_a), C.byref(ex))
    assert st == 0
    gm_s, gmu_s = mesh.zeros(loc), mesh.zeros(loc, 3)
    APIC.p2g(_dev(m), _dev(c), gm_s, gmu_s, sd)
    torch.cuda.synchronize()
    assert rel_err(gm_a.cpu().numpy(), gm_s.cpu().numpy()) <= TOL_F64
    assert rel_err(gmu_a.cpu().numpy(), gmu_s.cpu().numpy()) <= TOL_F64
