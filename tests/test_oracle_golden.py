"""Pin the oracle against the reference's known-answer tests.

tstAPIC.hpp / tstPolyPIC.hpp hold Mathematica values for one particle
(m = 0.134 at (9.31, -8.28, -3.34)) on the [-50, 50]^3, dx = 0.5, halo-2 mesh
with a polynomial grid field: g2p particle velocity / affine matrix / modes,
and p2g (of the g2p result) grid momentum and mass.  Tolerance 1e-11
absolute, as in the reference (tstAPIC.hpp:540, tstPolyPIC.hpp:196).
"""

import numpy as np
import pytest

import oracle
from helpers import (COLLOCATED_APIC, STAGGERED_APIC_KIND, golden, poly_fill, reference_mesh,
                     staggered_box_apic, staggered_box_polypic, stencil_range)
from picasso_b200 import FieldLocation, create_spline

EPS = 1e-11
BOX = [-50.0, -50.0, -50.0, 50.0, 50.0, 50.0]
G = golden()


def _particle(fx):
    return np.array([[fx["px"], fx["py"], fx["pz"]]]), np.array([fx["pm"]])


def _window_fill(shape, dims, c, width=6):
    """Polynomial values on a window around the particle cell, zero
    elsewhere (only the stencil entities are read)."""
    arr = np.zeros(tuple(shape) + (len(dims),))
    lo = [max(0, c[d] - width) for d in range(3)]
    hi = [min(shape[d], c[d] + width) for d in range(3)]
    full = poly_fill(hi, dims)
    arr[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = full[lo[0]:, lo[1]:, lo[2]:]
    return arr


def _idx(order, c):
    return [(i, j, k) for i in stencil_range(order, c[0]) for j in stencil_range(order, c[1])
            for k in stencil_range(order, c[2])]


@pytest.mark.parametrize("order", [1, 2, 3])
def test_apic_collocated_golden(order):
    fx = G["apic"]["fixture"]
    ck = G["apic"]["checks"][str(order)]
    loc = COLLOCATED_APIC[order]
    mesh = reference_mesh(BOX)
    sd = create_spline(loc, order, mesh, None).desc
    c = (fx["cx"], fx["cy"], fx["cz"])
    ext = mesh.extent(loc)
    u = _window_fill(ext, [0, 1, 2], c)
    nodes = _idx(order, c)
    # grid values (checkGridVelocity)
    gv = np.array(ck["checkGridVelocity"]["mathematica"])
    for n, (i, j, k) in enumerate(nodes):
        np.testing.assert_allclose(u[i, j, k], gv[n], rtol=0, atol=EPS)
    x, m = _particle(fx)
    cp = np.zeros((1, 4, 3))
    assert oracle.apic_g2p(sd, x, u, cp) == 0
    pu = ck["checkParticleVelocity"]
    for dim in range(3):
        assert abs(cp[0, 0, dim] - pu["mathematica_u"][dim]) < EPS
        for a in range(3):
            assert abs(cp[0, 1 + a, dim] - pu["mathematica_b"][dim][a]) < EPS
    gm = np.zeros(ext)
    gmu = np.zeros(ext + (3,))
    assert oracle.apic_p2g(sd, x, m, cp, gm, gmu) == 0
    mom = np.array(ck["checkGridMomentum"]["mathematica"])
    mass = np.array(ck["checkGridMass"]["mathematica"])
    for n, (i, j, k) in enumerate(nodes):
        np.testing.assert_allclose(gmu[i, j, k], mom[n], rtol=0, atol=EPS)
        assert abs(gm[i, j, k] - mass[n]) < EPS
    # nothing outside the stencil
    assert np.count_nonzero(gm) == len(nodes)


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("dim", [0, 1, 2])
def test_apic_staggered_golden(order, dim):
    fx = G["apic"]["fixture"]
    ck = G["apic"]["checks"][str(order)]
    mesh = reference_mesh(staggered_box_apic(STAGGERED_APIC_KIND[order], dim))
    loc = FieldLocation.Face(dim)  # the reference test always uses Face<Dim>
    sd = create_spline(loc, order, mesh, None).desc
    c = (fx["cx"], fx["cy"], fx["cz"])
    ext = mesh.extent(loc)
    u = _window_fill(ext, [dim], c)[..., 0]
    nodes = _idx(order, c)
    gv = np.array(ck["checkGridVelocity"]["mathematica"])
    for n, (i, j, k) in enumerate(nodes):
        assert abs(u[i, j, k] - gv[n][dim]) < EPS
    x, m = _particle(fx)
    cp = np.zeros((1, 4, 3))
    assert oracle.apic_g2p(sd, x, u, cp) == 0
    pu = ck["checkParticleVelocity"]
    assert abs(cp[0, 0, dim] - pu["mathematica_u"][dim]) < EPS
    for a in range(3):
        assert abs(cp[0, 1 + a, dim] - pu["mathematica_b"][dim][a]) < EPS
    gm = np.zeros(ext)
    gs = np.zeros(ext)
    assert oracle.apic_p2g(sd, x, m, cp, gm, gs) == 0
    mom = np.array(ck["checkGridMomentum"]["mathematica"])
    mass = np.array(ck["checkGridMass"]["mathematica"])
    for n, (i, j, k) in enumerate(nodes):
        assert abs(gs[i, j, k] - mom[n][dim]) < EPS
        assert abs(gm[i, j, k] - mass[n]) < EPS


def test_polypic_linear_collocated_golden():
    fx = G["polypic"]["fixture"]
    ck = G["polypic"]["checks"]["1"]
    mesh = reference_mesh(BOX)
    loc = FieldLocation.Node
    sd = create_spline(loc, 1, mesh, None).desc
    c = (fx["cx"], fx["cy"], fx["cz"])
    ext = mesh.extent(loc)
    u = _window_fill(ext, [0, 1, 2], c)
    x, m = _particle(fx)
    modes = np.zeros((1, 8, 3))
    assert oracle.polypic_g2p(sd, x, u, modes) == 0
    gold = np.array(ck["checkParticleVelocity"]["mathematica"])
    np.testing.assert_allclose(modes[0], gold, rtol=0, atol=EPS)
    gm = np.zeros(ext)
    gmu = np.zeros(ext + (3,))
    assert oracle.polypic_p2g(sd, x, m, modes, modes, gmu, gm, fx["dt"]) == 0
    mom = np.array(ck["checkGridMomentum"]["mathematica"])
    mass = np.array(ck["checkGridMass"]["mathematica"])
    for n, (i, j, k) in enumerate(_idx(1, c)):
        np.testing.assert_allclose(gmu[i, j, k], mom[n], rtol=0, atol=EPS)
        assert abs(gm[i, j, k] - mass[n]) < EPS


@pytest.mark.parametrize("dim", [0, 1, 2])
def test_polypic_linear_staggered_golden(dim):
    fx = G["polypic"]["fixture"]
    ck = G["polypic"]["checks"]["1"]
    mesh = reference_mesh(staggered_box_polypic("edge", dim))
    loc = FieldLocation.Edge(dim)
    sd = create_spline(loc, 1, mesh, None).desc
    c = (fx["cx"], fx["cy"], fx["cz"])
    ext = mesh.extent(loc)
    u = _window_fill(ext, [dim], c)[..., 0]
    x, m = _particle(fx)
    modes = np.zeros((1, 8, 3))
    assert oracle.polypic_g2p(sd, x, u, modes) == 0
    gold = np.array(ck["checkParticleVelocity"]["mathematica"])
    np.testing.assert_allclose(modes[0, :, dim], gold[:, dim], rtol=0, atol=EPS)
    # the other columns are untouched by the staggered g2p (PolyPIC.hpp:328)
    assert np.all(np.delete(modes[0], dim, axis=1) == 0.0)
    modes = np.array(ck["setParticleVelocity"]["mathematica"])[None].copy()
    gm = np.zeros(ext)
    gs = np.zeros(ext)
    assert oracle.polypic_p2g(sd, x, m, modes, modes, gs, gm, fx["dt"]) == 0
    mom = np.array(ck["checkGridMomentum"]["mathematica"])
    mass = np.array(ck["checkGridMass"]["mathematica"])
    for n, (i, j, k) in enumerate(_idx(1, c)):
        assert abs(gs[i, j, k] - mom[n][dim]) < EPS
        assert abs(gm[i, j, k] - mass[n]) < EPS
