"""Shared fixtures of the tests: the reference's single-particle test mesh
(unit_test/inputs/polypic_test.json with the [-50, 50]^3 box), its
polynomial grid fill, the golden vectors, and synthetic particle sets."""

import json
import os

import numpy as np

from picasso_b200 import FieldLocation, UniformMesh

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "apic_polypic_golden.json")


def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def reference_mesh(box):
    """UniformMesh of the reference's transfer tests: cell_size 0.5,
    non-periodic, halo_cell_width 2, minimum halo 0 (tstAPIC.hpp:543-552)."""
    g = golden()
    mi = g["mesh_input"]
    return UniformMesh(box, cell_size=mi["cell_size"], periodic=mi["periodic"],
                       halo_cell_width=mi["halo_cell_width"], minimum_halo_cell_width=0)


def poly_fill(shape, dims):
    """The reference test grid values (tstAPIC.hpp:577-589) on indices
    (i, j, k) for each component value d+1 in dims: returns an array of
    shape + (len(dims),)."""
    i = np.arange(shape[0], dtype=np.int64)[:, None, None] - 2
    j = np.arange(shape[1], dtype=np.int64)[None, :, None] - 2
    k = np.arange(shape[2], dtype=np.int64)[None, None, :] - 2
    out = np.empty(tuple(shape) + (len(dims),))
    for n, d in enumerate(dims):
        dd = d + 1
        out[..., n] = (1e-10 * dd * (i.astype(np.float64) ** 5)
                       - 1.2e-9 * ((dd + j * i).astype(np.float64) ** 3)
                       + 1e-10 * ((i * j * k).astype(np.float64) ** 2)
                       + float(dd * dd))
    return out


def stencil_range(order, c):
    lo = c if order == 1 else c - 1
    hi = c + 2 if order in (1, 2) else c + 3
    return range(lo, hi)


def staggered_box_apic(location_kind, dim):
    """Box shift of tstAPIC.hpp:698-716 (Edge: other dims -0.25; Face: dim
    +0.25)."""
    box = [-50.0, -50.0, -50.0, 50.0, 50.0, 50.0]
    if location_kind == "edge":
        for d in range(3):
            if d != dim:
                box[d] -= 0.25
                box[d + 3] -= 0.25
    else:
        box[dim] += 0.25
        box[dim + 3] += 0.25
    return box


def staggered_box_polypic(location_kind, dim):
    """Box shift of tstPolyPIC.hpp:363-381 (Face: other dims -0.25; Edge:
    dim -0.25)."""
    box = [-50.0, -50.0, -50.0, 50.0, 50.0, 50.0]
    if location_kind == "face":
        for d in range(3):
            if d != dim:
                box[d] -= 0.25
                box[d + 3] -= 0.25
    else:
        box[dim] -= 0.25
        box[dim + 3] -= 0.25
    return box


COLLOCATED_APIC = {1: FieldLocation.Node, 2: FieldLocation.Cell, 3: FieldLocation.Node}
STAGGERED_APIC_KIND = {1: "edge", 2: "face", 3: "edge"}


def splitmix64(x):
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    return z ^ (z >> np.uint64(31))
