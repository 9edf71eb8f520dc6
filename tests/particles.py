"""Seeded synthetic particle sets for the tests (numpy, host side)."""

import numpy as np

from picasso_b200 import UniformMesh


def periodic_mesh(n, halo=0, cell=None):
    """Periodic n^3 mesh on [0, 1)^3 (cell size 1/n) with a given halo."""
    cs = cell if cell is not None else 1.0 / n
    box = [0.0, 0.0, 0.0, n * cs, n * cs, n * cs]
    return UniformMesh(box, cell_size=cs, periodic=(True, True, True), halo_cell_width=halo)


def uniform_particles(mesh, ppc, seed, ncomp=3, affine_sigma=0.1, jitter_mass=True):
    """ppc particles uniformly placed in every owned cell; v ~ N(0,1),
    m ~ U[0.5, 1.5], affine rows ~ N(0, affine_sigma)."""
    rng = np.random.default_rng(seed)
    n = mesh.global_num_cell
    cs = mesh.cell_size
    lo = mesh.global_low_corner
    ii, jj, kk = np.meshgrid(np.arange(n[0]), np.arange(n[1]), np.arange(n[2]), indexing="ij")
    cells = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1)
    cells = np.repeat(cells, ppc, axis=0)
    x = (cells + rng.random(cells.shape)) * cs + np.array(lo)
    npart = x.shape[0]
    m = rng.uniform(0.5, 1.5, npart) if jitter_mass else np.ones(npart)
    c = np.empty((npart, 4, ncomp))
    c[:, 0, :] = rng.standard_normal((npart, ncomp))
    c[:, 1:, :] = affine_sigma * rng.standard_normal((npart, 3, ncomp))
    return np.ascontiguousarray(x), m, c


def clustered_particles(mesh, npart, nblob, sigma_cells, frac, seed, ncomp=3):
    """frac of the particles in nblob Gaussian blobs (sigma in cells, centres
    uniform), the rest uniform; positions wrapped into the periodic box."""
    rng = np.random.default_rng(seed)
    n = np.array(mesh.global_num_cell)
    cs = mesh.cell_size
    lo = np.array(mesh.global_low_corner)
    L = n * cs
    nb = int(npart * frac)
    centres = lo + rng.random((nblob, 3)) * L
    which = rng.integers(0, nblob, nb)
    xb = centres[which] + rng.standard_normal((nb, 3)) * sigma_cells * cs
    xu = lo + rng.random((npart - nb, 3)) * L
    x = np.concatenate([xb, xu])
    x = lo + np.mod(x - lo, L)
    x = np.where(x >= lo + L, lo, x)
    m = rng.uniform(0.5, 1.5, npart)
    c = np.empty((npart, 4, ncomp))
    c[:, 0, :] = rng.standard_normal((npart, ncomp))
    c[:, 1:, :] = 0.1 * rng.standard_normal((npart, 3, ncomp))
    return np.ascontiguousarray(x), m, c


def rel_err(a, b):
    """Normwise relative error max|a - b| / max|b|."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))


def node_rel_err(a, b, mask=None):
    """Largest per-entry relative error: for every entry (grid node or
    particle, leading axes) the max-norm of a - b over its components divided
    by the max-norm of b, over the entries selected by `mask` (e.g. nodes
    with mass above the velocity threshold) whose b is not zero."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.ndim == b.ndim and mask is not None and a.ndim > np.asarray(mask).ndim:
        axes = tuple(range(np.asarray(mask).ndim, a.ndim))
    else:
        axes = tuple(range(1, a.ndim)) if mask is None else ()
    num = np.max(np.abs(a - b), axis=axes) if axes else np.abs(a - b)
    den = np.max(np.abs(b), axis=axes) if axes else np.abs(b)
    sel = den > 0
    if mask is not None:
        sel &= np.asarray(mask, dtype=bool)
    return float(np.max(num[sel] / den[sel])) if np.any(sel) else 0.0
