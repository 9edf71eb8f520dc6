"""Pin the quadratic (27-mode) PolyPIC of the oracle to the reference's 2-D
derivation, doc/polypic/polypic_2d_quadratic.nb.

The reference has no 3-D quadratic PolyPIC; its notebook derives the 2-D one
for a particle at offset (px, py) from the centre node of its 3 x 3 stencil
(nodes at -h, 0, h), mass m:
  * weights M = diag(m N2(px/h, i) N2(py/h, j)) with N2(x, 1) = (1/2 - x)^2/2,
    N2(x, 2) = 3/4 - x^2, N2(x, 3) = (x + 1/2)^2/2;
  * distances r = node - particle;
  * modes, in the notebook's column order after its permutation
    {1, 2, 4, 5, 3, 7, 6, 8, 9}: 1, r_x, r_y, r_x r_y, s2x, s2y, s2x r_y,
    s2y r_x, s2x s2y, with the shifted quadratic s2 = r^2 - h^2/4 -
    p (h^2 - 4 p^2) / h^2 r;
  * B^T M B (its printed output: diagonal, entries below), the P2G map M B
    and the G2P projection (B^T M B)^-1 B^T M.
The oracle defines the 3-D form as the tensor product of those per-dimension
modes.  With only the 9 modes of z-degree 0 populated, P2G (dt = 0) summed
over the stencil's z-nodes is the notebook's M B c, and G2P of a grid that
does not vary along z is the notebook's projection on those 9 modes (the
other 18 modes come out zero).  Everything is restated here from the
notebook's formulas; tolerance 1e-12 relative.
"""

import numpy as np
import pytest

import oracle
from picasso_b200 import FieldLocation, UniformMesh, create_spline

H = 0.5
# the notebook's 9 modes as (x-degree, y-degree), in its column order, and
# the oracle's index of the 3-D mode with those degrees and z-degree 0
NB_DEGREES = [(0, 0), (1, 0), (0, 1), (1, 1), (2, 0), (0, 2), (2, 1), (1, 2), (2, 2)]
ORACLE_MODE = {(0, 0): 0, (1, 0): 1, (0, 1): 2, (1, 1): 4, (2, 0): 18, (0, 2): 10,
               (2, 1): 21, (1, 2): 15, (2, 2): 24}


def n2(x, i):
    return {1: 0.5 * (0.5 - x) ** 2, 2: 0.75 - x * x, 3: 0.5 * (x + 0.5) ** 2}[i]


def notebook(px, py, m, h=H):
    """M, B (9 nodes x 9 modes) of polypic_2d_quadratic.nb; node id
    3 (i1 - 1) + (j1 - 1) for i1, j1 in 1..3, at ((i1 - 2) h, (j1 - 2) h)."""
    r = np.zeros((9, 2))
    w = np.zeros(9)
    for i1 in (1, 2, 3):
        for j1 in (1, 2, 3):
            idx = 3 * (i1 - 1) + (j1 - 1)
            r[idx] = ((i1 - 2) * h - px, (j1 - 2) * h - py)
            w[idx] = m * n2(px / h, i1) * n2(py / h, j1)
    M = np.diag(w)
    # monomials r_x^(i1-1) r_y^(j1-1) in column (j1 - 1) 3 + (i1 - 1), then
    # the notebook's permutation
    Bm = np.zeros((9, 9))
    for i1 in (1, 2, 3):
        for j1 in (1, 2, 3):
            Bm[:, (j1 - 1) * 3 + (i1 - 1)] = r[:, 0] ** (i1 - 1) * r[:, 1] ** (j1 - 1)
    B = Bm[:, [0, 1, 3, 4, 2, 6, 5, 7, 8]].copy()
    B[:, 4] = B[:, 4] - h * h / 4 - px * (h * h - 4 * px * px) / (h * h) * B[:, 1]
    B[:, 5] = B[:, 5] - h * h / 4 - py * (h * h - 4 * py * py) / (h * h) * B[:, 2]
    B[:, 6] = B[:, 4] * B[:, 2]
    B[:, 7] = B[:, 5] * B[:, 1]
    B[:, 8] = B[:, 4] * B[:, 5]
    return M, B


def btmb_diagonal(px, py, m, h=H):
    """The notebook's printed B^T M B diagonal."""
    ax = (h * h - 4 * px * px) ** 2 * (3 * h * h - 4 * px * px)
    ay = (h * h - 4 * py * py) ** 2 * (3 * h * h - 4 * py * py)
    return m * np.array([1.0, h * h / 4, h * h / 4, h ** 4 / 16, ax / (16 * h * h),
                         ay / (16 * h * h), ax / 64, ay / 64, ax * ay / (256 * h ** 4)])


# particle offsets from the centre node (in [-h/2, h/2)) and masses
INSIDE = [(0.1, -0.2, 1.3), (-0.24, 0.05, 0.7), (0.0, 0.0, 1.0), (0.2499, -0.2499, 0.134)]
# on a cell face (px = -h/2) the quadratic x-modes have zero weight: B^T M B
# is singular there and the notebook's projection is the 0/0 limit, which
# the oracle evaluates in closed form; the face is checked where defined
SAMPLES = INSIDE + [(-0.25, 0.17, 2.0)]


@pytest.mark.parametrize("px,py,m", SAMPLES)
def test_notebook_modes_are_weight_orthogonal(px, py, m):
    M, B = notebook(px, py, m)
    btmb = B.T @ M @ B
    d = btmb_diagonal(px, py, m)
    scale = np.abs(btmb).max()
    np.testing.assert_allclose(np.diag(btmb), d, rtol=1e-12, atol=1e-14 * scale)
    off = btmb - np.diag(np.diag(btmb))
    assert np.abs(off).max() <= 1e-12 * scale


def _mesh():
    # non-periodic box with cell size h and two ghost layers; the particle
    # sits near node (8, 8, 8)
    return UniformMesh([0.0, 0.0, 0.0, 8.0, 8.0, 8.0], cell_size=H, halo_cell_width=2)


def _particle(mesh, px, py, pz):
    node = np.array([8, 8, 8])
    lo = np.array(mesh.low_corner)
    return (lo + node * H + np.array([px, py, pz]))[None, :], node


@pytest.mark.parametrize("px,py,m", SAMPLES)
def test_oracle_p2g_reduces_to_notebook(px, py, m):
    mesh = _mesh()
    loc = FieldLocation.Node
    sd = create_spline(loc, 2, mesh, None).desc
    x, node = _particle(mesh, px, py, 0.13)
    rng = np.random.default_rng(int(1000 * (px + 2 * py + 3)))
    c2 = rng.standard_normal((9, 3))
    c = np.zeros((1, 27, 3))
    for col, deg in enumerate(NB_DEGREES):
        c[0, ORACLE_MODE[deg]] = c2[col]
    ext = mesh.extent(loc)
    mu = np.zeros(ext + (3,))
    mi = np.zeros(ext)
    # dt = 0: the backtracked distance is the distance itself
    assert oracle.polypic_p2g(sd, x, np.array([m]), c.copy(), c.copy(), mu, mi, 0.0) == 0
    M, B = notebook(px, py, m)
    want = M @ B @ c2  # (9 nodes, 3)
    got = np.zeros((9, 3))
    got_m = np.zeros(9)
    for i1 in (1, 2, 3):
        for j1 in (1, 2, 3):
            i, j = node[0] + i1 - 2, node[1] + j1 - 2
            got[3 * (i1 - 1) + (j1 - 1)] = mu[i, j, node[2] - 1:node[2] + 2].sum(axis=0)
            got_m[3 * (i1 - 1) + (j1 - 1)] = mi[i, j, node[2] - 1:node[2] + 2].sum()
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
    np.testing.assert_allclose(got_m, np.diag(M), rtol=1e-12, atol=1e-12 * np.diag(M).max())


@pytest.mark.parametrize("px,py,m", INSIDE)
def test_oracle_g2p_reduces_to_notebook(px, py, m):
    mesh = _mesh()
    loc = FieldLocation.Node
    sd = create_spline(loc, 2, mesh, None).desc
    x, node = _particle(mesh, px, py, -0.21)
    ext = mesh.extent(loc)
    rng = np.random.default_rng(int(1000 * (px - py + 5)))
    U = rng.standard_normal((3, 3, 3))  # (i1, j1, component), constant along z
    u = np.zeros(ext + (3,))
    for i1 in (1, 2, 3):
        for j1 in (1, 2, 3):
            u[node[0] + i1 - 2, node[1] + j1 - 2, :] = U[i1 - 1, j1 - 1]
    c = np.zeros((1, 27, 3))
    assert oracle.polypic_g2p(sd, x, u, c) == 0
    M, B = notebook(px, py, m)
    proj = np.linalg.inv(B.T @ M @ B) @ B.T @ M  # (9 modes, 9 nodes)
    want = proj @ U.reshape(9, 3)
    got = np.array([c[0, ORACLE_MODE[deg]] for deg in NB_DEGREES])
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
    others = [r for r in range(27) if r not in ORACLE_MODE.values()]
    assert np.abs(c[0, others]).max() <= 1e-12 * np.abs(want).max()
