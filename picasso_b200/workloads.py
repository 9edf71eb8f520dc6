"""Seeded synthetic particle sets with the shapes of the benchmark
configurations, generated on the GPU.

  uniform:   ppc particles uniformly placed in every cell of a periodic n^3
             box [0, 1)^3 (dx = 1/n); v ~ N(0, 1)^3, m ~ U[0.5, 1.5],
             affine rows C ~ N(0, 0.1)
  clustered: 70 % of the particles in 32 Gaussian blobs (sigma = 2 dx,
             centres uniform), 30 % uniform, wrapped into the box; v, m, C
             as above

Arrays come back in the order generated (not cell-sorted).  Particle
matrices are (N, 4, 3) with row 0 = velocity, rows 1..3 = C^T, i.e. the
reference's c_p layout.
"""

import torch


def _gen(seed, device):
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return g


def positions(kind, n_cells, ppc, seed, device="cuda", nblob=32, sigma_cells=2.0, frac=0.7):
    dx = 1.0 / n_cells
    total = n_cells ** 3 * ppc
    g = _gen(seed, device)
    if kind == "uniform":
        cell = torch.arange(total, device=device, dtype=torch.int64) // ppc
        k = cell % n_cells
        j = (cell // n_cells) % n_cells
        i = cell // (n_cells * n_cells)
        x = torch.stack([i, j, k], dim=1).to(torch.float64)
        del cell, i, j, k
        x += torch.rand((total, 3), generator=g, device=device, dtype=torch.float64)
        x *= dx
        return x
    if kind != "clustered":
        raise ValueError("workload kind must be 'uniform' or 'clustered'")
    nb = int(total * frac)
    centres = torch.rand((nblob, 3), generator=g, device=device, dtype=torch.float64)
    which = torch.randint(0, nblob, (nb,), generator=g, device=device)
    x = torch.empty((total, 3), device=device, dtype=torch.float64)
    x[:nb] = torch.randn((nb, 3), generator=g, device=device, dtype=torch.float64)
    x[:nb] *= sigma_cells * dx
    x[:nb] += centres[which]
    del which
    x[nb:] = torch.rand((total - nb, 3), generator=g, device=device, dtype=torch.float64)
    x.remainder_(1.0)
    x[x >= 1.0] = 0.0
    return x


def particle_state(total, seed, device="cuda", dtype=torch.float64, ncomp=3, affine_sigma=0.1):
    """(m, c): m ~ U[0.5, 1.5], c[:, 0] ~ N(0, 1), c[:, 1:] ~ N(0, affine_sigma)."""
    g = _gen(seed + 7919, device)
    m = torch.rand((total,), generator=g, device=device, dtype=torch.float64)
    m += 0.5
    c = torch.randn((total, 4, ncomp), generator=g, device=device, dtype=torch.float64)
    c[:, 1:] *= affine_sigma
    if dtype != torch.float64:
        return m.to(dtype), c.to(dtype)
    return m, c


def polypic_modes(total, nmode, seed, device="cuda", dtype=torch.float64, hi_sigma=0.05):
    """Mode 0 ~ N(0, 1), higher modes ~ N(0, hi_sigma), 3 components."""
    g = _gen(seed + 104729, device)
    u = torch.randn((total, nmode, 3), generator=g, device=device, dtype=torch.float64)
    u[:, 1:] *= hi_sigma
    return u.to(dtype) if dtype != torch.float64 else u
