"""Parity at the benchmark's full size (256^3 periodic grid, 8 particles per
cell: 134,217,728 particles) through properties that do not depend on the
size, since the oracle cannot run there in a test's time:

* the cell sort: keys non-decreasing, the permutation a bijection, stable
  (equal keys keep their input order);
* P2G conserves mass and momentum: the B-spline weights of a particle sum to
  one and its weighted node offsets sum to zero, so sum_i m_i = sum_p m_p and
  sum_i mu_i = sum_p m_p v_p (the affine term cancels);
* G2P of a constant velocity field returns that velocity and a zero affine
  matrix;
* the FP32 precision form against the FP64 plain form on the same clustered
  particles: grid velocity within 1e-5 (normwise relative).
"""

import pytest
import torch

from picasso_b200 import (APIC, FieldLocation, FixedGrid, UniformMesh, cell_sort, create_spline,
                          grid_velocity, permute_members, workloads)

pytestmark = pytest.mark.gpu
N = 256
PPC = 8
BITS = 36


@pytest.fixture(scope="module")
def state(cuda):
    mesh = UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1.0 / N, periodic=(True,) * 3)
    x = workloads.positions("clustered", N, PPC, seed=1002)
    m, c = workloads.particle_state(x.shape[0], 1002)
    sd0 = create_spline(FieldLocation.Node, 2, mesh, x)
    key, perm, bins = cell_sort(sd0, (4, 8, 8), chunk=4096)
    xs, ms, cs = permute_members(perm, x, m, c)
    yield {"mesh": mesh, "x0": x, "key": key, "perm": perm, "bins": bins, "x": xs, "m": ms,
           "c": cs}
    torch.cuda.empty_cache()


def test_fullsize_sort_is_sorted_stable_bijective(state):
    key, perm = state["key"].long() & 0xFFFFFFFF, state["perm"].long() & 0xFFFFFFFF
    n = key.numel()
    assert n == N ** 3 * PPC
    assert bool((key[1:] >= key[:-1]).all())
    assert bool((torch.bincount(perm, minlength=n) == 1).all())
    same = key[1:] == key[:-1]
    assert bool((perm[1:][same] > perm[:-1][same]).all())
    # the tile offsets split the sorted keys by tile
    off = state["bins"].tile_offset
    assert int(off[0]) == 0 and int(off[-1]) == n


def _p2g32(state):
    mesh, bins = state["mesh"], state["bins"]
    sd = create_spline(FieldLocation.Node, 2, mesh, state["x"])
    ext = mesh.extent(FieldLocation.Node)
    acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
    gm, gmu = FixedGrid(acc[..., 0], BITS), FixedGrid(acc[..., 1:], BITS)
    m32, c32 = state["m"].float(), state["c"].float()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    APIC.p2g(m32, c32, gm, gmu, sd, bins=bins, error_count=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return sd, acc, gm, gmu, m32, c32


def test_fullsize_p2g_conserves_mass_and_momentum(state):
    _, acc, _, _, m32, c32 = _p2g32(state)
    # (the total of 1.3e8 particle masses at 2^36 would overflow an int64 sum)
    tot = acc.double().sum(dim=(0, 1, 2)) * 2.0 ** -BITS
    mass = m32.double().sum()
    mom = (m32.double()[:, None] * c32[:, 0, :].double()).sum(dim=0)
    scale = (m32.double()[:, None] * c32[:, 0, :].double()).abs().sum(dim=0)
    assert abs(float(tot[0] - mass)) <= 1e-6 * float(mass)
    assert float(((tot[1:] - mom).abs() / scale).max()) <= 1e-6


def test_fullsize_g2p_reproduces_constant_field(state):
    mesh, bins = state["mesh"], state["bins"]
    sd = create_spline(FieldLocation.Node, 2, mesh, state["x"])
    ext = mesh.extent(FieldLocation.Node)
    a = torch.tensor([0.75, -1.5, 0.3125], dtype=torch.float32, device="cuda")
    u = a.expand(ext + (3,)).contiguous()
    c = torch.zeros((state["x"].shape[0], 4, 3), dtype=torch.float32, device="cuda")
    APIC.g2p(u, c, sd, bins=bins)
    torch.cuda.synchronize()
    assert float((c[:, 0, :] - a).abs().max()) <= 1e-6
    assert float(c[:, 1:, :].abs().max()) <= 1e-6


def test_fullsize_fp32_form_velocity_vs_fp64(state):
    sd, acc, gm, gmu, _, _ = _p2g32(state)
    mesh = state["mesh"]
    desc = mesh.descriptor(FieldLocation.Node)
    ext = mesh.extent(FieldLocation.Node)
    u32 = torch.zeros(ext + (3,), dtype=torch.float32, device="cuda")
    grid_velocity(desc, gm, gmu, u32, 1e-12)
    del acc
    g64 = torch.zeros(ext + (4,), dtype=torch.float64, device="cuda")
    sd64 = create_spline(FieldLocation.Node, 2, mesh, state["x"])
    APIC.p2g(state["m"], state["c"], g64[..., 0], g64[..., 1:], sd64)
    u64 = torch.zeros(ext + (3,), dtype=torch.float64, device="cuda")
    grid_velocity(desc, g64[..., 0], g64[..., 1:], u64, 1e-12)
    torch.cuda.synchronize()
    rel = float((u32.double() - u64).abs().max() / u64.abs().max())
    assert rel <= 1e-5, rel
