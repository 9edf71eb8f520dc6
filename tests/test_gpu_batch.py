"""Batched independent APIC instances (picasso_batch_*) through the C ABI.

The batch runs fill, P2G, grid velocity and G2P of every instance in
persistent launches fed by one work queue.  Checked here:
  * precision form: fused and phased launches, with and without the CUDA
    graph, give bit-identical grids and particle outputs to the same step
    issued as single calls instance after instance (the items run the same
    arithmetic on the same particles), over two consecutive steps;
  * every instance against the FP64 oracle (normwise relative <= 1e-5 in the
    precision form, <= 1e-12 in the FP64 form);
  * FP64 form against its sequential calls (atomic order only: <= 1e-12);
  * the bounded dependency waits of the fused launch: a wait limit of 0
    polls and a host-side cancel make waits give up, the launch ends and
    the batch status reports it.
"""

import numpy as np
import pytest
import torch

import oracle
from particles import clustered_particles, periodic_mesh, rel_err, uniform_particles
from picasso_b200 import (Batch, BatchInstance, FieldLocation, FixedGrid, PicassoError, _abi,
                          cell_sort, create_spline, permute_members)

pytestmark = pytest.mark.gpu
BITS = 36

# (edge, particles per cell or None for clustered, order, bins per tile, chunk, P2G lanes)
SHAPES = [
    (16, 4, 2, (4, 8, 8), 512, 0),
    (12, 6, 3, (4, 4, 4), 256, 4),
    (20, 2, 2, (8, 8, 8), 2048, 2),
    (8, 9, 1, (4, 4, 8), 256, 4),
    (24, None, 2, (4, 8, 8), 1024, 1),
    (10, 1, 3, (8, 8, 8), 512, 0),
    (16, 3, 1, (8, 8, 8), 512, 2),
]


def _host_state(i, edge, ppc):
    mesh = periodic_mesh(edge, halo=0)
    if ppc is None:
        x, m, c = clustered_particles(mesh, edge ** 3 * 6, nblob=3, sigma_cells=1.5, frac=0.7,
                                      seed=300 + i)
    else:
        x, m, c = uniform_particles(mesh, ppc, seed=300 + i)
    return mesh, x, m, c


def _instance(shape, host, f32):
    edge, ppc, order, tile, chunk, lanes = shape
    mesh, x, m, c = host
    pt = torch.float32 if f32 else torch.float64
    xd = torch.as_tensor(x, device="cuda")
    md = torch.as_tensor(m, dtype=pt, device="cuda")
    cd = torch.as_tensor(c, dtype=pt, device="cuda").contiguous()
    sd = create_spline(FieldLocation.Node, order, mesh, xd)
    _, perm, bins = cell_sort(sd, tile, chunk=chunk, p2g_lanes=lanes if f32 else 0)
    xd, md, cd = permute_members(perm, xd, md, cd)
    sd = create_spline(FieldLocation.Node, order, mesh, xd)
    ext = mesh.extent(FieldLocation.Node)
    if f32:
        acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
        m_i, mu_i = FixedGrid(acc[..., 0], BITS), FixedGrid(acc[..., 1:], BITS)
        u = torch.zeros(ext + (3,), dtype=torch.float32, device="cuda")
    else:
        acc = torch.zeros(ext + (4,), dtype=torch.float64, device="cuda")
        m_i, mu_i = acc[..., 0], acc[..., 1:]
        u = torch.zeros(ext + (3,), dtype=torch.float64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    inst = BatchInstance(sd, md, cd, m_i, mu_i, u, bins, 1e-12, err)
    return {"inst": inst, "acc": acc, "u": u, "c": cd, "x": xd, "m": md, "perm": perm,
            "err": err, "mesh": mesh, "order": order}


def _build(f32, hosts):
    return [_instance(s, h, f32) for s, h in zip(SHAPES, hosts)]


@pytest.fixture(scope="module")
def hosts():
    return [_host_state(i, s[0], s[1]) for i, s in enumerate(SHAPES)]


def _state(runs):
    torch.cuda.synchronize()
    return [(r["acc"].clone(), r["u"].clone(), r["c"].clone()) for r in runs]


@pytest.mark.parametrize("mode,graph", [("fused", True), ("fused", False), ("phased", True),
                                        ("phased", False)])
def test_precision_batch_matches_sequential_bit_for_bit(cuda, hosts, mode, graph):
    ref_runs, runs = _build(True, hosts), _build(True, hosts)
    ref = Batch([r["inst"] for r in ref_runs], mode=mode)
    bat = Batch([r["inst"] for r in runs], mode=mode)
    for _ in range(2):  # the second step starts from the first step's c_p
        ref.step_sequential()
        bat.step(graph=graph)
    bat.status()
    for (a0, u0, c0), (a1, u1, c1) in zip(_state(ref_runs), _state(runs)):
        assert torch.equal(a0, a1)
        assert torch.equal(u0, u1)
        assert torch.equal(c0, c1)
    for r in runs:
        assert int(r["err"].item()) == 0
    info = bat.info()
    assert info["count"] == len(SHAPES) and info["precision_form"]
    assert info["particles"] == sum(r["x"].shape[0] for r in runs)
    ref.close()
    bat.close()


def _oracle_step(r, c_in):
    mesh, order = r["mesh"], r["order"]
    ext = mesh.extent(FieldLocation.Node)
    sdo = create_spline(FieldLocation.Node, order, mesh, None).desc
    x = r["x"].cpu().numpy()
    m = r["m"].double().cpu().numpy()
    gm, gmu, gu = np.zeros(ext), np.zeros(ext + (3,)), np.zeros(ext + (3,))
    oracle.apic_p2g(sdo, x, m, c_in, gm, gmu)
    oracle.grid_velocity(sdo.mesh, gm, gmu, gu, 1e-12)
    co = np.zeros_like(c_in)
    oracle.apic_g2p(sdo, x, gu, co)
    return gm, gmu, gu, co


@pytest.mark.parametrize("f32", [True, False])
def test_batch_vs_oracle(cuda, hosts, f32):
    runs = _build(f32, hosts)
    c_in = [r["c"].double().cpu().numpy() for r in runs]
    bat = Batch([r["inst"] for r in runs], mode="fused")
    bat.step(graph=True)
    bat.status()
    tol = 1e-5 if f32 else 1e-12
    for r, ci in zip(runs, c_in):
        gm_o, gmu_o, gu_o, c_o = _oracle_step(r, ci)
        a = r["acc"].double().cpu().numpy()
        if f32:
            a = a * 2.0 ** -BITS
        assert rel_err(a[..., 0], gm_o) <= tol
        assert rel_err(a[..., 1:], gmu_o) <= tol
        assert rel_err(r["u"].double().cpu().numpy(), gu_o) <= tol
        cg = r["c"].double().cpu().numpy()
        assert rel_err(cg[:, 0], c_o[:, 0]) <= tol
        assert rel_err(cg[:, 1:], c_o[:, 1:]) <= tol
        assert int(r["err"].item()) == 0
    bat.close()


def test_fp64_batch_matches_sequential(cuda, hosts):
    ref_runs, runs = _build(False, hosts), _build(False, hosts)
    ref = Batch([r["inst"] for r in ref_runs], mode="phased")
    bat = Batch([r["inst"] for r in runs], mode="fused")
    ref.step_sequential()
    bat.step(graph=True)
    bat.status()
    for (a0, u0, c0), (a1, u1, c1) in zip(_state(ref_runs), _state(runs)):
        assert rel_err(a1.cpu().numpy(), a0.cpu().numpy()) <= 1e-12
        assert rel_err(u1.cpu().numpy(), u0.cpu().numpy()) <= 1e-12
        assert rel_err(c1.cpu().numpy(), c0.cpu().numpy()) <= 1e-12
    ref.close()
    bat.close()


def _expect_timeout(bat):
    with pytest.raises(PicassoError) as e:
        bat.status()
    assert e.value.status == _abi.ERR_TIMEOUT


@pytest.mark.parametrize("graph", [False, True])
def test_wait_that_runs_out_ends_the_launch(cuda, hosts, graph):
    """A fused step whose dependency waits may poll 0 times: the items that
    find their instance's previous phase unfinished give up at once, the
    launch still ends, and status() reports PICASSO_ERR_TIMEOUT (the bounded
    device wait, run out on purpose; nothing faults or hangs).  Restoring
    the default limit gives complete steps again."""
    runs = _build(True, hosts)
    bat = Batch([r["inst"] for r in runs], mode="fused")
    # the first wave of persistent warps takes fill and P2G items together, so
    # the P2G items poll while their instance's fill is still running
    bat.set_wait_limit(0)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    bat.step(graph=graph)
    t1.record()
    torch.cuda.synchronize()
    assert t0.elapsed_time(t1) < 1000.0  # ms: the launch did not wait out a long bound
    _expect_timeout(bat)
    bat.set_wait_limit(1 << 22)
    bat.step(graph=graph)
    bat.status()  # complete again
    bat.close()


def test_cancel_ends_fused_steps_until_reported(cuda, hosts):
    """picasso_batch_cancel: every wait of the next fused steps gives up at
    once until status() has reported PICASSO_ERR_TIMEOUT; after that the
    batch steps normally and matches the sequential calls from the same
    particles."""
    runs = _build(True, hosts)
    bat = Batch([r["inst"] for r in runs], mode="fused")
    saved = [r["c"].clone() for r in runs]
    bat.cancel()
    bat.step(graph=False)
    bat.step(graph=True)
    _expect_timeout(bat)
    # restart from the saved particle state; the step is complete again
    for r, c0 in zip(runs, saved):
        r["c"].copy_(c0)
    ref_runs = _build(True, hosts)
    ref = Batch([r["inst"] for r in ref_runs], mode="fused")
    ref.step_sequential()
    bat.step(graph=True)
    bat.status()
    for (a0, u0, c0), (a1, u1, c1) in zip(_state(ref_runs), _state(runs)):
        assert torch.equal(a0, a1)
        assert torch.equal(u0, u1)
        assert torch.equal(c0, c1)
    ref.close()
    bat.close()
