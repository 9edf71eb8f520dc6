"""Slab decomposition over ranks (picasso_b200.dist) on the CPU with gloo.

2 and 3 ranks each take the particles of their slab of a periodic 12^3 mesh,
run the transfers of the oracle on their ghosted local mesh, and exchange
halos.  Checked against the single-domain oracle on the whole mesh:
  * scatter_sum after P2G: the owned planes of every rank equal the global
    grid mass and momentum (normwise relative <= 1e-12);
  * gather before G2P: the ghost planes hold the neighbours' owned planes,
    and G2P on the local mesh gives every particle the global c_p;
  * migrate after a move of up to one cell: every rank ends with exactly the
    particles it owns, none lost or duplicated, members moved with them.
The same code drives NCCL on GPUs; a run on several GPUs is not available to
this test suite (one GPU per job here).
"""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as tdist
import torch.multiprocessing as mp

import oracle
from particles import periodic_mesh, rel_err, uniform_particles
from picasso_b200 import FieldLocation, _abi, create_spline
from picasso_b200.dist import SlabDecomposition

N = 12


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _spline(desc, order):
    sp = _abi.Spline()
    sp.mesh = desc
    sp.location = FieldLocation.Node
    sp.order = order
    return sp


def _global_reference(order):
    mesh = periodic_mesh(N, halo=0)
    x, m, c = uniform_particles(mesh, 2, seed=600)
    sdo = create_spline(FieldLocation.Node, order, mesh, None).desc
    ext = mesh.extent(FieldLocation.Node)
    gm, gmu = np.zeros(ext), np.zeros(ext + (3,))
    oracle.apic_p2g(sdo, x, m, c, gm, gmu)
    u = np.random.default_rng(601).standard_normal(ext + (3,))
    co = np.zeros_like(c)
    oracle.apic_g2p(sdo, x, u, co)
    return x, m, c, gm, gmu, u, co


def _worker(rank, world, port, order, q):
    try:
        tdist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                                 world_size=world)
        x, m, c, gm_g, gmu_g, u_g, co_g = _global_reference(order)
        dec = SlabDecomposition((N, N, N), 1.0 / N, world, rank, halo=2)
        xt = torch.from_numpy(x)
        mine = (dec.owner(xt) == rank).numpy()
        xl, ml, cl = x[mine], m[mine], c[mine]
        sp = _spline(dec.descriptor(), order)
        ext = dec.extent()
        gm, gmu = np.zeros(ext), np.zeros(ext + (3,))
        assert oracle.apic_p2g(sp, xl, ml, cl, gm, gmu) == 0  # no stencil left the ghosts
        tgm, tgmu = torch.from_numpy(gm), torch.from_numpy(gmu)
        dec.scatter_sum(tgm, tgmu)
        own = slice(dec.x0, dec.x0 + dec.own)
        e_m = rel_err(dec.owned(tgm).numpy(), gm_g[own])
        e_mu = rel_err(dec.owned(tgmu).numpy(), gmu_g[own])
        ghosts_clear = bool((tgm[:dec.halo] == 0).all() and (tgm[dec.halo + dec.own:] == 0).all())
        # gather: owned planes from the global velocity, ghosts from neighbours
        u = torch.zeros(ext + (3,), dtype=torch.float64)
        dec.owned(u).copy_(torch.from_numpy(u_g[own]))
        dec.gather(u)
        planes = [(dec.x0 - dec.halo + i) % N for i in range(ext[0])]
        e_ghost = float((u.numpy() - u_g[planes]).__abs__().max())
        co = np.zeros_like(cl)
        oracle.apic_g2p(sp, xl, u.numpy(), co)
        e_c = rel_err(co, co_g[mine])
        # migrate: move every particle by up to one cell, hand off, check owners
        rng = np.random.default_rng(602)
        step = rng.uniform(-1.0, 1.0, x.shape) / N
        pid = torch.arange(x.shape[0], dtype=torch.int64)[torch.from_numpy(mine)]
        xm = torch.from_numpy(x[mine] + step[mine])
        cm = torch.from_numpy(cl.copy())
        xm, pid, cm = dec.migrate(xm, pid, cm)
        owned_ok = bool((dec.owner(xm) == rank).all())
        moved = (x + step - 0.0) % 1.0
        pos_ok = bool(np.allclose(xm.numpy(), moved[pid.numpy()], rtol=0, atol=1e-12))
        c_ok = bool(np.array_equal(cm.numpy(), c[pid.numpy()]))
        ids = [None] * world
        tdist.all_gather_object(ids, pid.tolist())
        allids = sorted(i for part in ids for i in part)
        complete = allids == list(range(x.shape[0]))
        q.put((rank, e_m, e_mu, ghosts_clear, e_ghost, e_c, owned_ok, pos_ok, c_ok, complete,
               int(mine.sum())))
        tdist.barrier()
        tdist.destroy_process_group()
    except Exception as exc:  # report instead of hanging the parent
        q.put((rank, "error: %r" % (exc,)))
        raise


@pytest.mark.parametrize("world,order", [(2, 2), (3, 3), (3, 2)])
def test_slab_decomposition_matches_single_domain(world, order):
    oracle.lib()  # build the oracle once, before the workers start
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, order, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    total = 0
    for r in results:
        assert not isinstance(r[1], str), r
        rank, e_m, e_mu, ghosts_clear, e_ghost, e_c, owned_ok, pos_ok, c_ok, complete, n = r
        assert e_m <= 1e-12 and e_mu <= 1e-12, (rank, e_m, e_mu)
        assert ghosts_clear
        assert e_ghost == 0.0
        assert e_c <= 1e-12
        assert owned_ok and pos_ok and c_ok and complete
        total += n
    assert total == N ** 3 * 2


def test_single_rank_is_the_periodic_mesh():
    dec = SlabDecomposition((8, 8, 8), 0.125, 1, 0)
    d = dec.descriptor()
    assert list(d.extent) == [8, 8, 8] and list(d.periodic) == [1, 1, 1]
    assert dec.halo == 0 and dec.own == 8
    x = torch.tensor([[1.05, -0.1, 0.5]], dtype=torch.float64)
    (xw,) = dec.migrate(x)
    assert torch.allclose(xw, torch.tensor([[0.05, 0.9, 0.5]], dtype=torch.float64))


def test_uneven_slabs_and_owner():
    dec = SlabDecomposition((10, 4, 4), 0.1, 3, 1)
    assert dec.sizes == [4, 3, 3] and dec.starts == [0, 4, 7]
    assert (dec.x0, dec.own, dec.lower, dec.upper) == (4, 3, 0, 2)
    d = dec.descriptor()
    assert list(d.extent) == [7, 4, 4] and list(d.periodic) == [0, 1, 1]
    assert abs(d.low_corner[0] - 0.2) < 1e-15
    x = torch.tensor([[0.05, 0, 0], [0.45, 0, 0], [0.75, 0, 0], [0.99, 0, 0], [1.01, 0, 0],
                      [-0.02, 0, 0]], dtype=torch.float64)
    assert dec.owner(x).tolist() == [0, 1, 2, 2, 0, 2]
    with pytest.raises(ValueError):
        SlabDecomposition((4, 4, 4), 0.25, 3, 0, halo=2)
