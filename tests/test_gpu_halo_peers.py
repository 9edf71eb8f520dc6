"""Halo exchange inside the tiled transfers (picasso_apic_p2g_halo /
picasso_apic_g2p_halo, SlabDecomposition.halo_peers / map_peer_grids).

With the neighbours' grids addressable, the P2G adds its ghost-plane sums
straight into the neighbour's owned planes and the G2P reads its ghost
velocities from the neighbour's owned planes.  Checked, bit for bit, against
the same kernels without peers followed by the explicit exchange (ghost
planes added into the owners' planes, owned planes copied into the ghosts):
  * all slabs in one process on one GPU, the neighbours' grids being the
    other slabs' arrays (the kernels do not wait on one another: each slab's
    launch only adds into, or reads from, the others' memory);
  * two processes on one GPU, the grids mapped through CUDA IPC handles
    exchanged over a gloo process group, the reference exchange done by
    SlabDecomposition.scatter_sum / gather over gloo on host copies.
Between GPUs the same loads and reductions cross NVLink (peer access).
"""

import datetime
import os
import socket

import numpy as np
import pytest
import torch

from particles import clustered_particles, periodic_mesh
from picasso_b200 import (APIC, FieldLocation, FixedGrid, cell_sort, create_spline,
                          grid_velocity, permute_members, spline_records)
from picasso_b200.dist import SlabDecomposition

pytestmark = pytest.mark.gpu
N = 24
BITS = 36


class _Slab:
    def __init__(self, dec):
        self.dec = dec

    def descriptor(self, location):
        return self.dec.descriptor(location)


def _particles(seed):
    mesh = periodic_mesh(N, halo=0)
    x, m, c = clustered_particles(mesh, N ** 3 * 4, nblob=4, sigma_cells=2.0, frac=0.6, seed=seed)
    xd = torch.as_tensor(x, device="cuda")
    md = torch.as_tensor(m, dtype=torch.float32, device="cuda")
    cd = torch.as_tensor(c, dtype=torch.float32, device="cuda").contiguous()
    return xd, md, cd


def _slab_state(dec, order, xd, md, cd, records):
    """The slab's particles, sorted, with their spline and bins."""
    mine = dec.owner(xd) == dec.rank
    sd0 = create_spline(FieldLocation.Node, order, _Slab(dec), xd[mine])
    _, perm, bins = cell_sort(sd0, (4, 4, 8))
    xs, ms, cs = permute_members(perm, xd[mine], md[mine], cd[mine])
    sd = create_spline(FieldLocation.Node, order, _Slab(dec), xs)
    if records:
        spline_records(sd, bins)
    return sd, ms, cs, bins


def _views(acc):
    return FixedGrid(acc[..., 0], BITS), FixedGrid(acc[..., 1:], BITS)


@pytest.mark.parametrize("world,order,records", [(2, 2, True), (3, 2, False), (3, 3, True)])
def test_halo_in_transfers_equals_explicit_exchange(cuda, world, order, records):
    xd, md, cd = _particles(700 + world + order)
    decs = [SlabDecomposition((N, N, N), 1.0 / N, world, r) for r in range(world)]
    states = [_slab_state(dec, order, xd, md, cd, records) for dec in decs]
    ext = [dec.extent() for dec in decs]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    # reference: local P2G, then ghost planes added into their owners
    local = []
    for dec, (sd, ms, cs, bins), e in zip(decs, states, ext):
        acc = torch.zeros(e + (4,), dtype=torch.int64, device="cuda")
        APIC.p2g(ms, cs, *_views(acc), sd, bins=bins, error_count=err)
        local.append(acc)
    ref = [a.clone() for a in local]
    for r, dec in enumerate(decs):
        h, o = dec.halo, dec.own
        ref[dec.upper][h:2 * h] += local[r][h + o:2 * h + o]
        ref[dec.lower][decs[dec.lower].own:decs[dec.lower].own + h] += local[r][0:h]
    # P2G with the exchange inside: slab after slab, each adding into the others
    accs = [torch.zeros(e + (4,), dtype=torch.int64, device="cuda") for e in ext]
    for dec, (sd, ms, cs, bins), acc in zip(decs, states, accs):
        peers = dec.halo_peers(_views(accs[dec.lower]), _views(accs[dec.upper]))
        APIC.p2g(ms, cs, *_views(acc), sd, bins=bins, error_count=err, peers=peers)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    for dec, acc, r_acc in zip(decs, accs, ref):
        assert torch.equal(dec.owned(acc), dec.owned(r_acc))
        h, o = dec.halo, dec.own
        assert int(acc[:h].abs().sum()) == 0 and int(acc[h + o:].abs().sum()) == 0
    # G2P: ghost velocities from the neighbours' owned planes
    us = []
    for dec, acc, e in zip(decs, accs, ext):
        u = torch.zeros(e + (3,), dtype=torch.float32, device="cuda")
        grid_velocity(dec.descriptor(), *_views(acc), u, 1e-12)
        us.append(u)
    for r, (dec, (sd, ms, cs, bins)) in enumerate(zip(decs, states)):
        h, o = dec.halo, dec.own
        filled = us[r].clone()  # what gather provides
        lo = decs[dec.lower]
        filled[0:h] = us[dec.lower][lo.own:lo.own + h]
        filled[h + o:2 * h + o] = us[dec.upper][h:2 * h]
        c_ref = torch.zeros_like(cs)
        APIC.g2p(filled, c_ref, sd, bins=bins)
        c_got = torch.full_like(cs, 7.0)
        APIC.g2p(us[r], c_got, sd, bins=bins, peers=dec.halo_peers(us[dec.lower], us[dec.upper]))
        torch.cuda.synchronize()
        assert torch.equal(c_got, c_ref)


def test_halo_peers_refuse_other_forms(cuda):
    from picasso_b200._abi import ERR_UNSUPPORTED, PicassoError
    xd, md, cd = _particles(710)
    dec = SlabDecomposition((N, N, N), 1.0 / N, 2, 0)
    sd, ms, cs, bins = _slab_state(dec, 2, xd, md, cd, False)
    acc = torch.zeros(dec.extent() + (4,), dtype=torch.int64, device="cuda")
    other = torch.zeros_like(acc)
    peers = dec.halo_peers(_views(other), _views(other))
    with pytest.raises(PicassoError) as e:  # no bins: the plain kernels have no peer form
        APIC.p2g(ms, cs, *_views(acc), sd, peers=peers)
    assert e.value.status == ERR_UNSUPPORTED


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as tdist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    tdist.init_process_group("gloo", rank=rank, world_size=world,
                             timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        xd, md, cd = _particles(720)
        dec = SlabDecomposition((N, N, N), 1.0 / N, world, rank)
        sd, ms, cs, bins = _slab_state(dec, 2, xd, md, cd, True)
        e = dec.extent()
        # reference: local P2G, the exchange over gloo on a host copy
        acc = torch.zeros(e + (4,), dtype=torch.int64, device="cuda")
        APIC.p2g(ms, cs, *_views(acc), sd, bins=bins)
        host = acc.cpu()
        dec.scatter_sum(host)
        # the exchange inside the P2G, through the neighbours' mapped grids
        shared = torch.zeros(e + (4,), dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        lower, upper = dec.map_peer_grids(shared)
        tdist.barrier()  # every rank's grid is zero before any rank adds into it
        APIC.p2g(ms, cs, *_views(shared), sd, bins=bins,
                 peers=dec.halo_peers(_views(lower[0]), _views(upper[0])))
        torch.cuda.synchronize()
        tdist.barrier()  # every rank's additions are complete
        p2g_ok = torch.equal(dec.owned(shared).cpu(), dec.owned(host))
        # G2P: reference with ghosts gathered over gloo
        u = torch.zeros(e + (3,), dtype=torch.float32, device="cuda")
        grid_velocity(dec.descriptor(), *_views(shared), u, 1e-12)
        torch.cuda.synchronize()
        u_host = u.cpu()
        dec.gather(u_host)
        c_ref = torch.zeros_like(cs)
        APIC.g2p(u_host.cuda(), c_ref, sd, bins=bins)
        ul, uu = dec.map_peer_grids(u)
        tdist.barrier()
        c_got = torch.zeros_like(cs)
        APIC.g2p(u, c_got, sd, bins=bins, peers=dec.halo_peers(ul[0], uu[0]))
        torch.cuda.synchronize()
        g2p_ok = torch.equal(c_got, c_ref)
        tdist.barrier()  # the neighbours are done reading this rank's grids
        out.put((rank, bool(p2g_ok), bool(g2p_ok)))
    finally:
        tdist.destroy_process_group()


def test_two_processes_through_ipc(cuda):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0]
    res = sorted(out.get(timeout=10) for _ in range(2))
    assert res == [(0, True, True), (1, True, True)]
