"""Autotuner for the sorted (tiled) transfers.

For an instance shape -- mesh edge, particles per cell, spline order and
form -- it picks the three launch knobs of the tiled path:
  * ``tile``: bins per tile (the sort's tile shape, which sets the node tile
    a work item stages in shared memory),
  * ``chunk``: particles per work item,
  * ``lanes``: lanes per particle of the tiled P2G (precision form only).
Each candidate is timed on a synthetic instance of the shape's class (uniform
positions, v ~ N(0, 1), m ~ U[0.5, 1.5], C ~ N(0, 0.1)) on the current GPU:
sort + permute once per (tile, chunk), then the median of a few
fill -> P2G -> velocity -> G2P steps with CUDA events.  With ``batched=True``
the step is that of a :class:`~picasso_b200.api.Batch` of enough copies of
the instance (each with its own grids and c_p) to fill the GPU, so that the
choice optimises throughput inside a batch rather than the latency of one
small launch.  Shapes are grouped in classes (order, form, edge bucket,
particles-per-cell bucket) so a batch of hundreds of instances needs a
handful of measurements; results are kept in memory and, with
``cache_path``, in a JSON file keyed by device name.
"""

import json
import os

import torch

from . import api, workloads

TILES = [(4, 4, 4), (4, 4, 8), (4, 8, 8), (8, 8, 8)]
CHUNKS = [1024, 4096]
EDGE_BUCKETS = [(0, 32), (33, 64), (65, 1 << 20)]
PPC_BUCKETS = [(0, 4), (5, 10), (11, 1 << 20)]


def lanes_for(order, f32):
    if not f32:
        return [0]
    return [4] if order == 3 else [1, 2]


def _bucket(v, buckets):
    for i, (lo, hi) in enumerate(buckets):
        if lo <= v <= hi:
            return i
    return len(buckets) - 1


class Tuner:
    def __init__(self, cache_path=None, trials=3, fixed_bits=36, seed=1234, batched=False,
                 max_tile_bins=None, batch_particles=4 << 20):
        self.cache_path = cache_path
        self.trials = trials
        self.batched = batched
        self.tiles = [t for t in TILES
                      if max_tile_bins is None or t[0] * t[1] * t[2] <= max_tile_bins]
        self.batch_particles = batch_particles
        self.fixed_bits = fixed_bits
        self.seed = seed
        self.device = torch.cuda.get_device_name() if torch.cuda.is_available() else "none"
        self.table = {}
        self.measurements = 0
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.table = json.load(f).get(self.device, {})

    def class_of(self, order, edge, ppc, f32):
        return "o%d-%s-e%d-p%d%s" % (order, "f32" if f32 else "f64",
                                     _bucket(edge, EDGE_BUCKETS), _bucket(ppc, PPC_BUCKETS),
                                     "-b" if self.batched else "")

    def representative(self, cls_shapes):
        """Median edge and particles per cell of the shapes in a class."""
        edges = sorted(s[0] for s in cls_shapes)
        ppcs = sorted(s[1] for s in cls_shapes)
        return edges[len(edges) // 2], ppcs[len(ppcs) // 2]

    def tune_shapes(self, shapes, f32):
        """shapes: iterable of (edge, ppc, order).  Returns {class: choice}
        and fills the table for every class the shapes fall in."""
        groups = {}
        for e, p, o in shapes:
            groups.setdefault(self.class_of(o, e, p, f32), []).append((e, p, o))
        for cls, members in groups.items():
            if cls not in self.table:
                e, p = self.representative(members)
                self.table[cls] = self.tune(members[0][2], e, p, f32)
        self.save()
        return {c: self.table[c] for c in groups}

    def choice(self, order, edge, ppc, f32):
        cls = self.class_of(order, edge, ppc, f32)
        if cls not in self.table:
            self.table[cls] = self.tune(order, edge, ppc, f32)
        return self.table[cls]

    def save(self):
        if not self.cache_path:
            return
        data = {}
        if os.path.exists(self.cache_path):
            with open(self.cache_path) as f:
                data = json.load(f)
        data[self.device] = self.table
        with open(self.cache_path, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)

    # -- measurement ---------------------------------------------------------
    def _instance(self, order, edge, ppc, f32):
        mesh = api.UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1.0 / edge, periodic=(True,) * 3)
        x = workloads.positions("uniform", edge, ppc, self.seed)
        m, c = workloads.particle_state(x.shape[0], self.seed,
                                        dtype=torch.float32 if f32 else torch.float64)
        return mesh, x, m, c.contiguous()

    def _grids(self, mesh, f32):
        ext = mesh.extent(api.FieldLocation.Node)
        if f32:
            acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
            gm = api.FixedGrid(acc[..., 0], self.fixed_bits)
            gmu = api.FixedGrid(acc[..., 1:], self.fixed_bits)
            u = torch.zeros(ext + (3,), dtype=torch.float32, device="cuda")
            fill = api.FixedGrid(acc, self.fixed_bits)
        else:
            acc = torch.zeros(ext + (4,), dtype=torch.float64, device="cuda")
            gm, gmu = acc[..., 0], acc[..., 1:]
            u = torch.zeros(ext + (3,), dtype=torch.float64, device="cuda")
            fill = acc
        return fill, gm, gmu, u

    def tune(self, order, edge, ppc, f32):
        mesh, x, m, c = self._instance(order, edge, ppc, f32)
        loc = api.FieldLocation.Node
        desc = mesh.descriptor(loc)
        fill, gm, gmu, u = self._grids(mesh, f32)
        best = None
        results = []
        copies = max(1, min(32, self.batch_particles // max(1, x.shape[0])))
        for tile in self.tiles:
            if any(t > edge for t in tile):
                continue
            for chunk in CHUNKS:
                sd0 = api.create_spline(loc, order, mesh, x)
                _, perm, bins = api.cell_sort(sd0, tile, chunk=chunk)
                xs, ms, cs = api.permute_members(perm, x, m, c)
                sd = api.create_spline(loc, order, mesh, xs)
                for lanes in lanes_for(order, f32):
                    bins.desc.p2g_lanes = lanes
                    if self.batched:
                        t = self._time_batch(mesh, f32, sd, ms, cs, bins, copies)
                    else:
                        t = self._time(desc, fill, gm, gmu, u, sd, ms, cs, bins)
                    self.measurements += 1
                    r = {"tile": list(tile), "chunk": chunk, "lanes": lanes, "ms": t}
                    results.append(r)
                    if best is None or t < best["ms"]:
                        best = r
                del xs, ms, cs, sd, perm, bins
        best = dict(best)
        best["edge"], best["ppc"], best["candidates"] = edge, ppc, len(results)
        best["copies"] = copies if self.batched else 1
        return best

    def _time_batch(self, mesh, f32, sd, m, c, bins, copies):
        """Step time per instance of a phased Batch of `copies` instances that
        share x_p and m_p and own their c_p and grids."""
        insts = []
        for _ in range(copies):
            _, gm, gmu, u = self._grids(mesh, f32)
            insts.append(api.BatchInstance(sd, m, c.clone(), gm, gmu, u, bins))
        b = api.Batch(insts, mode="phased")
        b.step(graph=True)
        torch.cuda.synchronize()
        times = []
        for _ in range(self.trials):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            b.step(graph=True)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1) / copies)
        b.status()
        b.close()
        times.sort()
        return times[len(times) // 2]

    def _time(self, desc, fill, gm, gmu, u, sd, m, c, bins):
        def step():
            api.grid_fill(desc, fill, 0.0, ncomp=4)
            api.APIC.p2g(m, c, gm, gmu, sd, bins=bins)
            api.grid_velocity(desc, gm, gmu, u, 1e-12)
            api.APIC.g2p(u, c, sd, bins=bins)

        step()
        torch.cuda.synchronize()
        times = []
        for _ in range(self.trials):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            step()
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        times.sort()
        return times[len(times) // 2]
