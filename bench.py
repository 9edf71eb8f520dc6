#!/usr/bin/env python
"""Benchmark of the APIC transfer step: P2G -> grid velocity update -> G2P.

Default workload: 256^3 periodic grid, 8 particles per cell (134,217,728
particles), quadratic B-spline on nodes, clustered positions (70 % of the
particles in 32 Gaussian blobs of sigma = 2 dx, 30 % uniform), particles
already cell-sorted and resident in HBM.  One step = zero the grid
accumulators, P2G, FP64 velocity update (u = p / m where m > 1e-12), G2P.

The headline `value` is the FP32 precision form (FP32 particle state and
arithmetic, 64-bit fixed-point grid accumulation, FP64 division and
positions); the plain FP64 form runs on the same particles and is reported
in `fp64_plain`.  The cell sort and the permutation of particle storage are
timed separately (`sort`).  `e2e` is the same step through the C ABI with
the particle arrays in pinned host memory, copies included.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs its own replica of the workload (no
collective in the data path); `value` is the sum over ranks of particles
divided by the slowest rank's time.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("P2G+G2P particles/s at 256³·8ppc, FP32 form vs FP64 plain, % HBM roofline")
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--ppc", type=int, default=8)
    ap.add_argument("--order", type=int, default=2)
    ap.add_argument("--workload", default="clustered", choices=["clustered", "uniform"])
    ap.add_argument("--tile", type=int, nargs=3, default=[4, 8, 8])
    ap.add_argument("--chunk", type=int, default=4096, help="particles per work item")
    ap.add_argument("--p2g-lanes", type=int, default=0,
                    help="lanes per particle of the tiled P2G (0 = library choice)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 plain leg")
    ap.add_argument("--fuse", action="store_true",
                    help="grid velocity inside the P2G launch (APIC.p2g_update) instead of "
                         "its own pass")
    ap.add_argument("--no-records", action="store_true",
                    help="tiled kernels read the positions instead of spline records")
    ap.add_argument("--batch-leg-instances", type=int, default=96,
                    help="instances of the bounded batched leg of the default run (0: none)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--unsorted", action="store_true",
                    help="keep the generated particle order (plain kernels)")
    ap.add_argument("--cpu-sample-grid", type=int, default=64)
    ap.add_argument("--json-out", default=None)
    ap.add_argument("--suite", default="step", choices=["step", "batch", "advect", "polypic"],
                    help="step: the APIC step on one mesh (default, includes the advect and "
                         "polypic legs unless --no-legs); batch: many independent instances; "
                         "advect / polypic: one leg alone")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the cubic advection and PolyPIC legs of the default run")
    ap.add_argument("--adv-grid", type=int, default=256)
    ap.add_argument("--adv-steps", type=int, default=10)
    ap.add_argument("--adv-tile", type=int, nargs=3, default=[4, 4, 8])
    ap.add_argument("--pp-grid", type=int, default=128)
    ap.add_argument("--pp-tile", type=int, nargs=3, default=[4, 8, 8])
    ap.add_argument("--pp-chunk", type=int, default=1024)
    ap.add_argument("--batch-instances", type=int, default=512)
    ap.add_argument("--batch-seed", type=int, default=4)
    ap.add_argument("--batch-forms", default="fp32,fp64")
    ap.add_argument("--batch-max-tile-bins", type=int, default=256,
                    help="largest tile (bins) the batch autotuner may pick")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": PEAKS_FALLBACK["hbm_gbs"], "source": "fallback"}


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "samples": len(sm),
                "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# reference arm: the oracle port of the reference's CPU path
# ---------------------------------------------------------------------------
def cpu_sample(args, steps, warmup, nthreads, check_gpu=False):
    """P2G -> velocity -> G2P of the CPU port (OpenMP, duplicated scatter
    grids as Kokkos' OpenMP ScatterView) on a bounded sample: the same
    workload generator on a grid^3 periodic box (grid = --cpu-sample-grid).
    check_gpu: the GPU forms then run the same step on the same particles
    and their errors against this FP64 result are returned as well."""
    import numpy as np
    import torch

    import oracle
    from picasso_b200 import FieldLocation, UniformMesh, create_spline, workloads

    n = args.cpu_sample_grid
    mesh = UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1.0 / n, periodic=(True, True, True))
    x = workloads.positions(args.workload, n, args.ppc, seed=1002, device="cpu").numpy()
    m, c = workloads.particle_state(x.shape[0], seed=1002, device="cpu")
    m, c = m.numpy(), np.ascontiguousarray(c.numpy())
    sd = create_spline(FieldLocation.Node, args.order, mesh, None).desc
    times = []
    for s in range(warmup + steps):
        cc = c.copy()
        t0 = time.perf_counter()
        grids = oracle.apic_step_omp(sd, x, m, cc, nthreads)
        t1 = time.perf_counter()
        if s >= warmup:
            times.append(t1 - t0)
    sec = sum(times) / len(times)
    out = {"value": x.shape[0] / sec, "unit": "particles/s", "cores": nthreads, "kind": "port",
           "sample": "%d^3 periodic grid, %d ppc (%d particles), order %d, %s positions, "
                     "FP64, OpenMP with duplicated scatter grids; mean of %d steps"
                     % (n, args.ppc, x.shape[0], args.order, args.workload, steps),
           "ms_per_step": 1e3 * sec}
    if check_gpu:
        out["errors_vs_oracle"] = gpu_errors_vs_oracle(args, mesh, x, m, c, grids, cc)
    return out


def _errs(got, ref, mask=None):
    """normwise max|a-b|/max|b| and the largest per-entry relative error (per
    grid node with m > threshold, or per particle: max-norm over components)."""
    import numpy as np
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.abs(ref).max()
    nw = float(np.abs(got - ref).max() / den) if den > 0 else 0.0
    axes = tuple(range(mask.ndim if mask is not None else 1, ref.ndim))
    num = np.abs(got - ref).max(axis=axes) if axes else np.abs(got - ref)
    dd = np.abs(ref).max(axis=axes) if axes else np.abs(ref)
    sel = dd > 0
    if mask is not None:
        sel &= mask
    rel = num[sel] / dd[sel]
    pe = float(rel.max()) if sel.any() else 0.0
    return {"normwise": nw, "per_entry": pe, "entries": int(sel.sum()),
            "entries_above_1e-5": int(np.count_nonzero(rel > 1e-5))}


def gpu_errors_vs_oracle(args, mesh, x, m, c, grids, c_ref):
    """Errors of the GPU forms against the oracle's FP64 step on the CPU
    sample: FP32 form (tiled kernels on cell-sorted particles with spline
    records, the headline path; and the plain fixed-point kernel) and FP64
    plain form (unsorted particles)."""
    import torch

    import picasso_b200 as pb

    gm_o, gmu_o, gu_o = grids
    heavy = gm_o > 1e-12
    loc = pb.FieldLocation.Node
    ext = mesh.extent(loc)
    xd = torch.as_tensor(x, device="cuda")
    res = {"sample": "the CPU-baseline sample (%d^3, %d ppc, %s, order %d); per_entry: per "
                     "grid node with m > 1e-12 or per particle, max-norm over components"
                     % (args.cpu_sample_grid, args.ppc, args.workload, args.order)}
    # FP32 form, tiled (the headline path)
    sd = pb.create_spline(loc, args.order, mesh, xd)
    _, perm, bins = pb.cell_sort(sd, tuple(args.tile), chunk=args.chunk,
                                 p2g_lanes=args.p2g_lanes)
    xs, ms, cs = pb.permute_members(perm, xd, torch.as_tensor(m, dtype=torch.float32,
                                                              device="cuda"),
                                    torch.as_tensor(c, dtype=torch.float32,
                                                    device="cuda").contiguous())
    sds = pb.create_spline(loc, args.order, mesh, xs)
    if not args.no_records:
        pb.spline_records(sds, bins)
    acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
    gm, gmu = pb.FixedGrid(acc[..., 0], FIXED_BITS), pb.FixedGrid(acc[..., 1:], FIXED_BITS)
    u = torch.zeros(ext + (3,), dtype=torch.float32, device="cuda")
    pb.APIC.p2g(ms, cs, gm, gmu, sds, bins=bins)
    pb.grid_velocity(sds.desc.mesh, gm, gmu, u, 1e-12)
    pb.APIC.g2p(u, cs, sds, bins=bins)
    back = torch.empty_like(cs)
    back[perm.long()] = cs
    cb = back.double().cpu().numpy()
    res["fp32_tiled"] = {"grid_mass": _errs(gm.to_float().cpu().numpy(), gm_o, heavy),
                         "grid_momentum": _errs(gmu.to_float().cpu().numpy(), gmu_o, heavy),
                         "grid_velocity": _errs(u.double().cpu().numpy(), gu_o, heavy),
                         "particle_velocity": _errs(cb[:, 0], c_ref[:, 0]),
                         "particle_affine": _errs(cb[:, 1:], c_ref[:, 1:])}
    # FP32 form, plain fixed-point kernel on the unsorted particles
    sd = pb.create_spline(loc, args.order, mesh, xd)
    accp = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
    gmp, gmup = pb.FixedGrid(accp[..., 0], FIXED_BITS), pb.FixedGrid(accp[..., 1:], FIXED_BITS)
    up = torch.zeros(ext + (3,), dtype=torch.float32, device="cuda")
    cp_ = torch.as_tensor(c, dtype=torch.float32, device="cuda").contiguous()
    pb.APIC.p2g(torch.as_tensor(m, dtype=torch.float32, device="cuda"), cp_, gmp, gmup, sd)
    pb.grid_velocity(sd.desc.mesh, gmp, gmup, up, 1e-12)
    pb.APIC.g2p(up, cp_, sd)
    cph = cp_.double().cpu().numpy()
    res["fp32_plain"] = {"grid_mass": _errs(gmp.to_float().cpu().numpy(), gm_o, heavy),
                         "grid_momentum": _errs(gmup.to_float().cpu().numpy(), gmu_o, heavy),
                         "grid_velocity": _errs(up.double().cpu().numpy(), gu_o, heavy),
                         "particle_velocity": _errs(cph[:, 0], c_ref[:, 0]),
                         "particle_affine": _errs(cph[:, 1:], c_ref[:, 1:])}
    # FP64 plain form, unsorted
    sd = pb.create_spline(loc, args.order, mesh, xd)
    g64 = torch.zeros(ext + (4,), dtype=torch.float64, device="cuda")
    u64 = torch.zeros(ext + (3,), dtype=torch.float64, device="cuda")
    c64 = torch.as_tensor(c, device="cuda").clone()
    pb.APIC.p2g(torch.as_tensor(m, device="cuda"), c64, g64[..., 0], g64[..., 1:], sd)
    pb.grid_velocity(sd.desc.mesh, g64[..., 0], g64[..., 1:], u64, 1e-12)
    pb.APIC.g2p(u64, c64, sd)
    c64h = c64.cpu().numpy()
    g64h = g64.cpu().numpy()
    res["fp64_plain"] = {"grid_mass": _errs(g64h[..., 0], gm_o, heavy),
                         "grid_momentum": _errs(g64h[..., 1:], gmu_o, heavy),
                         "grid_velocity": _errs(u64.cpu().numpy(), gu_o, heavy),
                         "particle_velocity": _errs(c64h[:, 0], c_ref[:, 0]),
                         "particle_affine": _errs(c64h[:, 1:], c_ref[:, 1:])}
    return res


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    cb = cpu_sample(args, max(1, args.steps), max(0, args.warmup), nthreads)
    line = {"metric": METRIC, "value": cb["value"], "unit": "particles/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": cb["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": config_of(args),
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "particles/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def config_of(args):
    return {"workload": "APIC order-%d P2G + FP64 grid velocity + G2P, %d^3 periodic nodes, "
                        "%d ppc, %s positions, cell-sorted, resident in HBM"
                        % (args.order, args.grid, args.ppc, args.workload),
            "grid": args.grid, "ppc": args.ppc, "order": args.order,
            "particles": args.grid ** 3 * args.ppc, "positions": args.workload,
            "tile": list(args.tile), "chunk": args.chunk, "p2g_lanes": args.p2g_lanes,
            "l2": "inputs >> 126 MB L2 (no flush needed)",
            "parallelism": "replicas"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
class Step:
    """Buffers and launches of one form of the APIC step.  With bins that
    carry spline records the tiled kernels read the records instead of the
    positions (16 instead of 24 bytes per particle and transfer).  fused:
    the precision form's grid velocity update runs inside the P2G launch
    (APIC.p2g_update), so the step has no separate velocity pass (its
    "velocity" interval is empty)."""

    def __init__(self, form, mesh, x, m, c, bins, stream, fused=False):
        import torch

        import picasso_b200 as pb

        self.pb = pb
        self.form = form
        self.mesh = mesh
        self.loc = pb.FieldLocation.Node
        self.desc = mesh.descriptor(self.loc)
        self.sd = pb.create_spline(self.loc, ORDER[0], mesh, x)
        self.m, self.c = m, c
        self.bins = bins
        self.stream = stream
        ext = mesh.extent(self.loc)
        dev = x.device
        if form == "fp32":
            self.acc = torch.zeros(ext + (4,), dtype=torch.int64, device=dev)
            self.gm = pb.FixedGrid(self.acc[..., 0], FIXED_BITS)
            self.gmu = pb.FixedGrid(self.acc[..., 1:], FIXED_BITS)
            self.u = torch.zeros(ext + (3,), dtype=torch.float32, device=dev)
        else:
            self.acc = torch.zeros(ext + (4,), dtype=torch.float64, device=dev)
            self.gm = self.acc[..., 0]
            self.gmu = self.acc[..., 1:]
            self.u = torch.zeros(ext + (3,), dtype=torch.float64, device=dev)
        self.acc_fill = pb.FixedGrid(self.acc, FIXED_BITS) if form == "fp32" else self.acc
        self.fused = bool(fused and form == "fp32" and bins is not None)
        self.ws = None
        if self.fused:
            self.ws = torch.empty(pb.p2g_update_workspace(bins), dtype=torch.uint8, device=dev)
        # memset + kernels of the library per step: fill (memset), P2G,
        # velocity, G2P; fused: fill, counter memset, empty-region kernel,
        # P2G + update, G2P
        self.launches_per_step = 4

    def run(self, events=None):
        pb = self.pb
        s = self.stream
        if events is not None:
            events[0].record(s)
        pb.grid_fill(self.desc, self.acc_fill, 0.0, ncomp=4, stream=s)
        if events is not None:
            events[1].record(s)
        if self.fused:
            # v = p / m where m > 1e-12 (dt = 0: no force, no gravity)
            pb.APIC.p2g_update(self.m, self.c, self.gm, self.gmu, self.u, self.sd, dt=0.0,
                               mass_threshold=1e-12, workspace=self.ws, stream=s,
                               bins=self.bins)
            if events is not None:
                events[2].record(s)
                events[3].record(s)
        else:
            pb.APIC.p2g(self.m, self.c, self.gm, self.gmu, self.sd, stream=s, bins=self.bins)
            if events is not None:
                events[2].record(s)
            pb.grid_velocity(self.desc, self.gm, self.gmu, self.u, 1e-12, stream=s)
            if events is not None:
                events[3].record(s)
        pb.APIC.g2p(self.u, self.c, self.sd, stream=s, bins=self.bins)
        if events is not None:
            events[4].record(s)

    @property
    def records(self):
        return self.bins is not None and self.bins.records is not None

    def kernel_bytes(self, n, nodes):
        """Algorithmic bytes per launch: fill, p2g, velocity, g2p.  The
        position costs 24 bytes per transfer (3 x FP64), or 16 with spline
        records."""
        if self.form == "fp32":
            sf, sg, su = 4, 8, 4
        else:
            sf, sg, su = 8, 8, 8
        px = 16 if self.records else 24
        if self.fused:
            # the update reads the accumulators the P2G has just added into
            # (L2) and writes the velocity
            return {"fill": nodes * 4 * sg,
                    "p2g": n * (px + 13 * sf) + nodes * (4 * sg + 3 * su),
                    "velocity": 0,
                    "g2p": n * (px + 12 * sf) + nodes * 3 * su}
        return {"fill": nodes * 4 * sg,
                "p2g": n * (px + 13 * sf) + nodes * 4 * sg,
                "velocity": nodes * (4 * sg + 3 * su),
                "g2p": n * (px + 12 * sf) + nodes * 3 * su}

    def model_bytes_per_particle(self, ppc):
        """Step bytes per particle: 2 position reads, 25 particle values
        (P2G reads m, v, C; G2P writes v, C), 14 grid values per node."""
        sf = 4 if self.form == "fp32" else 8
        px = 16 if self.records else 24
        return 2 * px + 25 * sf + 14 * 8 / ppc


ORDER = [2]
FIXED_BITS = 36


def time_form(step, steps, warmup, dist):
    import torch
    names = ["fill", "p2g", "velocity", "g2p"]
    for _ in range(warmup):
        step.run()
    torch.cuda.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in range(steps)]
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(step.stream)
    for k in range(steps):
        step.run(ev[k])
    t1.record(step.stream)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    ms = t0.elapsed_time(t1) / steps
    per = {nm: sum(ev[k][q].elapsed_time(ev[k][q + 1]) for k in range(steps)) / steps
           for q, nm in enumerate(names)}
    if dist:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    return ms, per


def measured_traffic(kernel, n, form):
    """DRAM bytes of one launch of a tiled FP32-form kernel, from the ncu
    capture summarised in profiles/ncu_traffic.json, scaled by the particle
    count (traffic grows in proportion to the particles processed)."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    name = {"p2g": "p2g_tiled", "g2p": "g2p_tiled"}.get(kernel)
    if form != "fp32" or name is None or not os.path.exists(path):
        return None
    with open(path) as f:
        t = json.load(f)
    return t[name]["dram_bytes_per_particle"] * n if name in t else None


def roofline(step, per_ms, n, nodes, peak):
    kb = step.kernel_bytes(n, nodes)
    dom = max(per_ms, key=lambda k: per_ms[k])
    ach = kb[dom] / (per_ms[dom] * 1e-3) / 1e9
    kernels = {k: {"ms": per_ms[k], "bytes": kb[k],
                   "gbs": kb[k] / (per_ms[k] * 1e-3) / 1e9 if per_ms[k] > 0 else None}
               for k in per_ms}
    return {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak["hbm_gbs"],
            "unit": "GB/s", "frac": ach / peak["hbm_gbs"],
            "peak_source": peak["source"],
            "traffic": measured_traffic(dom, n, step.form) if step.bins is not None else None,
            "algorithmic_bytes": kb[dom]}, kernels


def run_ours(args):
    import torch

    import picasso_b200 as pb
    from picasso_b200 import workloads

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = world > 1
    torch.cuda.set_device(local)
    if dist:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ORDER[0] = args.order
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    n_cells = args.grid
    mesh = pb.UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1.0 / n_cells,
                          periodic=(True, True, True))
    seed = 1000 + (2 if args.workload == "clustered" else 1) + 17 * rank
    x = workloads.positions(args.workload, n_cells, args.ppc, seed, device=dev)
    n = x.shape[0]
    nodes = n_cells ** 3
    m64, c64 = workloads.particle_state(n, seed, device=dev)
    sort_info = None
    bins = None
    # the generation-order particles stay for the FP64 plain form on unsorted
    # particles (the reference's own situation: no sort)
    unsorted = (x, m64, c64) if not args.no_fp64 else None
    if not args.unsorted:
        sd0 = pb.create_spline(pb.FieldLocation.Node, args.order, mesh, x)
        ws = None
        for it in range(2):  # second run is timed
            torch.cuda.synchronize()
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
            key, perm, bins = pb.cell_sort(sd0, tuple(args.tile), chunk=args.chunk,
                                           p2g_lanes=args.p2g_lanes)
            e1.record()
            xs, ms_, cs = pb.permute_members(perm, x, m64, c64)
            e2.record()
            torch.cuda.synchronize()
            sort_info = {"sort_ms": e0.elapsed_time(e1), "permute_ms": e1.elapsed_time(e2),
                         "tile": list(args.tile), "num_tiles": bins.num_tiles}
        x, m64, c64 = xs, ms_, cs
        del key, perm, xs, ms_, cs
        if not args.no_records:
            # spline records of the sorted particles (in-cell fractions and
            # sort key, 16 bytes each): built once per sort, like the sort
            sds = pb.create_spline(pb.FieldLocation.Node, args.order, mesh, x)
            rec = torch.empty((n, 4), dtype=torch.float32, device=dev)
            pb.spline_records(sds, bins, out=rec)
            torch.cuda.synchronize()
            e0, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
            e0.record()
            pb.spline_records(sds, bins, out=rec)
            e1.record()
            torch.cuda.synchronize()
            sort_info["records_ms"] = e0.elapsed_time(e1)
    m32, c32 = m64.float(), c64.float()
    peak = peaks()
    clk = Clocks(local)

    out = {}
    # FP32 precision form (headline)
    # the grid velocity as its own pass (measured faster than inside the P2G
    # launch, which is reported beside it); --fuse puts it inside
    fused = bins is not None and args.fuse
    s32 = Step("fp32", mesh, x, m32, c32.clone(), bins, stream, fused=fused)
    clk.start()
    ms32, per32 = time_form(s32, args.steps, args.warmup, dist)
    clocks = clk.stop()
    rf32, k32 = roofline(s32, per32, n, nodes, peak)
    out["fp32"] = (ms32, per32, rf32, k32)
    model_bytes = s32.model_bytes_per_particle(args.ppc)
    from_positions = None
    if bins is not None and bins.records is not None:
        # the same step with the tiled kernels reading the FP64 positions
        rec_keep = bins.records
        bins.attach_records(None)
        sx = Step("fp32", mesh, x, m32, c32.clone(), bins, stream, fused=fused)
        msx, perx = time_form(sx, args.steps, args.warmup, dist)
        rfx, _ = roofline(sx, perx, n, nodes, peak)
        from_positions = {"ms_per_step": msx, "particles_per_s": world * n / (msx * 1e-3),
                          "kernels_ms": perx, "p2g_frac": rfx["frac"] if rfx["kernel"] == "p2g"
                          else None}
        del sx
        bins.attach_records(rec_keep)
    other = None
    if bins is not None:
        # the same step with the grid velocity in the other place
        sf_ = Step("fp32", mesh, x, m32, c32.clone(), bins, stream, fused=not fused)
        msf, perf = time_form(sf_, args.steps, args.warmup, dist)
        other = {"ms_per_step": msf, "particles_per_s": world * n / (msf * 1e-3),
                 "kernels_ms": perf}
        del sf_
    # FP64 plain form: on the generation-order particles (no sort, as the
    # reference runs) and on the cell-sorted ones
    if not args.no_fp64:
        if unsorted is not None and not args.unsorted:
            xu, mu_, cu = unsorted
            su = Step("fp64", mesh, xu, mu_, cu.clone(), None, stream)
            msu, peru = time_form(su, args.steps, args.warmup, dist)
            rfu, ku = roofline(su, peru, n, nodes, peak)
            out["fp64_unsorted"] = (msu, peru, rfu, ku)
            del su, xu, mu_, cu
        unsorted = None
        s64 = Step("fp64", mesh, x, m64, c64.clone(), None, stream)
        ms64, per64 = time_form(s64, args.steps, args.warmup, dist)
        rf64, k64 = roofline(s64, per64, n, nodes, peak)
        out["fp64"] = (ms64, per64, rf64, k64)
        # per-field error of the FP32 form against the FP64 result of the
        # same step (the FP64 form is parity-checked against the oracle)
        s64.c.copy_(c64)
        s32.c.copy_(c32)
        s64.run()
        s32.run()
        torch.cuda.synchronize()
        u64 = s64.u
        u32 = s32.u.double()
        den = u64.abs().max()
        err = {"grid_velocity": float((u32 - u64).abs().max() / den),
               "grid_mass": float((s32.gm.to_float() - s64.gm).abs().max() / s64.gm.abs().max()),
               "grid_momentum": float((s32.gmu.to_float() - s64.gmu).abs().max()
                                      / s64.gmu.abs().max()),
               "particle_velocity": float((s32.c[:, 0].double() - s64.c[:, 0]).abs().max()
                                          / s64.c[:, 0].abs().max()),
               "particle_affine": float((s32.c[:, 1:].double() - s64.c[:, 1:]).abs().max()
                                        / s64.c[:, 1:].abs().max())}
        out["errors"] = err
        del s64
    # e2e through the C ABI with host buffers (FP32 form)
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(s32, x, m32, c32, args, stream, dist, world)
    legs = {}
    if world == 1 and not args.no_legs:
        # free the headline workload first: the legs hold their own particles
        del s32
        x = m32 = c32 = m64 = c64 = sd0 = None
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        legs["advect_cubic"] = run_advect(args, peak)
        legs["polypic"] = run_polypic(args, peak)
        if args.batch_leg_instances > 0:
            legs["batch"] = run_batch_leg(args, peak)
    cpu = None
    errors_vs_oracle = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_sample(args, 3, 1, os.cpu_count() or 1, check_gpu=True)
        errors_vs_oracle = cpu.get("errors_vs_oracle")
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}

    ms32, per32, rf32, k32 = out["fp32"]
    value = world * n / (ms32 * 1e-3)
    line = {"metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (i64 fixed-point grid, f64 division/positions)", "data": "synthetic",
            "config": config_of(args), "roofline": rf32,
            "step_roofline": {"bytes_per_particle_model": model_bytes,
                              "model": "2 position reads (%d B each: %s) + 25 particle values "
                                       "(FP32) + 14 grid values (8 B) per node / ppc"
                                       % (16 if bins is not None and bins.records is not None
                                          else 24,
                                          "spline record" if bins is not None
                                          and bins.records is not None else "3 x FP64"),
                              "achieved_gbs": n * model_bytes / (ms32 * 1e-3) / 1e9,
                              "frac": n * model_bytes / (ms32 * 1e-3) / 1e9 / peak["hbm_gbs"]},
            "kernels": k32,
            # kernels of this library per step: P2G (+ update), the empty-region
            # zeroing or the velocity pass, G2P (the fills are cudaMemsetAsync)
            "gpu_launches": 3 * args.steps,
            "clocks": clocks}
    if from_positions:
        line["fp32_from_positions"] = from_positions
    if other:
        line["fp32_separate_velocity_pass" if fused else "fp32_velocity_fused_into_p2g"] = other
    line["step"] = ("fill (memset), P2G with the grid velocity update fused into its flush, G2P"
                    if fused else "fill (memset), P2G, grid velocity, G2P")
    if "fp64" in out:
        ms64, per64, rf64, k64 = out["fp64"]
        line["fp64_plain"] = {"value": world * n / (ms64 * 1e-3), "ms_per_step": ms64,
                              "particles": "cell-sorted",
                              "roofline": rf64, "kernels": k64,
                              "step_frac": n * 262.0 / (ms64 * 1e-3) / 1e9 / peak["hbm_gbs"]}
        best64 = ms64
        if "fp64_unsorted" in out:
            msu, peru, rfu, ku = out["fp64_unsorted"]
            line["fp64_plain_unsorted"] = {
                "value": world * n / (msu * 1e-3), "ms_per_step": msu,
                "particles": "generation order (no sort)", "roofline": rfu, "kernels": ku,
                "step_frac": n * 262.0 / (msu * 1e-3) / 1e9 / peak["hbm_gbs"]}
            best64 = min(ms64, msu)
        # the 3x target compares with the faster of the two FP64 plain runs
        line["speedup_fp32_vs_fp64"] = best64 / ms32
        line["speedup_fp32_vs_fp64_basis"] = ("fp64_plain (sorted)" if best64 == ms64
                                              else "fp64_plain_unsorted")
        line["errors_vs_fp64"] = out["errors"]
    if sort_info:
        line["sort"] = sort_info
    if e2e:
        line["e2e"] = e2e
    if cpu:
        line["cpu_baseline"] = cpu
        ratios = {"fp32_gpu_vs_cpu": value / cpu["value"]}
        if "fp64_plain" in line:
            best = max(line["fp64_plain"]["value"],
                       line.get("fp64_plain_unsorted", {}).get("value", 0.0))
            # same arithmetic on both sides: FP64 GPU plain form vs the FP64 CPU port
            ratios["fp64_gpu_vs_fp64_cpu"] = best / cpu["value"]
        line["ratios_vs_cpu_baseline"] = ratios
    if errors_vs_oracle:
        line["errors_vs_oracle"] = errors_vs_oracle
    line.update(legs)
    if "advect_cubic" in legs:
        adv = legs["advect_cubic"]
        # the whole time-loop step (re-sort and permutation included) of the
        # cubic advection workload, next to the headline's transfer step
        line["time_loop"] = {"workload": adv["workload"],
                             "fp32_particles_per_s": adv["fp32"]["particles_per_s"],
                             "fp32_ms_per_step": adv["fp32"]["ms_per_step"],
                             "fp64_particles_per_s": adv["fp64"]["particles_per_s"],
                             "fp64_ms_per_step": adv["fp64"]["ms_per_step"],
                             "speedup_fp32_vs_fp64": adv["speedup_fp32_vs_fp64"]}
    if rank == 0:
        print(json.dumps(line))
        if args.json_out:
            with open(args.json_out, "w") as f:
                json.dump(line, f, indent=1)
    if dist:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def leg_roofline(kernels_ms, kernel_bytes, peak):
    """Per-kernel achieved GB/s of a leg from algorithmic bytes per launch,
    and the dominant kernel's fraction of the HBM peak."""
    ks = {}
    for k, ms in kernels_ms.items():
        if k in kernel_bytes and ms > 0:
            gbs = kernel_bytes[k] / (ms * 1e-3) / 1e9
            ks[k] = {"ms": ms, "bytes": kernel_bytes[k], "gbs": gbs, "frac": gbs / peak["hbm_gbs"]}
    dom = max(ks, key=lambda k: ks[k]["ms"]) if ks else None
    return {"bound": "hbm", "kernel": dom, "achieved": ks[dom]["gbs"] if dom else None,
            "peak": peak["hbm_gbs"], "unit": "GB/s", "frac": ks[dom]["frac"] if dom else None,
            "peak_source": peak["source"], "kernels": ks}


# ---------------------------------------------------------------------------
# advection leg: cubic APIC, P2G -> grid update -> G2P + x += dt v -> re-sort
# ---------------------------------------------------------------------------
def run_advect(args, peak):
    """256^3 periodic grid, 8 ppc uniform, cubic B-spline, dt = 0.1 dx: every
    step re-sorts the particles by cell and permutes every member, zeroes the
    grid, P2G, velocity update, then G2P fused with the position update, which
    also emits the moved particles' sort keys for the next step's sort (the
    first sort starts from the positions).  FP64 plain form (the reference's
    arithmetic) and FP32 precision form (tiled kernels); both forms start from
    the same particles."""
    import torch

    import picasso_b200 as pb
    from picasso_b200 import workloads

    g = args.adv_grid
    mesh = pb.UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1.0 / g, periodic=(True,) * 3)
    loc = pb.FieldLocation.Node
    desc = mesh.descriptor(loc)
    ext = mesh.extent(loc)
    dt = 0.1 / g
    seed = 1001
    res = {"workload": "cubic APIC, %d^3 periodic, 8 ppc uniform, dt = 0.1 dx, per step: "
                       "cell re-sort (from the keys the previous G2P emitted) + permute (FP32 "
                       "form: + spline records of the permuted particles), fill, P2G, "
                       "velocity, G2P + advection + sort keys" % g,
           "steps": args.adv_steps, "tile": list(args.adv_tile)}
    names = ["sort", "permute", "fill", "p2g", "velocity", "g2p_advect"]
    for form in ("fp64", "fp32"):
        f32 = form == "fp32"
        x = workloads.positions("uniform", g, 8, seed)
        m, c = workloads.particle_state(x.shape[0], seed,
                                        dtype=torch.float32 if f32 else torch.float64)
        c = c.contiguous()
        n = x.shape[0]
        if f32:
            acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
            gm = pb.FixedGrid(acc[..., 0], FIXED_BITS)
            gmu = pb.FixedGrid(acc[..., 1:], FIXED_BITS)
            fill = pb.FixedGrid(acc, FIXED_BITS)
            u = torch.zeros(ext + (3,), dtype=torch.float32, device="cuda")
        else:
            acc = torch.zeros(ext + (4,), dtype=torch.float64, device="cuda")
            gm, gmu, fill = acc[..., 0], acc[..., 1:], acc
            u = torch.zeros(ext + (3,), dtype=torch.float64, device="cuda")
        state = {"x": x, "m": m, "c": c, "keys": None}
        keybuf = torch.empty(n, dtype=torch.int32, device="cuda")
        tile = tuple(args.adv_tile)
        # the permutation writes into the other one of two member sets, so the
        # timed steps allocate no particle storage
        spare = {"x": torch.empty_like(x), "m": torch.empty_like(m), "c": torch.empty_like(c)}
        sort_bufs = pb.SortBuffers(pb.create_spline(loc, 3, mesh, x), tile)
        # FP32 form: spline records of the permuted particles for P2G, and the
        # grid velocity inside the P2G launch
        recbuf = torch.empty((n, 4), dtype=torch.float32, device="cuda") if f32 else None
        fws = {}

        def step(ev=None):
            def mark(i):
                if ev is not None:
                    ev[i].record()
            mark(0)
            sd0 = pb.create_spline(loc, 3, mesh, state["x"])
            _, perm, bins = pb.cell_sort(sd0, tile, chunk=4096, p2g_lanes=4 if f32 else 0,
                                         keys=state["keys"], out=sort_bufs)
            mark(1)
            for name in ("x", "m", "c"):
                pb.permute(perm, state[name], spare[name])
                state[name], spare[name] = spare[name], state[name]
            sd = pb.create_spline(loc, 3, mesh, state["x"])
            if f32:
                pb.spline_records(sd, bins, out=recbuf)
            mark(2)
            pb.grid_fill(desc, fill, 0.0, ncomp=4)
            mark(3)
            if f32 and args.fuse:
                if "ws" not in fws:
                    fws["ws"] = torch.empty(pb.p2g_update_workspace(bins), dtype=torch.uint8,
                                            device="cuda")
                pb.APIC.p2g_update(state["m"], state["c"], gm, gmu, u, sd, dt=0.0,
                                   mass_threshold=1e-12, workspace=fws["ws"], bins=bins)
                mark(4)
            else:
                pb.APIC.p2g(state["m"], state["c"], gm, gmu, sd, bins=bins)
                mark(4)
                pb.grid_velocity(desc, gm, gmu, u, 1e-12)
            mark(5)
            state["keys"] = pb.APIC.g2p_advect(u, state["c"], sd, dt, bins=bins, key_tile=tile,
                                               keys_out=keybuf)
            mark(6)

        step()
        torch.cuda.synchronize()
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(7)]
              for _ in range(args.adv_steps)]
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for k in range(args.adv_steps):
            step(ev[k])
        t1.record()
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1) / args.adv_steps
        per = {nm: sum(ev[k][q].elapsed_time(ev[k][q + 1]) for k in range(args.adv_steps))
               / args.adv_steps for q, nm in enumerate(names)}
        xs = state["x"]
        nodes = g ** 3
        sf = 4 if f32 else 8
        px = 16 if f32 else 24  # FP32 form: P2G reads the spline records
        kb = {"permute": n * (2 * (24 + sf + 12 * sf) + 3 * 4 + (24 + 16 if f32 else 0)),
              "fill": nodes * 32,
              "p2g": n * (px + 13 * sf) + nodes * (32 + (3 * sf if f32 and args.fuse else 0)),
              "velocity": 0 if f32 and args.fuse else nodes * (32 + 3 * sf),
              "g2p_advect": n * (24 + 24 + 12 * sf + 4) + nodes * 3 * sf}
        step_bytes = sum(kb.values())
        res[form] = {"ms_per_step": ms, "particles_per_s": n / (ms * 1e-3),
                     "transfer_ms": per["fill"] + per["p2g"] + per["velocity"]
                     + per["g2p_advect"], "kernels_ms": per,
                     "roofline": leg_roofline(per, kb, peak),
                     "step_frac_without_sort": step_bytes / ((ms - per["sort"]) * 1e-3) / 1e9
                     / peak["hbm_gbs"],
                     "positions_in_box": bool(float(xs.min()) >= 0.0 and float(xs.max()) < 1.0)}
        del state, spare, x, m, c, acc, u, keybuf, sort_bufs
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    res["speedup_fp32_vs_fp64"] = res["fp64"]["ms_per_step"] / res["fp32"]["ms_per_step"]
    return res


# ---------------------------------------------------------------------------
# PolyPIC leg: 128^3, 8 ppc, quadratic (27 modes) and linear (8 modes)
# ---------------------------------------------------------------------------
def run_polypic(args, peak):
    """128^3 periodic grid, 8 ppc uniform, mode 0 ~ N(0, 1), other modes
    ~ N(0, 0.05), m ~ U[0.5, 1.5]; step = fill, PolyPIC P2G (dt = 0.1 dx),
    velocity update, PolyPIC G2P; particles cell-sorted once.  FP64 and FP32
    forms; per-mode error of the FP32 form against the FP64 result."""
    import torch

    import picasso_b200 as pb
    from picasso_b200 import workloads

    g = args.pp_grid
    mesh = pb.UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1.0 / g, periodic=(True,) * 3)
    loc = pb.FieldLocation.Node
    desc = mesh.descriptor(loc)
    ext = mesh.extent(loc)
    seed = 1003
    x = workloads.positions("uniform", g, 8, seed)
    n = x.shape[0]
    m64, _ = workloads.particle_state(n, seed)
    res = {"workload": "PolyPIC, %d^3 periodic, 8 ppc uniform, cell-sorted, per step: fill, "
                       "P2G, velocity, G2P (FP32 form: tiled kernels, tile %s, work items of %d)"
                       % (g, list(args.pp_tile), args.pp_chunk), "particles": n}
    for order, nm in ((2, 27), (1, 8)):
        sd0 = pb.create_spline(loc, order, mesh, x)
        _, perm, bins = pb.cell_sort(sd0, tuple(args.pp_tile), chunk=args.pp_chunk)
        modes = workloads.polypic_modes(n, nm, seed)
        xs, ms, us = pb.permute_members(perm, x, m64, modes)
        sd = pb.create_spline(loc, order, mesh, xs)
        out = {}
        finals = {}
        for form in ("fp64", "fp32"):
            f32 = form == "fp32"
            mm = ms.float() if f32 else ms
            c0 = us.float() if f32 else us
            c = c0.clone()
            if f32:
                acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
                gm = pb.FixedGrid(acc[..., 0], FIXED_BITS)
                gmu = pb.FixedGrid(acc[..., 1:], FIXED_BITS)
                fill = pb.FixedGrid(acc, FIXED_BITS)
                u = torch.zeros(ext + (3,), dtype=torch.float32, device="cuda")
            else:
                acc = torch.zeros(ext + (4,), dtype=torch.float64, device="cuda")
                gm, gmu, fill = acc[..., 0], acc[..., 1:], acc
                u = torch.zeros(ext + (3,), dtype=torch.float64, device="cuda")

            def step(ev=None):
                if ev is not None:
                    ev[0].record()
                pb.grid_fill(desc, fill, 0.0, ncomp=4)
                # the FP32 form takes the tiled kernels (bins); FP64 the plain ones
                pb.PolyPIC.p2g(mm, c, c, gmu, gm, 0.1 / g, sd, bins=bins if f32 else None)
                if ev is not None:
                    ev[1].record()
                pb.grid_velocity(desc, gm, gmu, u, 1e-12)
                if ev is not None:
                    ev[2].record()
                pb.PolyPIC.g2p(u, c, sd, bins=bins if f32 else None)
                if ev is not None:
                    ev[3].record()

            c.copy_(c0)
            step()  # the error comparison uses this first step
            torch.cuda.synchronize()
            finals[form] = c.double().clone()
            for _ in range(max(args.warmup - 1, 0)):
                step()
            torch.cuda.synchronize()
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)]
                   for _ in range(args.steps)]
            t0.record()
            for k in range(args.steps):
                step(evs[k])
            t1.record()
            torch.cuda.synchronize()
            msp = t0.elapsed_time(t1) / args.steps
            kms = {nm: sum(e[q].elapsed_time(e[q + 1]) for e in evs) / args.steps
                   for q, nm in enumerate(["fill_p2g", "velocity", "g2p"])}
            sf = 4 if f32 else 8
            nodes = g ** 3
            kb = {"fill_p2g": nodes * 32 + n * (24 + sf + nm * 3 * sf) + nodes * 32,
                  "velocity": nodes * (32 + 3 * sf),
                  "g2p": n * (24 + nm * 3 * sf) + nodes * 3 * sf}
            out[form] = {"ms_per_step": msp, "particles_per_s": n / (msp * 1e-3),
                         "kernels_ms": kms, "roofline": leg_roofline(kms, kb, peak),
                         "step_frac": sum(kb.values()) / (msp * 1e-3) / 1e9 / peak["hbm_gbs"]}
            del acc, u, c
        ref = finals["fp64"]
        err = (finals["fp32"] - ref).abs().amax(dim=(0, 2)) / ref.abs().amax(dim=(0, 2))
        out["fp32_per_mode_rel_err_max"] = float(err.max())
        out["fp32_per_mode_rel_err"] = [float(e) for e in err]
        out["speedup_fp32_vs_fp64"] = out["fp64"]["ms_per_step"] / out["fp32"]["ms_per_step"]
        res["quadratic_27" if order == 2 else "linear_8"] = out
        del xs, ms, us, modes, perm, sd, sd0, finals
        torch.cuda.empty_cache()
    return res


def run_leg_alone(args):
    import torch
    torch.cuda.set_device(0)
    peak = peaks()
    clk = Clocks(0)
    clk.start()
    r = run_advect(args, peak) if args.suite == "advect" else run_polypic(args, peak)
    r["clocks"] = clk.stop()
    line = json.dumps({"suite": args.suite, **r})
    print(line)
    if args.json_out:
        with open(args.json_out, "w") as f:
            f.write(line + "\n")


def run_e2e(step, x, m32, c32, args, stream, dist, world):
    """Same step with the particle arrays in pinned host memory: every step
    copies x, m, c in, runs fill / P2G / velocity / G2P through the C ABI and
    copies c (the step's result) out.  Two device buffer sets and three
    streams pipeline consecutive steps the way an application would with the
    asynchronous API: the inputs of step s + 1 travel host -> device while
    step s computes and the result of step s - 1 travels device -> host
    (PCIe is full duplex)."""
    import torch
    n = x.shape[0]
    hx = torch.empty(x.shape, dtype=x.dtype, pin_memory=True)
    hm = torch.empty(m32.shape, dtype=m32.dtype, pin_memory=True)
    hc = torch.empty(c32.shape, dtype=c32.dtype, pin_memory=True)
    houts = [torch.empty(c32.shape, dtype=c32.dtype, pin_memory=True) for _ in range(2)]
    hx.copy_(x)
    hm.copy_(m32)
    hc.copy_(c32)
    h2d = hx.numel() * 8 + hm.numel() * 4 + hc.numel() * 4
    d2h = houts[0].numel() * 4
    # all K steps (not a shorter sample): the last result's device -> host
    # copy drains after the last step and is part of the timed region, so
    # fewer steps would overstate its share of a long run
    steps = max(2, args.steps)
    s_in, s_run, s_out = torch.cuda.Stream(), stream, torch.cuda.Stream()
    # a second buffer set: positions, members and grids of its own, same bins
    other = Step(step.form, step.mesh, torch.empty_like(x), torch.empty_like(m32),
                 torch.empty_like(c32), step.bins, s_run)
    bufs = [step, other]
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_run = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    for e in ev_run + ev_out:
        e.record(s_run)

    def one(k):
        b = bufs[k % 2]
        with torch.cuda.stream(s_in):
            s_in.wait_event(ev_run[k % 2])   # step k - 2 no longer reads these inputs
            b.sd.x.copy_(hx, non_blocking=True)
            b.m.copy_(hm, non_blocking=True)
            s_in.wait_event(ev_out[k % 2])   # step k - 2's result has left c
            b.c.copy_(hc, non_blocking=True)
            ev_in[k % 2].record(s_in)
        s_run.wait_event(ev_in[k % 2])
        b.run()
        ev_run[k % 2].record(s_run)
        with torch.cuda.stream(s_out):
            s_out.wait_event(ev_run[k % 2])
            houts[k % 2].copy_(b.c, non_blocking=True)
            ev_out[k % 2].record(s_out)

    one(0)
    one(1)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(s_run)
    s_in.wait_event(t0)
    for k in range(steps):
        one(k)
    s_run.wait_stream(s_out)
    t1.record(s_run)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / steps
    if dist:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    # both buffer sets computed the same step from the same inputs
    consistent = bool(torch.equal(houts[0], houts[1]))
    return {"value": world * n / (ms * 1e-3), "unit": "particles/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": ms, "steps": steps,
            "results_identical_across_buffers": consistent,
            "path": "pinned host buffers, torch copies on two copy streams + C-ABI transfer "
                    "calls, consecutive steps double-buffered"}


# ---------------------------------------------------------------------------
# batched independent instances
# ---------------------------------------------------------------------------
BATCH_METRIC = ("batched APIC step particles/s: independent instances, edges 16..96 step 8, "
                "1-16 ppc, quadratic/cubic, one persistent launch per step vs sequential "
                "single launches")


def batch_shapes(count, seed):
    """(edge, particles per cell, order) of every instance: edge uniform in
    {16, 24, ..., 96}, particles per cell uniform in 1..16, order 2 or 3."""
    import numpy as np
    rng = np.random.default_rng(seed)
    edges = rng.choice(np.arange(16, 97, 8), count)
    ppcs = rng.integers(1, 17, count)
    orders = rng.choice([2, 3], count)
    return [(int(e), int(p), int(o)) for e, p, o in zip(edges, ppcs, orders)]


def batch_bytes(shapes, f32):
    """Algorithmic HBM bytes of one batched step (the per-kernel model of the
    single-mesh step, summed over instances)."""
    sf, su = (4, 4) if f32 else (8, 8)
    total = 0
    for e, p, _ in shapes:
        n, nodes = e ** 3 * p, e ** 3
        total += nodes * 32                                   # fill
        total += n * (24 + 13 * sf) + nodes * 32              # p2g
        total += nodes * (32 + 3 * su)                        # velocity
        total += n * (24 + 12 * sf) + nodes * 3 * su          # g2p
    return total


def batch_measure(shapes, forms, steps, warmup, peak, max_tile_bins, clocks=None):
    """Times the batched step of the instance shapes in each form: fused and
    phased persistent launches (CUDA graph) and the sequential single
    launches, after autotuning tile, chunk and lanes per instance class."""
    import torch

    import picasso_b200 as pb
    from picasso_b200 import autotune, workloads

    tuner = autotune.Tuner(fixed_bits=FIXED_BITS, batched=True, max_tile_bins=max_tile_bins)
    out = {}
    for form in forms:
        f32 = form == "fp32"
        t0 = time.time()
        tuner.tune_shapes(shapes, f32)
        tune_s = time.time() - t0
        per_particle = 24 + (52 if f32 else 104)
        per_node = (32 + 12) if f32 else (32 + 24)
        # instances in groups that fit in 80 % of the free memory; each group
        # is one batch, the step time of all instances is the sum over groups
        budget = 0.8 * torch.cuda.mem_get_info()[0]
        groups, cur, cur_b = [], [], 0
        for i, (e, p, o) in enumerate(shapes):
            need = e ** 3 * p * per_particle + e ** 3 * per_node
            if cur and cur_b + need > budget:
                groups.append(cur)
                cur, cur_b = [], 0
            cur.append(i)
            cur_b += need
        groups.append(cur)
        pdt = torch.float32 if f32 else torch.float64
        n_total = sum(e ** 3 * p for e, p, _ in shapes)
        nbytes = batch_bytes(shapes, f32)
        res = {"instances": len(shapes), "particles": n_total, "tune_s": tune_s,
               "groups": len(groups), "algorithmic_bytes": nbytes, "modes": {}}
        acc_ms = {"fused": 0.0, "phased": 0.0, "sequential": 0.0}
        infos = {}
        for grp in groups:
            insts = []
            for i in grp:
                e, p, o = shapes[i]
                ch = tuner.choice(o, e, p, f32)
                mesh = pb.UniformMesh([0, 0, 0, 1, 1, 1], cell_size=1.0 / e,
                                      periodic=(True,) * 3)
                x = workloads.positions("uniform", e, p, seed=1000 + i)
                m, c = workloads.particle_state(x.shape[0], 1000 + i, dtype=pdt)
                loc = pb.FieldLocation.Node
                sd0 = pb.create_spline(loc, o, mesh, x)
                _, perm, bins = pb.cell_sort(sd0, tuple(ch["tile"]), chunk=ch["chunk"],
                                             p2g_lanes=ch["lanes"])
                x, m, c = pb.permute_members(perm, x, m, c.contiguous())
                del perm, sd0
                sd = pb.create_spline(loc, o, mesh, x)
                ext = mesh.extent(loc)
                if f32:
                    acc = torch.zeros(ext + (4,), dtype=torch.int64, device="cuda")
                    gm = pb.FixedGrid(acc[..., 0], FIXED_BITS)
                    gmu = pb.FixedGrid(acc[..., 1:], FIXED_BITS)
                    u = torch.zeros(ext + (3,), dtype=torch.float32, device="cuda")
                else:
                    acc = torch.zeros(ext + (4,), dtype=torch.float64, device="cuda")
                    gm, gmu = acc[..., 0], acc[..., 1:]
                    u = torch.zeros(ext + (3,), dtype=torch.float64, device="cuda")
                insts.append(pb.BatchInstance(sd, m, c, gm, gmu, u, bins, 1e-12))
            torch.cuda.synchronize()
            for mode in ("fused", "phased", "sequential"):
                b = pb.Batch(insts, mode="phased" if mode == "sequential" else mode)
                if mode == "sequential":
                    run = b.step_sequential
                else:
                    def run(b=b):
                        b.step(graph=True)
                for _ in range(warmup):
                    run()
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(steps):
                    run()
                e1.record()
                torch.cuda.synchronize()
                acc_ms[mode] += e0.elapsed_time(e1) / steps
                b.status()
                infos.setdefault(mode, []).append(b.info())
                b.close()
            del insts
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
        for mode, ms in acc_ms.items():
            gbs = nbytes / (ms * 1e-3) / 1e9
            launches = {"fused": 1, "phased": 4, "sequential": 5 * len(shapes) // len(groups)}
            res["modes"][mode] = {"ms_per_step": ms, "particles_per_s": n_total / (ms * 1e-3),
                                  "gbs": gbs, "frac_hbm": gbs / peak["hbm_gbs"],
                                  "launches_per_step": launches[mode] * len(groups),
                                  "grid_blocks": [i["grid_blocks"] for i in infos[mode]],
                                  "smem_bytes": [i["smem_bytes"] for i in infos[mode]]}
        seq = res["modes"]["sequential"]["ms_per_step"]
        for mode in ("fused", "phased"):
            res["modes"][mode]["speedup_vs_sequential"] = seq / res["modes"][mode]["ms_per_step"]
        res["tuned"] = {k: v for k, v in tuner.table.items() if ("f32" if f32 else "f64") in k}
        res["tuned_classes"] = len(res["tuned"])
        out[form] = res
    return out, tuner.measurements


def run_batch_leg(args, peak):
    """Bounded batched leg of the default run: the batch configuration's
    instance distribution with fewer instances."""
    shapes = batch_shapes(args.batch_leg_instances, args.batch_seed)
    forms, meas = batch_measure(shapes, ["fp32", "fp64"], max(3, min(args.steps, 5)),
                                max(1, args.warmup), peak, args.batch_max_tile_bins)
    return {"workload": "%d independent APIC instances, edge uniform in {16,24,...,96}, 1-16 "
                        "ppc, order 2 or 3 per instance, uniform positions, autotuned tile / "
                        "chunk / lanes; fused = one persistent launch per step, phased = one "
                        "per phase, both replayed from a CUDA graph; sequential = single "
                        "launches instance after instance" % len(shapes),
            "instances": len(shapes), "particles": sum(e ** 3 * p for e, p, _ in shapes),
            "forms": forms, "autotune_measurements": meas}


def run_batch(args):
    import torch

    torch.cuda.set_device(0)
    peak = peaks()
    shapes = batch_shapes(args.batch_instances, args.batch_seed)
    out = {"metric": BATCH_METRIC, "unit": "particles/s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "higher_is_better": True, "data": "synthetic",
           "config": {"workload": "%d independent APIC instances, edge uniform in "
                                  "{16,24,...,96}, 1-16 ppc, order 2 or 3 per instance, uniform "
                                  "positions" % len(shapes),
                      "instances": len(shapes), "seed": args.batch_seed,
                      "particles": sum(e ** 3 * p for e, p, _ in shapes),
                      "nodes": sum(e ** 3 for e, _, _ in shapes),
                      "quadratic": sum(1 for s in shapes if s[2] == 2),
                      "cubic": sum(1 for s in shapes if s[2] == 3),
                      "l2": "inputs >> 126 MB L2 (no flush needed)"}}
    clocks = Clocks(0)
    clocks.start()
    out["forms"], meas = batch_measure(shapes, args.batch_forms.split(","), args.steps,
                                       args.warmup, peak, args.batch_max_tile_bins)
    out["clocks"] = clocks.stop()
    best = out["forms"].get("fp32", next(iter(out["forms"].values())))
    out["value"] = best["modes"]["fused"]["particles_per_s"]
    out["ms_per_step"] = best["modes"]["fused"]["ms_per_step"]
    out["dtype"] = "f32 (i64 fixed-point grid)" if "fp32" in out["forms"] else "f64"
    out["roofline"] = {"bound": "hbm", "achieved": best["modes"]["fused"]["gbs"],
                       "peak": peak["hbm_gbs"], "unit": "GB/s",
                       "frac": best["modes"]["fused"]["frac_hbm"],
                       "peak_source": peak["source"], "traffic": None}
    out["autotune_measurements"] = meas
    line = json.dumps(out)
    print(line)
    if args.json_out:
        with open(args.json_out, "w") as f:
            f.write(line + "\n")


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.suite == "batch":
        run_batch(args)
    elif args.suite in ("advect", "polypic"):
        run_leg_alone(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
