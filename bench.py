"""Benchmark: 256^3 projections per second (one GPU per rank, independent grids: weak scaling).

One step = one projection of a 256^3 MAC velocity field with 4 seeded random spheres
(radii U(0.05, 0.15)): b = -div(a u) -> fractional multigrid to ||r||/||f|| <= 1e-10 (FP32 V-cycles
inside FP64 iterative refinement, trilinear prolongation, V(2,2), omega 2/3) -> u <- a (u - grad p)
-> max|div| -> wavelet potential recovery (9 forward passes, local projection, 9 inverse passes).
The inputs of every step are restored from a device copy inside the step (3 D2D copies, 0.2 GB).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 256]

Prints one JSON line (rank 0).  `--impl reference` times the reference algorithm's CPU
implementation (the FP64 oracle restatement; the reference has no CPU code of its own) on a
bounded sample per step, extrapolated to one full projection.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def make_problem(n, seed):
    """Seeded inputs (cached in the temp directory: the spectral generator takes ~10 s at 256^3)."""
    import tempfile
    from waveletpotentials_b200 import fields
    centers, radii = fields.random_spheres(4, 0.05, 0.15, seed + 1000)
    path = os.path.join(tempfile.gettempdir(), f"wp_bench_fields_{n}_{seed}.npz")
    if os.path.exists(path):
        d = np.load(path)
        return centers, radii, (d["xv"], d["yv"], d["zv"])
    xv, yv, zv = fields.velocity3d((n, n, n), seed, dtype=np.float32)
    try:
        np.savez(path, xv=xv, yv=yv, zv=zv)
    except OSError:
        pass
    return centers, radii, (xv, yv, zv)


def ncu_traffic(kernel, n):
    """DRAM bytes (read + write) per launch of `kernel` at n^3 from the ncu captures summarised in
    profiles/ncu_traffic.json, or (None, reason).  A capture counts only while the CUDA sources are
    the ones it was taken from (their SHA-256 is stored with it); otherwise the figure is stale."""
    import hashlib
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None, "no capture"
    rec = json.load(open(path)).get(f"{kernel}@{n}")
    if not rec:
        return None, "no capture of this kernel at this size"
    h = hashlib.sha256()
    csrc = os.path.join(ROOT, "waveletpotentials_b200", "csrc")
    for f in sorted(os.listdir(csrc)):
        if f.endswith((".cu", ".cuh")):
            h.update(open(os.path.join(csrc, f), "rb").read())
    if rec.get("csrc_sha256") != h.hexdigest():
        return None, "capture predates the current kernel sources"
    return int(rec["dram_bytes_per_launch"]), rec["source"]


def max_over_ranks(values, world):
    """Element-wise max of per-rank timings (device-timed ms) over all ranks; the tensor lives on
    the current CUDA device under NCCL and on the host under gloo."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(v) for v in values], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu().tolist()]


def throughput(world, units_per_rank, ms):
    """Whole-job rate: the units all ranks processed over the slowest rank's device time."""
    return world * units_per_rank / (ms / 1000.0)


def rank_seed(seed, rank):
    """Each rank projects its own independent seeded problem (weak scaling, no data-path collective)."""
    return seed + rank


# --------------------------------------------------------------------------------- our arm
def run_ours(args, rank, world, local_rank):
    import torch
    from waveletpotentials_b200 import api, build, _lib
    build.build()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.n
    nn = (n, n, n)
    h = 1.0 / n
    centers, radii, (xv, yv, zv) = make_problem(n, rank_seed(args.seed, rank))
    s = api.mac_shapes3d(*nn)
    sls = api.CuSolidLevelSet3D(nn, h)
    sls.InitLsSpheres(centers, radii)
    a = [torch.empty(s[k], device=dev) for k in ("xv", "yv", "zv")]
    sls.GetFrac(*a)
    u0 = [torch.as_tensor(x, device=dev) for x in (xv, yv, zv)]
    u = [x.clone() for x in u0]
    q = [torch.zeros(s[k], device=dev) for k in ("qx", "qy", "qz")]
    start = api.START_FMG if args.start == "fmg" else api.START_ZERO
    proj = api.Projector3D(*a, nn, h, rel_tol=args.tol, max_cycles=80, nu1=2, nu2=2, weight=2.0 / 3.0,
                           precision=api.PREC_MIXED, prolongation=api.PROLONG_TRILINEAR, start=start,
                           host_loop=args.host_loop, inner_cycles=args.inner_cycles)
    if args.launch_by_launch:
        proj.mg.SetTile(0, 3, 0, 0)
    if args.pin_jacobi >= 0:
        zc = proj.mg.Tiles()[0][0]
        proj.mg.SetTile(0, 0, zc, args.pin_jacobi)
    stream = torch.cuda.current_stream()

    def step():
        for d, src in zip(u, u0):
            d.copy_(src, non_blocking=True)
        return proj.run(*u, *q)

    for _ in range(args.warmup):
        rep = step()
    L = _lib.lib()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    L.wp_profile_reset()  # counts launches; per-kernel events stay off in the timed region
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = []
    with ClockSampler(local_rank) as clk:
        if args.profile_region:
            torch.cuda.profiler.start()
        e0.record(stream)
        for _ in range(args.steps):
            reps.append(step())
        e1.record(stream)
        torch.cuda.synchronize()
        if args.profile_region:
            torch.cuda.profiler.stop()
    ms = e0.elapsed_time(e1)
    launches = int(L.wp_launch_count())
    # a second timed region with CUDA events around every kernel: the per-kernel table and roofline
    psteps = max(3, args.steps // 5)
    L.wp_profile_reset()
    L.wp_profile_enable(1)
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _ in range(psteps):
        step()
    g1.record(stream)
    torch.cuda.synchronize()
    L.wp_profile_enable(0)
    prof_ms = g0.elapsed_time(g1) / psteps
    ncls = L.wp_profile_collect()
    prof = []
    import ctypes
    for i in range(ncls):
        name = ctypes.create_string_buffer(64)
        lc, t, b = ctypes.c_longlong(), ctypes.c_double(), ctypes.c_double()
        L.wp_profile_entry(i, name, 64, ctypes.byref(lc), ctypes.byref(t), ctypes.byref(b))
        prof.append({"kernel": name.value.decode(), "launches": lc.value, "ms": t.value, "bytes": b.value})
    prof.sort(key=lambda r: -r["ms"])
    ms, = max_over_ranks([ms], world)
    # the last step's outputs (every step projects the same input) and the initial divergence, for
    # the host-side checks against the oracle
    b0 = torch.empty(s["p"], device=dev)
    api.CuConvergence.GetB_3d_frac_vel(b0, *u0, *a, nn, h)
    outputs = {"u": [x.double().cpu().numpy() for x in u], "q": [x.double().cpu().numpy() for x in q],
               "u0": [np.asarray(x, np.float64) for x in (xv, yv, zv)],
               "p64": proj.mg.Iterate64(), "a": [x.double().cpu().numpy() for x in a],
               "max_abs_b0": api.max_abs(b0)}

    # end to end through the public API with host buffers: every step copies its pinned host velocity
    # in and its potential q out; HostPipeline3D overlaps those copies with the neighbouring steps'
    # projections (two device buffer sets, one copy stream per direction)
    host_u = [torch.from_numpy(x).pin_memory() for x in (xv, yv, zv)]
    host_q = [torch.empty(s[k], dtype=torch.float32).pin_memory() for k in ("qx", "qy", "qz")]
    pipe = api.HostPipeline3D(proj)
    h2d, d2h = pipe.h2d_bytes, pipe.d2h_bytes
    pipe.run([host_u], [host_q])
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    # as many steps as the device-timed region, so the first copy in and the last copy out (the only
    # ones no projection overlaps) weigh the same as there
    ek = max(2, args.steps)
    f0 = torch.cuda.Event(enable_timing=True)
    f0.record(pipe.comp)
    pipe.run([host_u] * ek, [host_q] * ek)
    torch.cuda.synchronize()
    ems = f0.elapsed_time(pipe.last_out)
    ems, = max_over_ranks([ems], world)

    # plain path: FP64 V-cycles throughout to the same tolerance (no mixed precision)
    plain = None
    if args.plain_steps > 0:
        proj64 = api.Projector3D(*a, nn, h, rel_tol=args.tol, max_cycles=80, nu1=2, nu2=2, weight=2.0 / 3.0,
                                 precision=api.PREC_FP64, prolongation=api.PROLONG_TRILINEAR)
        for d, src in zip(u, u0):
            d.copy_(src)
        proj64.run(*u, *q)
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        preps = []
        for _ in range(args.plain_steps):
            for d, src in zip(u, u0):
                d.copy_(src, non_blocking=True)
            preps.append(proj64.run(*u, *q))
        g1.record(stream)
        torch.cuda.synchronize()
        pms = g0.elapsed_time(g1) / args.plain_steps
        plain = {"precision": "fp64", "start": "zero", "ms_per_projection": pms, "projections_per_s": 1000.0 / pms,
                 "vcycles": preps[-1]["cycles"], "max_abs_div": preps[-1]["max_abs_div"],
                 "rel_residual": preps[-1]["rel_residual"]}
        def time_variant(pr):
            for d, src in zip(u, u0):
                d.copy_(src)
            pr.run(*u, *q)
            torch.cuda.synchronize()
            g0.record(stream)
            vreps = []
            for _ in range(args.plain_steps):
                for d, src in zip(u, u0):
                    d.copy_(src, non_blocking=True)
                vreps.append(pr.run(*u, *q))
            g1.record(stream)
            torch.cuda.synchronize()
            vms = g0.elapsed_time(g1) / args.plain_steps
            return {"ms_per_projection": vms, "projections_per_s": 1000.0 / vms, "vcycles": vreps[-1]["cycles"],
                    "rel_residual": vreps[-1]["rel_residual"]}

        mixed = dict(rel_tol=args.tol, max_cycles=80, nu1=2, nu2=2, weight=2.0 / 3.0, precision=api.PREC_MIXED,
                     prolongation=api.PROLONG_TRILINEAR)
        # the same mixed-precision solve with the other first cycle (zero start <-> full multigrid), and
        # with the convergence test on the host after every cycle instead of the device-side loop
        other = api.START_ZERO if start == api.START_FMG else api.START_FMG
        plain["mixed_" + ("zero" if other == api.START_ZERO else "fmg") + "_start"] = time_variant(
            api.Projector3D(*a, nn, h, start=other, **mixed))
        plain["mixed_host_loop"] = time_variant(api.Projector3D(*a, nn, h, start=start, host_loop=True, **mixed))
        # the recovery stage alone: the wavelet recovery against the reference's comparison baseline,
        # sweep + DST-I (CuParallelSweep3D Solve + Project), on the same projected velocity
        for d, src in zip(u, u0):
            d.copy_(src)
        proj.run(*u, *q)
        sw = api.CuParallelSweep3D(nn, h, "n")
        qs = [torch.empty_like(t) for t in q]

        def time_rec(fn, k=5):
            fn()
            torch.cuda.synchronize()
            g0.record(stream)
            for _ in range(k):
                fn()
            g1.record(stream)
            torch.cuda.synchronize()
            return g0.elapsed_time(g1) / k

        plain["recovery"] = {
            "wavelet_ms": time_rec(lambda: proj.rec.Solve(*q, *u)),
            "sweep_dst_ms": time_rec(lambda: (sw.Solve(*qs, *u), sw.Project(*qs))),
            # CuWaveletPotentialRecover3D::CutCoefficients of the recovered potential at level 2
            "cut_level2_ms": time_rec(lambda: proj.rec.CutCoefficients(*qs, *q, 2)),
        }
        # face fractions of the same spheres' level set by the static CuSolidLevelSet3D::GetFrac
        # (cut faces sub-sampled 128 x 128) against the two-point formula the projection uses
        fa = [torch.empty_like(t) for t in a]
        plain["fractions"] = {
            "subsampled_ms": time_rec(lambda: sls.GetFrac(*fa, ls=sls.ls, dim=nn, dx=h), k=3),
            "two_point_ms": time_rec(lambda: sls.GetFrac(*fa), k=3),
        }
        sw.close()
        # the index-sparse cycle (CuMultigridFrac3D::Solve_index) against the dense reference cycle
        # (CuMultigridFrac3D::Solve) on a mostly-solid domain of the same extent: balls of fluid
        # filling 15% of the cells, four V(2,2) cycles, omega 0.8 (the reference's defaults)
        from waveletpotentials_b200 import fields as wf
        fl, fa, frng = wf.porous_domain(nn, 0.15, args.seed)
        tff = torch.as_tensor(frng.standard_normal(fl.shape) * fl, dtype=torch.float32, device=dev)
        mgp = api.CuMultigridFrac3D(*(torch.as_tensor(x, dtype=torch.float32, device=dev) for x in fa), nn, h)
        dp = torch.zeros_like(tff)
        cells, _ = mgp.IndexSizes()
        plain["index_sparse"] = {
            "workload": f"{n}^3 cells, {fl.mean():.3f} fluid (balls in a solid block), 4 V(2,2) cycles, omega 0.8",
            "listed_cells": [int(c) for c in cells],
            "index_ms_per_cycle": time_rec(lambda: mgp.Solve_index(dp, None, tff, 4, 2, 2, 0.8)) / 4,
            "dense_ms_per_cycle": time_rec(lambda: mgp.Solve(dp, None, tff, 4, 2, 2, 0.8)) / 4,
        }
        mgp.close()
    tiles = proj.mg.Tiles(with_times=True)
    return ms, ems, ek, h2d, d2h, launches, prof, reps, clk.summary(), plain, (tiles, psteps, prof_ms, outputs)


# ------------------------------------------------------------------ batched workload
BATCH_3D = (32, 64, 128)
BATCH_2D = (256, 512, 1024)
# the small-grid mix (--batch-sizes small): the same counts, every grid a few V-cycles of kernels
# that each run for a few microseconds
BATCH_3D_SMALL = (16, 32)
BATCH_2D_SMALL = (64, 128)


def make_batch(count3, count2, seed, small=False):
    """Seeded uneven batch: 3D cubes drawn from {32,64,128}^3 and 2D squares from {256,512,1024}^2
    ({16,32}^3 and {64,128}^2 when small), each with 0-4 random spheres/circles r~U(0.05,0.15) and
    its own field seed."""
    import tempfile
    from waveletpotentials_b200 import fields
    rng = np.random.default_rng(seed + 77)
    specs = []
    sizes3, sizes2 = (BATCH_3D_SMALL, BATCH_2D_SMALL) if small else (BATCH_3D, BATCH_2D)
    for i in range(count3 + count2):
        d3 = i < count3
        n = int(rng.choice(sizes3 if d3 else sizes2))
        nsph = int(rng.integers(0, 5))
        specs.append(((n, n, n) if d3 else (n, n), nsph, seed * 1000 + i))
    path = os.path.join(tempfile.gettempdir(),
                        f"wp_bench_batch_{count3}_{count2}_{seed}{'_small' if small else ''}.npz")
    cache = dict(np.load(path)) if os.path.exists(path) else {}
    out, dirty = [], False
    for i, (d, nsph, sd) in enumerate(specs):
        c, r = fields.random_spheres(nsph, 0.05, 0.15, sd)
        keys = [f"g{i}_{k}" for k in ("xv", "yv", "zv")[:len(d)]]
        if all(k in cache for k in keys):
            u = [cache[k] for k in keys]
        else:
            u = list(fields.velocity3d(d, sd, dtype=np.float32) if len(d) == 3 else
                     fields.velocity2d(d, sd, dtype=np.float32))
            cache.update(dict(zip(keys, u)))
            dirty = True
        out.append((d, c, r, u))
    if dirty:
        try:
            np.savez(path, **cache)
        except OSError:
            pass
    return out


def run_batch(args, rank, world, local_rank):
    import ctypes
    import torch
    from waveletpotentials_b200 import api, build, _lib
    build.build()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    probs = make_batch(args.batch3d, args.batch2d, rank_seed(args.seed, rank), small=args.batch_sizes == "small")
    grids, u0, outs = [], [], []
    for d, c, r, u in probs:
        h = 1.0 / d[0]
        if len(d) == 3:
            s = api.mac_shapes3d(*d)
            sls = api.CuSolidLevelSet3D(d, h)
            sls.InitLsSpheres(c, r)
            a = [torch.empty(s[k], device=dev) for k in ("xv", "yv", "zv")]
            sls.GetFrac(*a)
            grids.append({"dim": d, "dx": h, "ax": a[0], "ay": a[1], "az": a[2]})
            outs.append([torch.zeros(s[k], device=dev) for k in ("qx", "qy", "qz")])
        else:
            s = api.mac_shapes2d(*d)
            sls = api.CuSolidLevelSet2D(d, h)
            sls.InitLsCircles(np.reshape(c, (-1, 3))[:, :2], r)
            a = [torch.empty(s[k], device=dev) for k in ("xv", "yv")]
            sls.GetFrac(*a)
            grids.append({"dim": d, "dx": h, "ax": a[0], "ay": a[1]})
            outs.append([torch.zeros(s["qz"], device=dev)])
        u0.append([torch.as_tensor(x, device=dev) for x in u])
    u = [[x.clone() for x in f] for f in u0]
    want = {"graph": api.BATCH_GRAPH, "persistent": api.BATCH_PERSISTENT, "auto": api.BATCH_AUTO}[args.batch_mode]
    bp = api.BatchProjector(grids, rel_tol=args.batch_tol, max_cycles=80, nstreams=args.nstreams,
                            tile_cells=args.batch_tile, mode=want)
    cycles = bp.plan(u)
    mode_info = bp.get_mode()
    # the way the timed region runs the solves (auto: the plan's choice)
    persistent = mode_info[0] == api.BATCH_PERSISTENT
    stream = torch.cuda.current_stream()
    count = len(grids)

    def restore():
        for f, f0 in zip(u, u0):
            for d, src in zip(f, f0):
                d.copy_(src, non_blocking=True)

    def step():
        restore()
        bp.run(u, outs)

    for _ in range(args.warmup):
        step()
    L = _lib.lib()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    L.wp_profile_reset()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        if args.profile_region:
            torch.cuda.profiler.start()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        if args.profile_region:
            torch.cuda.profiler.stop()
    ms = e0.elapsed_time(e1)
    # kernels of the graph outside the solve loops (counted per replay), then the loop bodies: those
    # are counted when the results are read (the number of passes is known on the device only), once
    # for the last replay; every timed replay ran the same input, so each ran as many passes
    launches = int(L.wp_launch_count())
    res = bp.results()
    launches += (int(L.wp_launch_count()) - launches) * (args.steps - 1)
    # persistent mode: where the persistent kernel's CTAs spend their cycles over one more run
    prof = None
    if persistent:
        bp.profile(True)
        step()
        torch.cuda.synchronize()
        pr = bp.profile(False)
        tot = pr["wait_cycles"] + pr["setup_cycles"] + pr["complete_cycles"] + sum(
            pr[k]["cycles"] for k in api.BatchProjector.PROFILE_NAMES)
        prof = {"cta_cycles": tot, "tiles": pr["tiles"],
                "share": {"waiting_for_work": pr["wait_cycles"] / tot, "setup": pr["setup_cycles"] / tot,
                          "complete_publish": pr["complete_cycles"] / tot,
                          **{k: pr[k]["cycles"] / tot for k in api.BatchProjector.PROFILE_NAMES}},
                "cycles_per_tile": {k: (pr[k]["cycles"] / pr[k]["tiles"] if pr[k]["tiles"] else 0.0)
                                    for k in api.BatchProjector.PROFILE_NAMES},
                "tiles_by_type": {k: pr[k]["tiles"] for k in api.BatchProjector.PROFILE_NAMES}}
    # the other way of running the solves, same grids and inputs, for comparison
    other = api.BATCH_GRAPH if persistent else api.BATCH_PERSISTENT
    bp.set_mode(other, args.batch_tile)
    if not persistent:
        bp.plan(u)  # orders the programs and, with --batch-tile 0, tunes the persistent tile
    pers_mode = bp.get_mode() if not persistent else None
    for _ in range(2):
        step()
    torch.cuda.synchronize()
    o0, o1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    o0.record(stream)
    for _ in range(args.steps):
        step()
    o1.record(stream)
    torch.cuda.synchronize()
    other_ms = o0.elapsed_time(o1) / args.steps
    ores = bp.results()
    # back to the timed mode (the persistent tile the plan chose, when it chose one)
    bp.set_mode(api.BATCH_PERSISTENT if persistent else api.BATCH_GRAPH, mode_info[1] if persistent else 0)
    # the same grids projected one after another through the one-grid path (eager launches)
    projs = []
    for g in grids:
        if len(g["dim"]) == 3:
            projs.append(api.Projector3D(g["ax"], g["ay"], g["az"], g["dim"], g["dx"], rel_tol=args.batch_tol,
                                         max_cycles=80))
        else:
            projs.append(api.Projector2D(g["ax"], g["ay"], g["dim"], g["dx"], rel_tol=args.batch_tol, max_cycles=80))

    def seq_step():
        restore()
        for i, p in enumerate(projs):
            p.run(*u[i], *outs[i])

    seq_step()
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _ in range(2):
        seq_step()
    g1.record(stream)
    torch.cuda.synchronize()
    seq_ms = g0.elapsed_time(g1) / 2
    # end to end: pinned host velocities in, potentials out, around each batched run
    host_u = [[torch.from_numpy(np.ascontiguousarray(x)).pin_memory() for x in p[3]] for p in probs]
    host_q = [[torch.empty(t.shape, dtype=torch.float32).pin_memory() for t in o] for o in outs]
    h2d = sum(x.numel() * 4 for f in host_u for x in f)
    d2h = sum(x.numel() * 4 for f in host_q for x in f)

    def e2e_step():
        for f, hf in zip(u, host_u):
            for d, src in zip(f, hf):
                d.copy_(src, non_blocking=True)
        bp.run(u, outs)
        for hq, q in zip(host_q, outs):
            for d, src in zip(hq, q):
                d.copy_(src, non_blocking=True)

    e2e_step()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ek = max(1, min(args.steps, 5))
    f0.record(stream)
    for _ in range(ek):
        e2e_step()
    f1.record(stream)
    torch.cuda.synchronize()
    ems = f0.elapsed_time(f1)
    cells = sum(int(np.prod(g["dim"])) for g in grids)
    info = {"grids": count, "grids_3d": args.batch3d, "grids_2d": args.batch2d, "cells": cells,
            "cycles_min": min(res["cycles"]), "cycles_max": max(res["cycles"]), "nstreams": args.nstreams,
            "mode": args.batch_mode,
            "mode_run": "persistent" if persistent else "graph",
            "auto_graph_solve_ms": mode_info[3] if args.batch_mode == "auto" else None,
            "solves": ("one persistent kernel over a device work queue of (grid, level, pass) tiles, "
                       f"{args.batch_tile or 32768} cells per tile" if persistent else
                       "a device loop of launches per grid (while-node) on the graph's branches"),
            "cycles_per_grid": "each replay's stopping rule runs on the device: it stops at the tolerance",
            "ms_per_batch": ms / args.steps, "sequential_eager_ms_per_batch": seq_ms,
            "speedup_vs_sequential": seq_ms / (ms / args.steps),
            ("graph_ms_per_batch" if persistent else "persistent_ms_per_batch"): other_ms,
            "other_mode_same_cycles": ores["cycles"] == res["cycles"],
            "persistent_profile": prof,
            "persistent_tile": (pers_mode if pers_mode else mode_info)[1],
            "persistent_tile_tuning_ms": dict(zip([str(c) for c in api.BatchProjector.TILE_CANDIDATES],
                                                  (pers_mode if pers_mode else mode_info)[2])),
            "max_rel_residual": max(res["rel_residual"]), "max_abs_div": max(res["max_abs_div"])}
    return ms, ems, ek, h2d, d2h, launches, clk.summary(), info, count


# ------------------------------------------------------------------ learned warm start
def run_warmstart(args, rank, world, local_rank):
    """Trains the warm-start U-Net on solves of the plain method at n^3 (1-8 spheres/boxes), then
    times projections to 1e-6 with and without the warm start on held-out problems."""
    import torch
    from waveletpotentials_b200 import api, build, trainer, _lib
    build.build()
    torch.cuda.set_device(local_rank)
    n = args.ws_n
    dim = (n, n, n)
    t0 = time.perf_counter()
    train = trainer.make_dataset(dim, args.ws_train, seed=rank_seed(args.seed, rank) * 7 + 1, tol=1e-6)
    held = trainer.make_dataset(dim, args.ws_eval, seed=10 ** 6 + rank, tol=1e-6)
    gen_s = time.perf_counter() - t0
    net = api.UNetWarmStart(dim, seed=args.seed)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = trainer.train(net, train, steps=args.ws_steps, lr=args.ws_lr, lr_end=args.ws_lr * 0.1)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream()
    s = api.mac_shapes3d(*dim)
    q = [torch.zeros(s[k], device="cuda") for k in ("qx", "qy", "qz")]
    rows = []
    for smp in held:
        projs = {"plain": api.Projector3D(*smp["a"], dim, smp["h"], rel_tol=1e-6, max_cycles=60),
                 "warm": api.Projector3D(*smp["a"], dim, smp["h"], rel_tol=1e-6, max_cycles=60, warm_start=net,
                                         sdf=smp["sdf"])}
        row = {}
        for name, pr in projs.items():
            u = [x.clone() for x in smp["u"]]
            pr.run(*u, *q)  # warm-up
            reps, ms = [], []
            for _ in range(args.steps):
                for d, src in zip(u, smp["u"]):
                    d.copy_(src)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                reps.append(pr.run(*u, *q))
                e1.record(stream)
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
            row[name] = {"ms": float(np.median(ms)), "cycles": reps[-1]["cycles"],
                         "max_abs_div": reps[-1]["max_abs_div"], "rel_residual": reps[-1]["rel_residual"]}
            if name == "warm":
                row[name]["used"] = reps[-1]["warm_start"]["used"]
                row[name]["first_cycle_rel_residual"] = reps[-1]["warm_start"]["first_cycle_rel_residual"]
            else:
                row[name]["first_cycle_rel_residual"] = reps[-1]["history"][0]
        rows.append(row)
    # network inference alone
    guess = torch.empty(s["p"], device="cuda")
    smp = held[0]
    net.predict(guess, smp["b"], smp["sdf"], smp["h"])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(5):
        net.predict(guess, smp["b"], smp["sdf"], smp["h"])
    e1.record(stream)
    torch.cuda.synchronize()
    infer_ms = e0.elapsed_time(e1) / 5
    plain_ms = float(np.mean([r["plain"]["ms"] for r in rows]))
    warm_ms = float(np.mean([r["warm"]["ms"] for r in rows]))
    out = {"metric": f"{n}^3 projections/s with the learned warm start (plain mixed-precision path beside it)",
           "value": 1000.0 / warm_ms, "unit": "projections/s", "n_gpus": 1, "steps": args.steps, "warmup": 1,
           "ms_per_step": warm_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "bf16 network (FP32 accumulate) + f32/f64 multigrid", "data": "synthetic (device generator)",
           "config": {"workload": f"{n}^3, 1-8 random spheres/boxes U(0.05,0.2), rel. residual 1e-6, U-Net "
                                  f"16/32/64 trained on {args.ws_train} plain solves x {args.ws_steps} Adam steps"},
           "warm_start": {"plain_ms": plain_ms, "warm_ms": warm_ms, "speedup": plain_ms / warm_ms,
                          "plain_cycles": float(np.mean([r["plain"]["cycles"] for r in rows])),
                          "warm_cycles": float(np.mean([r["warm"]["cycles"] for r in rows])),
                          "fallback_rate": float(np.mean([0.0 if r["warm"]["used"] else 1.0 for r in rows])),
                          "first_cycle_rel_residual_warm":
                              float(np.mean([r["warm"]["first_cycle_rel_residual"] for r in rows])),
                          "first_cycle_rel_residual_plain":
                              float(np.mean([r["plain"]["first_cycle_rel_residual"] for r in rows])),
                          "inference_ms": infer_ms, "train_s": train_s, "data_gen_s": gen_s,
                          "loss_first": float(np.mean(losses[:10])), "loss_last": float(np.mean(losses[-50:])),
                          "params": int(net.params(0).size)},
           "samples": rows}
    return out


# ------------------------------------------------------------------ convolution kernels
def run_conv(args):
    """The warm-start network's tensor-core 3x3x3 convolutions (forward and weight gradient) on one
    channels-last BF16 volume of conv_n^3 x conv_c: CUDA-event time and TFLOP/s
    (2 * 27 * c * c * n^3 flops); a profiling aid for the tcgen05 kernels."""
    import torch
    from waveletpotentials_b200 import api, build
    build.build()
    n, c = args.conv_n, args.conv_c
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn((n, n, n, c), device="cuda", generator=g).to(torch.bfloat16)
    w = (torch.randn((27, c, c), device="cuda", generator=g) * 0.05).to(torch.bfloat16)
    out = torch.empty_like(x)
    dw = torch.zeros((27, c, c), device="cuda")
    for _ in range(3):
        api.conv3_forward(out, x, w)
        api.conv3_wgrad(dw, x, out)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    if args.profile_region:
        torch.cuda.profiler.start()
    ev[0].record(st)
    for _ in range(args.conv_reps):
        api.conv3_forward(out, x, w)
    ev[1].record(st)
    for _ in range(args.conv_reps):
        api.conv3_wgrad(dw, x, out)
    ev[2].record(st)
    torch.cuda.synchronize()
    if args.profile_region:
        torch.cuda.profiler.stop()
    fl = 2.0 * 27 * c * c * n ** 3
    res = {}
    for name, t in (("conv3_forward", ev[0].elapsed_time(ev[1]) / args.conv_reps),
                    ("conv3_wgrad", ev[1].elapsed_time(ev[2]) / args.conv_reps)):
        res[name] = {"ms": t, "tflops": fl / t / 1e9}
    print(json.dumps({"workload": "conv", "n": n, "c": c, "kernels": res}))


# --------------------------------------------------------------------------- CPU arm
def cpu_inputs(n, seed, fractions=None):
    """The benchmark's inputs on the host in FP64: velocity (the FP32 values), face fractions (the
    GPU's FP32 ones when given, else the oracle's)."""
    from oracle import oracle as O
    O.build()
    nn = (n, n, n)
    h = 1.0 / n
    centers, radii, (xv, yv, zv) = make_problem(n, seed)
    if fractions is None:
        sdf = O.sdf_spheres3d(nn, h, centers, radii)
        fractions = O.fractions3d(sdf, nn, h)
    u = [np.asarray(x, np.float64) for x in (xv, yv, zv)]
    a = [np.asarray(x, np.float64) for x in fractions]
    return nn, h, u, a


def cpu_projection(n, seed, ncycles, fractions=None):
    """One whole projection with the FP64 oracle on the host cores (the same composition as a GPU
    step): divergence, its mean over the active cells removed, ncycles trilinear V(2,2) cycles,
    omega 2/3, from zero, the gradient update and the wavelet recovery.  Returns the wall times per
    stage and the fields."""
    from oracle import oracle as O
    nn, h, u, a = cpu_inputs(n, seed, fractions)
    d = (h,) * 3
    t0 = time.perf_counter()
    f = O.divergence3d(*u, *a, nn, d)
    act = cpu_active(a)
    f[act] -= f[act].mean()
    t1 = time.perf_counter()
    p, hist = O.mgfrac3d_solve(f, *a, nn, d, ncycles, 2, 2, 2.0 / 3.0, prolong=O.PROLONG_TRILINEAR)
    t2 = time.perf_counter()
    uu = O.grad_subtract3d(*u, p, *a, nn, d, True)
    t3 = time.perf_counter()
    q = O.recover3d(*uu, nn, d)
    t4 = time.perf_counter()
    return {"divergence_s": t1 - t0, "mg_s": t2 - t1, "gradient_s": t3 - t2, "recovery_s": t4 - t3,
            "total_s": t4 - t0, "rel_residual": float(hist[-1]), "p": p, "u": uu, "q": q, "act": act,
            "f": f, "a": a, "h": h}


def cpu_active(a):
    """cells with at least one open interior face (the Neumann problem's support)"""
    ax, ay, az = a
    act = np.zeros((ax.shape[0], ay.shape[1], ax.shape[2]), dtype=bool)
    act[:, :-1, :] |= ax[:, 1:-1, :] > 0
    act[:, 1:, :] |= ax[:, 1:-1, :] > 0
    act[:, :, :-1] |= ay[:, :, 1:-1] > 0
    act[:, :, 1:] |= ay[:, :, 1:-1] > 0
    act[:-1] |= az[1:-1] > 0
    act[1:] |= az[1:-1] > 0
    return act


def cpu_sample(n, seed, ncycles):
    """A bounded sample of the projection on the host cores with the FP64 oracle: the divergence,
    ONE trilinear V-cycle, the gradient update and the whole recovery at n^3.  Returns the sample's
    wall time and the projection time extrapolated to ncycles V-cycles."""
    from oracle import oracle as O
    nn, h, u, a = cpu_inputs(n, seed)
    d = (h,) * 3
    t0 = time.perf_counter()
    f = O.divergence3d(*u, *a, nn, d)
    t1 = time.perf_counter()
    p, _ = O.mgfrac3d_solve(f, *a, nn, d, 1, 2, 2, 2.0 / 3.0, prolong=O.PROLONG_TRILINEAR)
    t2 = time.perf_counter()
    uu = O.grad_subtract3d(*u, p, *a, nn, d, True)
    O.recover3d(*uu, nn, d)
    t3 = time.perf_counter()
    return t3 - t0, (t1 - t0) + ncycles * (t2 - t1) + (t3 - t2)


def rel_l2(ref, got):
    num = sum(float(np.sum((np.asarray(r, np.float64) - np.asarray(g, np.float64)) ** 2)) for r, g in zip(ref, got))
    den = sum(float(np.sum(np.asarray(r, np.float64) ** 2)) for r in ref)
    return float(np.sqrt(num / den))


def fp32_div_floor(u0, a, u, h):
    """The size of max|div| that FP32 rounding allows after the projection: the solver's right-hand
    side is the FP32 divergence of the input u0 (its rounding, 2^-24 x the cell's sum of |a u0| over
    its faces / h, cannot be projected out) and the projected u is stored in FP32 (2^-24 x its own
    sum of |face flux| / h); the largest per-cell sum of the two."""
    def fluxsum(v):
        vx, vy, vz = (np.abs(np.asarray(x, np.float64)) for x in v)
        return (vx[:, :-1, :] + vx[:, 1:, :]) + (vy[:, :, :-1] + vy[:, :, 1:]) + (vz[:-1] + vz[1:])
    au0 = [np.asarray(x, np.float64) * np.asarray(y, np.float64) for x, y in zip(u0, a)]
    return float(2.0 ** -24 * (fluxsum(au0) + fluxsum(u)).max() / h)


def cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=25)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--start", default="zero", choices=["fmg", "zero"],
                    help="first iterate of the mixed-precision solve: full-multigrid start or zero")
    ap.add_argument("--pin-jacobi", type=int, default=-1,
                    help="diagnostic: pin the finest-level Jacobi kernel variant (0-4) after autotuning")
    ap.add_argument("--inner-cycles", type=int, default=5,
                    help="FP32 V-cycles per refinement step of the mixed solve (5: the FP64 defect and the "
                         "tolerance test every fifth cycle; each step's FP32 correction solve then gains ~3e-3, "
                         "far inside FP32)")
    ap.add_argument("--launch-by-launch", action="store_true",
                    help="keep the levels below the finest launch by launch (the autotuner's choice at 256^3; under "
                         "ncu, whose serialised launches distort the timing, the autotuner would pick otherwise)")
    ap.add_argument("--host-loop", action="store_true",
                    help="test convergence on the host after every cycle instead of the device-side graph loop "
                         "(ncu does not profile kernels inside graphs with conditional nodes)")
    ap.add_argument("--profile-region", action="store_true",
                    help="bracket the timed steps with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    ap.add_argument("--conv-n", type=int, default=64)
    ap.add_argument("--conv-c", type=int, default=32)
    ap.add_argument("--conv-reps", type=int, default=10)
    ap.add_argument("--workload", default="single", choices=["single", "batch", "warmstart", "index", "conv"],
                    help="single: one 256^3 projection per step; batch: 64 uneven grids in one graph per step; "
                         "warmstart: train the U-Net, then projections with/without its guess; index: four "
                         "index-sparse V-cycles on a 15%%-fluid domain (profiling aid); conv: the tensor-core "
                         "convolutions alone (profiling aid)")
    ap.add_argument("--ws-n", type=int, default=128)
    ap.add_argument("--ws-train", type=int, default=128)
    ap.add_argument("--ws-eval", type=int, default=8)
    ap.add_argument("--ws-steps", type=int, default=3000)
    ap.add_argument("--ws-lr", type=float, default=2e-3)
    ap.add_argument("--batch3d", type=int, default=32)
    ap.add_argument("--batch2d", type=int, default=32)
    ap.add_argument("--batch-tol", type=float, default=1e-6)
    ap.add_argument("--batch-mode", default="graph", choices=["graph", "persistent", "auto"],
                    help="graph: each grid's solve a device loop of launches on a graph branch; persistent: every "
                         "grid's solve in one persistent kernel over a device work queue; auto: the plan times both "
                         "and the faster runs")
    ap.add_argument("--batch-tile", type=int, default=0,
                    help="persistent mode: cells per work-queue tile (0: the plan tunes it)")
    ap.add_argument("--batch-sizes", default="mixed", choices=["mixed", "small"],
                    help="mixed: 3D {32,64,128}^3 + 2D {256,512,1024}^2 (the configured batch); small: {16,32}^3 + "
                         "{64,128}^2")
    ap.add_argument("--nstreams", type=int, default=8)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    metric = "256^3 projections/s (mixed-precision path; plain path reported beside it) at max|div| of a 1e-10 solve"
    workload = {"workload": f"projection of a {args.n}^3 MAC field, 4 random spheres r~U(0.05,0.15), "
                            f"mixed-precision multigrid to rel. residual {args.tol:g} + wavelet potential recovery",
                "n": args.n, "spheres": 4, "rel_tol": args.tol, "mg": f"V(2,2) omega=2/3 trilinear, FP32 cycles + FP64 IR ({args.inner_cycles} "
                                                          f"cycle(s) per refinement step), {args.start} start",
                "l2_flush": "inputs larger than L2 (~1.3 GB working set per step)"}

    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import oracle as O
        O.build()
        ncyc = 20  # the V-cycles our arm needs for 1e-10 at this configuration
        vals = []
        for i in range(args.warmup + args.steps):
            sample_s, proj_s = cpu_sample(args.n, args.seed, ncyc)
            if i >= args.warmup:
                vals.append((sample_s, proj_s))
        proj_s = float(np.median([v[1] for v in vals]))
        sample_s = float(np.median([v[0] for v in vals]))
        value = 1.0 / proj_s
        sample = (f"each step: FP64 oracle at {args.n}^3 on {O.threads()} OpenMP threads, divergence + 1 trilinear "
                  f"V-cycle + gradient + full recovery ({sample_s:.2f} s); value extrapolated to {ncyc} V-cycles")
        out = {"impl": "reference", "metric": metric, "value": value, "unit": "projections/s", "n_gpus": 0,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": sample_s * 1000.0,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
               "data": "synthetic (seeded spectral fields)", "config": workload,
               "cpu_baseline": {"value": value, "unit": "projections/s", "cores": O.threads(), "kind": "port",
                                "extrapolated": True, "sample": sample},
               "e2e": {"value": value, "unit": "projections/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out))
        return

    if args.workload == "index" and args.impl == "ours":
        # the index-sparse cycle alone on the mostly-solid domain of plain["index_sparse"]: one
        # warm call, then one call of four V(2,2) cycles inside the profiler region (for ncu)
        import torch
        from waveletpotentials_b200 import api, fields as wf
        nn = (args.n,) * 3
        fl, fa, frng = wf.porous_domain(nn, 0.15, args.seed)
        tff = torch.as_tensor(frng.standard_normal(fl.shape) * fl, dtype=torch.float32, device="cuda")
        mgp = api.CuMultigridFrac3D(*(torch.as_tensor(x, dtype=torch.float32, device="cuda") for x in fa), nn,
                                    1.0 / args.n)
        dp = torch.zeros_like(tff)
        mgp.Solve_index(dp, None, tff, 4, 2, 2, 0.8)
        torch.cuda.synchronize()
        if args.profile_region:
            torch.cuda.cudart().cudaProfilerStart()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record()
        mgp.Solve_index(dp, None, tff, 4, 2, 2, 0.8)
        g1.record()
        torch.cuda.synchronize()
        if args.profile_region:
            torch.cuda.cudart().cudaProfilerStop()
        cells, segs = mgp.IndexSizes()
        print(json.dumps({"workload": "index", "n": args.n, "fluid": float(fl.mean()), "listed_cells": cells,
                          "segments": segs, "ms_per_cycle": g0.elapsed_time(g1) / 4}))
        return
    if args.workload == "conv" and args.impl == "ours":
        if rank == 0:
            run_conv(args)
        return
    if args.workload == "warmstart" and args.impl == "ours":
        if rank == 0:
            print(json.dumps(run_warmstart(args, rank, world, local_rank)))
        return

    if args.workload == "batch" and args.impl == "ours":
        if world > 1:
            import torch
            import datetime
            torch.cuda.set_device(local_rank)
            torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        ms, ems, ek, h2d, d2h, launches, clocks, info, count = run_batch(args, rank, world, local_rank)
        ms, ems = max_over_ranks([ms, ems], world)
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()
        if rank != 0:
            return
        small = args.batch_sizes == "small"
        s3 = "{16,32}" if small else "{32,64,128}"
        s2 = "{64,128}" if small else "{256,512,1024}"
        out = {"metric": "batched projections/s (64 uneven 2D/3D grids per CUDA-graph launch)",
               "value": throughput(world, count * args.steps, ms), "unit": "projections/s", "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 defect/refinement)",
               "data": "synthetic (seeded spectral fields)",
               "config": {"workload": f"{args.batch3d} 3D grids from {s3}^3 + {args.batch2d} 2D grids from "
                                      f"{s2}^2, 0-4 random spheres each, mixed-precision multigrid to "
                                      f"rel. residual {args.batch_tol:g} + wavelet recovery, one graph per batch",
                          "solves": args.batch_mode,
                          "l2_flush": ("inputs larger than L2 (batch working set > 1 GB)" if args.batch_sizes == "mixed"
                                       else "small grids: the batch's inputs fit L2; every timed step restores them "
                                            "from copies, and the step is launch- and latency-bound")},
               "e2e": {"value": throughput(world, count * ek, ems), "unit": "projections/s",
                       "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
               "gpu_launches": launches, "clocks": clocks, "batch": info}
        print(json.dumps(out))
        return

    if world > 1:
        import torch
        import datetime
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    ms, ems, ek, h2d, d2h, launches, prof, reps, clocks, plain, extra = run_ours(args, rank, world, local_rank)
    tiles, psteps, prof_ms = extra[:3]
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    value = throughput(world, args.steps, ms)
    hbm, peak_kind = peaks()
    top = prof[0] if prof else None
    roof = None
    if top and top["ms"] > 0:
        ach = top["bytes"] / (top["ms"] / 1000.0) / 1e9
        tr = ncu_traffic(top["kernel"], args.n)
        roof = {"bound": "hbm", "kernel": top["kernel"], "achieved": ach, "peak": hbm, "unit": "GB/s",
                "measured_over": f"{psteps} further timed steps with CUDA events around every kernel "
                                 f"({prof_ms:.2f} ms per step there)",
                "frac": ach / hbm, "peak_kind": peak_kind, "traffic": tr[0], "traffic_source": tr[1],
                "avg_launch_us": top["ms"] * 1000.0 / top["launches"],
                "bytes_per_launch": top["bytes"] / top["launches"]}
    cpu = parity = None
    ncyc = int(reps[-1]["cycles"])
    gout = extra[3]
    div = {"max_abs_div": reps[-1]["max_abs_div"], "max_abs_b0": gout["max_abs_b0"],
           "relative": reps[-1]["max_abs_div"] / gout["max_abs_b0"],
           "fp32_floor": fp32_div_floor(gout["u0"], gout["a"], gout["u"], 1.0 / args.n),
           "note": "max|div a(u - grad p)| of the FP32 projected field after the 1e-10 solve; fp32_floor: 2^-24 x the "
                   "largest per-cell sum of |a u0| (the FP32 right-hand side's rounding) and |u| (the FP32 storage) "
                   "over the cell's faces / h, what FP32 rounding alone leaves"}
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        nthr = O.threads()
        cp = cpu_projection(args.n, args.seed, ncyc, fractions=gout["a"])
        O.set_threads(1)
        s1, p1 = cpu_sample(args.n, args.seed, ncyc)
        O.set_threads(nthr)
        cpu = {"value": 1.0 / cp["total_s"], "unit": "projections/s", "cores": nthr, "kind": "port",
               "extrapolated": False,
               "sample": f"one whole projection at {args.n}^3 by the FP64 oracle on {nthr} OpenMP threads: divergence, "
                         f"{ncyc} trilinear V(2,2) cycles, gradient update, wavelet recovery ({cp['total_s']:.1f} s)",
               "stages_s": {k: round(cp[k], 3) for k in ("divergence_s", "mg_s", "gradient_s", "recovery_s")},
               "single_thread": {"value": 1.0 / p1, "unit": "projections/s", "cores": 1, "extrapolated": True,
                                 "sample": f"divergence + 1 V-cycle + gradient + recovery on one thread ({s1:.1f} s), "
                                           f"extrapolated to {ncyc} V-cycles"}}
        act = cp["act"]

        def no_mean(x):
            y = np.array(x, np.float64, copy=True)
            y[act] -= y[act].mean()
            y[~act] = 0.0
            return y

        parity = {"against": f"the FP64 oracle's projection of the same input (the GPU's FP32 face fractions), "
                             f"{ncyc} FP64 V-cycles of the same method (rel. residual {cp['rel_residual']:.1e})",
                  "p_rel_l2": rel_l2([no_mean(cp["p"])], [no_mean(gout["p64"])]),
                  "u_rel_l2": rel_l2(cp["u"], gout["u"]), "q_rel_l2": rel_l2(cp["q"], gout["q"])}
        ux, uy, uz = cp["u"]
        hh = cp["h"]
        odiv = np.abs((ux[:, 1:, :] - ux[:, :-1, :]) / hh + (uy[:, :, 1:] - uy[:, :, :-1]) / hh + (uz[1:] - uz[:-1]) / hh)
        div["oracle_fp64_max_abs_div"] = float(odiv.max())
    out = {
        "metric": metric, "value": value, "unit": "projections/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (FP64 defect/refinement)", "data": "synthetic (seeded spectral fields)",
        "config": workload,
        "e2e": {"value": throughput(world, ek, ems), "unit": "projections/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "solve": {"vcycles": reps[-1]["cycles"], "rel_residual": reps[-1]["rel_residual"],
                  "max_abs_div": reps[-1]["max_abs_div"]},
        "divergence": div,
        "parity": parity,
        "plain": plain,
        # every kernel of the event-instrumented steps (ms and algorithmic bytes summed over psteps),
        # with its achieved algorithmic GB/s and that as a fraction of the measured HBM copy bandwidth
        "kernels": [{**{k: (round(v, 4) if isinstance(v, float) else v) for k, v in r.items()},
                     "gbs": round(r["bytes"] / (r["ms"] * 1e6), 1) if r["ms"] > 0 else None,
                     "frac_of_peak": round(r["bytes"] / (r["ms"] * 1e6) / peaks()[0], 3) if r["ms"] > 0 else None}
                    for r in prof],
        "kernel_ms_per_step": round(sum(r["ms"] for r in prof) / psteps, 4),
        "mg_tiles": {"z_chunks_per_level": tiles[0], "variants_per_level": tiles[1], "tuned_ms_per_level": tiles[2]},
    }
    print(json.dumps(out))


if __name__ == "__main__":
    main()
