"""Benchmark of the filament-velocity hot path: point-velocity evaluations per second.

Default workload (--workload ensemble512): an ensemble of 512 independent random-ring systems
(seed 2), point counts log-uniform in [500, 20000] (about 2.7M points), delta = 0.002 cm,
periodic cube D = 0.1 cm; per system alpha ~ U[0.03,0.2], alpha' ~ U[0,0.02] and a uniform
normal flow of magnitude U[0,1] cm/s along a random axis; direct sum below the autotuned
direct/tree crossover, Barnes-Hut theta = 0.4 above it; dt = 2e-5 s; insertion, removal and
reconnection on; every system advanced by the same launches (one per stage).  The same line
carries the 1,048,576-point counterflow tangle (seed 3, delta = 0.0005 cm, theta = 0.5,
alpha = (0.1, 0.01), v_n = (1,0,0) cm/s, dt = 1e-6 s) as the sub-object "tangle1m", with its
own mixed/plain timing, error and event comparison over at least 20 steps.  Seeded synthetic
input (no dataset).  Other workloads (--workload): rings8 (8 rings, direct sum, FP64 small
case), tangle32k (32,768 points, theta = 0.4), tangle1m, ensemble32 (32 systems of
131k-262k points).

One step = one whole time step on the device (ghosts, tree build, velocity of every point
with 27 periodic images, AB3 update, insertion, closest-point search, reconnection, removal,
periodic wrap), replayed from a CUDA graph.  value = sum over timed steps of live points /
sum of per-step device time of whole steps (CUDA events recorded on the library's stream),
max over ranks; "velocity_stage" gives the same per velocity-stage time.  Between timed steps
a 256 MiB buffer is written to flush L2.

The product arm runs the mixed-precision path; the plain FP64 path (the drop-in that
reproduces the reference arithmetic) is measured beside it on the same initial state, and
the line reports both, their velocity difference, their error against the FP64 direct sum
on a seeded subsample of points, and whether their topology event logs agree.

Multi-GPU (torchrun, one rank per GPU): an ensemble's systems are split across the ranks by
a greedy balance of sum N^2 (nuvort_b200.dist.shard_systems), the same ensemble whatever the
rank count (strong scaling, no collective on the data path); a single-tangle workload runs one
replica per rank (seed + rank, weak scaling), or, with --split-tangle, one tangle over all the
ranks: each computes the velocities of its range of the walk order, the ranges are
all-gathered (NCCL) and every rank finishes the step on the full field (strong scaling; the
line checks that the ranks agree and that rank 0's state equals an unsplit run's).

--impl reference times the CPU oracle -- the line-by-line C++ restatement of the reference
Fortran (the Fortran itself cannot be built here: no Fortran compiler) -- on all host
threads, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "Biot-Savart point-evals/s on 1 B200: mixed+batched vs FP64 plain at ≤1e-6 err"
UNIT = "point-evals/s"


# ---- workloads -----------------------------------------------------------------------------
def _p(**kw):
    from nuvort_b200.abi import make_params
    base = dict(box_size=0.1, corea=1.3e-8)
    base.update(kw)
    return make_params(**base)


def workload(name: str, rank: int = 0, crossover: int = 3000, world: int = 1):
    """(params per system, states, config dict) of this rank.  Single tangles: one replica per
    rank (seed + rank).  Ensembles: the same ensemble on every rank, its systems split across
    the ranks by shard_systems (sum of N^2 balanced)."""
    from nuvort_b200.rings import random_rings
    L = (0.1, 0.1, 0.1)
    if name == "rings8":
        st = random_rings(0 + rank, 0.002, L, n_rings=8)
        return [_p(dt=2e-5, delta=0.002, velocity="BS", tree_theta=0.0)], [st], {
            "workload": "8 random rings, seed 0+rank, delta=0.002 cm, direct sum, no normal fluid",
            "points": int(st.pcount), "dt": 2e-5}
    if name == "tangle32k":
        st = random_rings(1 + rank, 0.001, L, n_points=32768)
        return [_p(dt=5e-6, delta=0.001, velocity="Tree", tree_theta=0.4, alpha=(0.1, 0.01),
                   normal_velocity="uniform", norm_vel_vec=(0.0, 0.0, 0.5))], [st], {
            "workload": "random-ring tangle, 32,768 points, delta=0.001 cm, D=0.1 cm periodic, seed 1+rank",
            "velocity": "Tree", "tree_theta": 0.4, "alpha": [0.1, 0.01], "v_n": [0.0, 0.0, 0.5], "dt": 5e-6,
            "points": 32768, "images": 27}
    if name == "tangle1m":
        st = random_rings(3 + rank, 0.0005, L, n_points=1048576)
        return [_p(dt=1e-6, delta=0.0005, velocity="Tree", tree_theta=0.5, alpha=(0.1, 0.01),
                   normal_velocity="xflow", norm_vel_xflow=1.0)], [st], {
            "workload": "random-ring counterflow tangle, 1,048,576 points, delta=0.0005 cm, seed 3+rank",
            "velocity": "Tree", "tree_theta": 0.5, "alpha": [0.1, 0.01], "v_n": [1.0, 0.0, 0.0], "dt": 1e-6,
            "points": 1048576, "images": 27}
    if name in ("ensemble512", "ensemble32"):
        from nuvort_b200.dist import shard_systems
        big = name == "ensemble32"
        seed = 4 if big else 2
        rng = np.random.Generator(np.random.PCG64(seed))
        nsys = 32 if big else 512
        if big:
            counts = rng.uniform(131072, 262144, size=nsys).astype(int)
        else:
            counts = np.round(np.exp(rng.uniform(math.log(500), math.log(20000), size=nsys))).astype(int)
        delta = 0.0005 if big else 0.002
        mine = set(shard_systems([int(c) for c in counts], world, rank))
        params, states = [], []
        for s in range(nsys):
            sub = int(rng.integers(0, 2**31 - 1))
            if big:
                a = float(rng.uniform(0.05, 0.15))
                alpha = (a, 0.1 * a)
                vmag = float(rng.uniform(0.2, 1.0))
                vec = (vmag, 0.0, 0.0)
            else:
                alpha = (float(rng.uniform(0.03, 0.2)), float(rng.uniform(0.0, 0.02)))
                vmag = float(rng.uniform(0.0, 1.0))
                ax = rng.standard_normal(3)
                ax /= np.linalg.norm(ax)
                vec = tuple(float(v) for v in vmag * ax)
            n = int(counts[s])
            vel = "Tree" if (big or n >= crossover) else "BS"
            theta = 0.5 if big else 0.4
            if s not in mine:
                continue
            params.append(_p(dt=1e-6 if big else 2e-5, delta=delta, velocity=vel, tree_theta=theta, alpha=alpha,
                             normal_velocity="uniform", norm_vel_vec=vec))
            states.append(random_rings(sub, delta, L, n_points=n))
        cfg = {"workload": (f"ensemble of {nsys} independent random-ring systems, points "
                            + ("U[131072,262144]" if big else "log-uniform [500,20000]") + f", seed {seed}"),
               "systems": nsys, "points": int(sum(int(c) for c in counts)),
               "direct_below": None if big else crossover, "tree_theta": 0.5 if big else 0.4,
               "dt": 1e-6 if big else 2e-5}
        if world > 1:
            cfg["sharding"] = (f"{world} ranks, systems split by a greedy balance of sum N^2; this line's "
                               "value counts every rank's points")
        return params, states, cfg
    raise ValueError(name)


def with_precision(params, precision: str):
    out = []
    for p in params:
        q = type(p).from_buffer_copy(p)
        q.precision = 1 if precision == "mixed" else 0
        out.append(q)
    return out


# ---- helpers ---------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while active."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def profile_traffic(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` on `workload` from its committed ncu summary
    (profiles/traffic.json), or None where no capture of that workload exists."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            entry = json.load(f).get(kernel, {}).get(workload)
        return dict(entry, workload=workload) if entry else None
    except Exception:
        return None


def rms_rel(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def timed_steps(h, steps, flush, torch, sampler=None):
    """Run `steps` single steps; per-step device time from the library's stage events."""
    pts = 0
    evals = tests = 0
    per_step = []
    vel = 0.0
    t_start = h.stage_times()
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        pts += sum(h.counters(s).live for s in range(h.nsys))
        before = h.stage_times()
        h.step(1)
        after = h.stage_times()
        per_step.append(after["step"] - before["step"])
        vel += after["velocity"] - before["velocity"]
        for s in range(h.nsys):
            c = h.counters(s)
            evals += c.tree_eval
            tests += c.tree_tests
    t_end = h.stage_times()
    timed_steps.stages = {k: (t_end[k] - t_start[k]) / steps for k in t_end}
    return pts, per_step, vel, evals, tests


def cpu_baseline_port(params, states, seconds: float = 15.0, max_steps: int = 40):
    """The CPU oracle (whole steps, all host threads) on the first system of the workload."""
    import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    o = oracle.Oracle(with_precision(params, "fp64")[0], states[0])
    o.step(1)  # warm-up (first tree build, page-in)
    pts, tot, n = 0, 0.0, 0
    while tot < seconds and n < max_steps:
        live = o.counters().live
        t0 = time.perf_counter()
        o.step(1)
        tot += time.perf_counter() - t0
        pts += live
        n += 1
    return {"value": pts / tot, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} whole steps of system 0 of the workload ({states[0].pcount} points) on the C++ oracle "
                      f"(OpenMP over points; tree build and topology serial as in the reference), {tot:.1f} s"}


# ---- arms ------------------------------------------------------------------------------------
def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    # the ensemble's direct/tree split: the crossover the product arm's autotuner measured on
    # the B200 (500 points, i.e. every system of at least 500 points walks the tree); the CPU
    # reference itself has no crossover, each system runs with the velocity scheme it is given
    params, states, cfg = workload(args.workload, 0, crossover=args.crossover or 500)
    import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    os_ = [oracle.Oracle(p, s) for p, s in zip(with_precision(params, "fp64"), states)]
    # bounded sample: the first systems up to the point budget (all of a single tangle)
    budget = max(states[0].pcount, 40000)
    use, tot_pts = [], 0
    for o, s in zip(os_, states):
        if tot_pts and tot_pts + s.pcount > budget:
            break
        use.append(o)
        tot_pts += s.pcount
    for _ in range(args.warmup):
        for o in use:
            o.step(1)
    pts, tot = 0, 0.0
    for _ in range(args.steps):
        for o in use:
            live = o.counters().live
            t0 = time.perf_counter()
            o.step(1)
            tot += time.perf_counter() - t0
            pts += live
    value = pts / tot
    sample = (f"{args.steps} whole steps of {len(use)} of {len(states)} system(s) ({tot_pts} points) on the C++ "
              "restatement of the reference (the Fortran is not buildable here: no Fortran compiler), "
              f"{threads} threads")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def compare_arms(params, states, args, local, flush, torch, dist, steps, warmup, e2e=False):
    """Mixed (product) and plain FP64 handles on the same initial state: errors on that state,
    then warm-up and timed steps of each, event comparison over every step run.  Returns
    (measurements dict, mixed handle, plain handle); the caller closes the handles."""
    from nuvort_b200 import api
    caps = [int(s.pcount * 1.6) + 256 for s in states]
    hm = api.Handle(with_precision(params, args.precision), caps, device=local, states=states)
    hp = api.Handle(with_precision(params, "fp64"), caps, device=local, states=states) if args.compare else None
    # block shapes of each arm's velocity pass, measured on these systems (velocity passes only)
    from nuvort_b200.autotune import tune_launch_shapes
    shapes = {"product": tune_launch_shapes(hm)}
    if hp is not None:
        shapes["plain_fp64"] = tune_launch_shapes(hp)
    err = {}
    if hp is not None:
        um = [hm.calc_velocity(s) for s in range(len(states))]
        up = [hp.calc_velocity(s) for s in range(len(states))]
        err["rms_rel_vs_plain_fp64"] = rms_rel(np.concatenate(um), np.concatenate(up))
        # FP64 direct-sum yardstick on a seeded subsample of the first system's points
        rng = np.random.Generator(np.random.PCG64(12345))
        n0 = states[0].pcount
        sub = np.sort(rng.choice(np.arange(1, n0 + 1), size=min(args.subsample, n0), replace=False))
        ud = hp.calc_velocity_direct_at(0, sub)
        err["rms_rel_vs_direct_fp64"] = {
            "mixed": rms_rel(um[0][sub - 1], ud), "plain": rms_rel(up[0][sub - 1], ud),
            "subsample": int(len(sub)), "system": 0,
            "note": "the tree approximation itself (theta); the same in both arms"}
        for h in (hm, hp):  # fresh state for the timed run
            for s, st in enumerate(states):
                h.upload(s, st, t=0.0, itime=0)
        hm.set_event_margins(True)  # how close the compared events came to flipping
    for _ in range(warmup):
        hm.step(1)
        if hp is not None:
            hp.step(1)
    launches = hm.step_launches()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        pts, per_step, vel_ms, evals, tests = timed_steps(hm, steps, flush, torch)
    stages = timed_steps.stages
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    out = {"pts": pts, "per_step": per_step, "vel_ms": vel_ms, "evals": evals, "tests": tests, "stages": stages,
           "launches": launches, "clocks": clk.summary(), "err": err, "plain": None, "shapes": shapes}
    if hp is not None:
        ppts, pper, pvel, _, _ = timed_steps(hp, steps, flush, torch)
        # every event of every system, through the device digest (the event log may be full)
        cm = [hm.counters(s) for s in range(len(states))]
        cp = [hp.counters(s) for s in range(len(states))]
        out["plain"] = {"pts": ppts, "step_ms": sum(pper), "vel_ms": pvel}
        err["events_match_plain"] = all(a.event_hash == b.event_hash and a.n_events == b.n_events
                                        for a, b in zip(cm, cp))
        err["events_compared"] = int(sum(c.n_events for c in cp))
        err["steps_compared"] = warmup + steps
        err["events_compared_by"] = "per-system event count and order-sensitive 64-bit digest"
        err.update(margin_report(hm, hp, params, len(states)))
    return out, hm, hp, caps


def margin_report(hm, hp, params, nsys):
    """The mixed arm's event margins (smallest relative distance of any topology test from
    its threshold, over every step run) against the largest position difference between the
    two arms at the end: a distance test moves by at most 2 dev / threshold and the tangent
    dot by about 4 dev / delta, so margins far above 4 dev / delta leave the events safe."""
    keys = ("insert", "remove", "recon_distance", "recon_dot")
    mins = {k: 1e300 for k in keys}
    dev, need = 0.0, 0.0
    for s in range(nsys):
        mg = hm.event_margins(s)
        for k in keys:
            mins[k] = min(mins[k], mg[k])
        a, b = hm.download(s), hp.download(s)
        if a.pcount == b.pcount and np.array_equal(a.infront, b.infront):
            d = float(np.max(np.abs(a.x - b.x))) if a.pcount else 0.0
            dev = max(dev, d)
            need = max(need, 4.0 * d / params[s].delta)
    worst = min(mins.values())
    return {"event_margins_min": {k: (v if v < 1e300 else None) for k, v in mins.items()},
            "position_dev_max_cm": dev,
            "margin_over_need": (worst / need) if need > 0 else None}


def roofline_of(params, states, m, steps, precision, local, workload):
    from nuvort_b200 import api
    from nuvort_b200.abi import NV_VEL_BS
    mixed = precision == "mixed"
    # direct-sum systems: 27 N^2 pair-images each (N = live points at the start)
    pairs = sum(27.0 * float(st.pcount) ** 2 for p, st in zip(params, states) if p.velocity == NV_VEL_BS)
    tree = m["evals"] / steps >= pairs
    kernel = ("k_tree_walk_mixed" if mixed else "k_tree_walk_fp64") if tree else (
        "k_direct_mixed" if mixed else "k_direct_fp64")
    peak = api.measure_fp32_peak(local) if mixed else api.measure_fp64_peak(local)
    flops = (43.0 * m["evals"] + 12.0 * m["tests"]) / steps + 43.0 * pairs
    per_launch = {"interactions": m["evals"] / steps, "opening_tests": m["tests"] / steps,
                  "direct_pair_images": pairs, "ms": m["vel_ms"] / steps}
    achieved = flops / (m["vel_ms"] / steps * 1e-3) / 1e12
    return {"bound": "fp32" if mixed else "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if peak else None, "traffic": profile_traffic(kernel, workload), "kernel": kernel,
            "peak_source": ("FP32" if mixed else "FP64") + " FMA rate measured on this GPU by nv_measure_fp"
                           + ("32" if mixed else "64") + "_peak (MEASURED_PEAKS.json covers HBM and bf16 tensor "
                           "only); algorithmic flops = 43 per interaction or pair-image + 12 per opening test; "
                           "time = the velocity stage (all velocity kernels of the step)",
            "per_launch": per_launch}


def tangle1m_summary(args, local, flush, torch):
    """The 1M-point counterflow tangle, mixed against plain, for the ensemble's line."""
    params, states, cfg = workload("tangle1m", 0)
    steps = args.steps
    warmup = max(args.warmup, 20 - steps)  # events compared over at least 20 steps
    m, hm, hp, _ = compare_arms(params, states, args, local, flush, torch, None, steps, warmup)
    hm.close()
    if hp is not None:
        hp.close()
    step_ms = sum(m["per_step"])
    out = {"config": cfg, "steps": steps, "warmup": warmup,
           "value": m["pts"] / (step_ms * 1e-3), "ms_per_step": step_ms / steps,
           "velocity_stage": {"ms_per_step": m["vel_ms"] / steps, "point_evals_per_s": m["pts"] / (m["vel_ms"] * 1e-3)},
           "stage_ms_per_step": {k: round(v, 4) for k, v in m["stages"].items()},
           "launch_shapes": m["shapes"],
           "roofline": roofline_of(params, states, m, steps, args.precision, local, "tangle1m"),
           "clocks": m["clocks"]}
    if m["plain"]:
        p = m["plain"]
        out["plain_fp64"] = {"value": p["pts"] / (p["step_ms"] * 1e-3), "ms_per_step": p["step_ms"] / steps,
                             "velocity_ms_per_step": p["vel_ms"] / steps}
        out["speedup_vs_plain"] = out["value"] / out["plain_fp64"]["value"]
        out["velocity_speedup_vs_plain"] = p["vel_ms"] / m["vel_ms"]
    out["error"] = m["err"]
    return out


def run_ours(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    from nuvort_b200 import api

    crossover, tuned = args.crossover, None
    if args.workload == "ensemble512" and crossover is None:
        # the direct/tree crossover of the batched ensemble, measured on this GPU
        from nuvort_b200.autotune import tune_crossover
        tuned = tune_crossover(device=local, precision=args.precision, delta=0.002, theta=0.4)
        crossover = tuned["crossover"]
    params, states, cfg = workload(args.workload, rank, crossover=crossover or 3000, world=world)
    ensemble = args.workload.startswith("ensemble")
    if tuned is not None:
        cfg["crossover_source"] = ("autotuned on this GPU (nuvort_b200/autotune.py): velocity + tree-build device "
                                   "time per point of batched systems, direct vs tree"
                                   + (", cached" if tuned.get("cached") else ""))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    m, hm, hp, caps = compare_arms(params, states, args, local, flush, torch, dist, args.steps, args.warmup)
    from nuvort_b200.dist import reduce_max_sum
    (step_ms, vel_ms), (all_pts,) = reduce_max_sum(dist, "cuda", [sum(m["per_step"]), m["vel_ms"]], [float(m["pts"])])
    value = all_pts / (step_ms * 1e-3)
    plain = None
    if m["plain"]:
        (pstep, pvel), (ppts,) = reduce_max_sum(dist, "cuda", [m["plain"]["step_ms"], m["plain"]["vel_ms"]],
                                                [float(m["plain"]["pts"])])
        plain = {"value": ppts / (pstep * 1e-3), "ms_per_step": pstep / args.steps,
                 "velocity_ms_per_step": pvel / args.steps}

    # end to end through the C ABI with host buffers: upload f(:), one step, download f(:)
    e2e = None
    if not args.no_e2e:
        # the caller's persistent host arrays f(:) (x, u, u1, u2, infront, behind), as the
        # reference keeps them between steps
        # (page-locked, one array per field with every system's rows packed one after another;
        # all systems in one call and one copy per array each way)
        fields = ("x", "u", "u1", "u2", "infront", "behind")
        hb = api.BatchBuffers(hm, fields)
        hb.download()
        h2d = d2h = e_pts = 0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            hb.upload()
            h2d += hb.bytes_of(fields)
            e_pts += hb.live_points()
            hm.step(1)
            hb.download()
            d2h += hb.bytes_of(fields)
        e2e_s = time.perf_counter() - t0
        hb.close()
        (e2e_s,), (e_pts,) = reduce_max_sum(dist, "cuda", [e2e_s], [float(e_pts)])
        e2e = {"value": e_pts / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps,
               "path": "nv_upload_packed (page-locked host f(:) of every system -> device) + nv_step(1) + "
                       "nv_download_packed (device -> host) per step"}
    hm.close()
    if hp is not None:
        hp.close()

    out = None
    if rank == 0:
        mixed = args.precision == "mixed"
        peaks = measured_peaks()
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_ms / args.steps, "higher_is_better": True,
                "scaling": "strong" if ensemble else "weak", "vs_baseline": None,
                "dtype": "f32+f64" if mixed else "f64", "data": "synthetic",
                "config": dict(cfg, precision=args.precision, l2="256 MiB buffer written between timed steps"),
                "impl": "ours",
                "value_basis": "whole steps (ghosts, tree build, velocity, AB3 update, topology); the velocity "
                               "stage alone is in velocity_stage",
                "velocity_stage": {"ms_per_step": vel_ms / args.steps, "point_evals_per_s": all_pts / (vel_ms * 1e-3)},
                "stage_ms_per_step": {k: round(v, 4) for k, v in m["stages"].items()},
                "launch_shapes": m["shapes"],
                "roofline": roofline_of(params, states, m, args.steps, args.precision, local, args.workload),
                "hbm_peak_gbs": peaks.get("hbm_gbs"), "clocks": m["clocks"],
                "gpu_launches": m["launches"] * args.steps, "per_step_ms": [round(x, 4) for x in m["per_step"]]}
        if plain:
            line["plain_fp64"] = plain
            line["speedup_vs_plain"] = value / plain["value"]
            line["velocity_speedup_vs_plain"] = plain["velocity_ms_per_step"] / (vel_ms / args.steps)
        if m["err"]:
            line["error"] = dict(m["err"], scope="rank 0's systems" if world > 1 else "every system")
        if e2e:
            line["e2e"] = e2e
        out = line
    # the 1M tangle beside the ensemble (rank 0's GPU; the other ranks wait at the barrier)
    if rank == 0 and args.workload == "ensemble512" and args.with_1m:
        out["tangle1m"] = tangle1m_summary(args, local, flush, torch)
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline_port(params, states, seconds=args.cpu_seconds)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if out:
        print(json.dumps(out), flush=True)
    return 0


def run_split_tangle(args):
    """One tangle on every rank, its velocity pass split over the ranks (TangleSplit: walk
    ranges of whole warps, an all-gather of the velocities, every rank finishing the step on
    the full field).  Strong scaling: the job advances one tangle whatever N.  Each timed
    step is bracketed by events on torch's stream with the device idle on both sides (the
    library's calls return with their stream drained), so a step's time covers the ranks'
    launches, the exchange and the host calls between them; max over ranks.  At the end the
    ranks' states are compared (a digest of every rank's positions and links), and rank 0
    runs the same steps unsplit (nv_step) and compares bit for bit."""
    import datetime
    import hashlib

    import torch
    import torch.distributed as dist
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180), device_id=dev)
    else:  # a one-rank group: the same code path, the exchange a copy
        import socket
        with socket.socket() as s:
            s.bind(("127.0.0.1", 0))
            port = s.getsockname()[1]
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=180), device_id=dev)
    from nuvort_b200 import api
    from nuvort_b200.dist import TangleSplit, reduce_max_sum
    params, states, cfg = workload(args.workload, 0)  # the same tangle (seed) on every rank
    caps = [int(s.pcount * 1.6) + 256 for s in states]
    hp = with_precision(params, args.precision)
    h = api.Handle(hp, caps, device=local, states=states)
    ts = TangleSplit(h, 0, dist, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        ts.step()
    dist.barrier()
    torch.cuda.synchronize()
    per_step, pts = [], 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            pts += int(h.counters(0).live)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            ts.step()
            torch.cuda.synchronize()
            e1.record()
            e1.synchronize()
            per_step.append(e0.elapsed_time(e1))
    dist.barrier()
    st = h.download(0)
    dig = hashlib.sha256(st.x.tobytes() + st.infront.tobytes() + st.behind.tobytes()).digest()
    d = torch.tensor(list(dig[:8]), dtype=torch.float64, device="cuda")
    (step_ms,), _ = reduce_max_sum(dist, "cuda", [sum(per_step)], [float(pts)])
    dmax, dsum = reduce_max_sum(dist, "cuda", list(d.tolist()), list(d.tolist()))
    identical = all(abs(a * world - b) < 0.5 for a, b in zip(dmax, dsum))  # every rank's digest equal
    launches = h.step_launches() + 1 + (world - 1)  # the step's kernels, the pack, the unpacks
    h.close()
    out = None
    if rank == 0:
        ref = api.Handle(hp, caps, device=local, states=states)
        ref.step(args.warmup + args.steps)
        sr = ref.download(0)
        ref.close()
        one_gpu = bool(np.array_equal(sr.x, st.x) and np.array_equal(sr.infront, st.infront)
                       and np.array_equal(sr.behind, st.behind))
        out = {"metric": METRIC, "value": pts / (step_ms * 1e-3), "unit": UNIT, "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms / args.steps,
               "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
               "dtype": "f32+f64" if args.precision == "mixed" else "f64", "data": "synthetic",
               "config": dict(cfg, workload=cfg["workload"].replace("seed 3+rank", "seed 3").replace(
                   "seed 1+rank", "seed 1"), precision=args.precision,
                   split=(f"one tangle on {world} rank(s): walk ranges of whole warps, all-gather of the "
                          "velocities, every rank finishing the step"),
                   l2="256 MiB buffer written between timed steps"),
               "impl": "ours", "clocks": clk.summary(), "gpu_launches": launches * args.steps,
               "ranks_identical": identical, "matches_one_gpu": one_gpu,
               "per_step_ms": [round(x, 4) for x in per_step]}
    dist.barrier()
    dist.destroy_process_group()
    if out:
        print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["rings8", "tangle32k", "ensemble512", "tangle1m", "ensemble32"],
                    default="ensemble512")
    ap.add_argument("--no-1m", dest="with_1m", action="store_false",
                    help="ensemble512: skip the 1M-tangle sub-object of the line")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--crossover", type=int, default=None,
                    help="ensembles: direct sum below this many points (default: autotuned for ensemble512, 3000 "
                         "otherwise)")
    ap.add_argument("--subsample", type=int, default=4096)
    ap.add_argument("--no-compare", dest="compare", action="store_false", help="skip the plain FP64 arm")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--split-tangle", action="store_true",
                    help="tangle workloads: one tangle over all ranks, its velocity pass split by walk ranges "
                         "(default: one replica per rank)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.split_tangle:
        if args.workload not in ("tangle32k", "tangle1m"):
            ap.error("--split-tangle takes a tangle workload (tangle32k, tangle1m)")
        return run_split_tangle(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
