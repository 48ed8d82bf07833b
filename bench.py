"""Benchmark of the filament-velocity hot path: point-velocity evaluations per second.

Workload (default): the tree-vs-direct tangle -- random vortex rings, seed 1, delta = 0.001
cm, exactly 32,768 points in a periodic cube D = 0.1 cm; Barnes-Hut theta = 0.4 with the
extra correction; mutual friction alpha = 0.1, alpha' = 0.01 against a uniform normal flow
v_n = (0, 0, 0.5) cm/s; dt = 5e-6 s; insertion, removal and reconnection on.  Synthetic
seeded input (no dataset).  One step = one whole time step (ghosts, tree build, velocity of
every point with 27 periodic images, AB3 update, insertion, closest-point search,
reconnection, removal, periodic wrap) on the device.

value = sum over timed steps of live points / sum of per-step device time (CUDA events on
the library's stream), max over ranks.  Between timed steps a 256 MiB buffer is written to
flush L2 (the workload's state is smaller than L2).

Arms: --impl ours (default) runs libnuvort_gpu; --impl reference times the CPU oracle -- the
line-by-line C++ restatement of the reference Fortran (the reference itself cannot be
compiled here: no Fortran compiler) -- on all host threads, on the same workload.
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

METRIC = "Biot-Savart point-evals/s on 1 B200: mixed+batched vs FP64 plain at ≤1e-6 err"
UNIT = "point-evals/s"


def workload(rank: int, precision: str, velocity: str = "Tree"):
    from nuvort_b200.abi import make_params
    from nuvort_b200.rings import random_rings
    st = random_rings(1 + rank, 0.001, (0.1, 0.1, 0.1), n_points=32768)
    p = make_params(dt=5e-6, delta=0.001, box_size=0.1, velocity=velocity, corea=1.3e-8, tree_theta=0.4,
                    alpha=(0.1, 0.01), normal_velocity="uniform", norm_vel_vec=(0.0, 0.0, 0.5),
                    precision=precision)
    cfg = {"workload": "random-ring tangle, 32,768 points, delta=0.001 cm, D=0.1 cm periodic, seed 1+rank",
           "velocity": velocity, "tree_theta": 0.4, "alpha": [0.1, 0.01], "v_n": [0.0, 0.0, 0.5], "dt": 5e-6,
           "points": int(st.pcount), "images": 27, "precision": precision,
           "l2": "256 MiB buffer written between timed steps (state < L2)"}
    return p, st, cfg


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
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def profile_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary (profiles/traffic.json)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            d = json.load(f)
        return d.get(kernel)
    except Exception:
        return None


def cpu_baseline_port(params, st, seconds: float = 15.0, max_steps: int = 40):
    """Time the CPU oracle (whole steps) on all host threads on the same workload."""
    import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    o = oracle.Oracle(params, st)
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
            "sample": f"{n} whole steps of the same 32,768-point workload on the C++ oracle "
                      f"(OpenMP over points, serial tree build and topology as in the reference), {tot:.1f} s"}


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    params, st, cfg = workload(0, "fp64")
    import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    o = oracle.Oracle(params, st)
    for _ in range(args.warmup):
        o.step(1)
    pts, tot = 0, 0.0
    for _ in range(args.steps):
        live = o.counters().live
        t0 = time.perf_counter()
        o.step(1)
        tot += time.perf_counter() - t0
        pts += live
    value = pts / tot
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{args.steps} whole steps on the C++ restatement of the reference "
                                       "(reference Fortran not buildable here: no Fortran compiler)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from nuvort_b200 import api

    precision = args.precision
    params, st, cfg = workload(rank, precision)
    h = api.Handle(params, [st.pcount * 2], device=local, states=[st])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    for _ in range(args.warmup):
        h.step(1)
    launches = h.step_launches()

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t_before = h.stage_times()
    pts = 0
    evals = tests = 0
    per_step_ms = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            c = h.counters()
            pts += c.live
            before = h.stage_times()["step"]
            h.step(1)
            per_step_ms.append(h.stage_times()["step"] - before)
            c2 = h.counters()
            evals += c2.tree_eval
            tests += c2.tree_tests
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t_after = h.stage_times()
    step_ms = t_after["step"] - t_before["step"]
    vel_ms = t_after["velocity"] - t_before["velocity"]
    tot_ms = torch.tensor([step_ms, vel_ms], dtype=torch.float64, device="cuda")
    tot_pts = torch.tensor([float(pts)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(tot_ms, op=dist.ReduceOp.MAX)
        dist.all_reduce(tot_pts, op=dist.ReduceOp.SUM)
    step_ms, vel_ms = float(tot_ms[0]), float(tot_ms[1])
    all_pts = float(tot_pts[0])
    value = all_pts / (step_ms * 1e-3)

    # end to end through the C ABI with host buffers: upload f(:), one step, download f(:)
    e2e = None
    if not args.no_e2e:
        host = h.download()
        nbytes_state = lambda s: sum(a.nbytes for a in (s.x, s.u, s.u1, s.u2, s.infront, s.behind) if a is not None)
        h2d = d2h = 0
        e_pts = 0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            hs = api.State(x=host.x, infront=host.infront, behind=host.behind, u=host.u, u1=host.u1, u2=host.u2)
            h.upload(0, hs)
            h2d += nbytes_state(hs)
            e_pts += int(np.count_nonzero(host.infront))
            h.step(1)
            host = h.download()
            d2h += nbytes_state(host)
        e2e_s = time.perf_counter() - t0
        e2e_t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        e2e_p = torch.tensor([float(e_pts)], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
            dist.all_reduce(e2e_p, op=dist.ReduceOp.SUM)
        e2e = {"value": float(e2e_p[0]) / float(e2e_t[0]), "unit": UNIT,
               "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps,
               "path": "nv_upload (host f(:) -> device) + nv_step(1) + nv_download (device -> host) per step"}

    out = None
    if rank == 0:
        fp64_peak = api.measure_fp64_peak(local)
        # dominant kernel: the tree walk; algorithmic flops = 43 per accepted interaction + 12 per
        # opening test (counted on the device), per launch (one launch per step)
        flops = (43.0 * evals + 12.0 * tests) / args.steps
        vel_launch_s = vel_ms / args.steps * 1e-3
        achieved = flops / vel_launch_s / 1e12
        roof = {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak if fp64_peak else None,
                "traffic": profile_traffic("k_tree_walk_fp64"),
                "kernel": "k_tree_walk_fp64",
                "peak_source": "FP64 FMA rate measured on this GPU by nv_measure_fp64_peak (MEASURED_PEAKS.json "
                               "covers HBM and bf16 tensor only)",
                "per_launch": {"interactions": evals / args.steps, "opening_tests": tests / args.steps,
                               "ms": vel_ms / args.steps}}
        peaks = measured_peaks()
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if precision == "fp64" else "f32+f64",
                "data": "synthetic", "config": cfg, "impl": "ours",
                "velocity_stage": {"ms_per_step": vel_ms / args.steps,
                                   "point_evals_per_s": all_pts / (vel_ms * 1e-3)},
                "roofline": roof, "hbm_peak_gbs": peaks.get("hbm_gbs"),
                "clocks": clk.summary(), "gpu_launches": launches * args.steps,
                "per_step_ms": [round(x, 4) for x in per_step_ms]}
        if e2e:
            line["e2e"] = e2e
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_baseline_port(params, st, seconds=args.cpu_seconds)
        out = line
    h.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if out:
        print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
