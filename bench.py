#!/usr/bin/env python
"""Benchmark of the SmokeSim per-frame smoke step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (default): the 256^3 scene of the mixed-precision configuration - two
r=16 emitters injecting density 1, temperature 1 and upward velocity 2, an
r=32 sphere at the centre, three seeded cubes of side 16-48, solid walls, a
unit-variance Gaussian random initial velocity (correlation length 8 cells),
dt = 0.1, buoyancy alpha 0.05 / beta 0.3, vorticity confinement 0.2, multigrid
V-cycles down to 8^3 with 2+2 red-black sweeps (80 on the coarsest level).
A step is one full frame of run_physics_step.  Seeded synthetic data only.

One process per GPU: under torchrun every rank runs its own replica of the
grid (the step is a single-grid computation; replicas only), the timed region
is bracketed by a barrier and synchronize, and the max over ranks is reported.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "Mcell-steps/s at 256³, mixed vs FP32 at equal divergence; fwd+adjoint ms/step"
UNIT = "Mcell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=256, help="grid cells per axis")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--vcycles", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="no timing: set up, run one step and a few level-0 smoother sweeps (for ncu)")
    return ap.parse_args()


def workload(args):
    from smokesim_b200 import scene
    sc = scene.grf256(seed=args.seed, n=args.n, with_grf=True)
    sc["params"].mg.n_vcycles = args.vcycles
    sc["params"].collect_stats = 0
    return sc


def workload_config(args, sc):
    p = sc["params"]
    return {
        "workload": f"grf{args.n}: {args.n}^3 MAC smoke step, 2 emitters + sphere + 3 cubes, GRF initial velocity "
                    f"(sigma 8), dt {p.time_step:g}, {p.mg.n_pre}+{p.mg.n_post} RB-GS sweeps, {p.mg.n_coarse} coarse, "
                    f"{p.mg.n_vcycles} V-cycles to 8^3, reference boundary rules",
        "grid": [args.n, args.n, args.n],
        "precision": "fp32",
        "vcycles_per_step": p.mg.n_vcycles,
        "l2": "inputs larger than L2 (working set ~100 B/cell, 1.6 GB at 256^3)",
    }


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ CPU arm
def cpu_step_rate(sc, steps, warmup):
    """The oracle (C/OpenMP FP32 restatement of the reference shaders) on the
    host cores: returns (Mcell-steps/s, seconds per step, threads)."""
    from oracle import oracle
    from smokesim_b200 import scene
    o = oracle.OracleSim(sc["desc"], "f32")
    scene.apply(o, sc)
    for _ in range(warmup):
        o.step(sc["params"])
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        o.step(sc["params"])
        times.append(time.perf_counter() - t0)
    n = sc["desc"].n
    cells = n[0] * n[1] * n[2]
    sec = statistics.median(times)
    return cells / sec / 1e6, sec, oracle.num_threads(), o


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sc = workload(args)
    value, sec, threads, _ = cpu_step_rate(sc, max(1, args.steps), max(0, args.warmup))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene + GRF)",
        "config": workload_config(args, sc),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"full {args.n}^3 steps, median of {args.steps} after {args.warmup} warm-up"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's own GLSL compute path needs an OpenGL 4.6 context: unavailable on this box; "
                "this arm runs the C/OpenMP restatement of its shaders (oracle/)",
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU arm
def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)

    from smokesim_b200 import Sim, abi, scene
    sc = workload(args)
    n = sc["desc"].n
    cells = n[0] * n[1] * n[2]
    with torch.cuda.stream(stream):
        sim = Sim(sc["desc"], stream=stream.cuda_stream)
        scene.apply(sim, sc)
        p = sc["params"]

        if args.profile:
            sim.step(p, 1)
            sim.smooth(p, 0, 2)
            torch.cuda.synchronize()
            print(json.dumps({"profile": "done", "levels": sim.level_sizes}))
            return 0

        def barrier():
            if world > 1:
                dist.barrier()

        # warm-up
        sim.step(p, args.warmup)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        clk = ClockSampler(local)
        clk.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.step(p, args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        clocks = clk.stop()
        ms = e0.elapsed_time(e1)
        launches = sim.stats().kernel_launches
        if world > 1:
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        value = world * cells * args.steps / (ms / 1e3) / 1e6

        # divergence actually left by this schedule (one extra, untimed step)
        p_stats = scene.workload_params(n_vcycles=args.vcycles, collect_stats=1)
        sim.step(p_stats, 1)
        st = sim.stats()

        # end to end through the C ABI: per step the emitter records go host->device
        # and the step's statistics (divergence norms) come back device->host
        pe = scene.workload_params(n_vcycles=args.vcycles, collect_stats=1)
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            sim.step(pe, 1)
            _ = sim.stats()
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        if world > 1:
            t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = {"value": world * cells * args.steps / e2e_s / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": C.sizeof(abi.Emitter) * len(sc["emitters"]),
               "d2h_bytes_per_step": 8 * 8}

        # roofline of the dominant kernel: the level-0 red-black smoother
        # (k_rb_smooth, one colour per launch on the colour-split arrays).
        # 13 B/cell per red+black sweep (read/write p, read rhs, read flag).
        reps = 10
        sim.smooth(p, 0, 1)
        torch.cuda.synchronize()
        a0, a1, b0, b1 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        a0.record(stream)
        sim.smooth(p, 0, 1)
        a1.record(stream)
        b0.record(stream)
        sim.smooth(p, 0, 1 + reps)
        b1.record(stream)
        torch.cuda.synchronize()
        sweep_ms = (b0.elapsed_time(b1) - a0.elapsed_time(a1)) / reps
        launch_ms = sweep_ms / 2.0
        alg_bytes = 13.0 / 2.0 * cells
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        peak = float(peaks.get("hbm_gbs", 6650.0))
        achieved = alg_bytes / (launch_ms / 1e3) / 1e9
        roofline = {"kernel": "k_rb_smooth<3> (one colour of a level-0 red-black sweep, 256^3)", "bound": "hbm",
                    "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                    "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": launch_ms, "traffic": None}

    line = {
        "impl": "b200", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene + GRF)",
        "config": workload_config(args, sc), "gpu_launches": int(launches), "clocks": clocks,
        "divergence": {"rel_div": st.rel_div, "div_before": st.div_before, "div_after": st.div_after,
                       "vcycles": st.vcycles},
        "e2e": e2e, "roofline": roofline,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cv, csec, threads, _ = cpu_step_rate(sc, 1, 1)
        line["cpu_baseline"] = {"value": cv, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"one full {args.n}^3 step after one warm-up step, C/OpenMP oracle"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sim.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
