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

import numpy as np

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
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the forward+adjoint rollout timing")
    ap.add_argument("--profile-adjoint", action="store_true",
                    help="no timing: a 4-step forward+reverse rollout of the plume scene at --n (for ncu)")
    ap.add_argument("--profile", action="store_true",
                    help="no timing: set up, run --profile-steps steps and a few level-0 smoother sweeps (for ncu)")
    ap.add_argument("--profile-steps", type=int, default=1,
                    help="steps of the --profile run (the first one starts from the GRF state)")
    ap.add_argument("--inverse", action="store_true",
                    help="instead of the benchmark: the inverse-control run (plume scene at --inverse-n, per-step emitter "
                         "forces + a 16^3 force field fitted by Adam to a target density)")
    ap.add_argument("--inverse-n", type=int, default=128)
    ap.add_argument("--inverse-steps", type=int, default=200)
    ap.add_argument("--inverse-iters", type=int, default=50)
    return ap.parse_args()


VARIANTS = {
    # name: (precision, ref_quirks, tol, V-cycle cap or count, warm start)
    # warm start 1: the mixed solve starts from 2 p(n-1) - p(n-2) once two
    # solved steps exist; 0: from p(n-1), as the reference's solve does
    "mixed_fp16": (1, 0, 1e-6, 40, 1),
    "mixed_bf16": (2, 0, 1e-6, 40, 1),
    "mixed_fp16_previous_pressure_start": (1, 0, 1e-6, 40, 0),
    "fp32": (0, 0, 1e-6, 40, 0),
    "fp32_reference_rules_4vc": (0, 1, 0.0, 4, 0),
}
HEADLINE = "mixed_fp16"


def variant_params(sc, name):
    from smokesim_b200 import scene
    prec, quirks, tol, cyc, ws = VARIANTS[name]
    p = scene.workload_params(ref_quirks=quirks, precision=prec, tol=tol, n_vcycles=cyc,
                              collect_stats=1 if tol > 0 else 0, warm_start=ws)
    return p


def workload(args):
    from smokesim_b200 import scene
    sc = scene.grf256(seed=args.seed, n=args.n, with_grf=True)
    sc["params"] = variant_params(sc, HEADLINE)
    return sc


def workload_config(args, sc):
    p = sc["params"]
    return {
        "workload": f"grf{args.n}: {args.n}^3 MAC smoke step, 2 emitters + sphere + 3 cubes, GRF initial velocity "
                    f"(sigma 8), dt {p.time_step:g}, {p.mg.n_pre}+{p.mg.n_post} RB-GS sweeps, {p.mg.n_coarse} coarse, "
                    f"V-cycles to 8^3 until the projected divergence is <= 1e-6 of the pre-projection divergence "
                    f"(cap 40); mixed precision: FP64 residual + refinement, FP32 smoothing, FP16 coarse corrections; "
                    f"each solve starts from " + ("the linear extrapolation 2 p(n-1) - p(n-2) of the last two solved "
                                                  "pressures (from the third step on)" if p.mg.warm_start == 1
                                                  else "the previous step's pressure"),
        "grid": [args.n, args.n, args.n],
        "precision": "mixed (f64 residual/refinement, f32 smoothing, f16 coarse)",
        "tolerance": p.mg.tol,
        "warm_start": "extrapolated" if p.mg.warm_start == 1 else "previous pressure",
        "l2": "inputs larger than L2 (working set ~100 B/cell, 1.6 GB at 256^3)",
    }


# ------------------------------------------------------------------ ranks
def max_over_ranks(value, world, device):
    """The largest of the ranks' values (every rank gets it): timings of a
    multi-rank run are the slowest rank's."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, cells, steps, ms):
    """Whole-job Mcell-steps/s: every rank advances its own replica of
    `cells` cells by `steps` steps in `ms` milliseconds (slowest rank)."""
    return world * cells * steps / (ms / 1e3) / 1e6


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
    vcycles = []
    for _ in range(steps):
        t0 = time.perf_counter()
        o.step(sc["params"])
        times.append(time.perf_counter() - t0)
        vcycles.append(o.stats().vcycles)
    n = sc["desc"].n
    cells = n[0] * n[1] * n[2]
    sec = statistics.median(times)
    cpu_step_rate.vcycles = vcycles   # refinement steps (V-cycles) of the sampled steps
    return cells / sec / 1e6, sec, oracle.num_threads(), o


# the reference arm stops taking steps once this much time has gone (a
# 256^3 step of the oracle takes seconds on the host cores)
REFERENCE_BUDGET_S = 150.0


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle
    sc = workload(args)
    o = oracle.OracleSim(sc["desc"], "f32")
    from smokesim_b200 import scene
    scene.apply(o, sc)
    t_start = time.perf_counter()
    w = 0
    for _ in range(args.warmup):
        o.step(sc["params"])
        w += 1
        if time.perf_counter() - t_start > REFERENCE_BUDGET_S / 4:
            break
    times = []
    vcycles = []
    t_timed = time.perf_counter()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.step(sc["params"])
        times.append(time.perf_counter() - t0)
        vcycles.append(o.stats().vcycles)
        if time.perf_counter() - t_start > REFERENCE_BUDGET_S:
            break
    total = time.perf_counter() - t_timed
    k = len(times)
    n = sc["desc"].n
    cells = n[0] * n[1] * n[2]
    value = cells * k / total / 1e6
    threads = oracle.num_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": k, "warmup": w, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": total / k * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 residual/refinement, f16 coarse storage)",
        "data": "synthetic (seeded scene + GRF)",
        "config": workload_config(args, sc),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{k} consecutive full {args.n}^3 steps after {w} warm-up steps, from the "
                                   f"workload's initial state (the steps that fit in {REFERENCE_BUDGET_S:.0f} s)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "vcycles_mean": sum(vcycles) / max(1, len(vcycles)),
        "note": "the reference's own GLSL compute path needs an OpenGL 4.6 context: unavailable on this box; this "
                "arm runs the C/OpenMP restatement of its compute shaders (oracle/) on all host threads, with the "
                "same step as the GPU arm: the reference's stage order, boundary rules and red-black ordering, "
                "and the same mixed-precision projection (FP64 residual and refinement, FP32 smoothing, FP16 "
                "coarse corrections, the same extrapolated warm start) to the same 1e-6 tolerance",
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU arm
# DRAM bytes per k_rb_smooth4<3> launch at 256^3 from one ncu capture of
# that launch (dram__bytes_read.sum + dram__bytes_write.sum: 76,061,440 +
# 10,889,472); the figure is for the 256^3 workload only.
RB_SMOOTH_TRAFFIC = 86950912


def step1(sim, p):
    """One step; a tolerance solve that hits its V-cycle cap completes the
    step and reports SS_E_NOT_CONVERGED, which its statistics record."""
    from smokesim_b200 import SmokeSimError, abi
    try:
        sim.step(p, 1)
    except SmokeSimError as e:
        if e.code != abi.SS_E_NOT_CONVERGED:
            raise


def run_variant(torch, sim_cls, scene, sc, name, args, stream, barrier, world, dev, timed_stats=True):
    """Fresh simulation of the scene, W warm-up steps, K steps timed with CUDA
    events on the simulation's stream (max over ranks).  Returns the timing and
    the per-step solver statistics of the timed steps."""
    import torch.distributed as dist
    p = variant_params(sc, name)
    sim = sim_cls(sc["desc"], stream=stream.cuda_stream)
    scene.apply(sim, sc)
    for _ in range(args.warmup):
        step1(sim, p)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    launches = 0
    e0.record(stream)
    for _ in range(args.steps):
        step1(sim, p)
        st = sim.stats()
        launches += st.kernel_launches
        stats.append((st.vcycles, st.converged, st.residual / st.div_before if st.div_before > 0 else 0.0, st.rel_div))
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    out = {"ms_per_step": ms / args.steps, "ms_total": ms, "gpu_launches": launches}
    if p.mg.tol > 0:
        out.update({
            "vcycles_mean": statistics.mean(x[0] for x in stats),
            "vcycles_max": max(x[0] for x in stats),
            "converged_steps": sum(x[1] for x in stats),
            "projected_rel_div_max": max(x[2] for x in stats),
            "rel_div_last": stats[-1][3],
        })
    return sim, p, out


ADJOINT_CASES = [
    # name, scene, steps, checkpoint interval (= steps: every intermediate kept,
    # no recomputation), projection precision of the forward, owner-computes
    # (deterministic) scatter-adds in the reverse pass
    ("rollout64", dict(kind="rollout64", n=64), 64, 8, 0, False),
    ("rollout64_no_recompute", dict(kind="rollout64", n=64), 64, 64, 0, False),
    ("plume128", dict(kind="plume3d", n=128), 200, 14, 0, False),
    # the inverse-control configuration: mixed-precision forward (FP16 coarse
    # corrections), the recorded refinement steps transposed in the adjoint
    ("plume128_mixed", dict(kind="plume3d", n=128), 200, 14, 1, False),
    # the same with every intermediate kept (25 GB of records at 128^3: HBM
    # holds them, so nothing is recomputed)
    ("plume128_mixed_no_recompute", dict(kind="plume3d", n=128), 200, 200, 1, False),
    ("plume128_deterministic", dict(kind="plume3d", n=128), 200, 14, 0, True),
]
# cases whose forward pass also stores every step's solved pressure, so the
# reverse pass recomputes segments without solving (ss_adjoint_set_pressure_store)
PRESSURE_STORE_CASES = [
    ("plume128_mixed_pressure_store", dict(kind="plume3d", n=128), 200, 14, 1, False),
]


def adjoint_bench(torch, stream):
    """Forward rollout with checkpoints + reverse pass (ss_adjoint_*) against
    the plain forward steps of the same scene: FP32 (or mixed-precision)
    projection with the corrected operators, 4 V-cycles (refinement steps) per
    step, L2 loss on the final density."""
    from smokesim_b200 import Sim, abi, scene
    from smokesim_b200.adjoint import Rollout
    out = {}
    cases = [c + (False,) for c in ADJOINT_CASES] + [c + (True,) for c in PRESSURE_STORE_CASES]
    for name, sa, nsteps, every, prec, det, pstore in cases:
        sc = scene.rollout64(seed=0, n=sa["n"]) if sa["kind"] == "rollout64" else scene.plume3d(seed=0, n=sa["n"])
        sc.pop("rng", None)
        p = scene.workload_params(ref_quirks=0, n_vcycles=4, collect_stats=0, precision=prec)
        cells = sa["n"] ** 3
        forces = np.zeros((nsteps, 3), np.float32)
        forces[:, 1] = 0.5
        e0, e_mid, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        # plain forward steps
        sim = Sim(sc["desc"], stream=stream.cuda_stream)
        scene.apply(sim, sc)
        sim.set_emitter_force((0.0, 0.5, 0.0))
        sim.step(p, 3)
        torch.cuda.synchronize()
        e0.record(stream)
        sim.step(p, nsteps)
        e1.record(stream)
        torch.cuda.synchronize()
        fwd_ms = e0.elapsed_time(e1) / nsteps
        sim.close()
        # rollout with checkpoints + reverse pass (the first repetition warms up;
        # the reverse pass leaves the simulation in the rollout's initial state)
        sim = Sim(sc["desc"], stream=stream.cuda_stream)
        scene.apply(sim, sc)
        ro = Rollout(sim, nsteps, every, deterministic=det, store_pressure=pstore)
        rho = torch.empty(abi.field_count(3, sim.n, abi.FIELD_DENSITY), device="cuda")
        for _ in range(2):
            torch.cuda.synchronize()
            e0.record(stream)
            ro.forward(p, forces, stream=stream.cuda_stream)
            e_mid.record(stream)
            sim.L.ss_get_field_device(sim.h, abi.FIELD_DENSITY, C.c_void_p(rho.data_ptr()), rho.numel(),
                                      C.c_void_p(stream.cuda_stream))
            with torch.cuda.stream(stream):
                gd = (2.0 * (rho - 0.1)).contiguous()
            ro.backward(p, grad_density=gd.data_ptr(), stream=stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
        f_ms = e0.elapsed_time(e_mid) / nsteps
        fb_ms = e0.elapsed_time(e1) / nsteps
        info = ro.info()
        ro.close()
        sim.close()
        out[name] = {"grid": [sa["n"]] * 3, "steps": nsteps, "checkpoint_every": every,
                     "precision": "mixed (f16 coarse)" if prec else "f32",
                     "scatter": "owner-computes" if det else "atomic",
                     "recompute": ("segments replay the stored pressures (no solve)" if pstore else
                                   "segments re-run every stage") if every < nsteps else "none",
                     "forward_ms_per_step": fwd_ms, "forward_with_checkpoints_ms_per_step": f_ms,
                     "fwd_adjoint_ms_per_step": fb_ms, "fwd_adjoint_over_forward": fb_ms / fwd_ms,
                     "fwd_adjoint_mcell_steps_per_s": cells / (fb_ms / 1e3) / 1e6,
                     "reverse_kernel_launches": info["kernel_launches"],
                     "checkpoint_bytes": info["checkpoint_bytes"], "workspace_bytes": info["workspace_bytes"]}
    return out


def config_runs(torch, stream, cpu):
    """The plain-method configurations at their own sizes and step counts
    (FP32, 4 V-cycles of 2+2 sweeps to 8, the reference's boundary rules):
    the 2D 256^2 plume for 200 steps and the 3D 128^3 plume for 500 steps,
    timed with CUDA events on the simulation's stream after 5 warm-up steps,
    each with the C/OpenMP oracle on a bounded sample of the same steps."""
    from smokesim_b200 import Sim, scene
    out = {}
    for name, sc, steps, sample in (("plume2d_256", scene.plume2d(seed=0, n=256), 200, 20),
                                    ("plume3d_128", scene.plume3d(seed=0, n=128), 500, 4)):
        sc.pop("rng", None)
        p = sc["params"]
        sim = Sim(sc["desc"], stream=stream.cuda_stream)
        scene.apply(sim, sc)
        sim.step(p, 5)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.step(p, steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        n = sc["desc"].n
        cells = n[0] * n[1] * (n[2] if sc["desc"].dim == 3 else 1)
        line = {"grid": [n[0], n[1]] + ([n[2]] if sc["desc"].dim == 3 else []), "steps": steps,
                "ms_per_step": ms, "mcell_steps_per_s": cells / (ms / 1e3) / 1e6,
                "schedule": "FP32, 4 V-cycles, 2+2 sweeps, 80 coarsest, down to 8, reference boundary rules"}
        sim.close()
        if cpu:
            cv, csec, threads, _ = cpu_step_rate(sc, sample, 1)
            line["cpu_baseline"] = {"value": cv, "unit": UNIT, "cores": threads, "kind": "port",
                                    "ms_per_step": csec * 1e3,
                                    "sample": f"median of {sample} steps after 1 warm-up from the initial state"}
        out[name] = line
    return out


def inverse_control(args, torch, stream):
    """Inverse control on the plume scene: per-step 3-vector emitter forces and
    a 16^3 coarse force field, fitted with Adam (lr 1e-2) so that the final
    density after --inverse-steps steps matches a target run whose emitters
    are moved 10 cells apart in x.  Mixed-precision projection (FP16 coarse
    corrections, tolerance 1e-6) in the forward; the adjoint transposes the
    recorded refinement steps; checkpoints every ~sqrt(steps)."""
    from smokesim_b200 import Sim, abi, scene
    from smokesim_b200.adjoint import Rollout
    n, nsteps, iters, nf = args.inverse_n, args.inverse_steps, args.inverse_iters, 16
    every = max(1, int(round(nsteps ** 0.5)))
    p = scene.workload_params(ref_quirks=0, precision=abi.PREC_MIXED, tol=1e-6, n_vcycles=40, collect_stats=0)
    sc = scene.plume3d(seed=0, n=n)
    sc.pop("rng", None)
    tgt = scene.plume3d(seed=0, n=n)
    tgt.pop("rng", None)
    tgt["emitters"][0].pos[0] -= 5.0
    tgt["emitters"][1].pos[0] += 5.0
    free0, total = torch.cuda.mem_get_info()
    ts = Sim(tgt["desc"], stream=stream.cuda_stream)
    scene.apply(ts, tgt)
    ts.step(p, nsteps)
    rho_t = torch.from_numpy(ts.get_field(abi.FIELD_DENSITY).ravel()).cuda()
    ts.close()
    sim = Sim(sc["desc"], stream=stream.cuda_stream)
    scene.apply(sim, sc)
    ro = Rollout(sim, nsteps, every, store_pressure=True)
    forces = torch.zeros((nsteps, 3), dtype=torch.float32, requires_grad=True)
    field = torch.zeros((3, nf, nf, nf), dtype=torch.float32, requires_grad=True)
    opt = torch.optim.Adam([forces, field], lr=1e-2)
    rho = torch.empty(abi.field_count(3, sim.n, abi.FIELD_DENSITY), device="cuda")
    losses, ms = [], []
    peak_used = 0
    e0, e_mid, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    fwd_ms, bwd_ms = [], []
    for it in range(iters):
        sim.set_force_field(field.detach().numpy())
        torch.cuda.synchronize()
        e0.record(stream)
        ro.forward(p, forces.detach().numpy(), stream=stream.cuda_stream)
        e_mid.record(stream)
        sim.L.ss_get_field_device(sim.h, abi.FIELD_DENSITY, C.c_void_p(rho.data_ptr()), rho.numel(),
                                  C.c_void_p(stream.cuda_stream))
        with torch.cuda.stream(stream):
            diff = rho - rho_t
            loss = float((diff * diff).sum())
            gd = (2.0 * diff).contiguous()
        gf = ro.backward(p, grad_density=gd.data_ptr(), stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        fwd_ms.append(e0.elapsed_time(e_mid) / nsteps)
        bwd_ms.append(e0.elapsed_time(e1) / nsteps)
        peak_used = max(peak_used, free0 - torch.cuda.mem_get_info()[0])
        losses.append(loss)
        forces.grad = torch.from_numpy(np.ascontiguousarray(gf, dtype=np.float32))
        field.grad = torch.from_numpy(ro.force_field_grad(nf))
        opt.step()
        opt.zero_grad()
    info = ro.info()
    ro.close()
    sim.close()
    return {"inverse_control": {
        "grid": [n] * 3, "steps": nsteps, "checkpoint_every": every, "iterations": iters,
        "controls": f"{nsteps} x 3 emitter forces + 3 x {nf}^3 force field", "optimizer": "Adam lr 1e-2",
        "precision": "mixed (f64 residual/refinement, f16 coarse), tolerance 1e-6",
        "recompute": "checkpoint every ~sqrt(steps) steps; segments recomputed with the stored per-step pressures",
        "loss_first": losses[0], "loss_last": losses[-1], "loss_min": min(losses),
        "loss_curve": losses,
        "forward_with_checkpoints_ms_per_step": float(np.median(fwd_ms)),
        "fwd_adjoint_ms_per_step": float(np.median(bwd_ms)),
        "device_bytes_in_use_peak": int(peak_used),
        "checkpoint_bytes": info["checkpoint_bytes"], "workspace_bytes": info["workspace_bytes"]}}


# The CPU-baseline leg steps the oracle PARITY_STEPS times from the initial
# state and times the last CPU_TIMED of them (past the steps of the start-up
# transient, which take several times the refinement steps); the parity block
# compares a GPU run of the same steps with the oracle's final state.
PARITY_STEPS = 6
CPU_TIMED = 3


def step_parity(sc, o, stream):
    """PARITY_STEPS steps of a fresh GPU simulation of the workload against the
    oracle `o` after the same steps from the same initial state (from the
    third on they start from the extrapolated warm start): every field bit for
    bit, plus the largest absolute difference and the relative L2 per field."""
    from smokesim_b200 import Sim, abi
    g = Sim(sc["desc"], stream=stream.cuda_stream)
    from smokesim_b200 import scene
    scene.apply(g, sc)
    for _ in range(PARITY_STEPS):
        step1(g, sc["params"])
    out = {"steps": PARITY_STEPS, "fields_equal": True, "max_abs": 0.0, "rel_l2": 0.0, "per_field": {}}
    names = {abi.FIELD_VX: "vx", abi.FIELD_VY: "vy", abi.FIELD_VZ: "vz", abi.FIELD_DENSITY: "density",
             abi.FIELD_TEMPERATURE: "temperature", abi.FIELD_PRESSURE: "pressure"}
    for f, name in names.items():
        a = g.get_field(f).astype(np.float64).ravel()
        b = o.get_field(f).astype(np.float64).ravel()
        eq = bool(np.array_equal(a, b))
        mx = float(np.max(np.abs(a - b))) if a.size else 0.0
        den = float(np.linalg.norm(b))
        rl = float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))
        out["per_field"][name] = {"equal": eq, "max_abs": mx, "rel_l2": rl}
        out["fields_equal"] = out["fields_equal"] and eq
        out["max_abs"] = max(out["max_abs"], mx)
        out["rel_l2"] = max(out["rel_l2"], rl)
    sg, so = g.stats(), o.stats()
    out["vcycles"] = [sg.vcycles, so.vcycles]
    out["div_after_rel_diff"] = abs(sg.div_after - so.div_after) / max(1e-300, abs(so.div_after))
    g.close()
    return out


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

    def barrier():
        if world > 1:
            dist.barrier()

    if args.inverse:
        out = inverse_control(args, torch, stream)
        print(json.dumps(out))
        return 0

    if args.profile_adjoint:
        from smokesim_b200.adjoint import Rollout
        sc = scene.plume3d(seed=0, n=args.n)
        sc.pop("rng", None)
        p = scene.workload_params(ref_quirks=0, n_vcycles=4, collect_stats=0)
        sim = Sim(sc["desc"], stream=stream.cuda_stream)
        scene.apply(sim, sc)
        ro = Rollout(sim, 4, 2)
        forces = np.zeros((4, 3), np.float32)
        forces[:, 1] = 0.5
        ro.forward(p, forces, stream=stream.cuda_stream)
        rho = torch.ones(abi.field_count(3, sim.n, abi.FIELD_DENSITY), device="cuda")
        torch.cuda.synchronize()
        ro.backward(p, grad_density=rho.data_ptr(), stream=stream.cuda_stream)
        torch.cuda.synchronize()
        print(json.dumps({"profile_adjoint": "done", "reverse": ro.info()}))
        return 0

    with torch.cuda.stream(stream):
        if args.profile:
            sim = Sim(sc["desc"], stream=stream.cuda_stream)
            scene.apply(sim, sc)
            sim.step(sc["params"], args.profile_steps)
            sim.smooth(sc["params"], 0, 2)
            torch.cuda.synchronize()
            print(json.dumps({"profile": "done", "levels": sim.level_sizes}))
            return 0

        variants = {}
        clocks = None
        for name in [HEADLINE] + [v for v in VARIANTS if v != HEADLINE]:
            if name == HEADLINE:
                clk = ClockSampler(local)
                clk.start()
            sim, p, out = run_variant(torch, Sim, scene, sc, name, args, stream, barrier, world, dev)
            if name == HEADLINE:
                clocks = clk.stop()
                head_sim, head_p = sim, p
            else:
                sim.close()
            out["value"] = job_rate(world, cells, 1, out["ms_per_step"])
            variants[name] = out
        head = variants[HEADLINE]
        value = head["value"]
        sim, p = head_sim, head_p

        # end to end through the C ABI on the headline variant, from the same
        # initial state and over the same steps as the timed run (a fresh
        # simulation of the scene, the same warm-up): per step the emitter
        # records go host->device (ss_run_physics_step uploads them) and the
        # step's statistics (divergence norms) come back device->host; wall
        # clock around the steps, synchronised on both sides
        sim.close()
        sim = Sim(sc["desc"], stream=stream.cuda_stream)
        scene.apply(sim, sc)
        for _ in range(args.warmup):
            step1(sim, p)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        vc = 0
        for _ in range(args.steps):
            step1(sim, p)
            vc += sim.stats().vcycles
        torch.cuda.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t0, world, dev)
        e2e = {"value": job_rate(world, cells, args.steps, e2e_s * 1e3), "unit": UNIT,
               "h2d_bytes_per_step": C.sizeof(abi.Emitter) * len(sc["emitters"]),
               "d2h_bytes_per_step": C.sizeof(abi.Stats), "vcycles_mean": vc / max(1, args.steps),
               "api": "ss_run_physics_step + ss_get_stats per step (smokesim_b200.Sim), wall clock"}

        # roofline of the dominant kernel: the level-0 red-black smoother
        # (k_rb_smooth4, one colour per launch on the colour-split arrays).
        # 13 B/cell per red+black sweep (read/write p, read rhs, read mask).
        reps = 10
        ps = variant_params(sc, "fp32")
        sim.smooth(ps, 0, 1)
        torch.cuda.synchronize()
        a0, a1, b0, b1 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        a0.record(stream)
        sim.smooth(ps, 0, 1)
        a1.record(stream)
        b0.record(stream)
        sim.smooth(ps, 0, 1 + reps)
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
        roofline = {"kernel": f"k_rb_smooth4<3> (one colour of a level-0 red-black sweep, {args.n}^3)", "bound": "hbm",
                    "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                    "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": launch_ms,
                    "traffic": RB_SMOOTH_TRAFFIC if args.n == 256 else None}

    # headless ray-marched frame of the final 256^3 smoke (k_raymarch), 1024x1024
    render = None
    with torch.cuda.stream(stream):
        d = sim.render_desc(1024, 1024)
        img = torch.empty(1024 * 1024 * 4, dtype=torch.uint8, device=dev)
        for _ in range(2):
            sim.L.ss_render(sim.h, C.byref(d), C.c_void_p(img.data_ptr()), 1, C.c_void_p(stream.cuda_stream))
        r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        r0.record(stream)
        for _ in range(5):
            sim.L.ss_render(sim.h, C.byref(d), C.c_void_p(img.data_ptr()), 1, C.c_void_p(stream.cuda_stream))
        r1.record(stream)
        torch.cuda.synchronize()
        render = {"image": [1024, 1024], "ms_per_frame": r0.elapsed_time(r1) / 5,
                  "step_size": d.step_size, "shadow_steps": d.shadow_steps}

    adjoint = None
    inverse = None
    configs = None
    if not args.no_adjoint and world == 1:
        adjoint = adjoint_bench(torch, stream)
        inverse = inverse_control(args, torch, stream)["inverse_control"]
    if world == 1:
        configs = config_runs(torch, stream, rank == 0 and not args.no_cpu_baseline)

    line = {
        "impl": "b200", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (f64 residual/refinement, f16 coarse storage)",
        "data": "synthetic (seeded scene + GRF)",
        "config": workload_config(args, sc), "gpu_launches": int(head["gpu_launches"]), "clocks": clocks,
        "variants": variants,
        "configs": configs,
        "adjoint": adjoint,
        "inverse_control": inverse,
        "render": render,
        "e2e": e2e, "roofline": roofline,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cv, csec, threads, o = cpu_step_rate(sc, CPU_TIMED, PARITY_STEPS - CPU_TIMED)
        line["cpu_baseline"] = {"value": cv, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"median of full {args.n}^3 steps {PARITY_STEPS - CPU_TIMED + 1}.."
                                          f"{PARITY_STEPS} of the same variant from the initial state, C/OpenMP "
                                          f"oracle (refinement steps of each in vcycles; the timed GPU steps come "
                                          f"later in the run and take fewer)",
                                "vcycles": list(cpu_step_rate.vcycles)}
        line["parity"] = step_parity(sc, o, stream)
    if rank == 0:
        print(json.dumps(line), flush=True)
    sim.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
