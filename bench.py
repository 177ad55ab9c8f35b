#!/usr/bin/env python
"""Benchmark of the SPH fluid step: particle-steps/s at 4M particles.

Workload: the precision-form dam break — a 128x256x128 jittered lattice
(4,194,304 particles, spacing h/2 = 0.1, SphParams::defaults() with bounds
[0, 51.2]^3, dt = 0.0025).  One "step" is one FluidWorld::step of the whole
scene.  The headline `value` is the FP32-compensated step with the state
resident in HBM; the f64 plain step is timed on the same scene beside it,
together with the compensated form's density error against it (the f64 plain
step is bit-identical to the f64 oracle).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 (under torchrun) every rank steps its own replica of the
scene: the single-scene step does not shard ("replicas only"), so value is
N x particles x K / (max over ranks of the timed region).  The batched form's
scenes are independent and are partitioned across the ranks by particle count
instead (its "batched" block: the whole batch's particle-steps over the max
over ranks).

--impl reference times the CPU restatement of the reference's rayon step
(oracle/, OpenMP over all host threads) on the same 4,194,304-particle scene,
without loading the product library; the Rust reference itself cannot be
built here.

Output: auxiliary blocks first, one JSON object per line with a "block" key
(precision errors along the trajectory, full trajectory, readback, batched,
adjoint, coupling); the headline object is the last line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SPH particle-steps/s @4M: FP32-comp vs f64 plain on B200 (density err <=1e-5)"
UNIT = "particle-steps/s"
DIMS = (128, 256, 128)
BOX = 51.2
DT = 0.0025

# Algorithmic bytes of the force pass per particle (compulsory traffic of its
# own arrays, each touched once; neighbour reads are reuse, not compulsory):
#   f64 form:  reads pos+vel (48), rho, p/rho^2, m/rho, mass (32), material (4);
#              writes pos+vel (48), acc (24), xsph (24), mu_eff (8)       = 188
#   f32c form: reads pos+vel (48), rho (8), material (4), packed f32 operands
#              cpos (16), cvel (16), m/rho (4); writes as above (104)      = 200
FORCE_BYTES = {"f64": 188, "comp": 200}
# DRAM traffic of one k_force_tiled launch per particle, dram__bytes_read.sum +
# dram__bytes_write.sum from an ncu capture of the 80x160x80 dam break (the
# 4M launch is larger than an ncu capture should be); at constant density the
# traffic grows with the particle count, so a full launch is scaled by it.
FORCE_TRAFFIC_PER_PARTICLE = (239.449344e6 + 80.680448e6) / 1024000
# Kernels one compensated step launches: the sort (tile histogram, the sums
# of the tile counts and occupied tiles per scan tile, their scan with the
# tile list, scatter by tile, per-tile cells and order, order of large cells,
# gather) and the passes (tiled and dense-cell density, tiled and dense-cell
# force).
LAUNCHES_PER_STEP = 7 + 4
# Whole-step compulsory state traffic (f64 pos, vel, mass in; pos, vel, rho, p out):
# the algorithmic bytes of one particle-step.
STEP_BYTES = 120
# Steps of the configured 1000-step trajectory at which the compensated form's
# per-output errors are probed (teacher-forced from that state), the last one in
# the collapsed regime.
PROBE_FRACTIONS = (0.0, 0.25, 0.5, 0.75, 1.0)


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def peaks():
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms."""

    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(gpu_index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[4 + k].lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


# Algorithmic flops of one particle-step: the candidate test (~8 flops: three
# differences, a sum of squares, a compare) in each of the two passes, the
# density term (~12) and the force terms (~60: distance, pressure, viscosity,
# XSPH, strain rate) per in-range pair, with candidates and pairs counted on the
# device (phy_fluid_step_counters).
FLOPS_PER_CANDIDATE_PASS = 8
FLOPS_PER_PAIR = 12 + 60


def flop_rate(counters: dict, n: int, step_ms: float) -> dict:
    """The flop side of the step's roofline: algorithmic flops per particle-step from the
    device counters of one counted step, and the rate they imply at step_ms per step.  No
    FP32 CUDA-core peak is measured on this hardware, so no fraction is formed."""
    c = counters["candidates"] / n if n else 0.0
    p = counters["pairs"] / n if n else 0.0
    per = 2 * FLOPS_PER_CANDIDATE_PASS * c + FLOPS_PER_PAIR * p
    return {"flops_per_particle_step": per, "candidates_per_particle": c, "pairs_per_particle": p,
            "achieved_tflops": per * n / (step_ms / 1e3) / 1e12 if step_ms > 0 else None,
            "peak": None, "unit": "TFLOP/s"}


def bench_config(dims, n: int, world_size: int) -> dict:
    """The workload both arms run (the precision of each arm is its line's dtype)."""
    return {"workload": f"dam_break_{dims[0]}x{dims[1]}x{dims[2]}: {n} particles, spacing 0.1 = h/2, "
                        f"bounds [0,{BOX}]^3, dt={DT}",
            "particles": n,
            "parallelism": f"replicas x{world_size}",
            "l2": "inputs larger than L2 (state ~1.4 GB per replica)"}


def make_params(pb):
    p = pb.SphParams.defaults()
    p.bounds_min, p.bounds_max = (0.0, 0.0, 0.0), (BOX, BOX, BOX)
    return p


BATCH_DT = 0.005
BATCH_CHUNK = 10  # steps per captured CUDA graph


def run_batched(pb, scenes, stream, n_scenes: int, steps: int, warmup: int, rank: int = 0, world_size: int = 1,
                max_over_ranks=lambda x: x, barrier=lambda: None) -> dict:
    """The batched form: n_scenes independent dam breaks (log-uniform 2k..200k particles,
    aspect U[0.5,2], fill U[0.2,0.5]) in one world, one sort and one persistent launch per
    pass, steps captured in CUDA graphs, launch knobs from the library's autotuner; against
    looping the single-scene step over the same scenes (each scene its own world and
    phy_fluid_step call).  With several ranks the scenes are partitioned across them by
    particle count (no collective in the step); times are the max over ranks and the
    values count every rank's particles (strong scaling: the batch is fixed)."""
    import torch
    every = scenes.batch_scenes(n_scenes)
    total_all = int(sum(b.n for b in every))
    parts = scenes.partition_scenes([b.n for b in every], world_size)
    if any(not part for part in parts):
        raise ValueError("the batched form needs at least one scene per rank")
    batch = [every[i] for i in parts[rank]]
    counts = [b.n for b in batch]
    total = int(sum(counts))
    mass = scenes.lattice_mass(scenes.SPACING)
    p = pb.SphParams.defaults()
    w = pb.FluidWorld(p, "comp")
    w.set_stream(stream.cuda_stream)
    w.add_particles(np.concatenate([b.pos for b in batch]), np.full(total, mass))
    w.set_scenes(counts, [b.bounds_min for b in batch], [b.bounds_max for b in batch])
    w.set_tuning(graph_chunk=BATCH_CHUNK)
    t0 = time.time()
    # Tuned over the run ahead: the states at 0, steps/2 and steps steps.
    trials = w.autotune(BATCH_DT, BATCH_CHUNK, horizon=steps)
    tune_s = time.time() - t0
    chosen = w.tuning()
    finalists = [t for t in trials if t["samples"] == max(t["samples"] for t in trials)]

    def timed(fn, k):
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn(k)
        e1.record(stream)
        e1.synchronize()
        return max_over_ranks(e0.elapsed_time(e1))

    w.step(BATCH_DT, max(warmup, BATCH_CHUNK))
    ms = timed(lambda k: w.step(BATCH_DT, k), steps)
    # The same batch without graph capture.
    w.set_tuning(graph_chunk=0)
    k_eager = max(BATCH_CHUNK, steps // 4)
    ms_eager = timed(lambda k: w.step(BATCH_DT, k), k_eager)
    del w
    # Looping the single-scene step: one world per scene, default configuration.
    worlds = []
    for b in batch:
        q = pb.SphParams.defaults()
        q.bounds_min, q.bounds_max = b.bounds_min, b.bounds_max
        ws = pb.FluidWorld(q, "comp")
        ws.set_stream(stream.cuda_stream)
        ws.add_particles(b.pos, np.full(b.n, mass))
        worlds.append(ws)
    for ws in worlds:
        ws.step(BATCH_DT, warmup)

    def loop(k):
        for ws in worlds:
            ws.step(BATCH_DT, k)

    ms_loop = timed(loop, steps)
    del worlds
    value = total_all * steps / (ms / 1e3)
    loop_value = total_all * steps / (ms_loop / 1e3)
    return {
        "workload": f"{n_scenes} dam-break scenes, {total_all} particles (log-uniform 2000..200000 per scene, "
                    f"aspect U[0.5,2], fill U[0.2,0.5]), dt={BATCH_DT}, FP32-compensated",
        "scenes": n_scenes,
        "particles": total_all,
        "ranks": world_size,
        "scaling": "strong (the scenes are partitioned across ranks by particle count)",
        "particles_rank0": total if rank == 0 else None,
        "steps": steps,
        "value": value,
        "unit": UNIT,
        "ms_per_step": ms / steps,
        "graph_chunk": BATCH_CHUNK,
        "eager_value": total_all * k_eager / (ms_eager / 1e3),
        "loop_single_scene_value": loop_value,
        "loop_single_scene_ms_per_step": ms_loop / steps,
        "speedup_vs_loop": value / loop_value,
        "tuning": {k: chosen[k] for k in ("comp_tile", "ctas_per_sm", "queue", "sort_block", "graph_chunk")},
        "autotune": {"trials": len(trials), "finalists": len(finalists), "horizon_steps": steps,
                     "seconds": tune_s,
                     "best_ms_per_step": min(t["ms_per_step"] for t in finalists),
                     "worst_finalist_ms_per_step": max(t["ms_per_step"] for t in finalists),
                     "best_over_timed": min(t["ms_per_step"] for t in finalists) / (ms / steps)},
    }


ADJ_DIMS = (32, 64, 32)
ADJ_BOX = 12.8
ADJ_DT = 0.005
ADJ_STEPS = 100
ADJ_EVERY = 10


def adjoint_problem(scenes, seed: int = 64):
    """The differentiation form: 64k-particle dam break, initial velocities f32-drawn
    N(0, 0.1^2), target = initial lattice + (0.5, 0, 0) + N(0, 0.01^2)."""
    pos = scenes.dam_break_positions(*ADJ_DIMS)
    rng = np.random.default_rng(seed)
    v0 = (rng.standard_normal(pos.shape, dtype=np.float32) * np.float32(0.1)).astype(np.float64)
    target = pos + np.array([0.5, 0.0, 0.0]) + rng.normal(0.0, 0.01, pos.shape)
    return pos, v0, target


def run_adjoint(pb, scenes, stream, directions: int) -> dict:
    """step_backward on the differentiation form: device time of the 100-step forward, of
    the recorded forward and of the reverse sweep (checkpoint every 10 steps, segments
    re-run forward), and the gradient against central finite differences (eps = 1e-4)
    of the same f64 plain forward on `directions` random unit directions."""
    import torch
    pos, v0, target = adjoint_problem(scenes)
    n = pos.shape[0]
    mass = scenes.lattice_mass(scenes.SPACING)

    def world(v, stiffness=None, visc=None, form="f64"):
        p = pb.SphParams.defaults()
        p.bounds_min, p.bounds_max = (0.0, 0.0, 0.0), (ADJ_BOX, ADJ_BOX, ADJ_BOX)
        if stiffness is not None:
            p.stiffness = stiffness
        if visc is not None:
            p.visc_k = [visc]
        w = pb.FluidWorld(p, form)
        w.set_stream(stream.cuda_stream)
        w.add_particles(pos, mass, vel=v)
        return w

    def loss(x):
        return float(np.mean(np.sum((x - target) ** 2, axis=1)))

    def timed(fn):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    warm = world(v0)
    warm.step(ADJ_DT, 10)
    w = world(v0)
    fwd_ms, _ = timed(lambda: w.step(ADJ_DT, ADJ_STEPS))
    w = world(v0)
    w.tape_begin(ADJ_EVERY)
    taped_ms, _ = timed(lambda: w.step(ADJ_DT, ADJ_STEPS))
    xT = w.pos
    L = loss(xT)
    gx = 2.0 * (xT - target) / n
    w.step_backward(gx, None)  # warm-up sweep (allocations)
    t0 = time.perf_counter()
    bwd_ms, g = timed(lambda: w.step_backward(gx, None))
    bwd_wall_ms = (time.perf_counter() - t0) * 1e3
    del w, warm

    def run_loss(v, **kw):
        q = world(v, **kw)
        q.step(ADJ_DT, ADJ_STEPS)
        return loss(q.pos)

    eps = 1e-4
    rng = np.random.default_rng(7)
    errs = []
    for _ in range(directions):
        d = rng.normal(size=v0.shape)
        d /= np.linalg.norm(d)
        fd = (run_loss(v0 + eps * d) - run_loss(v0 - eps * d)) / (2 * eps)
        errs.append(abs(float(np.sum(g["vel"] * d)) - fd) / abs(fd))
    fd_visc = (run_loss(v0, visc=3.5 + eps) - run_loss(v0, visc=3.5 - eps)) / (2 * eps)
    hk = 250.0 * eps
    fd_stiff = (run_loss(v0, stiffness=250.0 + hk) - run_loss(v0, stiffness=250.0 - hk)) / (2 * hk)

    # The same on the FP32-compensated world (its adjoint differentiates the step along
    # the compensated trajectory through f64 records of each state).
    cw = world(v0, form="comp")
    cw.step(ADJ_DT, 10)
    cw = world(v0, form="comp")
    cfwd_ms, _ = timed(lambda: cw.step(ADJ_DT, ADJ_STEPS))
    cw = world(v0, form="comp")
    cw.tape_begin(ADJ_EVERY)
    cw.step(ADJ_DT, ADJ_STEPS)
    cxT = cw.pos
    cgx = 2.0 * (cxT - target) / n
    cw.step_backward(cgx, None)
    cbwd_ms, cg = timed(lambda: cw.step_backward(cgx, None))
    del cw

    def run_closs(v):
        q = world(v, form="comp")
        q.step(ADJ_DT, ADJ_STEPS)
        return loss(q.pos)

    # Central differences of the smooth f64 map (eps 1e-4), and of the compensated forward
    # itself at eps 1e-2 (at 1e-4 its f32 rounding scatters them by ~1e-3 relative around
    # any smooth gradient): the compensated and the f64 adjoint's distances from the latter.
    cerrs, cspread = [], []
    for _ in range(min(directions, 8)):
        d = rng.normal(size=v0.shape)
        d /= np.linalg.norm(d)
        fd = (run_loss(v0 + eps * d) - run_loss(v0 - eps * d)) / (2 * eps)
        cerrs.append(abs(float(np.sum(cg["vel"] * d)) - fd) / abs(fd))
        fc = (run_closs(v0 + 1e-2 * d) - run_closs(v0 - 1e-2 * d)) / 2e-2
        cspread.append((abs(float(np.sum(cg["vel"] * d)) - fc) / abs(fc),
                        abs(float(np.sum(g["vel"] * d)) - fc) / abs(fc)))
    comp = {"forward_ms": cfwd_ms, "backward_ms": cbwd_ms, "backward_over_forward": cbwd_ms / cfwd_ms,
            "fd_directions": len(cerrs), "fd_of": "f64 map, eps 1e-4",
            "fd_max_rel_err": max(cerrs), "fd_median_rel_err": float(np.median(cerrs)),
            "grad_rel_diff_vs_f64_adjoint": float(np.linalg.norm(cg["vel"] - g["vel"]) / np.linalg.norm(g["vel"])),
            "comp_fd_eps": 1e-2,
            "comp_fd_max_rel_err": max(a for a, _ in cspread),
            "comp_fd_max_rel_err_of_f64_adjoint": max(b for _, b in cspread)}
    return {
        "workload": f"dam_break_{ADJ_DIMS[0]}x{ADJ_DIMS[1]}x{ADJ_DIMS[2]}: {n} particles, {ADJ_STEPS} steps at "
                    f"dt={ADJ_DT}, checkpoint every {ADJ_EVERY}; loss = mean |x_T - target|^2",
        "particles": n,
        "loss": L,
        "forward_ms": fwd_ms,
        "recorded_forward_ms": taped_ms,
        "backward_ms": bwd_ms,
        "backward_wall_ms": bwd_wall_ms,
        "backward_over_forward": bwd_ms / fwd_ms,
        "fd_directions": directions,
        "fd_eps": eps,
        "fd_max_rel_err": max(errs),
        "fd_median_rel_err": float(np.median(errs)),
        "grad_visc_k0": g["visc_k0"],
        "fd_visc_k0_rel_err": abs(g["visc_k0"] - fd_visc) / abs(fd_visc),
        "grad_stiffness": g["stiffness"],
        "fd_stiffness_rel_err": abs(g["stiffness"] - fd_stiff) / abs(fd_stiff),
        "fd_stiffness_step": hk,
        "comp": comp,
    }


def probe_errors(pb, new_world, w, n: int, params) -> dict:
    """Per-output error of one FP32-compensated step against one f64 plain step (itself
    bit-identical to the f64 oracle), both started from the state of world `w`
    (teacher-forced): density and acceleration (the force per unit density,
    world.rs:332-336) as max relative / max-normalised errors, pressure normalised by
    k*rho0 (p is ~0 near rest), position and velocity after the step."""
    pos, vel = w.pos.copy(), w.vel.copy()
    plain = new_world("f64", pos, vel)
    comp = new_world("comp", pos, vel)
    plain.step(DT)
    comp.step(DT)
    rp, rc = plain.rho, comp.rho
    live = np.abs(rp) > 0
    ap, ac = plain.acc, comp.acc
    amag = np.linalg.norm(ap, axis=1)
    aerr = np.linalg.norm(ac - ap, axis=1)
    amax = float(amag.max()) if n else 0.0
    big = amag > 1e-3 * amax
    xp, xc = plain.pos, comp.pos
    vp, vc = plain.vel, comp.vel
    vmax = float(np.linalg.norm(vp, axis=1).max())
    out = {
        "density_max_rel": float(np.max(np.abs(rc[live] - rp[live]) / np.abs(rp[live]))),
        "pressure_max_norm": float(np.max(np.abs(comp.p - plain.p)) / (params.stiffness * params.rest_density)),
        "acc_max_norm": float(aerr.max() / amax) if amax > 0 else 0.0,
        "acc_median_rel": float(np.median(aerr[big] / amag[big])) if big.any() else 0.0,
        "pos_max_abs_m": float(np.max(np.abs(xc - xp))),
        "vel_max_norm": float(np.max(np.linalg.norm(vc - vp, axis=1)) / vmax) if vmax > 0 else 0.0,
    }
    del plain, comp
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist
    import physics_b200 as pb
    from physics_b200 import scenes

    world_size = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    local_rank = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local_rank)
    if world_size > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    def barrier():
        if world_size > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world_size == 1:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def emit(block: str, obj) -> None:
        if rank == 0 and obj is not None:
            print(json.dumps({"block": block, **obj}), flush=True)

    K, W = args.steps, args.warmup
    dims = tuple(args.dims)
    pos = scenes.dam_break_positions(*dims)
    n = pos.shape[0]
    params = make_params(pb)
    stream = torch.cuda.Stream()

    def new_world(prec, p=pos, v=None):
        w = pb.FluidWorld(params, prec)
        w.set_stream(stream.cuda_stream)
        mass = w.lattice_mass(0.1)
        w.add_particles(p, mass, vel=v)
        if args.graph_chunk > 0:
            w.set_tuning(graph_chunk=args.graph_chunk)
        return w

    def timed(w, steps, warmup, sample_clocks=False, phase=False):
        """Device time of `steps` steps (CUDA events on the world's stream); with
        phase=True the world also records per-pass events inside the timed region
        (non-blocking) and their per-step means are returned."""
        w.step(DT, warmup)
        w.synchronize()
        barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(local_rank) if sample_clocks else None
        if sampler:
            time.sleep(0.3)
        if phase:
            w.set_timing(True)
            w.phase_times(reset=True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        w.step(DT, steps)
        e1.record(stream)
        e1.synchronize()
        clocks = sampler.stop() if sampler else None
        ms = max_over_ranks(e0.elapsed_time(e1))
        ph = None
        if phase:
            t = w.phase_times(reset=True)
            w.set_timing(False)
            ph = {k: t[k] / max(t["steps"], 1) for k in ("sort", "prep", "density", "force")}
        barrier()
        return ms, clocks, ph

    # ---- headline: FP32-compensated, state resident in HBM ----------------------------
    comp = new_world("comp")
    ms_comp, clocks, ph_comp = timed(comp, K, W, sample_clocks=(rank == 0), phase=True)
    value = world_size * n * K / (ms_comp / 1e3)

    # ---- the f64 plain step on the same scene ---------------------------------------
    plain = new_world("f64")
    k_plain = max(3, K // 4)
    ms_plain, _, ph_plain = timed(plain, k_plain, max(3, W // 2), phase=True)
    plain_value = world_size * n * k_plain / (ms_plain / 1e3)
    del plain

    comp.set_counting(True)
    comp.step(DT)
    cnt = comp.step_counters()
    comp.set_counting(False)

    # ---- the configured 1000-step trajectory, with per-output error probes ------------
    # Timed in segments between probe points (CUDA events around each segment); a
    # probe reads the state and steps an f64 plain and a compensated world from it
    # outside the timed segments.
    full, errors = None, None
    if args.full_steps > 0:
        traj = new_world("comp")
        probes = sorted({min(int(round(f * args.full_steps)), args.full_steps - 1) for f in PROBE_FRACTIONS})
        errors = {"workload": f"teacher-forced: one f32c step and one f64 plain step from the state of the "
                              f"{args.full_steps}-step trajectory at each listed step",
                  "reference": "f64 plain step (bit-identical to the f64 oracle)", "at_step": {}}
        done, ms_full, segments, seg_clocks = 0, 0.0, [], []
        for s_probe in probes + [args.full_steps]:
            seg = s_probe - done
            if seg > 0:
                ms_seg, clk, _ = timed(traj, seg, 0, sample_clocks=rank == 0)
                ms_full += ms_seg
                segments.append({"steps": [done, s_probe], "ms_per_step": ms_seg / seg,
                                 "sm_mhz": clk["sm_mhz"] if clk else None,
                                 "reasons": clk["reasons"] if clk else None})
                done = s_probe
            if s_probe < args.full_steps and rank == 0:
                errors["at_step"][str(s_probe)] = probe_errors(pb, new_world, traj, n, params)
        full = {"steps": args.full_steps, "value": world_size * n * args.full_steps / (ms_full / 1e3),
                "ms_per_step": ms_full / args.full_steps, "segments": segments}
        traj.set_timing(True)
        traj.phase_times(reset=True)
        traj.step(DT, 20)
        t = traj.phase_times(reset=True)
        traj.set_timing(False)
        full["phase_ms_at_end"] = {k: t[k] / max(t["steps"], 1) for k in ("sort", "prep", "density", "force")}
        traj.set_counting(True)
        traj.step(DT)
        full["pairs_per_particle_at_end"] = traj.step_counters()["pairs"] / n
        traj.set_counting(False)
        full["dense_masks_at_end"] = traj.dense_mask_info()
        del traj
        if rank == 0:
            at = errors["at_step"].values()
            errors["max_over_probes"] = {k: max(e[k] for e in at) for k in next(iter(at))}
    emit("precision_errors", errors)
    emit("full_trajectory", full)

    adjoint = None
    if args.adjoint_directions > 0:
        adjoint = run_adjoint(pb, scenes, stream, args.adjoint_directions)
    emit("adjoint", adjoint)

    batched = None
    if args.batch_scenes > 0 and args.batch_steps > 0:
        batched = run_batched(pb, scenes, stream, args.batch_scenes, args.batch_steps, W, rank, world_size,
                              max_over_ranks, barrier)
    emit("batched", batched)

    # ---- end to end through the C ABI with host buffers ------------------------------
    pin_pos = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    pin_vel = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    comp.synchronize()
    pin_pos[:] = comp.pos
    pin_vel[:] = comp.vel
    ke = max(3, K // 10)
    barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(ke):
        comp.set(pb.FIELD_POS, pin_pos)
        comp.set(pb.FIELD_VEL, pin_vel)
        comp.step(DT)
        comp.get(pb.FIELD_POS, pin_pos.reshape(-1))
        comp.get(pb.FIELD_VEL, pin_vel.reshape(-1))
    f1.record(stream)
    f1.synchronize()
    ms_e2e = max_over_ranks(f0.elapsed_time(f1))
    e2e_value = world_size * n * ke / (ms_e2e / 1e3)

    emit("readback", run_readback(pb, comp, n))

    coupling = None
    if not args.no_coupling and world_size == 1:
        coupling = run_coupling(pb, scenes, comp, n, dims)
    emit("coupling", coupling)

    hbm_peak, peak_kind = peaks()
    force_ms = ph_comp["force"]
    step_ms = ms_comp / K
    # Roofline of the dominant kernel against HBM with the whole step's algorithmic
    # bytes (120 B per particle-step) over the force pass's own event time.
    achieved = STEP_BYTES * n / (force_ms / 1e3) / 1e9
    step_gbs = STEP_BYTES * n / (step_ms / 1e3) / 1e9

    line = None
    if rank == 0:
        cpu = None if (args.no_cpu or world_size > 1) else cpu_baseline(scenes, pb, n, dims)
        err_max = errors["max_over_probes"] if errors else None
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world_size,
            "steps": K,
            "warmup": W,
            "ms_per_step": step_ms,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32c/f64",
            "data": "synthetic (seeded jittered dam-break lattice)",
            "config": bench_config(dims, n, world_size),
            "roofline": {
                "bound": "issue",
                "axis": "hbm",
                "kernel": "k_force_tiled",
                "achieved": achieved,
                "peak": hbm_peak,
                "unit": "GB/s",
                "frac": achieved / hbm_peak,
                "peak_kind": peak_kind,
                "traffic": FORCE_TRAFFIC_PER_PARTICLE * n,
                "bytes_per_particle": STEP_BYTES,
                "kernel_ms": force_ms,
                "step_achieved": step_gbs,
                "step_frac": step_gbs / hbm_peak,
                "force_own_bytes_frac": FORCE_BYTES["comp"] * n / (force_ms / 1e3) / 1e9 / hbm_peak,
            },
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * 24 * n,
                    "d2h_bytes_per_step": 2 * 24 * n, "steps": ke},
            "gpu_launches": LAUNCHES_PER_STEP * K,
            "clocks": clocks,
            "cpu_baseline": cpu,
            # The form-specific results last, the most read at the very end, so that a
            # reader of the output's last characters sees them.
            "phase_ms": {"comp": ph_comp, "plain_f64": ph_plain},
            "flops": flop_rate(cnt, n, step_ms),
            "pairs_per_particle": cnt["pairs"] / n,
            "full_trajectory": {"steps": full["steps"], "ms_per_step": full["ms_per_step"],
                                "value": full["value"]} if full else None,
            "errors_max_over_trajectory": err_max,
            "density_err_max_rel": err_max["density_max_rel"] if err_max else None,
            "plain_f64": {"value": plain_value, "ms_per_step": ms_plain / k_plain, "steps": k_plain},
            "ratio_comp_vs_plain": value / plain_value,
        }
        print(json.dumps(line), flush=True)
    if world_size > 1:
        dist.barrier()
        dist.destroy_process_group()
    return line


def run_readback(pb, w, n: int) -> dict:
    """phy_world_get_fluid_positions (lib.rs:399-429) of the 4M state into a pageable and
    into a pinned (phy_fluid_pin_host) host buffer: host clock per call, 3 calls each."""
    import ctypes as C
    lib = pb._lib.load()
    h = w._h
    out = {}
    for kind in ("pageable", "pinned"):
        buf = np.empty(3 * n, np.float64)
        buf[:] = 0.0  # touch the pages
        if kind == "pinned" and lib.phy_fluid_pin_host(buf.ctypes.data, buf.nbytes) != 0:
            out[kind] = {"error": pb._lib.last_error()}
            continue
        ptr = buf.ctypes.data_as(C.POINTER(C.c_double))
        lib.phy_world_get_fluid_positions(h, ptr, buf.size)
        t0 = time.perf_counter()
        for _ in range(3):
            got = lib.phy_world_get_fluid_positions(h, ptr, buf.size)
        t = (time.perf_counter() - t0) / 3
        if kind == "pinned":
            lib.phy_fluid_unpin_host(buf.ctypes.data)
        out[kind] = {"ms": t * 1e3, "gbs": buf.nbytes / t / 1e9, "particles": int(got)}
    out["workload"] = f"phy_world_get_fluid_positions of {n} particles (f64 xyz, {24 * n} bytes), host clock"
    return out


def run_coupling(pb, scenes, w, n: int, fluid_dims=DIMS) -> dict:
    """The fluid's coupling calls on the 4M state (after the timed steps), each timed by the
    host clock around the call (every call synchronises; the grid / point / body transfers
    are inside), next to the oracle on the 524,288-particle block of the same recipe."""
    from oracle import oracle as O
    O.build()
    rng = np.random.default_rng(17)
    dims = (64, 128, 64)  # heat grid: 0.2-cells over the 12.8 x 25.6 x 12.8 block
    temp = rng.uniform(0.0, 1.0, dims[::-1])
    src = np.zeros_like(temp)
    pts = rng.uniform((0.5, 0.5, 0.5), (12.3, 25.1, 12.3), (4096, 3))
    pvel = rng.normal(0.0, 0.2, pts.shape)
    pmass = np.full(len(pts), 0.02)
    centres = rng.uniform((1.0, 1.0, 1.0), (11.8, 24.6, 11.8), (8, 3))
    bodies = [{"shape": "sphere", "size": (0.5,), "pos": tuple(c), "vel": (0.0, -0.5, 0.0), "inv_mass": 0.01}
              for c in centres]

    def wall(fn, reps=3):
        fn()  # allocations
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        return (time.perf_counter() - t0) / reps

    t_heat = wall(lambda: w.couple_heat(temp, src, (0.0, 0.0, 0.0), 0.2, DT, 0.5, 2e-4, 0.1))
    t_pts = wall(lambda: w.couple_points(pts, pvel, pmass, DT, 1.0, 1000.0))
    t_bod = wall(lambda: w.couple_bodies(bodies, DT))
    # The oracle on the 64 x 128 x 64 block (a quarter of each extent's particles, same spacing).
    sdims = (64, 128, 64)
    spos = scenes.dam_break_positions(*sdims)
    p = pb.SphParams.defaults()
    p.bounds_min, p.bounds_max = (0.0, 0.0, 0.0), (BOX, BOX, BOX)
    ow = O.OracleWorld(p)
    ow.add_particles(spos, scenes.lattice_mass(0.1))
    ns = spos.shape[0]
    sgrid = (32, 64, 32)
    stemp = rng.uniform(0.0, 1.0, sgrid[::-1])
    spts = rng.uniform((0.5, 0.5, 0.5), (5.9, 12.3, 5.9), (1024, 3))
    sbodies = [dict(b, pos=tuple(np.asarray(b["pos"]) * 0.5)) for b in bodies[:4]]
    t0 = time.perf_counter()
    ow.couple_heat(stemp, np.zeros_like(stemp), (0.0, 0.0, 0.0), 0.2, DT, 0.5, 2e-4, 0.1)
    c_heat = time.perf_counter() - t0
    t0 = time.perf_counter()
    ow.couple_points(spts, np.zeros_like(spts), np.full(len(spts), 0.02), DT, 1.0, 1000.0)
    c_pts = time.perf_counter() - t0
    t0 = time.perf_counter()
    ow.couple_bodies(sbodies, DT)
    c_bod = time.perf_counter() - t0
    return {
        "workload": f"dam_break_{fluid_dims[0]}x{fluid_dims[1]}x{fluid_dims[2]} state ({n} particles) after the timed "
                    f"steps; heat grid "
                    f"{dims[0]}x{dims[1]}x{dims[2]} of 0.2 with sources; 4096 points; 8 spheres r=0.5; host-clock "
                    f"time per call including transfers",
        "couple_heat": {"ms": t_heat * 1e3, "particles_per_s": n / t_heat,
                        "cpu_particles_per_s": ns / c_heat},
        "couple_points": {"ms": t_pts * 1e3, "points_per_s": len(pts) / t_pts,
                          "cpu_points_per_s": len(spts) / c_pts},
        "couple_bodies": {"ms": t_bod * 1e3, "particles_per_s": n / t_bod, "cpu_particles_per_s": ns / c_bod},
        "cpu_sample": f"oracle, one thread: {sdims[0]}x{sdims[1]}x{sdims[2]} block ({ns} particles), heat grid "
                      f"{sgrid[0]}x{sgrid[1]}x{sgrid[2]}, 1024 points, 4 spheres",
    }


def _standalone_scenes():
    """physics_b200/scenes.py loaded as a lone module: the scene generator needs only
    numpy, and importing it this way keeps the product library (loaded by the package's
    __init__) out of the process."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("sph_bench_scenes", ROOT / "physics_b200" / "scenes.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod  # dataclasses resolve their module through sys.modules
    spec.loader.exec_module(mod)
    return mod


def _oracle_world(O, pos, threads: int):
    """The oracle world of the benchmark scene: SphParams::defaults() restated in the
    oracle module (params.rs:55-85), bounds [0, 51.2]^3, lattice_mass(0.1)."""
    p = O.RefParams.defaults()
    p.bounds_min, p.bounds_max = (0.0, 0.0, 0.0), (BOX, BOX, BOX)
    w = O.OracleWorld(p, threads=threads)
    w.add_particles(pos, w.lattice_mass(0.1))
    return w


def cpu_baseline(scenes, pb, n: int, dims, budget_s: float = 15.0):
    """The oracle (CPU restatement of the reference's rayon step) on all host threads, on
    the same scene as the headline, for about budget_s seconds of steps from the start."""
    from oracle import oracle as O
    O.build()
    threads = O.max_threads()
    w = _oracle_world(O, scenes.dam_break_positions(*dims), threads)
    steps, t = 0, 0.0
    while (t < budget_s and steps < 50) or steps < 2:
        t0 = time.perf_counter()
        w.step(DT)
        t += time.perf_counter() - t0
        steps += 1
    return {"value": n * steps / t, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"steps 1-{steps} of the same {n}-particle scene, OpenMP {threads} threads, f64 oracle"}


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's rayon step (oracle/, the
    reference op order, OpenMP over all host threads) on the headline's scene, W untimed
    and K timed steps from the initial state, as the headline.  Loads liboracle.so only."""
    rank = env_int("RANK", 0)
    if rank != 0:
        return None
    scenes = _standalone_scenes()
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O
    O.build()
    threads = O.max_threads()
    K, W = args.steps, args.warmup
    dims = tuple(args.dims)
    pos = scenes.dam_break_positions(*dims)
    n = pos.shape[0]
    w = _oracle_world(O, pos, threads)
    w.step(DT, W)
    t0 = time.perf_counter()
    w.step(DT, K)
    t = time.perf_counter() - t0
    value = n * K / t
    sample = (f"every step of the {n}-particle scene (steps {W + 1}-{W + K}); CPU restatement of the reference's "
              f"rayon step (oracle/), OpenMP {threads} threads; the Rust reference is not buildable here (no cargo, "
              f"crates not vendored)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": env_int("WORLD_SIZE", 1),
            "steps": K, "warmup": W, "ms_per_step": t / K * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered dam-break lattice)",
            "config": bench_config(dims, n, env_int("WORLD_SIZE", 1)),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return line


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--graph-chunk", type=int, default=0,
                    help="steps per captured CUDA graph of the single-scene worlds (0: launch every step)")
    ap.add_argument("--batch-scenes", type=int, default=256, help="scenes of the batched form (0: skip)")
    ap.add_argument("--adjoint-directions", type=int, default=32,
                    help="finite-difference directions of the adjoint check (0: skip the adjoint)")
    ap.add_argument("--batch-steps", type=int, default=200, help="timed steps of the batched form")
    ap.add_argument("--no-coupling", action="store_true", help="skip the coupling calls (couple_heat / _points / "
                    "_bodies)")
    ap.add_argument("--full-steps", type=int, default=1000,
                    help="also time this many steps from the initial dam (the configured 1000-step run; "
                         "the column compresses and splashes, so per-step cost changes along it); 0 = skip")
    ap.add_argument("--dims", type=int, nargs=3, default=list(DIMS),
                    help="lattice of the dam block (default 128 256 128 = 4,194,304 particles); smaller blocks "
                         "are for profiling captures only")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
