"""Throughput of the differentiable growth step: particle-steps/s of forward +
adjoint for the batched FP32 path on the 256-scene uneven workload
(n log-uniform in [2048, 65536], grids 32^3..64^3, mixed neo-Hookean/Hencky,
per-scene growth g, 200 steps forward + full-trajectory adjoint, one
graph-captured launch sequence per trajectory).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One bench step = one forward + loss + adjoint trajectory over the whole batch.
Prints one JSON line (rank 0).  Under torchrun the batch has 256 x ranks scenes
(one seed), LPT-sharded over the ranks by particles x steps, so every rank holds
about the 1-GPU work (weak scaling); no data-path collective; time = max over
ranks; per-scene results are gathered to every rank in scene order afterwards.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s fwd+adjoint: FP32 batched vs FP64 plain @ stated F error"
UNIT = "particle-steps/s"
WORKLOAD = "config4: 256 uneven growth scenes (2k-64k particles, 32^3-64^3 grids), 200 steps fwd+adj, FP32 batched"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scenes", type=int, default=256)
    ap.add_argument("--mpm-steps", type=int, default=200)
    ap.add_argument("--ckpt-every", default="auto",
                    help="checkpoint interval: an int, 'sqrt', or 'auto' (largest that fits 75%% of free HBM)")
    ap.add_argument("--no-plain", action="store_true", help="skip the FP64 plain-path leg")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-others", action="store_true", help="skip the configs 1, 2, 3, 5 leg")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--workload", default="config4", choices=["config1", "config2", "config3", "config4", "config5"],
                    help="config4 is the headline line; the others print one line each for the other growth "
                         "workloads (FP64 and FP32 where the workload names both)")
    ap.add_argument("--conditioning", action="store_true",
                    help="with --workload: how far FP64 moves when only the initial positions are rounded to "
                         "FP32, next to the FP32 error (one JSON line)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9 for i in range(4)
                          if r[5 + i].lower() in ("active", "1")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU legs (oracle port: numpy FP64 restatement of the reference)
# ---------------------------------------------------------------------------
def _oracle_scene_run(args):
    s, steps = args
    from oracle import mpm_oracle as O
    sp = s["dx"] / 2
    sc = O.Scene(shape=s["shape"], dx=s["dx"], dt=s["dt"], damping=s["damping"], pmass=s["density"] * sp ** 3,
                 vol0=sp ** 3, wall=s["wall"])
    m = O.Model.elastic(s["model"], s["E"], s["nu"])
    gr = O.Growth(A=s["growth_A"])
    t0 = time.perf_counter()
    st, caches = O.rollout(O.State.rest(s["x"]), m, sc, steps, advect=True, growth=gr)
    n = s["x"].shape[0]
    z3, z33 = np.zeros((n, 3)), np.zeros((n, 3, 3))
    O.rollout_vjp(caches, z3, z3, z33, O.seed_detF(st.F), z33, advect=True, growth=gr)
    return n * steps, time.perf_counter() - t0


def cpu_sample(scenes, seconds, steps=2):
    """Scenes of the workload (smallest first) until ~`seconds` of work."""
    order = sorted(range(len(scenes)), key=lambda i: scenes[i]["x"].shape[0])
    budget_units = None
    picked = []
    # calibrate on the smallest scene
    units, dt = _oracle_scene_run((scenes[order[0]], steps))
    rate = units / dt
    budget_units = rate * seconds
    acc = 0
    for i in order[1:]:
        u = scenes[i]["x"].shape[0] * steps
        if acc + u > budget_units:
            break
        picked.append(i)
        acc += u
    return picked, steps


def cpu_baseline(scenes, seconds):
    picked, steps = cpu_sample(scenes, seconds)
    tot_u, tot_t = 0, 0.0
    for i in picked:
        u, t = _oracle_scene_run((scenes[i], steps))
        tot_u += u
        tot_t += t
    return {"value": tot_u / max(tot_t, 1e-9), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{len(picked)} smallest scenes of the workload ({tot_u} particle-steps), {steps} steps "
                      f"fwd+adj each, numpy FP64 oracle, 1 thread",
            "note": "the port vectorises the reference's per-particle numpy loops; the reference's own "
                    "transfer.step + step_vjp ran at about 465 particle-steps/s on one core of the build "
                    "machine (config-1 cube), so the port is far faster than the reference itself"}


def cpp_reference_forward(seconds=4.0):
    """The reference's own C++ FP32 forward solver (growth_solver.h, built into
    oracle/_ref from the reference tree), one core, on the 4096-particle
    free-swell cube of config 1 with Hencky stress (the solver's only model).
    Forward only: the C++ code has no adjoint.  None when the library is absent."""
    from oracle import growth_ref as G
    if not G.available():
        return None
    from morphompm_b200 import scenes as S
    c = S.config1()
    n = c["x"].shape[0]
    sp = c["dx"] / 2

    def make():
        r = G.RefSolver(c["shape"][0], c["dx"], c["E"], c["nu"], c["damping"])
        r.add(c["x"], c["density"] * sp ** 3, c["density"])
        r.set_growth(1.0 + c["growth_A"])
        return r
    r = make()
    t0 = time.perf_counter()
    r.step(c["dt"], 2)
    per_step = (time.perf_counter() - t0) / 2
    steps = max(2, int(seconds / max(per_step, 1e-6)))
    r = make()
    t0 = time.perf_counter()
    r.step(c["dt"], steps)
    dt = time.perf_counter() - t0
    return {"value": n * steps / dt, "unit": "particle-steps/s (forward only)", "cores": 1, "kind": "reference",
            "sample": f"config-1 cube, {n} particles, {steps} forward steps, Hencky, FP32, C++ (growth_solver.h)"}


def run_reference(a):
    """--impl reference: the oracle port on all host cores (process pool over scenes)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from morphompm_b200 import scenes as S
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    scn = S.config4(n_scenes=a.scenes)
    cores = os.cpu_count() or 1
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    steps = 2
    # ~8 s of single-core work per process per bench step, scenes taken evenly
    # over the size range of the workload
    _, t1 = _oracle_scene_run((scn[0], steps))
    rate = scn[0]["x"].shape[0] * steps / max(t1, 1e-6)
    budget = rate * 8.0 * cores
    order = sorted(range(len(scn)), key=lambda i: scn[i]["x"].shape[0])
    stride = max(1, len(order) // 64)
    jobs, acc = [], 0
    for i in order[::stride]:
        u = scn[i]["x"].shape[0] * steps
        if acc + u > budget and jobs:
            break
        jobs.append((scn[i], steps))
        acc += u
    vals, wall = [], []
    with ctx.Pool(cores) as pool:
        for it in range(a.warmup + a.steps):
            t0 = time.perf_counter()
            res = pool.map(_oracle_scene_run, jobs)
            dt = time.perf_counter() - t0
            if it >= a.warmup:
                vals.append(sum(u for u, _ in res) / dt)
                wall.append(dt * 1e3)
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": float(np.median(wall)), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "scenes": a.scenes, "mpm_steps": a.mpm_steps},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{len(jobs)} scenes x {steps} steps fwd+adj per bench step, numpy FP64 "
                                       f"oracle, {cores} processes"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# algorithmic bytes per particle, per kernel kind (w = bytes per word)
# ---------------------------------------------------------------------------
def kernel_bytes_per_particle(kind, w):
    """Unique bytes a kernel must move per particle (state and cotangent
    fields it reads and writes, its payload record, 4-byte sort indices);
    node records are added separately."""
    table = {
        "prepass": 24 * w + 16 * w + 4,            # x v C F (+ growth law) -> P2G record, scene id
        "p2g": 16 * w + 4,                         # P2G record once, through perm
        # chained step: x F -> x v C F, the next step's record and key; perm, old key, scene id
        "g2p": 12 * w + 24 * w + 16 * w + 4 + 4 + 4 + 4,
        "bwd_p2g": 36 * w + 4,                     # x F + the x v C F cotangents, through perm
        "bwd_particle": (24 + 9 + 24 + 24) * w + 8 + 4 + 4 + 4,
    }
    return table.get(kind)


# DRAM bytes (read + write) per particle per launch of the heaviest kernels, from
# `ncu` captures of a 2,092,825-particle batch of the config-4 generator (FP32,
# chained steps; profiles/reverse_particle_dram_config4_128scenes.md and
# profiles/g2p_per_model_config4_128scenes.md); their traffic grows in
# proportion to the particles, so it is scaled to the workload.
MEASURED_TRAFFIC_PER_PARTICLE = {
    # the neo-Hookean and the Hencky run of one step (the kernels specialised per model)
    "bwd_particle": (281440768 + 89405440 + 244199680 + 81494016) / 2092825,
    "g2p": (73642240 + 131875328 + 63985408 + 110647808) / 2092825,
}


def node_bytes(kind, w):
    return {"p2g": 4 * w, "bwd_p2g": 8 * w, "g2p": 4 * w, "bwd_particle": 8 * w}.get(kind, 0)


# ---------------------------------------------------------------------------
def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    if a.conditioning:
        return run_conditioning(a)
    if a.workload != "config4":
        return run_other(a)
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = torch.device("cuda", torch.cuda.current_device())
    from morphompm_b200 import scenes as S
    from morphompm_b200.batch import Batch, host_slab, load_tuned
    from morphompm_b200.trajectory import sqrt_schedule

    # one fixed batch of scenes x ranks scenes (seed 4; its first 256 scenes are
    # the 1-GPU workload), LPT-sharded over the ranks by particles x steps:
    # every rank holds about the same work (weak scaling), no data-path collective
    from morphompm_b200.shard import lpt_assign, gather_scenes, fixed_order_sum
    scn_all = S.config4(seed=4, n_scenes=a.scenes * world)
    mine = lpt_assign([s["x"].shape[0] * a.mpm_steps for s in scn_all], world)[rank]
    scn = [scn_all[i] for i in mine]
    n_tot = sum(s["x"].shape[0] for s in scn)
    ck = a.ckpt_every if a.ckpt_every in ("auto", "sqrt") else int(a.ckpt_every)
    # the schedule tuned for this GPU (python -m morphompm_b200.batch --autotune);
    # a rank's shard of a larger batch takes the 1-GPU batch's schedule
    tuning = load_tuned(scn, torch.float32) or load_tuned(scn_all[:a.scenes], torch.float32) or {}
    slab_np = host_slab(scn, np.float32)
    b = Batch(scn, a.mpm_steps, dtype=torch.float32, ckpt_every=ck, tuning=tuning, slab_host=slab_np)
    k = b.ckpt_every
    slab_h = torch.from_numpy(slab_np).pin_memory()
    b.load(slab_h, non_blocking=False)
    plan = b.plan

    # capture once with every kernel bracketed to find the dominant kernel
    from morphompm_b200 import _lib as L
    counts = {}

    def start_all():
        counts["n0"] = plan.launch_count()
        plan.profile_begin(L.KERNELS, max_launches=20000)
    b.capture(pre_capture=start_all)
    launches_per_traj = plan.launch_count() - counts["n0"]
    b.replay()
    prof_all = plan.profile_end()
    dominant = max(prof_all, key=lambda kk: prof_all[kk][0])

    # re-capture with only the dominant kernel bracketed; this graph is timed
    b.graph = None
    b.capture(pre_capture=lambda: plan.profile_begin([dominant], max_launches=20000))
    for _ in range(a.warmup):
        b.replay()
    torch.cuda.synchronize()
    fb0 = plan.fp64_fallbacks()      # cumulative device counter: read its change over the timed replays
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(dev.index if dev.index is not None else 0)
    clocks.start()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(a.steps):
        b.replay()
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    fallbacks = (plan.fp64_fallbacks() - fb0) / a.steps
    prof = plan.profile_end()
    from morphompm_b200.shard import max_over_ranks, sum_over_ranks
    ms = max_over_ranks(ms, dev)
    ms_per = ms / a.steps
    # the job's particles: the sum over the ranks' shards
    n_all = int(sum_over_ranks(n_tot, dev))
    units = n_all * a.mpm_steps
    value = units / (ms_per / 1e3)

    # end to end through the public API: every step copies its pinned host slab
    # to the device (on a side stream, overlapping the previous trajectory),
    # runs the trajectory and reads the per-scene loss and dL/dg back
    loss_h = torch.empty(len(scn), dtype=torch.float64).pin_memory()
    grad_h = torch.empty(len(scn), dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0.record(s)
    for _ in range(a.steps):
        b.prefetch(slab_h)
        b.replay()
        loss_h.copy_(b.loss, non_blocking=True)
        grad_h.copy_(b.dloss_dg, non_blocking=True)
    e1.record(s)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1)
    ms_e2e = max_over_ranks(ms_e2e, dev)
    e2e = {"value": units / (ms_e2e / a.steps / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": int(slab_h.numel() * slab_h.element_size()),
           "d2h_bytes_per_step": int(2 * 8 * len(scn))}
    # every scene's loss and d loss / d g in scene order on every rank, and the
    # gradient of a growth amplitude shared by all scenes (fixed-order sum)
    full = gather_scenes(np.stack([loss_h.numpy(), grad_h.numpy()], 1), mine, len(scn_all), dev)
    gathered = {"scenes": len(scn_all), "loss_sum": fixed_order_sum(full[:, 0]),
                "shared_growth_grad": fixed_order_sum(full[:, 1])}

    # roofline of the dominant kernel (HBM bound: no dense contraction here)
    tot_ms, nl = prof.get(dominant, (float("nan"), 0))
    avg_ms = tot_ms / max(nl, 1)
    w = 4
    nodes_per_launch = None
    bpp = kernel_bytes_per_particle(dominant, w)
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    achieved = None
    if bpp is not None and nl:
        alg = bpp * n_tot + node_bytes(dominant, w) * 0.2 * n_tot
        achieved = alg / (avg_ms / 1e3) / 1e9
    roof = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "peak_source": peak_src,
            "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
            "traffic": (MEASURED_TRAFFIC_PER_PARTICLE[dominant] * n_tot
                        if dominant in MEASURED_TRAFFIC_PER_PARTICLE else None),
            "traffic_source": "ncu dram bytes per launch, 2.09M-particle capture scaled by particles "
                              "(profiles/reverse_particle_dram_config4_128scenes.md)",
            "avg_launch_ms": avg_ms, "launches": nl,
            "per_launch": "one MPM step of the kernel: its launches over every material-model run of slots "
                          f"({len({sc['model'] for sc in scn if sc['x'].shape[0]})} per step) between one pair of CUDA events"}
    # whole step against the algorithmic bytes per particle-step fwd+adj
    # (w*(156 + 32*G_touched/n), G_touched/n ~ 0.2 at 8 particles per cell)
    step_bytes = w * (156 + 32 * 0.2) * n_tot * a.mpm_steps
    step_roof = {"bytes_per_particle_step": w * (156 + 32 * 0.2), "achieved_gbs": step_bytes / (ms_per / 1e3) / 1e9,
                 "frac": step_bytes / (ms_per / 1e3) / 1e9 / peak}
    status = plan.status()
    # every Hencky particle is evaluated once per forward step and once per
    # reverse step (store-all schedule; recompute adds forward evaluations)
    n_hencky = sum(int(sc["x"].shape[0]) for sc in scn if sc["model"] == "hencky")
    recomputed = a.mpm_steps - a.mpm_steps // max(1, k) if k < a.mpm_steps else 0
    hencky_evals = n_hencky * (2 * a.mpm_steps + recomputed)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms_per, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "scenes": len(scn_all), "particles": n_all,
                       "mpm_steps": a.mpm_steps, "ckpt_every": k, "l2": "inputs larger than L2 "
                       f"({n_tot * 24 * 4 / 1e6:.0f} MB state per GPU)", "schedule": plan.tuning or "defaults",
                       "parallelism": f"{world} rank(s), one {len(scn_all)}-scene batch LPT-sharded by "
                                      "particles x steps (no data-path collective)"},
            "roofline": roof, "step_roofline": step_roof, "e2e": e2e,
            "gpu_launches": int(launches_per_traj * a.steps), "clocks": clk,
            "kernel_ms_per_trajectory": {kk: round(v[0], 3) for kk, v in prof_all.items()},
            "fp64_hencky_fallbacks_per_trajectory": fallbacks,
            "fp64_hencky_fallback_fraction": fallbacks / max(1, hencky_evals),
            "device_status": status, "active_tile_cap": plan.tuning.get("active_tile_cap"),
            "gathered": gathered}

    # the 1-GPU legs (FP64 plain path, CPU baselines, the other workloads)
    if world == 1 and not a.no_plain:
        line["fp64_plain"] = plain_leg(scn, a, value, peak, tuning)
    if world == 1 and not a.no_cpu:
        line["cpu_baseline"] = cpu_baseline(scn, a.cpu_seconds)
        line["cpu_reference_forward"] = cpp_reference_forward()
    if world == 1 and not a.no_others:
        # the other growth workloads, one timed trajectory each after one warm-up
        b.graph = None
        del b
        torch.cuda.empty_cache()
        others = {}
        for w in ("config1", "config2", "config3", "config5"):
            r = workload_line(w, 1, 1)
            others[w] = {"name": r["name"], "particles": r["particles"], "mpm_steps": r["mpm_steps"],
                         "results": {k: {kk: v[kk] for kk in ("value", "ms_per_trajectory", "ckpt_every",
                                                              "trajectory_storage_gb", "device_status")}
                                     for k, v in r["results"].items()},
                         "fp32_error_vs_fp64": r.get("fp32_error_vs_fp64")}
            torch.cuda.empty_cache()
        line["other_workloads"] = others
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        b.graph = None
        dist.barrier()
        dist.destroy_process_group()


def _timed_trajectories(b, steps, warmup):
    """Capture the batch's trajectory once, replay warmup + steps times; device
    ms per trajectory (CUDA events on the replay stream)."""
    import torch
    b.capture()
    for _ in range(warmup):
        b.replay()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(steps):
        b.replay()
    e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _curvature(final_slab):
    """Bending of the bilayer strip: least-squares parabola y(x) of the
    centreline (mean y per x-bin), curvature ~ 2a (the measure of the
    reference's Timoshenko test, tests/test_growth.cpp)."""
    x = final_slab[0].astype(np.float64)
    y = final_slab[1].astype(np.float64)
    nb = 9
    lo, hi = x.min(), x.max()
    idx = np.minimum(nb - 1, ((x - lo) / ((hi - lo) / nb + 1e-12)).astype(int))
    xm = np.array([x[idx == b].mean() for b in range(nb) if np.any(idx == b)])
    ym = np.array([y[idx == b].mean() for b in range(nb) if np.any(idx == b)])
    a2 = np.polyfit(xm - xm.mean(), ym, 2)[0]
    return abs(2 * a2)


def run_other(a):
    """One JSON line for configs 1, 2, 3 or 5 (particle-steps/s fwd+adj)."""
    print(json.dumps(workload_line(a.workload, a.steps, a.warmup)), flush=True)


def workload_line(w, steps, warmup):
    """Throughput of one of configs 1, 2, 3, 5 (FP64 and FP32 where the
    workload names both), with the FP32 error against FP64."""
    import torch
    from morphompm_b200 import scenes as S
    from morphompm_b200.batch import Batch, host_slab
    from morphompm_b200.trajectory import sqrt_schedule
    c = getattr(S, w)()
    n = c["x"].shape[0]
    line = {"metric": METRIC, "unit": UNIT, "workload": w, "name": c["name"], "n_gpus": 1, "steps": steps,
            "warmup": warmup, "higher_is_better": True, "data": "synthetic", "particles": n,
            "mpm_steps": c["steps"], "results": {}}
    loss, x_obs = "detF", None
    if w == "config3":
        # observation: final positions of the g* trajectory; gradient at g_eval
        c_true = dict(c, growth_A=c["g_true"] - 1.0, ramp_steps=0)
        ob = Batch([c_true], c["steps"], dtype=torch.float64, ckpt_every=c["ckpt_every"])
        ob.load(host_slab([c_true], np.float64), non_blocking=False)
        ob.rollout.forward(ob.slab0)
        x_obs = ob.final_state()[0:3].t().cpu().numpy()
        c = dict(c, growth_A=c["g_eval"] - 1.0, ramp_steps=0)
        loss = "mse"
        del ob
    dtypes = {"config1": [torch.float64, torch.float32], "config2": [torch.float64, torch.float32],
              "config3": [torch.float64, torch.float32], "config5": [torch.float64, torch.float32]}[w]
    finals = {}
    for dt in dtypes:
        ck = {"config1": "auto", "config2": "auto", "config3": c.get("ckpt_every", 20),
              "config5": sqrt_schedule(c["steps"])}[w]
        # config 5 keeps sqrt(N) checkpoints: its trajectory storage stays far
        # below the 80 GB cap (reported as trajectory_storage_gb)
        b = Batch([c], c["steps"], dtype=dt, ckpt_every=ck, loss=loss, x_obs=x_obs)
        npd = np.float64 if dt == torch.float64 else np.float32
        b.load(host_slab([c], npd), non_blocking=False)
        ms = _timed_trajectories(b, steps, warmup)
        key = "fp64" if dt == torch.float64 else "fp32"
        mem = b.rollout.memory_bytes() + b.plan.ws_bytes
        res = {"value": n * c["steps"] / (ms / 1e3), "ms_per_trajectory": ms, "ckpt_every": b.ckpt_every,
               "trajectory_storage_gb": round(mem / 1e9, 2), "loss": float(b.loss[0]),
               "dloss_dg": float(b.dloss_dg[0]), "device_status": b.plan.status(),
               "fp64_hencky_fallbacks": b.plan.fp64_fallbacks()}
        finals[key] = b.final_state().double().cpu().numpy()
        if w == "config2":
            res["curvature"] = _curvature(finals[key])
            res["curvature_timoshenko"] = 1.5 * 0.2 / (8 * c["dx"])
        line["results"][key] = res
        del b
        torch.cuda.empty_cache()
    if "fp64" in finals and "fp32" in finals:
        f64, f32 = finals["fp64"], finals["fp32"]
        g64, g32 = line["results"]["fp64"]["dloss_dg"], line["results"]["fp32"]["dloss_dg"]
        line["fp32_error_vs_fp64"] = {"F": float(np.max(np.abs(f64[15:24] - f32[15:24]))),
                                      "x": float(np.max(np.abs(f64[0:3] - f32[0:3]))),
                                      "dLdg_rel": abs(g64 - g32) / max(abs(g64), 1e-300)}
    main_key = "fp32" if "fp32" in line["results"] else "fp64"
    line["value"] = line["results"][main_key]["value"]
    line["dtype"] = "f32" if main_key == "fp32" else "f64"
    return line


def run_conditioning(a):
    """Conditioning of a workload's FP32 error: FP64 from the scene's initial
    positions, FP64 from the same positions rounded to FP32 (a perturbation of
    rounding size and nothing else), and FP32.  When the first two differ as
    much as FP64 and FP32 do, the FP32 error is the trajectory's amplification
    of rounding, not an error of the FP32 path."""
    import torch
    from morphompm_b200 import scenes as S
    from morphompm_b200.batch import Batch, host_slab
    from morphompm_b200.trajectory import sqrt_schedule
    c = getattr(S, a.workload)()

    def run(cc, dt):
        ck = cc.get("ckpt_every") or (sqrt_schedule(cc["steps"]) if a.workload == "config5" else "auto")
        b = Batch([cc], cc["steps"], dtype=dt, ckpt_every=ck)
        b.load(host_slab([cc], np.float64 if dt == torch.float64 else np.float32), non_blocking=False)
        b.run()
        torch.cuda.synchronize()
        out = (b.final_state().double().cpu().numpy(), float(b.loss[0]), float(b.dloss_dg[0]), b.plan.status())
        del b
        torch.cuda.empty_cache()
        return out

    def diff(u, v):
        return {"F": float(np.max(np.abs(u[0][15:24] - v[0][15:24]))),
                "x": float(np.max(np.abs(u[0][0:3] - v[0][0:3]))),
                "loss_rel": abs(u[1] - v[1]) / abs(u[1]), "dLdg_rel": abs(u[2] - v[2]) / abs(u[2])}
    r64 = run(c, torch.float64)
    cr = dict(c, x=c["x"].astype(np.float32).astype(np.float64))
    r64r = run(cr, torch.float64)
    r32 = run(c, torch.float32)
    print(json.dumps({"workload": a.workload, "name": c["name"], "mpm_steps": c["steps"],
                      "x0_rounding": float(np.max(np.abs(cr["x"] - c["x"]))),
                      "fp64_vs_fp64_x0_rounded": diff(r64, r64r), "fp32_vs_fp64": diff(r64, r32),
                      "device_status": [r64[3], r64r[3], r32[3]]}), flush=True)


def plain_leg(scn, a, value32, peak, tuning32=None):
    """FP64 plain path: one scene at a time, eager launches per step (the
    drop-in transfer path), same trajectory.  Timed on a sample of scenes
    spread over the size range, with the throughput and the FP32-batched ratio
    of each sampled scene, the HBM roofline of the plain path (1299.2 B per
    particle-step in FP64), and the FP32 error vs FP64 on the same scenes.
    The whole batch in FP64, graph-captured, separates the gain of batching
    from the gain of FP32."""
    import torch
    from morphompm_b200.batch import Batch, host_slab
    idx = sorted(range(len(scn)), key=lambda i: scn[i]["x"].shape[0])
    sample = [idx[int(round(q * (len(idx) - 1)))] for q in np.linspace(0.0, 1.0, 6)]
    units, secs = 0, 0.0
    errs = {"F": 0.0, "x": 0.0, "dLdg_rel": 0.0}
    per_scene = []
    for i in sample:
        s = scn[i]
        b64 = Batch([s], a.mpm_steps, dtype=torch.float64, ckpt_every="auto")
        b64.load(host_slab([s], np.float64), non_blocking=False)
        b64.run()                                     # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b64.run()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        secs += dt
        n_i = s["x"].shape[0]
        units += n_i * a.mpm_steps
        v_i = n_i * a.mpm_steps / dt
        per_scene.append({"particles": n_i, "grid": int(s["shape"][0]), "model": s["model"], "value": v_i,
                          "ms_per_mpm_step": dt * 1e3 / a.mpm_steps, "fp32_batched_over_this": value32 / v_i})
        b32 = Batch([s], a.mpm_steps, dtype=torch.float32, ckpt_every="auto", tuning=tuning32)
        b32.load(host_slab([s], np.float32), non_blocking=False)
        b32.run()
        torch.cuda.synchronize()
        f64 = b64.final_state().cpu().numpy()
        f32 = b32.final_state().double().cpu().numpy()
        errs["F"] = max(errs["F"], float(np.max(np.abs(f64[15:24] - f32[15:24]))))
        errs["x"] = max(errs["x"], float(np.max(np.abs(f64[0:3] - f32[0:3]))))
        g64, g32 = float(b64.dloss_dg[0]), float(b32.dloss_dg[0])
        errs["dLdg_rel"] = max(errs["dLdg_rel"], abs(g64 - g32) / max(abs(g64), 1e-300))
        del b64, b32
    v64 = units / secs
    bpp = 8 * (156 + 32 * 0.2)
    torch.cuda.empty_cache()
    # the whole batch in FP64, graph-captured (batching without the FP32 gain)
    bb = Batch(scn, a.mpm_steps, dtype=torch.float64, ckpt_every="auto", tuning=None)
    bb.load(host_slab(scn, np.float64), non_blocking=False)
    ms_b = _timed_trajectories(bb, 2, 1)
    n_all = sum(s["x"].shape[0] for s in scn)
    v64b = n_all * a.mpm_steps / (ms_b / 1e3)
    del bb
    torch.cuda.empty_cache()
    return {"value": v64, "unit": UNIT, "sample": f"{len(sample)} scenes spread over the size range, "
            f"{a.mpm_steps} steps fwd+adj each, eager launches, FP64", "fp32_batched_over_fp64_plain": value32 / v64,
            "per_scene": per_scene,
            "roofline": {"bound": "hbm", "bytes_per_particle_step": bpp, "achieved": v64 * bpp / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": v64 * bpp / 1e9 / peak},
            "fp64_batched": {"value": v64b, "ms_per_trajectory": ms_b,
                             "roofline_frac": v64b * bpp / 1e9 / peak,
                             "batching_gain": v64b / v64, "fp32_gain": value32 / v64b},
            "fp32_error_vs_fp64": errs}


if __name__ == "__main__":
    main()
