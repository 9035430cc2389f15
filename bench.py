"""Benchmark: frames/s of the foam hot path at 10k particles on a 128^3 JFA grid.

Workload (the headline foam): N = 10,000, uniform positions (seed 1),
lognormal radii (median 0.015, sigma_log 0.25, clipped [0.007, 0.03]), 128^3
int32 owner grid (8 JFA passes), 8 PBD and 20 Jacobi pressure iterations per
frame, FSC band [12, 16], JFA every frame for 20 warm-start frames and then
every 5th frame.  One step = one steady-state cadence cycle of 5 frames
(1 JFA frame + 4 non-JFA frames) replayed from CUDA graphs; value = frames/s.

Timing: W untimed warm-up steps after the 20 warm-start frames; each of the K
timed steps is bracketed by CUDA events on the launching stream, with a
256 MiB L2 flush between steps outside the events; barrier + synchronize
around the timed region; max over ranks.  e2e repeats the step through the
public API with host buffers: pinned H2D of pos/rad before and D2H of
pos/rad/fsc after the 5 frames, inside the timed region.  The resident and the
e2e steps alternate, so both cover the same stretch of the trajectory.

--impl reference times the CPU restatement of the reference (oracle/, the
reference itself is Python+Taichi and Taichi is not installable here) with all
host threads on the same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "fabric-of-space-taichi-jfa_b200"))

METRIC = "frames/s at 10k particles, 128^3 JFA: plain vs surrogate-FSC (>=99% FSC agree)"
UNIT = "frames/s"
FRAMES_PER_STEP = 5


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fos", choices=["fos", "reference"])
    ap.add_argument("--cpu-sample-steps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--jfa-form", default="multi", choices=["multi", "single", "staged", "label"],
                    help="JFA pass form for --profile jfa / frame: four voxels a thread "
                         "(default), one, TMA-staged rows, or the label-gather pass (the "
                         "lower-index tie rule)")
    ap.add_argument("--profile", default=None,
                    choices=["jfa", "frame", "surrogate", "ensemble", "inference"],
                    help="stage-timing mode for profiling (one small JSON line)")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--workload", default="headline", choices=["small", "headline", "stress"])
    ap.add_argument("--no-surrogate", action="store_true",
                    help="skip the surrogate-FSC arm of the metric")
    ap.add_argument("--no-surrogate-large", action="store_true",
                    help="skip the surrogate on the 50,000-particle 192^3 variant")
    ap.add_argument("--surrogate-mode", default="absolute", choices=["absolute", "anchored"])
    ap.add_argument("--no-warm-jfa", action="store_true",
                    help="skip the warm-started JFA arm (frames/s and agreement with the exact JFA)")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the batched-ensemble measurement")
    ap.add_argument("--ensemble-frames", type=int, default=500)
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# The workloads a line can be measured on: the headline foam (the metric's
# configuration, the default), the bandwidth-stress foam (200,000 particles
# on a 256^3 grid, JFA every frame) and the small CPU-runnable foam.
WORKLOADS = {
    "small": {"metric": "frames/s at 1k particles, 64^3 JFA every frame (small)",
              "frames_per_step": 1, "particles": 1000, "jfa_res": 64,
              "describe": "small foam: N=1000, r ~ U[0.025, 0.035], 64^3 int32 owner grid, 7 "
                          "JFA passes every frame, K=4 PBD, M=10 pressure, band [10,16]; step = "
                          "1 frame"},
    "headline": {"metric": METRIC, "frames_per_step": 5, "particles": 10000, "jfa_res": 128,
                 "describe": "headline foam: N=10000, 128^3 int32 owner grid, 8 JFA passes, "
                             "K=8 PBD, M=20 pressure, band [12,16], JFA every 5th frame after 20 "
                             "warm-start frames; step = 5-frame cadence cycle"},
    "stress": {"metric": "frames/s at 200k particles, 256^3 JFA every frame (bandwidth stress)",
               "frames_per_step": 1, "particles": 200000, "jfa_res": 256,
               "describe": "stress foam: N=200000, bimodal radii (50% U[0.004,0.005], 50% "
                           "U[0.007,0.009]), 256^3 int32 owner grid, 9 JFA passes every frame, "
                           "K=8 PBD, M=20 pressure, band [12,16]; step = 1 frame"},
}


def use_workload(name):
    """Set the module's metric and step length for the named workload."""
    global METRIC, FRAMES_PER_STEP, WORKLOAD
    WORKLOAD = name
    METRIC = WORKLOADS[name]["metric"]
    FRAMES_PER_STEP = WORKLOADS[name]["frames_per_step"]


WORKLOAD = "headline"


def workload_config(n_gpus):
    w = WORKLOADS[WORKLOAD]
    return {"workload": w["describe"],
            "particles": w["particles"], "jfa_res": w["jfa_res"], "frames_per_step": FRAMES_PER_STEP,
            "l2": "flushed between timed steps (256 MiB write outside the events)",
            "parallelism": f"replicas x{n_gpus} (independent foams, no collective)",
            "path": "plain exact JFA"}


def workload_foam(inputs):
    return {"small": inputs.small, "headline": inputs.headline,
            "stress": inputs.stress}[WORKLOAD]()


def warm_start_frames(foam):
    """Frames run before the first warm-up step: the warm start of a foam whose
    JFA cadence changes after it (20 frames on the headline foam), none on a
    foam that runs the JFA every frame."""
    return foam.jfa_warm if foam.jfa_warm < foam.frames else 0


# ----------------------------------------------------------------- clocks
class Clocks:
    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = f"/tmp/fos_clocks_{os.getpid()}.csv"

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = max(mx, float(f[2]))
                except ValueError:
                    continue
                for k, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(k)
        except OSError:
            return None
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


def profile_traffic():
    """Per-launch DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum)
    from the committed summary, each with the commit and command it came from."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        return json.load(open(path))
    except Exception:
        return None


def traffic_bytes(traffic, kernel):
    e = (traffic or {}).get(kernel)
    return e.get("bytes") if isinstance(e, dict) else None


def tkey(kernel):
    """traffic.json key of a kernel on the current workload."""
    return kernel if WORKLOAD == "headline" else f"{kernel}@{WORKLOAD}"


def traffic_source(traffic, kernel):
    e = (traffic or {}).get(kernel)
    if not isinstance(e, dict):
        return None
    return f"ncu capture at commit {e.get('commit')} ({e.get('workload')})"


# ------------------------------------------------------------- CPU arm
def oracle_sim(foam):
    from oracle import oracle as O
    p = O.OracleParams(n=foam.n, L=1.0, R=foam.res, r_max_cell=foam.r_max, f_low=foam.f_low,
                       f_high=foam.f_high, r_min=foam.r_min, r_max=foam.r_max, brownian=1e-4,
                       seed=foam.seed, pbd_iters=foam.pbd_iters,
                       pressure_iters=foam.pressure_iters, jfa_warm=foam.jfa_warm,
                       jfa_cadence=foam.jfa_cadence)
    sim = O.OracleSim(p, foam.pos, foam.rad)
    sim.initialize()
    return sim, O


def time_cpu(foam, steps, warmup):
    """The CPU restatement over the frames the GPU arm's resident steps time:
    the 20 warm-start frames (JFA every frame) and `warmup` cadence steps
    untimed, then `steps` timed 5-frame steps, each followed by one untimed
    step (the frames of the GPU arm's interleaved e2e step).  Returns
    (frames/s, timed seconds, threads, first timed frame)."""
    sim, O = oracle_sim(foam)
    for _ in range(warm_start_frames(foam) + warmup * FRAMES_PER_STEP):
        sim.step()
    first = sim.frame
    dt = 0.0
    for k in range(steps):
        t0 = time.perf_counter()
        for _ in range(FRAMES_PER_STEP):
            sim.step()
        dt += time.perf_counter() - t0
        if k + 1 < steps:
            for _ in range(FRAMES_PER_STEP):
                sim.step()
    return FRAMES_PER_STEP * steps / dt, dt, O.num_threads(), first


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle as O
    O.build()
    from fos import inputs
    foam = workload_foam(inputs)
    fps, dt, cores, first = time_cpu(foam, args.steps, args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(fps, 4), "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1000.0 * dt / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.gpus),
        "impl_path": "CPU restatement of the reference's kernels (oracle/, OpenMP), run on "
                     "the frames the GPU arm's resident steps time",
        "cpu_baseline": {"value": round(fps, 4), "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} timed {FRAMES_PER_STEP}-frame steps from "
                                   f"frame {first} ({warm_start_frames(foam)} warm-start frames "
                                   f"and {args.warmup} warm-up steps untimed; an untimed step "
                                   f"between timed ones, as the GPU arm's e2e steps); the "
                                   f"reference itself is Taichi, which is not installable here"},
        "e2e": {"value": round(fps, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------- GPU arm
def run_fos(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    from fos import inputs
    from fos.context import stream
    from fos.driver import FoamSim
    import ctypes as C
    from fos._lib import FosJfaStats, call

    foam = workload_foam(inputs)
    sim = FoamSim.from_foam(foam, use_graph=True)
    sim.initialize()
    for _ in range(warm_start_frames(foam)):  # headline: 20 frames with JFA every frame
        sim.step()
    assert sim.frame % foam.jfa_cadence == 0
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def one_step():
        for _ in range(FRAMES_PER_STEP):
            sim.step()

    for _ in range(args.warmup):
        one_step()
    barrier()
    clocks = Clocks(dev)
    clocks.start()
    launches0 = sim.ctx.launch_count()
    torch_kernels_before = 1 + 8  # flush buffer fill + state tensor fills
    s = torch.cuda.current_stream()
    times = []
    # e2e through the public API with host buffers, interleaved with the
    # resident steps so that both numbers cover the same stretch of the
    # trajectory (the foam packs over the run and frames slow down with it):
    # each iteration times one resident step, then refreshes the pinned host
    # copy of the particle state (outside the events) and times one step that
    # uploads it, runs and reads the state and the FSC back
    n = foam.n
    h_pos = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    h_rad = torch.empty((n,), dtype=torch.float32).pin_memory()
    h_fsc = torch.empty((n,), dtype=torch.int32).pin_memory()
    e2e_ms = 0.0
    launches = 0
    frame_evs = []
    barrier()
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = sim.ctx.launch_count()
        e0.record(s)
        # an event after every frame: the plain frames' intervals are the
        # dynamics kernel's live, in-step duration (roofline below)
        prev_ev = e0
        for _ in range(FRAMES_PER_STEP):
            kind = "jfa" if sim.cfg.is_jfa_frame(sim.frame) else "plain"
            sim.step()
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(s)
            frame_evs.append((kind, prev_ev, ev))
            prev_ev = ev
        e1 = prev_ev
        launches += sim.ctx.launch_count() - l0
        times.append((e0, e1))
        h_pos.copy_(sim.pos)
        h_rad.copy_(sim.rad)
        flush.fill_(1.0)
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        l0 = sim.ctx.launch_count()
        f0.record(s)
        sim.pos.copy_(h_pos, non_blocking=True)
        sim.rad.copy_(h_rad, non_blocking=True)
        one_step()
        h_pos.copy_(sim.pos, non_blocking=True)
        h_rad.copy_(sim.rad, non_blocking=True)
        h_fsc.copy_(sim.fsc, non_blocking=True)
        f1.record(s)
        launches += sim.ctx.launch_count() - l0
        f1.synchronize()
        e2e_ms += f0.elapsed_time(f1)
    barrier()
    clk = clocks.stop()
    total_ms = sum(a.elapsed_time(b) for a, b in times)
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    value = world * FRAMES_PER_STEP * args.steps / (total_ms / 1000.0)

    t = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = world * FRAMES_PER_STEP * args.steps / (float(t.item()) / 1000.0)

    # ---- late run: the last 200 frames of a 1,000-frame workload (the foam
    # packs over a run and its frames slow down), steps as above
    late_run = None
    if foam.frames >= 1000:
        while sim.frame < foam.frames - 200:
            sim.step()
        late_ms, late_steps, first_late = 0.0, 0, sim.frame
        while sim.frame + FRAMES_PER_STEP <= foam.frames:
            flush.fill_(1.0)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(s)
            one_step()
            b.record(s)
            b.synchronize()
            late_ms += a.elapsed_time(b)
            late_steps += 1
        t = torch.tensor([late_ms], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        late_run = {"frames": f"{first_late}-{sim.frame - 1}",
                    "value": round(world * FRAMES_PER_STEP * late_steps /
                                   (float(t.item()) / 1000.0), 3),
                    "unit": UNIT, "ms_per_step": round(float(t.item()) / late_steps, 4)}

    # ---- per-kernel timing on the launching stream, after the timed region
    ctx = sim.ctx
    peaks = measured_peaks()
    peak = peaks["hbm_gbs"] if peaks else 6650.0
    traffic = profile_traffic() or {}
    G3 = sim.cfg.grid_res() ** 3
    # (a) dominant kernel by time: k_frame_coop, the dynamics of one frame (one
    # launch per frame).  Its duration is the live one inside the timed steps:
    # the mean interval of the plain frames, whose graph holds k_frame_coop and
    # three small launches (a 16-byte reset kernel, one memset, the frame-end
    # kernel).  The JFA frame's interval is reported beside it.
    plain_ms = [a.elapsed_time(b) for k, a, b in frame_evs if k == "plain"]
    jfa_frame_ms = [a.elapsed_time(b) for k, a, b in frame_evs if k == "jfa"]
    coop_ms, coop_n = float(sum(plain_ms)), len(plain_ms)
    coop_s = coop_ms / 1000.0 / coop_n if coop_n else float("nan")
    K, M = foam.pbd_iters, foam.pressure_iters
    # algorithmic bytes per launch (first-touch, per particle / per cell), summed
    # over the frame's stages: (K+2) grid rebuilds x (68 B/particle + 16 B/cell),
    # max overlap 24 B, nudge 16 B, M pressure sweeps x 56 B, Brownian 24 B,
    # K PBD sweeps x 32 B.  Neighbour re-reads are L1/L2 reuse, not counted.
    coop_bytes = float(n) * ((K + 2) * 68 + 24 + 16 + M * 56 + 24 + K * 32) + (K + 2) * 16.0 * G3
    coop_achieved = coop_bytes / coop_s / 1e9
    # (b) the JFA pass (eight launches per JFA frame)
    reps = 10
    barrier()
    j0 = torch.cuda.Event(enable_timing=True)
    j1 = torch.cuda.Event(enable_timing=True)
    jfa_ms = 0.0
    for _ in range(reps):
        flush.fill_(1.0)
        ctx.jfa_init(sim.pos, sim.rad, n)
        j0.record(s)
        ctx.jfa_passes(n)
        j1.record(s)
        j1.synchronize()
        jfa_ms += j0.elapsed_time(j1)
    passes = ctx.num_passes
    # the interval holds the passes and the one record-grid build before them
    pass_s = jfa_ms / 1000.0 / (reps * passes)
    # the same passes with the record rows staged in shared memory by TMA
    # copies (off by default; measured here beside the default form)
    staged_ms = None
    if foam.res in (32, 64, 128, 256):
        ctx.set_jfa_staging(True)
        staged_ms = 0.0
        for _ in range(reps):
            flush.fill_(1.0)
            ctx.jfa_init(sim.pos, sim.rad, n)
            j0.record(s)
            ctx.jfa_passes(n)
            j1.record(s)
            j1.synchronize()
            staged_ms += j0.elapsed_time(j1)
        ctx.set_jfa_staging(False)
    staged_us = None if staged_ms is None else round(staged_ms * 1000.0 / (reps * passes), 3)
    # the default pass form at this size: four voxels a thread along x where
    # R^3 / 4 threads fill the GPU (R >= 128), else one
    multi = foam.res >= 128 and (foam.res & (foam.res - 1)) == 0
    pass_kernel = "k_jfa_pass_recx" if multi else "k_jfa_pass_rec"
    pass_note = ("four voxels a thread along x: 58 coalesced seed-record rows per 4 voxels"
                 if multi else "27 coalesced seed-record rows per voxel") + \
        "; labels and records are L2-resident at 128^3, not at 256^3"
    V = foam.res ** 3
    alg_bytes = 8.0 * V  # int32 label read + write per voxel per pass
    achieved = alg_bytes / pass_s / 1e9
    # FP32 work: 27 candidates x ~20 FP32 operations per voxel and pass (the
    # nominal count of the scope table), none of them FMAs (-fmad=false), so
    # the peak is the lane-operation rate 148 SMs x 128 lanes x 1.965 GHz.
    # The four-voxel form's first pass (step R/2) evaluates only the 8
    # distinct candidates of a voxel, so that pass counts 8 / 27 of the work.
    ops_per_voxel = 540.0 * ((passes - 1 + 8.0 / 27.0) / passes if multi else 1.0)
    fp32_ops = ops_per_voxel * V
    fp32_lane_peak = 148 * 128 * 1.965e9
    fp32_frac = fp32_ops / pass_s / fp32_lane_peak
    # (c) face extraction (accumulate_face_area: k_faces_reset, k_faces,
    # k_compact, k_rows) on the last passes' labels, majority-filtered first
    ctx.majority_filter()
    f_ms = 0.0
    for _ in range(reps):
        flush.fill_(1.0)
        j0.record(s)
        ctx.accumulate_faces(n)
        j1.record(s)
        j1.synchronize()
        f_ms += j0.elapsed_time(j1)
    faces_s = f_ms / 1000.0 / reps
    st = FosJfaStats()
    call("fos_jfa_stats", ctx.h, n, C.c_void_p(sim.rad.data_ptr()), C.byref(st), stream())
    # 4 B per voxel (filtered label read) + 8 B per distinct face pair
    faces_bytes = 4.0 * V + 8.0 * st.face_pairs
    headline_arms = WORKLOAD == "headline"

    surrogate = (None if args.no_surrogate or not headline_arms
                 else run_surrogate_arm(args, foam, flush, barrier, world))
    ensemble = (None if args.no_ensemble or not headline_arms
                else run_ensemble(args, barrier, world, rank))
    warm = None if args.no_warm_jfa or not headline_arms else run_warm_jfa(foam, flush)

    if world > 1:
        dist.barrier()
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0

    topo = run_topology(sim, foam, not args.no_cpu_baseline) if headline_arms else None
    # where the dynamics kernel's time goes: %globaltimer after every grid
    # barrier of one plain-frame dynamics kernel (block 0), taken after every
    # timed region (it advances the foam by one frame's dynamics)
    try:
        tr = sim.trace_dynamics()
        dyn_trace = {"phases_us": [round(x / 1000.0, 2) for x in tr],
                     "kernel_us": round(sum(tr) / 1000.0, 2), "phases": len(tr),
                     "source": "%globaltimer at kernel entry and after every grid barrier "
                               "(block 0), one plain frame after the timed steps"}
    except Exception as e:  # a diagnostic only: never fails the line
        dyn_trace = {"error": str(e)[:120]}
    cpu = None
    if not args.no_cpu_baseline:
        fps, dt, cores, first = time_cpu(foam, args.cpu_sample_steps, args.warmup)
        cpu = {"value": round(fps, 4), "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{args.cpu_sample_steps} timed {FRAMES_PER_STEP}-frame step(s) from "
                         f"frame {first}, the GPU arm's first timed frames, after the untimed "
                         f"warm-start and warm-up frames ({dt:.1f} s timed, OpenMP oracle)"}
    coop_roof = None
    if coop_n:
        coop_roof = {"bound": "hbm", "kernel": "k_frame_coop (dynamics of one frame)",
                     "achieved": round(coop_achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(coop_achieved / peak, 5),
                     "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peaks else
                                    "fallback 6650 GB/s",
                     "traffic": traffic_bytes(traffic, "k_frame_coop"),
                     "traffic_source": traffic_source(traffic, "k_frame_coop"),
                     "alg_bytes_per_launch": coop_bytes, "launch_us": round(coop_s * 1e6, 2),
                     "launch_us_source": f"live: mean of {coop_n} plain-frame graph intervals "
                                         "inside the timed steps (k_frame_coop + reset kernel, "
                                         "memset, frame-end kernel)",
                     "jfa_frame_us": round(1000.0 * sum(jfa_frame_ms) / max(1, len(jfa_frame_ms)),
                                           2),
                     "note": "latency/barrier bound: 14 phases (13 grid barriers) over L2-resident "
                             "data; HBM is not the limiting roof"}
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(world),
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": n * 16,
                "d2h_bytes_per_step": n * 20},
        "roofline": coop_roof,
        "roofline_jfa_pass": {"bound": "fp32-issue",
                              "kernel": f"{pass_kernel} ({foam.res}^3, one pass)",
                              "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                              "frac": round(achieved / peak, 4),
                              "fp32": {"achieved_T_ops_per_s": round(fp32_ops / pass_s / 1e12, 2),
                                       "peak_T_ops_per_s": round(fp32_lane_peak / 1e12, 2),
                                       "frac": round(fp32_frac, 4),
                                       "ops_per_voxel": round(ops_per_voxel, 1),
                                       "ops_note": "540 a voxel and pass (27 candidates x 20), "
                                                   "the first pass 8 / 27 of it (its distinct "
                                                   "candidates), averaged over the passes",
                                       "peak_note": "lane operations without FMA (148 x 128 x "
                                                    "1.965 GHz); 74.4 TFLOP/s counts an FMA "
                                                    "as two"},
                              "traffic": traffic_bytes(traffic, tkey(pass_kernel)),
                              "traffic_source": traffic_source(traffic, tkey(pass_kernel)),
                              "alg_bytes_per_launch": alg_bytes,
                              "pass_us": round(pass_s * 1e6, 3),
                              "tma_staged_pass_us": staged_us,
                              "pass_us_source": "CUDA events over 8 passes + the record-grid "
                                                "build, 10 JFA runs on the bench state",
                              "note": pass_note},
        "late_run": late_run,
        "surrogate": surrogate,
        "warm_jfa": warm,
        "ensemble": ensemble,
        "gpu_launches": int(launches),
        "clocks": clk,
        "cpu_baseline": cpu,
        "diagnostics": {"launches_before_timed": int(launches0 + torch_kernels_before),
                        "finalize_iterations": st.finalize_iterations,
                        "face_pairs": st.face_pairs, "mean_fsc": round(st.mean_fsc, 3),
                        "voxel_passes_per_s": round(V * passes * value / FRAMES_PER_STEP, 1),
                        "dynamics_trace": dyn_trace,

                        "topology": topo},
    }
    faces_achieved = faces_bytes / faces_s / 1e9
    line["roofline_faces"] = {
        "bound": "hbm", "kernel": f"face extraction ({foam.res}^3: k_faces_reset, k_faces_tile "
                                  f"(k_faces where R is not a multiple of 8), k_compact, "
                                  f"k_rows)",
        "achieved": round(faces_achieved, 2), "peak": peak, "unit": "GB/s",
        "frac": round(faces_achieved / peak, 4), "alg_bytes_per_launch": faces_bytes,
        "face_pairs": int(st.face_pairs), "us": round(faces_s * 1e6, 2),
        "traffic": traffic_bytes(traffic, tkey("k_faces")),
        "traffic_source": traffic_source(traffic, tkey("k_faces")),
        "note": "4 B per voxel + 8 B per distinct pair; the pair table is probed at random"}
    if WORKLOAD != "headline":
        # every frame runs the JFA: the dominant kernel is the pass (on the
        # stress foam the bandwidth case: two 67 MB label grids and two
        # 268 MB record grids do not fit the 126 MB L2)
        jr = line.pop("roofline_jfa_pass")
        jr["bound"] = "hbm"
        line["roofline"] = jr
        line["jfa_frame_ms"] = round(sum(jfa_frame_ms) / max(1, len(jfa_frame_ms)), 4)
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_topology(sim, foam, with_cpu):
    """One Gabriel-degree update (run.py:1273-1277: build_topo_candidates +
    gabriel_test_topological_degree) on the relaxed headline foam and its
    final grid: device time with CUDA events (median of 10), beside the oracle's
    serial restatement on the same state."""
    import ctypes as C

    import numpy as np
    import torch

    from fos._lib import call
    from fos.context import stream

    cfg, n = sim.cfg, sim.n
    cap = int(cfg.MAX_TOPO_NEIGHBORS)
    dev = sim.pos.device
    pairs = torch.zeros((n, cap), dtype=torch.int32, device=dev)
    cnt = torch.zeros(n, dtype=torch.int32, device=dev)
    tr = torch.zeros(n, dtype=torch.int32, device=dev)
    deg = torch.zeros(n, dtype=torch.int32, device=dev)
    ema = torch.zeros(n, dtype=torch.float32, device=dev)
    vp = lambda t: C.c_void_p(t.data_ptr())
    g = (vp(sim.cell_start), vp(sim.cell_count), vp(sim.cell_indices))
    s = torch.cuda.current_stream()
    times = []
    for r in range(13):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        call("fos_topo_candidates", sim.ctx.h, vp(sim.pos), vp(sim.rad), *g, n,
             float(cfg.TOPO_MAX_RADIUS_MULTIPLE), cap, vp(pairs), vp(cnt), vp(tr), stream())
        call("fos_topo_gabriel", sim.ctx.h, vp(sim.pos), *g, n, 60 * r, cfg.cell_size(),
             int(cfg.TOPO_PAIR_SUBSAMPLING_STRIDE), int(bool(cfg.TOPO_EARLY_EXIT_HIGH_DEGREE)),
             float(cfg.TOPO_DEG_HIGH), cap, vp(pairs), vp(cnt), vp(ema), vp(deg), stream())
        b.record(s)
        b.synchronize()
        if r >= 3:
            times.append(a.elapsed_time(b))
    out = {"workload": "Gabriel degree of the relaxed headline foam (candidates + witness test, "
                       "stride 3)", "gpu_ms": round(float(np.median(times)), 4),
           "mean_degree": round(float(deg.float().mean().item()), 3)}
    if with_cpu:
        from oracle import oracle as O
        p = O.OracleParams(n=n, L=1.0, R=foam.res, r_max_cell=foam.r_max)
        tp = O.TopoParams(mult=cfg.TOPO_MAX_RADIUS_MULTIPLE, cap=cap,
                          stride=cfg.TOPO_PAIR_SUBSAMPLING_STRIDE,
                          early_exit=cfg.TOPO_EARLY_EXIT_HIGH_DEGREE,
                          deg_high=cfg.TOPO_DEG_HIGH, cell_size=cfg.cell_size())
        pos, rad = sim.pos.cpu().numpy(), sim.rad.cpu().numpy()
        grid = (sim.cell_count.cpu().numpy(), sim.cell_start.cpu().numpy(),
                sim.cell_indices.cpu().numpy())
        t0 = time.perf_counter()
        op, opc, _ = O.topo_candidates(pos, rad, grid, p, tp)
        odeg = O.topo_gabriel(pos, grid, op, opc, np.zeros(n, np.float32), 60 * 12, p, tp)
        out["cpu_oracle_ms"] = round((time.perf_counter() - t0) * 1e3, 3)
        out["cpu_cores"] = O.num_threads()
        out["degrees_equal_oracle"] = bool(np.array_equal(odeg, deg.cpu().numpy()))
    return out


def surrogate_measure(args, foam, sur, flush, barrier, world, steps):
    """frames/s of `foam` with the learned FSC surrogate `sur` supplying FSC
    between exact JFA refreshes every 10 frames (the spec's "refresh every 5 or
    10 frames"), with the drift guard at the target and off, next to the plain
    path with JFA every 10 frames (the same JFA work with no FSC update
    between: the surrogate's cost floor).  Each run starts from the same
    warm-started foam; a step is one 10-frame refresh cycle, L2 flushed between
    steps; each judged JFA frame reads its counters on the host (one sync per
    cycle, inside the timed region).  Agreement: per-cell rint(surrogate FSC)
    == JFA fsc on the refresh frames of the timed region, beside the stale FSC
    the reference reuses (previous JFA fsc vs this one)."""
    import torch
    from fos import surrogate as S
    from fos.driver import FoamSim

    cycle = 10
    s = torch.cuda.current_stream()

    def timed(sim):
        for _ in range(foam.jfa_warm):
            sim.step()
        for _ in range(args.warmup * cycle):
            sim.step()
        barrier()
        if sim.policy is not None:
            sim.policy.judged.clear()
            forced0 = sim.policy.forced_total
        ms = 0.0
        jfa_frames = 0
        for _ in range(steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s)
            for _ in range(cycle):
                jfa_frames += 1 if sim.step() else 0
            e1.record(s)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
        t = torch.tensor([ms], dtype=torch.float64, device=flush.device)
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        fps = world * cycle * steps / (float(t.item()) / 1000.0)
        forced = sim.policy.forced_total - forced0 if sim.policy is not None else 0
        return fps, jfa_frames / float(cycle * steps), forced

    keys = ("exact_frac", "within1_frac", "mean_abs_err", "stale_exact_frac",
            "stale_within1_frac", "stale_mean_abs_err")

    def surrogate_run(pol):
        sim = FoamSim.from_foam(foam, surrogate=sur, policy=pol,
                                surrogate_mode=args.surrogate_mode)
        sim.initialize()
        fps, jfa_frac, forced = timed(sim)
        judged = list(pol.judged)
        sim.ctx.close()
        agree = {k: round(sum(d[k] for d in judged) / max(1, len(judged)), 4) for k in keys}
        return fps, jfa_frac, forced, judged, agree

    # the guard at the target (the policy's defaults: >= 99 % of cells exact,
    # mean error <= 0.05 faces), then the same run with the guard off
    pol = S.RefreshPolicy(every=cycle, warm_frames=foam.jfa_warm)
    fps_sur, jfa_frac, forced, judged, agree = surrogate_run(pol)
    off = S.RefreshPolicy(every=cycle, warm_frames=foam.jfa_warm, min_exact=0.0,
                          max_mean_abs_err=math.inf)
    fps_off, jfa_frac_off, _, judged_off, agree_off = surrogate_run(off)
    plain10 = FoamSim.from_foam(foam, JFA_CADENCE=cycle)
    plain10.initialize()
    fps_plain10, _, _ = timed(plain10)
    plain10.ctx.close()
    return {
        "value": round(fps_sur, 3), "unit": UNIT,
        "path": f"surrogate FSC ({args.surrogate_mode}) on every non-JFA frame, exact JFA "
                f"refresh every {cycle} frames, judged per cell on each refresh; drift guard "
                f"at the target (exact_frac >= {pol.min_exact}, mean_abs_err <= "
                f"{pol.max_mean_abs_err}) forces the next frame to a JFA refresh",
        "guard": {"min_exact": pol.min_exact, "max_mean_abs_err": pol.max_mean_abs_err,
                  "forced_refreshes": forced, "jfa_frame_fraction": round(jfa_frac, 4)},
        "guard_off": {"value": round(fps_off, 3), "jfa_frame_fraction": round(jfa_frac_off, 4),
                      "judged_frames": len(judged_off), "agreement": agree_off},
        "plain_jfa_every10_value": round(fps_plain10, 3),
        "judged_frames": len(judged), "agreement": agree,
        "meets_99pct_agreement": agree["exact_frac"] >= 0.99,
        "pairs_last": judged[-1]["pairs"] if judged else None,
        "overflow_last": judged[-1]["overflow"] if judged else None,
    }


def run_surrogate_arm(args, foam, flush, barrier, world):
    """The metric's second arm (surrogate_measure) on the headline foam, with
    the model trained on the headline law (seeds 10-19); then config 4's
    50,000-particle variant (the same law scaled by (1/5)^(1/3), 192^3 grid):
    a model trained on JFA frames of that variant's seeds 10-19, measured on
    held-out seed 20."""
    import time as _time
    import torch
    from fos import inputs
    from fos import surrogate as S

    t0 = _time.perf_counter()
    sur = S.train_default()
    torch.cuda.synchronize()
    train_s = _time.perf_counter() - t0
    out = surrogate_measure(args, foam, sur, flush, barrier, world, args.steps)
    out["train"] = {"seconds": round(train_s, 2), "foams": "headline law, seeds 10-19",
                    "frames": "JFA frames 20-200", "rows": "3,000,000 sampled pairs",
                    "epochs": 30, "lr": 1e-3, "batch": 65536}
    if args.no_surrogate_large:
        return out
    t0 = _time.perf_counter()
    frames = (20, 60, 100)
    big = S.train_default(foams=[inputs.surrogate_variant(s, large=True) for s in range(10, 20)],
                          frames=frames)
    torch.cuda.synchronize()
    train_big = _time.perf_counter() - t0
    held = inputs.surrogate_variant(20, large=True)
    res = surrogate_measure(args, held, big, flush, barrier, world, min(args.steps, 5))
    res["workload"] = (f"{held.name}: N={held.n}, {held.res}^3, held-out seed 20 of the "
                       f"variant law")
    res["train"] = {"seconds": round(train_big, 2), "foams": "50k variant, seeds 10-19",
                    "frames": "JFA frames " + ", ".join(str(f) for f in frames),
                    "rows": "3,000,000 sampled pairs", "epochs": 30, "lr": 1e-3,
                    "batch": 65536}
    out["large_variant"] = res
    return out


def run_warm_jfa(foam, flush):
    """The warm-started JFA (fos_jfa_warm, steps 4, 2, 1, 1 from the previous
    owner grid) beside the exact one: frames/s of the same 5-frame cycles
    (device time, graph replay), owner-label and FSC agreement from one
    relaxed state, and the dirty-tile fraction of the reference's marking
    between two JFA frames."""
    import ctypes as C

    import torch

    from fos import jfa as J
    from fos import runtime
    from fos._lib import call
    from fos.context import stream
    from fos.driver import FoamSim

    s = torch.cuda.current_stream()
    out = {"workload": foam.name, "first_step": None}
    fps = {}
    for name, warm in (("exact", False), ("warm", True)):
        sim = FoamSim.from_foam(foam, jfa_warm=warm)
        out["first_step"] = sim.cfg.JFA_WARM_STEP
        sim.initialize()
        sim.run(40)
        tot = 0.0
        for _ in range(20):
            flush.fill_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            sim.run(5)
            b.record(s)
            b.synchronize()
            tot += a.elapsed_time(b)
        fps[name] = 100.0 / (tot / 1000.0)
        if warm:
            # agreement from one relaxed state: frames 40..44 ran, the last JFA on frame 40
            fields = ("fsc", "fsc_ema", "face_ids", "face_counts", "neighbor_list",
                      "neighbor_used_count", "neighbor_prev_scores")
            snap = {k: getattr(sim.ctx, k).clone() for k in fields}
            n = sim.n

            def finish():
                lab = sim.ctx.labels().clone()
                sim.ctx.majority_filter()
                sim.ctx.accumulate_faces(n)
                sim.ctx.finalize(sim.rad, n)
                return lab, sim.fsc.clone()

            call("fos_jfa_warm", sim.ctx.h, C.c_void_p(sim.pos.data_ptr()),
                 C.c_void_p(sim.rad.data_ptr()), n, sim.cfg.JFA_WARM_STEP, stream())
            lw, fw = finish()
            for k, v in snap.items():
                getattr(sim.ctx, k).copy_(v)
            sim.ctx.jfa_init(sim.pos, sim.rad, n)
            sim.ctx.jfa_passes(n)
            lx, fx = finish()
            out["voxel_agreement"] = round((lw == lx).float().mean().item(), 6)
            out["fsc_agreement"] = round((fw == fx).float().mean().item(), 6)
            # dirty tiles between two JFA frames, as run.py marks them
            pp, rp = sim.pos.clone(), sim.rad.clone()
            sim.run(5)
            runtime.configure(sim.cfg)
            J.init_jfa(max_particles=n, max_res=sim.ctx.max_res)
            J.update_tile_cache(pp, rp, n)
            J.clear_dirty_tiles()
            J.mark_dirty_tiles(sim.pos, sim.rad, n)
            out["dirty_tiles"] = [J.count_dirty_tiles(), J.tiles_per_axis ** 3]
            runtime.ctx().close()
            runtime._ctx = None
    out["frames_per_s"] = {k: round(v, 2) for k, v in fps.items()}
    out["speedup"] = round(fps["warm"] / fps["exact"], 4)
    return out


def run_ensemble(args, barrier, world, rank):
    """Batched ensemble: the 64 foams of the ensemble workload (N ~ U[2k, 20k],
    seed 3; 64^3 / 96^3 / 128^3 grids; per-foam bands), split over the ranks by
    fos.ensemble.partition, advanced --ensemble-frames frames from the end of
    their 20-frame warm start, once with the fixed launch shapes and once with
    the autotuned ones (each from the same warm state).  value = foam-frames/s
    over all ranks (max time over ranks).  Beside it, the same foams run one
    after another through their single-foam frame graphs for 25 frames."""
    import time as _time
    import torch
    from fos import inputs
    from fos.driver import FoamSim
    from fos.ensemble import FIXED, Ensemble, partition

    foams_all = inputs.ensemble()
    mine = partition(foams_all, world)[rank]
    foams = [foams_all[k] for k in mine]
    frames = args.ensemble_frames
    s = torch.cuda.current_stream()
    dev = torch.cuda.current_device()

    def max_over_ranks(ms):
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    def timed_run(ens, n):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        ens.run(n)
        e1.record(s)
        e1.synchronize()
        return max_over_ranks(e0.elapsed_time(e1))

    out = {"foams": len(foams_all), "particles": int(sum(f.n for f in foams_all)),
           "jfa_res": {str(r): sum(f.res == r for f in foams_all) for r in (64, 96, 128)},
           "frames": frames, "unit": "foam-frames/s",
           "split": "foams partitioned over ranks (LPT greedy on N + R^3/450), no collective "
                    "inside a frame"}
    t0 = _time.perf_counter()
    ens = Ensemble(foams)
    ens.initialize()
    ens.run(20)
    torch.cuda.synchronize()
    out["setup_s"] = round(_time.perf_counter() - t0, 2)
    l0 = ens.launch_count()
    ens.run(5)  # one cadence cycle, graphs captured
    torch.cuda.synchronize()
    out["launches_per_5_frames"] = ens.launch_count() - l0
    snap = [t.clone() for t in (ens.pos, ens.rad, ens.rad_target)]
    frame0 = ens.frame
    ens.tuning = FIXED
    ms_fixed = timed_run(ens, frames)
    # the tuned run starts from a fresh ensemble at the same warm state
    ens.close()
    ens = Ensemble(foams)
    ens.initialize()
    ens.run(25)
    torch.cuda.synchronize()
    same_start = all(torch.equal(a, b) for a, b in zip(snap, (ens.pos, ens.rad, ens.rad_target)))
    t0 = _time.perf_counter()
    tuning, report = ens.autotune(reps=3)
    tune_s = _time.perf_counter() - t0
    assert ens.frame == frame0
    ms_tuned = timed_run(ens, frames)
    ens.close()
    nfoam = len(foams_all)
    out["fixed"] = {"tuning": FIXED, "ms_per_frame": round(ms_fixed / frames, 4),
                    "value": round(nfoam * frames / (ms_fixed / 1000.0), 2)}
    out["tuned"] = {"tuning": tuning, "ms_per_frame": round(ms_tuned / frames, 4),
                    "value": round(nfoam * frames / (ms_tuned / 1000.0), 2),
                    "autotune_s": round(tune_s, 2), "candidates_ms": report}
    out["same_start_state"] = same_start
    out["value"] = max(out["fixed"]["value"], out["tuned"]["value"])
    # unbatched: every foam through its own single-foam frame graph
    sims = [FoamSim.from_foam(f) for f in foams]
    for sm in sims:
        sm.initialize()
    for _ in range(25):
        for sm in sims:
            sm.step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(25):
        for sm in sims:
            sm.step()
    e1.record(s)
    e1.synchronize()
    ms_seq = max_over_ranks(e0.elapsed_time(e1))
    for sm in sims:
        sm.ctx.close()
    out["sequential_single_foam"] = {"frames": 25, "ms_per_frame": round(ms_seq / 25, 4),
                                     "value": round(nfoam * 25 / (ms_seq / 1000.0), 2)}
    # with the learned FSC surrogate on every frame between JFA refreshes (one
    # every 10 frames, drift guard off), the headline law's model
    import math
    from fos import surrogate as S
    sur = S.train_default()
    ens = Ensemble(foams)
    ens.initialize()
    ens.attach_surrogate(sur, S.RefreshPolicy(every=10, warm_frames=20, min_exact=0.0,
                                              max_mean_abs_err=math.inf), "absolute")
    ens.run(30)
    torch.cuda.synchronize()
    sframes = 100
    ens.policy.judged.clear()
    ms_sur = timed_run(ens, sframes)
    judged = list(ens.policy.judged)
    ens.close()

    def mean(key):
        return round(sum(d[key] for d in judged) / len(judged), 4) if judged else None
    out["with_surrogate"] = {
        "frames": sframes, "ms_per_frame": round(ms_sur / sframes, 4),
        "value": round(nfoam * sframes / (ms_sur / 1000.0), 2),
        "path": "surrogate FSC (absolute) on every frame between JFA refreshes every 10 frames, "
                "drift guard off; pairs on each foam's own grid",
        "model": "headline law, JFA frames 20-200 of seeds 10-19",
        "judged_frames": len(judged),
        "agreement": {"exact_frac": mean("exact_frac"), "within1_frac": mean("within1_frac"),
                      "mean_abs_err": mean("mean_abs_err"),
                      "stale_exact_frac": mean("stale_exact_frac"),
                      "stale_mean_abs_err": mean("stale_mean_abs_err")}}
    return out


def run_profile(args):
    """Stage timings of one workload with CUDA events (used under ncu as well)."""
    import numpy as np
    import torch

    from fos import inputs
    from fos.config import FosConfig
    from fos.context import Context
    from fos.driver import FoamSim

    torch.cuda.set_device(0)
    foam = inputs.WORKLOADS[args.workload]()
    s = torch.cuda.current_stream()
    out = {"profile": args.profile, "workload": foam.name, "reps": args.reps}
    form_cfg = {"TIE_LOWER_INDEX": True} if args.jfa_form == "label" else {}

    def set_form(ctx):
        ctx.set_jfa_multi_voxel(0 if args.jfa_form in ("single", "staged") else 1)
        ctx.set_jfa_staging(args.jfa_form == "staged")
    if args.profile == "jfa":
        cfg = FosConfig.for_foam(foam, **form_cfg)
        ctx = Context(cfg, max_n=foam.n, max_res=cfg.JFA_RES)
        set_form(ctx)
        f = np.float32
        p = foam.pos - np.floor(foam.pos + f(0.5))
        pos = torch.as_tensor(np.ascontiguousarray(p, np.float32)).cuda()
        rad = torch.as_tensor(foam.rad).cuda()
        stages = {"init": lambda: ctx.jfa_init(pos, rad, foam.n),
                  "passes": lambda: ctx.jfa_passes(foam.n),
                  "filter": ctx.majority_filter,
                  "faces": lambda: ctx.accumulate_faces(foam.n),
                  "finalize": lambda: ctx.finalize(rad, foam.n)}
        acc = {k: 0.0 for k in stages}
        for r in range(args.reps + 1):
            for k, fn in stages.items():
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(s)
                fn()
                b.record(s)
                b.synchronize()
                if r > 0:
                    acc[k] += a.elapsed_time(b)
        out["ms"] = {k: round(v / args.reps, 4) for k, v in acc.items()}
        out["passes"] = ctx.num_passes
        out["stats"] = {k: v for k, v in ctx.jfa_stats(foam.n, rad).items()
                        if k in ("finalize_iterations", "face_pairs", "mean_fsc",
                                 "max_row_candidates")}
    elif args.profile == "ensemble":
        # one 5-frame cadence cycle of the 64-foam ensemble between
        # cudaProfilerStart/Stop, for `ncu --profile-from-start off`
        from fos.ensemble import Ensemble
        ens = Ensemble(inputs.ensemble())
        ens.initialize()
        ens.run(25)
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStart()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        ens.run(5)
        b.record(s)
        b.synchronize()
        torch.cuda.cudart().cudaProfilerStop()
        out["ms_per_frame"] = round(a.elapsed_time(b) / 5, 4)
        out["workload"] = "ensemble-64"
        # one plain frame's dynamics kernel over all foams, phase by phase
        # (%globaltimer after every grid barrier, block 0), outside the
        # profiled range
        tr = ens.trace_dynamics()
        out["dynamics_phase_us"] = [round(x / 1000.0, 1) for x in tr]
        out["dynamics_total_us"] = round(sum(tr) / 1000.0, 1)
        ens.close()
    elif args.profile == "inference":
        # surrogate inference alone on the candidate pairs of the headline foam
        # at frame 60 (a seeded random model): 3 rounds of 1 + 20 predict calls
        # with the mma.sync kernel, then 1 + 20 with the tcgen05 kernel
        from fos import surrogate as S
        from fos._lib import call
        sim = FoamSim.from_foam(foam)
        sim.initialize()
        sim.run(60)
        torch.cuda.synchronize()
        sur = S.Surrogate(seed=3)
        ctx, n = sim.ctx, foam.n
        S.build_pairs(ctx, sur, sim.pos, sim.rad, n, float(sim.cfg.R_MAX), sim.cell_start,
                      sim.cell_count, sim.cell_indices)
        out["pairs"] = S.pair_count(ctx)[0]
        for rnd in range(3):
            for kind in (0, 1):
                call("fos_surrogate_set_inference", ctx.h, kind)
                S.predict(ctx, sur, sim.rad, n)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(s)
                for _ in range(20):
                    S.predict(ctx, sur, sim.rad, n)
                b.record(s)
                b.synchronize()
                key = "tcgen05_us" if kind else "mma_sync_us"
                out.setdefault(key, []).append(round(a.elapsed_time(b) / 20 * 1000, 2))
        out["device_error"] = ctx.device_error()
    elif args.profile == "surrogate":
        # 20 steady-state surrogate frames (2 refresh cycles) between
        # cudaProfilerStart/Stop, for `ncu --profile-from-start off`; the
        # drift guard is off, so 18 of the 20 frames are surrogate frames
        from fos import surrogate as S
        sur = S.train_default(frames=(20, 60, 100), max_rows=1_000_000, epochs=5)
        sim = FoamSim.from_foam(foam, surrogate=sur, surrogate_mode="absolute",
                                policy=S.RefreshPolicy(every=10, warm_frames=foam.jfa_warm,
                                                       min_exact=0.0,
                                                       max_mean_abs_err=math.inf))
        sim.initialize()
        for _ in range(60):
            sim.step()
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStart()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for _ in range(20):
            sim.step()
        b.record(s)
        b.synchronize()
        torch.cuda.cudart().cudaProfilerStop()
        out["ms_per_frame"] = round(a.elapsed_time(b) / 20, 4)
        out["judged"] = [{k: round(float(d[k]), 4) for k in ("exact_frac", "stale_exact_frac",
                                                              "pairs")}
                         for d in sim.policy.judged[-2:]]
    else:
        sim = FoamSim.from_foam(foam, use_graph=True, **form_cfg)
        set_form(sim.ctx)
        sim.initialize()
        for _ in range(min(foam.jfa_warm, 25)):
            sim.step()
        for _ in range(foam.jfa_cadence if foam.jfa_cadence > 1 else 2):  # capture both graphs
            sim.step()
        ms = {"jfa_frame": 0.0, "plain_frame": 0.0}
        cnt = {"jfa_frame": 0, "plain_frame": 0}
        for r in range(args.reps * 5):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            jfa = sim.step()
            b.record(s)
            b.synchronize()
            k = "jfa_frame" if jfa else "plain_frame"
            ms[k] += a.elapsed_time(b)
            cnt[k] += 1
        out["ms"] = {k: round(ms[k] / max(1, cnt[k]), 4) for k in ms}
        out["frames"] = cnt
        # per-stage breakdown (event after every stage, no graph)
        stages = {"jfa_frame": {}, "plain_frame": {}}
        nst = {"jfa_frame": 0, "plain_frame": 0}
        for r in range(args.reps * 5):
            d = sim.step_profiled()
            k = "jfa_frame" if d.pop("jfa") else "plain_frame"
            nst[k] += 1
            for st, v in d.items():
                stages[k][st] = stages[k].get(st, 0.0) + v
        out["stages_ms"] = {k: {st: round(v / max(1, nst[k]), 4) for st, v in d.items()}
                            for k, d in stages.items()}
        tr = sim.trace_dynamics()
        out["coop_phase_us"] = [round(x / 1000.0, 2) for x in tr]
        out["coop_total_us"] = round(sum(tr) / 1000.0, 2)
    print(json.dumps(out), flush=True)
    return 0


def main():
    args = parse()
    if not args.profile:
        use_workload(args.workload)
    if args.profile:
        return run_profile(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_fos(args)


if __name__ == "__main__":
    sys.exit(main())
