"""Ant env-steps/s on B200: the batched FP64 Newton substep behind Physics.

Workload (one bench step = one substep of every env, fresh controls):
  Ant (nq=15, nv=14, nu=8, 57 candidate pairs, plane floor), dt 0.01,
  Newton with tolerance 1e-10 and a 30-iteration cap, 16384 envs per GPU
  (the env count of the plain vs warm-started comparison on Ant),
  qpos = qpos0 + U[-0.1, 0.1], qvel ~ N(0, 0.1^2), ctrl ~ U[-1, 1] each step,
  from seeded generators (synthetic; no dataset), timed after 100 pre-roll
  substeps (the Ant has landed).

Output: one JSON line (rank 0). `value` times pg_step_device with the
controls already in HBM (L2 flushed between timed steps by writing a 256 MB
buffer outside the timed events); `e2e` times the C-ABI path with host
buffers (pinned controls in, qpos out) every step. `--impl reference` times
the CPU restatement of the reference engine (oracle/) on all host cores on
the same workload. Multi-GPU: one process per GPU, envs sharded (weak
scaling, no data-path collective), max time over ranks.
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

TOL = 1e-10
ITERS = 30

# oracle FLOP-counter stages computed by each phase kernel
PHASE_STAGES = {"smooth": ("kinematics", "crba", "vel_rne", "passive_act", "factor_solve"),
                "collide": ("collide",),
                "newton": ("rows", "newton", "pgs", "integrate")}
# DRAM bytes (read + write) per env of each phase kernel, from in-situ ncu
# captures (--cache-control none: the caches hold what the previous launches
# left) of the headline's phase kernels at 16384 Ant envs after 100 substeps:
# smooth 65.3 + 93.8 MB, collide 98.0 + 53.2 MB, Newton (newton_plain_kernel)
# 131.7 + 48.6 MB per launch. The work record the phases hand each other (12 KB per env, 200 MB
# at 16384 envs) is larger than the 126 MB L2, so most of it reaches HBM.
NCU_TRAFFIC_PER_ENV = {"smooth": 9711.0, "collide": 9227.0, "newton": 11004.0}
# DRAM bytes (read + write) per image of render_kernel, from one ncu capture of a
# whole frame of 4096 Ant images (the render benchmark's view): 8.2 + 274.0 MB
# at 64 x 64, 6.8 + 787.6 MB at 128 x 128 (the images written are 12 B a pixel:
# 49152 and 196608 B an image).
NCU_RENDER_TRAFFIC_PER_IMAGE = {64: 68894.0, 128: 193949.0}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--envs", type=int, default=16384, help="envs per GPU")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shape")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start variant")
    ap.add_argument("--lanes", type=int, default=0, help="force lanes per env (8, 16, 32)")
    ap.add_argument("--per-block", type=int, default=0, help="force envs per block")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--learned-eval", action="store_true",
                    help="the learned warm-start evaluation (Ant and tabletop) instead of the headline")
    ap.add_argument("--learned-samples", type=int, default=10_000_000, help="training pairs per scene")
    ap.add_argument("--preroll", type=int, default=100,
                    help="substeps run before the warm-up (the Ant lands first), outside every timed region")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip configs 2-5 (tabletop, hull tumble, contact-free, learned evaluation) in the line")
    ap.add_argument("--extras-steps", type=int, default=50, help="timed substeps of each extra config")
    ap.add_argument("--learned-envs", type=int, default=16384)
    ap.add_argument("--solver", default="newton", choices=["newton", "pgs"], help="solver of --scene")
    ap.add_argument("--scene", default="", choices=["", "tabletop", "hull_tumble", "cartpole", "arm3hinge", "big_hulls"],
                    help="phase timing of another workload (configs 2-4; big_hulls: hulls of 96 and 276 vertices) "
                    "beside the oracle, instead of the headline")
    ap.add_argument("--render", default="", help="batched rendering of Ant poses at these square resolutions "
                    "(comma-separated, e.g. 64,128) instead of the headline")
    ap.add_argument("--render-envs", type=int, default=4096, help="envs rendered per frame (the reference's "
                    "render benchmark renders 4096)")
    ap.add_argument("--aux", action="store_true", help="per-call device time of the auxiliary kernels (set_const, "
                    "pose export, reset, learned inference, network training, hull support) instead of the headline")
    return ap.parse_args()


def workload(envs, preroll=100):
    return {"workload": f"ant: {envs} envs/GPU, dt 0.01, Newton tol 1e-10 cap {ITERS}, "
                        f"qpos0+U[-0.1,0.1], qvel N(0,0.1^2), ctrl U[-1,1] per step, timed after {preroll} "
                        "pre-roll substeps (landed)",
            "model": "ant (nq 15, nv 14, nu 8)", "envs_per_gpu": envs, "substeps_per_step": 1,
            "l2": "flushed between timed steps (256 MB write)"}


def initial_state(m, n, seed):
    rng = np.random.default_rng(seed)
    q = np.tile(np.array(m.qpos0), (n, 1)) + rng.uniform(-0.1, 0.1, (n, m.nq))
    v = rng.normal(0.0, 0.1, (n, m.nv))
    return q, v, rng


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def shard_seeds(rank):
    """Seeds of a rank's own envs: every rank steps its own independent set
    (weak scaling; envs never cross ranks, so the step has no collective)."""
    return {"state": 1000 + rank, "train_state": 3000 + rank, "train_ctrl": 2000 + rank}


def whole_job(ms, envs_per_rank, steps, ws):
    """Max over ranks of each timed total (ms, a list) and the whole-job
    rates they give: every rank's envs count, the slowest rank's time
    decides. Takes part in one all-reduce when ws > 1 (every rank calls it)."""
    import torch
    t = torch.tensor(ms, dtype=torch.float64)
    if ws > 1:
        import torch.distributed as dist
        if dist.get_backend() == "nccl":
            t = t.cuda()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    mx = [float(x) for x in t.cpu()]
    total = envs_per_rank * ws * steps
    return mx, [total / (x * 1e-3) for x in mx]


# ------------------------------------------------------------------ CPU legs
def cpu_rollout_rate(blob, m, envs, seconds, fast=True):
    """Oracle rollout (batch.rs:46-59 shape) on all host threads, repeated
    until `seconds` of work; returns (env-steps/s, threads, sample text)."""
    from oracle.oracle import QPOS, QVEL, Oracle
    o = Oracle(blob, envs, threads=0, fast=fast)
    o.set_solver(tolerance=TOL, iterations=ITERS)
    q, v, rng = initial_state(m, envs, 1)
    o.set(QPOS, q)
    o.set(QVEL, v)
    nstep = 200
    done, t0, reps = 0, time.perf_counter(), 0
    while True:
        ctrl = rng.uniform(-1, 1, (envs, nstep, m.nu))
        o.rollout(ctrl, record=False)
        done += envs * nstep
        reps += 1
        el = time.perf_counter() - t0
        if el >= seconds or reps >= 50:
            break
    return done / el, o.threads, f"Ant {envs} envs x {nstep} steps rollout x {reps} (oracle, {o.threads} threads)"


def algorithmic_flops(blob, m, envs=256, steps=120):
    """FP64 operations per Ant env-step of the reference algorithm as written
    (the oracle's per-stage counters, averaged over a seeded trajectory)."""
    from oracle.oracle import QPOS, QVEL, Oracle
    o = Oracle(blob, envs, threads=0, fast=False)
    o.set_solver(tolerance=TOL, iterations=ITERS)
    q, v, rng = initial_state(m, envs, 2)
    o.set(QPOS, q)
    o.set(QVEL, v)
    o.flops(reset=True)
    o.rollout(rng.uniform(-1, 1, (envs, steps, m.nu)), record=False)
    f = o.flops()
    return sum(f.values()) / (envs * steps), {k: v / (envs * steps) for k, v in f.items()}


def run_reference(args):
    """--impl reference: the oracle on the host cores, same workload."""
    ws, rank, _ = dist_setup(args)
    if rank != 0:
        return
    from oracle.oracle import CTRL, QPOS, QVEL, Oracle
    from pippin_b200 import mjcf, scenes
    xml = scenes.ant_xml()
    m = mjcf.load_string(xml)
    blob = mjcf.to_blob(m)
    n = args.envs * max(args.gpus, 1)
    o = Oracle(blob, n, threads=0, fast=True)
    o.set_solver(tolerance=TOL, iterations=ITERS)
    q, v, rng = initial_state(m, n, 1)
    o.set(QPOS, q)
    o.set(QVEL, v)
    P = args.preroll
    ctrls = [rng.uniform(-1, 1, (n, m.nu)) for _ in range(P + args.warmup + args.steps)]
    for k in range(P + args.warmup):  # pre-roll (the Ant lands) and warm-up, untimed
        o.set(CTRL, ctrls[k])
        o.step(0, n, 1)
    t0 = time.perf_counter()
    for k in range(args.steps):
        o.set(CTRL, ctrls[P + args.warmup + k])
        o.step(0, n, 1)
    el = time.perf_counter() - t0
    value = n * args.steps / el
    line = {"metric": "Ant env-steps/s", "value": value, "unit": "env-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload(args.envs, P), parallelism=f"{o.threads} host threads"), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "env-steps/s", "cores": o.threads, "kind": "port",
                             "sample": f"Ant {n} envs x {args.steps} steps (Physics::step shape, per-step ctrl)"},
            "e2e": {"value": value, "unit": "env-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms. start()
    returns once the first sample is in (nvidia-smi's own start-up, which
    briefly disturbs the GPU, then falls before the timed region); stop()
    waits for the next sample and reports those taken from the return of
    start() to that one, so a region shorter than the period still has the
    sample that closes it."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.skip = 0

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
            return
        t0 = time.perf_counter()
        while not self.lines and self.proc.poll() is None and time.perf_counter() - t0 < 10.0:
            time.sleep(0.01)
        self.skip = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        n_end, t0 = len(self.lines), time.perf_counter()
        while len(self.lines) <= n_end and self.proc.poll() is None and time.perf_counter() - t0 < 1.0:
            time.sleep(0.01)
        n_end = min(len(self.lines), n_end + 1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[self.skip:n_end] or self.lines[-1:]:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for name, val in zip(names, p[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ our arm
def run_ours(args):
    import torch

    from pippin_b200 import CudaPhysics, Field, mjcf, scenes
    from pippin_b200.physics import WarmStart, fp64_peak

    ws, rank, local = dist_setup(args)
    if ws > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    xml = scenes.ant_xml(tolerance=TOL, iterations=ITERS)
    m = mjcf.load_string(xml)
    blob = mjcf.to_blob(m)
    n = args.envs
    phys = CudaPhysics(blob, n)
    q, v, rng = initial_state(m, n, shard_seeds(rank)["state"])
    phys.set(Field.QPOS, range(n), q)
    phys.set(Field.QVEL, range(n), v)
    K, W, P = args.steps, args.warmup, args.preroll
    ctrl_all = torch.from_numpy(rng.uniform(-1, 1, (P + W + K, n, m.nu))).to(dev)
    # pre-roll (outside every timed region): the Ant falls from qpos0 and
    # lands, so that the timed steps see ground contact; every variant then
    # starts from this state
    phys.set_solver(warm=int(WarmStart.REF_PREV_QACC))
    for k in range(P):
        phys.step_device(range(n), 1, ctrl_all[k].data_ptr())
    snap = {f: phys.get(f, range(n)) for f in (Field.QPOS, Field.QVEL, Field.QACC)}

    def restore():
        for f, x in snap.items():
            phys.set(f, range(n), x)

    if args.lanes or args.per_block:
        phys.set_launch(args.lanes, args.per_block)
    elif not args.no_autotune:
        phys.autotune(nstep=4)  # trial steps run on a saved copy of the state
    lanes, per_block, blocks = phys.launch()
    phase_shapes = phys.phase_launch()
    clocks = ClockSampler(local)
    clocks.start()

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.ExternalStream(phys.stream(), device=dev)

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    def timed_device_loop(warm):
        restore()
        phys.set_solver(warm=int(warm))
        for k in range(W):
            phys.step_device(range(n), 1, ctrl_all[P + k].data_ptr())
        phys.synchronize()
        barrier()
        total_ms = 0.0
        iters = []
        for k in range(K):
            flush.fill_(float(k))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            phys.step_device(range(n), 1, ctrl_all[P + W + k].data_ptr())
            e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
            st = phys.stats()
            iters.append(st["iters"][st["nrows"] > 0])
        barrier()
        return total_ms, st, np.concatenate(iters)

    ms_ref, st, it_ref = timed_device_loop(WarmStart.REF_PREV_QACC)
    ms_cold, st_cold, it_cold = timed_device_loop(WarmStart.COLD)
    # learned warm start (one GPU): a network trained on the plain solver's
    # converged contact forces (config 5's training set: 10M pairs from a
    # 16384-env Ant run), then the same workload again
    learned, extras = None, {}
    if not args.no_learned and ws == 1:
        ant_line, wts = learned_eval("ant", args.learned_envs, args.learned_samples, args.extras_steps, 5)
        extras["learned_ant"] = ant_line
        phys.set_warm_mlp(wts)
        ms_learned, st_l, it_l = timed_device_loop(WarmStart.LEARNED)
        learned = {"value": n * ws * K / (ms_learned * 1e-3), "ms_per_step": ms_learned / K,
                   "mean_iters": float(it_l.mean()) if len(it_l) else 0.0,
                   "p99_iters": float(np.percentile(it_l, 99)) if len(it_l) else 0.0,
                   "train_samples": ant_line["train"]["samples"], "train_loss": ant_line["train"]["loss"]}
    phys.set_solver(warm=int(WarmStart.REF_PREV_QACC))

    # end to end through the C-ABI with host buffers
    pin_ctrl = torch.empty((n, m.nu), dtype=torch.float64, pin_memory=True).numpy()
    pin_q = torch.empty((n, m.nq), dtype=torch.float64, pin_memory=True).numpy()
    ctrl_host = ctrl_all.cpu().numpy()
    restore()
    for k in range(W):
        pin_ctrl[:] = ctrl_host[P + k]
        phys.set(Field.CTRL, range(n), pin_ctrl)
        phys.step(range(n), 1)
        phys.get(Field.QPOS, range(n), out=pin_q)
    barrier()
    e2e_ms = 0.0
    for k in range(K):
        pin_ctrl[:] = ctrl_host[P + W + k]
        flush.fill_(float(k))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        phys.set(Field.CTRL, range(n), pin_ctrl)
        phys.step(range(n), 1)
        phys.get(Field.QPOS, range(n), out=pin_q)
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    barrier()

    # per-phase device time over K further substeps of the same workload
    # (same start state, same warm-up), one event pair per phase kernel
    restore()
    for k in range(W):
        phys.step_device(range(n), 1, ctrl_all[P + k].data_ptr())
    phys.synchronize()
    phase_ms = {"smooth": 0.0, "collide": 0.0, "newton": 0.0}
    torch.cuda.nvtx.range_push("phase_timing")  # profilers can limit themselves to these launches
    for k in range(K):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        for name, ms in phys.time_phases(range(n), 1, ctrl_all[P + W + k].data_ptr()).items():
            phase_ms[name] = phase_ms.get(name, 0.0) + ms
    torch.cuda.nvtx.range_pop()
    barrier()
    clock_info = clocks.stop()

    (ms_ref, ms_cold, e2e_ms), (value, value_cold, e2e) = whole_job([ms_ref, ms_cold, e2e_ms], n, K, ws)

    if rank == 0:
        peak = fp64_peak(local)
        flops_step, per_stage = algorithmic_flops(blob, m)
        phase_flops = {ph: sum(per_stage.get(st, 0.0) for st in stages) for ph, stages in PHASE_STAGES.items()}
        top = max(phase_ms, key=phase_ms.get)
        per_launch_ms = phase_ms[top] / K
        achieved = phase_flops[top] * n / (per_launch_ms * 1e-3) / 1e12
        phase_total = sum(phase_ms.values())
        bytes_step = (m.nq + m.nv + m.nv + m.nu) * 8 + (m.nq + m.nv + m.nv) * 8
        line = {
            "metric": "Ant env-steps/s", "value": value, "unit": "env-steps/s", "n_gpus": ws, "steps": K,
            "warmup": W, "ms_per_step": ms_ref / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload(n, P), parallelism=f"env-sharded x{ws} (no collective)",
                           launch={"lanes_per_env": lanes, "envs_per_block": per_block, "blocks": blocks}),
            "e2e": {"value": e2e, "unit": "env-steps/s", "h2d_bytes_per_step": n * m.nu * 8,
                    "d2h_bytes_per_step": n * m.nq * 8},
            "gpu_launches": 3 * K,
            "variants": {"newton_ref_prev_qacc": value, "newton_cold": value_cold,
                         "mean_iters_ref": float(it_ref.mean()) if len(it_ref) else 0.0,
                         "mean_iters_cold": float(it_cold.mean()) if len(it_cold) else 0.0,
                         "p99_iters_ref": float(np.percentile(it_ref, 99)) if len(it_ref) else 0.0,
                         "p99_iters_cold": float(np.percentile(it_cold, 99)) if len(it_cold) else 0.0,
                         "iters_over": "envs with constraint rows",
                         "newton_learned": learned,
                         "mean_ncon": float(st["ncon"].mean()), "mean_rows": float(st["nrows"].mean())},
            # (the headline's Newton phase runs the instance without the learned start's code)
            "roofline": {"bound": "fp64", "kernel": {"newton": "newton_plain_kernel"}.get(top, f"{top}_kernel"),
                         "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": NCU_TRAFFIC_PER_ENV.get(top, 0.0) * n or None,
                         "note": f"{phase_flops[top]:.0f} algorithmic FP64 ops per env in the {top} phase (oracle "
                                 f"counters, {flops_step:.0f} per whole env-step) x {n} envs per launch / that "
                                 "kernel's mean event-timed duration; peak = live DFMA microbenchmark (pg_fp64_peak); "
                                 "traffic = in-situ ncu DRAM bytes per env of that kernel x envs",
                         "hbm_achieved_gbs": bytes_step * n / (ms_ref / K * 1e-3) / 1e9},
            "phases": {ph: {"ms_per_launch": phase_ms[ph] / K, "share": phase_ms[ph] / phase_total,
                            "fp64_ops_per_env": phase_flops.get(ph),
                            "launch": dict(zip(("lanes_per_env", "envs_per_block", "blocks"), phase_shapes[ph]))}
                       for ph in phase_ms if ph in phase_shapes},
            "clocks": clock_info,
        }
        if ws == 1 and not args.no_cpu_baseline:
            rate, cores, sample = cpu_rollout_rate(blob, m, 1024, args.cpu_seconds)
            line["cpu_baseline"] = {"value": rate, "unit": "env-steps/s", "cores": cores, "kind": "port",
                                    "sample": sample}
    phys.close()
    if rank == 0 and ws == 1 and not args.no_extras:
        # configs 2-5 beside the headline, each with its oracle sample on the
        # host cores (bounded: a few seconds of GPU time each)
        E = args.extras_steps
        extras["tabletop"] = scene_measure("tabletop", 8192, E, 300)
        extras["hull_tumble"] = scene_measure("hull_tumble", 4096, E, 250)
        extras["hull_tumble_pgs"] = scene_measure("hull_tumble", 4096, E, 250, solver=1)
        extras["cartpole"] = scene_measure("cartpole", 16384, 4 * E, 50)
        extras["arm3hinge"] = scene_measure("arm3hinge", 16384, 4 * E, 50)
        if not args.no_learned:
            extras["learned_tabletop"], _ = learned_eval("tabletop", args.learned_envs, args.learned_samples, E, 5)
    if rank == 0:
        if extras:
            line["configs"] = extras
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def learned_eval(name, n, samples, K, W, weights=None, epochs=8):
    """The learned Newton warm start on Ant or the tabletop scene (config 5):
    training pairs (24 contact features -> converged frame forces) from the
    plain solver's own converged solves, a network fitted to them on the GPU
    (or `weights`, when given), then cold start vs learned start on the same
    workload at the same 1e-10 tolerance (iteration counts and CUDA-graph
    step time). Returns (the JSON line as a dict, the weights)."""
    import torch
    from pippin_b200 import CudaPhysics, Field, Param, WarmStart, mjcf, scenes, warm
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)

    def ant(seed):
        m = mjcf.load_string(scenes.ant_xml(tolerance=TOL, iterations=ITERS))
        p = CudaPhysics(mjcf.to_blob(m), n)
        q, v, rng = initial_state(m, n, seed)
        p.set(Field.QPOS, range(n), q)
        p.set(Field.QVEL, range(n), v)
        return m, p, (lambda t: rng.uniform(-1, 1, (n, m.nu))), 100

    def tabletop(seed):
        plan = scenes.tabletop(n, seed=seed)
        m = mjcf.load_string(plan.xml)
        p = CudaPhysics(mjcf.to_blob(m), n)
        p.set_solver(tolerance=TOL, iterations=ITERS)
        plan.apply(lambda pid, elem, vals: p.set_param(Param(pid), elem, range(n), vals), lambda: p.reset(range(n)))
        return m, p, None, 100

    make = ant if name == "ant" else tabletop
    train = None
    if weights is None:
        t0 = time.perf_counter()
        m, p, controls, skip = make(11)
        xs, fs, steps = [], [], 0
        for t in range(skip):
            if controls is not None:
                p.set(Field.CTRL, range(n), controls(t))
            p.step(range(n), 1)
        got = 0
        while got < samples and steps < 20000:
            if controls is not None:
                p.set(Field.CTRL, range(n), controls(steps))
            X, F = p.warm_samples(range(n))
            xs.append(X)
            fs.append(F)
            got += len(X)
            steps += 1
            if name == "tabletop" and steps % 200 == 0:  # objects at rest: drop a fresh batch
                p.close()
                m, p, controls, _ = make(11 + steps)
        p.close()
        X, F = np.concatenate(xs)[:samples], np.concatenate(fs)[:samples]
        t_collect = time.perf_counter() - t0
        t0 = time.perf_counter()
        weights, losses = warm.train(X, F, epochs=epochs, batch=8192, lr=1e-3, seed=1)
        train = {"samples": int(len(X)), "collect_steps": steps, "epochs": epochs,
                 "loss": [float(losses[0]), float(losses[-1])], "collect_s": t_collect,
                 "train_s": time.perf_counter() - t0}
    out = {}
    for mode, wm in (("cold", WarmStart.COLD), ("ref_prev_qacc", WarmStart.REF_PREV_QACC),
                     ("learned", WarmStart.LEARNED)):
        m, p, controls, skip = make(7)
        p.set_warm_mlp(weights)
        p.set_solver(warm=int(wm))
        ctrl = None
        if controls is not None:
            ctrl = torch.from_numpy(np.stack([controls(t) for t in range(skip + W + K)])).to(dev)
        for t in range(skip + W):
            p.step_device(range(n), 1, ctrl[t].data_ptr() if ctrl is not None else 0)
        p.synchronize()
        stream = torch.cuda.ExternalStream(p.stream(), device=dev)
        iters, ms = [], 0.0
        for k in range(K):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            p.step_device(range(n), 1, ctrl[skip + W + k].data_ptr() if ctrl is not None else 0)
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            st = p.stats()
            iters.append(st["iters"][st["nrows"] > 0])
        p.close()
        it = np.concatenate(iters)
        out[mode] = {"env_steps_per_s": n * K / (ms * 1e-3), "ms_per_step": ms / K,
                     "mean_iters": float(it.mean()) if len(it) else 0.0,
                     "p99_iters": float(np.percentile(it, 99)) if len(it) else 0.0}
    line = {"metric": f"learned warm start, {name}", "impl": "ours", "envs": n, "steps": K, "warmup": W,
            "tolerance": TOL, "dtype": "f64 physics, bf16 network (fp32 accumulate)", "data": "synthetic",
            "train": train, "iters_over": "envs with constraint rows", "timed_after_substeps": skip + W}
    line.update(out)
    return line, weights


def run_learned_eval(args):
    """--learned-eval: one JSON line per scene (Ant, tabletop), rank 0, one GPU."""
    for name in ("ant", "tabletop"):
        line, _ = learned_eval(name, args.learned_envs, args.learned_samples, args.steps, max(args.warmup, 3))
        print(json.dumps(line), flush=True)


def scene_measure(scene, n, K, W, cpu=True, solver=0):
    """Device env-steps/s and per-phase time of the tabletop (config 3), the
    hull tumble (config 4), the large-hull scene (scenes.big_hulls_xml, with
    the hull tumble's initial velocities) or a contact-free model (config 2: random states
    over the joint ranges, qvel N(0, 1), per-env masses x U[0.5, 2], random
    controls held) after W settling substeps, with the oracle's rate on a
    bounded sample of the same workload on the host cores beside it; solver
    0 is Newton, 1 PGS (both sides). Returns the JSON line as a dict (one
    GPU)."""
    import torch
    from oracle.oracle import CTRL, QPOS, QVEL, Oracle
    from pippin_b200 import CudaPhysics, Field, Param, mjcf, scenes
    torch.cuda.set_device(0)
    if scene == "tabletop":
        plan = scenes.tabletop(n, seed=5)
        m = mjcf.load_string(plan.xml)
        desc = (f"tabletop: {n} envs, 2-6 objects each (boxes, cylinders, spheres), dropped 5-15 cm, dt 0.002, "
                f"Newton tol 1e-10 cap {ITERS}; timed after {W} substeps")
    elif scene in ("cartpole", "arm3hinge"):
        m = mjcf.load_string(scenes.cartpole_xml() if scene == "cartpole" else scenes.arm3hinge_xml())
        desc = (f"{scene}: {n} envs, qpos uniform over the joint ranges (hinges [-pi, pi], slides +-0.5), "
                f"qvel N(0,1), per-env masses x U[0.5,2], controls U[-1,1] held; timed after {W} substeps")
    elif scene == "big_hulls":
        m = mjcf.load_string(scenes.big_hulls_xml())
        desc = (f"big hulls: {n} envs of two 276-vertex hulls, two 96-vertex prisms (48-gon faces), a box, a sphere "
                f"and a capsule, v N(0,0.5^2), w N(0,3^2), dt 0.002, Newton tol 1e-10 cap {ITERS}; timed after {W} "
                "substeps")
    else:
        m = mjcf.load_string(scenes.hull_tumble_xml())
        desc = (f"hull tumble: {n} envs of 8 hulls (8-32 vertices), v N(0,0.5^2), w N(0,3^2), dt 0.002, "
                f"Newton tol 1e-10 cap {ITERS}; timed after {W} substeps")
    blob = mjcf.to_blob(m)

    def setup(sim, count, set_param, reset, set_q, set_v, set_ctrl=None):
        if scene == "tabletop":
            pl = scenes.tabletop(count, seed=5)
            for pid, elem, vals in pl.params:
                set_param(pid, elem, vals)
            set_param(11, 0, pl.qpos0)
            reset()
        elif scene in ("cartpole", "arm3hinge"):
            rng = np.random.default_rng(5)
            q = np.tile(np.array(m.qpos0), (count, 1))
            for j in range(m.njnt):
                qa = m.jnt_qposadr[j]
                if m.jnt_type[j] == mjcf.JNT_HINGE:
                    q[:, qa] = rng.uniform(-np.pi, np.pi, count)
                elif m.jnt_type[j] == mjcf.JNT_SLIDE:
                    q[:, qa] = rng.uniform(-0.5, 0.5, count)
            for b in range(1, m.nbody):
                set_param(5, b, (np.array(m.body_mass[b]) * rng.uniform(0.5, 2.0, count)).reshape(count, 1))
            set_q(q)
            set_v(rng.normal(0, 1, (count, m.nv)))
            set_ctrl(rng.uniform(-1, 1, (count, m.nu)))
        else:
            rng = np.random.default_rng(5)
            v = np.zeros((count, m.nv))
            for b in range(m.nv // 6):
                v[:, 6 * b:6 * b + 3] = rng.normal(0, 0.5, (count, 3))
                v[:, 6 * b + 3:6 * b + 6] = rng.normal(0, 3.0, (count, 3))
            set_q(np.tile(np.array(m.qpos0), (count, 1)))
            set_v(v)

    p = CudaPhysics(blob, n)
    p.set_solver(kind=solver, tolerance=TOL, iterations=ITERS)
    setup(p, n, lambda pid, elem, vals: p.set_param(Param(pid), elem, range(n), vals), lambda: p.reset(range(n)),
          lambda q: p.set(Field.QPOS, range(n), q), lambda v: p.set(Field.QVEL, range(n), v),
          lambda c: p.set(Field.CTRL, range(n), c))
    p.step(range(n), W)
    p.autotune(nstep=2)
    stream = torch.cuda.ExternalStream(p.stream(), device=torch.device("cuda", 0))
    # the held controls, in device memory for pg_step_device
    ctrl = torch.from_numpy(p.get(Field.CTRL, range(n))).cuda() if m.nu > 0 else None
    p.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    p.step_device(range(n), K, ctrl.data_ptr() if ctrl is not None else 0)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    ph = {"smooth": 0.0, "collide": 0.0, "newton": 0.0}
    torch.cuda.nvtx.range_push("phase_timing")  # profilers can limit themselves to these launches
    for k in range(K):
        for name, t in p.time_phases(range(n), 1).items():
            ph[name] = ph.get(name, 0.0) + t
    torch.cuda.nvtx.range_pop()
    st = p.stats()
    launch = p.phase_launch()
    p.close()
    # the oracle on a sample of the same workload (same settling, then timed)
    # (the oracle tests every edge pair of the 276-vertex hulls: a small sample)
    cn = 4096 if scene in ("cartpole", "arm3hinge") else (16 if scene == "big_hulls" else 256)
    if solver == 1:
        desc = desc.replace("Newton tol 1e-10 cap", "PGS cap")
    line = {"metric": f"{scene}{' (PGS)' if solver == 1 else ''} env-steps/s", "value": n * K / (ms * 1e-3),
            "unit": "env-steps/s",
            "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic", "config": {"workload": desc, "envs": n},
            "phases": {k: {"ms_per_launch": v / K, "launch": dict(zip(("lanes_per_env", "envs_per_block", "blocks"),
                                                                       launch[k]))} for k, v in ph.items()},
            "mean_ncon": float(st["ncon"].mean()), "mean_rows": float(st["nrows"].mean()),
            "mean_iters": float(st["iters"].mean())}
    if not cpu:
        return line
    o = Oracle(blob, cn, threads=0, fast=True)
    o.set_solver(kind=solver, tolerance=TOL, iterations=ITERS)
    setup(o, cn, lambda pid, elem, vals: o.set_param(pid, elem, np.asarray(vals), 0, cn),
          lambda: o.reset(list(range(cn))), lambda q: o.set(QPOS, q), lambda v: o.set(QVEL, v),
          lambda c: o.set(CTRL, c))
    o.step(0, cn, W)
    t0 = time.perf_counter()
    ck = max(1, min(K, 100 if cn > 256 else 50))
    o.step(0, cn, ck)
    cpu_rate = cn * ck / (time.perf_counter() - t0)
    line["cpu_baseline"] = {"value": cpu_rate, "unit": "env-steps/s", "cores": o.threads, "kind": "port",
                            "sample": f"{scene} {cn} envs x {ck} substeps after the same settling (oracle)"}
    o.close()
    return line


def run_scene(args):
    line = scene_measure(args.scene, args.envs, args.steps, max(args.warmup, 3),
                         solver=1 if args.solver == "pgs" else 0)
    print(json.dumps(line), flush=True)


def run_aux(args):
    """Device time per call of the kernels outside the substep's three phases,
    each on a small workload through the public API (CUDA events on the
    handle's stream): set_const after a per-env mass change
    (set_const_kernel), pose export into device buffers (poses_kernel), reset
    (reset_kernel), a substep with the learned start (learn_kernel, between
    the collision and Newton phases), the network's forward pass and a
    training epoch (mlp_forward_kernel; gemm_kernel, gemm_atb_kernel,
    sum_splits_kernel, colsum_split_kernel, mse_kernel, loss_add_kernel,
    adam_kernel, gather_kernel) and the hull support walk
    (hull_support_kernel) over 2000 directions on a 276-vertex hull. Each
    runs once inside the NVTX range "aux_once" (one launch of each kernel,
    one training batch, for profilers) before it is timed."""
    import ctypes as C

    import torch
    from pippin_b200 import CudaPhysics, Field, Param, _native, mjcf, scenes, warm
    from pippin_b200.physics import WarmStart
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    n = args.envs
    m = mjcf.load_string(scenes.ant_xml(tolerance=TOL, iterations=ITERS))
    p = CudaPhysics(mjcf.to_blob(m), n)
    stream = torch.cuda.ExternalStream(p.stream(), device=dev)
    rng = np.random.default_rng(7)
    L = _native.load()
    out = {}

    def timed(name, fn, reps=5):
        p.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        out[name] = e0.elapsed_time(e1) / reps

    # states, contacts and a network fitted to them, outside the range
    q = np.tile(np.array(m.qpos0), (n, 1)) + rng.uniform(-0.1, 0.1, (n, m.nq))
    p.set(Field.QPOS, range(n), q)
    p.set(Field.QVEL, range(n), rng.normal(0, 0.1, (n, m.nv)))
    X, F = warm.collect(p, 120, controls=lambda t: rng.uniform(-1, 1, (n, m.nu)), skip=60)
    k = min(len(X), 1 << 18)
    w, _ = warm.train(X[:k], F[:k], epochs=1, batch=8192, lr=1e-3, seed=1)
    masses = np.array(m.body_mass[1]) * rng.uniform(0.5, 2.0, (n, 1))
    sc = p.scene()
    gd = torch.empty(n * len(sc.geoms) * 12, dtype=torch.float32, device=dev)
    hm = mjcf.load_string(scenes.lumpy_hull_xml())
    h = CudaPhysics(mjcf.to_blob(hm), 1)
    d = np.ascontiguousarray(scenes.support_directions())
    v = np.zeros(len(d), dtype=np.int32)

    def hull_support():
        rc = L.pg_hull_support(h._h, 0, d.ctypes.data_as(C.POINTER(C.c_double)), len(d),
                               v.ctypes.data_as(C.POINTER(C.c_int32)))
        if rc != 0:
            raise RuntimeError(_native.last_error())

    p.set_warm_mlp(w)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("aux_once")
    p.set_param(Param.BODY_MASS, 1, range(n), masses)
    p.poses_device(range(n), gd.data_ptr(), 0)
    p.reset(range(n))
    p.synchronize()
    torch.cuda.nvtx.range_pop()
    p.set(Field.QPOS, range(n), q)  # the Ant lands: the learned substep has contacts
    p.step(range(n), 100)
    p.synchronize()
    torch.cuda.nvtx.range_push("aux_once")
    warm.forward(w, X[:8192])
    warm.train(X[:8192], F[:8192], epochs=1, batch=8192, lr=1e-3, seed=2)
    p.set_solver(warm=int(WarmStart.LEARNED))
    p.time_phases(range(n), 1)
    hull_support()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()

    timed("set_param_body_mass_ms", lambda: p.set_param(Param.BODY_MASS, 1, range(n), masses))
    timed("poses_device_ms", lambda: p.poses_device(range(n), gd.data_ptr(), 0))
    timed("reset_ms", lambda: p.reset(range(n)))
    p.set(Field.QPOS, range(n), q)
    p.step(range(n), 100)
    ph = {}
    for _ in range(5):
        for name, ms in p.time_phases(range(n), 1).items():
            ph[name] = ph.get(name, 0.0) + ms / 5
    out["learned_substep_phase_ms"] = ph
    t0 = time.perf_counter()
    warm.forward(w, X[:k])
    out["mlp_forward_host_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    warm.train(X[:k], F[:k], epochs=1, batch=8192, lr=1e-3, seed=3)
    out["train_epoch_host_s"] = time.perf_counter() - t0
    out["train_samples"] = int(k)
    t0 = time.perf_counter()
    hull_support()
    out["hull_support_host_s"] = time.perf_counter() - t0
    hv = np.asarray(hm.hull_vert[0])
    out["hull_support_exact"] = bool(np.abs((hv @ d.T).max(axis=0) - np.einsum("ij,ij->i", hv[v], d)).max() < 1e-12)
    h.close()
    p.close()
    print(json.dumps({"metric": "auxiliary kernels, time per call", "envs": n, "workload": "ant", **out}), flush=True)


def hbm_peak() -> float:
    """Measured HBM copy bandwidth (GB/s) from MEASURED_PEAKS.json, else the
    pool's earlier measurement of 6650 GB/s."""
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


def run_render(args):
    """Frames/s of the batched rasteriser on Ant poses (the reference's
    render benchmark, crates/pippin-render/examples/render_bench.rs: Ant
    after 50 steps, one fixed view, RGB + depth + segmentation), one JSON line
    per resolution. `value` times the kernel from device-resident poses with
    CUDA events; `e2e` times the host call (poses up, images down)."""
    import torch

    from pippin_b200 import CudaPhysics, Field, mjcf, scenes
    from pippin_b200 import render as R

    dev = torch.device("cuda", 0)
    n, K, W = args.render_envs, args.steps, max(args.warmup, 3)
    m = mjcf.load_string(scenes.ant_xml(tolerance=TOL, iterations=ITERS))
    phys = CudaPhysics(mjcf.to_blob(m), n)
    q, v, rng = initial_state(m, n, shard_seeds(0)["state"])
    phys.set(Field.QPOS, range(n), q)
    phys.set(Field.QVEL, range(n), v)
    phys.step(range(n), 50)
    g, c = phys.poses(range(n))  # host copies, for the e2e leg
    sc = phys.scene()
    ctrl = torch.from_numpy(rng.uniform(-1, 1, (n, m.nu))).to(dev)
    pstream = torch.cuda.ExternalStream(phys.stream(), device=dev)
    published = {64: 310_000.0, 128: 195_000.0}  # README.md:115-116, 4096 Ant envs on an Apple GPU
    for res in [int(x) for x in args.render.split(",")]:
        cfg = R.RenderConfig(res, res, [R.ViewSource.look_at([1.5, -1.5, 1.2], [0.0, 0.0, 0.3], 45.0)], 0.01, 20.0)
        r = R.CudaRenderer(sc, cfg)
        # poses straight from the physics into the renderer's input buffers
        gd = torch.empty(n * len(sc.geoms) * 12, dtype=torch.float32, device=dev)
        cd = torch.empty(max(n * len(sc.cameras) * 12, 1), dtype=torch.float32, device=dev)
        phys.poses_device(range(n), gd.data_ptr(), cd.data_ptr() if sc.cameras else 0)
        phys.synchronize()
        ad = torch.from_numpy(np.tile(r.base_appearance, (n, 1)).reshape(-1)).to(dev)
        px = n * res * res
        rgba = torch.empty(px * 4, dtype=torch.uint8, device=dev)
        depth = torch.empty(px, dtype=torch.float32, device=dev)
        seg = torch.empty(px, dtype=torch.int32, device=dev)
        stream = torch.cuda.ExternalStream(r.stream(), device=dev)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

        def frame():
            r.render_device(n, gd.data_ptr(), cd.data_ptr(), ad.data_ptr(), rgba.data_ptr(), depth.data_ptr(),
                            seg.data_ptr())

        for _ in range(W):
            frame()
        r.synchronize()
        clocks = ClockSampler(0)
        clocks.start()
        total = 0.0
        for k in range(K):
            flush.fill_(float(k))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            frame()
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
        ms = total / K
        clock_info = clocks.stop()
        # end to end through the host API: poses in from host memory, images back to host memory
        for _ in range(2):
            r.render(0, n, g, c)
        t0 = time.perf_counter()
        for _ in range(max(K // 4, 3)):
            r.render(0, n, g, c)
        e2e_ms = (time.perf_counter() - t0) * 1e3 / max(K // 4, 3)
        # a physics step, its poses into the renderer's buffers and a frame,
        # all on the device (the renderer's stream waits on the physics one)
        def chain():
            phys.step_device(range(n), 1, ctrl.data_ptr())
            phys.poses_device(range(n), gd.data_ptr(), cd.data_ptr() if sc.cameras else 0)
            ev = torch.cuda.Event()
            ev.record(pstream)
            stream.wait_event(ev)
            frame()

        for _ in range(W):
            chain()
        torch.cuda.synchronize()
        chain_ms = 0.0
        for k in range(K):
            flush.fill_(float(k))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(pstream)
            chain()
            e1.record(stream)
            e1.synchronize()
            chain_ms += e0.elapsed_time(e1)
        chain_ms /= K
        out_bytes = px * 12
        line = {"metric": f"Ant frames/s at {res}x{res} (RGBA8 + depth + segmentation)", "value": n / (ms * 1e-3),
                "unit": "frames/s", "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"ant: {n} envs after 50 steps from qpos0+U[-0.1,0.1], one fixed view "
                                       f"look_at((1.5,-1.5,1.2),(0,0,0.3)) fovy 45, near 0.01 far 20, {res}x{res}",
                           "triangles": int(len(r.triangles)), "vertices": int(len(r.vertices)),
                           "l2": "flushed between timed frames (256 MB write)"},
                "reference_published": {"value": published.get(res), "unit": "frames/s",
                                        "note": "Metal renderer, 4096 Ant envs, Apple GPU (README.md:115-116)"},
                "e2e": {"value": n / (e2e_ms * 1e-3), "unit": "frames/s", "h2d_bytes_per_step": int(g.nbytes + c.nbytes),
                        "d2h_bytes_per_step": int(out_bytes)},
                "physics_step_then_frame": {"value": n / (chain_ms * 1e-3), "unit": "env-steps/s with a frame each",
                                            "ms": chain_ms, "note": "pg_step_device, pg_poses_device into the "
                                            "renderer's buffers, pg_render_frames_device; no host round trip"},
                "gpu_launches": K, "clocks": clock_info,
                "roofline": {"bound": "hbm", "kernel": "render_kernel", "achieved": out_bytes / (ms * 1e-3) / 1e9,
                             "peak": hbm_peak(), "unit": "GB/s", "frac": out_bytes / (ms * 1e-3) / 1e9 / hbm_peak(),
                             "traffic": NCU_RENDER_TRAFFIC_PER_IMAGE.get(res, 0.0) * n or None,
                             "note": "algorithmic bytes = the images written (12 B a pixel); the poses read are "
                                     "48 B a geom; traffic = ncu DRAM bytes per image of one frame's capture x "
                                     "images"}}
        print(json.dumps(line), flush=True)
        r.close()
    phys.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.learned_eval:
        run_learned_eval(args)
    elif args.scene:
        run_scene(args)
    elif args.render:
        run_render(args)
    elif args.aux:
        run_aux(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
