#!/usr/bin/env python
"""Benchmark: particle-steps/s of the MPM snow step on B200.

Workload (default): the two-ball collision -- 1,048,576 particles in two
spheres, 128^3 grid, cubic B-spline APIC, dt 5e-5 (seeded synthetic input).
A "step" is one simulateOneStep of the whole scene.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mpm_b200|reference]

N > 1 runs one process per GPU (torchrun); every rank advances its own
replica of the scene (scene-parallel, no data-path collective), and the value
is the whole-job particle-steps/s over the max-over-ranks device time.
`--impl reference` times the reference's step math restated on the host CPU
(oracle/, FP32, OpenMP on every host core) on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s"
WORKLOADS = ("two_balls", "snow_cube", "large_slab")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="mpm_b200", choices=["mpm_b200", "reference"])
    ap.add_argument("--workload", default="two_balls", choices=WORKLOADS)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched and served legs")
    ap.add_argument("--serve-seconds", type=float, default=10.0)
    ap.add_argument("--serve-scale", type=float, default=0.02)
    ap.add_argument("--cpu-budget-s", type=float, default=20.0)
    ap.add_argument("--no-naive", action="store_true", help="skip the reference-naive GPU baseline leg")
    ap.add_argument("--naive-budget-s", type=float, default=10.0)
    return ap.parse_args()


def make_scene(name):
    from mpm_b200 import scenes
    return {"two_balls": scenes.two_balls, "snow_cube": scenes.snow_cube, "large_slab": scenes.large_slab}[name]()


def config_of(sc, n_gpus):
    from mpm_b200 import _abi
    return {"workload": sc.name, "particles_per_gpu": sc.n, "grid": list(sc.resolution),
            "transfer": "APIC" if sc.transfer == _abi.TRANSFER_APIC else "PIC-FLIP",
            "interpolation": ["linear", "quadratic", "cubic"][sc.interpolation], "dt": sc.dt,
            "parallelism": f"scene-replicas x{n_gpus}",
            "l2": "inputs larger than L2 (particle state %.0f MB)" % (sc.n * 41 * 4 * 2 / 1e6)}


# --- distributed plumbing ---------------------------------------------------
def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(ws, x):
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allsum(ws, x):
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# --- clocks -----------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# --- roofline ---------------------------------------------------------------
def algorithmic_bytes(sc, family, stats):
    """Algorithmic bytes of one launch: per particle-step SoA FP32 state read
    once and written once, plus per active grid node (m and momentum/force
    into the grid, v* out of it)."""
    from mpm_b200 import _abi
    apic = sc.transfer == _abi.TRANSFER_APIC
    n, nodes = sc.n, stats["active_nodes"]
    if family == "p2g":  # x v Fe Fp m V0 (+B) in; m, p(+dt f) (or p, f) out
        return n * (140 if apic else 104) + nodes * (16 if apic else 28)
    if family == "g2p":  # state in (no m, V0), state out, v* (v) gathered
        return n * ((132 + 132) if apic else (96 + 96)) + nodes * (12 if apic else 24)
    if family == "grid":  # tile sums in, v* (v) out
        return nodes * ((16 + 12) if apic else (28 + 24))
    return 0


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_of(family, workload):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get(workload, {}).get(family)


# --- CPU baseline -------------------------------------------------------------
def cpu_rate(sc, budget_s, steps_hint=None):
    """Reference step math (oracle, FP32 restatement) on all host cores: full
    steps of the same scene, as many as fit the time budget (at least one)."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    o = O.OracleSolver(sc.desc(), sc.particles, bits=32, threads=threads)
    t0 = time.perf_counter()
    o.step(1)
    t1 = time.perf_counter() - t0
    k = max(1, min(int(budget_s / max(t1, 1e-9)), steps_hint or 10 ** 9))
    t0 = time.perf_counter()
    o.step(k)
    dt = time.perf_counter() - t0
    return sc.n * k / dt, threads, k, dt


def naive_rate(sc, budget_s):
    """The reference-naive GPU restatement (baseline/naive) on the same scene
    and GPU: AoS state, float atomics, per-node spline evaluation, one
    synchronised launch per sub-step.  Steps timed with CUDA events on the
    legacy stream, as many as fit the budget (at least 3)."""
    sys.path.insert(0, os.path.join(ROOT, "baseline", "naive"))
    import naive as NV
    g = NV.NaiveSolver(sc.desc(), sc.particles)
    g.step(2)
    t1 = g.timed_step(2) / 2e3
    k = int(max(3, min(1000, budget_s / max(t1, 1e-6))))
    ms = g.timed_step(k)
    g.close()
    return {"value": sc.n * k / (ms / 1e3), "unit": METRIC, "ms_per_step": ms / k, "steps": k,
            "kind": "reference-naive CUDA restatement on the same B200 (AoS 236 B APIC / 128 B FLIP points, "
                    "52 B nodes, 7 float atomics per particle-node, per-node FP64-literal splines, "
                    "2 SVDs per particle, synchronised launch per sub-step)"}


def run_reference(args, ws, rank):
    if rank != 0:
        return
    sc = make_scene(args.workload)
    # budget: the whole --steps/--warmup run finishes within a few minutes
    value, threads, k, dt = cpu_rate(sc, budget_s=min(150.0, 1.5 * (args.steps + args.warmup)), steps_hint=args.steps)
    out = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus, "steps": k,
           "warmup": 1, "ms_per_step": dt / k * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "impl": "reference",
           "config": config_of(sc, 1),
           "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
                            "sample": f"{k} full steps of the {sc.n}-particle scene after 1 untimed step"},
           "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# --- our arm -------------------------------------------------------------------
def run_ours(args, ws, rank, local):
    from mpm_b200 import _abi
    lib = _abi.load()
    _abi.check(lib.mpm_set_device(local), "mpm_set_device")
    sc = make_scene(args.workload)
    g = sc.solver()
    g.step(args.warmup)
    g.synchronize()
    launches0 = C.c_uint64()
    launches1 = C.c_uint64()
    g.profile(True)
    barrier(ws)
    with ClockSampler(index=local) as clk:
        lib.mpm_kernel_launches(C.byref(launches0))
        ms = g.timed_step(args.steps)
        lib.mpm_kernel_launches(C.byref(launches1))
    barrier(ws)
    prof = g.profile_read()
    g.profile(False)
    stats = g.stats()
    t_max = allmax(ws, ms) / 1e3
    total = allsum(ws, float(sc.n * args.steps))
    value = total / t_max

    fams = {k: v for k, v in prof.items() if k in ("p2g", "g2p", "grid", "sort")}
    dom = max(fams, key=lambda k: fams[k][0] * fams[k][1])
    dur = fams[dom][0] * 1e-3
    byt = algorithmic_bytes(sc, dom, stats)
    peak, peak_kind = peaks()
    achieved = byt / dur / 1e9 if dur > 0 and byt > 0 else None
    roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
            "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
            "traffic": traffic_of(dom, sc.name), "algorithmic_bytes": byt, "avg_launch_ms": fams[dom][0],
            "kernel_ms": {k: v[0] for k, v in prof.items()}}

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(sc, args.steps, ws)

    forms = None
    if not args.no_forms:
        forms = run_forms(args, ws, local)

    naive = None
    if rank == 0 and ws == 1 and not args.no_naive:
        naive = naive_rate(sc, args.naive_budget_s)
        naive["speedup"] = value / naive["value"]

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, threads, k, dt = cpu_rate(sc, args.cpu_budget_s)
        cpu = {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
               "sample": f"{k} full steps of the {sc.n}-particle scene (oracle FP32, OpenMP)"}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
               "config": config_of(sc, ws), "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
               "gpu_launches": int(launches1.value - launches0.value), "clocks": clk.summary(),
               "stats": stats, "naive_gpu": naive, "forms": forms}
        print(json.dumps(out), flush=True)
    g.close()


def run_forms(args, ws, local):
    """Batched vs plain on the 64-scene workload, and a served stream.

    batched: the 64 seeded scenes (10k-500k particles, 32^3-128^3 grids,
             half APIC / half PIC-FLIP, quadratic, dt 1e-4) in one Batch;
    plain:   the same 64 scenes as 64 separate solvers stepped round-robin
             (each on its own stream), i.e. the reference's API used per scene;
    served:  a Poisson stream of scene requests (rate 20/s) replayed for
             --serve-seconds with particle counts scaled by --serve-scale."""
    from mpm_b200 import scenes
    from mpm_b200.batch import Batch
    from mpm_b200.serving import Server
    from mpm_b200.sharding import scenes_for_rank
    out = {}
    steps = min(args.steps, 100)
    # with several GPUs the 64 scenes are split across ranks (scene-parallel)
    rank = int(os.environ.get("RANK", "0"))
    scs = scenes_for_rank(scenes.batched_scenes(), rank, ws)
    ntot = sum(s.n for s in scs)
    with Batch(device=local) as b:
        for s in scs:
            b.add(s)
        b.step(3)
        b.synchronize()
        b.profile(True)
        barrier(ws)
        ms = b.timed_step(steps)
        prof = b.profile_read()
        st = b.stats()
    t = allmax(ws, ms) / 1e3
    out["batched"] = {"workload": "64 seeded scenes split over %d GPU(s); %d particles on rank %d" % (ws, ntot, rank),
                      "steps": steps,
                      "value": allsum(ws, float(ntot * steps)) / t, "ms_per_step": t / steps * 1e3,
                      "kernel_ms": {k: v[0] for k, v in prof.items()}, "stats": st}
    solvers = [s.solver() for s in scs]
    for g in solvers:
        g.step(3)
    for g in solvers:
        g.synchronize()
    barrier(ws)
    t0 = time.perf_counter()
    for _ in range(steps):
        for g in solvers:
            g.step(1)
    for g in solvers:
        g.synchronize()
    t = allmax(ws, time.perf_counter() - t0)
    for g in solvers:
        g.close()
    out["plain"] = {"workload": "same 64 scenes as 64 solvers", "steps": steps,
                    "value": allsum(ws, float(ntot * steps)) / t, "ms_per_step": t / steps * 1e3}
    out["batched_over_plain"] = out["batched"]["value"] / out["plain"]["value"]
    reqs = scenes.serving_requests(rate=20.0, duration=args.serve_seconds, scale=args.serve_scale)
    srv = Server(budget_bytes=150e9, device=local, keep_state=False)
    rep = srv.run(reqs, time_scale=1.0)
    srv.close()
    s = rep.summary()
    s["stream"] = ("Poisson 20 req/s for %.0f s, particles log-uniform in [%d, %d], 100-500 steps each"
                   % (args.serve_seconds, max(1, int(5000 * args.serve_scale)), int(2_000_000 * args.serve_scale)))
    out["served"] = s
    return out


def run_e2e(sc, steps, ws):
    """Same metric through the public API with host buffers: construct the
    solver from pinned host arrays (H2D), then every step download the
    (x, y, z, 1) positions into pinned host memory (D2H, asynchronous, into
    two alternating buffers, so the copy of step k overlaps step k + 1); the
    clock stops after the last copy has landed."""
    import torch
    from mpm_b200 import _abi
    from mpm_b200.solver import APICMPMSolver3D, MPMSolver3D, Particles
    n = sc.n
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    p = Particles(pin(sc.particles.positions), pin(sc.particles.velocities), pin(sc.particles.mass),
                  sc.particles.materials, None, None)
    outs = [torch.empty((n, 4), dtype=torch.float32).pin_memory() for _ in range(2)]
    opts = dict(gravity=sc.gravity, boundary=sc.boundary, sticky_cells=sc.sticky_cells, volume_mode=sc.volume_mode)
    barrier(ws)
    t0 = time.perf_counter()
    if sc.transfer == _abi.TRANSFER_APIC:
        g = APICMPMSolver3D(p, sc.origin, sc.resolution, sc.stride, sc.friction, sc.interpolation, sc.dt, **opts)
    else:
        g = MPMSolver3D(p, sc.origin, sc.resolution, sc.stride, sc.friction, sc.blend, sc.interpolation, sc.dt,
                        **opts)
    for k in range(steps):
        g.step(1)
        # this step's positions into alternating pinned buffers; the copy
        # overlaps the next step (download_async)
        g.download_async(_abi.FIELD_POSITION4, outs[k % 2].data_ptr())
    g.download_wait()
    dt = time.perf_counter() - t0
    g.close()
    barrier(ws)
    t = allmax(ws, dt)
    h2d = n * (3 + 3 + 1) * 4
    return {"value": allsum(ws, float(n * steps)) / t, "unit": METRIC, "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": 16 * n, "timed": "solver construction (H2D of the particles) + per step: "
            "step + asynchronous download of float4 positions into pinned host memory, "
            "until the last copy has landed"}


def main():
    args = parse()
    ws, rank, local = dist_init()
    if args.impl == "reference":
        run_reference(args, ws, rank)
    else:
        run_ours(args, ws, rank, local)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
