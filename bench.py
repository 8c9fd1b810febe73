#!/usr/bin/env python
"""Benchmark: particle-steps/s of the MPM snow step on B200.

Workload (default): the two-ball collision -- 1,048,576 particles in two
spheres, 128^3 grid, cubic B-spline APIC, dt 5e-5 (seeded synthetic input).
A "step" is one simulateOneStep of the whole scene.  `--workload batch64`
times the 64-scene batch (8.56M particles, quadratic, half APIC / half
PIC-FLIP) as one batched step; `snow_cube` (65,536 particles, 64^3) and
`large_slab` (8,388,608 particles, 256^3) are the other single scenes.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mpm_b200|reference]

N > 1 runs one process per GPU (torchrun); every rank advances its own
replica of the scene (batch64: its share of the 64 scenes; scene-parallel,
no data-path collective), and the value is the whole-job particle-steps/s
over the max-over-ranks device time.  `--impl reference` times the
reference's step math restated on the host CPU (oracle/, FP32, OpenMP on
every host core) on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import dataclasses
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
WORKLOADS = ("two_balls", "snow_cube", "large_slab", "batch64")
NAIVE_KIND = ("reference-naive CUDA restatement on the same B200 (AoS 236 B APIC / 128 B FLIP points, 52 B nodes, "
              "7 float atomics per particle-node, per-node FP64-literal splines, 2 SVDs per particle, "
              "synchronised launch per sub-step)")


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
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--serve-scale", type=float, default=1.0)
    ap.add_argument("--cpu-budget-s", type=float, default=20.0)
    ap.add_argument("--no-naive", action="store_true", help="skip the reference-naive GPU baseline leg")
    ap.add_argument("--naive-budget-s", type=float, default=10.0)
    ap.add_argument("--batch-scenes", type=int, default=64,
                    help="batch64: use only the first K scenes (small cases for profiling)")
    return ap.parse_args()


# --- workloads --------------------------------------------------------------
class Work:
    """The scenes one rank advances: a single scene (one solver) or a share of
    the 64-scene batch (one Batch)."""

    def __init__(self, name, rank=0, ws=1, batch_scenes=64):
        from mpm_b200 import scenes
        from mpm_b200.sharding import scenes_for_rank
        self.name = name
        self.batched = name == "batch64"
        if self.batched:
            self.scenes = scenes_for_rank(scenes.batched_scenes()[:batch_scenes], rank, ws)
        else:
            self.scenes = [{"two_balls": scenes.two_balls, "snow_cube": scenes.snow_cube,
                            "large_slab": scenes.large_slab}[name]()]
        self.n = sum(s.n for s in self.scenes)
        self.nscenes = min(batch_scenes, 64) if self.batched else 1

    def engine(self, device=None, scenes=None):
        scenes = scenes if scenes is not None else self.scenes
        if not self.batched:
            return scenes[0].solver(device=device)
        from mpm_b200.batch import Batch
        b = Batch(device=device)
        b.scene_ids = [b.add(s) for s in scenes]
        return b

    def config(self, ws):
        from mpm_b200 import _abi
        if not self.batched:
            sc = self.scenes[0]
            return {"workload": sc.name, "particles_per_gpu": sc.n, "grid": list(sc.resolution),
                    "transfer": "APIC" if sc.transfer == _abi.TRANSFER_APIC else "PIC-FLIP",
                    "interpolation": ["linear", "quadratic", "cubic"][sc.interpolation], "dt": sc.dt,
                    "parallelism": f"scene-replicas x{ws}",
                    "l2": "inputs larger than L2 (particle state %.0f MB)" % (sc.n * 41 * 4 * 2 / 1e6)}
        return {"workload": "batch64: %d of the 64 seeded scenes (N log-uniform 10k-500k, grids 32-128^3, "
                            "quadratic, half APIC / half PIC-FLIP, dt 1e-4) in one batched step" % self.nscenes,
                "scenes_on_rank0": len(self.scenes), "particles_on_rank0": self.n,
                "parallelism": f"scenes split over {ws} GPU(s)",
                "l2": "inputs larger than L2 (particle state %.0f MB)" % (self.n * 41 * 4 * 2 / 1e6)}


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
    """SM clock, power and clock-event (throttle) reasons of one GPU, sampled
    through NVML every ~2 ms by a thread while the timed region runs, plus one
    sample on entry and one on exit (so even a region of a few milliseconds is
    covered).  Falls back to `nvidia-smi -lms` when NVML is unavailable."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, index=0):
        self.index = index
        self.samples = []  # (sm_mhz, max_mhz, reasons bitmask)
        self.rows = []     # nvidia-smi fallback rows
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        # CUDA device indices count only the visible GPUs: find the GPU by the
        # UUID CUDA reports for it, else by CUDA_VISIBLE_DEVICES, else by index
        h = None
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid).encode())
        except Exception:
            h = None
        if h is None:
            ids = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
            idx = int(ids[self.index]) if len(ids) > self.index and ids[self.index].isdigit() else self.index
            h = pynvml.nvmlDeviceGetHandleByIndex(idx)
        self.bits = [(name, getattr(pynvml, const)) for name, const in self.REASONS]
        return pynvml, h

    def _sample(self):
        nv, h = self.nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        try:
            rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        except AttributeError:
            rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        self.samples.append((float(sm), float(mx), int(rs)))

    def _poll(self):
        while not self.stop.is_set():
            try:
                self._sample()
            except Exception:
                return
            self.stop.wait(0.002)

    def __enter__(self):
        try:
            self.nvml = self._nvml_handle()
            self._sample()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
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
        if self.nvml:
            self.stop.set()
            self.t.join(timeout=5)
            try:
                self._sample()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=5)

    def summary(self):
        if self.samples:
            sm = [a for a, _, _ in self.samples]
            reasons = sorted({name for _, _, r in self.samples for name, bit in self.bits if r & bit})
            return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(b for _, b, _ in self.samples),
                    "reasons": reasons, "samples": len(self.samples), "source": "nvml"}
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows), "source": "nvidia-smi"}


# --- roofline ---------------------------------------------------------------
# Algorithmic bytes per particle-step and per active grid node, (APIC, PIC-FLIP):
# the SoA FP32 state read once and written once.
PARTICLE_BYTES = {
    "p2g": (140, 104),            # x v Fe Fp m V0 (+B) in
    "g2p": (132 + 132, 96 + 96),  # state in (no m, V0), state out
    "grid": (0, 0),
}
NODE_BYTES = {
    "p2g": (16, 28),              # m, p + dt f (or p, f) out
    "g2p": (12, 24),              # v* (and v) gathered
    "grid": (16 + 12, 28 + 24),   # tile sums in, v* (v) out
}


def algorithmic_bytes(scenes, family, stats):
    """Algorithmic bytes of one launch family.  Active nodes are counted over
    all scenes; their per-node bytes are weighted by the APIC / PIC-FLIP
    particle split."""
    from mpm_b200 import _abi
    if family not in PARTICLE_BYTES:
        return 0
    n_apic = sum(s.n for s in scenes if s.transfer == _abi.TRANSFER_APIC)
    n_flip = sum(s.n for s in scenes) - n_apic
    pa, pf = PARTICLE_BYTES[family]
    na, nf = NODE_BYTES[family]
    frac = n_apic / max(n_apic + n_flip, 1)
    return n_apic * pa + n_flip * pf + stats["active_nodes"] * (frac * na + (1 - frac) * nf)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of a
# kernel family, from ncu captures of this bench run separately (ncu --set full
# --clock-control none -k regex:<kernel> -c 1 on `bench.py --steps 10 --warmup 3
# --no-e2e --no-cpu-baseline --no-naive --no-forms`, per workload); ncu cannot
# run inside the timed run, so these are not measured in the run they are
# printed with.
TRAFFIC_SOURCE = ("ncu capture of one launch of the kernel in a separate run of this bench on the same workload "
                  "(dram__bytes_read.sum + dram__bytes_write.sum)")
NCU_TRAFFIC = {
    "two_balls": {"p2g": 104.8e6, "g2p": 240.4e6, "grid": 4.45e6},
}


def traffic_of(family, workload):
    return NCU_TRAFFIC.get(workload, {}).get(family)


# FP32 pipe use of one launch of each kernel family (sm__pipe_fma_cycles_active,
# fraction of the peak sustained while active) from the same ncu captures: the
# cubic configurations are FP32-issue bound rather than HBM bound, so this
# fraction is reported beside the HBM one.
FP32_SOURCE = ("ncu capture of one launch of the kernel in a separate run of this bench on the same workload "
               "(sm__pipe_fma_cycles_active.avg.pct_of_peak_sustained_active / 100)")
NCU_FP32 = {
    "two_balls": {"p2g": 0.401, "g2p": 0.447, "grid": 0.048},
}


def fp32_of(family, workload):
    return NCU_FP32.get(workload, {}).get(family)


# --- CPU and naive-GPU baselines --------------------------------------------------
def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_rate(work, budget_s, steps_hint=None, threads=None):
    """Reference step math (oracle, FP32 restatement) on the host cores: full
    steps of the workload's scenes, as many as fit the time budget.
    Returns (rate, threads, sample description, steps, seconds)."""
    from oracle import oracle as O
    threads = threads or os.cpu_count() or 1
    if len(work.scenes) == 1:
        sc = work.scenes[0]
        o = O.OracleSolver(sc.desc(), sc.particles, bits=32, threads=threads)
        t0 = time.perf_counter()
        o.step(1)
        t1 = time.perf_counter() - t0
        k = max(1, min(int(budget_s / max(t1, 1e-9)), steps_hint or 10 ** 9))
        t0 = time.perf_counter()
        o.step(k)
        dt = time.perf_counter() - t0
        return sc.n * k / dt, threads, f"{k} full steps of the {sc.n}-particle scene", k, dt
    done, dt, used = 0, 0.0, 0
    for sc in work.scenes:  # one step of each scene in turn, within the budget
        o = O.OracleSolver(sc.desc(), sc.particles, bits=32, threads=threads)
        o.step(1)
        t0 = time.perf_counter()
        o.step(1)
        dt += time.perf_counter() - t0
        done += sc.n
        used += 1
        if dt > budget_s:
            break
    return done / dt, threads, f"1 step of each of the first {used} scenes ({done} particle-steps)", 1, dt


def cpu_single_thread(work, max_particles=65536):
    """The same FP32 step math on one host thread, over a bounded sample: one
    step (after one untimed step) of a seeded random subset of at most
    max_particles particles of the workload's first scene, on its full grid."""
    from oracle import oracle as O
    from mpm_b200.solver import Particles
    sc = work.scenes[0]
    p = sc.particles
    if sc.n > max_particles:
        idx = np.sort(np.random.default_rng(0).choice(sc.n, max_particles, replace=False))
        p = Particles(p.positions[idx], p.velocities[idx], p.mass[idx], p.materials,
                      None if p.material is None else p.material[idx], None if p.volume is None else p.volume[idx])
    o = O.OracleSolver(sc.desc(), p, bits=32, threads=1)
    o.step(1)
    t0 = time.perf_counter()
    o.step(1)
    dt = time.perf_counter() - t0
    return {"value": p.n / dt, "unit": METRIC, "cores": 1,
            "sample": f"1 step of a seeded random {p.n}-particle subset of {sc.name} (full grid), after 1 untimed step"}


def naive_rate(work, budget_s):
    """The reference-naive GPU restatement (baseline/naive) on the same scenes
    and GPU: AoS state, float atomics, per-node spline evaluation, one
    synchronised launch per sub-step, scenes stepped one after the other.
    Steps timed with CUDA events, as many as fit the budget (at least 3)."""
    sys.path.insert(0, os.path.join(ROOT, "baseline", "naive"))
    import naive as NV
    gs = [NV.NaiveSolver(s.desc(), s.particles) for s in work.scenes]
    for g in gs:
        g.step(2)
    t1 = sum(g.timed_step(1) for g in gs) / 1e3
    k = int(max(3, min(1000, budget_s / max(t1, 1e-6))))
    ms = 0.0
    for _ in range(k):
        ms += sum(g.timed_step(1) for g in gs)
    for g in gs:
        g.close()
    return {"value": work.n * k / (ms / 1e3), "unit": METRIC, "ms_per_step": ms / k, "steps": k, "kind": NAIVE_KIND}


def run_reference(args, ws, rank):
    if rank != 0:
        return
    work = Work(args.workload, batch_scenes=args.batch_scenes)
    # budget: the whole --steps/--warmup run finishes within a few minutes
    value, threads, sample, k, dt = cpu_rate(work, budget_s=min(150.0, 1.5 * (args.steps + args.warmup)),
                                             steps_hint=args.steps)
    out = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus, "steps": k,
           "warmup": 1, "ms_per_step": dt / k * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "impl": "reference",
           "config": work.config(1),
           "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
                            "sample": sample + " after 1 untimed step", "cpu_model": cpu_model(),
                            "nproc": os.cpu_count()},
           "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# --- our arm -------------------------------------------------------------------
def run_ours(args, ws, rank, local):
    from mpm_b200 import _abi
    lib = _abi.load()
    _abi.check(lib.mpm_set_device(local), "mpm_set_device")
    work = Work(args.workload, rank, ws, args.batch_scenes)
    g = work.engine()
    # launch settings from the autotuner (its steps are real steps, before warm-up)
    tuning = g.autotune(steps_per_candidate=3)
    g.step(args.warmup)
    g.synchronize()
    launches0 = C.c_uint64()
    launches1 = C.c_uint64()
    barrier(ws)
    g.kernel_spans()  # restart the device-side kernel spans
    with ClockSampler(index=local) as clk:
        lib.mpm_kernel_launches(C.byref(launches0))
        ms = g.timed_step(args.steps)
        lib.mpm_kernel_launches(C.byref(launches1))
    barrier(ws)
    # P2G / grid / G2P time per step measured on the device inside the timed,
    # graph-replayed steps (first CTA start to last CTA end of each launch)
    spans = g.kernel_spans()
    # Per-kernel times: the same steps again with CUDA events around every
    # kernel family on the library's stream (this mode launches the kernels
    # of a batch's stencil/transfer combinations one after another and
    # without graph replay, so it is not the timed configuration).
    prof_steps = min(args.steps, 200)
    g.profile(True)
    g.timed_step(prof_steps)
    prof = g.profile_read()
    g.profile(False)
    stats = g.stats()
    g.close()
    t_max = allmax(ws, ms) / 1e3
    total = allsum(ws, float(work.n * args.steps))
    value = total / t_max

    # the roofline kernel: the longest family among those that move the
    # state (the sort and compaction are overhead without algorithmic bytes),
    # timed inside the timed steps themselves
    dom = max(spans, key=lambda k: spans[k][0])
    dur = spans[dom][0] * 1e-3
    byt = algorithmic_bytes(work.scenes, dom, stats)
    peak, peak_kind = peaks()
    achieved = byt / dur / 1e9 if dur > 0 and byt > 0 else None
    roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
            "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
            "traffic": traffic_of(dom, work.name), "traffic_source": TRAFFIC_SOURCE,
            "fp32_pipe_frac": fp32_of(dom, work.name), "fp32_source": FP32_SOURCE,
            "algorithmic_bytes": byt, "avg_launch_ms": spans[dom][0],
            "kernel_ms_in_step": {k: v[0] for k, v in spans.items()}, "span_steps": spans[dom][1],
            "kernel_timing": "device-measured span of every launch (first CTA start to last CTA end, %globaltimer) "
                             "inside the timed graph-replayed steps",
            "kernel_ms": {k: v[0] for k, v in prof.items()},
            "kernel_ms_timing": "CUDA events around each kernel family over %d further non-graph steps "
                                "(sequential launches; includes the sort and compaction)" % prof_steps}

    e2e = None
    if not args.no_e2e:
        # one untimed pass of the same leg first: the process's first DMA
        # through freshly pinned pages and its first downloads (memory-pool
        # growth) are start-up costs of the process, as the warm-up steps'
        # are of the device leg
        run_e2e(work, min(args.steps, 3), ws, tuning)
        e2e = run_e2e(work, args.steps, ws, tuning)
        e2e["timed"] += "; after one untimed 3-step pass of the same leg (process warm-up)"

    naive = None
    if rank == 0 and ws == 1 and not args.no_naive:
        naive = naive_rate(work, args.naive_budget_s)
        naive["speedup"] = value / naive["value"]

    forms = None
    if not args.no_forms and not work.batched:
        forms = run_forms(args, ws, local)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, threads, sample, k, dt = cpu_rate(work, args.cpu_budget_s)
        cpu = {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
               "sample": sample + " (oracle FP32, OpenMP)", "cpu_model": cpu_model(), "nproc": os.cpu_count(),
               "single_thread": cpu_single_thread(work)}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
               "config": work.config(ws), "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
               "gpu_launches": int(launches1.value - launches0.value), "clocks": clk.summary(), "tuning": tuning,
               "stats": stats, "naive_gpu": naive, "forms": forms}
        print(json.dumps(out), flush=True)


def run_forms(args, ws, local):
    """Batched vs plain on the 64-scene workload, and a served stream.

    batched: the 64 seeded scenes (10k-500k particles, 32^3-128^3 grids,
             half APIC / half PIC-FLIP, quadratic, dt 1e-4) in one Batch;
    plain:   the same 64 scenes as 64 separate solvers stepped round-robin
             (each on its own stream), i.e. the reference's API used per scene;
    served:  a Poisson stream of scene requests (rate 20/s) replayed for
             --serve-seconds with particle counts scaled by --serve-scale."""
    from mpm_b200 import scenes
    from mpm_b200.serving import Server
    out = {}
    steps = min(args.steps, 100)
    rank = int(os.environ.get("RANK", "0"))
    work = Work("batch64", rank, ws)  # with several GPUs the 64 scenes are split across ranks
    with work.engine(device=local) as b:
        tuning = b.autotune(steps_per_candidate=3)
        b.step(3)
        b.synchronize()
        barrier(ws)
        b.kernel_spans()
        ms = b.timed_step(steps)
        spans = b.kernel_spans()
        b.profile(True)
        b.timed_step(steps)
        prof = b.profile_read()
        b.profile(False)
        st = b.stats()
    t = allmax(ws, ms) / 1e3
    out["batched"] = {"workload": "64 seeded scenes split over %d GPU(s); %d particles on rank %d" % (ws, work.n, rank),
                      "steps": steps,
                      "value": allsum(ws, float(work.n * steps)) / t, "ms_per_step": t / steps * 1e3,
                      "kernel_ms_in_step": {k: v[0] for k, v in spans.items()},
                      "kernel_ms": {k: v[0] for k, v in prof.items()}, "stats": st, "tuning": tuning}
    solvers = [s.solver(device=local) for s in work.scenes]
    # warm-up as for the batch: the autotuner (cached keys: one step), the
    # first step decides a default P2G staging size (read back at the
    # synchronize), the next steps capture the step graphs
    for g in solvers:
        g.autotune(steps_per_candidate=3)
        g.step(1)
    for g in solvers:
        g.synchronize()
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
                    "value": allsum(ws, float(work.n * steps)) / t, "ms_per_step": t / steps * 1e3}
    out["batched_over_plain"] = out["batched"]["value"] / out["plain"]["value"]
    reqs = scenes.serving_requests(rate=20.0, duration=args.serve_seconds, scale=args.serve_scale, lazy=True)
    srv = Server(budget_bytes=150e9, device=local, keep_state=False)
    rep = srv.run(reqs, time_scale=1.0)
    srv.close()
    s = rep.summary()
    s["stream"] = ("Poisson 20 req/s for %.0f s, particles log-uniform in [%d, %d], 100-500 steps each, "
                   "grid = bounding box + 4 cells (<= 128^3), 150 GB admission budget; scenes built from their "
                   "seeds by a helper thread up to 2 s before arrival" % (
                       args.serve_seconds, max(1, int(5000 * args.serve_scale)), int(2_000_000 * args.serve_scale)))
    out["served"] = s
    return out


def run_e2e(work, steps, ws, tuning=None):
    """Same metric through the public API with host buffers: construct the
    solver (or batch) from pinned host arrays (H2D), then every step download
    every scene's (x, y, z, 1) positions into pinned host memory (D2H,
    asynchronous, into two alternating buffers per scene, so the copy of step
    k overlaps step k + 1); the clock stops after the last copy has landed."""
    import torch
    from mpm_b200 import _abi
    from mpm_b200.solver import Particles
    pin = lambda a: torch.from_numpy(np.array(a, copy=True)).pin_memory().numpy()
    pinned = []
    for sc in work.scenes:
        p = sc.particles
        pp = Particles(pin(p.positions), pin(p.velocities), pin(p.mass), p.materials,
                       None if p.material is None else pin(p.material), None if p.volume is None else pin(p.volume))
        pinned.append(dataclasses.replace(sc, particles=pp))
    outs = [[torch.empty((sc.n, 4), dtype=torch.float32).pin_memory() for _ in range(2)] for sc in work.scenes]
    barrier(ws)
    t0 = time.perf_counter()
    g = work.engine(scenes=pinned)
    if tuning and not work.batched:  # the settings the autotuner chose for this scene
        g.set_tuning(tuning["g2p_chunk"], tuning["p2g_stage"], tuning["p2g_warp_max"])
    elif tuning:
        for c in tuning["combinations"]:
            g.set_tuning(c["g2p_chunk"], c["p2g_stage"], c["interpolation"], c["transfer"], c["p2g_warp_max"])
    for k in range(steps):
        g.step(1)
        if work.batched:
            for j, sid in enumerate(g.scene_ids):
                g.download_async(sid, _abi.FIELD_POSITION4, outs[j][k % 2].data_ptr())
        else:
            g.download_async(_abi.FIELD_POSITION4, outs[0][k % 2].data_ptr())
    g.download_wait()
    dt = time.perf_counter() - t0
    g.close()
    barrier(ws)
    t = allmax(ws, dt)
    h2d = sum(sc.n * (7 + (1 if sc.particles.volume is not None else 0)) * 4 +
              (2 * sc.n if sc.particles.material is not None else 0) for sc in work.scenes)
    return {"value": allsum(ws, float(work.n * steps)) / t, "unit": METRIC, "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": 16 * work.n, "timed": "construction from pinned host arrays (H2D of the "
            "particles) + per step: step + asynchronous download of every scene's float4 positions into pinned "
            "host memory, until the last copy has landed"}


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
