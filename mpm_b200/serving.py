"""Serving loop: continuous batching of scene-simulation requests.

Requests (a scene plus a number of steps) arrive over time.  The server keeps
every admitted scene's particle and grid state resident on the device in one
Batch and advances all of them by one step per iteration; between
iterations it retires finished requests (downloading their final state) and
admits newly arrived ones while their device memory fits the budget.  So
requests that arrive while others are running join the next step: their work
overlaps on the device with everyone else's.  Each result is bitwise the
result of solving the scene alone (per-scene reductions run in a fixed,
scene-local order).

Reported: per-step latency (p50/p99 of the batched step), time to completion
(arrival to result), queueing delay, and aggregate particle-steps/s.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

import numpy as np

from . import _abi
from .batch import Batch

FIELDS_OUT = (_abi.FIELD_POSITION, _abi.FIELD_VELOCITY, _abi.FIELD_DET_FE, _abi.FIELD_DET_FP)


def scene_device_bytes(scene) -> int:
    """Device memory a scene holds while admitted: two particle buffers (41
    float planes, id, material), the dense grid (v*, and v for PIC-FLIP), its
    share of the batch's sort buffers and block tables, and P2G tiles for its
    blocks (bounded by its particle count)."""
    n = scene.n
    res = scene.resolution
    nodes = int(res[0]) * int(res[1]) * int(res[2])
    nb = [((int(r) + 3) >> 2) + 1 for r in res]
    blocks = nb[0] * nb[1] * nb[2] + 1
    flip = scene.transfer == _abi.TRANSFER_PIC_FLIP
    particles = 2 * n * (41 * 4 + 4 + 2)
    grid = nodes * 16 * (2 if flip else 1)
    sort = n * (16 + 24) + (n + 2047) // 2048 * 256 * 4 * 2  # radix + incremental sort scratch
    tables = blocks * (4 + 8 + 8 + 4)
    S = {0: 2, 1: 3, 2: 4}[scene.interpolation]
    tiles = min(blocks, max(n, 1)) * 7 * (S + 3) ** 3 * 4
    return particles + grid + sort + tables + tiles


@dataclass
class RequestResult:
    rid: int
    n: int
    steps: int
    arrival: float
    admitted: float
    finished: float
    state: Dict[int, np.ndarray] = field(default_factory=dict)

    @property
    def time_to_completion(self) -> float:
        return self.finished - self.arrival

    @property
    def queue_delay(self) -> float:
        return self.admitted - self.arrival


@dataclass
class ServeReport:
    results: List[RequestResult]
    step_latency_ms: List[float]
    batch_sizes: List[int]
    particle_steps: int
    wall_s: float
    rejected: List[int]

    def summary(self) -> dict:
        lat = np.asarray(self.step_latency_ms) if self.step_latency_ms else np.zeros(1)
        ttc = np.asarray([r.time_to_completion for r in self.results]) if self.results else np.zeros(1)
        qd = np.asarray([r.queue_delay for r in self.results]) if self.results else np.zeros(1)
        return {"requests": len(self.results), "rejected": len(self.rejected), "steps": len(self.step_latency_ms),
                "p50_step_ms": float(np.percentile(lat, 50)), "p99_step_ms": float(np.percentile(lat, 99)),
                "mean_batch_scenes": float(np.mean(self.batch_sizes)) if self.batch_sizes else 0.0,
                "p50_ttc_s": float(np.percentile(ttc, 50)), "p99_ttc_s": float(np.percentile(ttc, 99)),
                "p50_queue_s": float(np.percentile(qd, 50)), "p99_queue_s": float(np.percentile(qd, 99)),
                "particle_steps": int(self.particle_steps), "wall_s": self.wall_s,
                "particle_steps_per_s": self.particle_steps / self.wall_s if self.wall_s > 0 else 0.0}


class Server:
    """Continuous-batching server over one Batch on one GPU."""

    def __init__(self, budget_bytes: float = 150e9, device: Optional[int] = None, keep_state: bool = True,
                 clock: Callable[[], float] = time.perf_counter):
        self.batch = Batch(device=device)
        self.budget = float(budget_bytes)
        self.keep_state = keep_state
        self.clock = clock

    def close(self):
        self.batch.close()

    def run(self, requests, time_scale: float = 1.0, max_wall_s: Optional[float] = None,
            prefetch_s: float = 2.0) -> ServeReport:
        """Replay `requests` (mpm_b200.scenes.Request, arrival-ordered).
        Arrival times are divided by `time_scale` (10 replays a 60 s stream in
        6 s).  Requests larger than the whole budget are rejected.

        The loop keeps the GPU fed: step k + 1 is queued before the host waits
        for step k (at most one step in flight behind the running one), and
        per-step latencies are the device times of the steps, read from events
        without synchronizing.  A request whose last step has been queued is
        retired once that step has completed: its final state is downloaded
        (keep_state) and its memory returns to the pool in stream order.  Scene
        uploads do not wait for the GPU; a change of the scene set costs one
        rebuild of the scene table at the next step.  Lazy requests
        (scenes.serving_requests(lazy=True)) are built by a helper thread up to
        prefetch_s ahead of their arrival, as a client's upload would arrive,
        and their host copy is dropped once uploaded."""
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        live: Dict[int, dict] = {}  # scene id -> request bookkeeping
        done_queue: List[int] = []   # scene ids whose last step is queued
        used = 0.0
        results, lat, sizes, rejected = [], [], [], []
        psteps = 0
        self.batch.time_steps(True)
        t0 = self.clock()
        qi = 0
        waiting: List = []
        stop = threading.Event()

        def prefetch():
            for req in pending:
                while not stop.is_set() and req.arrival / time_scale > self.clock() - t0 + prefetch_s:
                    time.sleep(0.01)
                if stop.is_set():
                    return
                req.materialize()

        helper = threading.Thread(target=prefetch, daemon=True)
        helper.start()

        def retire(sid):
            nonlocal used
            rec = live.pop(sid)
            req = rec["req"]
            state = {f: self.batch.download(sid, f) for f in FIELDS_OUT} if self.keep_state else {}
            self.batch.remove(sid)
            used -= rec["need"]
            results.append(RequestResult(req.rid, rec["n"], rec["steps"], req.arrival / time_scale,
                                         rec["admitted"], self.clock() - t0, state))

        while qi < len(pending) or waiting or live:
            now = self.clock() - t0
            if max_wall_s is not None and now > max_wall_s:
                break
            while qi < len(pending) and pending[qi].arrival / time_scale <= now:
                waiting.append(pending[qi])
                qi += 1
            # retire the requests whose last step has been queued, once it has
            # completed (the scene set changes anyway: the next step rebuilds)
            if done_queue:
                self.batch.wait_steps(0)
                for sid in done_queue:
                    retire(sid)
                done_queue = []
            # admission: first fit in arrival order against the memory budget
            still = []
            for req in waiting:
                need = scene_device_bytes(req.scene)
                if need > self.budget:
                    rejected.append(req.rid)
                    continue
                if used + need <= self.budget:
                    sc = req.scene
                    sid = self.batch.add(sc)
                    live[sid] = dict(req=req, left=sc.steps, need=need, admitted=self.clock() - t0, n=sc.n,
                                     steps=sc.steps)
                    used += need
                    if req._factory is not None:
                        req.release()  # uploaded: the host copy is no longer needed
                else:
                    still.append(req)
            waiting = still
            stepping = [sid for sid in live if live[sid]["left"] > 0]
            if not stepping:
                if qi < len(pending):  # idle until the next arrival
                    delay = pending[qi].arrival / time_scale - (self.clock() - t0)
                    if delay > 0:
                        time.sleep(min(delay, 0.05))
                continue
            # one batched step of every in-flight scene, queued behind the running one
            self.batch.step(1)
            sizes.append(len(stepping))
            psteps += sum(live[sid]["n"] for sid in stepping)
            for sid in stepping:
                live[sid]["left"] -= 1
                if live[sid]["left"] == 0:
                    done_queue.append(sid)
            self.batch.wait_steps(1)
            lat.extend(self.batch.step_times())
        stop.set()
        helper.join()
        self.batch.synchronize()
        for sid in done_queue:
            retire(sid)
        lat.extend(self.batch.step_times())
        self.batch.time_steps(False)
        wall = self.clock() - t0
        return ServeReport(results, lat, sizes, psteps, wall, rejected)


def main():
    import argparse
    import json

    from . import scenes
    ap = argparse.ArgumentParser(description="Replay a seeded Poisson stream of snow-scene requests.")
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--duration", type=float, default=60.0)
    ap.add_argument("--scale", type=float, default=1.0, help="particle-count scale of every request")
    ap.add_argument("--time-scale", type=float, default=1.0)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--max-requests", type=int, default=None)
    a = ap.parse_args()
    reqs = scenes.serving_requests(rate=a.rate, duration=a.duration, scale=a.scale, max_requests=a.max_requests)
    srv = Server(budget_bytes=a.budget_gb * 1e9, keep_state=False)
    rep = srv.run(reqs, time_scale=a.time_scale)
    print(json.dumps(rep.summary()))


if __name__ == "__main__":
    main()
