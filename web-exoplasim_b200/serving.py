"""Serving: continuous batching of many planet runs on one GPU.

Requests (a seeded planet, a resolution and a duration in simulated days)
arrive over time. Each resolution (T, L) has one batched engine whose slot
count is sized from an HBM budget by the per-slot state footprint. A request
waits until a slot of its resolution is free, is admitted at the next batch
boundary (configured into the slot while the other slots keep their state on
the device), steps with everyone else in the same launches, and leaves when
its last step is done: the engine stops a slot exactly at its final step
(exogcm_set_stop), so a result does not depend on what else was running.
Engines of different resolutions step concurrently on their own streams.

Reported: time-to-result p50/p99, admission queue depth, and aggregate
simulated days per second over the window.
"""
from __future__ import annotations

import importlib
import math
import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

pkg = importlib.import_module("web-exoplasim_b200")
planets_mod = importlib.import_module("web-exoplasim_b200.planets")

# Model timestep per truncation: 45 minutes, and 30 at T63 where the
# reference documents 45-minute runs going unstable.
STEP_MINUTES = {21: 45.0, 42: 45.0, 63: 30.0}


@dataclass
class Request:
    id: int
    truncation: int
    levels: int
    days: float
    seed: int
    arrival: float = 0.0
    overrides: dict = field(default_factory=dict)
    planet: object = None  # a prebuilt planets.Planet (the client's input); else made from the seed
    # filled in by the server
    admitted: float | None = None
    finished: float | None = None
    steps: int = 0
    status: str = "queued"
    result: dict | None = None


def slot_bytes(truncation: int, levels: int) -> int:
    """Device bytes one slot of a (T, L) engine holds (state plus tables)."""
    e = pkg.Engine(truncation, levels, 1)
    try:
        names = [n for n in FIELD_NAMES]
        return sum(e.field_size(n) for n in names) * 4 + 64 * 1024
    finally:
        e.close()


FIELD_NAMES: list[str] = []


def _field_names():
    import os
    import re
    src = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "fields.h")
    return re.findall(r"X\((\w+),[SFGT],", open(src).read())


class Group:
    """One (T, L) engine and its slots."""

    def __init__(self, truncation, levels, slots, chunk):
        self.truncation, self.levels, self.slots, self.chunk = truncation, levels, slots, chunk
        self.engine = pkg.Engine(truncation, levels, slots, mode=1)
        self.free = deque(range(slots))
        self.running: dict[int, Request] = {}
        self.stop_step: dict[int, int] = {}
        self.sim_days = 0.0

    def admit(self, req: Request, now: float):
        slot = self.free.popleft()
        planet = req.planet
        if planet is None:
            planet = planets_mod.make_planet(req.seed, truncation=req.truncation, levels=req.levels,
                                             timestepMinutes=STEP_MINUTES[req.truncation], **req.overrides)
        self.engine.configure(slot, planet)
        steps_per_day = 1440.0 / STEP_MINUTES[req.truncation]
        req.steps = max(1, int(round(req.days * steps_per_day)))
        start = self.engine.slot_info(slot)["step"]
        self.stop_step[slot] = start + req.steps
        self.engine.set_stop(slot, start + req.steps)
        req.admitted = now
        req.status = "running"
        self.running[slot] = req

    def step(self):
        if self.running:
            self.engine.step(self.chunk, publish_every=1 << 30)

    def collect(self, now: float, done: list):
        unstable = self.engine.unstable() if self.running else None
        for slot, req in list(self.running.items()):
            info = self.engine.slot_info(slot)
            failed = unstable is not None and unstable[slot]
            if failed or (info["startup_left"] == 0 and info["step"] >= self.stop_step[slot]):
                req.finished = now
                req.status = "failed" if failed else "finished"
                if not failed:
                    self.sim_days += req.days
                    req.result = {name: self.engine.read(slot, name) for name in ("st", "sz", "sd", "sq", "sp")}
                self.engine.release(slot)
                del self.running[slot]
                self.free.append(slot)
                done.append(req)


class Server:
    """Continuous-batching loop over per-resolution engines."""

    def __init__(self, capacity: dict, chunk: int = 16, keep_results: bool = True):
        self.groups = {key: Group(key[0], key[1], n, chunk) for key, n in capacity.items() if n > 0}
        self.queue: deque[Request] = deque()
        self.done: list[Request] = []
        self.queue_depth: list[int] = []
        self.keep_results = keep_results

    @staticmethod
    def capacity_for(budget_bytes: float, mix: dict, max_slots: int = 256) -> dict:
        """Slots per (T, L) from an HBM budget split by the expected mix of
        work (fraction of requests per resolution times its per-slot bytes)."""
        global FIELD_NAMES
        if not FIELD_NAMES:
            FIELD_NAMES = _field_names()
        sizes = {key: slot_bytes(*key) for key in mix}
        weight = sum(mix[k] * sizes[k] for k in mix)
        return {k: int(min(max_slots, max(1, budget_bytes * mix[k] / weight))) for k in mix}

    def submit(self, req: Request):
        self.queue.append(req)

    def _admit(self, now: float):
        waiting = deque()
        while self.queue:
            req = self.queue.popleft()
            group = self.groups.get((req.truncation, req.levels))
            if group is None:
                req.status = "rejected"
                req.finished = now
                self.done.append(req)
                continue
            if req.arrival > now:
                waiting.append(req)
                continue
            if group.free:
                group.admit(req, now)
            else:
                waiting.append(req)
        self.queue = waiting

    def run(self, requests: list[Request], window: float, drain: bool = False, clock=time.perf_counter):
        """Serves `requests` (arrival times relative to the start) for
        `window` seconds of wall time, or until all finish with `drain`."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        t0 = clock()
        while True:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                self.queue.append(pending.popleft())
            self._admit(now)
            self.queue_depth.append(len(self.queue))
            active = [g for g in self.groups.values() if g.running]
            if not active:
                if not pending and not self.queue:
                    break
                if now > window and not drain:
                    break
                time.sleep(0.001)
                continue
            threads = [threading.Thread(target=g.step) for g in active]
            for t in threads:
                t.start()
            for t in threads:
                t.join()
            now = clock() - t0
            for g in active:
                g.collect(now, self.done)
            if not self.keep_results:
                for r in self.done:
                    r.result = None
            if now > window and not drain:
                break
        elapsed = clock() - t0
        return self.report(elapsed)

    def report(self, elapsed: float) -> dict:
        finished = [r for r in self.done if r.status == "finished"]
        latency = np.array([r.finished - r.arrival for r in finished]) if finished else np.array([np.nan])
        days = sum(r.days for r in finished)
        partial = 0.0
        for g in self.groups.values():
            for slot, req in g.running.items():
                info = g.engine.slot_info(slot)
                done_steps = req.steps - max(0, g.stop_step[slot] - info["step"])
                partial += done_steps * STEP_MINUTES[g.truncation] / 1440.0
        return {
            "completed": len(finished),
            "failed": sum(r.status == "failed" for r in self.done),
            "p50_s": float(np.nanpercentile(latency, 50)),
            "p99_s": float(np.nanpercentile(latency, 99)),
            "queue_depth_mean": float(np.mean(self.queue_depth)) if self.queue_depth else 0.0,
            "queue_depth_max": int(max(self.queue_depth)) if self.queue_depth else 0,
            "sim_days_per_s": (days + partial) / elapsed,
            "window_s": elapsed,
            "slots": {f"T{k[0]}L{k[1]}": g.slots for k, g in self.groups.items()},
        }


def poisson_requests(rate: float, window: float, seed: int, max_days: float = 365.0, min_days: float = 1.0,
                     resolutions=((21, 5), (21, 10), (42, 5), (42, 10), (63, 5), (63, 10))) -> list[Request]:
    """Poisson arrivals at `rate` per second over `window` seconds, each with a
    resolution drawn uniformly and a duration uniform in [min_days, max_days]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    i = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > window:
            break
        tr, lv = resolutions[rng.integers(len(resolutions))]
        out.append(Request(id=i, truncation=int(tr), levels=int(lv), days=float(rng.uniform(min_days, max_days)),
                           seed=int(rng.integers(1 << 30)), arrival=t))
        i += 1
    return out


if __name__ == "__main__":
    import argparse
    import json

    ap = argparse.ArgumentParser(description="Serve Poisson planet-run requests on one GPU")
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--window", type=float, default=600.0)
    ap.add_argument("--max-days", type=float, default=365.0)
    ap.add_argument("--budget-gb", type=float, default=60.0)
    ap.add_argument("--drain", action="store_true")
    args = ap.parse_args()
    reqs = poisson_requests(args.rate, args.window, seed=5, max_days=args.max_days)
    mix = {}
    for r in reqs:
        mix[(r.truncation, r.levels)] = mix.get((r.truncation, r.levels), 0) + r.days
    total = sum(mix.values())
    mix = {k: v / total for k, v in mix.items()}
    server = Server(Server.capacity_for(args.budget_gb * 1e9, mix), keep_results=False)
    print(json.dumps(server.run(reqs, args.window, drain=args.drain)))
