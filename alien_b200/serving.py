"""Continuous-batching serving loop for simulation requests.

No counterpart in the reference (its EngineWorker serves one world,
source/EngineImpl/EngineWorker.cpp:450-476).  A request is a world (DataTO,
size, parameters) and a number of timesteps.  Every admitted world lives in
one live arena (alien_b200_arena_create) whose memory is reserved once for
the HBM budget, and all resident worlds step in the same launches:

* admission: a waiting request is admitted as soon as the arena has free
  ranges for it (alien_b200_world_admit); its upload and ingest are queued
  on the arena's stream behind the steps already enqueued, so the resident
  worlds keep stepping while it is admitted.  Admission waves can be held
  ``admit_interval`` seconds apart; the default admits at every tick;
* a tick = ``steps_per_tick`` timesteps of the arena, then one wait; its wall
  time per step is the per-step latency every resident request sees (p50 /
  p99 reported);
* every world carries its step budget on the device, so it stops exactly
  after its requested steps; the loop counts the same steps on the host,
  reads the results of finished requests and evicts them, which frees their
  ranges for the next admissions.

Results do not depend on what else is resident: every world evolves under the
same deterministic step as alone (tests/test_batch_gpu.py checks alone vs in
the mix, with admissions and evictions in between).
"""
from __future__ import annotations

import dataclasses
import time
from typing import Callable

import numpy as np

from ._lib import AlienError
from .params import PhysicsParams
from .to import DataTO

ERR_CAPACITY = 6  # ALIEN_B200_ERR_CAPACITY


@dataclasses.dataclass
class Request:
    rid: int
    data: DataTO
    world: tuple
    params: PhysicsParams
    steps: int
    arrival: float = 0.0
    admitted: float | None = None
    finished: float | None = None
    result: DataTO | None = None
    cells: int = 0
    steps_done: int = 0
    slot: int = -1


class ServingLoop:
    def __init__(self, hbm_budget_bytes: int, keep_results: bool = False, steps_per_tick: int = 4,
                 admit_interval: float = 0.0, max_worlds: int = 1024, arena=None, max_misses: int = 8,
                 max_wave_ms: float = 25.0):
        """``arena``: a LiveArena (default: one sized for the budget);
        ``max_misses``: requests that did not fit after which a wave ends;
        ``max_wave_ms``: host time after which a wave ends (the enqueued
        steps keep the GPU busy meanwhile; the rest waits for the next tick)"""
        if not 1 <= steps_per_tick <= 64:
            raise ValueError("steps_per_tick must be in [1, 64]")
        if admit_interval < 0:
            raise ValueError("admit_interval must be >= 0")
        if arena is None:
            from .facade import LiveArena
            arena = LiveArena(LiveArena.capacity_for(int(hbm_budget_bytes), max_worlds=max_worlds))
        self.arena = arena
        self.max_misses = int(max_misses)
        self.max_wave_ms = float(max_wave_ms)
        self.steps_per_tick = int(steps_per_tick)
        self.admit_interval = float(admit_interval)
        self.last_admit: float | None = None
        self.keep_results = keep_results
        self.waiting: list[Request] = []
        self.resident: dict[int, Request] = {}
        self.finished: list[Request] = []
        self.tick_ms: list[float] = []
        self.waits: list[float] = []  # seconds from arrival to admission
        self.admit_ms: list[float] = []  # host time of each admission wave
        self.admit_call_ms: list[float] = []  # host time of each successful admission
        self.sync_ms: list[float] = []  # host wait for the tick's steps
        self.evict_ms: list[float] = []
        self.cell_steps = 0
        self.capacity_events = 0  # synchronisations that reported dropped particles

    def submit(self, req: Request) -> None:
        self.waiting.append(req)

    def _admit(self, now: float) -> None:
        if not self.waiting:
            return
        if self.resident and self.last_admit is not None and now - self.last_admit < self.admit_interval:
            return
        t0 = time.perf_counter()
        rest = []
        misses = 0
        for i, r in enumerate(self.waiting):
            if misses >= self.max_misses or (time.perf_counter() - t0) * 1000.0 > self.max_wave_ms:
                rest.extend(self.waiting[i:])  # the arena is full, or the wave's time is up
                break
            ta = time.perf_counter()
            try:
                slot = self.arena.admit(r.data, r.world, r.params, 0, r.steps)
                self.admit_call_ms.append((time.perf_counter() - ta) * 1000.0)
            except AlienError as e:
                if e.code != ERR_CAPACITY:
                    raise
                rest.append(r)  # waits for ranges to free up; smaller requests behind it may fit
                misses += 1
                continue
            r.slot = slot
            r.admitted = now
            r.cells = r.data.num_cells
            r.steps_done = 0
            self.waits.append(max(0.0, now - r.arrival))
            self.resident[slot] = r
        if len(rest) < len(self.waiting):
            self.last_admit = now
        self.waiting = rest
        self.admit_ms.append((time.perf_counter() - t0) * 1000.0)

    def tick(self, now: float) -> float:
        """``steps_per_tick`` timesteps of every resident world, with the
        admission of waiting requests done while they run; returns the
        per-step latency in ms (wall time of the tick / steps)"""
        k = self.steps_per_tick
        t0 = time.perf_counter()
        running = list(self.resident.items())
        if running:
            self.arena.enqueue_timesteps(k)
        # admission overlaps the steps just enqueued; new worlds step from
        # the next tick on
        self._admit(now)
        if not running:
            return 0.0
        ts = time.perf_counter()
        try:
            self.arena.synchronize()
        except AlienError as e:
            if e.code != ERR_CAPACITY:
                raise
            # a world created more particles than its range held (and no
            # larger range was free): the excess was dropped; the loop goes on
            self.capacity_events += 1
        self.sync_ms.append((time.perf_counter() - ts) * 1000.0)
        ms = (time.perf_counter() - t0) * 1000.0 / k
        self.tick_ms.append(ms)
        done_now = time.perf_counter()
        for slot, r in running:
            n = max(0, min(k, r.steps - r.steps_done))
            self.cell_steps += r.cells * n
            r.steps_done += n
            if r.steps_done >= r.steps:
                r.finished = done_now
                te = time.perf_counter()
                if self.keep_results:
                    r.result = self.arena.get_simulation_data(slot)
                self.arena.evict(slot)
                self.evict_ms.append((time.perf_counter() - te) * 1000.0)
                del self.resident[slot]
                self.finished.append(r)
        return ms

    def idle(self) -> bool:
        return not self.resident and not self.waiting

    def close(self) -> None:
        self.arena.close()

    def report(self, wall_s: float) -> dict:
        t = np.array(self.tick_ms) if self.tick_ms else np.zeros(1)
        wq = np.array(self.waits) if self.waits else np.zeros(1)
        am = np.array(self.admit_ms) if self.admit_ms else np.zeros(1)

        def pct(xs, q):
            return float(np.percentile(np.array(xs), q)) if xs else 0.0
        return {
            "p50_admission_wait_s": float(np.percentile(wq, 50)),
            "p99_admission_wait_s": float(np.percentile(wq, 99)),
            "p50_admission_wave_ms": float(np.percentile(am, 50)),
            "p99_admission_wave_ms": float(np.percentile(am, 99)),
            "admissions": len(self.admit_call_ms),
            "p50_admit_call_ms": pct(self.admit_call_ms, 50), "p99_admit_call_ms": pct(self.admit_call_ms, 99),
            "p50_sync_ms": pct(self.sync_ms, 50), "p50_evict_ms": pct(self.evict_ms, 50),
            "requests_finished": len(self.finished),
            "requests_waiting": len(self.waiting),
            "requests_resident": len(self.resident),
            "capacity_events": self.capacity_events,
            "ticks": len(self.tick_ms),
            "p50_step_ms": float(np.percentile(t, 50)),
            "p99_step_ms": float(np.percentile(t, 99)),
            "cell_steps": int(self.cell_steps),
            "mcell_steps_per_s": self.cell_steps / max(wall_s, 1e-9) / 1e6,
        }


def run_poisson(make_request: Callable[[int, np.random.Generator], Request], rate_per_s: float, duration_s: float,
                hbm_budget_bytes: int, seed: int = 0, keep_results: bool = False, drain: bool = True,
                steps_per_tick: int = 4, admit_interval: float = 0.0, max_worlds: int = 1024) -> dict:
    """Poisson arrivals at ``rate_per_s`` for ``duration_s`` seconds of wall
    time; requests are built by ``make_request(rid, rng)``."""
    rng = np.random.default_rng(seed)
    loop = ServingLoop(hbm_budget_bytes, keep_results, steps_per_tick=steps_per_tick, admit_interval=admit_interval,
                       max_worlds=max_worlds)
    try:
        t0 = time.perf_counter()
        next_arrival = rng.exponential(1.0 / rate_per_s)
        rid = 0
        while True:
            now = time.perf_counter() - t0
            while now < duration_s and next_arrival <= now:
                req = make_request(rid, rng)
                req.arrival = next_arrival
                loop.submit(req)
                rid += 1
                next_arrival += rng.exponential(1.0 / rate_per_s)
            if now >= duration_s and (not drain or loop.idle()):
                break
            if loop.idle():
                time.sleep(max(0.0, min(next_arrival - now, 0.01)))
                continue
            loop.tick(now)
        wall = time.perf_counter() - t0
        out = loop.report(wall)
        out["requests_submitted"] = rid
        out["wall_s"] = wall
        out["arena_bytes"] = loop.arena.device_bytes()
        out["arena_cell_slots"] = int(loop.arena.capacity.cellSlots)
    finally:
        loop.close()
    return out
