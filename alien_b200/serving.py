"""Continuous-batching serving loop for simulation requests.

No counterpart in the reference (its EngineWorker serves one world).  A
request is a world (DataTO, size, parameters) and a number of timesteps.  The
loop keeps every admitted world resident on the device and steps all of them
together:

* admission: a waiting request is admitted when its estimated device bytes fit
  into the HBM budget next to the resident worlds; requests that arrive while
  others run are admitted at the next admission wave (no queue barrier).
  Waves can be held ``admit_interval`` seconds apart while cohorts run, so
  that arrivals gather into fewer, larger cohorts (fewer launches per step)
  at the price of a longer wait before admission; the default admits at
  every tick;
* cohorts: each admission wave becomes one batch arena (alien_b200_batch)
  whose worlds carry per-world step budgets, so a world stops exactly after
  its requested steps without host synchronisation;
* a tick = a few timesteps (``steps_per_tick``) of every cohort with active
  worlds, each cohort on its own CUDA stream so that their kernels overlap on
  the device; the tick's wall time per step is the per-step latency every
  running request sees (p50 / p99 reported);
* a request whose steps are done is finished at once (its world no longer
  steps; its results are read while the cohort runs on); a cohort whose
  worlds are all done is freed, which returns its bytes to the budget.

Results do not depend on what else is resident: every world evolves under the
same deterministic step as alone (tests/test_batch_gpu.py checks alone vs in
the mix).
"""
from __future__ import annotations

import dataclasses
import time
from typing import Callable

import numpy as np

from .facade import BatchSimulation
from .params import PhysicsParams
from .to import DataTO

# device bytes per cell and per particle slot of an arena (engine.cu::build),
# plus the per-world particle map; used for admission before allocating
BYTES_PER_CELL_SLOT = 760
BYTES_PER_PARTICLE_SLOT = 130


def estimate_bytes(data: DataTO, world) -> int:
    n, p = data.num_cells, data.num_particles
    cell_slots = n + 256
    part_slots = p + n + max(4096, (p + n) // 2) + 256
    return (BYTES_PER_CELL_SLOT * cell_slots + BYTES_PER_PARTICLE_SLOT * part_slots
            + 4 * world[0] * world[1] + 304 * n)


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


class _Cohort:
    def __init__(self, requests: list[Request]):
        self.requests = requests
        self.batch = BatchSimulation([(r.data, r.world, r.params) for r in requests])
        for w, r in enumerate(requests):
            self.batch.set_step_budget(w, r.steps)
        self.bytes = self.batch.device_bytes()
        self.max_steps = max(r.steps for r in requests)
        self.steps_done = 0

    @property
    def done(self) -> bool:
        return self.steps_done >= self.max_steps

    def finish_done(self, now: float, keep_results: bool) -> list[Request]:
        """requests whose step budget is used up, finished now: their worlds no
        longer step, so their results can be read while the cohort runs on"""
        out = []
        for w, r in enumerate(self.requests):
            if r.finished is None and r.steps <= self.steps_done:
                r.finished = now
                if keep_results:
                    r.result = self.batch.get_simulation_data(w)
                out.append(r)
        return out

    def close(self):
        self.batch.close()


class ServingLoop:
    def __init__(self, hbm_budget_bytes: int, keep_results: bool = False, max_cohort_worlds: int = 256,
                 steps_per_tick: int = 4, admit_interval: float = 0.0):
        if not 1 <= steps_per_tick <= 64:
            raise ValueError("steps_per_tick must be in [1, 64]")
        if admit_interval < 0:
            raise ValueError("admit_interval must be >= 0")
        self.steps_per_tick = int(steps_per_tick)
        self.admit_interval = float(admit_interval)
        self.last_admit: float | None = None
        self.budget = int(hbm_budget_bytes)
        self.keep_results = keep_results
        self.max_cohort_worlds = max_cohort_worlds
        self.waiting: list[Request] = []
        self.cohorts: list[_Cohort] = []
        self.finished: list[Request] = []
        self.tick_ms: list[float] = []
        self.waits: list[float] = []  # seconds from arrival to admission
        self.cell_steps = 0

    def resident_bytes(self) -> int:
        return sum(c.bytes for c in self.cohorts)

    def submit(self, req: Request) -> None:
        self.waiting.append(req)

    def _admit(self, now: float) -> None:
        if not self.waiting:
            return
        if self.cohorts and self.last_admit is not None and now - self.last_admit < self.admit_interval:
            return
        free = self.budget - self.resident_bytes()
        wave, wave_bytes = [], 0
        rest = []
        for r in self.waiting:
            b = estimate_bytes(r.data, r.world)
            if len(wave) < self.max_cohort_worlds and wave_bytes + b <= free:
                wave.append(r)
                wave_bytes += b
            else:
                rest.append(r)
        self.waiting = rest
        if wave:
            for r in wave:
                r.admitted = now
                r.cells = r.data.num_cells
                self.waits.append(max(0.0, now - r.arrival))
            self.cohorts.append(_Cohort(wave))
            self.last_admit = now

    def tick(self, now: float) -> float:
        """``steps_per_tick`` timesteps of every running cohort, each cohort
        on its own stream so that their kernels overlap, with the admission
        of waiting requests done while they run; returns the per-step
        latency in ms (wall time of the tick / steps)"""
        k = self.steps_per_tick
        t0 = time.perf_counter()
        running = list(self.cohorts)
        for c in running:
            c.batch.enqueue_timesteps(k)
        # admission (host work and the new arenas' uploads on their own
        # streams) overlaps the steps just enqueued; new cohorts step from
        # the next tick on
        self._admit(now)
        if not running:
            return 0.0
        for c in running:
            c.batch.synchronize()
        ms = (time.perf_counter() - t0) * 1000.0 / k
        for c in running:
            for r in c.requests:
                self.cell_steps += r.cells * max(0, min(k, r.steps - c.steps_done))
            c.steps_done += k
        self.tick_ms.append(ms)
        done_now = time.perf_counter()
        for c in running:
            self.finished.extend(c.finish_done(done_now, self.keep_results))
        keep = []
        for c in self.cohorts:
            if c in running and c.done:
                c.close()
            else:
                keep.append(c)
        self.cohorts = keep
        return ms

    def idle(self) -> bool:
        return not self.cohorts and not self.waiting

    def report(self, wall_s: float) -> dict:
        t = np.array(self.tick_ms) if self.tick_ms else np.zeros(1)
        wq = np.array(self.waits) if self.waits else np.zeros(1)
        return {
            "p50_admission_wait_s": float(np.percentile(wq, 50)),
            "p99_admission_wait_s": float(np.percentile(wq, 99)),
            "requests_finished": len(self.finished),
            "requests_waiting": len(self.waiting),
            "ticks": len(self.tick_ms),
            "p50_step_ms": float(np.percentile(t, 50)),
            "p99_step_ms": float(np.percentile(t, 99)),
            "cell_steps": int(self.cell_steps),
            "mcell_steps_per_s": self.cell_steps / max(wall_s, 1e-9) / 1e6,
        }


def run_poisson(make_request: Callable[[int, np.random.Generator], Request], rate_per_s: float, duration_s: float,
                hbm_budget_bytes: int, seed: int = 0, keep_results: bool = False, drain: bool = True,
                steps_per_tick: int = 4, admit_interval: float = 0.0) -> dict:
    """Poisson arrivals at ``rate_per_s`` for ``duration_s`` seconds of wall
    time; requests are built by ``make_request(rid, rng)``."""
    rng = np.random.default_rng(seed)
    loop = ServingLoop(hbm_budget_bytes, keep_results, steps_per_tick=steps_per_tick, admit_interval=admit_interval)
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
    return out
