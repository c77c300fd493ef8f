"""Admission logic of the serving loop on CPU, with cohorts that stand in for
the device arenas (the GPU tests in test_batch_gpu.py run the real ones)."""
import numpy as np
import pytest

from alien_b200 import serving, worldgen
from alien_b200 import params as P


class FakeBatch:
    def __init__(self):
        self.enqueued = 0

    def enqueue_timesteps(self, k):
        self.enqueued += k

    def synchronize(self):
        pass


class FakeCohort:
    def __init__(self, requests):
        self.requests = requests
        self.batch = FakeBatch()
        self.bytes = sum(serving.estimate_bytes(r.data, r.world) for r in requests)
        self.max_steps = max(r.steps for r in requests)
        self.steps_done = 0

    @property
    def done(self):
        return self.steps_done >= self.max_steps

    def finish_done(self, now, keep_results):
        out = []
        for r in self.requests:
            if r.finished is None and r.steps <= self.steps_done:
                r.finished = now
                out.append(r)
        return out

    def close(self):
        pass


@pytest.fixture
def fake_cohorts(monkeypatch):
    monkeypatch.setattr(serving, "_Cohort", FakeCohort)


def _request(rid, steps, cells=2000, arrival=0.0):
    data, world = worldgen.mixed_world(rid, cells)
    return serving.Request(rid, data, world, P.benchmark_parameters(P.MOTION_FLUID), steps, arrival=arrival)


def test_admission_waves_respect_interval(fake_cohorts):
    loop = serving.ServingLoop(hbm_budget_bytes=1 << 40, steps_per_tick=4, admit_interval=1.0)
    loop.submit(_request(0, 400))
    loop.tick(0.0)                      # nothing runs: admitted at once
    assert len(loop.cohorts) == 1
    t = 0.1
    for rid in range(1, 6):             # arrivals while a cohort runs, within the interval
        loop.submit(_request(rid, 40, arrival=t))
        loop.tick(t)
        t += 0.2
    assert len(loop.cohorts) == 1 and len(loop.waiting) == 5
    loop.tick(1.05)                     # the next wave takes all five
    assert [len(c.requests) for c in loop.cohorts] == [1, 5] and not loop.waiting
    loop.submit(_request(6, 40, arrival=1.2))
    loop.tick(1.2)
    assert len(loop.cohorts) == 2 and len(loop.waiting) == 1
    assert loop.report(1.0)["p99_admission_wait_s"] <= 1.0 + 1e-9


def test_admission_respects_budget_and_frees_bytes(fake_cohorts):
    r0, r1 = _request(0, 8), _request(1, 8)
    b = serving.estimate_bytes(r0.data, r0.world)
    loop = serving.ServingLoop(hbm_budget_bytes=int(1.5 * b), steps_per_tick=4)
    loop.submit(r0)
    loop.submit(r1)
    loop.tick(0.0)
    assert [len(c.requests) for c in loop.cohorts] == [1] and len(loop.waiting) == 1
    loop.tick(0.0)                      # budget full: the second request waits
    assert len(loop.waiting) == 1
    loop.tick(0.0)                      # first cohort done and freed after 8 steps
    loop.tick(0.0)
    assert len(loop.waiting) == 0 and [r.rid for r in loop.finished] == [0]
    while not loop.idle():
        loop.tick(0.0)
    assert [r.rid for r in loop.finished] == [0, 1]
    assert loop.cell_steps == 8 * (r0.data.num_cells + r1.data.num_cells)


def test_interval_validation():
    with pytest.raises(ValueError):
        serving.ServingLoop(1 << 30, admit_interval=-1.0)
    with pytest.raises(ValueError):
        serving.ServingLoop(1 << 30, steps_per_tick=0)


def test_requests_finish_before_their_cohort(fake_cohorts):
    loop = serving.ServingLoop(hbm_budget_bytes=1 << 40, steps_per_tick=4)
    short, long_ = _request(0, 4), _request(1, 40)
    loop.submit(short)
    loop.submit(long_)
    loop.tick(0.0)                      # one cohort with both
    loop.tick(0.0)                      # 4 steps: the short one is finished
    assert [r.rid for r in loop.finished] == [0] and len(loop.cohorts) == 1
    while not loop.idle():
        loop.tick(0.0)
    assert [r.rid for r in loop.finished] == [0, 1]
