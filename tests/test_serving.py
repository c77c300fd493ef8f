"""Host logic of the serving loop on CPU, with a fake live arena that stands
in for the device arena (test_batch_gpu.py runs the real one): admission as
ranges free up, admission intervals, exact step counting, results read and
worlds evicted when their steps are done."""
import pytest

from alien_b200 import serving, worldgen
from alien_b200 import params as P
from alien_b200._lib import AlienError


class FakeCapacity:
    def __init__(self, cells):
        self.cellSlots = cells


class FakeArena:
    """admits while the cells fit; records the steps each world received"""

    def __init__(self, cells):
        self.capacity = FakeCapacity(cells)
        self.free = cells
        self.worlds = {}      # slot -> [cells, budget, steps done]
        self.next_slot = 0
        self.enqueued = 0
        self.evicted = []
        self.closed = False

    def admit(self, data, world, params, timestep, steps):
        n = data.num_cells
        if n > self.free:
            raise AlienError(serving.ERR_CAPACITY, "no free cell range in the arena")
        self.free -= n
        slot = self.next_slot
        self.next_slot += 1
        self.worlds[slot] = [n, steps, 0]
        return slot

    def enqueue_timesteps(self, k):
        self.enqueued += k
        for w in self.worlds.values():
            w[2] = min(w[1], w[2] + k)  # the device budget stops a world exactly

    def synchronize(self):
        pass

    def get_simulation_data(self, slot):
        return ("result", slot, self.worlds[slot][2])

    def evict(self, slot):
        self.free += self.worlds.pop(slot)[0]
        self.evicted.append(slot)

    def device_bytes(self):
        return 0

    def close(self):
        self.closed = True


def _request(rid, steps, cells=2000, arrival=0.0):
    data, world = worldgen.mixed_world(rid, cells)
    return serving.Request(rid, data, world, P.benchmark_parameters(P.MOTION_FLUID), steps, arrival=arrival)


def _loop(cells=1 << 40, **kw):
    return serving.ServingLoop(0, arena=FakeArena(cells), **kw)


def test_admission_waves_respect_interval():
    loop = _loop(steps_per_tick=4, admit_interval=1.0)
    loop.submit(_request(0, 400))
    loop.tick(0.0)                      # nothing runs: admitted at once
    assert list(loop.resident) == [0]
    t = 0.1
    for rid in range(1, 6):             # arrivals while a world runs, within the interval
        loop.submit(_request(rid, 40, arrival=t))
        loop.tick(t)
        t += 0.2
    assert len(loop.resident) == 1 and len(loop.waiting) == 5
    loop.tick(1.05)                     # the next wave takes all five
    assert len(loop.resident) == 6 and not loop.waiting
    loop.submit(_request(6, 40, arrival=1.2))
    loop.tick(1.2)
    assert len(loop.resident) == 6 and len(loop.waiting) == 1
    assert loop.report(1.0)["p99_admission_wait_s"] <= 1.0 + 1e-9


def test_admission_waits_for_free_ranges_and_counts_steps_exactly():
    r0, r1, r2 = _request(0, 8), _request(1, 8), _request(2, 6, cells=500)
    arena = FakeArena(int(1.5 * r0.data.num_cells))
    loop = serving.ServingLoop(0, arena=arena, steps_per_tick=4, keep_results=True)
    for r in (r0, r1, r2):
        loop.submit(r)
    loop.tick(0.0)                      # r0 fits; r1 does not; the smaller r2 behind it does
    assert sorted(loop.resident) == [0, 1] and [r.rid for r in loop.waiting] == [1]
    loop.tick(0.0)                      # 4 steps each
    loop.tick(0.0)                      # r0 done at 8 steps, r2 done at 6: both evicted
    assert sorted(r.rid for r in loop.finished) == [0, 2] and arena.evicted == [0, 1]
    assert r0.result == ("result", 0, 8) and r2.result == ("result", 1, 6)
    while not loop.idle():
        loop.tick(0.0)
    assert [r.rid for r in loop.finished][-1] == 1 and r1.result[2] == 8
    assert loop.cell_steps == 8 * (r0.data.num_cells + r1.data.num_cells) + 6 * r2.data.num_cells
    loop.close()
    assert arena.closed


def test_interval_validation():
    with pytest.raises(ValueError):
        serving.ServingLoop(1 << 30, admit_interval=-1.0, arena=FakeArena(1))
    with pytest.raises(ValueError):
        serving.ServingLoop(1 << 30, steps_per_tick=0, arena=FakeArena(1))


def test_requests_finish_at_their_own_step_count():
    loop = _loop(steps_per_tick=4)
    short, long_ = _request(0, 4), _request(1, 40)
    loop.submit(short)
    loop.submit(long_)
    loop.tick(0.0)                      # both admitted
    loop.tick(0.0)                      # 4 steps: the short one is finished and evicted
    assert [r.rid for r in loop.finished] == [0] and list(loop.resident) == [1]
    while not loop.idle():
        loop.tick(0.0)
    assert [r.rid for r in loop.finished] == [0, 1]
    assert loop.report(1.0)["requests_resident"] == 0


def test_other_admission_errors_propagate():
    class Broken(FakeArena):
        def admit(self, *a):
            raise AlienError(2, "invalid cell transfer objects")

    loop = serving.ServingLoop(0, arena=Broken(1 << 30))
    loop.submit(_request(0, 4))
    with pytest.raises(AlienError):
        loop.tick(0.0)
