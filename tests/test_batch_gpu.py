"""Batched multi-world arena, live arena and serving loop: every world
evolves exactly as it does alone (bit for bit: the step is deterministic and
all sums are order-independent), also when worlds are admitted into and
evicted from a live arena between its steps; step budgets stop worlds
exactly, and the serving loop's results equal the results of running each
request alone."""
import numpy as np
import pytest

from alien_b200 import params as P
from alien_b200 import serving, worldgen
from alien_b200._lib import AlienError, ArenaCapacity
from alien_b200.facade import BatchSimulation, LiveArena, SimulationFacade

pytestmark = pytest.mark.gpu


def alone(data, world, prm, steps):
    s = SimulationFacade()
    s.new_simulation(0, world, prm)
    s.set_simulation_data(data)
    s.calc_timesteps(steps)
    out = s.get_simulation_data()
    s.close_simulation()
    return out


def mixed_worlds():
    a = worldgen.random_test_world(31, world=(64, 64)) + (P.benchmark_parameters(P.MOTION_FLUID),)
    b = worldgen.random_test_world(32, world=(96, 80), free_cells=400) + (P.benchmark_parameters(P.MOTION_COLLISION),)
    c = worldgen.mixed_world(33, 3000) + (P.benchmark_parameters(P.MOTION_FLUID),)
    prm = P.benchmark_parameters(P.MOTION_FLUID)
    prm.smoothingLength = 1.2  # different tile side in the same arena
    d = worldgen.random_test_world(34, world=(50, 70)) + (prm,)
    return [a, b, c, d]


def test_batch_equals_alone_bit_for_bit():
    worlds = mixed_worlds()
    batch = BatchSimulation(worlds)
    batch.calc_timesteps(25)
    for w, (data, world, prm) in enumerate(worlds):
        got = batch.get_simulation_data(w)
        ref = alone(data, world, prm, 25)
        assert np.array_equal(got.cells, ref.cells), w
        assert np.array_equal(got.particles, ref.particles), w
    batch.close()


def test_step_budgets_stop_worlds_exactly():
    worlds = mixed_worlds()
    batch = BatchSimulation(worlds)
    budgets = [5, 12, 1, 20]
    for w, n in enumerate(budgets):
        batch.set_step_budget(w, n)
    batch.calc_timesteps(30)
    assert batch.num_active() == 0
    for w, (data, world, prm) in enumerate(worlds):
        t, remaining, active = batch.world_status(w)
        assert (t, remaining, active) == (budgets[w], 0, False)
        got = batch.get_simulation_data(w)
        ref = alone(data, world, prm, budgets[w])
        assert np.array_equal(got.cells, ref.cells), w
    batch.close()


def test_serving_results_equal_alone():
    specs = []

    def make(rid, rng):
        data, world = worldgen.mixed_world(100 + rid, int(rng.integers(500, 4000)))
        steps = int(rng.integers(3, 40))
        specs.append((data, world, steps))
        return serving.Request(rid, data, world, P.benchmark_parameters(P.MOTION_FLUID), steps)

    loop = serving.ServingLoop(hbm_budget_bytes=2 << 30, keep_results=True)
    rng = np.random.default_rng(0)
    # requests arrive while others are running
    for tick in range(60):
        if tick % 5 == 0 and tick < 40:
            loop.submit(make(len(specs), rng))
        loop.tick(float(tick))
    while not loop.idle():
        loop.tick(0.0)
    assert len(loop.finished) == len(specs)
    for r in loop.finished:
        data, world, steps = specs[r.rid]
        ref = alone(data, world, P.benchmark_parameters(P.MOTION_FLUID), steps)
        assert np.array_equal(r.result.cells, ref.cells), r.rid
        assert np.array_equal(r.result.particles, ref.particles), r.rid


def test_worlds_at_different_timestep_phases_equal_alone():
    """a world stopped by its budget and started again runs one step behind
    the others, so the angle-force steps (timestep % 3 == 0) of the worlds
    differ within one launch; each world still evolves as it does alone"""
    worlds = mixed_worlds()
    batch = BatchSimulation(worlds)
    batch.set_step_budget(0, 1)
    batch.set_step_budget(2, 2)
    batch.calc_timesteps(3)            # world 0 at t = 1, world 2 at t = 2, others at t = 3
    batch.set_step_budget(0, 10)
    batch.set_step_budget(2, 10)
    batch.calc_timesteps(10)
    expect = [11, 13, 12, 13]
    for w, (data, world, prm) in enumerate(worlds):
        t, _, _ = batch.world_status(w)
        assert t == expect[w], w
        got = batch.get_simulation_data(w)
        ref = alone(data, world, prm, expect[w])
        assert np.array_equal(got.cells, ref.cells), w
        assert np.array_equal(got.particles, ref.particles), w
    batch.close()


def small_capacity(worlds=8, cells=40_000):
    c = ArenaCapacity()
    c.maxWorlds = worlds
    c.cellSlots = cells
    c.particleSlots = 4 * cells + 16 * 4096
    c.tiles = 64 * cells
    c.particleMapSlots = 64 * cells
    c.auxBytes = 1 << 20
    return c


def assert_equals_alone(arena, slot, spec, steps):
    data, world, prm = spec
    got = arena.get_simulation_data(slot)
    ref = alone(data, world, prm, steps)
    assert np.array_equal(got.cells, ref.cells), slot
    assert np.array_equal(got.particles, ref.particles), slot


def test_live_arena_admit_evict_equals_alone():
    """worlds admitted between steps and into ranges an evicted world freed
    evolve as alone, and the worlds already resident are not disturbed"""
    a, b, c, d = mixed_worlds()
    arena = LiveArena(small_capacity())
    assert LiveArena.bytes_for(arena.capacity) == arena.device_bytes()
    wa = arena.admit(*a)
    wb = arena.admit(*b)
    arena.calc_timesteps(7)
    wc = arena.admit(*c)                    # a third world while two have stepped
    arena.enqueue_timesteps(5)
    arena.synchronize()
    assert_equals_alone(arena, wa, a, 12)
    arena.evict(wa)
    assert arena.num_resident() == 2
    wd = arena.admit(*d)                    # into the freed ranges
    assert wd == wa
    arena.calc_timesteps(9)
    assert_equals_alone(arena, wb, b, 21)
    assert_equals_alone(arena, wc, c, 14)
    assert_equals_alone(arena, wd, d, 9)
    with pytest.raises(AlienError):
        arena.get_simulation_data(5)        # never admitted
    arena.close()


def test_live_arena_full_rejects_and_keeps_its_worlds():
    a, b = mixed_worlds()[2], mixed_worlds()[1]
    arena = LiveArena(small_capacity(worlds=2, cells=3600))
    wa = arena.admit(*a)
    with pytest.raises(AlienError) as e:
        arena.admit(*b)                     # no free cell range: the arena is unchanged
    assert e.value.code == 6
    arena.calc_timesteps(6)
    assert_equals_alone(arena, wa, a, 6)
    arena.evict(wa)
    wb = arena.admit(*b)
    arena.calc_timesteps(4)
    assert_equals_alone(arena, wb, b, 4)
    arena.close()


def test_live_arena_budgets_and_mixed_motion_types():
    worlds = mixed_worlds()
    arena = LiveArena(small_capacity())
    slots = [arena.admit(data, world, prm, 0, steps) for (data, world, prm), steps in zip(worlds, [3, 8, 5, 11])]
    arena.calc_timesteps(12)
    assert arena.num_active() == 0
    for slot, spec, steps in zip(slots, worlds, [3, 8, 5, 11]):
        assert arena.world_status(slot)[0] == steps
        assert_equals_alone(arena, slot, spec, steps)
    arena.close()


def test_live_arena_grows_a_world_that_fills_its_particles():
    """radiation without absorption fills a world's particle range: the world
    moves to larger ranges (same index) while the other keeps stepping"""
    data, world, prm = growing_world()
    other = mixed_worlds()[0]
    arena = LiveArena(small_capacity(cells=20_000))
    wo = arena.admit(*other)
    wg = arena.admit(data, world, prm)
    first = arena.particle_slots(wg)
    for _ in range(16):
        arena.calc_timesteps(16)
    assert arena.particle_slots(wg) > first, "the world did not outgrow its first particle range"
    assert_equals_alone(arena, wg, (data, world, prm), 256)
    assert_equals_alone(arena, wo, other, 256)
    arena.close()


def test_live_arena_first_in_a_fresh_process():
    """a live arena as the process's first handle steps (its kernels' launch
    attributes are set by the arena itself, not by an earlier handle)"""
    import os
    import subprocess
    import sys
    code = (
        "from alien_b200 import params as P, worldgen\n"
        "from alien_b200._lib import ArenaCapacity\n"
        "from alien_b200.facade import LiveArena\n"
        "c = ArenaCapacity(); c.maxWorlds = 4; c.cellSlots = 20000; c.particleSlots = 100000\n"
        "c.tiles = 200000; c.particleMapSlots = 400000; c.auxBytes = 1024\n"
        "a = LiveArena(c)\n"
        "d, w = worldgen.random_test_world(7)\n"
        "k = a.admit(d, w, P.benchmark_parameters(P.MOTION_COLLISION))\n"
        "a.calc_timesteps(5)\n"
        "assert a.world_status(k)[0] == 5\n"
        "a.close()\n"
        "print('ok')\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip().endswith("ok"), out.stderr[-2000:]


def growing_world():
    """radiation without absorption: about 48 new particles per step fill
    the first particle range within 200 steps"""
    data, world = worldgen.random_test_world(36, world=(384, 384), free_cells=4000, particles=0)
    data.cells["age"] = 1000
    prm = P.default_parameters()
    prm.radiationProb = 0.01
    for c in range(P.MAX_COLORS):
        prm.radiationCellAgeStrength[c] = 0.002
        prm.radiationAbsorption[c] = 0.0
    return data, world, prm


def test_growing_particle_storage_changes_no_state():
    """a world that outgrows its particle storage (export, larger arena,
    re-import, fluid densities and absorbers carried) ends bit for bit where
    the same world with room reserved from the start ends"""
    data, world, prm = growing_world()
    grown = alone(data, world, prm, 256)
    s = SimulationFacade()
    s.new_simulation(0, world, prm)
    s.set_simulation_data(data)
    s.resize_arrays_if_necessary(particles=200_000)
    s.calc_timesteps(256)
    roomy = s.get_simulation_data()
    s.close_simulation()
    assert roomy.num_particles > 4000
    assert np.array_equal(grown.cells, roomy.cells)
    assert np.array_equal(grown.particles, roomy.particles)


def feature_worlds():
    """worlds with zones and flows, radiation sources with the backflow, and
    rigidity, beside a plain one"""
    import tests.test_zones_gpu as tz
    a = tz.zone_world(71) + (tz.zone_params(P.MOTION_FLUID),)
    data, world = tz.zone_world(72)
    data.cells["age"] = 1000
    prm = P.default_parameters()
    prm.motionType = P.MOTION_COLLISION
    for c in range(P.MAX_COLORS):
        prm.radiationCellAgeStrength[c] = 0.002
        prm.externalEnergyBackflowFactor[c] = 0.3
    prm.externalEnergyControl = 1
    prm.externalEnergy = 20.0
    prm.numRadiationSources = 1
    prm.radiationSources[0].posX, prm.radiationSources[0].posY = 30.0, 40.0
    prm.radiationSources[0].strength, prm.radiationSources[0].radius = 1.0, 4.0
    prm.radiationSources[0].velX = 0.25
    b = (data, world, prm)
    rp = P.benchmark_parameters(P.MOTION_FLUID)
    rp.rigidity = 0.5
    c = worldgen.random_test_world(73, world=(96, 96), clusters=8) + (rp,)
    d = mixed_worlds()[1]
    return [a, b, c, d]


def test_batch_with_zones_sources_and_rigidity_equals_alone():
    """zones move, sources emit, the pool takes the backflow and clusters
    blend per world: a batch and a live arena give every world its results
    alone, bit for bit"""
    worlds = feature_worlds()
    batch = BatchSimulation(worlds)
    batch.calc_timesteps(7)
    arena = LiveArena(small_capacity())
    slots = [arena.admit(*spec) for spec in worlds]
    arena.calc_timesteps(7)
    for w, (data, world, prm) in enumerate(worlds):
        s = SimulationFacade()
        s.new_simulation(0, world, prm)
        s.set_simulation_data(data)
        s.calc_timesteps(7)
        ref = s.get_simulation_data()
        s.close_simulation()
        for got in (batch.get_simulation_data(w), arena.get_simulation_data(slots[w])):
            assert np.array_equal(got.cells, ref.cells), w
            assert np.array_equal(got.particles, ref.particles), w
    batch.close()
    arena.close()
