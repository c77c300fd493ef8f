"""Particle storage that runs out inside a step: the world halts before its
step writes the new particles, the host grows its range on the device and
completes the step, then runs the steps the world missed.  Nothing is
dropped and nothing differs from a run whose storage was large enough from
the start, in a single world, a batch and a live arena.  Only a live arena
without a free range large enough drops the excess (and reports it), as the
reference's Array::tryGetEntries does (Array.cuh:246-267).

Also the last step of a step budget: the particles that step creates by
splitting are written although the world stops with it."""
import numpy as np
import pytest

from alien_b200 import params as P
from alien_b200 import worldgen
from alien_b200._lib import AlienError, ArenaCapacity
from alien_b200.facade import BatchSimulation, LiveArena, SimulationFacade

pytestmark = pytest.mark.gpu


def burst_world(seed=91, cells=3000, size=256):
    """every cell radiates every step and no particle is absorbed: about one
    new particle per cell per step, so the first particle range (cells +
    4096 slots) overflows in the third step, and the larger ones again"""
    data, world = worldgen.random_test_world(seed, world=(size, size), free_cells=cells, particles=0)
    data.cells["age"] = 1000
    data.cells["energy"] = 200.0
    prm = P.default_parameters()
    prm.radiationProb = 1.0
    for c in range(P.MAX_COLORS):
        prm.radiationCellAgeStrength[c] = 0.0005
        prm.radiationAbsorption[c] = 0.0
    return data, world, prm


def split_world(seed=95):
    """energetic particles that split (1 % of them per step)"""
    data, world = worldgen.random_test_world(seed, world=(128, 128), free_cells=300, particles=3000)
    data.particles["energy"] = 50.0
    prm = P.default_parameters()
    for c in range(P.MAX_COLORS):
        prm.particleSplitEnergy[c] = 2.0
        prm.radiationAbsorption[c] = 0.0
    return data, world, prm


def run(spec, steps, room=0):
    data, world, prm = spec
    s = SimulationFacade()
    s.new_simulation(0, world, prm)
    s.set_simulation_data(data)
    if room:
        s.resize_arrays_if_necessary(particles=room)
    first = s.get_array_sizes().particleArraySize
    s.calc_timesteps(steps)
    out = s.get_simulation_data()
    last = s.get_array_sizes().particleArraySize
    s.close_simulation()
    return out, first, last


def assert_same(a, b, label=""):
    assert np.array_equal(a.cells, b.cells), label
    assert np.array_equal(a.particles, b.particles), label


def test_single_world_grows_inside_a_check_interval():
    spec = burst_world()
    grown, first, last = run(spec, 40)
    roomy, roomy_first, roomy_last = run(spec, 40, room=400_000)
    assert grown.num_particles > first, "the first range did not overflow"
    assert last > first and roomy_last == roomy_first
    assert_same(grown, roomy)


def test_batch_worlds_grow_and_catch_up():
    """two bursting worlds halt at different steps, a plain world keeps
    stepping; every world ends where it ends alone with room"""
    specs = [burst_world(92), worldgen.random_test_world(93, world=(64, 64)) + (P.benchmark_parameters(P.MOTION_FLUID),),
             burst_world(94, cells=1500, size=200)]
    batch = BatchSimulation(specs)
    first = [batch.particle_slots(w) for w in range(3)]
    batch.calc_timesteps(30)
    assert batch.particle_slots(0) > first[0] and batch.particle_slots(2) > first[2]
    for w, spec in enumerate(specs):
        assert batch.world_status(w)[0] == 30
        ref, _, _ = run(spec, 30, room=200_000)
        assert_same(batch.get_simulation_data(w), ref, w)
    batch.close()


def live_capacity(particles):
    c = ArenaCapacity()
    c.maxWorlds = 4
    c.cellSlots = 20_000
    c.particleSlots = particles
    c.tiles = 1_000_000
    c.particleMapSlots = 1_000_000
    c.auxBytes = 1 << 20
    return c


def test_live_arena_world_grows_mid_interval_within_its_budget():
    """a bursting world with a step budget halts, moves to a larger range and
    catches up exactly its budget; the other world's budget is untouched"""
    burst = burst_world(96, cells=2000, size=200)
    other = worldgen.random_test_world(97, world=(80, 80)) + (P.benchmark_parameters(P.MOTION_COLLISION),)
    arena = LiveArena(live_capacity(600_000))
    wb = arena.admit(*burst, 0, 25)
    wo = arena.admit(*other, 0, 33)
    first = arena.particle_slots(wb)
    arena.enqueue_timesteps(12)
    arena.synchronize()
    assert arena.particle_slots(wb) > first
    assert arena.world_status(wb)[:2] == (12, 13)
    arena.calc_timesteps(40)
    assert arena.world_status(wb)[0] == 25 and arena.world_status(wo)[0] == 33
    assert arena.num_active() == 0
    assert_same(arena.get_simulation_data(wb), run(burst, 25, room=200_000)[0], "burst")
    assert_same(arena.get_simulation_data(wo), run(other, 33)[0], "other")
    arena.close()


def test_live_arena_without_room_drops_and_reports():
    """no larger particle range is free: the step completes with the excess
    dropped, the next synchronisation reports it, and the world keeps its
    step count"""
    burst = burst_world(98, cells=2000, size=200)
    arena = LiveArena(live_capacity(9_000))
    wb = arena.admit(*burst)
    with pytest.raises(AlienError) as e:
        arena.calc_timesteps(6)
    assert e.value.code == 6
    assert arena.world_status(wb)[0] == 6
    got = arena.get_simulation_data(wb)
    assert got.num_particles <= arena.particle_slots(wb)
    arena.close()


def test_last_budgeted_step_writes_its_split_particles():
    spec = split_world()
    for steps in (1, 4, 9):
        batch = BatchSimulation([spec, spec])
        batch.set_step_budget(0, steps)
        batch.calc_timesteps(steps + 3)
        assert batch.world_status(0)[0] == steps
        ref, _, _ = run(spec, steps)
        assert_same(batch.get_simulation_data(0), ref, steps)
        ref2, _, _ = run(spec, steps + 3)
        assert_same(batch.get_simulation_data(1), ref2, steps)
        batch.close()
