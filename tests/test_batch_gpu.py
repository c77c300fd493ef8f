"""Batched multi-world arena and serving loop: every world evolves exactly as
it does alone (bit for bit: the step is deterministic and all sums are
order-independent), step budgets stop worlds exactly, and the serving loop's
results equal the results of running each request alone."""
import numpy as np
import pytest

from alien_b200 import params as P
from alien_b200 import serving, worldgen
from alien_b200.facade import BatchSimulation, SimulationFacade

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
