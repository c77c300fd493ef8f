"""The neuron cell function on the GPU against the FP64 oracle.

Neuron cells (CellFunction_Neuron) run in the steps of their execution order
number: input = bonded cells of the input execution order number (clamped
sums), output = activation(W x + b) (NeuronProcessor.cuh:33-90).  Each case
steps a seeded world with neurons through the C ABI and through the oracle
and compares, by id: signal channels within NEURON_ATOL, signal origin,
targets and the function-used flag exactly or within tolerance; the physics
state one step in as in test_parity_gpu.py.  The oracle itself is pinned
against the reference engine by tests/test_golden.py.
"""
import numpy as np
import pytest

from alien_b200 import params as P
from alien_b200 import worldgen
from alien_b200._lib import AlienError
from alien_b200.facade import SimulationFacade
from oracle.oracle import OracleSimulation
from tests.helpers import compare_cells, compare_particles

pytestmark = pytest.mark.gpu

NEURON_ATOL = 1e-5


def run_both(data, world, prm, steps, timestep=0):
    eng = SimulationFacade()
    eng.new_simulation(timestep, world, prm)
    eng.set_simulation_data(data)
    eng.calc_timesteps(steps)
    got = eng.get_simulation_data()
    eng.close_simulation()
    ora = OracleSimulation(world, prm, timestep)
    ora.set_simulation_data(data)
    ora.calc_timesteps(steps)
    return got, ora.get_simulation_data()


def by_id(cells):
    return cells[np.argsort(cells["id"])]


def compare_signals(got, ref):
    g, r = by_id(got), by_id(ref)
    assert np.array_equal(g["id"], r["id"])
    assert np.array_equal(g["cellFunctionUsed"], r["cellFunctionUsed"])
    assert np.array_equal(g["signalOrigin"], r["signalOrigin"])
    np.testing.assert_allclose(g["signalChannels"], r["signalChannels"], rtol=0, atol=NEURON_ATOL)
    np.testing.assert_allclose(g["signalTargetX"], r["signalTargetX"], rtol=1e-6, atol=NEURON_ATOL)
    np.testing.assert_allclose(g["signalTargetY"], r["signalTargetY"], rtol=1e-6, atol=NEURON_ATOL)


@pytest.mark.parametrize("motion,timestep", [(P.MOTION_FLUID, 0), (P.MOTION_COLLISION, 3)])
def test_neurons_one_step(motion, timestep):
    data, world = worldgen.random_test_world(51 + motion, free_cells=150)
    data = worldgen.add_neurons(data, 51 + motion, fraction=0.7)
    got, ref = run_both(data, world, P.benchmark_parameters(motion), 1, timestep)
    compare_cells(got.cells, ref.cells, world)
    compare_particles(got.particles, ref.particles, world)
    compare_signals(got.cells, ref.cells)


@pytest.mark.parametrize("orders", [6, 3, 1])
def test_neuron_chains_over_all_execution_orders(orders):
    """13 steps cover every execution order number twice; signals travel
    along chains of neurons"""
    data, world = worldgen.calm_test_world(61 + orders)
    data = worldgen.add_neurons(data, 61 + orders, fraction=0.8, num_orders=orders)
    prm = P.benchmark_parameters(P.MOTION_FLUID)
    prm.cellNumExecutionOrderNumbers = orders
    got, ref = run_both(data, world, prm, 13)
    compare_signals(got.cells, ref.cells)
    changed = np.any(by_id(got.cells)["signalChannels"] != by_id(data.cells)["signalChannels"], axis=1)
    assert changed.sum() >= (data.cells["cellFunction"] == 0).sum() // 2


def test_neurons_in_a_batch_equal_alone():
    from alien_b200.facade import BatchSimulation

    worlds = []
    for k in range(3):
        d, w = worldgen.calm_test_world(70 + k)
        worlds.append((worldgen.add_neurons(d, 70 + k, fraction=0.5), w, P.benchmark_parameters(P.MOTION_FLUID)))
    worlds.append((worldgen.random_test_world(74)[0], (64, 64), P.benchmark_parameters(P.MOTION_FLUID)))
    batch = BatchSimulation(worlds)
    batch.calc_timesteps(7)
    for i, (d, w, p) in enumerate(worlds):
        eng = SimulationFacade()
        eng.new_simulation(0, w, p)
        eng.set_simulation_data(d)
        eng.calc_timesteps(7)
        alone = eng.get_simulation_data()
        eng.close_simulation()
        assert np.array_equal(batch.get_simulation_data(i).cells, alone.cells), i
    batch.close()


def test_other_cell_functions_are_rejected():
    data, world = worldgen.random_test_world(80)
    data.cells["cellFunction"][3] = 2  # constructor
    eng = SimulationFacade()
    eng.new_simulation(0, world, P.benchmark_parameters())
    with pytest.raises(AlienError, match="cell function 2"):
        eng.set_simulation_data(data)
    eng.close_simulation()
