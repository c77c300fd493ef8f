"""One-step and multi-step parity of the CUDA engine against the FP64 oracle.

Each case builds a seeded world, runs the engine through its C ABI
(``SimulationFacade`` -> libalien_b200.so) and the oracle from the same
DataTO, and compares the exported state by id.  Tolerance: one step,
|engine - oracle| <= 1e-5 * max(|oracle|, 1) for positions, velocities,
energies, bond rest distances and angles; ids, bond partners (in order),
bond counts, living states and ages must be identical.
"""
import numpy as np
import pytest

from alien_b200 import params as P
from alien_b200 import worldgen
from alien_b200.facade import SimulationFacade
from oracle.oracle import OracleSimulation
from tests.helpers import compare_cells, compare_particles, slot_sets, total_energy

pytestmark = pytest.mark.gpu


def run_both(data, world, prm, steps=1, timestep=0):
    eng = SimulationFacade()
    eng.new_simulation(timestep, world, prm)
    eng.set_simulation_data(data)
    eng.calc_timesteps(steps)
    got = eng.get_simulation_data()
    t_eng = eng.get_current_timestep()
    eng.close_simulation()
    ora = OracleSimulation(world, prm, timestep)
    ora.set_simulation_data(data)
    ora.calc_timesteps(steps)
    ref = ora.get_simulation_data()
    assert t_eng == ora.current_timestep() == timestep + steps
    return got, ref


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("timestep", [0, 1])
def test_fluid_one_step(seed, timestep):
    data, world = worldgen.random_test_world(seed)
    prm = P.benchmark_parameters(P.MOTION_FLUID)
    got, ref = run_both(data, world, prm, 1, timestep)
    compare_cells(got.cells, ref.cells, world, before=data.cells)
    compare_particles(got.particles, ref.particles, world, before=data.particles)


@pytest.mark.parametrize("seed", [4, 5, 6])
@pytest.mark.parametrize("timestep", [0, 2])
def test_collision_one_step(seed, timestep):
    data, world = worldgen.random_test_world(seed, vmax=0.9)
    prm = P.benchmark_parameters(P.MOTION_COLLISION)
    got, ref = run_both(data, world, prm, 1, timestep)
    compare_cells(got.cells, ref.cells, world, before=data.cells)
    compare_particles(got.particles, ref.particles, world, before=data.particles)


def test_barriers_one_step():
    data, world = worldgen.random_test_world(7, barriers=20, free_cells=200)
    prm = P.benchmark_parameters(P.MOTION_FLUID)
    got, ref = run_both(data, world, prm, 1, 0)
    compare_cells(got.cells, ref.cells, world, before=data.cells)
    compare_particles(got.particles, ref.particles, world, before=data.particles)


def test_structural_operations_one_step():
    """dense, fast world: fusion, overstretched bonds, force-decay RNG,
    dying cells (energy below cellMinEnergy) and deletion"""
    data, world = worldgen.random_test_world(8, world=(48, 48), free_cells=400, vmax=1.2, particles=200)
    c = data.cells
    c["energy"][::7] = 20.0          # below cellMinEnergy: dying
    c["livingState"][::11] = 3       # detaching: deleted with cellDeathProbability
    prm = P.benchmark_parameters(P.MOTION_COLLISION)
    for i in range(7):
        prm.cellDeathProbability[i] = 0.5
        prm.cellMaxForce[i] = 0.05
    got, ref = run_both(data, world, prm, 1, 0)
    compare_cells(got.cells, ref.cells, world, before=data.cells)
    compare_particles(got.particles, ref.particles, world, before=data.particles)


def test_cell_map_sets_bit_exact():
    """slot contents of the map built from identical input (order-independent sets)"""
    data, world = worldgen.random_test_world(9, free_cells=600)
    got = slot_sets(data.cells, world)
    ora = OracleSimulation(world, P.benchmark_parameters())
    ora.set_simulation_data(data)
    slots = ora.cell_slots()
    ids = ora.get_simulation_data().cells["id"]
    ref = {}
    for s, i in zip(slots.tolist(), ids.tolist()):
        ref.setdefault(s, set()).add(i)
    assert got == {k: frozenset(v) for k, v in ref.items()}


@pytest.mark.parametrize("motion", [P.MOTION_FLUID, P.MOTION_COLLISION])
def test_multi_step_statistics(motion):
    """30 steps: cell/particle counts and total energy agree; bit-exact run to run."""
    data, world = worldgen.random_test_world(10, world=(96, 96), free_cells=500, particles=300)
    prm = P.benchmark_parameters(motion)
    got, ref = run_both(data, world, prm, 30, 0)
    assert abs(len(got.cells) - len(ref.cells)) <= max(2, len(ref.cells) // 100)
    e0 = total_energy(data)
    assert abs(total_energy(got) - e0) / e0 < 1e-4
    assert abs(total_energy(ref) - e0) / e0 < 1e-6
    eng = SimulationFacade()
    eng.new_simulation(0, world, prm)
    eng.set_simulation_data(data)
    eng.calc_timesteps(30)
    again = eng.get_simulation_data()
    assert np.array_equal(again.cells, got.cells) and np.array_equal(again.particles, got.particles)


@pytest.mark.parametrize("motion", [P.MOTION_FLUID, P.MOTION_COLLISION])
def test_world_too_small_for_regions(motion):
    """7x7 torus: the pair phase reads neighbours from global tile lists"""
    data, world = worldgen.random_test_world(41, world=(7, 7), clusters=0, hex_clusters=0, free_cells=30,
                                             particles=5)
    got, ref = run_both(data, world, P.benchmark_parameters(motion), 1, 0)
    compare_cells(got.cells, ref.cells, world, before=data.cells)
    compare_particles(got.particles, ref.particles, world, before=data.particles)


@pytest.mark.parametrize("motion", [P.MOTION_FLUID, P.MOTION_COLLISION])
def test_region_denser_than_shared_buffer(motion):
    """about 6 cells per slot: a region's halo exceeds the shared buffer"""
    data, world = worldgen.random_test_world(42, world=(16, 16), clusters=0, hex_clusters=0, free_cells=1500,
                                             particles=20, vmax=0.2)
    got, ref = run_both(data, world, P.benchmark_parameters(motion), 1, 1)
    compare_cells(got.cells, ref.cells, world, before=data.cells)
    compare_particles(got.particles, ref.particles, world, before=data.particles)
