"""The facade surface through the C ABI (the reference's DataTransferTests,
EngineTests/DataTransferTests.cpp:19-148, and the _SimulationCudaFacade calls
around the step): exact round trips at small and 1M-cell scale, empty and
particle-only worlds, rectangle selection, timestep and clear, parameter
changes that re-lay out the tile grid, particle storage growth, and rejected
inputs that leave the previous world in place.  Physics after a step is
compared with the FP64 oracle as in test_parity_gpu.py.
"""
import numpy as np
import pytest

from alien_b200 import params as P
from alien_b200 import worldgen
from alien_b200._lib import AlienError
from alien_b200.facade import SimulationFacade
from alien_b200.to import DataTO
from oracle.oracle import OracleSimulation
from tests.helpers import compare_cells, compare_particles, total_energy

pytestmark = pytest.mark.gpu


def facade(world, prm, data=None, timestep=0):
    f = SimulationFacade()
    f.new_simulation(timestep, world, prm)
    if data is not None:
        f.set_simulation_data(data)
    return f


def test_round_trip_exact_with_neurons_and_aux():
    data, world = worldgen.random_test_world(90)
    data = worldgen.add_neurons(data, 90, fraction=0.5)
    f = facade(world, P.benchmark_parameters(), data)
    out = f.get_simulation_data()
    assert np.array_equal(out.cells, data.cells)
    assert np.array_equal(out.particles, data.particles)
    assert np.array_equal(out.aux, data.aux)
    f.close_simulation()


def test_auxiliary_data_survives_rebuilds_with_neurons():
    """neuron weights live only on the device: a parameter change that
    re-lays out the tile grid and a resize both rebuild the arena from a
    download, and the auxiliary bytes come back unchanged"""
    data, world = worldgen.random_test_world(92)
    data = worldgen.add_neurons(data, 92, fraction=0.5)
    f = facade(world, P.benchmark_parameters(), data)
    assert f.get_array_sizes().auxiliaryDataSize == len(data.aux)
    f.calc_timesteps(2)
    p2 = P.benchmark_parameters(P.MOTION_COLLISION)
    p2.cellMaxCollisionDistance = 2.5
    f.set_simulation_parameters(p2)
    f.resize_arrays_if_necessary(particles=4 * f.get_array_sizes().particleArraySize)
    f.calc_timesteps(2)
    out = f.get_simulation_data()
    assert np.array_equal(out.aux, data.aux)
    assert out.num_cells == data.num_cells
    f.close_simulation()


def test_round_trip_exact_at_one_million_cells():
    data, world = worldgen.hex_world(seed=91, world=(2048, 2048), clusters=10000)
    f = facade(world, P.benchmark_parameters(P.MOTION_COLLISION), data)
    out = f.get_simulation_data()
    assert out.num_cells == 1_000_000
    assert np.array_equal(out.cells, data.cells)
    f.close_simulation()


def test_empty_world_steps():
    f = facade((64, 64), P.benchmark_parameters(), DataTO(None, None))
    f.calc_timesteps(10)
    out = f.get_simulation_data()
    assert out.num_cells == 0 and out.num_particles == 0
    st = f.get_raw_statistics()
    assert st.timestep == 10 and st.numCells == 0 and st.numParticles == 0
    f.close_simulation()


def test_particles_only_world_matches_oracle():
    data, world = worldgen.random_test_world(92, clusters=0, hex_clusters=0, free_cells=0, particles=400)
    prm = P.benchmark_parameters()
    f = facade(world, prm, data)
    f.calc_timesteps(3)
    got = f.get_simulation_data()
    f.close_simulation()
    o = OracleSimulation(world, prm)
    o.set_simulation_data(data)
    o.calc_timesteps(3)
    compare_particles(got.particles, o.get_simulation_data().particles, world)


def test_rectangle_selection():
    data, world = worldgen.random_test_world(93, free_cells=300)
    f = facade(world, P.benchmark_parameters(), data)
    out = f.get_simulation_data((10, 12), (40, 50))
    pos = data.cells["pos"]
    inside = (pos[:, 0] >= 10) & (pos[:, 0] <= 40) & (pos[:, 1] >= 12) & (pos[:, 1] <= 50)
    assert set(out.cells["id"].tolist()) == set(data.cells["id"][inside].tolist())
    f.close_simulation()


def test_timestep_and_clear():
    data, world = worldgen.random_test_world(94)
    f = facade(world, P.benchmark_parameters(), data, timestep=5)
    assert f.get_current_timestep() == 5
    f.calc_timesteps(4)
    assert f.get_current_timestep() == 9
    f.set_current_timestep(100)
    assert f.get_current_timestep() == 100
    f.clear()
    out = f.get_simulation_data()
    assert out.num_cells == 0 and out.num_particles == 0
    assert f.get_current_timestep() == 100
    f.close_simulation()


def test_parameter_change_relayouts_and_matches_oracle():
    """fluid (scan radius 2 * 0.8) to collision with a larger radius, midway"""
    data, world = worldgen.random_test_world(95, free_cells=200)
    p1 = P.benchmark_parameters(P.MOTION_FLUID)
    p2 = P.benchmark_parameters(P.MOTION_COLLISION)
    p2.cellMaxCollisionDistance = 2.5
    f = facade(world, p1, data)
    o = OracleSimulation(world, p1)
    o.set_simulation_data(data)
    f.calc_timesteps(2)
    o.calc_timesteps(2)
    f.set_simulation_parameters(p2)
    o.set_simulation_parameters(p2)
    assert f.get_simulation_parameters().cellMaxCollisionDistance == pytest.approx(2.5)
    f.calc_timesteps(1)
    o.calc_timesteps(1)
    got, ref = f.get_simulation_data(), o.get_simulation_data()
    f.close_simulation()
    assert len(got.cells) == len(ref.cells)
    compare_cells(got.cells, ref.cells, world, rtol=1e-4)


def test_particle_storage_grows():
    """every cell dies within a few steps: the particles outgrow the initial
    capacity (cells + particles + 4096) and storage grows between steps"""
    cells = np.concatenate([worldgen.random_test_world(96 + k, world=(128, 128), clusters=0, hex_clusters=0,
                                                      free_cells=3000, particles=0)[0].cells for k in range(3)])
    cells["id"] = np.arange(1, len(cells) + 1, dtype=np.uint64)
    cells["energy"] = 20.0  # below cellMinEnergy: dying
    data = DataTO(cells, None)
    prm = P.benchmark_parameters()
    for c in range(7):
        prm.cellDeathProbability[c] = 1.0
    f = facade((128, 128), prm, data)
    cap0 = f.get_array_sizes().particleArraySize
    f.calc_timesteps(6)
    out = f.get_simulation_data()
    assert out.num_cells == 0
    assert out.num_particles > 0
    assert abs(total_energy(out) - total_energy(data)) / total_energy(data) < 1e-5
    assert f.get_array_sizes().particleArraySize >= cap0
    f.close_simulation()


def test_rejected_input_keeps_previous_world():
    data, world = worldgen.random_test_world(97)
    f = facade(world, P.benchmark_parameters(), data)
    bad = DataTO(data.cells.copy(), data.particles)
    bad.cells["connections"]["cellIndex"][0, 0] = len(bad.cells) + 5
    bad.cells["numConnections"][0] = max(1, bad.cells["numConnections"][0])
    with pytest.raises(AlienError, match="cellIndex out of range"):
        f.set_simulation_data(bad)
    out = f.get_simulation_data()
    assert np.array_equal(out.cells, data.cells)
    f.calc_timesteps(1)
    f.close_simulation()


def test_resize_arrays_if_necessary_adds_particle_room():
    data, world = worldgen.random_test_world(98)
    f = facade(world, P.benchmark_parameters(), data)
    before = f.get_array_sizes().particleArraySize
    f.resize_arrays_if_necessary(particles=before * 4)
    assert f.get_array_sizes().particleArraySize > before
    out = f.get_simulation_data()
    assert np.array_equal(out.cells, data.cells)
    f.close_simulation()
