"""CPU tests of the oracle (the checker) against the reference's own known
answers for this path, restated at the DataTO level, and of its
invariants.  No GPU needed."""
import numpy as np
import pytest

from alien_b200 import params as P
from alien_b200 import worldgen
from alien_b200.to import DataTO, empty_cells
from oracle.oracle import OracleSimulation
from tests.helpers import topology, total_energy


def decay_world():
    """CellConnectionTests.decay (EngineTests/CellConnectionTests.cpp:19-37):
    a 10x10 rect (createRect, centred at the origin) with energy
    cellMinEnergy/2 in a 1000x1000 world (IntegrationTestFramework.cpp:11-21)"""
    tmpl = worldgen.rect_template()
    cells = worldgen._clusters_to_cells(tmpl, np.zeros((1, 2)), np.zeros((1, 2)), np.zeros(1), 25.0, 1, (1000, 1000))
    prm = P.benchmark_parameters()
    prm.radiationAbsorption[0] = 0.0
    prm.cellDeathConsequences = 1  # CellDeathConsquences_CreatureDies
    prm.cellDeathProbability[0] = 0.5
    return DataTO(cells), (1000, 1000), prm


def approx_compare(expected, actual, precision=1e-3):
    """IntegrationTestFramework::approxCompare (IntegrationTestFramework.cpp:108-115)"""
    norm = abs(expected) + abs(actual)
    return norm < precision or abs(expected - actual) / norm < precision


def test_decay_known_answer():
    data, world, prm = decay_world()
    o = OracleSimulation(world, prm)
    o.set_simulation_data(data)
    for _ in range(1000):
        o.calc_timesteps(1)
    out = o.get_simulation_data()
    assert out.num_cells == 0
    assert 0 < out.num_particles <= 100  # energy particles of deleted cells, some merged
    assert approx_compare(total_energy(out), total_energy(data))


def test_data_round_trip_exact():
    """DataTransferTests.singleCell/singleParticle/cellCluster
    (EngineTests/DataTransferTests.cpp:19-103): set then get returns the
    same transfer objects"""
    data, world = worldgen.random_test_world(3)
    data.cells["cellFunction"][:5] = 0          # neurons: weights in auxiliary data
    data.cells["cellFunctionData"][:5, 0] = np.arange(5) * 288
    aux = np.arange(5 * 288, dtype=np.uint8)
    data = DataTO(data.cells, data.particles, aux)
    o = OracleSimulation(world, P.benchmark_parameters())
    o.set_simulation_data(data)
    out = o.get_simulation_data()
    assert np.array_equal(out.cells, data.cells)
    assert np.array_equal(out.particles, data.particles)
    assert np.array_equal(out.aux, data.aux)


@pytest.mark.parametrize("motion", [P.MOTION_FLUID, P.MOTION_COLLISION])
def test_deterministic_and_energy_conserving(motion):
    data, world = worldgen.random_test_world(11, free_cells=300, particles=200)
    prm = P.benchmark_parameters(motion)
    runs = []
    for _ in range(2):
        o = OracleSimulation(world, prm)
        o.set_simulation_data(data)
        o.calc_timesteps(40)
        runs.append(o.get_simulation_data())
    assert np.array_equal(runs[0].cells, runs[1].cells)
    assert np.array_equal(runs[0].particles, runs[1].particles)
    e0 = total_energy(data)
    assert abs(total_energy(runs[0]) - e0) / e0 < 1e-6


def test_bonds_stay_symmetric_and_angles_sum_to_360():
    data, world = worldgen.random_test_world(12, world=(48, 48), free_cells=400, vmax=1.2)
    prm = P.benchmark_parameters(P.MOTION_COLLISION)
    o = OracleSimulation(world, prm)
    o.set_simulation_data(data)
    o.calc_timesteps(25)
    out = o.get_simulation_data()
    topo = topology(out.cells)
    assert all((b, a) in topo for a, b in topo)
    c = out.cells
    for i in range(len(c)):
        n = int(c["numConnections"][i])
        if n:
            assert abs(float(np.sum(c["connections"]["angleFromPrevious"][i, :n], dtype=np.float64)) - 360.0) < 1e-2


def test_fusion_creates_bonds():
    """two free cells approaching faster than cellFusionVelocity bond"""
    cells = empty_cells(2)
    cells["id"] = [1, 2]
    cells["pos"] = [[10.0, 10.0], [11.0, 10.0]]
    cells["vel"] = [[0.4, 0.0], [-0.4, 0.0]]
    cells["maxConnections"] = 6
    for motion in (P.MOTION_FLUID, P.MOTION_COLLISION):
        o = OracleSimulation((32, 32), P.benchmark_parameters(motion))
        o.set_simulation_data(DataTO(cells))
        o.calc_timesteps(1)
        out = o.get_simulation_data()
        assert topology(out.cells) == {(1, 2), (2, 1)}, motion


def test_overstretched_bond_breaks_and_detaches():
    tmpl = worldgen.rect_template()
    cells = worldgen._clusters_to_cells(tmpl, np.array([[20.0, 20.0]]), np.zeros((1, 2)), np.zeros(1), 100.0, 1, (64, 64))
    cells["pos"][0] += np.array([0.0, -8.0], np.float32)  # corner cell beyond cellMaxBindingDistance of its partners
    o = OracleSimulation((64, 64), P.benchmark_parameters())
    o.set_simulation_data(DataTO(cells))
    o.calc_timesteps(1)
    out = o.get_simulation_data()
    first = out.cells[out.cells["id"] == 1][0]
    assert first["numConnections"] == 0
    # its former partners detach (checkConnections, CellProcessor.cuh:515-520)
    assert set(out.cells["livingState"][np.isin(out.cells["id"], [2, 11])]) == {3}


def test_particle_absorbed_by_cell():
    cells = empty_cells(1)
    cells["id"] = 1
    cells["pos"] = [[10.5, 10.5]]
    from alien_b200.to import PARTICLE_TO
    p = np.zeros(1, PARTICLE_TO)
    p["id"] = 2
    p["pos"] = [[8.5, 10.5]]  # moves to 9.5; the cell at floor(pos + vel) absorbs it
    p["vel"] = [[1.0, 0.0]]
    p["energy"] = 3.0
    o = OracleSimulation((32, 32), P.benchmark_parameters())
    o.set_simulation_data(DataTO(cells, p))
    o.calc_timesteps(1)
    out = o.get_simulation_data()
    assert out.num_particles == 0
    assert abs(float(out.cells["energy"][0]) - 103.0) < 1e-5
