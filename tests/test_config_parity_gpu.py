"""Parity of the CUDA engine with the FP64 oracle on the benchmark worlds
themselves, on the engine's own cell map, and on the parts of the step that
the default parameters leave off (radiation emission, particle splitting).

* One step of each benchmark world at full size: the 512x512 soft-body world
  (20k lattice cells, 20k energy particles, fluid motion), the 1M-cell SPH
  fluid world (2048x2048) and the 4M-cell hexagonal soft-body world
  (4096x4096, collision motion, bond breaking on).  These exercise the pair
  kernel's paths that small worlds never reach (bands of dense regions, the
  per-motion region shapes, thousands of regions per launch).  Bar: ids,
  bond partners in order, bond counts, living states and ages identical;
  positions, velocities, energies, bond rest lengths and angles within
  |engine - oracle| <= 1e-5 * max(|oracle|, 1) (tests/helpers.py).  The
  oracle is the multithreaded FP64 build (per-cell gathers; only the order
  of its FP64 angle-force additions depends on the thread count).
* The cell map: the engine bins the input state with its step kernels and
  returns the map (alien_b200_debug_cell_map); per slot, the set of cell
  ids must equal the oracle's (Map.cuh:95-130, order independent), every
  record must lie in the tile of its slot, tiles in ascending order, and a
  cell's "visible" flag (among the first 10 cells of its slot in storage
  order, Map.cuh:117-125) and "head" flag (first of its slot) must match
  the storage-order ranks exactly.
* Radiation (CellProcessor::radiation, CellProcessor.cuh:725-773) with the
  reference's default age strength and a high-energy factor, and particle
  splitting (RadiationProcessor::splitting, RadiationProcessor.cuh:172-204)
  with a finite split energy: the new particles' ids must be identical and
  their values within the same tolerance.
* get_raw_statistics of the engine against counts and FP64 energy sums of
  the oracle's state after the same steps.
"""
import numpy as np
import pytest

from alien_b200 import params as P
from alien_b200 import worldgen
from alien_b200.facade import SimulationFacade
from oracle.oracle import OracleSimulation
from tests.helpers import compare_cells, compare_particles

pytestmark = pytest.mark.gpu


def run_both(data, world, prm, steps=1, timestep=0, precision="f64mt"):
    eng = SimulationFacade()
    eng.new_simulation(timestep, world, prm)
    eng.set_simulation_data(data)
    eng.calc_timesteps(steps)
    got = eng.get_simulation_data()
    stats = eng.get_raw_statistics()
    eng.close_simulation()
    ora = OracleSimulation(world, prm, timestep, precision=precision)
    ora.set_simulation_data(data)
    ora.calc_timesteps(steps)
    ref = ora.get_simulation_data()
    ora.close()
    return got, ref, stats


CONFIGS = {
    # name: (generator, motion)
    "softbody": (lambda: worldgen.soft_body_world(seed=0), P.MOTION_FLUID),
    "fluid1m": (lambda: worldgen.fluid_world(seed=0), P.MOTION_FLUID),
    "hex4m": (lambda: worldgen.hex_world(seed=0), P.MOTION_COLLISION),
}
_WORLDS = {}


def config_world(name):
    if name not in _WORLDS:
        _WORLDS[name] = CONFIGS[name][0]()
    return _WORLDS[name]


@pytest.mark.parametrize("name,timestep", [("softbody", 0), ("softbody", 1), ("fluid1m", 0), ("fluid1m", 1),
                                           ("hex4m", 0), ("hex4m", 1)])
def test_benchmark_world_one_step(name, timestep):
    """timestep 0: angle forces and inner friction on; timestep 1: off (the
    position update runs inside the first bond-force kernel)"""
    data, world = config_world(name)
    prm = P.benchmark_parameters(CONFIGS[name][1])
    got, ref, _ = run_both(data, world, prm, 1, timestep)
    errs = compare_cells(got.cells, ref.cells, world, before=data.cells)
    errs.update(compare_particles(got.particles, ref.particles, world, before=data.particles))
    print(f"{name} t={timestep}: {len(got.cells)} cells, {len(got.particles)} particles, "
          + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))


def _assert_map_matches(data, world, prm):
    eng = SimulationFacade()
    eng.new_simulation(0, world, prm)
    eng.set_simulation_data(data)
    ids, slots, tiles, flags = eng.debug_cell_map()
    eng.close_simulation()
    cells = data.cells
    assert len(ids) == len(cells)
    # the oracle's map of the same input (slot of every cell, storage order)
    ora = OracleSimulation(world, prm, precision="f64mt")
    ora.set_simulation_data(data)
    oslots = ora.cell_slots().astype(np.int64)
    ora.close()
    W, H = world
    # tile geometry: tiles of ceil(interaction radius) slots, row-major
    R = prm.smoothingLength * 2 if prm.motionType == P.MOTION_FLUID else prm.cellMaxCollisionDistance
    T = max(1, int(np.ceil(np.float32(R))))
    nTX = -(-W // T)
    s = slots.astype(np.int64)
    assert np.array_equal(tiles.astype(np.int64), (s % W) // T + ((s // W) // T) * nTX), "record outside its slot's tile"
    assert np.all(np.diff(tiles.astype(np.int64)) >= 0), "map records not grouped by tile"
    # per-slot id sets, order independent
    id_of = cells["id"].astype(np.uint64)
    eng_pairs = np.stack([s, ids.astype(np.int64)], 1)
    ora_pairs = np.stack([oslots, id_of.astype(np.int64)], 1)
    eng_pairs = eng_pairs[np.lexsort((eng_pairs[:, 1], eng_pairs[:, 0]))]
    ora_pairs = ora_pairs[np.lexsort((ora_pairs[:, 1], ora_pairs[:, 0]))]
    assert np.array_equal(eng_pairs, ora_pairs), "cell-map slot sets differ from the oracle's"
    # visibility and head flags from the storage-order rank within the slot
    by_id = np.argsort(id_of, kind="stable")
    order = by_id[np.searchsorted(id_of[by_id], ids)].astype(np.int64)  # storage index of each record
    by = np.lexsort((order, s))
    ss, so = s[by], order[by]
    start = np.r_[0, np.nonzero(np.diff(ss))[0] + 1]
    rank = np.arange(len(ss)) - np.repeat(start, np.diff(np.r_[start, len(ss)]))
    want_visible = np.zeros(len(ids), bool)
    want_head = np.zeros(len(ids), bool)
    want_visible[by] = rank < 10
    want_head[by] = rank == 0
    assert np.array_equal((flags & 2) != 0, want_visible), "visible flags differ from the storage-order ranks"
    assert np.array_equal((flags & 4) != 0, want_head), "slot-head flags differ from the storage-order ranks"
    assert np.array_equal((flags & 1) != 0, cells["barrier"][order] != 0)
    return int(np.max(np.bincount(s)))


@pytest.mark.parametrize("motion", [P.MOTION_FLUID, P.MOTION_COLLISION])
def test_engine_cell_map_matches_oracle(motion):
    data, world = worldgen.random_test_world(9, free_cells=600, barriers=12)
    _assert_map_matches(data, world, P.benchmark_parameters(motion))


def test_engine_cell_map_dense_slots():
    """more than 10 cells in some slots: only the first 10 in storage order
    are visible to the pair scans"""
    data, world = worldgen.random_test_world(43, world=(16, 16), clusters=0, hex_clusters=0, free_cells=900,
                                             particles=0)
    rng = np.random.default_rng(43)
    c = data.cells
    c["pos"][:120] = (np.array([3.5, 7.5]) + rng.uniform(-0.45, 0.45, (120, 2))).astype(np.float32)
    most = _assert_map_matches(data, world, P.benchmark_parameters(P.MOTION_FLUID))
    assert most > 10


@pytest.mark.parametrize("name", ["fluid1m", "hex4m"])
def test_engine_cell_map_benchmark_worlds(name):
    data, world = config_world(name)
    _assert_map_matches(data, world, P.benchmark_parameters(CONFIGS[name][1]))


def _radiation_world(seed):
    data, world = worldgen.random_test_world(seed, free_cells=400, particles=100)
    rng = np.random.default_rng(seed)
    data.cells["age"] = rng.integers(0, 200, len(data.cells)).astype(np.uint32)
    return data, world


@pytest.mark.parametrize("motion", [P.MOTION_FLUID, P.MOTION_COLLISION])
@pytest.mark.parametrize("steps", [1, 3])
def test_radiation_emission(motion, steps):
    """the reference's default radiation (age strength 2e-5, probability
    0.03) plus a high-energy factor for cells above 90 energy units"""
    data, world = _radiation_world(31)
    prm = P.default_parameters()
    prm.motionType = motion
    for c in range(P.MAX_COLORS):
        prm.highRadiationFactor[c] = 0.002
        prm.highRadiationMinCellEnergy[c] = 90.0
        prm.radiationMinCellAge[c] = 50
    got, ref, _ = run_both(data, world, prm, steps, 0, precision="f64")
    new_ids = ref.particles["id"] > max(int(data.cells["id"].max()), int(data.particles["id"].max()))
    assert np.count_nonzero(new_ids) > 0, "no radiation particle was emitted"
    compare_cells(got.cells, ref.cells, world, before=data.cells)
    compare_particles(got.particles, ref.particles, world, before=data.particles)


@pytest.mark.parametrize("steps", [1, 4])
def test_particle_splitting(steps):
    """particles above the split energy split with probability 0.01 per step"""
    data, world = worldgen.random_test_world(32, free_cells=100, particles=3000)
    data.particles["energy"] = np.random.default_rng(32).uniform(0.5, 6.0, len(data.particles)).astype(np.float32)
    prm = P.benchmark_parameters(P.MOTION_FLUID)
    for c in range(P.MAX_COLORS):
        prm.particleSplitEnergy[c] = 2.0
    got, ref, _ = run_both(data, world, prm, steps, 0, precision="f64")
    new_ids = ref.particles["id"] > max(int(data.cells["id"].max()), int(data.particles["id"].max()))
    assert np.count_nonzero(new_ids) > 0, "no particle split"
    compare_cells(got.cells, ref.cells, world, before=data.cells)
    compare_particles(got.particles, ref.particles, world, before=data.particles)


@pytest.mark.parametrize("motion", [P.MOTION_FLUID, P.MOTION_COLLISION])
def test_statistics_match_oracle(motion):
    """getRawStatistics after 5 steps (structural operations and decay on):
    counts exact, energies within the one-step tolerance of the state"""
    data, world = worldgen.random_test_world(33, world=(48, 48), free_cells=400, vmax=1.2, particles=200)
    c = data.cells
    c["energy"][::9] = 20.0
    prm = P.default_parameters()
    prm.motionType = motion
    for i in range(P.MAX_COLORS):
        prm.cellDeathProbability[i] = 0.3
    got, ref, stats = run_both(data, world, prm, 5, 0, precision="f64")
    cells, parts = ref.cells, ref.particles
    assert stats.timestep == 5
    assert stats.numCells == len(cells) and stats.numParticles == len(parts)
    assert stats.numConnections == int(np.sum(cells["numConnections"]))
    assert list(stats.numCellsByColor) == np.bincount(cells["color"] % 7, minlength=7).tolist()
    ce = float(np.sum(cells["energy"], dtype=np.float64))
    pe = float(np.sum(parts["energy"], dtype=np.float64))
    assert abs(stats.totalCellEnergy - ce) <= 1e-5 * max(ce, 1.0)
    assert abs(stats.totalParticleEnergy - pe) <= 1e-5 * max(pe, 1.0)


def _expected_statistics(data, neuron_activities):
    """RawStatisticsData of a state, computed from its transfer objects
    (StatisticsKernels.cu:12-46, 73-105)"""
    cells, parts = data.cells, data.particles
    col = cells["color"].astype(np.int64) % 7
    pcol = parts["color"].astype(np.int64) % 7
    energy = np.zeros(7)
    np.add.at(energy, col, cells["energy"].astype(np.float64))
    np.add.at(energy, pcol, parts["energy"].astype(np.float64))
    ages = cells["age"].astype(np.int64)
    live = cells["barrier"] == 0
    max_age = int(ages[live].max()) if np.any(live) else 0
    hist = np.zeros((7, 20), np.int64)
    np.add.at(hist, (col[live], ages[live] * 20 // (max_age + 1)), 1)
    return {
        "numCells": np.bincount(col, minlength=7),
        "numFreeCells": np.bincount(col[cells["mutationId"] == 1], minlength=7),
        "numParticles": np.bincount(pcol, minlength=7),
        "totalEnergy": energy,
        "maxValue": max_age,
        "histogram": hist,
        "numNeuronActivities": np.asarray(neuron_activities, np.int64),
    }


@pytest.mark.parametrize("motion", [P.MOTION_FLUID, P.MOTION_COLLISION])
def test_raw_statistics_data_match_oracle(motion):
    """the full RawStatisticsData after 13 steps of a world with neuron
    cells, free cells (mutation id 1), barriers, decaying cells and energy
    particles: counts, histogram and neuron activities exact, energies per
    color within the one-step tolerance of the state"""
    data, world = worldgen.calm_test_world(61)
    data = worldgen.add_neurons(data, 61, fraction=0.5)
    rng = np.random.default_rng(61)
    c = data.cells
    c["mutationId"] = np.where(rng.random(len(c)) < 0.3, 1, 7).astype(np.uint32)
    c["age"] = rng.integers(0, 500, len(c)).astype(np.uint32)
    c["color"] = rng.integers(0, 7, len(c)).astype(np.uint8)
    c["energy"][::13] = 30.0
    c["barrier"][5:8] = 1
    prm = P.benchmark_parameters(motion)
    for i in range(P.MAX_COLORS):
        prm.cellDeathProbability[i] = 0.2
    steps = 13
    eng = SimulationFacade()
    eng.new_simulation(0, world, prm)
    eng.set_simulation_data(data)
    eng.calc_timesteps(steps)
    got = eng.get_raw_statistics_data()
    ora = OracleSimulation(world, prm, precision="f64")
    ora.set_simulation_data(data)
    ora.calc_timesteps(steps)
    want = _expected_statistics(ora.get_simulation_data(), ora.neuron_activities())
    ts = got.timeline.timestep
    for field in ("numCells", "numFreeCells", "numParticles"):
        assert list(getattr(ts, field)) == want[field].tolist(), field
    assert np.sum(want["numFreeCells"]) > 0 and np.sum(want["numParticles"]) > 0
    e = np.array(list(ts.totalEnergy), np.float64)
    assert np.all(np.abs(e - want["totalEnergy"]) <= 1e-5 * np.maximum(want["totalEnergy"], 1.0))
    assert got.histogram.maxValue == want["maxValue"]
    assert np.array_equal(np.array([list(r) for r in got.histogram.numCellsByColorBySlot]), want["histogram"])
    acc = np.array(list(got.timeline.accumulated.numNeuronActivities), np.int64)
    assert np.array_equal(acc, want["numNeuronActivities"]) and acc.sum() > 0
    for field in ("numSelfReplicators", "numColonies", "numViruses"):
        assert list(getattr(ts, field)) == [0] * 7
    eng.reset_time_interval_statistics()
    assert list(eng.get_raw_statistics_data().timeline.accumulated.numNeuronActivities) == [0] * 7
    eng.close_simulation()
