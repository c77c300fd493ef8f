"""The density map (DensityMap.cuh:8-230).

CPU: the restatement in oracle/density_map.py against the reference engine's
own maps after one step (tests/golden/ref_density_*.npz, written by
tests/golden/make_golden.py from oracle/_ref/ref_run), and against small
hand-made cases (byte-lane carries, truncation, the flattened index check).

GPU: the engine's map (alien_b200_get_density_map) against the reference's
maps and against the restatement, alone, in a batch and in a live arena.
"""
import os

import numpy as np
import pytest

from alien_b200 import params as P
from alien_b200 import worldgen
from alien_b200.to import DataTO
from oracle import density_map as dm

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = ["density_collision_t47", "density_fluid_t70"]


def fixture(name):
    f = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    seed, motion, t, W, H, ts = (int(v) for v in f["meta"])
    return f, (W, H), t, motion


def assert_maps_equal(got, want, label=""):
    for k in dm.FIELDS:
        assert got[k].shape == want[k].shape, (label, k)
        assert np.array_equal(got[k], want[k]), f"{label}: {k} differs in {np.count_nonzero(got[k] != want[k])} slots"


@pytest.mark.parametrize("name", FIXTURES)
def test_restatement_matches_reference_maps(name):
    f, world, t, _ = fixture(name)
    want = {k: f["map_" + k] for k in dm.FIELDS}
    assert_maps_equal(dm.from_cells(f["in_cells"], world, t), want, name)
    # the fixture reaches every branch of addCell
    c = f["in_cells"]
    assert (c["mutationId"] == 0).any() and (c["mutationId"] == 1).any() and (c["mutationId"] > 1).any()
    buckets = 32 - dm._clz32(np.trunc(c["genomeComplexity"] * np.float32(10)).astype(np.int64))
    assert (buckets < 8).any() and ((buckets >= 8) & (buckets < 16)).any() and (buckets >= 16).any()


def test_byte_lanes_carry_and_index_rules():
    # 300 cells of color 2 in slot (1, 0): the color byte carries into byte 3
    pos = np.tile(np.array([[9.5, 3.0]], np.float32), (300, 1))
    m = dm.density_map(pos, np.full(300, 2), np.zeros(300, np.uint32), np.zeros(300, np.float32), (32, 16), 0)
    assert int(m["color"][0, 1]) == 300 * ((1 << 16) | (1 << 56)) % (1 << 64)
    assert int(m["specificMutant"][0, 1]) == 300
    # x beyond the last full slot column wraps into the next row through the
    # flattened index (world 20 wide: 2 columns; x = 17 gives column 2)
    m = dm.density_map(np.array([[17.0, 1.0], [17.0, 15.0], [-0.5, 2.0]], np.float32), np.zeros(3, int),
                       np.zeros(3, np.uint32), np.zeros(3, np.float32), (20, 16), 0)
    assert int(m["specificMutant"][1, 0]) == 1  # index 2 = (x 0, y 1)
    assert int(m["specificMutant"][0, 0]) == 1  # -0.5 truncates to 0
    assert int(m["specificMutant"].sum()) == 2  # index 2 + 1 * 2 = 4 is past the map
    # genome complexity buckets: 0 -> bucket 0, 12.8 -> 128 -> bucket 8, 7000 -> 70000 -> bucket 17 (none)
    m = dm.density_map(np.array([[1.0, 1.0]] * 3, np.float32), np.zeros(3, int), np.array([2, 2, 2], np.uint32),
                       np.array([0.0, 12.8, 7000.0], np.float32), (8, 8), 0)
    lanes = 0x0101010101010101
    assert int(m["lessComplexity1"][0, 0]) == lanes
    assert int(m["lessComplexity2"][0, 0]) == lanes + lanes
    assert int(m["moreComplexity1"][0, 0]) == 1 + lanes
    assert int(m["moreComplexity2"][0, 0]) == 1  # bucket 8: byte lanes 0..0


# ------------------------------------------------------------------ GPU --


def engine_map(data, world, prm, steps, timestep=0):
    from alien_b200.facade import SimulationFacade
    s = SimulationFacade()
    s.new_simulation(timestep, world, prm)
    s.set_simulation_data(data)
    if steps:
        s.calc_timesteps(steps)
    m = s.get_density_map()
    out = s.get_simulation_data()
    s.close_simulation()
    return m, out


@pytest.mark.gpu
@pytest.mark.parametrize("name", FIXTURES)
def test_engine_matches_reference_maps(name):
    f, world, t, motion = fixture(name)
    data = DataTO(f["in_cells"].copy(), f["in_particles"].copy())
    prm = P.benchmark_parameters(motion)
    m, _ = engine_map(data, world, prm, 1, timestep=t)
    assert_maps_equal(m, {k: f["map_" + k] for k in dm.FIELDS}, name)


@pytest.mark.gpu
def test_engine_map_before_and_after_steps():
    """before any step: the set positions at the current timestep; after k
    steps: the positions the k-th step started from (what get_data returned
    after k - 1 steps) at timestep t0 + k - 1"""
    import tests.golden.make_golden as mg
    data, world = mg.density_world(43)
    prm = P.benchmark_parameters(P.MOTION_COLLISION)
    t0 = 45
    m, _ = engine_map(data, world, prm, 0, timestep=t0)
    assert_maps_equal(m, dm.from_cells(data.cells, world, t0), "no step")
    for k in (2, 5):
        _, before = engine_map(data, world, prm, k - 1, timestep=t0)
        m, _ = engine_map(data, world, prm, k, timestep=t0)
        assert_maps_equal(m, dm.from_cells(before.cells, world, t0 + k - 1), f"{k} steps")


@pytest.mark.gpu
def test_engine_map_of_a_world_not_a_multiple_of_the_slot():
    data, world = worldgen.random_test_world(44, world=(100, 60), free_cells=400, particles=0)
    rng = np.random.default_rng(44)
    data.cells["mutationId"] = rng.integers(0, 40, data.num_cells).astype(np.uint32)
    data.cells["genomeComplexity"] = rng.uniform(0, 20, data.num_cells).astype(np.float32)
    m, _ = engine_map(data, world, P.benchmark_parameters(P.MOTION_FLUID), 0, timestep=3)
    assert m["color"].shape == (7, 12)
    assert_maps_equal(m, dm.from_cells(data.cells, world, 3), "100 x 60")


@pytest.mark.gpu
def test_batch_and_live_arena_maps_equal_alone():
    import tests.golden.make_golden as mg
    import tests.test_batch_gpu as tb
    from alien_b200.facade import BatchSimulation, LiveArena
    specs = [mg.density_world(45) + (P.benchmark_parameters(P.MOTION_COLLISION),),
             mg.density_world(46) + (P.benchmark_parameters(P.MOTION_FLUID),)]
    alone = [engine_map(d, w, p, 3)[0] for d, w, p in specs]
    batch = BatchSimulation(specs)
    batch.calc_timesteps(3)
    arena = LiveArena(tb.small_capacity())
    slots = [arena.admit(*spec) for spec in specs]
    arena.calc_timesteps(3)
    for w, want in enumerate(alone):
        assert_maps_equal(batch.get_density_map(w), want, f"batch {w}")
        assert_maps_equal(arena.get_density_map(slots[w]), want, f"live {w}")
    batch.close()
    arena.close()
