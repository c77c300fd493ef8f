"""The pair kernel's launch configuration and its autotuner.

The pair kernel splits each cell's neighbour candidates across a group of
2, 4, 8 or 16 lanes and sums in fixed point, so the lane count must change
no result: worlds stepped with every fixed lane count and with the
autotuner's choice must agree bit for bit (cells, bonds and particles).
The autotuner's choice rule is a pure host function, checked on the CPU.
"""
import ctypes

import numpy as np
import pytest

from alien_b200 import _lib
from alien_b200 import params as P
from alien_b200 import worldgen


def choose(ms):
    lib = _lib.load()
    arr = (ctypes.c_float * len(ms))(*ms)
    return lib.alien_b200_choose_pair_lanes(arr, len(ms))


def test_choice_rule():
    assert choose([1.0, 0.9, 0.95, 1.2]) == 4
    assert choose([1.0, 0.99, 0.985, 0.5]) == 16
    # within 2 % of a smaller lane count: the smaller one stays
    assert choose([1.0, 0.99, 1.0, 1.0]) == 2
    assert choose([1.0, 0.97, 0.96, 0.955]) == 4
    # nothing measured: the default
    assert choose([0.0, 0.0, 0.0, 0.0]) == 4
    assert choose([-1.0, 2.0, 0.0, 0.0]) == 4
    assert choose([]) == 4


def _run(data, world, prm, steps, fluid_lanes=0, collision_lanes=0):
    from alien_b200.facade import SimulationFacade

    eng = SimulationFacade()
    eng.new_simulation(0, world, prm)
    eng.set_pair_lanes(fluid_lanes, collision_lanes)
    eng.set_simulation_data(data)
    eng.calc_timesteps(steps)
    out = eng.get_simulation_data()
    cfg = eng.launch_config()
    eng.close_simulation()
    return out, cfg


@pytest.mark.gpu
@pytest.mark.parametrize("motion", [P.MOTION_FLUID, P.MOTION_COLLISION])
def test_results_do_not_depend_on_lanes(motion):
    data, world = worldgen.random_test_world(51, world=(96, 96), free_cells=800, particles=200, vmax=0.9,
                                             barriers=6)
    prm = P.benchmark_parameters(motion)
    tuned, cfg = _run(data, world, prm, 4)
    assert cfg.tuned == 1
    assert cfg.pairLanes[motion] in _lib.PAIR_LANE_CHOICES
    assert all(cfg.tunedMs[motion][i] > 0 for i in range(len(_lib.PAIR_LANE_CHOICES)))
    for lanes in _lib.PAIR_LANE_CHOICES:
        fixed, fcfg = _run(data, world, prm, 4, lanes, lanes)
        assert fcfg.pairLanes[motion] == lanes and fcfg.pairLanesFixed[motion] == lanes
        assert np.array_equal(fixed.cells, tuned.cells), f"cells differ with {lanes} lanes per cell"
        assert np.array_equal(fixed.particles, tuned.particles), f"particles differ with {lanes} lanes per cell"


@pytest.mark.gpu
def test_dense_rows_and_small_worlds_do_not_depend_on_lanes():
    """regions denser than the shared buffer and worlds too small for
    regions defer cells to the overflow kernel; results stay identical"""
    for world_size, cells in (((16, 16), 1500), ((7, 7), 30)):
        data, world = worldgen.random_test_world(52, world=world_size, clusters=0, hex_clusters=0, free_cells=cells,
                                                 particles=10, vmax=0.2)
        for motion in (P.MOTION_FLUID, P.MOTION_COLLISION):
            prm = P.benchmark_parameters(motion)
            ref, _ = _run(data, world, prm, 2, 2, 2)
            got, _ = _run(data, world, prm, 2, 16, 16)
            assert np.array_equal(ref.cells, got.cells) and np.array_equal(ref.particles, got.particles)
