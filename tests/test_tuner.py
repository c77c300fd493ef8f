"""The pair kernel's launch configuration and its autotuner.

The pair kernel works on regions of tiles, one CTA each; the region shape
is one of six candidates per motion type.  A cell's neighbours are visited
in the same order whatever the shape, so the shape must change no result:
worlds stepped with every fixed shape and with the autotuner's choice must
agree bit for bit (cells, bonds and particles).  The autotuner's choice
rule is a pure host function, checked on the CPU.
"""
import ctypes

import numpy as np
import pytest

from alien_b200 import _lib
from alien_b200 import params as P
from alien_b200 import worldgen


def choose(ms):
    lib = _lib.load()
    arr = (ctypes.c_float * max(len(ms), 1))(*ms)
    return lib.alien_b200_choose_region(arr, len(ms))


def test_choice_rule():
    assert choose([1.0, 0.9, 0.95, 1.2]) == 1
    assert choose([1.0, 0.99, 0.985, 0.5]) == 3
    # within 2 % of an earlier candidate: the earlier one stays
    assert choose([1.0, 0.99, 1.0, 1.0]) == 0
    assert choose([1.0, 0.97, 0.96, 0.955]) == 1
    # nothing measured: the default (first) candidate
    assert choose([0.0, 0.0, 0.0, 0.0]) == 0
    assert choose([-1.0, 2.0, 0.0, 0.0]) == 1
    assert choose([]) == 0


def _run(data, world, prm, steps, fluid_choice=0, collision_choice=0):
    from alien_b200.facade import SimulationFacade

    eng = SimulationFacade()
    eng.new_simulation(0, world, prm)
    eng.set_region_choice(fluid_choice, collision_choice)
    eng.set_simulation_data(data)
    eng.calc_timesteps(steps)
    out = eng.get_simulation_data()
    cfg = eng.launch_config()
    eng.close_simulation()
    return out, cfg


@pytest.mark.gpu
@pytest.mark.parametrize("motion", [P.MOTION_FLUID, P.MOTION_COLLISION])
def test_results_do_not_depend_on_region_shape(motion):
    data, world = worldgen.random_test_world(51, world=(160, 160), free_cells=2000, particles=200, vmax=0.9,
                                             barriers=6)
    prm = P.benchmark_parameters(motion)
    tuned, cfg = _run(data, world, prm, 4)
    assert cfg.tuned == 1
    assert 0 <= cfg.regionChoice[motion] < _lib.REGION_CHOICES
    assert all(cfg.tunedMs[motion][i] > 0 for i in range(_lib.REGION_CHOICES))
    for i in range(_lib.REGION_CHOICES):
        fixed, fcfg = _run(data, world, prm, 4, i + 1, i + 1)
        shape = tuple(fcfg.candidates[motion][i])
        assert fcfg.regionChoice[motion] == i and tuple(fcfg.regionTiles[motion]) == shape
        assert np.array_equal(fixed.cells, tuned.cells), f"cells differ with regions of {shape} tiles"
        assert np.array_equal(fixed.particles, tuned.particles), f"particles differ with regions of {shape} tiles"


@pytest.mark.gpu
def test_dense_rows_and_small_worlds_do_not_depend_on_region_shape():
    """regions denser than the shared buffer and worlds too small for
    regions defer cells to the overflow kernel; results stay identical"""
    for world_size, cells in (((16, 16), 1500), ((7, 7), 30)):
        data, world = worldgen.random_test_world(52, world=world_size, clusters=0, hex_clusters=0, free_cells=cells,
                                                 particles=10, vmax=0.2)
        for motion in (P.MOTION_FLUID, P.MOTION_COLLISION):
            prm = P.benchmark_parameters(motion)
            ref, _ = _run(data, world, prm, 2, 1, 1)
            got, _ = _run(data, world, prm, 2, 4, 4)
            assert np.array_equal(ref.cells, got.cells) and np.array_equal(ref.particles, got.particles)
