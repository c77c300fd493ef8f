"""The reference's .settings.json format for the physics-stage parameters
(AuxiliaryDataParserService.cpp, ParameterParser.h): the reader against the
general settings and physics keys of the reference's own sample file
(tests/golden/ref_settings_subset.json, made by make_settings_fixture.py),
and write/read round trips."""
import json
import os

import numpy as np
import pytest

from alien_b200 import params as P
from alien_b200 import settings

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_settings_subset.json")


def test_reads_the_reference_sample_file():
    t, world, prm, unsupported = settings.read_settings(GOLDEN)
    assert t == 85540 and world == (2000, 1000)
    assert prm.motionType == P.MOTION_FLUID
    assert prm.smoothingLength == pytest.approx(0.66, abs=1e-7)
    assert prm.pressureStrength == pytest.approx(0.1) and prm.viscosityStrength == pytest.approx(0.1)
    assert prm.friction == pytest.approx(0.002)
    assert list(prm.cellMaxBindingDistance) == pytest.approx([3.6] * 7)
    assert prm.cellMinDistance == pytest.approx(0.1)
    assert prm.cellFusionVelocity == pytest.approx(0.824)
    assert prm.cellMaxBindingEnergy == pytest.approx(500000.0)
    assert prm.cellDeathConsequences == 2 and prm.cellNumExecutionOrderNumbers == 6
    assert prm.cellMaxAge[0] == 223872
    assert list(prm.radiationCellAgeStrength)[:2] == pytest.approx([0.000026, 0.000093])
    assert prm.radiationMinCellAge[0] == 29648 and prm.radiationMinCellAge[1] == 0
    assert prm.radiationAbsorption[1] == pytest.approx(0.0679)
    assert prm.highRadiationMinCellEnergy[3] == pytest.approx(1483.98205566)
    assert prm.particleSplitEnergy[0] == np.finfo(np.float32).max
    # the sample uses zones, radiation sources and external energy control
    assert set(unsupported) == {"numZones", "numRadiationSources", "externalEnergyControl"}
    assert prm.numZones == 3 and prm.numRadiationSources == 3


def test_write_read_round_trip(tmp_path):
    prm = P.benchmark_parameters(P.MOTION_COLLISION)
    prm.cellMaxCollisionDistance = 1.25
    prm.cellMaxForce[3] = 0.75
    prm.cellMaxAge[6] = 12345
    prm.friction = 0.0015
    path = tmp_path / "w.settings.json"
    settings.write_settings(str(path), 42, (512, 256), prm)
    t, world, got, unsupported = settings.read_settings(str(path))
    assert (t, world, unsupported) == (42, (512, 256), [])
    for name, _, kind, color in settings._FIELDS:
        if name in settings._MOTION_KEYS[P.MOTION_FLUID]:
            continue  # not written for a collision world
        a, b = getattr(got, name), getattr(prm, name)
        if color:
            assert list(a) == pytest.approx(list(b), rel=1e-7, abs=1e-8), name
        else:
            assert a == pytest.approx(b, rel=1e-7, abs=1e-8), name


def test_written_layout_is_the_reference_layout(tmp_path):
    prm = P.benchmark_parameters(P.MOTION_FLUID)
    tree = settings.encode(7, (64, 32), prm)
    assert tree["general"]["world size"] == {"x": "64", "y": "32"}
    sp = tree["simulation parameters"]
    assert sp["motion"]["type"] == "0"
    assert "collision" not in sp["motion"]
    assert sp["fluid"]["smoothing length"] == f"{prm.smoothingLength:.8f}"
    assert [sp["cell"][f"max force[{c}]"] for c in range(7)] == [f"{v:.8f}" for v in prm.cellMaxForce]
    assert sp["features"]["external energy"] == "false"
    json.dumps(tree)  # every value is a string, every path a nested object
    assert all(isinstance(v, str) for v in _leaves(tree))


def test_missing_keys_take_defaults_and_bad_values_fail():
    t, world, prm, unsupported = settings.decode({"simulation parameters": {"friction": "0.5"}})
    default = P.default_parameters()
    assert prm.friction == pytest.approx(0.5) and prm.cellMinDistance == default.cellMinDistance
    assert (t, world, unsupported) == (0, (0, 0), [])
    with pytest.raises(ValueError):
        settings.decode({"simulation parameters": {"friction": 0.5}})
    with pytest.raises(ValueError):
        settings.decode({"simulation parameters": {"features": {"external energy": "yes"}}})


def _leaves(tree):
    for v in tree.values():
        if isinstance(v, dict):
            yield from _leaves(v)
        else:
            yield v
