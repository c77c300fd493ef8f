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
    # the sample's zones, radiation sources and external-energy backflow
    assert unsupported == []
    assert prm.numZones == 3 and prm.numRadiationSources == 3
    z0, z2 = prm.zones[0], prm.zones[2]
    assert (z0.posX, z0.posY, z0.shapeType, z0.flowType) == (500.0, 500.0, P.SHAPE_CIRCULAR, P.FLOW_RADIAL)
    assert z0.coreRadius == pytest.approx(367.7) and z0.fadeoutRadius == pytest.approx(154.8)
    assert z0.flowStrength == pytest.approx(0.00305) and z0.flowDriftAngle == pytest.approx(2.6)
    assert z0.radiationCellAgeStrengthActivated == 1 and z0.frictionActivated == 0
    assert (z2.shapeType, z2.width, z2.flowType) == (P.SHAPE_RECTANGULAR, 2000.0, P.FLOW_NONE)
    assert z2.height == pytest.approx(54.8)
    s0, s2 = prm.radiationSources[0], prm.radiationSources[2]
    assert (s0.posX, s0.posY, s0.shapeType, s0.radius) == (502.0, 502.0, P.SHAPE_CIRCULAR, 82.0)
    assert (s2.shapeType, s2.useAngle, s2.angle, s2.height) == (P.SHAPE_RECTANGULAR, 1, 90.0, 164.0)
    assert s0.strength == pytest.approx(1 / 3)
    assert prm.externalEnergyControl == 1 and prm.externalEnergyBackflowFactor[0] == pytest.approx(0.1436)
    assert prm.externalEnergyBackflowFactor[1] == 0.0


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


def test_zones_and_sources_round_trip(tmp_path):
    """a reference file read and written again keeps its zones, sources and
    backflow values, zone rigidity included"""
    _, _, prm, _ = settings.read_settings(GOLDEN)
    path = tmp_path / "z.settings.json"
    settings.write_settings(str(path), 5, (2000, 1000), prm)
    _, _, got, unsupported = settings.read_settings(str(path))
    assert unsupported == []
    for i in range(prm.numZones):
        for name, _ in P.Zone._fields_:
            a, b = getattr(got.zones[i], name), getattr(prm.zones[i], name)
            if hasattr(a, "__len__"):
                assert list(a) == pytest.approx(list(b), rel=1e-7), (i, name)
            else:
                assert a == pytest.approx(b, rel=1e-7), (i, name)
    for i in range(prm.numRadiationSources):
        for name, _ in P.RadiationSource._fields_:
            assert getattr(got.radiationSources[i], name) == pytest.approx(getattr(prm.radiationSources[i], name),
                                                                           rel=1e-7), (i, name)
    assert list(got.externalEnergyBackflowFactor) == pytest.approx(list(prm.externalEnergyBackflowFactor), rel=1e-7)
    prm.zones[1].rigidityActivated, prm.zones[1].rigidity = 1, 0.5
    settings.write_settings(str(path), 5, (2000, 1000), prm)
    _, _, got, unsupported = settings.read_settings(str(path))
    assert unsupported == [] and got.zones[1].rigidityActivated == 1 and got.zones[1].rigidity == 0.5


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
