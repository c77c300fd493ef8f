"""Zones, flow fields, radiation sources and the external-energy backflow.

* Zones (SimulationParametersZone.h, SpotCalculator.cuh:12-251): a zone
  value blends from the base value into the zone's own by the zone's weight
  at the position (core: the zone value, beyond core + fade-out: the base).
  The physics stage reads friction, cell max force, min energy, death
  probability, fusion velocity, max binding energy, radiation absorption and
  age strength there, and the zone's flow field (FlowFieldKernels.cu:10-89)
  accelerates cells and particles.
* Radiation sources (RadiationProcessor.cuh:42-59, 277-343): emitted
  particles start at a randomly chosen active source; a zone can switch the
  sources inside it off.
* External-energy backflow (RadiationProcessor.cuh:345-354): with external
  energy control on, a share of every emitted particle's energy goes into
  the pool, up to the pool's limit.
* Zones and sources move by their velocities after each step.

The CPU part checks the oracle's zone rules directly; the GPU part compares
the CUDA engine with the FP64 oracle on the same seeded worlds, with the
one-step tolerance of the other parity tests.
"""
import math
import os

import numpy as np
import pytest

from alien_b200 import params as P
from alien_b200 import settings
from alien_b200 import worldgen
from oracle.oracle import OracleSimulation
from tests.helpers import compare_cells, compare_particles

SAMPLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_settings_subset.json")


def zone(prm, i, x, y, **kw):
    z = P.default_zone(prm.zones[i], prm)
    z.posX, z.posY = x, y
    for k, v in kw.items():
        if isinstance(v, (list, tuple)):
            arr = getattr(z, k)
            for c in range(P.MAX_COLORS):
                arr[c] = v[c] if len(v) > 1 else v[0]
        else:
            setattr(z, k, v)
    prm.numZones = max(prm.numZones, i + 1)
    return z


def zone_params(motion):
    """three zones over a 128x128 world: a radial flow with friction and max
    force, a rectangular central flow with fusion velocity and binding
    energy, a linear flow with min energy and death probability"""
    prm = P.benchmark_parameters(motion)
    zone(prm, 0, 40.0, 40.0, coreRadius=12.0, fadeoutRadius=20.0, flowType=P.FLOW_RADIAL, flowStrength=0.004,
         flowDriftAngle=10.0, frictionActivated=1, friction=0.02, cellMaxForceActivated=1, cellMaxForce=[0.3])
    zone(prm, 1, 100.0, 30.0, shapeType=P.SHAPE_RECTANGULAR, width=30.0, height=20.0, fadeoutRadius=15.0,
         flowType=P.FLOW_CENTRAL, flowStrength=0.05, cellFusionVelocityActivated=1, cellFusionVelocity=0.2,
         cellMaxBindingEnergyActivated=1, cellMaxBindingEnergy=80.0)
    zone(prm, 2, 64.0, 100.0, coreRadius=20.0, fadeoutRadius=30.0, flowType=P.FLOW_LINEAR, flowAngle=30.0,
         flowStrength=0.003, cellMinEnergyActivated=1, cellMinEnergy=[90.0], cellDeathProbabilityActivated=1,
         cellDeathProbability=[0.3])
    return prm


def zone_world(seed):
    data, world = worldgen.random_test_world(seed, world=(128, 128), clusters=10, hex_clusters=4, free_cells=800,
                                             particles=300)
    return data, world


# ---- the oracle's zone rules (CPU) --------------------------------------------------------------

def _one_particle_world(x, y, world=(128, 128)):
    data, _ = worldgen.random_test_world(1, world=world, clusters=0, hex_clusters=0, free_cells=0, particles=1)
    data.particles["pos"][0] = (x, y)
    data.particles["vel"][0] = (0.0, 0.0)
    return data, world


def _particle_velocity(prm, x, y):
    data, world = _one_particle_world(x, y)
    o = OracleSimulation(world, prm)
    o.set_simulation_data(data)
    o.calc_timesteps(1)
    v = o.get_simulation_data().particles["vel"][0].astype(np.float64)
    o.close()
    return v


def test_oracle_flow_fields():
    """a particle at rest picks up the flow at its position: the radial flow
    turns around the centre (clockwise on screen: +x above, -x below), the
    central flow pulls towards the centre, the linear flow points along its
    angle (0 = up, clockwise); outside core + fade-out nothing"""
    prm = P.benchmark_parameters(P.MOTION_FLUID)
    zone(prm, 0, 64.0, 64.0, coreRadius=30.0, fadeoutRadius=10.0, flowType=P.FLOW_RADIAL, flowStrength=0.01)
    above = _particle_velocity(prm, 64.0, 54.0)
    below = _particle_velocity(prm, 64.0, 74.0)
    # the flow is the rotated forward-difference gradient of strength *
    # sqrt(distance) (one-unit steps), about strength / (2 sqrt(10)) here
    assert above[0] > 0 and below[0] < 0 and abs(above[1]) < 0.1 * abs(above[0])
    assert above[0] == pytest.approx(0.01 / (2 * math.sqrt(10.0)), rel=0.05)
    assert np.allclose(_particle_velocity(prm, 5.0, 5.0), 0.0)
    prm.zones[0].flowType = P.FLOW_CENTRAL
    left = _particle_velocity(prm, 54.0, 64.0)
    assert left[0] > 0 and abs(left[1]) < 1e-9
    prm.zones[0].flowType = P.FLOW_LINEAR
    prm.zones[0].flowAngle = 90.0
    v = _particle_velocity(prm, 60.0, 60.0)
    assert v[0] == pytest.approx(0.01, rel=1e-6) and abs(v[1]) < 1e-8


def test_oracle_zone_weights_blend_values():
    """death probability 1 in a zone's core kills every detaching cell there,
    base 0 outside keeps every one; the fade-out ring blends"""
    prm = P.benchmark_parameters(P.MOTION_FLUID)
    for c in range(P.MAX_COLORS):
        prm.cellDeathProbability[c] = 0.0
    zone(prm, 0, 32.0, 32.0, coreRadius=10.0, fadeoutRadius=10.0, cellDeathProbabilityActivated=1,
         cellDeathProbability=[1.0])
    data, world = worldgen.random_test_world(2, clusters=0, hex_clusters=0, free_cells=400, particles=0)
    data.cells["numConnections"] = 0
    data.cells["livingState"] = 3  # detaching
    data.cells["vel"] = 0
    o = OracleSimulation(world, prm)
    o.set_simulation_data(data)
    o.calc_timesteps(1)
    survivors = set(o.get_simulation_data().cells["id"].tolist())
    o.close()
    d = np.hypot(data.cells["pos"][:, 0] - 32.0, data.cells["pos"][:, 1] - 32.0)
    core = data.cells["id"][d < 9.5]
    outside = data.cells["id"][d > 20.5]
    assert len(core) and len(outside)
    assert not (set(core.tolist()) & survivors)
    assert set(outside.tolist()) <= survivors


def test_oracle_zone_and_source_movement():
    prm = P.benchmark_parameters(P.MOTION_FLUID)
    zone(prm, 0, 10.0, 20.0, velX=0.5, velY=-0.25)
    prm.numRadiationSources = 1
    s = prm.radiationSources[0]
    s.posX, s.posY, s.velX, s.velY, s.strength = 100.0, 5.0, -1.5, 2.0, 1.0
    data, world = _one_particle_world(1.0, 1.0)
    o = OracleSimulation(world, prm)
    o.set_simulation_data(data)
    o.calc_timesteps(4)
    got = o.get_simulation_parameters()
    o.close()
    assert (got.zones[0].posX, got.zones[0].posY) == pytest.approx((12.0, 19.0))
    assert (got.radiationSources[0].posX, got.radiationSources[0].posY) == pytest.approx((94.0, 13.0))


def test_oracle_backflow_limit():
    """emitted energy goes into the pool at the backflow factor while the pool
    stays under its limit; cell energy + particle energy + pool is conserved"""
    data, world = worldgen.random_test_world(3, free_cells=300, particles=50)
    data.cells["age"] = 1000
    prm = P.default_parameters()
    for c in range(P.MAX_COLORS):
        prm.radiationCellAgeStrength[c] = 0.01
        prm.externalEnergyBackflowFactor[c] = 0.5
    prm.externalEnergyControl = 1
    prm.externalEnergy = 10.0
    e0 = _energy(data) + prm.externalEnergy
    for limit, grows in ((P.FLT_MAX, True), (10.0, False)):
        prm.externalEnergyBackflowLimit = limit
        o = OracleSimulation(world, prm)
        o.set_simulation_data(data)
        o.calc_timesteps(3)
        pool = o.get_simulation_parameters().externalEnergy
        out = o.get_simulation_data()
        o.close()
        assert (pool > 10.0) == grows
        assert _energy(out) + pool == pytest.approx(e0, rel=1e-9)


def _energy(data):
    return float(data.cells["energy"].astype(np.float64).sum() + data.particles["energy"].astype(np.float64).sum())


# ---- the CUDA engine against the oracle (GPU) ---------------------------------------------------

def run_both(data, world, prm, steps, timestep=0):
    from alien_b200.facade import SimulationFacade

    eng = SimulationFacade()
    eng.new_simulation(timestep, world, prm)
    eng.set_simulation_data(data)
    eng.calc_timesteps(steps)
    got = eng.get_simulation_data()
    got_prm = eng.get_simulation_parameters()
    eng.close_simulation()
    ora = OracleSimulation(world, prm, timestep)
    ora.set_simulation_data(data)
    ora.calc_timesteps(steps)
    ref = ora.get_simulation_data()
    ref_prm = ora.get_simulation_parameters()
    ora.close()
    return got, ref, got_prm, ref_prm


@pytest.mark.gpu
@pytest.mark.parametrize("motion", [P.MOTION_FLUID, P.MOTION_COLLISION])
@pytest.mark.parametrize("steps", [1, 3])
def test_zones_match_oracle(motion, steps):
    data, world = zone_world(41)
    data.cells["livingState"][::9] = 3  # detaching: zone death probability
    prm = zone_params(motion)
    got, ref, _, _ = run_both(data, world, prm, steps)
    rtol = 1e-5 if steps == 1 else 5e-5  # FP32 rounding compounds over steps
    compare_cells(got.cells, ref.cells, world, rtol=rtol, before=data.cells)
    compare_particles(got.particles, ref.particles, world, rtol=rtol, before=data.particles)


@pytest.mark.gpu
@pytest.mark.parametrize("motion", [P.MOTION_FLUID, P.MOTION_COLLISION])
def test_radiation_sources_match_oracle(motion):
    """three sources, one of them switched off by a zone; emitted particles
    start inside the active sources.  A source is drawn by comparing one
    uniform draw in [0, 1) with the running sum of the active sources'
    strengths (RadiationProcessor.cuh:253-270), so the strengths of the
    active sources sum to 1 here, as the reference's editor keeps them"""
    data, world = zone_world(42)
    data.cells["age"] = np.random.default_rng(42).integers(0, 400, len(data.cells)).astype(np.uint32)
    prm = P.default_parameters()
    prm.motionType = motion
    for c in range(P.MAX_COLORS):
        prm.radiationCellAgeStrength[c] = 0.002
    prm.numRadiationSources = 3
    shapes = [(20.0, 20.0, 0.4, P.SHAPE_CIRCULAR, 5.0, 0, 0.0), (90.0, 60.0, 0.6, P.SHAPE_RECTANGULAR, 0.0, 1, 45.0),
              (60.0, 110.0, 0.5, P.SHAPE_CIRCULAR, 3.0, 0, 0.0)]
    for s, (x, y, strength, shape, radius, use_angle, angle) in zip(prm.radiationSources, shapes):
        s.posX, s.posY, s.strength, s.shapeType, s.radius, s.useAngle, s.angle = x, y, strength, shape, radius, \
            use_angle, angle
        s.width, s.height = 10.0, 4.0
    zone(prm, 0, 60.0, 110.0, coreRadius=6.0, fadeoutRadius=2.0, radiationDisableSourcesActivated=1,
         radiationDisableSources=1)
    got, ref, _, _ = run_both(data, world, prm, 2)
    compare_cells(got.cells, ref.cells, world, before=data.cells)
    compare_particles(got.particles, ref.particles, world, before=data.particles)
    first_new = max(int(data.cells["id"].max()), int(data.particles["id"].max()))
    new = got.particles[got.particles["id"] > first_new]
    assert len(new) > 10, "too few radiation particles"
    p = new["pos"].astype(np.float64)
    near0 = np.hypot(p[:, 0] - 20.0, p[:, 1] - 20.0) < 5.0 + 2.5
    near1 = (np.abs(p[:, 0] - 90.0) < 5.0 + 2.5) & (np.abs(p[:, 1] - 60.0) < 2.0 + 2.5)
    assert np.all(near0 | near1), "a particle started outside the active sources"
    assert np.any(near0) and np.any(near1)


@pytest.mark.gpu
@pytest.mark.parametrize("limit", [P.FLT_MAX, 40.0])
def test_external_energy_backflow_matches_oracle(limit):
    data, world = zone_world(43)
    data.cells["age"] = 1000
    data.cells["livingState"][::7] = 3
    prm = P.default_parameters()
    for c in range(P.MAX_COLORS):
        prm.radiationCellAgeStrength[c] = 0.003
        prm.externalEnergyBackflowFactor[c] = 0.1 * (c + 1)
        prm.cellDeathProbability[c] = 0.2
    prm.externalEnergyControl = 1
    prm.externalEnergy = 30.0
    prm.externalEnergyBackflowLimit = limit
    got, ref, gp, rp = run_both(data, world, prm, 3)
    compare_cells(got.cells, ref.cells, world, before=data.cells)
    compare_particles(got.particles, ref.particles, world, before=data.particles)
    assert rp.externalEnergy > 30.0
    assert gp.externalEnergy == pytest.approx(rp.externalEnergy, rel=1e-5)
    e0 = _energy(data) + 30.0
    assert _energy(got) + gp.externalEnergy == pytest.approx(e0, rel=1e-5)


@pytest.mark.gpu
def test_zone_and_source_movement_matches_oracle():
    data, world = zone_world(44)
    prm = zone_params(P.MOTION_FLUID)
    prm.zones[0].velX, prm.zones[0].velY = 0.75, -0.5
    prm.zones[2].velX = -1.25
    prm.numRadiationSources = 1
    prm.radiationSources[0].posX, prm.radiationSources[0].posY = 10.0, 10.0
    prm.radiationSources[0].velX, prm.radiationSources[0].velY = 0.5, 0.25
    prm.radiationSources[0].strength = 1.0
    got, ref, gp, rp = run_both(data, world, prm, 6)
    compare_cells(got.cells, ref.cells, world, rtol=5e-5, before=data.cells)
    compare_particles(got.particles, ref.particles, world, rtol=5e-5, before=data.particles)
    for i in range(prm.numZones):
        assert (gp.zones[i].posX, gp.zones[i].posY) == pytest.approx((rp.zones[i].posX, rp.zones[i].posY), rel=1e-6)
    assert (gp.zones[0].posX, gp.zones[0].posY) == pytest.approx((44.5, 37.0), rel=1e-6)
    s, r = gp.radiationSources[0], rp.radiationSources[0]
    assert (s.posX, s.posY) == pytest.approx((r.posX, r.posY), rel=1e-6) == (13.0, 11.5)


@pytest.mark.gpu
@pytest.mark.parametrize("dt", [0, 1, 2])
def test_reference_sample_settings_match_oracle(dt):
    """the reference's own sample settings (fluid motion, three zones with
    radial flows, three radiation sources, backflow on) over a random world
    of the sample's size, one step from each phase of the three-step cycle.
    One step only: the world reaches x = 2000, where FP32 positions (the
    transfer objects' type) resolve 1.2e-4, so two close cells' distance
    after a stored step carries ~1e-3 relative error into the next step's
    fluid forces."""
    t, world, prm, unsupported = settings.read_settings(SAMPLE)
    assert unsupported == []
    data, world = worldgen.random_test_world(45, world=world, clusters=60, hex_clusters=20, free_cells=6000,
                                             particles=2000)
    data.cells["age"] = np.random.default_rng(45).integers(0, 300000, len(data.cells)).astype(np.uint32)
    got, ref, gp, rp = run_both(data, world, prm, 1, t + dt)
    compare_cells(got.cells, ref.cells, world, before=data.cells)
    compare_particles(got.particles, ref.particles, world, before=data.particles)
    first_new = max(int(data.cells["id"].max()), int(data.particles["id"].max()))
    assert np.count_nonzero(got.particles["id"] > first_new) > 50, "the sample's radiation emitted too little"
    assert gp.externalEnergy == pytest.approx(rp.externalEnergy, rel=1e-5, abs=1e-3)
    for i in range(prm.numZones):
        assert (gp.zones[i].posX, gp.zones[i].posY) == (rp.zones[i].posX, rp.zones[i].posY)
