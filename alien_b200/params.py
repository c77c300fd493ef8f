"""``AlienPhysicsParams``: the physics-stage subset of the reference's
``SimulationParameters`` (source/EngineInterface/SimulationParameters.h:18-206,
SimulationParametersZoneValues.h:10-30, Motion.h:7-43), as a ctypes struct
with the reference's field names and defaults."""
from __future__ import annotations

import ctypes

MAX_COLORS = 7
FLT_MAX = 3.4028234663852886e38  # Infinity<float>::value = numeric_limits<float>::max()
INT_MAX = 2147483647

MOTION_FLUID = 0
MOTION_COLLISION = 1


MAX_ZONES = 20
MAX_RADIATION_SOURCES = 40
SHAPE_CIRCULAR, SHAPE_RECTANGULAR = 0, 1
FLOW_NONE, FLOW_RADIAL, FLOW_CENTRAL, FLOW_LINEAR = 0, 1, 2, 3

_C = ctypes.c_float * MAX_COLORS


class Zone(ctypes.Structure):
    """AlienZone (include/alien_b200.h): SimulationParametersZone's physics-stage part"""
    _fields_ = [
        ("posX", ctypes.c_float), ("posY", ctypes.c_float), ("velX", ctypes.c_float), ("velY", ctypes.c_float),
        ("fadeoutRadius", ctypes.c_float),
        ("shapeType", ctypes.c_int32),
        ("coreRadius", ctypes.c_float), ("width", ctypes.c_float), ("height", ctypes.c_float),
        ("flowType", ctypes.c_int32), ("flowOrientation", ctypes.c_int32),
        ("flowStrength", ctypes.c_float), ("flowDriftAngle", ctypes.c_float), ("flowAngle", ctypes.c_float),
        ("friction", ctypes.c_float), ("rigidity", ctypes.c_float),
        ("radiationAbsorption", _C), ("radiationCellAgeStrength", _C), ("cellMaxForce", _C), ("cellMinEnergy", _C),
        ("cellDeathProbability", _C),
        ("cellFusionVelocity", ctypes.c_float), ("cellMaxBindingEnergy", ctypes.c_float),
        ("radiationDisableSources", ctypes.c_uint8),
        ("frictionActivated", ctypes.c_uint8), ("rigidityActivated", ctypes.c_uint8),
        ("radiationAbsorptionActivated", ctypes.c_uint8), ("radiationCellAgeStrengthActivated", ctypes.c_uint8),
        ("cellMaxForceActivated", ctypes.c_uint8), ("cellMinEnergyActivated", ctypes.c_uint8),
        ("cellDeathProbabilityActivated", ctypes.c_uint8), ("cellFusionVelocityActivated", ctypes.c_uint8),
        ("cellMaxBindingEnergyActivated", ctypes.c_uint8), ("radiationDisableSourcesActivated", ctypes.c_uint8),
        ("reserved", ctypes.c_uint8 * 1),
    ]


class RadiationSource(ctypes.Structure):
    """AlienRadiationSource (include/alien_b200.h)"""
    _fields_ = [
        ("strength", ctypes.c_float), ("posX", ctypes.c_float), ("posY", ctypes.c_float), ("velX", ctypes.c_float),
        ("velY", ctypes.c_float), ("useAngle", ctypes.c_int32), ("angle", ctypes.c_float), ("shapeType", ctypes.c_int32),
        ("radius", ctypes.c_float), ("width", ctypes.c_float), ("height", ctypes.c_float),
    ]


class PhysicsParams(ctypes.Structure):
    _fields_ = [
        ("timestepSize", ctypes.c_float),
        ("motionType", ctypes.c_int32),
        ("smoothingLength", ctypes.c_float),
        ("viscosityStrength", ctypes.c_float),
        ("pressureStrength", ctypes.c_float),
        ("cellMaxCollisionDistance", ctypes.c_float),
        ("cellRepulsionStrength", ctypes.c_float),
        ("innerFriction", ctypes.c_float),
        ("cellMaxVelocity", ctypes.c_float),
        ("cellMaxBindingDistance", ctypes.c_float * MAX_COLORS),
        ("cellMinDistance", ctypes.c_float),
        ("cellMaxForceDecayProb", ctypes.c_float),
        ("radiationProb", ctypes.c_float),
        ("radiationVelocityMultiplier", ctypes.c_float),
        ("radiationVelocityPerturbation", ctypes.c_float),
        ("radiationMinCellAge", ctypes.c_int32 * MAX_COLORS),
        ("highRadiationFactor", ctypes.c_float * MAX_COLORS),
        ("highRadiationMinCellEnergy", ctypes.c_float * MAX_COLORS),
        ("cellDeathConsequences", ctypes.c_int32),
        ("cellMaxAge", ctypes.c_int32 * MAX_COLORS),
        ("particleSplitEnergy", ctypes.c_float * MAX_COLORS),
        ("friction", ctypes.c_float),
        ("rigidity", ctypes.c_float),
        ("radiationAbsorption", ctypes.c_float * MAX_COLORS),
        ("radiationCellAgeStrength", ctypes.c_float * MAX_COLORS),
        ("cellMaxForce", ctypes.c_float * MAX_COLORS),
        ("cellMinEnergy", ctypes.c_float * MAX_COLORS),
        ("cellDeathProbability", ctypes.c_float * MAX_COLORS),
        ("cellFusionVelocity", ctypes.c_float),
        ("cellMaxBindingEnergy", ctypes.c_float),
        ("numZones", ctypes.c_int32),
        ("numRadiationSources", ctypes.c_int32),
        ("particleTransformationAllowed", ctypes.c_uint8),
        ("cellAgeLimiter", ctypes.c_uint8),
        ("cellColorTransitionRules", ctypes.c_uint8),
        ("advancedAbsorptionControl", ctypes.c_uint8),
        ("externalEnergyControl", ctypes.c_uint8),
        ("radiationDisableSources", ctypes.c_uint8),
        ("reserved", ctypes.c_uint8 * 2),
        ("cellNumExecutionOrderNumbers", ctypes.c_int32),
        ("externalEnergy", ctypes.c_float),
        ("externalEnergyBackflowFactor", ctypes.c_float * MAX_COLORS),
        ("externalEnergyBackflowLimit", ctypes.c_float),
        ("zones", Zone * MAX_ZONES),
        ("radiationSources", RadiationSource * MAX_RADIATION_SOURCES),
    ]

    def copy(self) -> "PhysicsParams":
        out = PhysicsParams()
        ctypes.memmove(ctypes.byref(out), ctypes.byref(self), ctypes.sizeof(self))
        return out


def _fill(arr, value):
    for i in range(len(arr)):
        arr[i] = value


def default_parameters() -> PhysicsParams:
    """Reference defaults (SimulationParameters.h, ZoneValues.h, Motion.h)."""
    p = PhysicsParams()
    p.timestepSize = 1.0
    p.motionType = MOTION_FLUID
    p.smoothingLength = 0.8
    p.viscosityStrength = 0.1
    p.pressureStrength = 0.1
    p.cellMaxCollisionDistance = 1.3
    p.cellRepulsionStrength = 0.08
    p.innerFriction = 0.3
    p.cellMaxVelocity = 2.0
    _fill(p.cellMaxBindingDistance, 3.6)
    p.cellMinDistance = 0.3
    p.cellMaxForceDecayProb = 0.2
    p.radiationProb = 0.03
    p.radiationVelocityMultiplier = 1.0
    p.radiationVelocityPerturbation = 0.5
    _fill(p.radiationMinCellAge, 0)
    _fill(p.highRadiationFactor, 0.0)
    _fill(p.highRadiationMinCellEnergy, 500.0)
    p.cellDeathConsequences = 2  # CellDeathConsquences_DetachedPartsDie
    _fill(p.cellMaxAge, INT_MAX)
    _fill(p.particleSplitEnergy, FLT_MAX)
    p.friction = 0.001
    p.rigidity = 0.0
    _fill(p.radiationAbsorption, 1.0)
    _fill(p.radiationCellAgeStrength, 0.00002)
    _fill(p.cellMaxForce, 0.8)
    _fill(p.cellMinEnergy, 50.0)
    _fill(p.cellDeathProbability, 0.001)
    p.cellFusionVelocity = 0.6
    p.cellMaxBindingEnergy = FLT_MAX
    p.cellNumExecutionOrderNumbers = 6
    p.externalEnergyBackflowLimit = FLT_MAX
    for z in p.zones:
        default_zone(z, p)
    for r in p.radiationSources:
        r.radius = 1.0
        r.width, r.height = 100.0, 200.0
    return p


def default_zone(z: Zone, base: PhysicsParams) -> Zone:
    """the reference's zone defaults (SimulationParametersZone.h): circular,
    core radius 100, fade-out radius 100, no flow, the base values, nothing
    activated"""
    z.fadeoutRadius = 100.0
    z.shapeType = SHAPE_CIRCULAR
    z.coreRadius = 100.0
    z.width, z.height = 100.0, 200.0
    z.flowType = FLOW_NONE
    z.flowStrength = 0.001
    z.friction, z.rigidity = base.friction, base.rigidity
    for c in range(MAX_COLORS):
        z.radiationAbsorption[c] = base.radiationAbsorption[c]
        z.radiationCellAgeStrength[c] = base.radiationCellAgeStrength[c]
        z.cellMaxForce[c] = base.cellMaxForce[c]
        z.cellMinEnergy[c] = base.cellMinEnergy[c]
        z.cellDeathProbability[c] = base.cellDeathProbability[c]
    z.cellFusionVelocity, z.cellMaxBindingEnergy = base.cellFusionVelocity, base.cellMaxBindingEnergy
    return z


def benchmark_parameters(motion_type: int = MOTION_FLUID) -> PhysicsParams:
    """Defaults with radiation off, as the reference's integration tests set
    them (EngineTests/IntegrationTestFramework.cpp:14-20)."""
    p = default_parameters()
    _fill(p.radiationCellAgeStrength, 0.0)
    p.motionType = motion_type
    return p
