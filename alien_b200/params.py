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
        ("reserved", ctypes.c_uint8 * 3),
        ("cellNumExecutionOrderNumbers", ctypes.c_int32),
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
    return p


def benchmark_parameters(motion_type: int = MOTION_FLUID) -> PhysicsParams:
    """Defaults with radiation off, as the reference's integration tests set
    them (EngineTests/IntegrationTestFramework.cpp:14-20)."""
    p = default_parameters()
    _fill(p.radiationCellAgeStrength, 0.0)
    p.motionType = motion_type
    return p
