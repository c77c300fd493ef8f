"""Reader and writer of the reference's ``.settings.json`` files, for the
physics-stage parameters.

The reference stores the settings of a saved simulation next to it as
``<name>.settings.json`` (SerializerService.cpp:850-870, 886-900): a JSON
tree written by boost's property_tree, so every value is a string and every
dotted key path is a chain of nested objects.  The keys are those of
AuxiliaryDataParserService.cpp (general settings :1105-1112, simulation
parameters :12-1100); color-dependent values are seven keys ``name[0]`` ..
``name[6]`` (ParameterParser.h:54-82).  A key that is missing takes the
default, as in the reference's decoder.

Only the fields of ``AlienPhysicsParams`` are read or written: the
physics-stage parameters, the zones ("spots", AuxiliaryDataParserService.cpp
:765-900) with their shapes, flow fields and physics-stage values, the
radiation sources ("particle sources", :723-763) and the external-energy
backflow (:271-300); the rest of the file (rendering, genome mutation,
cell-function parameters) belongs to other parts of the reference.  A zone
value has an ``activated`` flag: ``<key>.activated`` with ``<key>.value``, or
with ``<key>[c]`` for color-dependent values (ParameterParser.h:155-210).  The
fields whose non-default values the engine rejects (particle transformation,
cell-function feature flags) are read so that ``read_settings`` can name
them.  ``innerFriction`` has no key in the
reference's files.
"""
from __future__ import annotations

import json
import math
from typing import Any

from . import params as P

_SP = "simulation parameters."

# field, key below "simulation parameters.", kind ("f" float, "i" int, "b" bool),
# color-dependent.  Motion-specific keys are present only for their motion type.
_FIELDS = [
    ("timestepSize", "time step size", "f", False),
    ("motionType", "motion.type", "i", False),
    ("smoothingLength", "fluid.smoothing length", "f", False),
    ("pressureStrength", "fluid.pressure strength", "f", False),
    ("viscosityStrength", "fluid.viscosity strength", "f", False),
    ("cellMaxCollisionDistance", "motion.collision.max distance", "f", False),
    ("cellRepulsionStrength", "motion.collision.repulsion strength", "f", False),
    ("friction", "friction", "f", False),
    ("rigidity", "rigidity", "f", False),
    ("cellMaxVelocity", "cell.max velocity", "f", False),
    ("cellMaxBindingDistance", "cell.max binding distance", "f", True),
    ("cellMinDistance", "cell.min distance", "f", False),
    ("cellMaxForce", "cell.max force", "f", True),
    ("cellMaxForceDecayProb", "cell.max force decay probability", "f", False),
    ("cellMinEnergy", "cell.min energy", "f", True),
    ("cellFusionVelocity", "cell.fusion velocity", "f", False),
    ("cellMaxBindingEnergy", "cell.max binding energy", "f", False),
    ("cellDeathProbability", "cell.death probability", "f", True),
    ("cellDeathConsequences", "cell.death consequences", "i", False),
    ("cellMaxAge", "cell.max age", "i", True),
    ("cellNumExecutionOrderNumbers", "cell.max execution order number", "i", False),
    ("radiationCellAgeStrength", "radiation.factor", "f", True),
    ("radiationProb", "radiation.probability", "f", False),
    ("radiationVelocityMultiplier", "radiation.velocity multiplier", "f", False),
    ("radiationVelocityPerturbation", "radiation.velocity perturbation", "f", False),
    ("radiationMinCellAge", "radiation.min cell age", "i", True),
    ("radiationAbsorption", "radiation.absorption", "f", True),
    ("highRadiationFactor", "high radiation.factor", "f", True),
    ("highRadiationMinCellEnergy", "high radiation.min cell energy", "f", True),
    ("particleSplitEnergy", "particle.split energy", "f", True),
    ("particleTransformationAllowed", "particle.transformation allowed", "b", False),
    ("numZones", "spots.num spots", "i", False),
    ("numRadiationSources", "particle sources.num sources", "i", False),
    ("cellAgeLimiter", "features.cell age limiter", "b", False),
    ("cellColorTransitionRules", "features.cell color transition rules", "b", False),
    ("advancedAbsorptionControl", "features.additional absorption control", "b", False),
    ("externalEnergyControl", "features.external energy", "b", False),
    ("radiationDisableSources", "radiation.disable sources", "b", False),
    ("externalEnergy", "cell.function.constructor.external energy", "f", False),
    ("externalEnergyBackflowFactor", "cell.function.constructor.external energy backflow", "f", True),
    ("externalEnergyBackflowLimit", "cell.function.constructor.external energy backflow limit", "f", False),
]
# zone ("spots.<i>.") fields: plain, then values with an activated flag
_ZONE_PLAIN = [
    ("posX", "pos.x", "f"), ("posY", "pos.y", "f"), ("velX", "vel.x", "f"), ("velY", "vel.y", "f"),
    ("fadeoutRadius", "fadeout radius", "f"), ("shapeType", "shape.type", "i"),
    ("coreRadius", "shape.circular.core radius", "f"), ("width", "shape.rectangular.core width", "f"),
    ("height", "shape.rectangular.core height", "f"), ("flowType", "flow.type", "i"),
]
_ZONE_FLOW = {  # flow type: [(field, key, kind)]
    P.FLOW_RADIAL: [("flowOrientation", "flow.radial.orientation", "i"), ("flowStrength", "flow.radial.strength", "f"),
                    ("flowDriftAngle", "flow.radial.drift angle", "f")],
    P.FLOW_CENTRAL: [("flowStrength", "flow.central.strength", "f")],
    P.FLOW_LINEAR: [("flowAngle", "flow.linear.angle", "f"), ("flowStrength", "flow.linear.strength", "f")],
}
# (value field, activated flag, key, kind, color-dependent)
_ZONE_VALUES = [
    ("friction", "frictionActivated", "friction", "f", False),
    ("rigidity", "rigidityActivated", "rigidity", "f", False),
    ("radiationDisableSources", "radiationDisableSourcesActivated", "radiation.disable sources", "b", False),
    ("radiationAbsorption", "radiationAbsorptionActivated", "radiation.absorption", "f", True),
    ("radiationCellAgeStrength", "radiationCellAgeStrengthActivated", "radiation.factor", "f", True),
    ("cellMaxForce", "cellMaxForceActivated", "cell.max force", "f", True),
    ("cellMinEnergy", "cellMinEnergyActivated", "cell.min energy", "f", True),
    ("cellDeathProbability", "cellDeathProbabilityActivated", "cell.death probability", "f", True),
    ("cellFusionVelocity", "cellFusionVelocityActivated", "cell.fusion velocity", "f", False),
    ("cellMaxBindingEnergy", "cellMaxBindingEnergyActivated", "cell.max binding energy", "f", False),
]
_SOURCE_FIELDS = [
    ("posX", "pos.x", "f"), ("posY", "pos.y", "f"), ("velX", "vel.x", "f"), ("velY", "vel.y", "f"),
    ("useAngle", "use angle", "b"), ("strength", "strength", "f"), ("angle", "angle", "f"),
    ("shapeType", "shape.type", "i"), ("radius", "shape.circular.radius", "f"),
    ("width", "shape.rectangular.width", "f"), ("height", "shape.rectangular.height", "f"),
]
_MOTION_KEYS = {
    P.MOTION_FLUID: {"smoothingLength", "pressureStrength", "viscosityStrength"},
    P.MOTION_COLLISION: {"cellMaxCollisionDistance", "cellRepulsionStrength"},
}
# fields whose non-default values the engine rejects (ALIEN_B200_ERR_UNSUPPORTED)
_UNSUPPORTED = ("particleTransformationAllowed", "cellAgeLimiter", "cellColorTransitionRules",
                "advancedAbsorptionControl")


def _get(tree: dict, path: str) -> Any:
    """value at a dotted path; the last segment may itself contain dots only
    inside a color suffix, which never happens in these keys"""
    node: Any = tree
    for part in path.split("."):
        if not isinstance(node, dict) or part not in node:
            return None
        node = node[part]
    return node


def _set(tree: dict, path: str, value: str) -> None:
    parts = path.split(".")
    node = tree
    for part in parts[:-1]:
        node = node.setdefault(part, {})
    node[parts[-1]] = value


def _parse(text: Any, kind: str):
    if not isinstance(text, str):
        raise ValueError(f"expected a string value, got {text!r}")
    if kind == "b":
        if text not in ("true", "false"):
            raise ValueError(f"expected true/false, got {text!r}")
        return 1 if text == "true" else 0
    if kind == "i":
        return int(text)
    return float(text)


def _format(value, kind: str) -> str:
    if kind == "b":
        return "true" if value else "false"
    if kind == "i":
        return str(int(value))
    v = float(value)
    if math.isinf(v) or math.isnan(v):
        raise ValueError("settings files hold finite numbers")
    return f"{v:.8f}"  # the reference writes 8 decimals


def decode(tree: dict) -> tuple[int, tuple[int, int], P.PhysicsParams, list[str]]:
    """(timestep, (worldSizeX, worldSizeY), parameters, names of fields the
    engine does not support that hold non-default values) from a parsed file"""
    prm = P.default_parameters()
    general = tree.get("general", {}) if isinstance(tree, dict) else {}
    timestep = int(_parse(_get(general, "time step") or "0", "i"))
    wx = _get(general, "world size.x")
    wy = _get(general, "world size.y")
    world = (int(_parse(wx, "i")) if wx is not None else 0, int(_parse(wy, "i")) if wy is not None else 0)
    motion_text = _get(tree, _SP + "motion.type")
    motion = int(_parse(motion_text, "i")) if motion_text is not None else prm.motionType
    for name, key, kind, color in _FIELDS:
        other_motion = any(name in keys for m, keys in _MOTION_KEYS.items() if m != motion)
        if other_motion:
            continue
        if color:
            arr = getattr(prm, name)
            for c in range(P.MAX_COLORS):
                v = _get(tree, _SP + f"{key}[{c}]")
                if v is not None:
                    arr[c] = _parse(v, kind)
        else:
            v = _get(tree, _SP + key)
            if v is not None:
                setattr(prm, name, _parse(v, kind))
    prm.numZones = max(0, min(prm.numZones, P.MAX_ZONES))
    prm.numRadiationSources = max(0, min(prm.numRadiationSources, P.MAX_RADIATION_SOURCES))
    _decode_zones(tree, prm)
    _decode_sources(tree, prm)
    default = P.default_parameters()
    unsupported = [n for n in _UNSUPPORTED if getattr(prm, n) != getattr(default, n)]
    return timestep, world, prm, unsupported


def _read(tree: dict, path: str, kind: str, fallback):
    v = _get(tree, path)
    return _parse(v, kind) if v is not None else fallback


def _decode_zones(tree: dict, prm: P.PhysicsParams) -> None:
    base_defaults = P.default_parameters()  # a missing zone key takes the struct default
    for i in range(prm.numZones):
        z = P.default_zone(prm.zones[i], base_defaults)
        base = _SP + f"spots.{i}."
        for field, key, kind in _ZONE_PLAIN:
            setattr(z, field, _read(tree, base + key, kind, getattr(z, field)))
        for field, key, kind in _ZONE_FLOW.get(z.flowType, []):
            setattr(z, field, _read(tree, base + key, kind, getattr(z, field)))
        for field, flag, key, kind, color in _ZONE_VALUES:
            setattr(z, flag, _read(tree, base + key + ".activated", "b", 0))
            if color:
                arr = getattr(z, field)
                for c in range(P.MAX_COLORS):
                    arr[c] = _read(tree, base + f"{key}[{c}]", kind, arr[c])
            else:
                setattr(z, field, _read(tree, base + key + ".value", kind, getattr(z, field)))


def _decode_sources(tree: dict, prm: P.PhysicsParams) -> None:
    for i in range(prm.numRadiationSources):
        r = prm.radiationSources[i]
        base = _SP + f"particle sources.{i}."
        for field, key, kind in _SOURCE_FIELDS:
            setattr(r, field, _read(tree, base + key, kind, getattr(r, field)))


def encode(timestep: int, world: tuple[int, int], prm: P.PhysicsParams) -> dict:
    """the physics-stage subset of a settings file; the reference's decoder
    fills every other key with its default"""
    tree: dict = {}
    _set(tree, "general.time step", _format(timestep, "i"))
    _set(tree, "general.world size.x", _format(world[0], "i"))
    _set(tree, "general.world size.y", _format(world[1], "i"))
    for name, key, kind, color in _FIELDS:
        if any(name in keys for m, keys in _MOTION_KEYS.items() if m != prm.motionType):
            continue
        if color:
            arr = getattr(prm, name)
            for c in range(P.MAX_COLORS):
                _set(tree, _SP + f"{key}[{c}]", _format(arr[c], kind))
        else:
            _set(tree, _SP + key, _format(getattr(prm, name), kind))
    for i in range(prm.numZones):
        z = prm.zones[i]
        base = _SP + f"spots.{i}."
        for field, key, kind in _ZONE_PLAIN + _ZONE_FLOW.get(z.flowType, []):
            _set(tree, base + key, _format(getattr(z, field), kind))
        for field, flag, key, kind, color in _ZONE_VALUES:
            _set(tree, base + key + ".activated", _format(getattr(z, flag), "b"))
            if color:
                arr = getattr(z, field)
                for c in range(P.MAX_COLORS):
                    _set(tree, base + f"{key}[{c}]", _format(arr[c], kind))
            else:
                _set(tree, base + key + ".value", _format(getattr(z, field), kind))
    for i in range(prm.numRadiationSources):
        r = prm.radiationSources[i]
        for field, key, kind in _SOURCE_FIELDS:
            _set(tree, _SP + f"particle sources.{i}." + key, _format(getattr(r, field), kind))
    return tree


def read_settings(path: str):
    """decode() of the file at ``path``"""
    with open(path, encoding="utf-8") as f:
        return decode(json.load(f))


def write_settings(path: str, timestep: int, world: tuple[int, int], prm: P.PhysicsParams) -> None:
    with open(path, "w", encoding="utf-8") as f:
        json.dump(encode(timestep, world, prm), f, indent=4)
