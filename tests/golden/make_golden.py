"""Generates the golden fixtures of the reference engine (run on a GPU box).

    python tests/golden/make_golden.py [<out_dir>]   (default: tests/golden)

For each seeded input below it runs the reference's own CUDA engine
(oracle/_ref/ref_run, built from the reference sources by oracle/ref/Makefile)
and stores the input DataTO and the reference's output (one step) as
compressed npz, or, for long runs, the reference's aggregate observables as
JSON.  The CPU tests (tests/test_golden.py) check the oracle against these
files; the inputs are regenerated from their seeds and compared byte for
byte with the stored copy.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from alien_b200 import params as P  # noqa: E402
from alien_b200 import worldgen  # noqa: E402
from oracle import refrun  # noqa: E402

ONE_STEP = [
    # name, seed, motion, timestep, innerFriction (None = default)
    ("calm_fluid_t0", 21, P.MOTION_FLUID, 0, None),
    ("calm_fluid_t1", 22, P.MOTION_FLUID, 1, None),
    ("calm_collision_t0", 23, P.MOTION_COLLISION, 0, None),
    ("calm_collision_t2", 24, P.MOTION_COLLISION, 2, None),
    # angle forces on, lock-guarded inner friction off
    ("calm_fluid_t3_nofric", 25, P.MOTION_FLUID, 3, 0.0),
    ("calm_collision_t3_nofric", 26, P.MOTION_COLLISION, 3, 0.0),
]

ZONE_ONE_STEP = [
    # name, seed, motion, timestep: calm worlds under three zones with flow
    # fields and friction (see zone_params)
    ("calm_zone_fluid_t1", 27, P.MOTION_FLUID, 1),
    ("calm_zone_collision_t2", 28, P.MOTION_COLLISION, 2),
]


NEURON_RUNS = [
    # name, seed, motion, timestep, steps: calm worlds with neuron cells; the
    # steps cover every execution order number (6) and chains of neurons
    ("neuron_fluid_t0", 41, P.MOTION_FLUID, 0, 13),
    ("neuron_collision_t4", 42, P.MOTION_COLLISION, 4, 13),
]


def neuron_world(seed):
    data, world = worldgen.calm_test_world(seed)
    return worldgen.add_neurons(data, seed, fraction=0.6), world


def one_step_params(motion, inner_friction):
    prm = P.benchmark_parameters(motion)
    if inner_friction is not None:
        prm.innerFriction = inner_friction
    return prm


RIGID_ONE_STEP = [
    # name, seed, motion, timestep: calm worlds with rigidity (a step with
    # timestep % 3 == 0 runs the cluster pass); inner friction off, since it
    # runs in the same steps under the reference's tryLock
    ("calm_rigid_fluid_t0", 29, P.MOTION_FLUID, 0),
    ("calm_rigid_collision_t3", 30, P.MOTION_COLLISION, 3),
]


def rigid_params(motion):
    """base rigidity 0.6, and 1.0 in a circular zone around the world's
    centre (the rigidity blend of ClusterProcessor::applyClusterData)"""
    prm = P.benchmark_parameters(motion)
    prm.innerFriction = 0.0
    prm.rigidity = 0.6
    prm.numZones = 1
    z = P.default_zone(prm.zones[0], prm)
    z.posX, z.posY, z.coreRadius, z.fadeoutRadius = 32.0, 32.0, 12.0, 8.0
    z.rigidityActivated, z.rigidity = 1, 1.0
    return prm


def zone_params(motion):
    """three zones over the 64x64 calm world: a clockwise radial flow with
    drift and zone friction, a rectangular central flow, a linear flow with a
    second friction value; everything else at the benchmark values"""
    prm = P.benchmark_parameters(motion)
    prm.numZones = 3
    z0, z1, z2 = (P.default_zone(prm.zones[i], prm) for i in range(3))
    z0.posX, z0.posY, z0.coreRadius, z0.fadeoutRadius = 18.0, 20.0, 9.0, 12.0
    z0.flowType, z0.flowStrength, z0.flowDriftAngle = P.FLOW_RADIAL, 0.004, 15.0
    z0.frictionActivated, z0.friction = 1, 0.02
    z1.posX, z1.posY, z1.shapeType, z1.width, z1.height, z1.fadeoutRadius = 46.0, 18.0, P.SHAPE_RECTANGULAR, 18.0, \
        14.0, 10.0
    z1.flowType, z1.flowStrength = P.FLOW_CENTRAL, 0.05
    z2.posX, z2.posY, z2.coreRadius, z2.fadeoutRadius = 32.0, 48.0, 10.0, 14.0
    z2.flowType, z2.flowAngle, z2.flowStrength = P.FLOW_LINEAR, 120.0, 0.003
    z2.frictionActivated, z2.friction = 1, 0.0
    return prm


def calm(seed):
    return worldgen.calm_test_world(seed)


def observables(data):
    c, p = data.cells, data.particles
    speed = np.hypot(c["vel"][:, 0].astype(np.float64), c["vel"][:, 1].astype(np.float64))
    hist, _ = np.histogram(speed, bins=20, range=(0.0, 2.0))
    return {
        "cells": int(len(c)), "particles": int(len(p)),
        "bonds": int(np.sum(c["numConnections"])),
        "cell_energy": float(np.sum(c["energy"], dtype=np.float64)),
        "particle_energy": float(np.sum(p["energy"], dtype=np.float64)),
        "mean_speed": float(speed.mean()) if len(c) else 0.0,
        "speed_hist": hist.tolist(),
        "dying_or_detaching": int(np.sum((c["livingState"] == 3) | (c["livingState"] == 5))),
    }


LONG_RUNS = {
    # name: (builder, motion, steps)
    "stats_softbody": (lambda: worldgen.soft_body_world(seed=5, world=(128, 128), clusters=20, particles=1500), P.MOTION_FLUID, 300),
    "stats_fluid": (lambda: worldgen.fluid_world(seed=6, world=(128, 128), cells=3900), P.MOTION_FLUID, 300),
    "stats_hex": (lambda: worldgen.hex_world(seed=7, world=(256, 256), clusters=120), P.MOTION_COLLISION, 300),
}


def decay_input():
    """CellConnectionTests.decay (EngineTests/CellConnectionTests.cpp:19-37)"""
    tmpl = worldgen.rect_template()
    cells = worldgen._clusters_to_cells(tmpl, np.zeros((1, 2)), np.zeros((1, 2)), np.zeros(1), 25.0, 1, (1000, 1000))
    prm = P.benchmark_parameters()
    prm.radiationAbsorption[0] = 0.0
    prm.cellDeathConsequences = 1
    prm.cellDeathProbability[0] = 0.5
    from alien_b200.to import DataTO
    return DataTO(cells), (1000, 1000), prm


DENSITY_ONE_STEP = [
    # name, seed, motion, timestep
    ("density_collision_t47", 41, P.MOTION_COLLISION, 47),
    ("density_fluid_t70", 42, P.MOTION_FLUID, 70),
]


def density_world(seed):
    """a calm world (no overlap correction moves a cell in the step, so the
    density map holds the cells at their input positions) whose cells carry
    colors, mutation ids (0, 1 and others) and genome complexities that reach
    every bucket of DensityMap::addCell (DensityMap.cuh:150-205)"""
    data, world = worldgen.calm_test_world(seed, world=(96, 96), clusters=10, hex_clusters=4, free_cells=700)
    rng = np.random.default_rng(seed)
    n = data.num_cells
    c = data.cells
    c["color"] = rng.integers(0, 7, n).astype(c["color"].dtype)
    c["mutationId"] = rng.choice(np.array([0, 1, 2, 3, 5, 7, 11, 24, 105, 1000003], np.uint32), n)
    c["genomeComplexity"] = np.where(rng.random(n) < 0.1, rng.uniform(7000.0, 9000.0, n),
                                     rng.uniform(0.0, 30.0, n)).astype(np.float32)
    return data, world


def density_fixtures(out_dir):
    for name, seed, motion, t in DENSITY_ONE_STEP:
        data, world = density_world(seed)
        prm = P.benchmark_parameters(motion)
        out, _, ts, dm = refrun.run(data, world, prm, steps=1, timestep=t, density_map=True)
        np.savez_compressed(os.path.join(out_dir, f"ref_{name}.npz"), in_cells=data.cells, in_particles=data.particles,
                            out_cells=out.cells, params=np.frombuffer(bytes(prm), np.uint8),
                            meta=np.array([seed, motion, t, world[0], world[1], ts], np.int64),
                            **{f"map_{k}": v for k, v in dm.items()})
        print(name, out.num_cells, ts, {k: int(np.count_nonzero(v)) for k, v in dm.items()})


def main(out_dir):
    """ZONES_ONLY=1 writes only the zone and rigidity fixtures; NEURON_ONLY=1
    stops after the one-step and neuron fixtures; DENSITY_ONLY=1 writes only
    the density-map fixtures"""
    os.makedirs(out_dir, exist_ok=True)
    density_fixtures(out_dir)
    if os.environ.get("DENSITY_ONLY"):
        return
    zone_fixtures(out_dir)
    rigid_fixtures(out_dir)
    if os.environ.get("ZONES_ONLY"):
        return
    one_step_fixtures(out_dir)
    more_fixtures(out_dir)


def one_step_fixtures(out_dir):
    for name, seed, motion, t, fric in ONE_STEP:
        data, world = calm(seed)
        prm = one_step_params(motion, fric)
        out, _, ts = refrun.run(data, world, prm, steps=1, timestep=t)
        np.savez_compressed(os.path.join(out_dir, f"ref_{name}.npz"), in_cells=data.cells, in_particles=data.particles,
                            out_cells=out.cells, out_particles=out.particles,
                            params=np.frombuffer(bytes(prm), np.uint8),
                            meta=np.array([seed, motion, t, world[0], world[1], ts], np.int64))
        print(name, out.num_cells, out.num_particles, ts)


def zone_fixtures(out_dir):
    for name, seed, motion, t in ZONE_ONE_STEP:
        data, world = calm(seed)
        prm = zone_params(motion)
        out, _, ts = refrun.run(data, world, prm, steps=1, timestep=t)
        np.savez_compressed(os.path.join(out_dir, f"ref_{name}.npz"), in_cells=data.cells, in_particles=data.particles,
                            out_cells=out.cells, out_particles=out.particles,
                            params=np.frombuffer(bytes(prm), np.uint8),
                            meta=np.array([seed, motion, t, world[0], world[1], ts], np.int64))
        print(name, out.num_cells, out.num_particles, ts)


def rigid_world(seed):
    """a calm world whose bonded cells carry velocity noise of 0.02, so that
    the rigid-body blend changes their velocities noticeably"""
    data, world = calm(seed)
    rng = np.random.default_rng(seed)
    bonded = data.cells["numConnections"] > 0
    data.cells["vel"][bonded] += rng.uniform(-0.02, 0.02, (int(bonded.sum()), 2)).astype(np.float32)
    return data, world


def rigid_fixtures(out_dir):
    for name, seed, motion, t in RIGID_ONE_STEP:
        data, world = rigid_world(seed)
        prm = rigid_params(motion)
        out, _, ts = refrun.run(data, world, prm, steps=1, timestep=t)
        np.savez_compressed(os.path.join(out_dir, f"ref_{name}.npz"), in_cells=data.cells, in_particles=data.particles,
                            out_cells=out.cells, out_particles=out.particles,
                            params=np.frombuffer(bytes(prm), np.uint8),
                            meta=np.array([seed, motion, t, world[0], world[1], ts], np.int64))
        print(name, out.num_cells, out.num_particles, ts)


def more_fixtures(out_dir):
    for name, seed, motion, t, steps in NEURON_RUNS:
        data, world = neuron_world(seed)
        prm = P.benchmark_parameters(motion)
        out, _, ts = refrun.run(data, world, prm, steps=steps, timestep=t)
        np.savez_compressed(os.path.join(out_dir, f"refneuron_{name}.npz"), in_cells=data.cells,
                            in_particles=data.particles, in_aux=data.aux, out_cells=out.cells,
                            params=np.frombuffer(bytes(prm), np.uint8),
                            meta=np.array([seed, motion, t, world[0], world[1], ts, steps], np.int64))
        print(name, out.num_cells, ts)
    if os.environ.get("NEURON_ONLY"):
        return
    summary = {}
    for name, (builder, motion, steps) in LONG_RUNS.items():
        data, world = builder()
        prm = P.benchmark_parameters(motion)
        out, seconds, ts = refrun.run(data, world, prm, steps=steps)
        summary[name] = {"steps": steps, "motion": motion, "world": list(world), "initial": observables(data),
                         "final": observables(out)}
        print(name, summary[name]["final"])
    data, world, prm = decay_input()
    out, _, _ = refrun.run(data, world, prm, steps=1000)
    summary["decay"] = {"steps": 1000, "initial": observables(data), "final": observables(out)}
    print("decay", summary["decay"]["final"])
    with open(os.path.join(out_dir, "ref_observables.json"), "w") as f:
        json.dump(summary, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
