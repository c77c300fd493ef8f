"""Rigidity clusters (ClusterProcessor.cuh:8-168): in every third step, after
friction, the velocity of each cell of a bonded cluster is blended with
weight rigidity * stiffness^2 into the rigid-body velocity of its cluster
(mean velocity plus the rotation that carries the cluster's angular
momentum), rigidity from the base value or a zone.

The CPU part checks the oracle's pass against the rigid projection computed
here in numpy; the GPU part compares the CUDA engine with the FP64 oracle,
including a cluster across the torus seam, a chain whose labels need more
rounds than the propagation runs, and rigidity switched on by
set_simulation_parameters."""
import numpy as np
import pytest

from alien_b200 import params as P
from alien_b200 import worldgen
from alien_b200.to import DataTO
from oracle.oracle import OracleSimulation
from tests.helpers import compare_cells, compare_particles


def cluster_world(centres, world=(64, 64), seed=0, stiffness=1.0, template=None):
    """rect clusters at ``centres`` with random velocity noise, so that the
    velocity field is not rigid already"""
    rng = np.random.default_rng(seed)
    tmpl = template or worldgen.rect_template()
    centres = np.asarray(centres, np.float64)
    vel = rng.uniform(-0.2, 0.2, (len(centres), 2))
    omega = rng.uniform(-0.02, 0.02, len(centres))
    cells = worldgen._clusters_to_cells(tmpl, centres, vel, omega, 100.0, 1, world)
    cells["vel"] += rng.uniform(-0.05, 0.05, cells["vel"].shape).astype(np.float32)
    cells["stiffness"] = stiffness
    return DataTO(cells), world


def chain_world(n=150, world=(8192, 64), seed=0):
    """one chain of ``n`` cells along x, stored in random order: the smallest
    storage index sits somewhere inside the chain"""
    rng = np.random.default_rng(seed)
    pos = np.stack([np.arange(n, dtype=np.float64) - n / 2, np.zeros(n)], axis=1)
    perm = rng.permutation(n)
    tmpl = worldgen.ClusterTemplate(pos[perm], 1.1, 2)
    cells = worldgen._clusters_to_cells(tmpl, np.array([[world[0] / 2, world[1] / 2]]), np.zeros((1, 2)), np.zeros(1),
                                        100.0, 1, world)
    cells["vel"] = rng.uniform(-0.1, 0.1, cells["vel"].shape).astype(np.float32)
    cells["stiffness"] = 1.0
    return DataTO(cells), world


def rigid_params(rigidity, motion=P.MOTION_FLUID):
    prm = P.benchmark_parameters(motion)
    prm.rigidity = rigidity
    for z in prm.zones:
        z.rigidity = rigidity
    return prm


def oracle_step(data, world, prm, t, steps=1):
    o = OracleSimulation(world, prm, t)
    o.set_simulation_data(data)
    o.calc_timesteps(steps)
    out = o.get_simulation_data()
    o.close()
    return out


def rigid_projection(cells, world, k):
    """ClusterProcessor's blend for one cluster, in FP64: offsets from the
    first cell by minimal image, mean velocity, angular velocity in degrees"""
    pos = cells["pos"].astype(np.float64)
    vel = cells["vel"].astype(np.float64)
    W, H = world
    rel = pos - pos[0]
    rel[:, 0] -= np.round(rel[:, 0] / W) * W
    rel[:, 1] -= np.round(rel[:, 1] / H) * H
    r = rel - rel.mean(axis=0)
    cv = vel.mean(axis=0)
    dv = vel - cv
    mass = np.sum(r[:, 0] ** 2 + r[:, 1] ** 2)
    mom = np.sum(r[:, 0] * dv[:, 1] - r[:, 1] * dv[:, 0])
    av = mom / mass * 180.0 / np.pi
    tangential = np.stack([cv[0] - av * r[:, 1] * np.pi / 180.0, cv[1] + av * r[:, 0] * np.pi / 180.0], axis=1)
    return vel * (1 - k[:, None]) + tangential * k[:, None]


@pytest.mark.parametrize("centre", [(32.0, 32.0), (0.5, 63.0)])
def test_oracle_rigidity_is_the_rigid_projection(centre):
    """with rigidity 0.7 the step's final velocities are the rigidity-free
    step's velocities blended into the rigid-body motion (stiffness 0.8, so
    weight 0.7 * 0.64); in steps with T % 3 != 0 nothing changes"""
    data, world = cluster_world([centre], stiffness=0.8)
    free = oracle_step(data, world, rigid_params(0.0), 0)
    rigid = oracle_step(data, world, rigid_params(0.7), 0)
    f = free.cells[np.argsort(free.cells["id"])]
    g = rigid.cells[np.argsort(rigid.cells["id"])]
    assert np.array_equal(f["pos"], g["pos"])
    want = rigid_projection(f, world, np.full(len(f), 0.7 * 0.8 * 0.8))
    np.testing.assert_allclose(g["vel"].astype(np.float64), want, rtol=0, atol=2e-7)
    assert np.abs(g["vel"] - f["vel"]).max() > 1e-3
    later = oracle_step(data, world, rigid_params(0.7), 1)
    same = oracle_step(data, world, rigid_params(0.0), 1)
    assert np.array_equal(later.cells["vel"], same.cells["vel"])


def test_oracle_rigidity_keeps_clusters_apart_and_conserves_momentum():
    data, world = cluster_world([(16.0, 16.0), (46.0, 40.0)], seed=3)
    free = oracle_step(data, world, rigid_params(0.0), 3)
    rigid = oracle_step(data, world, rigid_params(1.0), 3)
    n = worldgen.rect_template().n
    for part in (slice(0, n), slice(n, 2 * n)):
        f = free.cells[np.argsort(free.cells["id"])][part]
        g = rigid.cells[np.argsort(rigid.cells["id"])][part]
        np.testing.assert_allclose(g["vel"].astype(np.float64), rigid_projection(f, world, np.ones(n)), atol=2e-7)
        np.testing.assert_allclose(g["vel"].astype(np.float64).sum(axis=0), f["vel"].astype(np.float64).sum(axis=0),
                                   atol=2e-6)


def test_zone_rigidity_is_blended():
    """rigidity 0 in the base and 1 in a zone's core: cells far outside the
    zone keep the rigidity-free velocities"""
    data, world = cluster_world([(16.0, 16.0), (48.0, 48.0)], seed=4)
    prm = rigid_params(0.0)
    prm.numZones = 1
    z = P.default_zone(prm.zones[0], prm)
    z.posX, z.posY, z.coreRadius, z.fadeoutRadius = 16.0, 16.0, 10.0, 5.0
    z.rigidityActivated, z.rigidity = 1, 1.0
    free = oracle_step(data, world, rigid_params(0.0), 0)
    rigid = oracle_step(data, world, prm, 0)
    n = worldgen.rect_template().n
    f = free.cells[np.argsort(free.cells["id"])]
    g = rigid.cells[np.argsort(rigid.cells["id"])]
    assert np.abs(g["vel"][:n] - f["vel"][:n]).max() > 1e-3
    assert np.array_equal(g["vel"][n:], f["vel"][n:])


# ---- the CUDA engine against the oracle (GPU) ---------------------------------------------------

def run_both(data, world, prm, steps, timestep=0, new_params=None):
    from alien_b200.facade import SimulationFacade

    eng = SimulationFacade()
    eng.new_simulation(timestep, world, prm if new_params is None else rigid_params(0.0, prm.motionType))
    eng.set_simulation_data(data)
    if new_params is not None:
        eng.set_simulation_parameters(prm)
    eng.calc_timesteps(steps)
    got = eng.get_simulation_data()
    eng.close_simulation()
    return got, oracle_step(data, world, prm, timestep, steps)


@pytest.mark.gpu
@pytest.mark.parametrize("motion", [P.MOTION_FLUID, P.MOTION_COLLISION])
@pytest.mark.parametrize("steps", [1, 4])
def test_rigidity_matches_oracle(motion, steps):
    data, world = worldgen.random_test_world(61, world=(96, 96), clusters=8, hex_clusters=3, free_cells=300,
                                             particles=80)
    prm = rigid_params(0.4, motion)
    prm.numZones = 1
    z = P.default_zone(prm.zones[0], prm)
    z.posX, z.posY, z.coreRadius, z.fadeoutRadius = 30.0, 60.0, 20.0, 15.0
    z.rigidityActivated, z.rigidity = 1, 0.9
    got, ref = run_both(data, world, prm, steps)
    rtol = 1e-5 if steps == 1 else 5e-5
    compare_cells(got.cells, ref.cells, world, rtol=rtol, before=data.cells)
    compare_particles(got.particles, ref.particles, world, rtol=rtol, before=data.particles)


@pytest.mark.gpu
def test_rigidity_across_the_seam_matches_oracle():
    data, world = cluster_world([(0.5, 63.0), (40.0, 0.2)], seed=5, stiffness=0.9)
    got, ref = run_both(data, world, rigid_params(0.8), 1)
    compare_cells(got.cells, ref.cells, world, before=data.cells)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [150, 5000])
def test_rigidity_chains_match_oracle(n):
    """chains stored in random order: 150 cells converge to one cluster in
    8 rounds; 5000 cells need 14, so their labels stop after the last of the
    12 rounds before they meet, in the engine as in the oracle"""
    data, world = chain_world(n=n, world=(8192, 64))
    got, ref = run_both(data, world, rigid_params(1.0), 1)
    compare_cells(got.cells, ref.cells, world, before=data.cells)


@pytest.mark.gpu
def test_rigidity_switched_on_by_new_parameters():
    """an engine created without rigidity gets it from set_simulation_parameters
    (the arena is rebuilt with the cluster arrays)"""
    data, world = cluster_world([(20.0, 20.0), (44.0, 40.0)], seed=6)
    got, ref = run_both(data, world, rigid_params(0.6), 1, new_params=True)
    compare_cells(got.cells, ref.cells, world, before=data.cells)
