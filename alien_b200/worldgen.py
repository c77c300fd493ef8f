"""Seeded synthetic worlds in the reference's DataTO format.

The reference publishes no benchmark inputs; these generators build the
workloads its physics stage is measured on from seeded random numbers:

* ``rect_cluster`` / ``hex_patch`` restate DescriptionEditService::createRect
  and createHex (source/EngineInterface/DescriptionEditService.cpp:13-81):
  lattice cells at spacing 1.0, bonded by ``reconnect`` (the rule of
  DescriptionEditService::reconnectCells, :356-381, neighbours visited in
  order of distance) whose angles follow DataDescription::addConnection
  (source/EngineInterface/Descriptions.cpp:273-355).
* ``soft_body_world`` (10x10 lattices + energy particles, 512x512),
  ``fluid_world`` (1M unbonded cells, 2048x2048) and ``hex_world``
  (40k hexagonal 100-cell patches, 4096x4096) build the three single-world
  workloads; ``batched_worlds`` the 256-world mix.
"""
from __future__ import annotations

import math

import numpy as np

from .to import CELL_TO, PARTICLE_TO, DataTO, empty_cells

NEAR_ZERO = 1.0e-4


def angle_of_vector(dx: float, dy: float) -> float:
    """Math::angleOfVector (source/Base/Math.cpp:10-24): degrees, 0 = (0,-1)."""
    length = math.sqrt(dx * dx + dy * dy)
    if length < NEAR_ZERO:
        return 0.0
    s = math.degrees(math.asin(max(-1.0, min(1.0, -dy / length))))
    return 90.0 - s if dx >= 0.0 else s + 270.0


def _add_connection_one_way(conns, pos, cell, other):
    """One side of DataDescription::addConnection (Descriptions.cpp:278-349).
    ``conns[cell]`` is a list of [otherIndex, distance, angleFromPrevious]."""
    d = pos[other] - pos[cell]
    new_angle = angle_of_vector(d[0], d[1])
    dist = float(math.hypot(d[0], d[1]))
    lst = conns[cell]
    if not lst:
        lst.append([other, dist, 360.0])
        return
    if len(lst) == 1:
        dc = pos[lst[0][0]] - pos[cell]
        prev = angle_of_vector(dc[0], dc[1])
        diff = new_angle - prev
        if diff >= 0:
            lst[0][2] = 360.0 - diff
            lst.append([other, dist, diff])
        else:
            lst[0][2] = -diff
            lst.append([other, dist, 360.0 + diff])
        return
    df = pos[lst[0][0]] - pos[cell]
    angle = angle_of_vector(df[0], df[1])
    it = 1
    for _ in range(4 * len(lst) + 4):
        next_angle = angle + lst[it][2]
        if (angle < new_angle <= next_angle) or (angle < new_angle + 360.0 <= next_angle):
            break
        it += 1
        if it == len(lst):
            it = 0
        angle = next_angle
        if angle > 360.0:
            angle -= 360.0
    else:
        raise RuntimeError("addConnection: no angular gap found")
    diff1 = new_angle - angle
    if diff1 < 0:
        diff1 += 360.0
    diff2 = lst[it][2]
    factor = diff1 / diff2 if diff2 != 0 else 0.5
    lst.insert(it, [other, dist, diff2 * factor])
    nxt = it + 1
    if nxt == len(lst):
        nxt = 0
    lst[nxt][2] = diff2 * (1 - factor)


def reconnect(pos: np.ndarray, max_distance: float, max_connections: int):
    """DescriptionEditService::reconnectCells for one cluster template."""
    n = len(pos)
    conns = [[] for _ in range(n)]
    for i in range(n):
        d = np.hypot(pos[:, 0] - pos[i, 0], pos[:, 1] - pos[i, 1])
        near = [j for j in np.lexsort((np.arange(n), d)) if d[j] <= max_distance]
        for j in near:
            if j == i or len(conns[i]) >= max_connections or len(conns[j]) >= max_connections:
                continue
            if any(c[0] == j for c in conns[i]):
                continue
            _add_connection_one_way(conns, pos, i, j)
            _add_connection_one_way(conns, pos, j, i)
    return conns


def rect_cluster(width: int = 10, height: int = 10, spacing: float = 1.0) -> np.ndarray:
    """createRect cell positions (DescriptionEditService.cpp:17-20), centred."""
    pos = np.array([[i * spacing, j * spacing] for i in range(width) for j in range(height)], np.float64)
    return pos - pos.mean(axis=0)


def hex_patch(num_cells: int = 100, spacing: float = 1.0) -> np.ndarray:
    """``num_cells`` sites of a hexagonal lattice (the createHex geometry,
    DescriptionEditService.cpp:44-72) nearest to its centre, ties broken by
    angle; 100 is not a centred-hexagonal number, so the patch is the 100
    sites of the 7-layer hexagon (127 sites) closest to the centre."""
    layers = 7
    inc_y = math.sqrt(3.0) * spacing / 2.0
    sites = []
    for j in range(layers):
        for i in range(-(layers - 1), layers - j):
            sites.append((i * spacing + j * spacing / 2.0, -j * inc_y))
            if j > 0:
                sites.append((i * spacing + j * spacing / 2.0, j * inc_y))
    sites = np.array(sites, np.float64)
    r = np.hypot(sites[:, 0], sites[:, 1])
    ang = np.arctan2(sites[:, 1], sites[:, 0])
    order = np.lexsort((ang, np.round(r, 9)))
    patch = sites[order[:num_cells]]
    return patch - patch.mean(axis=0)


class ClusterTemplate:
    """Bonded cluster in local coordinates, replicated by translation."""

    def __init__(self, pos: np.ndarray, max_distance: float, max_connections: int = 6):
        self.pos = pos
        self.n = len(pos)
        conns = reconnect(pos, max_distance, max_connections)
        self.num = np.array([len(c) for c in conns], np.uint8)
        self.index = np.zeros((self.n, 6), np.int32)
        self.dist = np.zeros((self.n, 6), np.float32)
        self.angle = np.zeros((self.n, 6), np.float32)
        for i, c in enumerate(conns):
            for k, (j, d, a) in enumerate(c):
                self.index[i, k] = j
                self.dist[i, k] = d
                self.angle[i, k] = a
        self.radius = float(np.hypot(pos[:, 0], pos[:, 1]).max())


def _place_clusters_stratified(rng, count, world, radius):
    """Non-overlapping centres for large counts: ``count`` distinct cells of a
    grid of side 2*radius + 2, chosen uniformly at random, each with a
    uniform jitter that keeps the cluster inside its grid cell."""
    sx, sy = world
    d = 2.0 * radius + 2.0
    nx, ny = int(sx // d), int(sy // d)
    if nx * ny < count:
        raise RuntimeError("world too small for the clusters")
    pick = rng.choice(nx * ny, size=count, replace=False)
    gx, gy = pick % nx, pick // nx
    slack = d - (2.0 * radius + 1.0)
    cx = gx * d + radius + 0.5 + rng.uniform(0, slack, count)
    cy = gy * d + radius + 0.5 + rng.uniform(0, slack, count)
    return np.stack([cx, cy], axis=1)


def _place_clusters(rng, count, world, radius, max_tries=200):
    """Uniform cluster centres, rejecting overlaps (bins of side 2*radius);
    stratified placement beyond 2000 clusters."""
    if count > 2000:
        return _place_clusters_stratified(rng, count, world, radius)
    sx, sy = world
    min_d = 2.0 * radius + 1.0
    centres = np.zeros((count, 2), np.float64)
    grid = {}
    cell = min_d
    nbx, nby = max(1, int(sx // cell)), max(1, int(sy // cell))
    k = 0
    tries = 0
    while k < count:
        c = rng.uniform(0, 1, 2) * (sx, sy)
        bx, by = int(c[0] // cell) % nbx, int(c[1] // cell) % nby
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for o in grid.get(((bx + dx) % nbx, (by + dy) % nby), ()):
                    d = c - centres[o]
                    d -= np.round(d / (sx, sy)) * (sx, sy)
                    if d[0] * d[0] + d[1] * d[1] < min_d * min_d:
                        ok = False
                        break
                if not ok:
                    break
            if not ok:
                break
        tries += 1
        if tries > max_tries * count:
            raise RuntimeError("cannot place clusters without overlap")
        if ok:
            centres[k] = c
            grid.setdefault((bx, by), []).append(k)
            k += 1
    return centres


def _clusters_to_cells(tmpl: ClusterTemplate, centres, vel, omega, energy, first_id, world, creature_base=1):
    m = len(centres)
    n = tmpl.n
    cells = empty_cells(m * n)
    pos = (centres[:, None, :] + tmpl.pos[None, :, :]).reshape(-1, 2)
    pos = np.mod(pos, world)
    r = np.broadcast_to(tmpl.pos[None, :, :], (m, n, 2))
    v = vel[:, None, :] + omega[:, None, None] * np.stack([-r[..., 1], r[..., 0]], axis=-1)
    cells["id"] = np.arange(first_id, first_id + m * n, dtype=np.uint64)
    cells["pos"] = pos.astype(np.float32)
    cells["vel"] = v.reshape(-1, 2).astype(np.float32)
    cells["energy"] = energy
    cells["maxConnections"] = 6
    cells["numConnections"] = np.tile(tmpl.num, m)
    base = (np.arange(m, dtype=np.int64) * n)[:, None, None]
    idx = (tmpl.index[None, :, :] + base).reshape(-1, 6)
    mask = np.arange(6)[None, :] < np.tile(tmpl.num, m)[:, None]
    cells["connections"]["cellIndex"] = np.where(mask, idx, 0).astype(np.int32)
    cells["connections"]["distance"] = np.where(mask, np.tile(tmpl.dist, (m, 1)), 0)
    cells["connections"]["angleFromPrevious"] = np.where(mask, np.tile(tmpl.angle, (m, 1)), 0)
    cells["creatureId"] = np.repeat(np.arange(creature_base, creature_base + m, dtype=np.uint32), n)
    return cells


def _particles(rng, count, world, first_id, energy=1.0, vmax=0.1):
    parts = np.zeros(count, PARTICLE_TO)
    parts["id"] = np.arange(first_id, first_id + count, dtype=np.uint64)
    parts["pos"] = (rng.uniform(0, 1, (count, 2)) * world).astype(np.float32)
    parts["vel"] = rng.uniform(-vmax, vmax, (count, 2)).astype(np.float32)
    parts["energy"] = energy
    return parts


_RECT = None
_HEX = None


def rect_template() -> ClusterTemplate:
    global _RECT
    if _RECT is None:
        _RECT = ClusterTemplate(rect_cluster(10, 10, 1.0), max_distance=1.1)
    return _RECT


def hex_template() -> ClusterTemplate:
    global _HEX
    if _HEX is None:
        _HEX = ClusterTemplate(hex_patch(100, 1.0), max_distance=1.5)
    return _HEX


def soft_body_world(seed: int = 0, world=(512, 512), clusters: int = 200, particles: int = 20000,
                    particle_energy: float = 1.0):
    """Plain single world, small: 200 10x10 square-lattice clusters (4-neighbour
    bonds, rest distance 1.0, energy 100), velocities U[-0.1,0.1], plus 20k
    energy particles (energy 1.0: the workload leaves it unspecified)."""
    rng = np.random.default_rng(seed)
    tmpl = rect_template()
    centres = _place_clusters(rng, clusters, world, tmpl.radius)
    vel = rng.uniform(-0.1, 0.1, (clusters, 2))
    cells = _clusters_to_cells(tmpl, centres, vel, np.zeros(clusters), 100.0, 1, world)
    parts = _particles(rng, particles, world, 1 + len(cells), particle_energy, 0.1)
    return DataTO(cells, parts), world


def fluid_world(seed: int = 0, world=(2048, 2048), cells: int = 1_000_000, sigma: float = 0.5,
                energy: float = 50.0, spatially_sorted: bool = True):
    """SPH fluid stress: unbonded cells (maxConnections 0, the CellDescription
    default), uniform positions, Gaussian velocities, energy 50."""
    rng = np.random.default_rng(seed)
    c = empty_cells(cells)
    pos = rng.uniform(0, 1, (cells, 2)) * world
    if spatially_sorted:
        key = np.floor(pos[:, 1]).astype(np.int64) * world[0] + np.floor(pos[:, 0]).astype(np.int64)
        pos = pos[np.argsort(key, kind="stable")]
    c["id"] = np.arange(1, cells + 1, dtype=np.uint64)
    c["pos"] = pos.astype(np.float32)
    c["vel"] = rng.normal(0.0, sigma, (cells, 2)).astype(np.float32)
    c["energy"] = energy
    c["maxConnections"] = 0
    return DataTO(c, None), world


def hex_world(seed: int = 0, world=(4096, 4096), clusters: int = 40000, vmax: float = 0.5,
              omega_max: float = 0.02):
    """Soft-body heavy: hexagonal 100-cell patches (up to 6 bonds, rest
    distance 1.0), rigid velocity U[-0.5,0.5]^2 plus angular velocity
    U[-0.02,0.02] rad/step (v_i = v + omega x r_i)."""
    rng = np.random.default_rng(seed)
    tmpl = hex_template()
    centres = _place_clusters(rng, clusters, world, tmpl.radius)
    vel = rng.uniform(-vmax, vmax, (clusters, 2))
    omega = rng.uniform(-omega_max, omega_max, clusters)
    cells = _clusters_to_cells(tmpl, centres, vel, omega, 100.0, 1, world)
    return DataTO(cells, None), world


def mixed_world(seed: int, num_cells: int, density: float = 0.2, fluid_fraction: float = 0.5):
    """One world of the batched workload: side scaled to the density, half
    free fluid cells and half 10x10 lattice clusters."""
    rng = np.random.default_rng(seed)
    side = max(32, int(math.ceil(math.sqrt(num_cells / density))))
    world = (side, side)
    tmpl = rect_template()
    n_clusters = max(1, int(round(num_cells * (1 - fluid_fraction) / tmpl.n)))
    centres = _place_clusters(rng, n_clusters, world, tmpl.radius)
    vel = rng.uniform(-0.1, 0.1, (n_clusters, 2))
    cl = _clusters_to_cells(tmpl, centres, vel, np.zeros(n_clusters), 100.0, 1, world)
    n_free = max(0, num_cells - len(cl))
    free = empty_cells(n_free)
    free["id"] = np.arange(1 + len(cl), 1 + len(cl) + n_free, dtype=np.uint64)
    free["pos"] = (rng.uniform(0, 1, (n_free, 2)) * world).astype(np.float32)
    free["vel"] = rng.normal(0.0, 0.5, (n_free, 2)).astype(np.float32)
    free["energy"] = 50.0
    free["maxConnections"] = 0
    return DataTO(np.concatenate([cl, free]), None), world


def batched_sizes(seed: int = 0, count: int = 256, lo: int = 1000, hi: int = 200_000):
    """Log-uniform world sizes in [lo, hi]."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(math.log(lo), math.log(hi), count)).astype(np.int64)


def random_test_world(seed: int, world=(64, 64), clusters: int = 6, free_cells: int = 150,
                      particles: int = 60, hex_clusters: int = 2, vmax: float = 0.6,
                      free_max_connections: int = 6, barriers: int = 0):
    """Small mixed world for parity tests: lattice and hex clusters, free
    cells that can fuse (maxConnections 6, speeds up to ``vmax``), energy
    particles and optional barrier cells."""
    rng = np.random.default_rng(seed)
    parts_list = []
    next_id = 1
    rect = rect_template()
    hexa = hex_template()
    all_cells = []
    offset = 0
    items = [(rect, clusters), (hexa, hex_clusters)]
    centres_all = _place_clusters(rng, clusters + hex_clusters, world, max(rect.radius, hexa.radius))
    ci = 0
    for tmpl, count in items:
        if count == 0:
            continue
        centres = centres_all[ci:ci + count]
        ci += count
        vel = rng.uniform(-vmax, vmax, (count, 2))
        omega = rng.uniform(-0.02, 0.02, count)
        c = _clusters_to_cells(tmpl, centres, vel, omega, rng.uniform(60, 140), next_id, world,
                               creature_base=1 + len(all_cells))
        c["connections"]["cellIndex"] += np.where(
            np.arange(6)[None, :] < c["numConnections"][:, None], offset, 0).astype(np.int32)
        c["stiffness"] = rng.uniform(0.5, 1.0)
        next_id += len(c)
        offset += len(c)
        all_cells.append(c)
    free = empty_cells(free_cells)
    free["id"] = np.arange(next_id, next_id + free_cells, dtype=np.uint64)
    free["pos"] = (rng.uniform(0, 1, (free_cells, 2)) * world).astype(np.float32)
    free["vel"] = rng.uniform(-vmax, vmax, (free_cells, 2)).astype(np.float32)
    free["energy"] = rng.uniform(40, 120, free_cells).astype(np.float32)
    free["maxConnections"] = free_max_connections
    free["color"] = rng.integers(0, 7, free_cells)
    if barriers:
        free["barrier"][:barriers] = 1
        free["vel"][:barriers] = 0
    next_id += free_cells
    all_cells.append(free)
    cells = np.concatenate(all_cells)
    parts = _particles(rng, particles, world, next_id, energy=1.0, vmax=0.5)
    parts["energy"] = rng.uniform(0.005, 3.0, particles).astype(np.float32)
    parts_list.append(parts)
    return DataTO(cells, np.concatenate(parts_list)), world


def _separated_points(rng, count, world, occupied: np.ndarray, min_sep: float, max_tries: int = 200):
    """uniform points at least ``min_sep`` from each other and from ``occupied``"""
    sx, sy = world
    pts = [p for p in occupied]
    out = []
    cell = max(min_sep, 1.0)
    nbx, nby = max(1, int(sx // cell)), max(1, int(sy // cell))
    grid = {}

    def key(p):
        return int(p[0] // cell) % nbx, int(p[1] // cell) % nby

    for i, p in enumerate(pts):
        grid.setdefault(key(p), []).append(p)
    tries = 0
    while len(out) < count:
        tries += 1
        if tries > max_tries * max(count, 1):
            raise RuntimeError("cannot place separated points")
        c = rng.uniform(0, 1, 2) * (sx, sy)
        bx, by = key(c)
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for q in grid.get(((bx + dx) % nbx, (by + dy) % nby), ()):
                    d = c - q
                    d -= np.round(d / (sx, sy)) * (sx, sy)
                    if d[0] * d[0] + d[1] * d[1] < min_sep * min_sep:
                        ok = False
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            out.append(c)
            grid.setdefault((bx, by), []).append(c)
    return np.array(out, np.float64).reshape(-1, 2)


def calm_test_world(seed: int, world=(64, 64), clusters: int = 4, hex_clusters: int = 1, free_cells: int = 120,
                    particles: int = 20, vmax: float = 0.05, particle_speed: float = 0.3):
    """A world in which no lock, no random draw and no in-place update of the
    reference can change the outcome of a step: slow objects (no fusion, no
    force decay), free cells and particles at least 1.5 apart from everything,
    energies above cellMinEnergy.  Used to pin the oracle against the
    reference engine step for step."""
    rng = np.random.default_rng(seed)
    rect, hexa = rect_template(), hex_template()
    centres = _place_clusters(rng, clusters + hex_clusters, world, max(rect.radius, hexa.radius) + 1.0)
    parts_cells = []
    next_id, offset = 1, 0
    for tmpl, cs in ((rect, centres[:clusters]), (hexa, centres[clusters:])):
        if len(cs) == 0:
            continue
        c = _clusters_to_cells(tmpl, cs, rng.uniform(-vmax, vmax, (len(cs), 2)), rng.uniform(-0.005, 0.005, len(cs)),
                               100.0, next_id, world, creature_base=1 + len(parts_cells))
        c["connections"]["cellIndex"] += np.where(np.arange(6)[None, :] < c["numConnections"][:, None], offset, 0).astype(np.int32)
        next_id += len(c)
        offset += len(c)
        parts_cells.append(c)
    cluster_cells = np.concatenate(parts_cells)
    occupied = cluster_cells["pos"].astype(np.float64)
    free_pos = _separated_points(rng, free_cells, world, occupied, 1.5)
    free = empty_cells(free_cells)
    free["id"] = np.arange(next_id, next_id + free_cells, dtype=np.uint64)
    free["pos"] = free_pos.astype(np.float32)
    free["vel"] = rng.uniform(-vmax, vmax, (free_cells, 2)).astype(np.float32)
    free["energy"] = rng.uniform(60, 120, free_cells).astype(np.float32)
    free["maxConnections"] = 6
    next_id += free_cells
    cells = np.concatenate([cluster_cells, free])
    ppos = _separated_points(rng, particles, world, cells["pos"].astype(np.float64), 3.0)
    parts = np.zeros(particles, PARTICLE_TO)
    parts["id"] = np.arange(next_id, next_id + particles, dtype=np.uint64)
    parts["pos"] = ppos.astype(np.float32)
    parts["vel"] = rng.uniform(-particle_speed, particle_speed, (particles, 2)).astype(np.float32)
    parts["energy"] = rng.uniform(0.5, 2.0, particles).astype(np.float32)
    return DataTO(cells, parts), world


def add_neurons(data: DataTO, seed: int, fraction: float = 0.5, cells: np.ndarray | None = None,
                num_orders: int = 6) -> DataTO:
    """Turns a share of the bonded cells into neuron cells (CellFunction_Neuron)
    with their weights and biases in the auxiliary data
    (NeuronTO.weightsAndBiasesDataIndex, TOs.cuh:45-49): weights ~ N(0, 0.5),
    biases ~ N(0, 0.1), random activation functions and execution order
    numbers, and random initial signals on every cell so that inputs carry
    something.  ``cells`` selects the candidate cells (default: all bonded)."""
    rng = np.random.default_rng(seed)
    c = data.cells.copy()
    n = len(c)
    cand = np.nonzero(c["numConnections"] > 0)[0] if cells is None else np.asarray(cells)
    pick = cand[rng.random(len(cand)) < fraction]
    c["executionOrderNumber"] = rng.integers(0, num_orders, n).astype(np.uint8)
    c["inputExecutionOrderNumber"] = rng.integers(-1, num_orders, n).astype(np.int8)
    c["outputBlocked"] = (rng.random(n) < 0.1).astype(np.uint8)
    c["signalChannels"] = rng.normal(0.0, 1.0, (n, 8)).astype(np.float32)
    sensor = rng.random(n) < 0.2
    c["signalOrigin"] = sensor.astype(np.uint8)
    c["signalTargetX"] = np.where(sensor, rng.uniform(-50, 50, n), 0).astype(np.float32)
    c["signalTargetY"] = np.where(sensor, rng.uniform(-50, 50, n), 0).astype(np.float32)
    c["cellFunctionUsed"] = 0
    aux_old = data.aux
    stride = 8 * 9 * 4
    base = len(aux_old)
    aux = np.zeros(base + stride * len(pick), np.uint8)
    aux[:base] = aux_old
    for r, i in enumerate(pick):
        wb = np.concatenate([rng.normal(0.0, 0.5, 64), rng.normal(0.0, 0.1, 8)]).astype(np.float32)
        aux[base + r * stride: base + (r + 1) * stride] = wb.view(np.uint8)
        c["cellFunction"][i] = 0
        fd = np.zeros(8, np.uint64)
        fd[0] = base + r * stride
        acts = rng.integers(0, 5, 8).astype(np.int32)
        fd.view(np.uint8)[8:40] = acts.view(np.uint8)
        c["cellFunctionData"][i] = fd
    return DataTO(c, data.particles.copy(), aux)
