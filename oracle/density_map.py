"""CPU restatement of the reference's DensityMap (TEST INFRASTRUCTURE: only
tests compare the engine with it; the engine never calls it).

DensityMap (source/EngineGpuKernels/DensityMap.cuh:8-230) is filled in every
step of the reference: cleared at SimulationKernels.cu:33, and
DensityMap::addCell (DensityMap.cuh:150-205) is called for every cell in the
pair-force kernels (SimulationKernels.cu:39, :47), at the cell's position
after its own overlap correction.  Slots are 8 x 8
(PreprocessedSimulationData.cuh:13); the map holds packed byte counters that
are added as 64-bit (or 32-bit) integers, so counts above 255 carry into the
next byte lane exactly as here (numpy uint64 arithmetic wraps the same way).

Pinned by tests/golden/ref_density_*.npz, the reference engine's own maps
after one step (written by tests/golden/make_golden.py).
"""
from __future__ import annotations

import numpy as np

SLOT = 8  # PreprocessedSimulationData.cuh:13
MAX_COLORS = 7
FIELDS = ("color", "otherMutant", "sameMutant1", "sameMutant2", "specificMutant", "lessComplexity1",
          "lessComplexity2", "moreComplexity1", "moreComplexity2")
LANES = np.uint64(0x0101010101010101)


def _clz32(v: np.ndarray) -> np.ndarray:
    """leading zeros of the 32-bit pattern of v (__clz)"""
    u = v.astype(np.int64) & 0xFFFFFFFF
    out = np.full(u.shape, 32, np.int64)
    nz = u != 0
    out[nz] = 32 - np.floor(np.log2(u[nz].astype(np.float64))).astype(np.int64) - 1
    return out


def density_map(pos: np.ndarray, color: np.ndarray, mutation_id: np.ndarray, genome_complexity: np.ndarray, world,
                timestep: int) -> dict:
    """the map addCell builds for cells at pos (n x 2, FP32) at the given
    timestep; returns field -> (sizeY, sizeX) array"""
    sx, sy = int(world[0]) // SLOT, int(world[1]) // SLOT
    out = {f: np.zeros(sx * sy, np.uint32 if f == "specificMutant" else np.uint64) for f in FIELDS}
    if sx * sy == 0 or len(pos) == 0:
        return {f: v.reshape(sy, sx) for f, v in out.items()}
    p = np.asarray(pos, np.float32)
    # toInt (Base.cuh:29-32) truncates; the flattened index is checked (DensityMap.cuh:152-153)
    ix = np.trunc(p[:, 0]).astype(np.int64) // 1
    iy = np.trunc(p[:, 1]).astype(np.int64) // 1
    # C++ integer division truncates toward zero
    ix = np.where(ix >= 0, ix // SLOT, -((-ix) // SLOT))
    iy = np.where(iy >= 0, iy // SLOT, -((-iy) // SLOT))
    index = ix + iy * sx
    keep = (index >= 0) & (index < sx * sy)
    index = index[keep]
    col = (np.asarray(color)[keep].astype(np.int64)) % MAX_COLORS
    mid = np.asarray(mutation_id, np.uint64)[keep]
    gc = np.asarray(genome_complexity, np.float32)[keep]

    def add(field, idx, values):
        np.add.at(out[field], idx, values.astype(out[field].dtype))

    add("color", index, (np.uint64(1) << (col.astype(np.uint64) * np.uint64(8))) | (np.uint64(1) << np.uint64(56)))
    zero, one = mid == 0, mid == 1
    add("specificMutant", index[zero], np.full(int(zero.sum()), 1, np.uint32))
    add("specificMutant", index[one], np.full(int(one.sum()), 0x100, np.uint32))
    rest = ~(zero | one)
    ir, mr, gr = index[rest], mid[rest], gc[rest]
    other = (mr + np.uint64(timestep // 23)) % np.uint64(8)  # calcOtherMutantsBucket, :208-211
    add("otherMutant", ir, LANES ^ (np.uint64(1) << (other * np.uint64(8))))
    b1, b2, b3 = mr % np.uint64(3), mr % np.uint64(5), mr % np.uint64(7)
    add("sameMutant1", ir, (np.uint64(1) << (b1 * np.uint64(8))) | (np.uint64(1) << ((b2 + np.uint64(3)) * np.uint64(8))))
    add("sameMutant2", ir, np.uint64(1) << (b3 * np.uint64(8)))
    # bucket = 32 - __clz(toInt(genomeComplexity * 10)) (:169, convertGenomeComplexityToIntValue :214)
    value = (gr * np.float32(10.0)).astype(np.float32)
    bucket = 32 - _clz32(np.trunc(value).astype(np.int64))
    lo = bucket < 8
    mid_b = (bucket >= 8) & (bucket < 16)
    bl = bucket[lo].astype(np.uint64)
    # lanes bucket..7 (the shift-or loop of :174-177), lanes 0..bucket (:182-185)
    add("lessComplexity1", ir[lo], LANES << (bl * np.uint64(8)))
    add("lessComplexity2", ir[lo], np.full(int(lo.sum()), LANES, np.uint64))
    add("moreComplexity1", ir[lo], LANES >> ((np.uint64(7) - bl) * np.uint64(8)))
    bm = (bucket[mid_b] - 8).astype(np.uint64)
    add("lessComplexity2", ir[mid_b], LANES << (bm * np.uint64(8)))
    add("moreComplexity2", ir[mid_b], LANES >> ((np.uint64(7) - bm) * np.uint64(8)))
    add("moreComplexity1", ir[mid_b], np.full(int(mid_b.sum()), LANES, np.uint64))
    return {f: v.reshape(sy, sx) for f, v in out.items()}


def from_cells(cells: np.ndarray, world, timestep: int) -> dict:
    """the map of CellTO records at their positions"""
    return density_map(cells["pos"], cells["color"], cells["mutationId"], cells["genomeComplexity"], world, timestep)
