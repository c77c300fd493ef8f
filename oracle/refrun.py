"""Driver of oracle/_ref/ref_run: the reference's own CUDA engine stepped from
a given DataTO (test infrastructure; reference arm of the benchmark)."""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess
import tempfile

import numpy as np

from alien_b200.params import PhysicsParams
from alien_b200.to import CELL_TO, PARTICLE_TO, DataTO

HERE = os.path.dirname(os.path.abspath(__file__))
REF_RUN = os.path.join(HERE, "_ref", "ref_run")


def available() -> bool:
    return os.path.exists(REF_RUN)


def write_input(path, data: DataTO, world, params: PhysicsParams, timestep=0, warmup=0, steps=1):
    with open(path, "wb") as f:
        f.write(b"ALRF")
        f.write(struct.pack("<Iiiqqq", 1, int(world[0]), int(world[1]), int(timestep), int(warmup), int(steps)))
        f.write(bytes(params))
        f.write(struct.pack("<QQQ", data.num_cells, data.num_particles, data.num_aux))
        f.write(data.cells.tobytes())
        f.write(data.particles.tobytes())
        f.write(data.aux.tobytes())


def read_output(path):
    with open(path, "rb") as f:
        raw = f.read()
    assert raw[:4] == b"ALRO", "bad output file"
    _, nc, np_, na, seconds, ts = struct.unpack_from("<IQQQdQ", raw, 4)
    off = 4 + struct.calcsize("<IQQQdQ")
    cells = np.frombuffer(raw, CELL_TO, nc, off).copy()
    off += nc * CELL_TO.itemsize
    parts = np.frombuffer(raw, PARTICLE_TO, np_, off).copy()
    off += np_ * PARTICLE_TO.itemsize
    aux = np.frombuffer(raw, np.uint8, na, off).copy()
    return DataTO(cells, parts, aux), seconds, ts


# Largest cell count the reference engine can hold in one world.  Its
# dynamic-memory bound (SimulationData::resizeObjects, SimulationData.cu:93)
# is an int: 336 bytes x (cell array size + 1000), where the cell array is
# 3 x (300000 + requested cells) after the facade's first resize
# (SimulationData.cu:51-56, 121-126).  Above 6,391,320 array entries the
# product wraps; a 4M-cell world then gets a dynamic memory of about 40 MB
# instead of 4.3 GB, and its first step ended in cudaErrorLaunchFailure
# (an out-of-bounds access inside the reference's kernels).  Such worlds
# are refused here before the reference engine ever sees them.
REF_MAX_CELLS = (2**31 - 1) // 336 - 1000
REF_MAX_CELLS = REF_MAX_CELLS // 3 - 300000


DENSITY_MAP_NAMES = ("color", "otherMutant", "sameMutant1", "sameMutant2", "specificMutant", "lessComplexity1",
                     "lessComplexity2", "moreComplexity1", "moreComplexity2")


def read_density_map(path):
    """the reference's DensityMap arrays as its last step filled them
    (DensityMap.cuh:8-230): name -> (sizeY, sizeX) array"""
    with open(path, "rb") as f:
        raw = f.read()
    assert raw[:4] == b"ALDM", "bad density map file"
    sx, sy = struct.unpack_from("<ii", raw, 4)
    off, out = 12, {}
    for name in DENSITY_MAP_NAMES:
        dt = np.uint32 if name == "specificMutant" else np.uint64
        out[name] = np.frombuffer(raw, dt, sx * sy, off).reshape(sy, sx).copy()
        off += sx * sy * np.dtype(dt).itemsize
    return out


def run(data: DataTO, world, params: PhysicsParams, steps=1, warmup=0, timestep=0, timeout=1800, density_map=False):
    """returns (DataTO after warmup + steps, seconds of the timed steps, timestep), and with density_map the
    reference's density map of the last step as a fourth element"""
    if not available():
        raise FileNotFoundError(f"{REF_RUN} not built")
    if data.num_cells > REF_MAX_CELLS:
        raise ValueError(f"the reference engine holds at most {REF_MAX_CELLS} cells in one world "
                         f"(int overflow of its dynamic-memory bound), got {data.num_cells}")
    with tempfile.TemporaryDirectory() as d:
        inp, out, dm = os.path.join(d, "in.bin"), os.path.join(d, "out.bin"), os.path.join(d, "dm.bin")
        write_input(inp, data, world, params, timestep, warmup, steps)
        r = subprocess.run([REF_RUN, inp, out] + ([dm] if density_map else []), capture_output=True, text=True,
                           timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_run failed ({r.returncode}): {r.stderr.strip()[-500:]}")
        if density_map:
            return read_output(out) + (read_density_map(dm),)
        return read_output(out)
