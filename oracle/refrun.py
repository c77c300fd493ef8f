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


def run(data: DataTO, world, params: PhysicsParams, steps=1, warmup=0, timestep=0, timeout=1800):
    """returns (DataTO after warmup + steps, seconds of the timed steps, timestep)"""
    if not available():
        raise FileNotFoundError(f"{REF_RUN} not built")
    with tempfile.TemporaryDirectory() as d:
        inp, out = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        write_input(inp, data, world, params, timestep, warmup, steps)
        r = subprocess.run([REF_RUN, inp, out], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_run failed ({r.returncode}): {r.stderr.strip()[-500:]}")
        return read_output(out)
