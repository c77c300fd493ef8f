"""Transfer objects: numpy views of the reference's DataTO layout.

The dtypes below are byte-for-byte the reference's ``CellTO`` (304 bytes),
``ParticleTO`` (40 bytes) and ``ConnectionTO`` (12 bytes) from
``source/EngineGpuKernels/TOs.cuh:10-193``; ``include/alien_b200.h`` pins the
same offsets with static asserts on the C side.  ``DataTO`` owns host arrays
and hands out the ``AlienDataTO`` pointer struct that the C ABI consumes
(``TOs.cuh:195-236``).
"""
from __future__ import annotations

import ctypes

import numpy as np

MAX_CELL_BONDS = 6
MAX_COLORS = 7

CONNECTION_TO = np.dtype({
    "names": ["cellIndex", "distance", "angleFromPrevious"],
    "formats": ["<i4", "<f4", "<f4"],
    "offsets": [0, 4, 8],
    "itemsize": 12,
})

CELL_TO = np.dtype({
    "names": [
        "id", "connections", "pos", "vel", "energy", "stiffness", "color", "maxConnections",
        "numConnections", "barrier", "age", "livingState", "creatureId", "mutationId",
        "ancestorMutationId", "genomeComplexity", "executionOrderNumber", "inputExecutionOrderNumber",
        "outputBlocked", "cellFunction", "cellFunctionData", "signalChannels", "signalOrigin",
        "signalTargetX", "signalTargetY", "activationTime", "detectedByCreatureId", "cellFunctionUsed",
        "metadataNameSize", "metadataNameDataIndex", "metadataDescriptionSize",
        "metadataDescriptionDataIndex", "selected",
    ],
    "formats": [
        "<u8", (CONNECTION_TO, (MAX_CELL_BONDS,)), ("<f4", (2,)), ("<f4", (2,)), "<f4", "<f4", "u1", "u1",
        "u1", "u1", "<u4", "<i4", "<u4", "<u4",
        "u1", "<f4", "u1", "i1",
        "u1", "<i4", ("<u8", (8,)), ("<f4", (8,)), "u1",
        "<f4", "<f4", "<u4", "<u2", "u1",
        "<u2", "<u8", "<u2",
        "<u8", "u1",
    ],
    "offsets": [
        0, 8, 80, 88, 96, 100, 104, 105,
        106, 107, 108, 112, 116, 120,
        124, 128, 132, 133,
        134, 136, 144, 208, 240,
        244, 248, 252, 256, 258,
        264, 272, 280,
        288, 296,
    ],
    "itemsize": 304,
})

PARTICLE_TO = np.dtype({
    "names": ["id", "energy", "pos", "vel", "color", "selected"],
    "formats": ["<u8", "<f4", ("<f4", (2,)), ("<f4", (2,)), "u1", "u1"],
    "offsets": [0, 8, 16, 24, 32, 33],
    "itemsize": 40,
})

# CellFunction_None, EngineInterface/CellFunctionConstants.h:21
CELL_FUNCTION_NONE = 11


class CDataTO(ctypes.Structure):
    """``AlienDataTO``: six pointers, the reference's DataTO."""

    _fields_ = [
        ("numCells", ctypes.POINTER(ctypes.c_uint64)),
        ("cells", ctypes.c_void_p),
        ("numParticles", ctypes.POINTER(ctypes.c_uint64)),
        ("particles", ctypes.c_void_p),
        ("numAuxiliaryData", ctypes.POINTER(ctypes.c_uint64)),
        ("auxiliaryData", ctypes.c_void_p),
    ]


def empty_cells(n: int) -> np.ndarray:
    """Cell TOs with the CellDescription defaults that the physics stage
    reads (EngineInterface/Descriptions.h:363-380)."""
    cells = np.zeros(n, dtype=CELL_TO)
    cells["stiffness"] = 1.0
    cells["energy"] = 100.0
    cells["cellFunction"] = CELL_FUNCTION_NONE
    cells["executionOrderNumber"] = 0
    cells["inputExecutionOrderNumber"] = -1
    return cells


def _grown(arr: np.ndarray, cap: int) -> np.ndarray:
    out = np.zeros(cap, arr.dtype)
    out[: len(arr)] = arr
    return out


class DataTO:
    """Host-side DataTO with owned numpy buffers (``DataTO::init``,
    TOs.cuh:204-215).  ``capacity`` sizes the arrays for egress."""

    def __init__(self, cells: np.ndarray | None = None, particles: np.ndarray | None = None,
                 aux: np.ndarray | None = None, cell_capacity: int | None = None,
                 particle_capacity: int | None = None, aux_capacity: int | None = None):
        cells = np.zeros(0, CELL_TO) if cells is None else np.ascontiguousarray(cells, dtype=CELL_TO)
        particles = (np.zeros(0, PARTICLE_TO) if particles is None
                     else np.ascontiguousarray(particles, dtype=PARTICLE_TO))
        aux = np.zeros(0, np.uint8) if aux is None else np.ascontiguousarray(aux, dtype=np.uint8)
        ncap = max(len(cells), cell_capacity or 0, 1)
        pcap = max(len(particles), particle_capacity or 0, 1)
        acap = max(len(aux), aux_capacity or 0, 1)
        self._cells = cells if len(cells) == ncap else _grown(cells, ncap)
        self._particles = particles if len(particles) == pcap else _grown(particles, pcap)
        self._aux = aux if len(aux) == acap else _grown(aux, acap)
        self._counts = np.array([len(cells), len(particles), len(aux)], dtype=np.uint64)
        self._c = CDataTO()
        base = self._counts.ctypes.data
        u64p = ctypes.POINTER(ctypes.c_uint64)
        self._c.numCells = ctypes.cast(base, u64p)
        self._c.numParticles = ctypes.cast(base + 8, u64p)
        self._c.numAuxiliaryData = ctypes.cast(base + 16, u64p)
        self._c.cells = self._cells.ctypes.data
        self._c.particles = self._particles.ctypes.data
        self._c.auxiliaryData = self._aux.ctypes.data

    @property
    def num_cells(self) -> int:
        return int(self._counts[0])

    @property
    def num_particles(self) -> int:
        return int(self._counts[1])

    @property
    def num_aux(self) -> int:
        return int(self._counts[2])

    @property
    def cells(self) -> np.ndarray:
        return self._cells[: self.num_cells]

    @property
    def particles(self) -> np.ndarray:
        return self._particles[: self.num_particles]

    @property
    def aux(self) -> np.ndarray:
        return self._aux[: self.num_aux]

    @property
    def cell_capacity(self) -> int:
        return len(self._cells)

    @property
    def particle_capacity(self) -> int:
        return len(self._particles)

    def c_ptr(self) -> ctypes.POINTER(CDataTO):
        return ctypes.pointer(self._c)

    def copy(self) -> "DataTO":
        return DataTO(self.cells.copy(), self.particles.copy(), self.aux.copy())

    def nbytes(self) -> int:
        return self.num_cells * CELL_TO.itemsize + self.num_particles * PARTICLE_TO.itemsize + self.num_aux
