"""ctypes binding of the CPU oracle (test infrastructure only).

Loaded by the tests, by ``__graft_entry__.smoke`` as the checker, and by the
benchmark's CPU-baseline leg.  The product path never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from alien_b200.params import PhysicsParams
from alien_b200.to import CELL_TO, PARTICLE_TO, DataTO

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load(name: str) -> ctypes.CDLL:
    path = os.path.join(LIB_DIR, name)
    if not os.path.exists(path):
        build()
    lib = ctypes.CDLL(path)
    lib.oracle_create.restype = ctypes.c_void_p
    lib.oracle_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(PhysicsParams), ctypes.c_uint64]
    lib.oracle_destroy.argtypes = [ctypes.c_void_p]
    lib.oracle_set_data.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.oracle_get_data.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.oracle_get_counts.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_uint64)] * 3
    lib.oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
    lib.oracle_set_parameters.argtypes = [ctypes.c_void_p, ctypes.POINTER(PhysicsParams)]
    lib.oracle_timestep.restype = ctypes.c_uint64
    lib.oracle_timestep.argtypes = [ctypes.c_void_p]
    lib.oracle_cell_slots.restype = ctypes.c_int64
    lib.oracle_cell_slots.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
    lib.oracle_num_threads.restype = ctypes.c_int
    lib.oracle_set_threads.argtypes = [ctypes.c_int]
    lib.oracle_neuron_activities.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.oracle_get_parameters.argtypes = [ctypes.c_void_p, ctypes.POINTER(PhysicsParams)]
    return lib


def available_cpus() -> int:
    """CPUs this process may use: the affinity mask, capped by a cgroup
    CPU quota when one is set"""
    n = len(os.sched_getaffinity(0))
    try:
        with open("/sys/fs/cgroup/cpu.max") as f:
            quota, period = f.read().split()[:2]
        if quota != "max":
            n = min(n, max(1, int(int(quota) // int(period))))
    except (OSError, ValueError):
        pass
    return max(1, n)


_LIBS: dict[str, ctypes.CDLL] = {}


def library(precision: str = "f64") -> ctypes.CDLL:
    name = {"f64": "liboracle_f64.so", "f32": "liboracle_f32.so", "f64mt": "liboracle_f64mt.so"}[precision]
    if name not in _LIBS:
        # OpenMP threads must not outnumber the CPUs: spinning waiters on an
        # oversubscribed host stall every barrier
        os.environ.setdefault("OMP_WAIT_POLICY", "PASSIVE")
        os.environ.setdefault("OMP_NUM_THREADS", str(available_cpus()))
        _LIBS[name] = _load(name)
        _LIBS[name].oracle_set_threads(available_cpus())
    return _LIBS[name]


class OracleSimulation:
    """Same call shape as the engine facade: set data, step, get data."""

    def __init__(self, world, params: PhysicsParams, timestep: int = 0, precision: str = "f64"):
        self.lib = library(precision)
        self.world = tuple(world)
        self._params = params.copy()
        self.h = self.lib.oracle_create(int(world[0]), int(world[1]), ctypes.byref(self._params), timestep)
        if not self.h:
            raise ValueError("oracle_create failed")

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_simulation_data(self, data: DataTO):
        self.lib.oracle_set_data(self.h, ctypes.cast(data.c_ptr(), ctypes.c_void_p))

    def set_simulation_parameters(self, params: PhysicsParams):
        self._params = params.copy()
        self.lib.oracle_set_parameters(self.h, ctypes.byref(self._params))

    def get_simulation_parameters(self) -> PhysicsParams:
        """the parameters as they stand after the steps so far: zones and
        radiation sources moved by their velocities, the external-energy
        pool after backflow"""
        out = PhysicsParams()
        self.lib.oracle_get_parameters(self.h, ctypes.byref(out))
        return out

    def calc_timesteps(self, n: int):
        self.lib.oracle_step(self.h, n)

    def current_timestep(self) -> int:
        return int(self.lib.oracle_timestep(self.h))

    def counts(self):
        c, p, a = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self.lib.oracle_get_counts(self.h, ctypes.byref(c), ctypes.byref(p), ctypes.byref(a))
        return c.value, p.value, a.value

    def get_simulation_data(self) -> DataTO:
        c, p, a = self.counts()
        out = DataTO(np.zeros(0, CELL_TO), np.zeros(0, PARTICLE_TO), None, cell_capacity=c,
                     particle_capacity=p, aux_capacity=a)
        self.lib.oracle_get_data(self.h, ctypes.cast(out.c_ptr(), ctypes.c_void_p))
        return out

    def neuron_activities(self) -> np.ndarray:
        """neuron cells that ran, per color, since creation"""
        out = np.zeros(7, np.uint64)
        self.lib.oracle_neuron_activities(self.h, out.ctypes.data)
        return out

    def cell_slots(self) -> np.ndarray:
        c, _, _ = self.counts()
        out = np.zeros(max(c, 1), np.int32)
        n = self.lib.oracle_cell_slots(self.h, out.ctypes.data, len(out))
        return out[:n]
