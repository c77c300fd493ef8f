"""Loader of the in-tree CUDA library ``libalien_b200.so``.

There is no fallback: if the library is missing or no CUDA device is present,
the facade raises instead of computing anything on the CPU.
"""
from __future__ import annotations

import ctypes
import os

from .params import MAX_COLORS, PhysicsParams

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libalien_b200.so")

ERRORS = {
    1: "invalid argument",
    2: "out of memory",
    3: "CUDA error",
    4: "device error flag",
    5: "unsupported",
    6: "capacity",
    7: "no CUDA device",
}


class AlienError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, 'error')} ({code}): {message}")
        self.code = code


class Int2(ctypes.Structure):
    _fields_ = [("x", ctypes.c_int32), ("y", ctypes.c_int32)]


class GeneralSettings(ctypes.Structure):
    _fields_ = [("worldSizeX", ctypes.c_int32), ("worldSizeY", ctypes.c_int32)]


class ArraySizes(ctypes.Structure):
    _fields_ = [("cellArraySize", ctypes.c_uint64), ("particleArraySize", ctypes.c_uint64),
                ("auxiliaryDataSize", ctypes.c_uint64)]


class RawStatistics(ctypes.Structure):
    _fields_ = [
        ("timestep", ctypes.c_uint64),
        ("numCells", ctypes.c_uint64),
        ("numParticles", ctypes.c_uint64),
        ("numConnections", ctypes.c_uint64),
        ("numCellsByColor", ctypes.c_uint64 * 7),
        ("totalCellEnergy", ctypes.c_double),
        ("totalParticleEnergy", ctypes.c_double),
    ]


MAX_HISTOGRAM_SLOTS = 20
_C7 = MAX_COLORS


class TimestepStatistics(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32 * _C7) for n in ("numCells", "numSelfReplicators", "numColonies", "numViruses",
                                                    "numFreeCells", "numParticles")] + [
        ("numGenomeCells", ctypes.c_uint64 * _C7),
        ("genomeComplexity", ctypes.c_float * _C7),
        ("maxGenomeComplexityOfColonies", ctypes.c_float * _C7),
        ("genomeComplexityVariance", ctypes.c_double * _C7),
        ("totalEnergy", ctypes.c_float * _C7),
    ]


class AccumulatedStatistics(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64 * _C7) for n in (
        "numCreatedCells", "numCreatedReplicators", "numAttacks", "numMuscleActivities", "numDefenderActivities",
        "numTransmitterActivities", "numInjectionActivities", "numCompletedInjections", "numNervePulses",
        "numNeuronActivities", "numSensorActivities", "numSensorMatches", "numReconnectorCreated",
        "numReconnectorRemoved", "numDetonations")]


class TimelineStatistics(ctypes.Structure):
    _fields_ = [("timestep", TimestepStatistics), ("accumulated", AccumulatedStatistics)]


class HistogramData(ctypes.Structure):
    _fields_ = [("maxValue", ctypes.c_int32), ("numCellsByColorBySlot", (ctypes.c_int32 * MAX_HISTOGRAM_SLOTS) * _C7)]


class RawStatisticsData(ctypes.Structure):
    """AlienRawStatisticsData = RawStatisticsData (EngineInterface/RawStatisticsData.h)"""
    _fields_ = [("timeline", TimelineStatistics), ("histogram", HistogramData)]


REGION_CHOICES = 6


class LaunchConfig(ctypes.Structure):
    """AlienLaunchConfig (include/alien_b200.h)"""
    _fields_ = [
        ("regionTiles", (ctypes.c_int32 * 2) * 2),
        ("regionChoice", ctypes.c_int32 * 2),
        ("regionChoiceFixed", ctypes.c_int32 * 2),
        ("tuned", ctypes.c_int32),
        ("tunedMs", (ctypes.c_float * REGION_CHOICES) * 2),
        ("candidates", ((ctypes.c_int32 * 2) * REGION_CHOICES) * 2),
    ]


class ArenaCapacity(ctypes.Structure):
    """AlienArenaCapacity (include/alien_b200_batch.h): what a live arena reserves"""
    _fields_ = [
        ("maxWorlds", ctypes.c_int32),
        ("cellSlots", ctypes.c_uint64),
        ("particleSlots", ctypes.c_uint64),
        ("tiles", ctypes.c_uint64),
        ("particleMapSlots", ctypes.c_uint64),
        ("auxBytes", ctypes.c_uint64),
    ]


DENSITY_MAP_FIELDS = ("color", "otherMutant", "sameMutant1", "sameMutant2", "specificMutant", "lessComplexity1",
                      "lessComplexity2", "moreComplexity1", "moreComplexity2")


class DensityMap(ctypes.Structure):
    """AlienDensityMap: sizes, and host arrays the call fills (null: skipped)"""
    _fields_ = [("sizeX", ctypes.c_int32), ("sizeY", ctypes.c_int32)] + [
        (name, ctypes.POINTER(ctypes.c_uint32 if name == "specificMutant" else ctypes.c_uint64))
        for name in DENSITY_MAP_FIELDS]


# every symbol declared in include/alien_b200.h and include/alien_b200_batch.h
EXPORTED_SYMBOLS = [
    "alien_b200_version", "alien_b200_select_device", "alien_b200_time_timesteps",
    "alien_b200_batch_time_timesteps", "alien_b200_default_parameters", "alien_b200_last_error", "alien_b200_create",
    "alien_b200_destroy", "alien_b200_calc_timesteps", "alien_b200_set_data", "alien_b200_get_data",
    "alien_b200_set_parameters", "alien_b200_get_parameters", "alien_b200_get_array_sizes",
    "alien_b200_resize_arrays_if_necessary", "alien_b200_get_current_timestep", "alien_b200_set_current_timestep",
    "alien_b200_clear", "alien_b200_get_raw_statistics", "alien_b200_enqueue_timesteps", "alien_b200_stream",
    "alien_b200_kernel_launch_count", "alien_b200_timed_timesteps", "alien_b200_step_kernel_name",
    "alien_b200_batch_create", "alien_b200_batch_destroy", "alien_b200_batch_num_worlds",
    "alien_b200_batch_calc_timesteps", "alien_b200_batch_enqueue_timesteps", "alien_b200_batch_get_data",
    "alien_b200_batch_get_array_sizes", "alien_b200_batch_get_raw_statistics", "alien_b200_batch_stream",
    "alien_b200_batch_kernel_launch_count", "alien_b200_batch_kernels_per_step", "alien_b200_batch_timed_timesteps",
    "alien_b200_batch_set_step_budget", "alien_b200_batch_world_status", "alien_b200_batch_num_active",
    "alien_b200_batch_device_bytes", "alien_b200_statistics_no_alloc", "alien_b200_batch_synchronize",
    "alien_b200_debug_cell_map", "alien_b200_set_launch_config", "alien_b200_get_launch_config",
    "alien_b200_choose_region", "alien_b200_batch_set_launch_config", "alien_b200_batch_get_launch_config",
    "alien_b200_get_raw_statistics_data", "alien_b200_reset_time_interval_statistics",
    "alien_b200_batch_get_raw_statistics_data", "alien_b200_batch_reset_time_interval_statistics",
    "alien_b200_arena_bytes", "alien_b200_arena_create", "alien_b200_world_admit", "alien_b200_world_evict",
    "alien_b200_arena_num_resident", "alien_b200_get_density_map", "alien_b200_batch_get_density_map",
]

_lib: ctypes.CDLL | None = None


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m alien_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    vp, u64, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int
    P = ctypes.POINTER
    lib.alien_b200_version.restype = i32
    lib.alien_b200_default_parameters.argtypes = [P(PhysicsParams)]
    lib.alien_b200_default_parameters.restype = None
    lib.alien_b200_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    lib.alien_b200_create.argtypes = [P(GeneralSettings), P(PhysicsParams), u64, P(vp)]
    lib.alien_b200_destroy.argtypes = [vp]
    lib.alien_b200_calc_timesteps.argtypes = [vp, u64]
    lib.alien_b200_enqueue_timesteps.argtypes = [vp, u64]
    lib.alien_b200_set_data.argtypes = [vp, vp]
    lib.alien_b200_get_data.argtypes = [vp, Int2, Int2, vp]
    lib.alien_b200_set_parameters.argtypes = [vp, P(PhysicsParams)]
    lib.alien_b200_get_parameters.argtypes = [vp, P(PhysicsParams)]
    lib.alien_b200_get_array_sizes.argtypes = [vp, P(ArraySizes)]
    lib.alien_b200_resize_arrays_if_necessary.argtypes = [vp, P(ArraySizes)]
    lib.alien_b200_get_current_timestep.argtypes = [vp, P(u64)]
    lib.alien_b200_set_current_timestep.argtypes = [vp, u64]
    lib.alien_b200_clear.argtypes = [vp]
    lib.alien_b200_get_raw_statistics.argtypes = [vp, P(RawStatistics)]
    lib.alien_b200_stream.argtypes = [vp]
    lib.alien_b200_stream.restype = vp
    lib.alien_b200_kernel_launch_count.argtypes = [vp]
    lib.alien_b200_kernel_launch_count.restype = u64
    lib.alien_b200_batch_create.argtypes = [i32, P(GeneralSettings), P(PhysicsParams), vp, u64, P(vp)]
    lib.alien_b200_batch_destroy.argtypes = [vp]
    lib.alien_b200_batch_num_worlds.argtypes = [vp]
    lib.alien_b200_batch_calc_timesteps.argtypes = [vp, u64]
    lib.alien_b200_batch_enqueue_timesteps.argtypes = [vp, u64]
    lib.alien_b200_batch_get_data.argtypes = [vp, i32, vp]
    lib.alien_b200_batch_get_array_sizes.argtypes = [vp, i32, P(ArraySizes)]
    lib.alien_b200_batch_get_raw_statistics.argtypes = [vp, i32, P(RawStatistics)]
    lib.alien_b200_batch_stream.argtypes = [vp]
    lib.alien_b200_batch_stream.restype = vp
    lib.alien_b200_batch_kernel_launch_count.argtypes = [vp]
    lib.alien_b200_batch_kernel_launch_count.restype = u64
    lib.alien_b200_batch_kernels_per_step.argtypes = [vp]
    lib.alien_b200_timed_timesteps.argtypes = [vp, u64, P(ctypes.c_double), i32, P(i32)]
    lib.alien_b200_batch_timed_timesteps.argtypes = [vp, u64, P(ctypes.c_double), i32, P(i32)]
    lib.alien_b200_batch_set_step_budget.argtypes = [vp, i32, u64]
    lib.alien_b200_batch_world_status.argtypes = [vp, i32, P(u64), P(u64), P(i32)]
    lib.alien_b200_batch_num_active.argtypes = [vp]
    lib.alien_b200_batch_device_bytes.argtypes = [vp]
    lib.alien_b200_batch_device_bytes.restype = u64
    lib.alien_b200_batch_synchronize.argtypes = [vp]
    lib.alien_b200_statistics_no_alloc.argtypes = [vp, u64, vp, u64, u64, vp, vp]
    lib.alien_b200_debug_cell_map.argtypes = [vp, u64, vp, vp, vp, vp, P(u64)]
    lib.alien_b200_set_launch_config.argtypes = [vp, P(LaunchConfig)]
    lib.alien_b200_get_launch_config.argtypes = [vp, P(LaunchConfig)]
    lib.alien_b200_batch_set_launch_config.argtypes = [vp, P(LaunchConfig)]
    lib.alien_b200_batch_get_launch_config.argtypes = [vp, P(LaunchConfig)]
    lib.alien_b200_choose_region.argtypes = [P(ctypes.c_float), i32]
    lib.alien_b200_choose_region.restype = i32
    lib.alien_b200_get_raw_statistics_data.argtypes = [vp, P(RawStatisticsData)]
    lib.alien_b200_get_density_map.argtypes = [vp, P(DensityMap)]
    lib.alien_b200_batch_get_density_map.argtypes = [vp, ctypes.c_int, P(DensityMap)]
    lib.alien_b200_reset_time_interval_statistics.argtypes = [vp]
    lib.alien_b200_batch_get_raw_statistics_data.argtypes = [vp, i32, P(RawStatisticsData)]
    lib.alien_b200_batch_reset_time_interval_statistics.argtypes = [vp, i32]
    lib.alien_b200_select_device.argtypes = [i32]
    lib.alien_b200_time_timesteps.argtypes = [vp, u64, P(ctypes.c_double)]
    lib.alien_b200_batch_time_timesteps.argtypes = [vp, u64, P(ctypes.c_double)]
    lib.alien_b200_step_kernel_name.argtypes = [i32]
    lib.alien_b200_step_kernel_name.restype = ctypes.c_char_p
    lib.alien_b200_arena_bytes.argtypes = [P(ArenaCapacity), P(u64)]
    lib.alien_b200_arena_create.argtypes = [P(ArenaCapacity), P(vp)]
    lib.alien_b200_world_admit.argtypes = [vp, P(GeneralSettings), P(PhysicsParams), vp, u64, u64, P(i32)]
    lib.alien_b200_world_evict.argtypes = [vp, i32]
    lib.alien_b200_arena_num_resident.argtypes = [vp]
    _lib = lib
    return lib


def select_device(device: int) -> None:
    check(load().alien_b200_select_device(int(device)))


def last_error() -> str:
    lib = load()
    buf = ctypes.create_string_buffer(1024)
    lib.alien_b200_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(code: int) -> None:
    if code != 0:
        raise AlienError(code, last_error())
