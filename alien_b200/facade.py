"""Python mirror of the reference's engine surface for the physics stage.

``SimulationFacade`` follows ``_SimulationFacade``
(source/EngineInterface/SimulationFacade.h:13-110) at the DataTO level of
``_SimulationCudaFacade`` (source/EngineGpuKernels/SimulationCudaFacade.cuh
:27-139): the same operations, argument meaning and error behaviour
(failures raise).  Every call goes through the C ABI of ``libalien_b200.so``.
``BatchSimulation`` steps many worlds in one arena.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import ArenaCapacity, ArraySizes, GeneralSettings, Int2, LaunchConfig, RawStatistics, RawStatisticsData, check
from .params import PhysicsParams
from .to import CELL_TO, PARTICLE_TO, DataTO


class SimulationFacade:
    """One world on the current CUDA device."""

    def __init__(self):
        self._lib = _lib.load()
        self._h = ctypes.c_void_p()
        self._world = None

    # _SimulationFacade::newSimulation (SimulationFacade.h:18)
    def new_simulation(self, timestep: int, world_size, parameters: PhysicsParams) -> None:
        self.close_simulation()
        g = GeneralSettings(int(world_size[0]), int(world_size[1]))
        check(self._lib.alien_b200_create(ctypes.byref(g), ctypes.byref(parameters), int(timestep), ctypes.byref(self._h)))
        self._world = (int(world_size[0]), int(world_size[1]))

    # closeSimulation (:67)
    def close_simulation(self) -> None:
        if self._h:
            check(self._lib.alien_b200_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close_simulation()
        except Exception:
            pass

    def _handle(self):
        if not self._h:
            raise RuntimeError("no simulation: call new_simulation first")
        return self._h

    @property
    def world_size(self):
        return self._world

    # calcTimesteps (:60)
    def calc_timesteps(self, timesteps: int) -> None:
        check(self._lib.alien_b200_calc_timesteps(self._handle(), int(timesteps)))

    def enqueue_timesteps(self, timesteps: int) -> None:
        check(self._lib.alien_b200_enqueue_timesteps(self._handle(), int(timesteps)))

    def time_timesteps(self, timesteps: int) -> float:
        """milliseconds of ``timesteps`` steps between CUDA events on the engine stream"""
        ms = ctypes.c_double()
        check(self._lib.alien_b200_time_timesteps(self._handle(), int(timesteps), ctypes.byref(ms)))
        return ms.value

    # setSimulationData (:47)
    def set_simulation_data(self, data: DataTO) -> None:
        check(self._lib.alien_b200_set_data(self._handle(), ctypes.cast(data.c_ptr(), ctypes.c_void_p)))

    # getSimulationData (:40); the reference reads the world +- 10
    # (EngineImpl/SimulationFacadeImpl.cpp:87-91)
    def get_simulation_data(self, upper_left=None, lower_right=None, out: DataTO | None = None) -> DataTO:
        if upper_left is None:
            upper_left = (-10, -10)
        if lower_right is None:
            lower_right = (self._world[0] + 10, self._world[1] + 10)
        if out is None:
            sizes = self.get_array_sizes()
            out = DataTO(np.zeros(0, CELL_TO), np.zeros(0, PARTICLE_TO), None, cell_capacity=sizes.cellArraySize,
                         particle_capacity=sizes.particleArraySize, aux_capacity=sizes.auxiliaryDataSize)
        check(self._lib.alien_b200_get_data(self._handle(), Int2(*upper_left), Int2(*lower_right),
                                            ctypes.cast(out.c_ptr(), ctypes.c_void_p)))
        return out

    # get/setSimulationParameters (:75-79)
    def set_simulation_parameters(self, parameters: PhysicsParams) -> None:
        check(self._lib.alien_b200_set_parameters(self._handle(), ctypes.byref(parameters)))

    def get_simulation_parameters(self) -> PhysicsParams:
        p = PhysicsParams()
        check(self._lib.alien_b200_get_parameters(self._handle(), ctypes.byref(p)))
        return p

    def get_array_sizes(self) -> ArraySizes:
        s = ArraySizes()
        check(self._lib.alien_b200_get_array_sizes(self._handle(), ctypes.byref(s)))
        return s

    def resize_arrays_if_necessary(self, cells: int = 0, particles: int = 0, aux: int = 0) -> None:
        s = ArraySizes(cells, particles, aux)
        check(self._lib.alien_b200_resize_arrays_if_necessary(self._handle(), ctypes.byref(s)))

    # getCurrentTimestep / setCurrentTimestep (:69-70)
    def get_current_timestep(self) -> int:
        t = ctypes.c_uint64()
        check(self._lib.alien_b200_get_current_timestep(self._handle(), ctypes.byref(t)))
        return t.value

    def set_current_timestep(self, timestep: int) -> None:
        check(self._lib.alien_b200_set_current_timestep(self._handle(), int(timestep)))

    def clear(self) -> None:
        check(self._lib.alien_b200_clear(self._handle()))

    # getRawStatistics (:98)
    def get_raw_statistics(self) -> RawStatistics:
        r = RawStatistics()
        check(self._lib.alien_b200_get_raw_statistics(self._handle(), ctypes.byref(r)))
        return r

    def get_raw_statistics_data(self) -> RawStatisticsData:
        """RawStatisticsData: timeline of this timestep, accumulated counts, age histogram"""
        r = RawStatisticsData()
        check(self._lib.alien_b200_get_raw_statistics_data(self._handle(), ctypes.byref(r)))
        return r

    # resetTimeIntervalStatistics (SimulationFacade.h)
    def reset_time_interval_statistics(self) -> None:
        check(self._lib.alien_b200_reset_time_interval_statistics(self._handle()))

    def get_density_map(self) -> dict:
        """the density map the last step filled (DensityMap.cuh:8-230): field
        name -> (sizeY, sizeX) array, entry [y, x] for slot x + y * sizeX"""
        return _density_map(lambda m: self._lib.alien_b200_get_density_map(self._handle(), m))

    def launch_config(self) -> LaunchConfig:
        """pair-kernel region shapes in use, and the autotuner's timings"""
        c = LaunchConfig()
        check(self._lib.alien_b200_get_launch_config(self._handle(), ctypes.byref(c)))
        return c

    def set_region_choice(self, fluid: int = 0, collision: int = 0) -> None:
        """fix the pair-kernel region shape per motion type: candidate index
        + 1, or 0 for the autotuner"""
        c = LaunchConfig()
        c.regionChoiceFixed[0], c.regionChoiceFixed[1] = int(fluid), int(collision)
        check(self._lib.alien_b200_set_launch_config(self._handle(), ctypes.byref(c)))

    def debug_cell_map(self):
        """The engine's cell map of the current state (alien_b200_debug_cell_map):
        (ids, slots, tiles, flags) of every binned cell in the map's tile order."""
        import numpy as np

        count = ctypes.c_uint64()
        code = self._lib.alien_b200_debug_cell_map(self._handle(), 0, None, None, None, None, ctypes.byref(count))
        if code not in (0, 6):  # 6: capacity (the count is still returned)
            check(code)
        n = int(count.value)
        ids = np.zeros(max(n, 1), np.uint64)
        slots = np.zeros(max(n, 1), np.uint32)
        tiles = np.zeros(max(n, 1), np.uint32)
        flags = np.zeros(max(n, 1), np.uint8)
        check(self._lib.alien_b200_debug_cell_map(self._handle(), n, ids.ctypes.data, slots.ctypes.data, tiles.ctypes.data,
                                                  flags.ctypes.data, ctypes.byref(count)))
        return ids[:n], slots[:n], tiles[:n], flags[:n]

    def stream(self) -> int:
        return int(self._lib.alien_b200_stream(self._handle()) or 0)

    def kernel_launches(self) -> int:
        return int(self._lib.alien_b200_kernel_launch_count(self._handle()))

    def timed_timesteps(self, timesteps: int):
        """{kernel name: summed ms} over ``timesteps`` steps, launch by launch"""
        return _timed(self._lib, self._lib.alien_b200_timed_timesteps, self._handle(), timesteps)


class BatchSimulation:
    """Many independent worlds stepped together in one arena."""

    def __init__(self, worlds, timestep: int = 0):
        """``worlds``: list of (DataTO, (sizeX, sizeY), PhysicsParams)."""
        self._lib = _lib.load()
        n = len(worlds)
        self._datas = [w[0] for w in worlds]
        self._sizes = [tuple(w[1]) for w in worlds]
        gs = (GeneralSettings * n)(*[GeneralSettings(int(s[0]), int(s[1])) for s in self._sizes])
        ps = (PhysicsParams * n)(*[w[2] for w in worlds])
        from .to import CDataTO
        tos = (CDataTO * n)(*[d._c for d in self._datas])
        self._h = ctypes.c_void_p()
        check(self._lib.alien_b200_batch_create(n, gs, ps, ctypes.cast(tos, ctypes.c_void_p), int(timestep),
                                                ctypes.byref(self._h)))
        self.num_worlds = n

    def close(self) -> None:
        if self._h:
            check(self._lib.alien_b200_batch_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def calc_timesteps(self, timesteps: int) -> None:
        check(self._lib.alien_b200_batch_calc_timesteps(self._h, int(timesteps)))

    def enqueue_timesteps(self, timesteps: int) -> None:
        check(self._lib.alien_b200_batch_enqueue_timesteps(self._h, int(timesteps)))

    def synchronize(self) -> None:
        """wait for enqueued steps; grow particle storage if needed"""
        check(self._lib.alien_b200_batch_synchronize(self._h))

    def time_timesteps(self, timesteps: int) -> float:
        ms = ctypes.c_double()
        check(self._lib.alien_b200_batch_time_timesteps(self._h, int(timesteps), ctypes.byref(ms)))
        return ms.value

    def get_simulation_data(self, world: int) -> DataTO:
        s = ArraySizes()
        check(self._lib.alien_b200_batch_get_array_sizes(self._h, int(world), ctypes.byref(s)))
        out = DataTO(np.zeros(0, CELL_TO), np.zeros(0, PARTICLE_TO), None, cell_capacity=s.cellArraySize,
                     particle_capacity=s.particleArraySize, aux_capacity=s.auxiliaryDataSize)
        check(self._lib.alien_b200_batch_get_data(self._h, int(world), ctypes.cast(out.c_ptr(), ctypes.c_void_p)))
        return out

    def get_raw_statistics_data(self, world: int) -> RawStatisticsData:
        r = RawStatisticsData()
        check(self._lib.alien_b200_batch_get_raw_statistics_data(self._h, int(world), ctypes.byref(r)))
        return r

    def reset_time_interval_statistics(self, world: int) -> None:
        check(self._lib.alien_b200_batch_reset_time_interval_statistics(self._h, int(world)))

    def get_density_map(self, world: int) -> dict:
        """world's density map (SimulationFacade.get_density_map)"""
        return _density_map(lambda m: self._lib.alien_b200_batch_get_density_map(self._h, int(world), m))

    def get_raw_statistics(self, world: int) -> RawStatistics:
        r = RawStatistics()
        check(self._lib.alien_b200_batch_get_raw_statistics(self._h, int(world), ctypes.byref(r)))
        return r

    def particle_slots(self, world: int) -> int:
        """the particle slots the world holds in the arena"""
        s = ArraySizes()
        check(self._lib.alien_b200_batch_get_array_sizes(self._h, int(world), ctypes.byref(s)))
        return int(s.particleArraySize)

    def set_step_budget(self, world: int, steps: int) -> None:
        """world steps ``steps`` more times and then stops (0 = no limit)"""
        check(self._lib.alien_b200_batch_set_step_budget(self._h, int(world), int(steps)))

    def world_status(self, world: int):
        """(timestep, steps remaining, active)"""
        t, r, a = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_int()
        check(self._lib.alien_b200_batch_world_status(self._h, int(world), ctypes.byref(t), ctypes.byref(r),
                                                      ctypes.byref(a)))
        return t.value, r.value, bool(a.value)

    def num_active(self) -> int:
        n = int(self._lib.alien_b200_batch_num_active(self._h))
        if n < 0:
            raise RuntimeError(_lib.last_error())
        return n

    def device_bytes(self) -> int:
        return int(self._lib.alien_b200_batch_device_bytes(self._h))

    def stream(self) -> int:
        return int(self._lib.alien_b200_batch_stream(self._h) or 0)

    def kernel_launches(self) -> int:
        return int(self._lib.alien_b200_batch_kernel_launch_count(self._h))

    def launch_config(self) -> LaunchConfig:
        c = LaunchConfig()
        check(self._lib.alien_b200_batch_get_launch_config(self._h, ctypes.byref(c)))
        return c

    def set_region_choice(self, fluid: int = 0, collision: int = 0) -> None:
        c = LaunchConfig()
        c.regionChoiceFixed[0], c.regionChoiceFixed[1] = int(fluid), int(collision)
        check(self._lib.alien_b200_batch_set_launch_config(self._h, ctypes.byref(c)))

    def kernels_per_step(self) -> int:
        return int(self._lib.alien_b200_batch_kernels_per_step(self._h))

    def timed_timesteps(self, timesteps: int):
        return _timed(self._lib, self._lib.alien_b200_batch_timed_timesteps, self._h, timesteps)


class LiveArena(BatchSimulation):
    """A batch whose worlds are admitted and evicted while the others step
    (alien_b200_arena_create, include/alien_b200_batch.h).  Device memory for
    ``capacity`` is reserved once; ``admit`` places a world into free ranges
    and returns its index, which every BatchSimulation method takes."""

    def __init__(self, capacity: ArenaCapacity):
        self._lib = _lib.load()
        self._h = ctypes.c_void_p()
        self.capacity = capacity
        check(self._lib.alien_b200_arena_create(ctypes.byref(capacity), ctypes.byref(self._h)))
        self.num_worlds = int(capacity.maxWorlds)

    @staticmethod
    def bytes_for(capacity: ArenaCapacity) -> int:
        """device bytes an arena of this capacity reserves"""
        b = ctypes.c_uint64()
        check(_lib.load().alien_b200_arena_bytes(ctypes.byref(capacity), ctypes.byref(b)))
        return int(b.value)

    @staticmethod
    def capacity_for(budget_bytes: int, max_worlds: int = 1024, area_per_cell: float = 5.0, tile_side: int = 2,
                     particles_per_cell: float = 1.6, aux_per_cell: float = 100.0) -> ArenaCapacity:
        """the largest capacity of this mix that fits ``budget_bytes``: cell
        slots C, particle slots particles_per_cell * C, tiles and particle-map
        slots for worlds of area_per_cell slots per cell (density 0.2 at 5),
        aux_per_cell bytes of neuron data per cell"""
        def cap(cells):
            c = ArenaCapacity()
            c.maxWorlds = int(max_worlds)
            c.cellSlots = int(cells)
            c.particleSlots = int(cells * particles_per_cell) + 4096 * max_worlds // 4
            area = cells * area_per_cell
            c.tiles = int(area / (tile_side * tile_side) * 1.1) + 64 * max_worlds
            c.particleMapSlots = int(area * 1.1) + 256 * max_worlds
            c.auxBytes = int(cells * aux_per_cell)
            return c
        def fits(cells):
            try:
                return LiveArena.bytes_for(cap(cells)) <= budget_bytes
            except _lib.AlienError:  # beyond the arena's slot limits
                return False
        lo, hi = 1 << 12, 1 << 30
        if not fits(lo):
            raise ValueError("budget too small for a live arena")
        while not fits(hi):  # bisect the cell slots
            mid = (lo + hi) // 2
            if mid == lo:
                break
            if fits(mid):
                lo = mid
            else:
                hi = mid
        return cap(hi if fits(hi) else lo)

    def admit(self, data: DataTO, world_size, params: PhysicsParams, timestep: int = 0, steps: int = 0) -> int:
        """places the world into free ranges, behind the steps already
        enqueued; it steps ``steps`` times (0 = no limit).  Raises AlienError
        with ALIEN_B200_ERR_CAPACITY when it does not fit."""
        g = GeneralSettings(int(world_size[0]), int(world_size[1]))
        w = ctypes.c_int()
        check(self._lib.alien_b200_world_admit(self._h, ctypes.byref(g), ctypes.byref(params),
                                               ctypes.cast(data.c_ptr(), ctypes.c_void_p), int(timestep), int(steps),
                                               ctypes.byref(w)))
        return int(w.value)

    def evict(self, world: int) -> None:
        check(self._lib.alien_b200_world_evict(self._h, int(world)))

    def num_resident(self) -> int:
        n = int(self._lib.alien_b200_arena_num_resident(self._h))
        if n < 0:
            raise RuntimeError(_lib.last_error())
        return n


def _timed(lib, fn, handle, timesteps):
    buf = (ctypes.c_double * 64)()
    n = ctypes.c_int()
    check(fn(handle, int(timesteps), buf, 64, ctypes.byref(n)))
    out = {}
    for k in range(n.value):
        name = lib.alien_b200_step_kernel_name(k)
        out[name.decode() if name else f"k{k}"] = buf[k]
    return out


def _density_map(call) -> dict:
    """two calls of an AlienDensityMap entry point: the sizes, then the arrays"""
    m = _lib.DensityMap()
    check(call(ctypes.byref(m)))
    sx, sy = int(m.sizeX), int(m.sizeY)
    out = {name: np.zeros((sy, sx), np.uint32 if name == "specificMutant" else np.uint64)
           for name in _lib.DENSITY_MAP_FIELDS}
    if sx * sy == 0:
        return out
    for name, arr in out.items():
        ctype = ctypes.c_uint32 if name == "specificMutant" else ctypes.c_uint64
        setattr(m, name, arr.ctypes.data_as(ctypes.POINTER(ctype)))
    check(call(ctypes.byref(m)))
    return out
