"""alien_b200_statistics_no_alloc against alien_b200_get_raw_statistics.

The allocation-free statistics entry point reduces transfer objects that the
caller keeps in device memory, with its scratch in a fixed device array of
the library.  Each case exports a stepped world through the facade, copies
its cells and particles into device buffers, calls the entry point through
the C ABI and compares with the facade's own statistics of the same world.
Tolerance: counts exact; energies |a - b| <= 1e-9 * max(|b|, 1) (both sum
the same 2^-16 fixed-point terms, so they agree to the last bit in
practice).  Two different worlds are reduced in a row so that the second
call reads only partials written by itself.  The file name sorts last so
that the entry point also runs after every other GPU test in one process.
"""
import ctypes

import numpy as np
import pytest

from alien_b200 import _lib
from alien_b200 import params as P
from alien_b200 import worldgen
from alien_b200.facade import SimulationFacade

pytestmark = pytest.mark.gpu

MAX_OBJECTS = 4096 * 2048


def _device_bytes(array):
    import torch

    return torch.from_numpy(np.ascontiguousarray(array).view(np.uint8).copy()).cuda()


def _no_alloc_statistics(cells, particles, timestep):
    import torch

    lib = _lib.load()
    d_cells = _device_bytes(cells) if len(cells) else None
    d_particles = _device_bytes(particles) if len(particles) else None
    d_out = torch.zeros(ctypes.sizeof(_lib.RawStatistics), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(lib.alien_b200_statistics_no_alloc(
        d_cells.data_ptr() if d_cells is not None else None, len(cells),
        d_particles.data_ptr() if d_particles is not None else None, len(particles),
        int(timestep), d_out.data_ptr(), stream))
    torch.cuda.synchronize()
    host = d_out.cpu().numpy().tobytes()
    return _lib.RawStatistics.from_buffer_copy(host)


def _stepped_world(data, world, prm, steps):
    eng = SimulationFacade()
    eng.new_simulation(0, world, prm)
    eng.set_simulation_data(data)
    eng.calc_timesteps(steps)
    out = eng.get_simulation_data()
    stats = eng.get_raw_statistics()
    eng.close_simulation()
    return out, stats


def _assert_same(got, ref):
    assert got.timestep == ref.timestep
    assert got.numCells == ref.numCells
    assert got.numParticles == ref.numParticles
    assert got.numConnections == ref.numConnections
    assert list(got.numCellsByColor) == list(ref.numCellsByColor)
    for a, b in ((got.totalCellEnergy, ref.totalCellEnergy), (got.totalParticleEnergy, ref.totalParticleEnergy)):
        assert abs(a - b) <= 1e-9 * max(abs(b), 1.0)


def test_no_alloc_statistics_two_calls_in_a_row():
    cases = [
        (worldgen.random_test_world(11, barriers=10, free_cells=300), P.benchmark_parameters(P.MOTION_FLUID), 5),
        (worldgen.soft_body_world(3, world=(256, 256), clusters=40, particles=5000),
         P.benchmark_parameters(P.MOTION_COLLISION), 3),
    ]
    results = []
    for (data, world), prm, steps in cases:
        out, ref = _stepped_world(data, world, prm, steps)
        assert ref.numCells > 0 and ref.numConnections > 0
        results.append((out, ref))
    # second call right after the first, with different sizes
    for out, ref in results:
        got = _no_alloc_statistics(out.cells, out.particles, ref.timestep)
        _assert_same(got, ref)


def test_no_alloc_statistics_empty_and_limit():
    got = _no_alloc_statistics(np.zeros(0, np.uint8), np.zeros(0, np.uint8), 7)
    assert got.timestep == 7 and got.numCells == 0 and got.numParticles == 0
    assert got.totalCellEnergy == 0.0 and got.totalParticleEnergy == 0.0
    lib = _lib.load()
    out = ctypes.c_void_p(1)  # never dereferenced: the size check comes first
    code = lib.alien_b200_statistics_no_alloc(ctypes.c_void_p(1), MAX_OBJECTS + 1, None, 0, 0, out, None)
    assert code == 6
    assert "at most 8388608 cells" in _lib.last_error()


def test_no_alloc_statistics_with_device_memory_reserved():
    """A caller that reserves the device's remaining memory after the first
    call (the set-up on this device) can still call the entry point: later
    calls need no device memory.  The reservation leaves 64 MB free for the
    driver's own needs and is released at the end of the test."""
    import torch

    data, world = worldgen.random_test_world(12, free_cells=200)
    out, ref = _stepped_world(data, world, P.benchmark_parameters(P.MOTION_FLUID), 2)
    first = _no_alloc_statistics(out.cells, out.particles, ref.timestep)  # set-up call
    _assert_same(first, ref)
    lib = _lib.load()
    d_cells = _device_bytes(out.cells)
    d_particles = _device_bytes(out.particles)
    d_out = torch.zeros(ctypes.sizeof(_lib.RawStatistics), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info()
    reserve = max(0, free - (64 << 20))
    hold = torch.empty(reserve, dtype=torch.uint8, device="cuda") if reserve else None
    try:
        for _ in range(2):
            _lib.check(lib.alien_b200_statistics_no_alloc(
                d_cells.data_ptr(), len(out.cells), d_particles.data_ptr(), len(out.particles),
                int(ref.timestep), d_out.data_ptr(), stream))
            torch.cuda.synchronize()
            got = _lib.RawStatistics.from_buffer_copy(d_out.cpu().numpy().tobytes())
            _assert_same(got, ref)
    finally:
        del hold
        torch.cuda.empty_cache()
