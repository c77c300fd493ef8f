"""CPU checks of the C ABI boundary: the library loads without a GPU, exports
every function declared in include/*.h, and the transfer-object layouts
match the reference's TOs.cuh (304 / 40 / 12 bytes, pinned offsets)."""
import ctypes
import os
import re

import numpy as np

from alien_b200 import _lib, build
from alien_b200.params import PhysicsParams
from alien_b200.to import CELL_TO, CONNECTION_TO, PARTICLE_TO

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("alien_b200.h", "alien_b200_batch.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"^\s*(?:const\s+)?(?:int|void|uint64_t|char)\s*\*?\s*(alien_b200_\w+)\s*\(", text, re.M))
    return names


def test_library_exports_every_declared_symbol():
    build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    declared = declared_functions()
    assert len(declared) >= 25
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    assert set(declared) == set(_lib.EXPORTED_SYMBOLS)


def test_transfer_object_layout():
    assert CELL_TO.itemsize == 304 and PARTICLE_TO.itemsize == 40 and CONNECTION_TO.itemsize == 12
    assert CELL_TO.fields["pos"][1] == 80 and CELL_TO.fields["livingState"][1] == 112
    assert CELL_TO.fields["cellFunctionData"][1] == 144 and CELL_TO.fields["selected"][1] == 296
    assert PARTICLE_TO.fields["pos"][1] == 16 and PARTICLE_TO.fields["color"][1] == 32


def test_default_parameters_match_reference_defaults():
    lib = _lib.load()
    p = PhysicsParams()
    lib.alien_b200_default_parameters(ctypes.byref(p))
    from alien_b200.params import default_parameters
    q = default_parameters()
    assert bytes(p) == bytes(q)


def test_no_device_reports_error_without_fallback():
    """on a machine without a GPU, create fails loudly (no CPU path)"""
    import torch
    if torch.cuda.is_available():
        return
    lib = _lib.load()
    g = _lib.GeneralSettings(64, 64)
    p = PhysicsParams()
    lib.alien_b200_default_parameters(ctypes.byref(p))
    h = ctypes.c_void_p()
    rc = lib.alien_b200_create(ctypes.byref(g), ctypes.byref(p), 0, ctypes.byref(h))
    assert rc == 7 and not h


def test_raw_statistics_data_layout():
    """AlienRawStatisticsData mirrors RawStatisticsData byte for byte (ColorVector<T> = T[7],
    EngineInterface/Colors.h; MAX_HISTOGRAM_SLOTS = 20, EngineConstants.h)"""
    assert ctypes.sizeof(_lib.TimestepStatistics) == 368
    assert _lib.TimestepStatistics.numGenomeCells.offset == 168
    assert _lib.TimestepStatistics.genomeComplexityVariance.offset == 280
    assert ctypes.sizeof(_lib.AccumulatedStatistics) == 15 * 7 * 8
    assert _lib.RawStatisticsData.histogram.offset == 1208
    assert ctypes.sizeof(_lib.RawStatisticsData) == 1776
