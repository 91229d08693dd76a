"""The C ABI library loads on a machine without a GPU and exports every symbol that
include/avbd_cuda.h declares; no compute call is made here."""
import ctypes
import os
import re

import numpy as np

import checkers
from avbd_demo3d_b200 import _lib, box_properties, scenes
from avbd_demo3d_b200 import build as b

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "avbd_cuda.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(avbd_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    b.build()
    lib = ctypes.CDLL(b.OUT)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the same set
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_backend_name_without_gpu():
    lib = _lib.load()
    assert lib.avbd_backend_name().decode().startswith("CUDA AVBD")


def test_header_constants_match_binding():
    text = open(HEADER).read()
    consts = dict(re.findall(r"#define (AVBD_\w+) (-?\d+)", text))
    assert int(consts["AVBD_OK"]) == _lib.AVBD_OK
    for code, name in _lib.ERRORS.items():
        assert int(consts[f"AVBD_ERR_{name.upper()}"]) == code
    assert int(consts["AVBD_PHASE_COUNT"]) == len(_lib.PHASES)
    assert int(consts["AVBD_BROADPHASE_GRID"]) == scenes.BROADPHASE_GRID
    assert int(consts["AVBD_BROADPHASE_ALL_PAIRS"]) == scenes.BROADPHASE_ALL_PAIRS


def test_struct_sizes_match_header_layout():
    # plain C layouts: int32 count + pointers, all 8-byte aligned on x86-64
    assert ctypes.sizeof(_lib.AvbdBodies) == 8 + 13 * 8
    assert ctypes.sizeof(_lib.AvbdParams) == 32
    assert ctypes.sizeof(_lib.AvbdStats) == 16 * 8 + 8


def test_host_derived_properties_match_oracle():
    for sc in (scenes.pyramid(20), scenes.bridge(), scenes.mixed_drop(800, 6, 8, 0.1, extent=(20, 20, 12), seed=3)):
        p = checkers.World(sc, "oracle").body_props()
        m, mo, r = box_properties(sc.size, sc.density)
        assert np.array_equal(p["mass"], m[::-1])
        assert np.array_equal(p["moment"], mo[::-1])
        assert np.array_equal(p["radius"], r[::-1])
