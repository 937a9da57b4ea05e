"""The C ABI: the library loads, exports every declared symbol, and the
Python structs match the header's layouts.  No device compute."""
import ctypes as C
import os
import re
import subprocess

import pytest

from parex_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "parex_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.findall(r"\b(pxr_[a-z0-9_]+)\s*\(", text)


def test_header_lists_every_binding():
    decl = declared_functions()
    assert sorted(set(decl)) == sorted(_lib.SYMBOLS)


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    for name in declared_functions():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (pxr_\w+)", out))
    assert set(declared_functions()) <= exported


def test_struct_sizes_match_header():
    # pxr_config: 10 four-byte fields + reserved[6]
    assert C.sizeof(_lib.Config) == 64
    assert C.sizeof(_lib.SweepCut) == 12      # SweepCutData
    assert C.sizeof(_lib.NodeData) == 16      # NodeData
    assert C.sizeof(_lib.Stats) == 104
    assert C.sizeof(_lib.Schedule) == 32
    assert C.sizeof(_lib.RowPlan) == 32
    assert C.sizeof(_lib.ClusterRecord) == 128 == _lib.RECORD_DTYPE.itemsize
    assert C.sizeof(_lib.PhaseStat) == 40


def test_config_defaults_match_reference_globals():
    L = _lib.load()
    cfg = _lib.Config()
    L.pxr_config_default(C.byref(cfg))
    assert cfg.seed == 6582                   # randSeed, lib/core/definitions.h:46
    assert abs(cfg.sc_threshold - 0.3) < 1e-7  # sc_threshold, definitions.h:50
    assert abs(cfg.rw_threshold - 1e-4) < 1e-10
    assert cfg.max_rounds == 200000           # MAX_NUM_ITER, cuda/device.h:371


def test_status_strings():
    L = _lib.load()
    for s in range(7):
        assert L.pxr_status_string(s)


def test_null_arguments_are_rejected_without_device_work():
    L = _lib.load()
    assert L.pxr_create(None, None) == 1          # PXR_INVALID_ARG
    assert L.pxr_walk_step(None) == 1
    assert L.pxr_decompose(None, None) == 1


@pytest.mark.skipif(__import__("conftest").gpu_available(), reason="checks the no-device path")
def test_create_fails_loudly_without_a_device():
    L = _lib.load()
    cfg = _lib.Config()
    L.pxr_config_default(C.byref(cfg))
    h = C.c_void_p()
    assert L.pxr_create(C.byref(cfg), C.byref(h)) == 4   # PXR_CUDA_ERROR: no CPU fallback
    assert not h.value


def test_out_of_range_options_are_refused_before_any_device_work():
    L = _lib.load()
    for field, bad in (("division", 2), ("driver", 2), ("components", 3)):
        cfg = _lib.Config()
        L.pxr_config_default(C.byref(cfg))
        assert cfg.components == _lib.COMPONENTS_AUTO
        setattr(cfg, field, bad)
        h = C.c_void_p()
        assert L.pxr_create(C.byref(cfg), C.byref(h)) == 1, field   # PXR_INVALID_ARG
        assert not h.value
