"""The C-ABI library builds, loads and exports every entry point declared in
include/pt_b200.h (no compute call: this runs without a GPU)."""
import ctypes
import os
import re
import subprocess

import numpy as np

from lsystemeditor_b200 import _build
from lsystemeditor_b200.pathtracer import EXPORTED_SYMBOLS, PtProfile, PtStats
from lsystemeditor_b200.records import CAMERA_DTYPE, MATERIAL_DTYPE, PARAMS_DTYPE, TEXTURE_DTYPE

HEADER = os.path.join(_build.INCLUDE, "pt_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|void|float|size_t|const char\*)\s+(pt_\w+)\s*\(", text, re.M)))


def test_library_builds_and_exports_every_declared_symbol():
    lib = _build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(pt_\w+)", out))
    declared = declared_functions()
    assert declared, "no declarations parsed"
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    assert sorted(EXPORTED_SYMBOLS) == declared
    L = ctypes.CDLL(lib)
    for s in declared:
        getattr(L, s)


def test_record_layouts_match_header():
    text = open(HEADER).read()
    assert MATERIAL_DTYPE.itemsize == 96 and TEXTURE_DTYPE.itemsize == 64 and CAMERA_DTYPE.itemsize == 80
    assert PARAMS_DTYPE.itemsize == 80
    # field order of the params record follows the header
    body = re.search(r"typedef struct pt_render_params \{(.*?)\} pt_render_params;", text, re.S).group(1)
    names = re.findall(r"(\w+)(?:\s*,\s*(\w+))?(?:\s*,\s*(\w+))?;", re.sub(r"\[\d+\]", "", re.sub(r"/\*.*?\*/", "", body, flags=re.S)))
    flat = [n for tup in names for n in tup if n]
    assert list(PARAMS_DTYPE.names) == flat
    assert ctypes.sizeof(PtStats) == 72 and ctypes.sizeof(PtProfile) == 15 * 8


def test_default_params_match_reference_defaults():
    lib = ctypes.CDLL(_build.build())
    p = np.zeros((), PARAMS_DTYPE)
    lib.pt_default_params(ctypes.c_void_p(p.ctypes.data))
    assert abs(float(p["background_r"]) - 10.0 / 255.0) < 1e-7
    assert int(p["max_path_depth"]) == 32 and int(p["russian_roulette_min_depth"]) == 3
    assert int(p["min_samples"]) == 16 and int(p["max_samples_per_pixel"]) == 1024
    assert abs(float(p["relative_error_threshold"]) - 0.02) < 1e-7


def test_null_handle_errors_without_device():
    lib = ctypes.CDLL(_build.build())
    lib.pt_render.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.pt_destroy.argtypes = [ctypes.c_void_p]
    lib.pt_create.argtypes = [ctypes.c_void_p, ctypes.c_int]
    assert lib.pt_render(None, 1) == 1          # PT_ERR_INVALID_ARGUMENT
    assert lib.pt_destroy(None) == 1
    assert lib.pt_create(None, 0) == 1
    lib.pt_set_extend_mode.argtypes = [ctypes.c_void_p, ctypes.c_int]
    assert lib.pt_set_extend_mode(None, 0) == 1
