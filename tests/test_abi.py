"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute call: this runs without a GPU)."""
import ctypes
import glob
import os
import re

from phcpack_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(?:int|void|const char\s*\*|double|long long|long)\s+\**\s*(phc_\w+|GPU_\w+|gpu\w+)\s*\(",
                             text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared()
    assert "phc_system_evaldiff" in names
    # entry points returning long long are collected too
    assert "phc_bals_solve_static_capacity_bytes" in names and "phc_dense_workspace_bytes" in names


def test_library_exports_all_declared_symbols():
    lib = _lib.lib()
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version():
    assert _lib.lib().phc_abi_version() == 2


def test_tuning_knobs_set_get_and_reject():
    # host-side state only: no device work
    lib = _lib.lib()
    for knob, good, bad in ((0, 4, 9), (1, 2, 3), (2, 6, 33), (3, 2, 3)):
        assert _lib.call("phc_tune_set", knob, good) == 0
        assert _lib.call("phc_tune_get", knob) == good
        assert lib.phc_tune_set(knob, bad) < 0
        assert _lib.call("phc_tune_get", knob) == good
        assert _lib.call("phc_tune_set", knob, 0) == 0
    assert lib.phc_tune_set(4, 1) < 0 and lib.phc_tune_get(-1) < 0
    assert lib.phc_tune_set(0, -1) < 0
