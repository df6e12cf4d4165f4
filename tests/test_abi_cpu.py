"""CPU checks of the C ABI: the library loads and exports every symbol that
include/*.h declares; host-only entry points behave (no GPU calls here)."""
import ctypes as C
import glob
import os
import re

import numpy as np

from infernox_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(cmgpu_\w+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    L = N.lib()
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert set(N.EXPORTED) <= names


def test_version_and_error_string():
    L = N.lib()
    assert b"sm_100a" in L.cmgpu_version()
    assert isinstance(L.cmgpu_last_error(), bytes)


def test_tables_host_only():
    L = N.lib()
    t = np.zeros(23000, np.int32)
    assert L.cmgpu_ilogsum_table(t.ctypes.data_as(C.POINTER(C.c_int32)), 23000) == 0
    f = np.zeros(23000, np.float32)
    assert L.cmgpu_flogsum_table(f.ctypes.data_as(C.POINTER(C.c_float)), 23000) == 0
    assert abs(f[0] - 1.0) < 1e-6 and f[-1] < 1e-6
    assert L.cmgpu_ilogsum_table(t.ctypes.data_as(C.POINTER(C.c_int32)), 23001) != 0


def test_bad_arguments_are_rejected_without_gpu():
    L = N.lib()
    assert L.cmgpu_prep_configure(None, 0, 0, 1e-7, 1e-15, 1e-7, None) == -1
    m = C.c_void_p()
    assert L.cmgpu_model_upload(None, 0, C.byref(m)) == -1
