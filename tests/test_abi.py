"""C ABI of the product library: every entry point declared in include/*.h is
exported, host-only entry points behave, argument errors are reported as status
codes (no GPU needed)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from falm_b200 import _lib, cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:int|const char \*|long long)\s*(falm_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(lib_built):
    lib = _lib.load()
    names = declared()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_abi_version(lib_built):
    assert _lib.load().falm_abi_version() == 1


def test_null_arguments_are_rejected(lib_built):
    lib = _lib.load()
    assert lib.falm_create(None, 0, None) == 1
    assert lib.falm_destroy(None) == 1
    assert lib.falm_cfd_init(None, 1e3, 1, 1, 0.1) == 1
    assert lib.falm_step(None, None, 0.1, 0.0, None, None) == 1
    assert lib.falm_eq_solve(None, None, None, None, None, None, None) == 1
    assert lib.falm_alm_build_aps(0, None, None, None, None, None, 0, 0, 0, 1.0, 0.0, None, None, None, None, None) == 1


def test_build_aps_host_entry_point(lib_built):
    from falm_b200.api import build_aps
    st = cases.blade_stations()
    got = build_aps(st, 1, 3, 32, 1.0, 0.0)
    ref = cases.build_aps_py(st, 96, 32, 1.0, 0.0)
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k])


def test_inflow_box_statistics():
    box = cases.inflow_box(24, 20, 0.05, nb=16, corr=8, seed=cases.INFLOW_SEED)
    assert box.shape == (3, 16, 20, 24)
    np.testing.assert_allclose(box.reshape(3, -1).std(axis=1), 0.05, rtol=1e-12)
    again = cases.inflow_box(24, 20, 0.05, nb=16, corr=8, seed=cases.INFLOW_SEED)
    np.testing.assert_array_equal(box, again)
