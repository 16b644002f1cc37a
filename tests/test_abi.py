"""CPU-side checks of the C ABI: the library loads without a GPU and exports
every entry point include/dicegpu.h declares; argument validation that needs
no device behaves like the reference's (dice_correlate returns -1 on bad
arguments, DICe_api.cpp:71-76)."""
import ctypes
import os
import re

import numpy as np

from dice_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names.update(re.findall(r"\b(dicegpu_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    lib = abi.load_library()
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_defaults_match_reference():
    lib = abi.load_library()
    p = abi.Params()
    assert lib.dicegpu_default_params(ctypes.byref(p)) == 0
    q = abi.default_params()
    assert bytes(p) == bytes(q)
    assert p.max_solver_iterations_fast == 25
    assert p.fast_solver_tolerance == 1e-4
    assert p.optimization == abi.GRADIENT_BASED_THEN_SIMPLEX
    assert p.interpolation == abi.KEYS_FOURTH


def test_num_params():
    lib = abi.load_library()
    for kw, n in [({}, 2), (dict(enable_rotation=1), 3), (dict(enable_normal_strain=1), 4),
                  (dict(enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1), 6),
                  (dict(shape_function=abi.QUADRATIC_SF), 12)]:
        p = abi.default_params(**kw)
        assert lib.dicegpu_num_params(ctypes.byref(p)) == n == abi.num_params(p)


def test_correlate_rejects_bad_arguments_like_reference():
    lib = abi.load_library()
    pts = np.zeros((1, 9), np.float32)
    img = np.zeros((32, 32), np.float32)
    img2 = np.zeros((32, 33), np.float32)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    assert lib.dicegpu_correlate(P(pts), 1, 21, P(img), 32, 32, P(img2), 33, 32, None, 0) == -1
    assert lib.dicegpu_correlate(P(pts), 1, 0, P(img), 32, 32, P(img), 32, 32, None, 0) == -1
    assert lib.dicegpu_correlate(P(pts), 0, 21, P(img), 32, 32, P(img), 32, 32, None, 0) == -1


def test_version_string():
    lib = abi.load_library()
    assert b"sm_100a" in lib.dicegpu_version()
