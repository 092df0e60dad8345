"""The C-ABI library loads and exports every entry point include/*.h declares.

CPU-only: nothing here launches a kernel.
"""
import ctypes
import glob
import os
import re

import pytest

from gpu_tracking_b200 import _ffi, build
from gpu_tracking_b200._params import GtParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        for m in re.finditer(r"GT_API\s+[\w\s\*]+?\b(gt_\w+)\s*\(", open(h).read()):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def libso():
    build.build()
    return ctypes.CDLL(_ffi.LIB_PATH)


def test_every_declared_symbol_is_exported(libso):
    names = declared_symbols()
    assert len(names) >= 18
    for n in names:
        assert hasattr(libso, n), n


def test_params_layout_and_defaults(libso):
    p = GtParams()
    libso.gt_params_default(ctypes.byref(p))
    # TrackingParams::default (src/gpu_setup.rs:61-97)
    assert (p.diameter, p.separation, p.max_iterations) == (9, 10, 10)
    assert abs(p.shift_threshold - 0.6) < 1e-7 and p.noise_size == 1.0
    assert p.truncate_preprocessed == 1 and p.characterize == 0 and p.doughnut_correction == 0
    from oracle import loader
    assert loader.lib().oracle_params_sizeof() == ctypes.sizeof(GtParams)


def test_version_string(libso):
    libso.gt_version.restype = ctypes.c_char_p
    assert b"sm_100a" in libso.gt_version()
