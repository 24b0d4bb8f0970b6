"""CPU checks of the C-ABI library: it loads without a GPU, exports every symbol that
include/anitowave.h declares, and its host-only helpers agree with the oracle."""
import ctypes as C
import os
import re

import numpy as np

import anitowave_adaptive_b200 as aw
from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "anitowave.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(aw_[a-z0-9_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    L = aw.lib()
    names = declared_symbols()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding types every one of them
    assert set(names) <= set(aw.SIGNATURES), set(names) - set(aw.SIGNATURES)


def test_host_helpers_match_oracle():
    assert aw.version().startswith("anitowave-b200")
    rng = np.random.default_rng(0)
    for x, y, z in rng.integers(0, 1024, size=(100, 3)):
        assert aw.morton3d(int(x), int(y), int(z)) == po.morton3d(int(x), int(y), int(z))
    for R0, L in ((16, 3), (8, 4)):
        for lv in range(L):
            assert aw.block_layout(R0, lv) == list(po.block_layout(R0, lv))


def test_default_solver_descriptors():
    d = aw.solver_default_desc(aw.OPERATOR_REFERENCE)
    # Smoother.cuh:9-11, Smoother.cuh:286, VCycle.cuh:255-303
    assert d.block_iterations == 10 and abs(d.omega - 0.85714) < 1e-6 and abs(d.target_reduction - 0.33) < 1e-6
    assert abs(d.theta - 1e-4) < 1e-9 and d.pre_smooth == 2 and d.post_smooth == 2 and d.coarsest_iterations == 50
    with np.testing.assert_raises(aw.AWError):
        aw.solver_default_desc(7)


def test_invalid_descriptor_rejected_before_any_gpu_work():
    d = aw.GridDesc()
    d.dims[:] = [2, 2, 2]
    d.block_size = 1.0
    d.base_res = 6  # not a power of two
    d.num_levels = 2
    h = C.c_void_p()
    st = aw.lib().aw_msbg_create(C.byref(d), C.byref(h))
    assert st == 1 and "power of two" in aw.lib().aw_last_error().decode()
    assert not h.value
