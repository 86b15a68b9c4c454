"""CPU tests of the C ABI: the library loads, exports everything the public
header declares, and validates arguments before touching a device."""
import ctypes
import os
import re
import subprocess

import pytest

from analyticalreconbigpatient_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "helixrecon.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(?:void|int|size_t|const char\*)\s+(\w+)\s*\(", src)
    return sorted(set(names))


def test_header_declares_reference_entry_points():
    names = declared_functions()
    for ref in ("ParallelRebinningCBCurve_GPU", "filtering", "ParallekFDKHelical3DWeighting_GPU_float",
                "ParallekFDKHelical3DWeighting_GPU_double", "ParallelFDKHelical3DWeighting"):
        assert ref in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_functions()) <= set(_lib.exported_symbols())


def test_library_is_built_for_sm100a_only():
    out = subprocess.run(["cuobjdump", "--list-elf", _lib.LIB_PATH], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    arches = set(re.findall(r"sm_\w+", out.stdout))
    assert arches == {"sm_100a"}, arches


def test_argument_validation_precedes_device_use():
    lib = _lib.load()
    plan = ctypes.c_void_p()
    st = lib.hr_rebin_plan_create(ctypes.byref(plan), 0, 4, 10, 1.0, 0.01, 0.1, 1.0, 1.0, 0.1, 541.0)
    assert st == 1 and b"sizes" in lib.hr_last_error()
    st = lib.hr_filter_plan_create(ctypes.byref(plan), 4096, 4, 10, 1.0, 1.0, 1.0, 1.0, 541.0)
    assert st == 1 and b"2048" in lib.hr_last_error()
    g = _lib.BpGeom(N_2pi=984, XN=4, YN=4, ZN=4, YL=888, ZL=64, PN=100, h=0.0, DeltaFai=0.1, dYL=1, dZL=1, SO=541)
    w = (ctypes.c_double * 984)()
    st = lib.hr_bp_plan_create(ctypes.byref(plan), ctypes.byref(g), ctypes.cast(w, ctypes.c_void_p), 0)
    assert st == 1 and b"non-zero" in lib.hr_last_error()
    st = lib.hr_rebin_host(None, None, 4, 4, 4, 1.0, 0.01, 0.1, 1.0, 1.0, 0.1, 541.0)
    assert st == 1
    descs = (_lib.ReconDesc * 17)()
    st = lib.hr_batch_plan_create(ctypes.byref(plan), descs, 17)
    assert st == 1 and b"1..16" in lib.hr_last_error()
    st = lib.hr_batch_plan_create(ctypes.byref(plan), descs, 2)
    assert st == 1 and b"weight table" in lib.hr_last_error()
    st = lib.hr_batch_execute_host(None, None, None)
    assert st == 1 and b"hr_batch_execute_host" in lib.hr_last_error()
    st = lib.hr_add_poisson_noise(None, 10, 1e5, 1, None)
    assert st == 1


def test_no_device_is_reported_not_crashed():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = _lib.load()
    plan = ctypes.c_void_p()
    st = lib.hr_rebin_plan_create(ctypes.byref(plan), 8, 4, 10, 3.5, 0.01, 0.1, 3.5, 1.0, 0.1, 541.0)
    assert st == 4  # HR_ERR_NO_DEVICE
    assert b"no CUDA device" in lib.hr_last_error()


def test_view_weights_host_function_matches_oracle():
    import numpy as np

    import oracle
    from analyticalreconbigpatient_b200 import api

    for n2, hs, de in ((984, 0.68, 60), (492, 0.68, 60), (120, 0.7, 8), (101, 0.6, 5)):
        np.testing.assert_array_equal(api.weight_table(n2, hs, de), oracle.weight_table(n2, hs, de))
