"""The C-ABI libraries load without a GPU and export every entry point of
include/fasteddy_b200.h (no compute calls here)."""
from __future__ import annotations

import ctypes
import os
import re

from conftest import ROOT


def _declared_functions() -> list[str]:
    text = open(os.path.join(ROOT, "include", "fasteddy_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:int|void|size_t|long long|char)\s*\*?\s*([A-Za-z_]\w*)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_reference_entry_points():
    names = _declared_functions()
    for ref in ("cuda_gridInit", "cuda_hydroCoreInit", "cuda_timeIntInit", "cuda_timeIntCommence",
                "cuda_hydroCoreDeviceBuildFrhs", "fecuda_Init", "fecuda_SetBlocksPerGrid"):
        assert ref in names
    assert len(names) > 40


def test_every_declared_symbol_is_exported(fe):
    libs = fe.load()
    missing = [n for n in _declared_functions() if not any(hasattr(libs[k], n) for k in ("engine", "refabi"))]
    assert missing == []


def test_host_library_defines_the_reference_globals(fe):
    libs = fe.load()
    for g in ("Nxp", "Nyp", "Nzp", "Nh", "dt", "NtBatch", "simTime_it", "advectionSelector", "TKESelector"):
        assert ctypes.c_int.in_dll(libs["host"], g) is not None
    for g in ("hydroFlds", "hydroBaseStateFlds", "J31", "zPos", "sgstkeScalars", "moistScalars", "htFlux"):
        ctypes.c_void_p.in_dll(libs["host"], g)


def test_engine_reports_missing_gpu_instead_of_falling_back(fe):
    libs = fe.load()
    if libs["engine"].fe_device_count() > 0:
        return  # a GPU is present; the GPU tests cover the device path
    host = fe.cases.setup_host("cbl_dry", 8, 8, 8)
    try:
        with __import__("pytest").raises(fe.FeError, match="no CUDA device"):
            fe.Domain(host.config())
        assert libs["refabi"].fecuda_Init() != 0
    finally:
        host.cleanup()
