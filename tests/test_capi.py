"""The C-ABI library builds, loads and exports every symbol include/esys_dem.h
declares (no compute: runs without a GPU); without a GPU dem_create fails
with a status instead of falling back to the CPU."""
import os
import re

import pytest

from conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "esys_dem.h")


def declared_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(dem_[a-z_0-9]+)\s*\(", txt)))


def test_header_declares_the_abi():
    syms = declared_symbols()
    assert "dem_create" in syms and "dem_step" in syms and len(syms) >= 25


def test_library_exports_every_declared_symbol(dem_lib):
    from esys.lsm import _capi

    for s in declared_symbols():
        assert hasattr(dem_lib, s), s
        assert s in _capi.SIGNATURES, f"{s} not bound in esys/lsm/_capi.py"


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_create_without_gpu_fails_loudly(dem_lib):
    from esys.lsm import _capi

    with pytest.raises(_capi.DemError):
        _capi.DemSim("NRotSphere", 1.2, 0.2, (0, 0, 0), (5, 5, 5))
