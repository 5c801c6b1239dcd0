import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "esys-particle_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def dem_lib():
    """The built B200 DEM library (built on demand; never a CPU fallback)."""
    import build  # esys-particle_b200/build.py

    build.build()
    from esys.lsm import _capi

    return _capi.load_library()


@pytest.fixture(scope="session")
def oracle_libs():
    """Build the CPU restatement (and the reference harness when the reference tree is present)."""
    import subprocess

    odir = os.path.join(ROOT, "oracle")
    subprocess.run(["make", "-s", "-C", odir, "restate"], check=True)
    ref = os.environ.get("ESYS_REFERENCE_DIR", "/root/reference")
    if os.path.isdir(ref):
        subprocess.run(["make", "-s", "-j8", "-C", odir, "ref", f"REF={ref}"], check=True)
    import oracle

    return oracle


@pytest.fixture(scope="session")
def binding_lib(dem_lib):
    """The ASubLattice binding's test build (tests/binding): rebuilt when the reference tree is
    present, else the prebuilt library; skipped when neither exists."""
    import ctypes
    import subprocess

    bdir = os.path.join(ROOT, "tests", "binding")
    ref = os.environ.get("ESYS_REFERENCE_DIR", "/root/reference")
    if os.path.isdir(ref):
        subprocess.run(["make", "-s", "-j8", "-C", bdir, f"REF={ref}"], check=True)
    path = os.path.join(bdir, "_build", "libsublattice_binding.so")
    if not os.path.exists(path):
        pytest.skip("binding test build absent (needs the reference tree to build)")
    return ctypes.CDLL(path)
