"""The ASubLattice binding (esys-particle_b200/integration/GpuSubLattice.h) compiled against the
reference's headers: the test build loads, holds the TGpuSubLattice operations the worker's
command loop calls, and, without a GPU, a worker that cannot open the device reports the
failure to the master through the reference's own protocol instead of hanging it."""
import subprocess

import pytest

import binding_driver as B
from conftest import gpu_available

OPERATIONS = ("initNeighborTable", "receiveParticles", "receiveConnections", "addWall", "addElasticWIG",
              "addPairIG", "addRotBondedIG", "addBondedIG", "addDamping", "addSingleIG", "setExIG",
              "checkNeighbors", "searchNeighbors", "updateInteractions", "oneStep", "exchangePos", "getWallForce",
              "getWallPos", "moveWallBy", "getParticleData", "countParticles", "saveCheckPointData",
              "loadCheckPointData")


def test_binding_builds_and_holds_the_worker_operations(binding_lib):
    B.bind(binding_lib)
    out = subprocess.run(["nm", "-C", binding_lib._name], capture_output=True, text=True, check=True).stdout
    for particle in ("CRotParticle", "CParticle"):
        for op in OPERATIONS:
            assert f"TGpuSubLattice<{particle}>::{op}(" in out, (particle, op)


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU path")
def test_worker_failure_reaches_the_master_without_a_gpu(binding_lib):
    with pytest.raises(B.BindingError) as e:
        B.SubLatticeMaster(binding_lib, "RotSphere", 1.2, 0.2, (0, 0, 0), (5, 5, 5))
    assert "no usable GPU" in str(e.value) and "other party failed" in str(e.value)
    assert binding_lib.slm_finish() == -1  # the worker's failure is reported again at the end
    # a bad domain is refused by the worker's initNeighborTable the same way
    with pytest.raises(B.BindingError) as e:
        B.SubLatticeMaster(binding_lib, "RotSphere", 1.2, 0.2, (0, 0, 0), (5, 5, 5), circ=(0, 1, 0))
    assert "only x may be periodic" in str(e.value)
    binding_lib.slm_finish()
