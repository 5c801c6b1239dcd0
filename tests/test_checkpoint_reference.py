"""Restart checkpoints on the CPU, with the reference-built harness: its own writers and
readers (TSubLattice::saveCheckPointData / loadCheckPointData order) round-trip a bonded
block, which pins the file layout the GPU library writes and reads (tests/test_gpu_checkpoint.py).

The RotFriction storage's writer runs the record count into the first record
(pis/pi_storage_ed.hpp:202-214), so the reference cannot read back a checkpoint that has
RotFriction interactions; the round trip here has bonds only, and the reader of these tests
(scenarios.parse_checkpoint) handles the run-together form.
"""
import numpy as np
import pytest

import scenarios as S

RATE = 0.002
STRONG = (5.0, 5.0, 5.0, 5.0)   # bonds that hold through the loading


@pytest.fixture(scope="module")
def ref(oracle_libs):
    if not oracle_libs.available("ref"):
        pytest.skip("reference harness not built")
    return lambda *a: oracle_libs.OracleSim("ref", *a)


def test_reference_round_trip(ref, tmp_path):
    a = S.bonded_block(ref, with_friction=False, strength=STRONG)
    S.run_loaded(a, 40, RATE)
    path = tmp_path / "cp_t=40_1.txt"
    a.save_checkpoint(path, 12)
    cp = S.parse_checkpoint(path)
    assert len(cp["particles"]) == len(a.particles()["id"])
    assert len(cp["bonds"]) == len(a.pairs("bonds")[0]) > 20
    b = S.bonded_block_script(ref, with_friction=False, strength=STRONG)
    b.load_checkpoint(path, a.timestep)
    assert b.timestep == a.timestep
    pa, pb = a.particles(), b.particles()
    oa, ob = np.argsort(pa["id"]), np.argsort(pb["id"])
    for k in ("pos", "vel", "angvel", "quat"):
        x, y = pa[k][oa], pb[k][ob]
        assert np.abs(x - y).max() <= 1e-11 * max(np.abs(x).max(), 1.0), k  # 12 significant digits
    ia, _, _ = a.pairs("bonds")
    ib, _, _ = b.pairs("bonds")
    assert len(ia) == len(ib)
    # the restarted run follows the original to within the file's precision
    S.run_loaded(a, 40, RATE)
    S.run_loaded(b, 40, RATE)
    pa, pb = a.particles(), b.particles()
    x, y = pa["pos"][np.argsort(pa["id"])], pb["pos"][np.argsort(pb["id"])]
    assert np.abs(x - y).max() <= 1e-8 * np.abs(x).max()
