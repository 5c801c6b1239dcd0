"""Restart checkpoints of the GPU worker against the reference's own writers and readers
(the reference-built harness).  All tests need a GPU.

- The file the GPU writes equals, field by field, the one the reference writes on the same run:
  particle records, RotBond restart records, RotFriction records, walls.  Bars: integers,
  flags and pair / bond sets exact; creation vectors and scaled constants to 1e-10 relative;
  dynamic state within 1e-9 of each field's scale (the two runs differ by summation order).
- The reference reads the GPU's file; the GPU reads the reference's (whose RotFriction record
  count runs into the first record).  Restarted runs continue alike (1e-9 of scale, identical
  bond-failure events), and a restart follows the uninterrupted run to within the file's 12
  digits.
"""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu

RATE = 0.002
STEPS = 40


@pytest.fixture(scope="module")
def gpu(dem_lib):
    from esys.lsm import _capi

    return lambda *a: _capi.DemSim(*a)


@pytest.fixture(scope="module")
def ref(oracle_libs):
    if not oracle_libs.available("ref"):
        pytest.skip("reference harness not built")
    return lambda *a: oracle_libs.OracleSim("ref", *a)


def _by_id(p, k):
    return p[k][np.argsort(p["id"])]


def _close(x, y, rel, what):
    x, y = np.asarray(x, float), np.asarray(y, float)
    scale = max(np.abs(y).max(), 1e-300)
    assert np.abs(x - y).max() <= rel * scale, (what, np.abs(x - y).max() / scale)


@pytest.fixture(scope="module")
def written(gpu, ref, tmp_path_factory):
    d = tmp_path_factory.mktemp("cp")
    g, r = S.bonded_block(gpu), S.bonded_block(ref)
    g.set_option("store_forces", 1)
    S.run_loaded(g, STEPS, RATE)
    S.run_loaded(r, STEPS, RATE)
    pg, pr = d / "gpu_t=40_1.txt", d / "ref_t=40_1.txt"
    g.save_checkpoint(pg, 12)
    r.save_checkpoint(pr, 12)
    return g, r, pg, pr


def test_gpu_file_matches_reference_writer(written):
    g, r, pg, pr = written
    cg, cr = S.parse_checkpoint(pg), S.parse_checkpoint(pr)
    assert cg["base"] == cr["base"]
    assert cg["particles"].keys() == cr["particles"].keys()
    ids = sorted(cr["particles"])
    A = np.array([cg["particles"][i] for i in ids])
    B = np.array([cr["particles"][i] for i in ids])
    assert A.shape == B.shape == (len(ids), 32)
    exact = [3, 4, 5, 6, 7, 8, 9, 19, 20, 21, 22, 23, 31]  # radius, id, tag, mass, initial position, shift, flags, inertia
    assert np.array_equal(A[:, exact], B[:, exact])
    for name, cols in (("pos", [0, 1, 2]), ("oldpos", [10, 11, 12]), ("vel", [13, 14, 15]), ("force", [16, 17, 18]),
                       ("quat", [24, 25, 26, 27]), ("angvel", [28, 29, 30])):
        _close(A[:, cols], B[:, cols], 1e-9, name)
    # RotBond restart records: same bonds, constants and creation vectors
    assert cg["bonds"].keys() == cr["bonds"].keys() and len(cr["bonds"]) > 0
    for k in cr["bonds"]:
        _close(cg["bonds"][k], cr["bonds"][k], 1e-10, ("bond", k))
    # RotFriction records: same pairs, flags; histories within the dynamic-state bar
    assert cg["friction"].keys() == cr["friction"].keys() and len(cr["friction"]) > 0
    keys = sorted(cr["friction"])
    Fa = np.array([cg["friction"][k] for k in keys])
    Fb = np.array([cr["friction"][k] for k in keys])
    # fields after the first: r0, mu_d, mu_s, ks, dt, scaling, meanR, id1, id2, slipping, touching, Ffric
    assert np.array_equal(Fa[:, 5:11], Fb[:, 5:11])
    _close(Fa[:, 0:5], Fb[:, 0:5], 1e-10, "friction constants")
    _close(Fa[:, 11:14], Fb[:, 11:14], 1e-9, "friction history")
    assert cg["walls"].keys() == cr["walls"].keys()
    for w in cr["walls"]:
        _close(cg["walls"][w], cr["walls"][w], 1e-12, w)


def test_reference_reads_gpu_file_and_both_continue_alike(gpu, ref, written):
    g, r, pg, pr = written
    r2, g2 = S.bonded_block_script(ref), S.bonded_block_script(gpu)
    r2.load_checkpoint(pg, g.timestep)
    g2.load_checkpoint(pg, g.timestep)
    assert r2.timestep == g2.timestep == g.timestep
    S.run_loaded(r2, STEPS, RATE)
    S.run_loaded(g2, STEPS, RATE)
    pa, pb = g2.particles(), r2.particles()
    for k in ("pos", "vel", "angvel", "quat"):
        _close(_by_id(pa, k), _by_id(pb, k), 1e-9, k)
    ea, eb = g2.breaks(), r2.breaks()
    assert set(zip(*(x.tolist() for x in ea))) == set(zip(*(x.tolist() for x in eb)))
    fa, fb = g2.pairs("friction"), r2.pairs("friction")
    assert set(zip(fa[0].tolist(), fa[1].tolist())) == set(zip(fb[0].tolist(), fb[1].tolist()))


def test_gpu_reads_reference_file(gpu, ref, written):
    g, r, pg, pr = written
    g3 = S.bonded_block_script(gpu)
    g3.load_checkpoint(pr, r.timestep)
    pa, pb = g3.particles(), r.particles()
    for k in ("pos", "vel", "angvel", "quat"):
        _close(_by_id(pa, k), _by_id(pb, k), 1e-11, k)  # the file's 12 significant digits
    # touching friction pairs keep their history through the load's neighbour search
    fa, fb = g3.pairs("friction"), r.pairs("friction")
    ka = {(int(a), int(b)): s for a, b, s in zip(*fa)}
    kb = {(int(a), int(b)): s for a, b, s in zip(*fb)}
    touching = [k for k, s in kb.items() if s[4] > 0]  # state: tangential force (3), slipping, touching
    assert touching, "no touching friction pair in the checkpoint"
    for k in touching:
        assert k in ka
        _close(ka[k][:3], kb[k][:3], 1e-10, ("history", k))
    # the restart follows the uninterrupted run to within the file's precision
    S.run_loaded(g3, STEPS, RATE)
    S.run_loaded(r, STEPS, RATE)
    pa, pb = g3.particles(), r.particles()
    _close(_by_id(pa, "pos"), _by_id(pb, "pos"), 1e-8, "pos after restart")
