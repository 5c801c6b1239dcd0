"""Pin the CPU restatement (oracle/dem_oracle.cpp) against the reference itself.

The reference's own hot-path classes are compiled into oracle/_ref by
oracle/Makefile (single-rank MPI shim).  On non-periodic inputs the restatement
follows the reference's interaction-list order, so every particle field, pair
set, pair state and bond-break event must be bit-identical.  The committed
golden fixtures (tests/golden, made by tests/golden/make_golden.py from the
reference harness) pin the restatement where the reference tree is absent.
"""
import os

import numpy as np
import pytest

import scenarios as S

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _mk(oracle, backend):
    return lambda *a: oracle.OracleSim(backend, *a)


def _need_ref(oracle):
    if not oracle.available("ref"):
        pytest.skip("reference harness not built (reference tree absent)")


def _same_state(a, b, groups):
    pa, pb = a.particles(), b.particles()
    for k in ("id", "pos", "vel", "angvel", "quat", "force", "moment"):
        assert np.array_equal(pa[k], pb[k]), k
    for g in groups:
        x, y = a.pairs(g), b.pairs(g)
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1]), g
        assert np.array_equal(x[2], y[2]), g


def test_kat_two_sphere_friction(oracle_libs):
    """Two-sphere RotFriction known answer (values from a run of the reference's own classes)."""
    m = S.sphere_mass([0.5, 0.5])
    for backend in ("ref", "orc"):
        if backend == "ref" and not oracle_libs.available("ref"):
            continue
        s = oracle_libs.OracleSim(backend, "RotSphere", 2.5, 0.2, (-5, -5, -5), (5, 5, 5), dt=5e-5)
        s.add_particles([0, 1], [[0, 0, 0], [0.95, 0.01, 0]], [0.5, 0.5], m, vel=[[0, 0, 0], [0, 0.1, 0]])
        s.add_rot_friction_group("f", 1e4, 0.6, 0.6, 1e4, 5e-5)
        s.step(1)
        p = s.particles()
        assert p["force"][0][0] == pytest.approx(-124.861638918223, rel=1e-14)
        assert p["force"][0][1] == pytest.approx(-1.30183304124445, rel=1e-14)
        assert p["moment"][0][2] == pytest.approx(0.0059375, rel=1e-12)


def test_kat_two_sphere_elastic(oracle_libs):
    """Non-rotational spheres 0.9 apart with k=1000: F0 = (-25, 0, 0), the elastic law by hand."""
    m = S.sphere_mass([0.5, 0.5])
    s = oracle_libs.OracleSim("orc", "NRotSphere", 2.5, 0.2, (-5, -5, -5), (5, 5, 5), dt=1e-4)
    s.add_particles([0, 1], [[0, 0, 0], [0.9, 0, 0]], [0.5, 0.5], m)
    s.add_elastic_group("e", 1000.0, True)
    s.step(1)
    p = s.particles()
    assert np.allclose(p["force"][0], [-25.0, 0, 0], rtol=1e-13, atol=1e-12)
    assert np.allclose(p["force"][1], [25.0, 0, 0], rtol=1e-13, atol=1e-12)


def test_kat_two_sphere_bond(oracle_libs):
    """Bonded pair stretched by 0.001 in x after creation: F0 and M0z of the reference's own classes."""
    m = S.sphere_mass([0.5, 0.5])
    for backend in ("ref", "orc"):
        if backend == "ref" and not oracle_libs.available("ref"):
            continue
        s = oracle_libs.OracleSim(backend, "RotSphere", 2.5, 0.2, (-5, -5, -5), (5, 5, 5), dt=5e-5)
        s.add_particles([0, 1], [[0, 0, 0], [0.95, 0.01, 0]], [0.5, 0.5], m, tag=[0, 1],
                        vel=[[0, 0, 0], [0, 0.1, 0]])
        s.add_connections([1], [0], [1])
        s.add_rot_bond_group("b", 1, 1e5, 1e5, 1e3, 1e3, 0.5, 1.0, 1.0, 0.5)
        s.move_tagged(1, [0.001, 0, 0])
        s.step(1)
        p = s.particles()
        assert p["force"][0][0] == pytest.approx(-1162.49872032201, rel=1e-12)
        assert p["force"][0][1] == pytest.approx(-12.4868428309419, rel=1e-12)
        assert p["moment"][0][2] == pytest.approx(-0.125000164502805, rel=1e-12)
        assert len(s.breaks()[0]) == 0


@pytest.mark.parametrize("steps", [1, 250])
def test_restatement_matches_reference_gravity(oracle_libs, steps):
    _need_ref(oracle_libs)
    a = S.gravity_box(_mk(oracle_libs, "ref"), 5)
    b = S.gravity_box(_mk(oracle_libs, "orc"), 5)
    a.step(steps)
    b.step(steps)
    _same_state(a, b, ["elastic"])
    for w in ("xlo", "zlo"):
        assert np.array_equal(a.wall(w)[1], b.wall(w)[1])


@pytest.mark.parametrize("steps", [1, 250])
def test_restatement_matches_reference_friction(oracle_libs, steps):
    _need_ref(oracle_libs)
    a = S.friction_pack(_mk(oracle_libs, "ref"))
    b = S.friction_pack(_mk(oracle_libs, "orc"))
    a.step(steps)
    b.step(steps)
    _same_state(a, b, ["friction"])


def test_restatement_matches_reference_bond_breaking(oracle_libs):
    """Bonds break under platen loading; RotFriction takes over through the
    exclusion and the flagged-pair list: break events must be identical."""
    _need_ref(oracle_libs)
    a = S.bonded_block(_mk(oracle_libs, "ref"), strength=(0.05, 0.1, 0.1, 0.05))
    b = S.bonded_block(_mk(oracle_libs, "orc"), strength=(0.05, 0.1, 0.1, 0.05))
    S.run_loaded(a, 400, 2e-4)
    S.run_loaded(b, 400, 2e-4)
    _same_state(a, b, ["bonds", "friction"])
    ea, eb = a.breaks(), b.breaks()
    assert len(ea[0]) > 0
    for x, y in zip(ea, eb):
        assert np.array_equal(x, y)


def test_restatement_matches_reference_wall_servo(oracle_libs):
    _need_ref(oracle_libs)
    sims = []
    for backend in ("ref", "orc"):
        s = S.gravity_box(_mk(oracle_libs, backend), 4)
        s.step(50)
        s.apply_force_to_wall("zhi_w", (0, 0, -50.0))
        s.step(20)
        sims.append(s)
    assert np.array_equal(sims[0].wall("zhi")[0], sims[1].wall("zhi")[0])
    _same_state(sims[0], sims[1], ["elastic"])


@pytest.mark.parametrize("name", ["gravity_box", "friction_pack", "bonded_block"])
def test_restatement_matches_golden(oracle_libs, name):
    """The restatement reproduces the golden fixtures produced by the reference harness."""
    import golden_cases

    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.skip("golden fixture missing")
    g = np.load(path)
    sim = golden_cases.run(name, _mk(oracle_libs, "orc"))
    golden_cases.assert_matches(g, sim, exact=True, name=name)
