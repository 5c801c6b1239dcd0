"""Error paths that need no GPU.

The library checks a domain on the host before it touches a device, so a bad
domain returns DEM_ERR_ARG here as on a GPU box; a valid one returns
DEM_ERR_CUDA without a GPU.  The esys.lsm layer follows the reference's
worker-side handling of names that name nothing (TSubLattice::moveWallBy,
getWallPos, getWallForce, applyForceToWall, setExIG: SubLattice.hpp:2878-2891,
835-860, 897-921, 2935-2948, 1980-2009), checked on the CPU oracle backend.
The reference's damping fall-back (Damping.hpp:116-119: v_rel = 0 once
maxIterations is reached) is pinned for the restatement against the
reference's own classes.
"""
import ctypes
import math
import threading

import numpy as np
import pytest

import scenarios as S
from conftest import gpu_available

BAD_DOMAINS = [
    # (grid spacing, verlet distance, min, max, circ, dt, particle type, message fragment)
    (1.2, 0.2, (0, 0, 0), (0, 5, 5), (0, 0, 0), 1e-4, 0, "max must exceed min"),
    (1.2, 0.2, (0, 0, 0), (5, -1, 5), (0, 0, 0), 1e-4, 0, "max must exceed min"),
    (1.2, 0.2, (0, 0, 0), (5, 5, math.nan), (0, 0, 0), 1e-4, 0, "not finite"),
    (1.2, 0.2, (-math.inf, 0, 0), (5, 5, 5), (0, 0, 0), 1e-4, 0, "not finite"),
    (0.0, 0.2, (0, 0, 0), (5, 5, 5), (0, 0, 0), 1e-4, 0, "grid spacing"),
    (-1.0, 0.2, (0, 0, 0), (5, 5, 5), (0, 0, 0), 1e-4, 0, "grid spacing"),
    (1.2, -0.1, (0, 0, 0), (5, 5, 5), (0, 0, 0), 1e-4, 0, "verlet distance"),
    (1.2, 0.2, (0, 0, 0), (5, 5, 5), (0, 0, 0), 0.0, 0, "time step"),
    (1.2, 0.2, (0, 0, 0), (5, 5, 5), (0, 1, 0), 1e-4, 0, "only x may be periodic"),
    (1.2, 0.2, (0, 0, 0), (5, 5, 5), (0, 0, 1), 1e-4, 0, "only x may be periodic"),
    (1.2, 0.2, (0, 0, 0), (3.5, 5, 5), (1, 0, 0), 1e-4, 0, "at least 3 cells"),
    (1e-4, 0.0, (0, 0, 0), (100, 100, 100), (0, 0, 0), 1e-4, 0, "2^31 - 1 cells"),
    (1.2, 0.2, (0, 0, 0), (5, 5, 5), (0, 0, 0), 1e-4, 2, "particle type"),
]


def _create(lib, gs, vd, mn, mx, circ, dt, pt):
    h = ctypes.c_void_p()
    d3 = ctypes.c_double * 3
    rc = lib.dem_create(ctypes.byref(h), pt, gs, vd, d3(*mn), d3(*mx), (ctypes.c_int * 3)(*circ), dt)
    return rc, h


@pytest.mark.parametrize("case", BAD_DOMAINS, ids=lambda c: c[-1].replace(" ", "_"))
def test_bad_domain_is_an_argument_error_before_any_device_work(dem_lib, case):
    from esys.lsm import _capi

    *args, frag = case
    rc, h = _create(dem_lib, *args)
    assert rc == _capi.DEM_ERR_ARG and not h.value
    assert frag in dem_lib.dem_last_error(None).decode()
    # the Python binding raises with the same text and status
    gs, vd, mn, mx, circ, dt, pt = args
    with pytest.raises(_capi.DemError) as e:
        _capi.DemSim(pt, gs, vd, mn, mx, circ, dt)
    assert e.value.status == _capi.DEM_ERR_ARG and frag in str(e.value)


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU status of a valid domain")
def test_valid_domains_reach_the_device_check(dem_lib):
    """Domains the reference accepts pass the host checks: a periodic x side of 10 with
    range 3 (the reference adjusts the range to 10/3, SubLattice.hpp:506-515), exactly
    3 cells, a non-periodic side that is no multiple of the range (grown to whole cells)."""
    from esys.lsm import _capi

    for gs, mx, circ in ((3.0, (10, 4, 4), (1, 0, 0)), (1.0, (3, 1, 1), (1, 0, 0)), (1.2, (5.05, 0.3, 7.7), (0, 0, 0))):
        rc, h = _create(dem_lib, gs, 0.2, (0, 0, 0), mx, circ, 1e-4, 1)
        assert rc == _capi.DEM_ERR_CUDA and not h.value, (gs, mx, circ)
        assert "no usable GPU" in dem_lib.dem_last_error(None).decode()


def test_null_handle_text_is_per_thread(dem_lib):
    """dem_last_error(NULL) gives this thread's last dem_create failure, "null handle" before one."""
    out = []
    t = threading.Thread(target=lambda: out.append(dem_lib.dem_last_error(None)))
    t.start()
    t.join()
    assert out == [b"null handle"]
    rc, _ = _create(dem_lib, 1.2, 0.2, (0, 0, 0), (0, 5, 5), (0, 0, 0), 1e-4, 0)
    assert rc < 0 and dem_lib.dem_last_error(None).startswith(b"dem_create: ")


class OrcBackend:
    """The oracle's ctypes front end under the DemSim method names LsmMpi uses."""

    def __new__(cls, *a):
        import oracle

        sim = oracle.OracleSim("orc", *a)
        sim.set_timestep = lambda dt: None
        sim.num_particles = lambda: len(sim.particles()["id"])
        sim.close = lambda: None
        return sim


def _lsm_box(with_exclusion_typo=False):
    from esys.lsm import (LsmMpi, NRotElasticWallPrms, RotBondPrms, RotFrictionPrms, RotSphere)
    from esys.lsm.util import BoundingBox, Vec3

    sim = LsmMpi(numWorkerProcesses=1, mpiDimList=[1, 1, 1], _backend=OrcBackend)
    sim.initNeighbourSearch(particleType="RotSphere", gridSpacing=1.25, verletDist=0.2)
    sim.setTimeStepSize(1e-5)
    sim.setSpatialDomain(BoundingBox(Vec3(0, 0, 0), Vec3(3, 4, 3)))
    parts = []
    for i in range(12):
        p = RotSphere(id=i, posn=Vec3(0.5 + i % 3, 0.5 + (i // 3) % 4, 1.5), radius=0.5, mass=float(S.sphere_mass(0.5)))
        p.setLinearVelocity(Vec3(0.0, 0.3 * ((i % 2) - 0.5), 0.0))
        parts.append(p)
    sim.createParticles(parts)
    sim.createConnections([(1, i, i + 1) for i in range(0, 11, 3)])
    sim.createInteractionGroup(RotBondPrms("bonds", 1e5, 1e5, 1e3, 1e3, 1.0, 1.0, 1.0, 1.0, 1))
    sim.createInteractionGroup(RotFrictionPrms("friction", 1e5, 0.6, 0.6, 1e5))
    sim.createExclusion("bonds", "friction")
    if with_exclusion_typo:
        sim.createExclusion("bondz", "friction")
        sim.createExclusion("bonds", "fiction")
    sim.createWall(name="floor", posn=Vec3(0, 0, 0), normal=Vec3(0, 1, 0))
    sim.createInteractionGroup(NRotElasticWallPrms(name="floor_w", wallName="floor", normalK=1e5))
    return sim


def test_lsm_unknown_names_follow_the_reference(oracle_libs, capsys):
    """Unknown wall and group names: no exception, no effect, zero vectors read back, the
    exclusion error on the error console; the run is the one without the bad calls."""
    from esys.lsm.util import Vec3

    a, b = _lsm_box(with_exclusion_typo=True), _lsm_box()
    assert capsys.readouterr().err.count("nonexisting interaction group") == 2
    a.moveWallBy("no_such_wall", Vec3(0, 1, 0))
    a.applyForceToWall("no_such_group", Vec3(0, 5, 0))
    assert list(a.getWallPosition("no_such_wall")) == [0.0, 0.0, 0.0]
    assert list(a.getWallForce("no_such_wall")) == [0.0, 0.0, 0.0]
    for s in (a, b):
        s.setNumTimeSteps(30)
        s.run()
    assert list(a.getWallForce("floor")) == list(b.getWallForce("floor"))
    pa, pb = a._sim.particles(), b._sim.particles()
    for k in ("pos", "vel", "force"):
        assert np.array_equal(pa[k], pb[k]), k


def test_lsm_unknown_interaction_type_raises(oracle_libs):
    """CLatticeMaster / TSubLattice throw on an interaction type they do not know
    (SubLattice.hpp:1709-1714); the layer raises before anything reaches the worker."""
    from esys.lsm import LsmMpi
    from esys.lsm.util import BoundingBox, Vec3

    class FluidPrms:
        name = "fluid"

    sim = LsmMpi(_backend=OrcBackend)
    sim.initNeighbourSearch(particleType="NRotSphere", gridSpacing=1.2, verletDist=0.2)
    sim.setSpatialDomain(BoundingBox(Vec3(0, 0, 0), Vec3(4, 4, 4)))
    with pytest.raises(NotImplementedError):
        sim.createInteractionGroup(FluidPrms())
    with pytest.raises(NotImplementedError):
        sim.setSpatialDomain(BoundingBox(Vec3(0, 0, 0), Vec3(4, 4, 4)), circDimList=[False, True, False])


@pytest.mark.parametrize("max_iter", [0, 1, 3, 5, 100])
def test_damping_iteration_cap_matches_the_reference(oracle_libs, max_iter):
    """The restatement's damping equals the reference's CDamping / CRotDamping bit for bit at
    every maxIterations, including 0 and 1 (never damped: count >= maxIterations always)."""
    if not oracle_libs.available("ref"):
        pytest.skip("reference harness not built (reference tree absent)")
    a = S.damped_cloud(lambda *x: oracle_libs.OracleSim("orc", *x), max_iter=max_iter)
    b = S.damped_cloud(lambda *x: oracle_libs.OracleSim("ref", *x), max_iter=max_iter)
    a.step(5)
    b.step(5)
    pa, pb = a.particles(), b.particles()
    for k in ("pos", "vel", "angvel", "force", "moment"):
        assert np.array_equal(pa[k], pb[k]), k


def test_damping_cap_splits_the_cloud(oracle_libs):
    """With maxIterations = 3 the cloud holds both kinds of particle (damped and capped), so
    the cap is exercised both ways by the tests that use this case."""
    sim = S.damped_cloud(lambda *x: oracle_libs.OracleSim("orc", *x), max_iter=3)
    p = sim.particles()
    m = S.sphere_mass(0.4)
    f = np.array([0.0, 0.0, -9.81 * m])
    counts = [S.damping_iterations(v, f, 1.0 / m, m, 100.0, 1e-3, 3) for v in p["vel"]]
    capped = sum(c >= 3 for c in counts)
    assert 0 < capped < len(counts), counts
