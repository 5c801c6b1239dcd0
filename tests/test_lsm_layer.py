"""The esys.lsm scripting surface (LsmMpi, *Prms, particles, runnables): host
logic checked on the CPU by running a reference-style script on the CPU
oracle backend and comparing with the same calls made directly."""
import numpy as np

import scenarios as S


class OrcBackend:
    """Adapts the oracle's ctypes front end to the DemSim methods LsmMpi uses."""

    def __new__(cls, *a):
        import oracle

        sim = oracle.OracleSim("orc", *a)
        sim.set_timestep = lambda dt: None
        sim.num_particles = lambda: len(sim.particles()["id"])
        sim.close = lambda: None
        return sim


def test_lsmmpi_gravity_script_matches_direct_calls(oracle_libs):
    from esys.lsm import (GravityPrms, LinDampingPrms, LsmMpi, NRotElasticPrms, NRotElasticWallPrms, NRotSphere,
                          Runnable)
    from esys.lsm.util import BoundingBox, Vec3

    class Loader(Runnable):
        def __init__(self, sim):
            Runnable.__init__(self)
            self.sim, self.n = sim, 0

        def run(self):
            self.sim.moveWallBy("floor", Vec3(0, 0, 1e-4))
            self.n += 1

    sim = LsmMpi(numWorkerProcesses=1, mpiDimList=[1, 1, 1], _backend=OrcBackend)
    sim.initNeighbourSearch(particleType="NRotSphere", gridSpacing=1.2, verletDist=0.2)
    sim.setNumTimeSteps(60)
    sim.setTimeStepSize(1e-4)
    sim.setSpatialDomain(BoundingBox(Vec3(0, 0, 0), Vec3(4, 4, 8)))
    rng = np.random.default_rng(7)
    parts = []
    for i in range(12):
        p = NRotSphere(id=i, posn=Vec3(0.6 + (i % 3) * 1.1, 0.6 + (i // 3 % 2) * 1.1, 0.6 + (i // 6) * 1.0),
                       radius=0.45, mass=float(S.sphere_mass(0.45)))
        p.setLinearVelocity(Vec3(*rng.normal(0, 0.5, 3)))
        parts.append(p)
    sim.createParticles(parts)
    sim.createInteractionGroup(NRotElasticPrms(name="elastic", normalK=1000.0))
    sim.createInteractionGroup(GravityPrms(name="g", acceleration=Vec3(0, 0, -9.81)))
    sim.createWall(name="floor", posn=Vec3(0, 0, 0), normal=Vec3(0, 0, 1))
    sim.createInteractionGroup(NRotElasticWallPrms(name="floor_w", wallName="floor", normalK=1000.0))
    sim.createInteractionGroup(LinDampingPrms(name="damp", viscosity=0.01, maxIterations=100))
    loader = Loader(sim)
    sim.addPreTimeStepRunnable(loader)
    sim.run()
    assert loader.n == 60 and sim.getTimeStep() == 60

    d = OrcBackend("NRotSphere", 1.2, 0.2, (0, 0, 0), (4, 4, 8), (0, 0, 0), 1e-4)
    d.add_particles([p.getId() for p in parts], [list(p.getPosn()) for p in parts], [0.45] * 12,
                    [float(S.sphere_mass(0.45))] * 12, tag=[0] * 12, vel=[list(p.getLinearVelocity()) for p in parts])
    d.add_elastic_group("elastic", 1000.0, True)
    d.add_gravity("g", (0, 0, -9.81))
    d.add_wall("floor", (0, 0, 0), (0, 0, 1))
    d.add_wall_group("floor_w", "floor", 1000.0)
    d.add_damping(0, 0.01, 100)
    for _ in range(60):
        d.move_wall("floor", (0, 0, 1e-4))
        d.step(1)
    a, b = sim._sim.particles(), d.particles()
    for k in ("pos", "vel", "force"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(np.array(list(sim.getWallForce("floor"))), d.wall("floor")[1])
    assert len(sim.getParticleList()) == 12


def test_lsmmpi_rejects_groups_outside_the_path(oracle_libs):
    import pytest

    from esys.lsm import LsmMpi
    from esys.lsm.util import BoundingBox, Vec3

    sim = LsmMpi(_backend=OrcBackend)
    with pytest.raises(NotImplementedError):
        sim.initNeighbourSearch(particleType="RotThermSphere", gridSpacing=1.0, verletDist=0.1)
    sim.initNeighbourSearch(particleType="RotSphere", gridSpacing=1.0, verletDist=0.1)
    sim.setSpatialDomain(BoundingBox(Vec3(0, 0, 0), Vec3(3, 3, 3)))
    with pytest.raises(NotImplementedError):
        sim.readMesh("x.msh", "mesh")


def test_connection_finder_bonds_touching_pairs():
    from esys.lsm import ConnectionFinder, RotSphere
    from esys.lsm.util import Vec3

    ps = [RotSphere(0, Vec3(0, 0, 0), 0.5, 1.0), RotSphere(1, Vec3(1.0005, 0, 0), 0.5, 1.0),
          RotSphere(2, Vec3(3, 0, 0), 0.5, 1.0)]
    c = list(ConnectionFinder(maxDist=1e-3, bondTag=4, pList=ps))
    assert c == [(4, 0, 1)]


class RefBackend(OrcBackend):
    """The reference-built harness behind the same adapter."""

    def __new__(cls, *a):
        import oracle

        sim = oracle.OracleSim("ref", *a)
        sim.set_timestep = lambda dt: None
        sim.num_particles = lambda: len(sim.particles()["id"])
        sim.close = lambda: None
        return sim


def test_lsmmpi_widened_law_prms_match_direct_calls(oracle_libs):
    """HertzMindlinPrms, NRotFrictionPrms, LocalDampingPrms and the older createDamping /
    createGravity spellings reach the same groups (time step included: LsmMpiPy's
    createHertzMindlinIG and createNRotFrictionInteractGrp take it from the model) as direct calls."""
    import pytest

    from esys.lsm import (GravityPrms, HertzMindlinPrms, LocalDampingPrms, LsmMpi, NRotFrictionPrms, NRotSphere)
    from esys.lsm.util import BoundingBox, Vec3

    if not oracle_libs.available("ref"):
        pytest.skip("reference harness not built")
    for law in ("hm", "nfric"):
        sim = LsmMpi(numWorkerProcesses=1, mpiDimList=[1, 1, 1], _backend=RefBackend)
        sim.initNeighbourSearch(particleType="NRotSphere", gridSpacing=1.2, verletDist=0.1)
        sim.setNumTimeSteps(80)
        sim.setTimeStepSize(1e-4)
        sim.setSpatialDomain(BoundingBox(Vec3(0, 0, 0), Vec3(4, 4, 8)))
        rng = np.random.default_rng(11)
        parts = []
        for i in range(18):
            p = NRotSphere(id=i, posn=Vec3(0.6 + (i % 3) * 0.9, 0.6 + (i // 3 % 2) * 0.9, 0.6 + (i // 6) * 0.9),
                           radius=0.47, mass=float(S.sphere_mass(0.47)))
            p.setLinearVelocity(Vec3(*rng.normal(0, 0.5, 3)))
            parts.append(p)
        sim.createParticles(parts)
        if law == "hm":
            sim.createInteractionGroup(HertzMindlinPrms(name="c", youngsModulus=1e4, poissonsRatio=0.3,
                                                        dynamicMu=0.4))
        else:
            sim.createInteractionGroup(NRotFrictionPrms(name="c", normalK=1e4, dynamicMu=0.4, shearK=5e3))
        sim.createGravity(GravityPrms(name="g", acceleration=Vec3(0, 0, -9.81)))
        sim.createDamping(LocalDampingPrms(name="local", viscosity=0.05))
        sim.run()

        d = RefBackend("NRotSphere", 1.2, 0.1, (0, 0, 0), (4, 4, 8), (0, 0, 0), 1e-4)
        d.add_particles([p.getId() for p in parts], [list(p.getPosn()) for p in parts], [0.47] * 18,
                        [float(S.sphere_mass(0.47))] * 18, tag=[0] * 18,
                        vel=[list(p.getLinearVelocity()) for p in parts])
        if law == "hm":
            d.add_hertz_mindlin_group("c", 1e4, 0.3, 0.4, 1e-4)
        else:
            d.add_nrot_friction_group("c", 1e4, 0.4, 5e3, 1e-4, True)
        d.add_gravity("g", (0, 0, -9.81))
        d.add_local_damping("local", 0, 0.05)
        d.step(80)
        a, b = sim._sim.particles(), d.particles()
        for k in ("pos", "vel", "force"):
            assert np.array_equal(a[k], b[k]), (law, k)
        st = np.array(d.pairs("c")[2])
        assert st[:, 4].sum() > 5, law  # contacts were touching
