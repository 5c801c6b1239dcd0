"""esys.lsm on a B200: the ESyS-Particle scripting surface for the DEM hot path.

Scripts written for the reference (``from esys.lsm import *``) drive the GPU
worker through the same names, keywords and parameter classes:
``LsmMpi`` (Python/esys/lsm/LsmMpiPy.cpp:2056-3514), the ``*Prms`` classes
(Python/esys/lsm/InteractionParamsPy.cpp, WallPrmsPy.cpp), ``NRotSphere`` /
``RotSphere`` (ParticlePy.cpp, RotParticlePy.cpp) and ``Runnable`` hooks.
There are no MPI ranks: ``numWorkerProcesses`` and ``mpiDimList`` are accepted
and ignored, the single worker is one ``dem_sim`` handle on the current GPU.
Interaction groups outside the GPU path (meshes, fluids, the ~35 other laws)
raise ``NotImplementedError``.
"""
from __future__ import annotations

import sys

import numpy as np

from . import _capi
from .checkpoint import CheckPointer, CheckPointPrms, RestartCheckPointPrms, read_info, walls_in, worker_file
from .fields import (FieldSaver, InteractionScalarFieldSaverPrms, ParticleScalarFieldSaverPrms,
                     ParticleVectorFieldSaverPrms, TaggedParticleScalarFieldSaverPrms,
                     TaggedParticleVectorFieldSaverPrms, WallVectorFieldSaverPrms)
from .util import BoundingBox, Vec3

__all__ = [
    "LsmMpi", "NRotSphere", "RotSphere", "Runnable", "NRotElasticPrms", "RotFrictionPrms", "RotBondPrms",
    "NRotElasticWallPrms", "LinDampingPrms", "RotDampingPrms", "GravityPrms", "Vec3", "BoundingBox",
    "ConnectionFinder", "ParticleScalarFieldSaverPrms", "InteractionScalarFieldSaverPrms", "WallVectorFieldSaverPrms",
    "ParticleVectorFieldSaverPrms", "TaggedParticleScalarFieldSaverPrms", "TaggedParticleVectorFieldSaverPrms",
    "CheckPointPrms", "RestartCheckPointPrms", "NRotFrictionPrms", "NRotBondPrms", "LocalDampingPrms",
    "RotLocalDampingPrms", "HertzMindlinPrms", "BrittleBeamDZCPrms", "BrittleBeamSCPrms", "HertzMindlinViscoPrms",
]


# ---- particles (ParticlePy.cpp:90-140, RotParticlePy.cpp:143-230) ---------------------------
class NRotSphere:
    _rot = False

    def __init__(self, id=0, posn=Vec3(), radius=1.0, mass=1.0):
        self._id, self._pos, self._rad, self._mass = int(id), Vec3(*posn), float(radius), float(mass)
        self._tag, self._vel, self._angvel = 0, Vec3(), Vec3()

    def getId(self):
        return self._id

    def getTag(self):
        return self._tag

    def setTag(self, tag):
        self._tag = int(tag)

    def getPosn(self):
        return self._pos

    getPosition = getPosn
    getCentre = getCenter = getPosn

    def setPosn(self, p):
        self._pos = Vec3(*p)

    setPosition = setPosn

    def getRadius(self):
        return self._rad

    getRad = getRadius

    def getMass(self):
        return self._mass

    def getLinearVelocity(self):
        return self._vel

    getVelocity = getLinearVelocity

    def setLinearVelocity(self, v):
        self._vel = Vec3(*v)

    setVelocity = setLinearVelocity


class RotSphere(NRotSphere):
    _rot = True

    def getAngularVelocity(self):
        return self._angvel

    def setAngularVelocity(self, w):
        self._angvel = Vec3(*w)


# ---- interaction parameters (InteractionParamsPy.cpp, WallPrmsPy.cpp) ------------------------
class NRotElasticPrms:  # InteractionParamsPy.cpp:195-226
    def __init__(self, name, normalK, scaling=True):
        self.name, self.normalK, self.scaling = name, float(normalK), bool(scaling)


class RotFrictionPrms:  # InteractionParamsPy.cpp:772-834
    def __init__(self, name, normalK, dynamicMu, staticMu, shearK, scaling=True, rigid=False, meanR_scaling=True):
        self.name, self.normalK, self.dynamicMu, self.staticMu = name, float(normalK), float(dynamicMu), float(staticMu)
        self.shearK, self.scaling, self.rigid, self.meanR_scaling = float(shearK), bool(scaling), bool(rigid), bool(
            meanR_scaling)


class RotBondPrms:  # InteractionParamsPy.cpp:414-547, 2048-2170
    def __init__(self, name, normalK, shearK, torsionK, bendingK, normalBrkForce, shearBrkForce, torsionBrkForce,
                 bendingBrkForce, tag, scaling=True, meanR_scaling=True, truncated=1.0):
        self.name, self.tag = name, int(tag)
        self.normalK, self.shearK, self.torsionK, self.bendingK = (float(x) for x in (normalK, shearK, torsionK,
                                                                                      bendingK))
        self.normalBrkForce, self.shearBrkForce = float(normalBrkForce), float(shearBrkForce)
        self.torsionBrkForce, self.bendingBrkForce = float(torsionBrkForce), float(bendingBrkForce)
        self.scaling, self.meanR_scaling, self.truncated = bool(scaling), bool(meanR_scaling), float(truncated)


class NRotFrictionPrms:  # InteractionParamsPy.cpp:1446-1480 (CFrictionIGP)
    def __init__(self, name, normalK, dynamicMu, shearK, scaling=True):
        self.name, self.normalK, self.dynamicMu, self.shearK = name, float(normalK), float(dynamicMu), float(shearK)
        self.scaling = bool(scaling)


class NRotBondPrms:  # InteractionParamsPy.cpp:1090-1130 (CBondedIGP)
    def __init__(self, name, normalK, breakDistance, tag, scaling=True):
        self.name, self.normalK, self.breakDistance, self.tag = name, float(normalK), float(breakDistance), int(tag)
        self.scaling = bool(scaling)


class NRotElasticWallPrms:  # WallPrmsPy.cpp:213-243
    def __init__(self, name, wallName, normalK):
        self.name, self.wallName, self.normalK = name, wallName, float(normalK)


class LinDampingPrms:  # InteractionParamsPy.cpp:46-53, 998-1016
    def __init__(self, name, viscosity, maxIterations=100):
        self.name, self.viscosity, self.maxIterations = name, float(viscosity), int(maxIterations)


class RotDampingPrms(LinDampingPrms):
    pass


class HertzMindlinPrms:  # InteractionParamsPy.cpp:1350-1380 (CHertzMindlinIGP)
    def __init__(self, name, youngsModulus, poissonsRatio, dynamicMu):
        self.name, self.youngsModulus, self.poissonsRatio = name, float(youngsModulus), float(poissonsRatio)
        self.dynamicMu = float(dynamicMu)


class BrittleBeamDZCPrms:  # InteractionParamsPy.cpp:711-727, 1733-1760 (BrittleBeamDZCIGP)
    """Stiffnesses from the beam's Young's modulus and Poisson's ratio as ARotBondedIGP forms them
    (Model/ARotBondedInteraction.cpp: kr = kb = pi E, ks = kt = pi E / (2 (1 + nu)))."""

    def __init__(self, name, youngsModulus, poissonsRatio, cohesion, frictionAngle, tensileCutoff, compressCutoff,
                 beta1, beta2, tag):
        import math

        self.name, self.tag = name, int(tag)
        E, nu = float(youngsModulus), float(poissonsRatio)
        G = E / (2.0 * (1. + nu))
        self.kr, self.ks, self.kb, self.kt = math.pi * E, math.pi * G, math.pi * E, math.pi * G
        self.cohesion, self.frictionAngle = float(cohesion), float(frictionAngle)
        self.tensileCutoff, self.compressCutoff = float(tensileCutoff), float(compressCutoff)
        self.beta1, self.beta2 = float(beta1), float(beta2)


class BrittleBeamSCPrms:  # InteractionParamsPy.cpp:1689-1715 (BrittleBeamSCIGP)
    """Stiffnesses from E and nu as for BrittleBeamDZCPrms."""

    def __init__(self, name, youngsModulus, poissonsRatio, cohesion, frictionAngle, tensileCutoff, tag):
        import math

        self.name, self.tag = name, int(tag)
        E, nu = float(youngsModulus), float(poissonsRatio)
        G = E / (2.0 * (1. + nu))
        self.kr, self.ks, self.kb, self.kt = math.pi * E, math.pi * G, math.pi * E, math.pi * G
        self.cohesion, self.frictionAngle, self.tensileCutoff = float(cohesion), float(frictionAngle), float(tensileCutoff)


class HertzMindlinViscoPrms:  # InteractionParamsPy.cpp:1390-1420 (CHertzMindlinViscoIGP)
    def __init__(self, name, youngsModulus, poissonsRatio, dynamicMu, restitution):
        self.name, self.youngsModulus, self.poissonsRatio = name, float(youngsModulus), float(poissonsRatio)
        self.dynamicMu, self.restitution = float(dynamicMu), float(restitution)


class LocalDampingPrms:  # InteractionParamsPy.cpp:1033-1048 (CLocalDampingIGP "LocalDamping")
    def __init__(self, name, viscosity):
        self.name, self.viscosity = name, float(viscosity)


class RotLocalDampingPrms(LocalDampingPrms):  # InteractionParamsPy.cpp:1050-1065 ("RotLocalDamping")
    pass


class GravityPrms:  # InteractionParamsPy.cpp:922, 2375-2398
    def __init__(self, name, acceleration):
        self.name, self.acceleration = name, Vec3(*acceleration)


class Runnable:
    """Pre/post time-step hook (LsmMpiPy.cpp:1051-1059): subclasses implement run()."""

    def __init__(self):
        pass

    def run(self):
        raise NotImplementedError


class ConnectionFinder:
    """Bonds between particles whose gap is at most maxDist (Geometry/DistConnections.hpp);
    iterable of (tag, id1, id2) like the reference's connection iterable."""

    def __init__(self, maxDist, bondTag, pList):
        plist = list(pList)
        pos = np.array([list(p.getPosn()) for p in plist], dtype=np.float64)
        rad = np.array([p.getRadius() for p in plist], dtype=np.float64)
        ids = np.array([p.getId() for p in plist], dtype=np.int64)
        self._conn = []
        if len(plist) < 2:
            return
        cell = 2.0 * rad.max() + maxDist
        key = np.floor((pos - pos.min(0)) / cell).astype(np.int64)
        buckets = {}
        for i, k in enumerate(map(tuple, key)):
            buckets.setdefault(k, []).append(i)
        for k, members in buckets.items():
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        other = buckets.get((k[0] + dx, k[1] + dy, k[2] + dz))
                        if not other:
                            continue
                        for i in members:
                            for j in other:
                                if ids[j] <= ids[i]:
                                    continue
                                d = np.linalg.norm(pos[i] - pos[j]) - rad[i] - rad[j]
                                if d <= maxDist:
                                    self._conn.append((int(bondTag), int(ids[i]), int(ids[j])))

    def __iter__(self):
        return iter(self._conn)

    def __len__(self):
        return len(self._conn)


# ---- the simulation object (LsmMpiPy.cpp) ----------------------------------------------------
class LsmMpi:
    """One B200 worker behind the LsmMpi interface."""

    def __init__(self, numWorkerProcesses=1, mpiDimList=(1, 1, 1), _backend=None):
        self._backend = _backend or _capi.DemSim
        self._ptype = None
        self._grid = self._skin = None
        self._dt = 1e-3
        self._nsteps = 0
        self._sim = None
        self._pre, self._post = [], []
        self._savers, self._saved0 = [], False
        self._pending = []  # particles created before setSpatialDomain
        self._walls = {}
        self._wig_of_wall = {}
        self._bonded, self._dynamic = set(), set()  # group names, for createExclusion
        self._bbox, self._circ = None, (False, False, False)

    # -- set-up (LsmMpiPy.cpp:2187-2300) --
    def initNeighbourSearch(self, particleType, gridSpacing, verletDist):
        if particleType not in ("NRotSphere", "RotSphere"):
            raise NotImplementedError(f"particle type {particleType!r} is not on the GPU path")
        self._ptype, self._grid, self._skin = particleType, float(gridSpacing), float(verletDist)

    initNeighborSearch = initNeighbourSearch
    initVerletModel = initNeighbourSearch

    def getParticleType(self):
        return self._ptype

    def setTimeStepSize(self, dt):
        self._dt = float(dt)
        if self._sim is not None:
            self._sim.set_timestep(self._dt)

    def getTimeStepSize(self):
        return self._dt

    def setNumTimeSteps(self, n):
        self._nsteps = int(n)

    def getNumTimeSteps(self):
        return self._nsteps

    def getTimeStep(self):
        return self._sim.timestep if self._sim is not None else 0

    def setSpatialDomain(self, bBox, circDimList=(False, False, False)):
        if self._ptype is None:
            raise RuntimeError("call initNeighbourSearch before setSpatialDomain")
        if any(circDimList[1:]):
            raise NotImplementedError("periodic y or z is not on the GPU path (x only)")
        mn, mx = bBox.getMinPt(), bBox.getMaxPt()
        self._bbox, self._circ = (list(mn), list(mx)), tuple(bool(c) for c in circDimList)
        self._sim = self._backend(self._ptype, self._grid, self._skin, list(mn), list(mx),
                                 (1 if circDimList[0] else 0, 0, 0), self._dt)
        if self._pending:
            self.createParticles(self._pending)
            self._pending = []

    def _require(self):
        if self._sim is None:
            raise RuntimeError("setSpatialDomain has not been called")
        return self._sim

    def createParticle(self, p):
        self.createParticles([p])

    def createParticles(self, particles):
        plist = list(particles)
        if self._sim is None:
            self._pending.extend(plist)
            return
        if not plist:
            return
        ids = np.array([p.getId() for p in plist], np.int32)
        tags = np.array([p.getTag() for p in plist], np.int32)
        pos = np.array([list(p.getPosn()) for p in plist], np.float64)
        rad = np.array([p.getRadius() for p in plist], np.float64)
        mass = np.array([p.getMass() for p in plist], np.float64)
        vel = np.array([list(p.getLinearVelocity()) for p in plist], np.float64)
        angvel = np.array([list(getattr(p, "_angvel", Vec3())) for p in plist], np.float64)
        self._sim.add_particles(ids, pos, rad, mass, tag=tags, vel=vel, angvel=angvel)

    def createConnections(self, connections):
        c = [(x.getTag(), x.getP1Id(), x.getP2Id()) if hasattr(x, "getTag") else tuple(x) for x in connections]
        if c:
            a = np.array(c, np.int64)
            self._require().add_connections(a[:, 0], a[:, 1], a[:, 2])

    def createWall(self, name, posn, normal):
        self._require().add_wall(name, list(posn), list(normal))
        self._walls[name] = True

    def createInteractionGroup(self, prms):
        s = self._require()
        if isinstance(prms, NRotElasticPrms):
            s.add_elastic_group(prms.name, prms.normalK, prms.scaling)
            self._dynamic.add(prms.name)
        elif isinstance(prms, RotFrictionPrms):
            if prms.rigid:
                raise NotImplementedError("RotFrictionPrms(rigid=True) is not on the GPU path")
            s.add_rot_friction_group(prms.name, prms.normalK, prms.staticMu, prms.dynamicMu, prms.shearK, self._dt,
                                     prms.scaling, prms.meanR_scaling)
            self._dynamic.add(prms.name)
        elif isinstance(prms, RotBondPrms):
            s.add_rot_bond_group(prms.name, prms.tag, prms.normalK, prms.shearK, prms.torsionK, prms.bendingK,
                                 prms.normalBrkForce, prms.shearBrkForce, prms.torsionBrkForce, prms.bendingBrkForce,
                                 prms.scaling, prms.meanR_scaling, prms.truncated)
            self._bonded.add(prms.name)
        elif isinstance(prms, NRotFrictionPrms):  # LsmMpiPy::createNRotFrictionInteractGrp sets dt
            s.add_nrot_friction_group(prms.name, prms.normalK, prms.dynamicMu, prms.shearK, self._dt, prms.scaling)
            self._dynamic.add(prms.name)
        elif isinstance(prms, HertzMindlinPrms):  # LsmMpiPy::createHertzMindlinIG sets dt (LsmMpiPy.cpp:508-517)
            s.add_hertz_mindlin_group(prms.name, prms.youngsModulus, prms.poissonsRatio, prms.dynamicMu, self._dt)
            self._dynamic.add(prms.name)
        elif isinstance(prms, BrittleBeamDZCPrms):  # LsmMpiPy::createBrittleBeamDZCInteractGrp
            s.add_brittle_beam_dzc_group(prms.name, prms.tag, prms.kr, prms.ks, prms.kt, prms.kb, prms.cohesion,
                                         prms.tensileCutoff, prms.compressCutoff, prms.frictionAngle, prms.beta1,
                                         prms.beta2)
            self._bonded.add(prms.name)
        elif isinstance(prms, BrittleBeamSCPrms):  # LsmMpiPy::createBrittleBeamSCInteractGrp
            s.add_brittle_beam_sc_group(prms.name, prms.tag, prms.kr, prms.ks, prms.kt, prms.kb, prms.cohesion,
                                        prms.tensileCutoff, prms.frictionAngle)
            self._bonded.add(prms.name)
        elif isinstance(prms, HertzMindlinViscoPrms):  # LsmMpiPy::createHertzMindlinViscoIG sets dt
            s.add_hertz_mindlin_visco_group(prms.name, prms.youngsModulus, prms.poissonsRatio, prms.dynamicMu,
                                            prms.restitution, self._dt)
            self._dynamic.add(prms.name)
        elif isinstance(prms, NRotBondPrms):
            s.add_nrot_bond_group(prms.name, prms.tag, prms.normalK, prms.breakDistance, prms.scaling)
            self._bonded.add(prms.name)
        elif isinstance(prms, NRotElasticWallPrms):
            s.add_wall_group(prms.name, prms.wallName, prms.normalK)
            self._wig_of_wall[prms.name] = prms.wallName
        elif isinstance(prms, RotLocalDampingPrms):
            s.add_local_damping(prms.name, 1, prms.viscosity)
        elif isinstance(prms, LocalDampingPrms):
            s.add_local_damping(prms.name, 0, prms.viscosity)
        elif isinstance(prms, RotDampingPrms):
            s.add_damping(1, prms.viscosity, prms.maxIterations)
        elif isinstance(prms, LinDampingPrms):
            s.add_damping(0, prms.viscosity, prms.maxIterations)
        elif isinstance(prms, GravityPrms):
            s.add_gravity(prms.name, list(prms.acceleration))
        else:
            raise NotImplementedError(f"{type(prms).__name__} is not on the GPU path")
        return prms.name

    # LsmMpiPy::createDamping / createLocalDamping / createRotLocalDamping / createGravity
    # (LsmMpiPy.cpp:706-737): the older spellings of createInteractionGroup for these groups
    def createDamping(self, prms):
        return self.createInteractionGroup(prms)

    createLocalDamping = createRotLocalDamping = createGravity = createDamping

    def createExclusion(self, interactionName1, interactionName2):
        """TSubLattice::setExIG (SubLattice.hpp:1980-2009): a name that names no group is
        reported on the error console and the run goes on without the exclusion."""
        s = self._require()
        if interactionName1 not in self._bonded or interactionName2 not in self._dynamic:
            print("TSubLattice<T>::setExIG() - nonexisting interaction group", file=sys.stderr)
            return
        s.add_exclusion(interactionName1, interactionName2)

    # -- walls and particles during the run --
    # A wall (or wall group) name that names nothing is ignored by the workers, and its
    # position and force read as zero (TSubLattice::moveWallBy, getWallPos, getWallForce,
    # applyForceToWall: SubLattice.hpp:2878-2891, 835-860, 897-921, 2935-2948).
    def moveWallBy(self, name, move):
        if name in self._walls:
            self._require().move_wall(name, list(move))

    def getWallPosition(self, name):
        if name not in self._walls:
            return Vec3(0.0, 0.0, 0.0)
        return Vec3(*self._require().wall(name)[0])

    def getWallForce(self, name):
        if name not in self._walls:
            return Vec3(0.0, 0.0, 0.0)
        return Vec3(*self._require().wall(name)[1])

    def applyForceToWall(self, interactionName, force):
        if interactionName in self._wig_of_wall:
            self._require().apply_force_to_wall(interactionName, list(force))

    def moveTaggedParticlesBy(self, tag, displacement):
        self._require().move_tagged(int(tag), list(displacement))

    def getNumParticles(self):
        return self._require().num_particles()

    def getParticleList(self):
        p = self._require().particles()
        cls = RotSphere if self._ptype == "RotSphere" else NRotSphere
        out = []
        for k in range(len(p["id"])):
            q = cls(int(p["id"][k]), Vec3(*p["pos"][k]), 0.0, 0.0)
            q.setLinearVelocity(Vec3(*p["vel"][k]))
            if cls is RotSphere:
                q.setAngularVelocity(Vec3(*p["angvel"][k]))
            out.append(q)
        return out

    # -- runnables and stepping (LsmMpiPy.cpp:1051-1069; LatticeMaster.cpp:2602-2740) --
    def addPreTimeStepRunnable(self, r):
        self._pre.append(r)

    def addPostTimeStepRunnable(self, r):
        self._post.append(r)

    # -- field savers (LsmMpiPy.cpp:2160-2175, 3272-3297; saved in runOneStep after the step,
    #    LatticeMaster.cpp:2612-2700) --
    def createFieldSaver(self, prms):
        self._savers.append(FieldSaver(prms))

    # -- checkpoints (LsmMpiPy.cpp:847-884, 2807-2840; CheckPointController) --
    def createRestartCheckPointer(self, prms):
        self._savers.append(CheckPointer(self, prms, restart=True))

    # the reference gathers the workers' data through the master; with one worker the files are the same
    createCheckPointerWriteThroughMaster = createRestartCheckPointer

    def createCheckPointer(self, prms):
        """Snapshots for visualisation / post-processing (LsmMpiPy::createSnapShots)."""
        self._savers.append(CheckPointer(self, prms, restart=False))

    def loadCheckPoint(self, fileName):
        """CLatticeMaster::loadCheckPointData (Parallel/LatticeMaster.cpp:780-820): the info file's
        geometry (if no spatial domain was set), the step counter, and the worker file into this
        particle-less worker, whose interaction groups the script has created."""
        info = read_info(fileName)
        if self._sim is None:
            self.setSpatialDomain(BoundingBox(Vec3(*info["bbox_min"]), Vec3(*info["bbox_max"])), info["periodic"])
        wf = worker_file(fileName, info)
        self._sim.load_checkpoint(wf, info["t"])
        for name in walls_in(wf):
            self._walls[name] = True
        self._saved0 = True  # the initial-state savers ran in the original run

    def _save_fields(self, t):
        for f in self._savers:
            if f.need_save(t):
                f.save(self._sim)

    def runTimeStep(self):
        s = self._require()
        if s.timestep == 0 and not self._saved0:
            self._save_fields(0)
            self._saved0 = True
        for r in self._pre:
            r.run()
        s.step(1)
        self._save_fields(s.timestep)
        for r in self._post:
            r.run()

    def run(self):
        s = self._require()
        if self._pre or self._post:
            while s.timestep < self._nsteps:
                self.runTimeStep()
            return
        if s.timestep == 0 and not self._saved0:
            self._save_fields(0)
            self._saved0 = True
        while s.timestep < self._nsteps:  # step in stretches up to the next save
            nxt = [f.next_save(s.timestep) for f in self._savers]
            nxt = [x for x in nxt if x is not None]
            stop = min([self._nsteps] + nxt)
            s.step(stop - s.timestep)
            self._save_fields(s.timestep)

    def exit(self):
        if self._sim is not None:
            self._sim.close()
            self._sim = None

    def setVerbosity(self, *a, **k):
        pass

    setVerbosityLevel = setVerbosity

    def force2dComputations(self, do2d=True):
        if do2d:
            raise NotImplementedError("2-D computations are not on the GPU path")

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        raise NotImplementedError(f"LsmMpi.{name} is outside the GPU hot path")
