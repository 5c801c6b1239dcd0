"""Seeded synthetic scenarios shared by the parity tests.

Each builder takes a ``make(particle_type, grid_spacing, verlet_dist, bbox_min,
bbox_max, circ, dt)`` factory and returns the simulation it set up, so the same
scenario drives the CUDA path and the CPU oracles through identical calls.
Particle masses follow CParticle::setDensity with rho = 1 and pi = 3.141592654
(Model/Particle.cpp:108-122).
"""
from __future__ import annotations

import numpy as np

PI_REF = 3.141592654


def sphere_mass(r, rho=1.0):
    r = np.asarray(r, dtype=np.float64)
    return (4.0 / 3.0) * rho * PI_REF * r * r * r


def gravity_box(make, n_side=6, seed=1, steps_dt=1e-4, layers=None, gap=1.0):
    """Small form of the NRotSphere gravity packing: jittered cubic lattice,
    NRotElastic k=1000, gravity -9.81 z, linear damping 0.01, six elastic walls."""
    rng = np.random.default_rng(seed)
    layers = layers or n_side
    L = n_side * gap
    H = 2 * layers * gap
    g = np.stack(np.meshgrid(np.arange(n_side), np.arange(n_side), np.arange(layers), indexing="ij"), -1).reshape(-1, 3)
    pos = (g + 0.5) * gap + rng.uniform(-0.05, 0.05, size=g.shape)
    rad = rng.uniform(0.4, 0.5, size=len(g))
    n = len(g)
    sim = make("NRotSphere", 1.2, 0.2, (0, 0, 0), (L, L, H), (0, 0, 0), steps_dt)
    sim.add_particles(np.arange(n), pos, rad, sphere_mass(rad), tag=np.zeros(n, np.int32))
    sim.add_elastic_group("elastic", 1000.0, True)
    sim.add_gravity("gravity", (0, 0, -9.81))
    sim.add_damping(0, 0.01, 100)
    for name, o, nrm in (("xlo", (0, 0, 0), (1, 0, 0)), ("xhi", (L, 0, 0), (-1, 0, 0)),
                         ("ylo", (0, 0, 0), (0, 1, 0)), ("yhi", (0, L, 0), (0, -1, 0)),
                         ("zlo", (0, 0, 0), (0, 0, 1)), ("zhi", (0, 0, H), (0, 0, -1))):
        sim.add_wall(name, o, nrm)
        sim.add_wall_group(name + "_w", name, 1000.0)
    return sim


def nrot_friction_pack(make, rot=False, n_side=5, seed=8, dt=1e-4, vscale=0.5):
    """Jittered lattice of spheres in contact under gravity with an NRotFriction group
    (CFrictionInteraction: k = ks = 1000, mu = 0.6), linear damping, floor and side walls; random
    initial velocities so that contacts slide.  NRotSphere, or RotSphere (forces only, as the
    reference's applyForce gives no moments)."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(n_side), np.arange(n_side), np.arange(n_side), indexing="ij"), -1).reshape(-1, 3)
    pos = (g + 0.5) * 0.95 + rng.uniform(-0.03, 0.03, size=g.shape)
    rad = rng.uniform(0.46, 0.5, size=len(g))
    n = len(g)
    L = n_side * 0.95
    sim = make("RotSphere" if rot else "NRotSphere", 1.2, 0.2, (0, 0, 0), (L, L, 2 * L), (0, 0, 0), dt)
    vel = rng.normal(0, vscale, size=(n, 3))
    sim.add_particles(np.arange(n), pos, rad, sphere_mass(rad), tag=np.zeros(n, np.int32), vel=vel)
    sim.add_nrot_friction_group("friction", 1000.0, 0.6, 1000.0, dt, True)
    sim.add_gravity("gravity", (0, 0, -9.81))
    sim.add_damping(0, 0.01, 100)
    for name, o, nrm in (("xlo", (0, 0, 0), (1, 0, 0)), ("xhi", (L, 0, 0), (-1, 0, 0)),
                         ("zlo", (0, 0, 0), (0, 0, 1))):
        sim.add_wall(name, o, nrm)
        sim.add_wall_group(name + "_w", name, 1000.0)
    return sim


def hertz_mindlin_pack(make, rot=False, n_side=5, seed=10, dt=1e-4, vscale=1.0, skin=0.05, restitution=None):
    """nrot_friction_pack's lattice with a HertzMindlin group (CHertzMindlinInteraction,
    E = 1e4, nu = 0.3, mu = 0.5) and a small Verlet skin, so that neighbour rebuilds (which
    restart the law's tangential history, its storage being PIS_NE) fall inside a short run."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(n_side), np.arange(n_side), np.arange(n_side), indexing="ij"), -1).reshape(-1, 3)
    pos = (g + 0.5) * 0.95 + rng.uniform(-0.03, 0.03, size=g.shape)
    rad = rng.uniform(0.46, 0.5, size=len(g))
    n = len(g)
    L = n_side * 0.95
    sim = make("RotSphere" if rot else "NRotSphere", 1.2, skin, (0, 0, 0), (L, L, 2 * L), (0, 0, 0), dt)
    vel = rng.normal(0, vscale, size=(n, 3))
    sim.add_particles(np.arange(n), pos, rad, sphere_mass(rad), tag=np.zeros(n, np.int32), vel=vel)
    if restitution is None:
        sim.add_hertz_mindlin_group("hm", 1e4, 0.3, 0.5, dt)
    else:  # HertzMindlinVisco (CHertzMindlinViscoInteraction) with this restitution coefficient
        sim.add_hertz_mindlin_visco_group("hm", 1e4, 0.3, 0.5, restitution, dt)
    sim.add_gravity("gravity", (0, 0, -9.81))
    sim.add_damping(0, 0.01, 100)
    for name, o, nrm in (("xlo", (0, 0, 0), (1, 0, 0)), ("xhi", (L, 0, 0), (-1, 0, 0)),
                         ("zlo", (0, 0, 0), (0, 0, 1))):
        sim.add_wall(name, o, nrm)
        sim.add_wall_group(name + "_w", name, 1000.0)
    return sim


def nrot_bonded_block(make, nx=5, ny=6, nz=5, seed=9, dt=1e-4, k=1e4, rbreak=0.02, load_rate=0.01):
    """NRotSphere block with NRotBond (CBondedInteraction) between lattice neighbours (gap within
    0.015), failing on extension beyond r0 * rbreak, and an NRotFriction group for the contacts
    after failure (excluded while the bond holds); platens at y, closed by run_loaded."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    pos = (g + 0.5) * 1.0 + rng.uniform(-0.01, 0.01, size=g.shape)
    n = len(g)
    rad = np.full(n, 0.495)
    d = np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=-1)
    np.fill_diagonal(d, np.inf)
    i1, i2 = np.nonzero(np.triu(d - 2 * 0.495 <= 0.015, 1))
    vel = rng.normal(0, 0.05, size=(n, 3))
    Ly = ny * 1.0
    sim = make("NRotSphere", 1.25, 0.2, (0, 0, 0), (nx * 1.0, Ly, nz * 1.0), (0, 0, 0), dt)
    sim.add_particles(np.arange(n), pos, rad, sphere_mass(rad), tag=np.zeros(n, np.int32), vel=vel)
    sim.add_connections(np.ones(len(i1), np.int32), i1, i2)
    sim.add_nrot_bond_group("bonds", 1, k, rbreak, True)
    sim.add_nrot_friction_group("friction", k, 0.6, k, dt, True)
    sim.add_exclusion("bonds", "friction")
    sim.add_wall("bottom", (0, 0, 0), (0, 1, 0))
    sim.add_wall("top", (0, Ly, 0), (0, -1, 0))
    sim.add_wall_group("bottom_w", "bottom", k)
    sim.add_wall_group("top_w", "top", k)
    sim.add_damping(0, 0.05, 100)
    sim._load_rate = load_rate
    return sim


def nrot_bonded_block_script(make, nx=5, ny=6, nz=5, dt=1e-4, k=1e4, rbreak=0.02, load_rate=0.01):
    """The restart script of nrot_bonded_block: its groups, walls and damping, no particles."""
    Ly = ny * 1.0
    sim = make("NRotSphere", 1.25, 0.2, (0, 0, 0), (nx * 1.0, Ly, nz * 1.0), (0, 0, 0), dt)
    sim.add_nrot_bond_group("bonds", 1, k, rbreak, True)
    sim.add_nrot_friction_group("friction", k, 0.6, k, dt, True)
    sim.add_exclusion("bonds", "friction")
    sim.add_wall("bottom", (0, 0, 0), (0, 1, 0))
    sim.add_wall("top", (0, Ly, 0), (0, -1, 0))
    sim.add_wall_group("bottom_w", "bottom", k)
    sim.add_wall_group("top_w", "top", k)
    sim.add_damping(0, 0.05, 100)
    sim._load_rate = load_rate
    return sim


def friction_pack(make, nx=6, ny=5, nz=6, seed=2, periodic=False, dt=5e-5, vscale=0.5, squeeze=0.93):
    """Small rotational frictional pack: slightly overlapping jittered lattice of
    RotSpheres (lognormal radii), RotFriction kn=ks=1e4 mu=0.6, elastic floor and
    roof, random initial linear and angular velocities, linear + rotational damping."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    spacing = 1.0 * squeeze
    pos = (g + 0.5) * spacing + rng.uniform(-0.03, 0.03, size=g.shape)
    rad = np.clip(np.exp(np.log(0.5) + 0.25 * rng.standard_normal(len(g))) * 0.5 + 0.25, 0.3, 0.5)
    n = len(g)
    Lx, Ly, Lz = nx * spacing, ny * spacing + 0.2, nz * spacing
    sim = make("RotSphere", 1.2, 0.2, (0, -0.1, 0), (Lx, Ly - 0.1, Lz), (1 if periodic else 0, 0, 0), dt)
    vel = rng.normal(0, vscale, size=(n, 3))
    angvel = rng.normal(0, vscale, size=(n, 3))
    sim.add_particles(np.arange(n)[::-1].copy(), pos, rad, sphere_mass(rad), tag=np.zeros(n, np.int32), vel=vel,
                      angvel=angvel)
    sim.add_rot_friction_group("friction", 1e4, 0.6, 0.6, 1e4, dt, True, True)
    sim.add_wall("floor", (0, -0.1, 0), (0, 1, 0))
    sim.add_wall("roof", (0, Ly - 0.1, 0), (0, -1, 0))
    sim.add_wall_group("floor_w", "floor", 1e4)
    sim.add_wall_group("roof_w", "roof", 1e4)
    sim.add_damping(0, 0.002, 50)
    sim.add_damping(1, 0.002, 50)
    return sim


def bonded_block(make, nx=5, ny=6, nz=5, seed=3, dt=1e-5, strength=(0.5, 1.0, 1.0, 0.5), load_rate=0.02,
                 with_friction=True, bonds=True):
    """Small bonded block: jittered cubic RotSpheres, every pair within gap 1e-3
    of touching bonded (cf. Geometry/DistConnections), RotBond with brittle
    failure, RotFriction + exclusion for post-break contacts, platens at y."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    pos = (g + 0.5) * 1.0 + rng.uniform(-0.02, 0.02, size=g.shape)
    n = len(g)
    rad = np.full(n, 0.5)
    # radii chosen so that lattice neighbours touch: r_i = min over neighbours of half distance
    d = np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=-1)
    np.fill_diagonal(d, np.inf)
    rad = np.clip(0.5 * d.min(axis=1), 0.3, 0.5)
    gap = d - (rad[:, None] + rad[None, :])
    i1, i2 = np.nonzero(np.triu(gap <= 1e-3, 1))
    Ly = ny * 1.0
    sim = make("RotSphere", 1.25, 0.2, (0, 0, 0), (nx * 1.0, Ly, nz * 1.0), (0, 0, 0), dt)
    sim.add_particles(np.arange(n), pos, rad, sphere_mass(rad), tag=np.zeros(n, np.int32))
    sim.add_connections(np.ones(len(i1), np.int32), i1, i2)
    mn, ms, mt, mb = strength
    if bonds:
        sim.add_rot_bond_group("bonds", 1, 1e5, 1e5, 1e3, 1e3, mn, ms, mt, mb, True, True, 1.0)
    if with_friction:
        sim.add_rot_friction_group("friction", 1e5, 0.6, 0.6, 1e5, dt, True, True)
        sim.add_exclusion("bonds", "friction")
    sim.add_wall("bottom", (0, 0, 0), (0, 1, 0))
    sim.add_wall("top", (0, Ly, 0), (0, -1, 0))
    sim.add_wall_group("bottom_w", "bottom", 1e5)
    sim.add_wall_group("top_w", "top", 1e5)
    sim.add_damping(0, 0.01, 50)
    sim.add_damping(1, 0.01, 50)
    sim._load_rate = load_rate
    return sim


def dzc_block(make, nx=5, ny=6, nz=5, seed=3, dt=1e-5, crit=(3.0, 5.0, 20.0, 30.0, 1.0, 1.0), load_rate=0.02):
    """bonded_block's specimen with BrittleBeamDZC bonds (BrittleBeamDZCInteraction: RotBond forces,
    a cut-off Mohr-Coulomb failure of the beam's normal and shear stress) instead of RotBond.
    crit = (cohesion, tCutoff, cCutoff, fAngle in degrees, beta1, beta2)."""
    sim = bonded_block(make, nx, ny, nz, seed, dt, load_rate=load_rate, with_friction=False, bonds=False)
    coh, tcut, ccut, fang, b1, b2 = crit
    sim.add_brittle_beam_dzc_group("bonds", 1, 1e5, 1e5, 1e3, 1e3, coh, tcut, ccut, fang, b1, b2)
    sim.add_rot_friction_group("friction", 1e5, 0.6, 0.6, 1e5, dt, True, True)
    sim.add_exclusion("bonds", "friction")
    return sim


def sc_block(make, nx=5, ny=6, nz=5, seed=3, dt=1e-5, crit=(50.0, 50.0, 30.0), load_rate=0.02):
    """bonded_block's specimen with BrittleBeamSC bonds (BrittleBeamSCInteraction: RotBond forces, a
    truncated Mohr-Coulomb failure of the particles' mean stress across the bond) instead of RotBond.
    crit = (cohesion, tCutoff, fAngle in degrees)."""
    sim = bonded_block(make, nx, ny, nz, seed, dt, load_rate=load_rate, with_friction=False, bonds=False)
    coh, tcut, fang = crit
    sim.add_brittle_beam_sc_group("bonds", 1, 1e5, 1e5, 1e3, 1e3, coh, tcut, fang)
    sim.add_rot_friction_group("friction", 1e5, 0.6, 0.6, 1e5, dt, True, True)
    sim.add_exclusion("bonds", "friction")
    return sim


def bonded_block_script(make, nx=5, ny=6, nz=5, dt=1e-5, strength=(0.5, 1.0, 1.0, 0.5), with_friction=True):
    """The restart script of bonded_block: the same domain, groups, walls and damping, and no
    particles or connections (they come from the checkpoint, as with LsmMpi.loadCheckPoint)."""
    Ly = ny * 1.0
    sim = make("RotSphere", 1.25, 0.2, (0, 0, 0), (nx * 1.0, Ly, nz * 1.0), (0, 0, 0), dt)
    mn, ms, mt, mb = strength
    sim.add_rot_bond_group("bonds", 1, 1e5, 1e5, 1e3, 1e3, mn, ms, mt, mb, True, True, 1.0)
    if with_friction:
        sim.add_rot_friction_group("friction", 1e5, 0.6, 0.6, 1e5, dt, True, True)
        sim.add_exclusion("bonds", "friction")
    sim.add_wall("bottom", (0, 0, 0), (0, 1, 0))
    sim.add_wall("top", (0, Ly, 0), (0, -1, 0))
    sim.add_wall_group("bottom_w", "bottom", 1e5)
    sim.add_wall_group("top_w", "top", 1e5)
    sim.add_damping(0, 0.01, 50)
    sim.add_damping(1, 0.01, 50)
    return sim


def parse_checkpoint(path):
    """Restart-checkpoint worker file -> dict: particles {id: fields}, bonds {(id1, id2): fields},
    friction {(id1, id2): fields}, walls {name: 9 values}.  Reads this library's files and the
    reference's (whose RotFriction record count runs into the first record's first field)."""
    lines = open(path).read().split("\n")
    pos = [0]

    def nxt(blank_ok=False):
        while pos[0] < len(lines):
            ln = lines[pos[0]].split()
            pos[0] += 1
            if ln or blank_ok:
                return ln
        raise ValueError("unexpected end of checkpoint")

    out = {"base": nxt() + nxt(), "particles": {}, "bonds": {}, "friction": {}, "walls": {}}
    for _ in range(int(nxt()[0])):
        t = nxt()
        out["particles"][int(t[4])] = [float(x) for x in t]
    for _ in range(int(nxt()[0])):
        typ = nxt()[0]
        assert typ in ("RotBonded", "Bonded"), typ
        ids = (0, 1) if typ == "RotBonded" else (5, 6)   # RotBonded: id1 id2 first; Bonded: after 5 values
        for _ in range(int(nxt()[0])):
            t = nxt()
            out["bonds"][(int(t[ids[0]]), int(t[ids[1]]))] = [float(x) for x in t]
    for _ in range(int(nxt()[0])):
        typ = nxt()[0]
        assert typ in ("RotFriction", "Friction"), typ
        ids = (8, 9) if typ == "RotFriction" else (6, 7)
        t = nxt()
        recs = []
        if len(t) == 1:
            recs = [nxt() for _ in range(int(t[0]))]
        else:
            while t:
                recs.append(t)
                t = nxt(blank_ok=True)
        for r in recs:
            out["friction"][(int(r[ids[0]]), int(r[ids[1]]))] = [float(x) for x in r[1:]]
    t = nxt()
    assert t[0] == "Walls"
    for _ in range(int(t[1])):
        name = nxt()[0]
        out["walls"][name] = [float(x) for x in nxt()]
    return out


def run_loaded(sim, steps, rate):
    """Advance with a platen loader: both platens move toward each other by
    ``rate`` per step (a pre-step runnable like WallLoaderRunnable)."""
    for _ in range(steps):
        sim.move_wall("top", (0, -rate, 0))
        sim.move_wall("bottom", (0, rate, 0))
        sim.step(1)


def loaded_friction_pack(make, **kw):
    """friction_pack with its floor and roof moved onto the pack (up to ~0.09 overlap), so
    that the wall reactions of a short window are carried by the frictional contacts."""
    sim = friction_pack(make, vscale=0.2, **kw)
    sim.move_wall("floor", (0, 0.12, 0))
    sim.move_wall("roof", (0, -0.12, 0))
    return sim


WINDOW_SEEDS = ("param:bonds:normalK", "param:bonds:shearK", "param:bonds:torsionK", "param:bonds:bendingK",
                "param:Damping:viscosity", "param:RotDamping:viscosity")
WINDOW_PARAMS = (("bonds", "normalK"), ("bonds", "shearK"), ("bonds", "torsionK"), ("bonds", "bendingK"),
                 ("Damping", "viscosity"), ("RotDamping", "viscosity"))


def mse_target(R, seed=7):
    """A seeded target curve for the platen-force MSE: the window's own
    reactions smoothed and scaled by a seeded factor per wall."""
    rng = np.random.default_rng(seed)
    k = np.ones(9) / 9.0
    sm = np.empty_like(R)
    for g in range(R.shape[1]):
        for c in range(3):
            sm[:, g, c] = np.convolve(R[:, g, c], k, mode="same")
    return sm * rng.uniform(0.8, 1.2, size=(1, R.shape[1], 1))


def mse(R, tgt):
    return float(((R - tgt) ** 2).mean())


def mse_grad(R, tgt):
    return 2.0 * (R - tgt) / R.size


def window_block(make, nx=4, ny=5, nz=4, seed=4, dt=1e-4, kr=1e5, ks=1e5, kt=1e5, kb=1e5, visc=1.0, vscale=1.0,
                 platen_speed=0.5, friction=False, vel=None, angvel=None, tilt=(0.5, 0.3), strength=1e6):
    """Bonded block for the differentiable window: a cubic lattice of RotSpheres
    (r ~ U[0.49, 0.5]) with every lattice neighbour bonded, strengths far above
    the loads (elastic regime, no breaks), platens that
    start just touching the block and move inward at ``platen_speed`` (so the
    reactions are carried by the bonds), seeded initial linear and angular
    velocities (``vel`` / ``angvel`` override them, rows by id) and the
    stiffness / damping parameters as arguments.  A ``strength`` (all four
    bond strengths) near the loads makes bonds fail inside the window.  The defaults give every
    parameter a loss sensitivity well above the FP64 rounding noise of a
    200-step window, so that central differences at h = 1e-6 relative resolve
    the gradient (torsion / bending stiffness as large as the normal one, and a
    damping viscosity that changes the reactions by percents).  The lattice is tilted by
    ``tilt`` (radians about x, then y) so that no bond lies near the z axis,
    where the RotBond law's frame quaternion (ARotBondedInteraction.cpp:349-364)
    takes square roots of cancelling differences and its derivatives are
    ill-conditioned in any arithmetic."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    pos = (g + 0.5) * 1.0
    ax, ay = tilt
    rx = np.array([[1, 0, 0], [0, np.cos(ax), -np.sin(ax)], [0, np.sin(ax), np.cos(ax)]])
    ry = np.array([[np.cos(ay), 0, np.sin(ay)], [0, 1, 0], [-np.sin(ay), 0, np.cos(ay)]])
    c = pos.mean(axis=0)
    pos = (pos - c) @ (ry @ rx).T
    pos = pos - pos.min(axis=0) + 1.0
    n = len(g)
    rad = rng.uniform(0.49, 0.5, size=n)
    d = np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=-1)
    np.fill_diagonal(d, np.inf)
    gap = d - (rad[:, None] + rad[None, :])
    i1, i2 = np.nonzero(np.triu(gap <= 0.021, 1))   # every lattice neighbour: a connected solid
    v0 = rng.normal(0, vscale, size=(n, 3)) if vel is None else np.asarray(vel, dtype=np.float64)
    w0 = rng.normal(0, vscale, size=(n, 3)) if angvel is None else np.asarray(angvel, dtype=np.float64)
    top = pos.max(axis=0) + 1.0
    sim = make("RotSphere", 1.25, 0.2, (0, 0, 0), tuple(float(x) for x in top), (0, 0, 0), dt)
    sim.add_particles(np.arange(n), pos, rad, sphere_mass(rad), tag=np.zeros(n, np.int32), vel=v0, angvel=w0)
    sim.add_connections(np.ones(len(i1), np.int32), i1, i2)
    sim.add_rot_bond_group("bonds", 1, kr, ks, kt, kb, strength, strength, strength, strength, True, True, 1.0)
    if friction:
        sim.add_rot_friction_group("friction", 1e5, 0.6, 0.6, 1e5, dt, True, True)
        sim.add_exclusion("bonds", "friction")
    sim.add_wall("bottom", (0, float((pos[:, 1] - rad).min()), 0), (0, 1, 0))
    sim.add_wall("top", (0, float((pos[:, 1] + rad).max()), 0), (0, -1, 0))
    sim.add_wall_group("bottom_w", "bottom", 1e5)
    sim.add_wall_group("top_w", "top", 1e5)
    sim.add_damping(0, visc, 50)
    sim.add_damping(1, visc, 50)
    sim.set_wall_velocity("bottom", (0, platen_speed, 0))
    sim.set_wall_velocity("top", (0, -platen_speed, 0))
    return sim


def wall_force_history(sim, nsteps, groups=("bottom_w", "top_w"), walls=("bottom", "top")):
    """Step one at a time and collect each wall's reaction after every step."""
    out = np.zeros((nsteps, len(walls), 3))
    for t in range(nsteps):
        sim.step(1)
        for k, w in enumerate(walls):
            out[t, k] = sim.wall(w)[1]
    return out


def shear_cell(make, n=250_000, periodic=True, seed=2, moving_walls=False):
    """The headline shear cell: n RotSpheres with lognormal radii (median 0.5, sigma 0.25, in
    [0.2, 1.0]) packed by the seeded RSI packer into 100 x 50 x 100 (periodic in x), RotFriction
    kn = ks = 1e4, mu = 0.6, elastic walls (k = 1e4) at y = 0 and y = 50, dt = 5e-5, seeded
    N(0, 0.1) velocities and spins.  Walls static unless moving_walls (then the caller moves
    them); gridSpacing 2.2, verletDist 0.2."""
    from esys.lsm import geometry as G

    pos, rad = G.rsi_pack(n, (0, 0, 0), (100, 50, 100), seed=seed, periodic_x=True, lognormal=(0.5, 0.25),
                          rmin=0.2, rmax=1.0, max_attempts=5000)
    assert len(rad) == n
    rng = np.random.default_rng(seed + 100)
    vel = rng.normal(0.0, 0.1, size=(n, 3))
    angvel = rng.normal(0.0, 0.1, size=(n, 3))
    sim = make("RotSphere", 2.2, 0.2, (0, 0, 0), (100, 50, 100), (1 if periodic else 0, 0, 0), 5e-5)
    sim.add_particles(np.arange(n, dtype=np.int32), pos, rad, sphere_mass(rad), tag=np.zeros(n, np.int32), vel=vel,
                      angvel=angvel)
    sim.add_rot_friction_group("friction", 1e4, 0.6, 0.6, 1e4, 5e-5, True, True)
    sim.add_wall("bottom", (0, 0, 0), (0, 1, 0))
    sim.add_wall("top", (0, 50, 0), (0, -1, 0))
    sim.add_wall_group("bottom_w", "bottom", 1e4)
    sim.add_wall_group("top_w", "top", 1e4)
    return sim


def assert_forces_within_contribution_scale(a, orc_sim, rtol=1e-12):
    """Per-particle bar of the first force evaluation: |F_gpu - F_oracle| <= rtol times the sum of
    the magnitudes of the forces summed into F (and likewise for moments), the restatement's
    contribution sums (rounding of a different summation order is bounded by that sum)."""
    pa, pb = a.particles(), orc_sim.particles()
    assert np.array_equal(pa["id"], pb["id"])
    gf, gm = orc_sim.gross()
    for k, g in (("force", gf), ("moment", gm)):
        d = np.linalg.norm(pa[k] - pb[k], axis=1)
        bad = d > rtol * g + 1e-300
        assert not bad.any(), (k, int(bad.sum()), float((d / np.maximum(g, 1e-300)).max()))


class _Recorder:
    """Stands in for a simulation and records the calls a scenario builder makes."""

    def __init__(self, *args):
        self.args, self.calls = args, []

    def __getattr__(self, name):
        def call(*a, **k):
            self.calls.append((name, a, k))
        return call


def record(builder, edit=None, **kw):
    """(particles, connections, configure, creation args) of the scenario `builder(make, **kw)`:
    its add_particles arrays (after `edit(particles)`), its connections, and a function that makes
    its other calls (groups, walls) on another simulation."""
    rec = builder(lambda *a: _Recorder(*a), **kw)
    add = [c for c in rec.calls if c[0] == "add_particles"]
    assert len(add) == 1
    a, k = add[0][1], add[0][2]
    n = len(a[0])
    particles = {"id": np.asarray(a[0], np.int32), "pos": np.asarray(a[1], float), "rad": np.asarray(a[2], float),
                 "mass": np.asarray(a[3], float), "tag": k.get("tag", np.zeros(n, np.int32)), "vel": k.get("vel"),
                 "angvel": k.get("angvel"), "quat": k.get("quat")}
    if edit is not None:
        edit(particles)
    cc = [c for c in rec.calls if c[0] == "add_connections"]
    conns = tuple(np.asarray(x) for x in cc[0][1]) if cc else None
    rest = [c for c in rec.calls if c[0] not in ("add_particles", "add_connections")]

    def configure(sim):
        for name, a2, k2 in rest:
            getattr(sim, name)(*a2, **k2)

    return particles, conns, configure, rec.args


def split(make, world, builder, history_groups=("friction",), transport=None, edit=None, **kw):
    """The scenario `builder(make, **kw)` as a slab decomposition (esys.lsm.slabs.SlabDomain) over
    `world` workers made by `make`; `edit(particles)` may change the particle arrays first (apply
    the same edit to the one-worker run it is compared with, see replay)."""
    from esys.lsm.slabs import SlabDomain

    particles, conns, configure, args = record(builder, edit, **kw)
    return SlabDomain(make, configure, *args, particles, connections=conns, world=world, transport=transport,
                      history_groups=history_groups)


def replay(make, builder, edit=None, **kw):
    """The scenario on one worker, with the same particle edit as split's."""
    particles, conns, configure, args = record(builder, edit, **kw)
    sim = make(*args)
    p = particles
    sim.add_particles(p["id"], p["pos"], p["rad"], p["mass"], tag=p["tag"], vel=p["vel"], angvel=p["angvel"],
                      quat=p["quat"])
    if conns is not None:
        sim.add_connections(*conns)
    configure(sim)
    return sim


def drift_x(v):
    """Particle edit: a uniform velocity v along x on top of the scenario's own."""
    def edit(p):
        vel = np.zeros((len(p["id"]), 3)) if p["vel"] is None else np.array(p["vel"], float)
        vel[:, 0] += v
        p["vel"] = vel
    return edit


def wide_friction_pack(make, nx=12, ny=5, nz=6, extra_x=8.0, skin=0.05, **kw):
    """friction_pack in a box longer in x by extra_x (room to drift) with a small Verlet skin, so
    that neighbour rebuilds are frequent."""
    def wider(pt, gs, vd, lo, hi, circ, dt):
        return make(pt, gs, skin, lo, (hi[0] + extra_x, hi[1], hi[2]), circ, dt)
    return friction_pack(wider, nx=nx, ny=ny, nz=nz, **kw)


def damped_cloud(make, rot=True, n_side=4, seed=5, dt=1e-3, visc=100.0, max_iter=3, vdecades=(-6.0, 1.0)):
    """Isolated spheres (no contacts) under gravity with linear (and rotational) damping of
    viscosity * dt = 0.1, speeds spread over decades: the damping fixed point converges in
    a few iterations for slow particles and in more for fast ones, so a small maxIterations
    splits them into damped particles and particles left undamped (v_rel = 0)."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(*[np.arange(n_side)] * 3, indexing="ij"), -1).reshape(-1, 3)
    n = len(g)
    pos = (g + 0.5) * 3.0
    rad = np.full(n, 0.4)

    def spread():
        d = rng.normal(size=(n, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        return d * 10.0 ** rng.uniform(*vdecades, size=(n, 1))

    L = 3.0 * n_side
    sim = make("RotSphere" if rot else "NRotSphere", 1.2, 0.2, (0, 0, 0), (L, L, L), (0, 0, 0), dt)
    sim.add_particles(np.arange(n), pos, rad, sphere_mass(rad), tag=np.zeros(n, np.int32), vel=spread(),
                      angvel=spread() if rot else None)
    sim.add_elastic_group("elastic", 1000.0, True)
    sim.add_gravity("gravity", (0, 0, -9.81))
    sim.add_damping(0, visc, max_iter)
    if rot:
        sim.add_damping(1, visc, max_iter)
    return sim


def damping_iterations(v, f, inv_mass, mass, visc, dt, max_iter):
    """Iteration count of CDamping<T>::calcForces (Model/Damping.hpp:99-124) for one particle."""
    v_rel, error, count = np.zeros(3), 1.0, 0
    while error * error > 1e-12 and count < max_iter:
        count += 1
        old = v_rel
        v_rel = v + inv_mass * dt * (f - v_rel * visc * mass)
        error = float(np.dot(v_rel - old, v_rel - old))
    return count


def fitted_window_block(make, n=2000, L=10.0, seed=4, kt=1e3, kb=1e3, visc=0.05, dt=1e-5):
    """The differentiable-window benchmark's block at a small size: n spheres of radii in
    [0.2, 1.0] fitted by the packer into L x 2L x L, every pair within a 1e-3 gap bonded, seeded
    small initial velocities and spins, platens closing at 1.0, linear and rotational damping."""
    from esys.lsm import geometry as G

    pos, rad = G.fit_pack(n, (0, 0, 0), (L, 2 * L, L), 0.2, 1.0, seed=seed, max_failures=2000)
    i1, i2 = G.distance_connections(pos, rad, 1e-3)
    rng = np.random.default_rng(seed + 100)
    m = len(rad)
    sim = make("RotSphere", 2.2, 0.2, (0, 0, 0), (L, 2 * L, L), (0, 0, 0), dt)
    sim.add_particles(np.arange(m), pos, rad, sphere_mass(rad), tag=np.zeros(m, np.int32),
                      vel=rng.normal(0, 0.01, size=(m, 3)), angvel=rng.normal(0, 0.01, size=(m, 3)))
    sim.add_connections(np.ones(len(i1), np.int32), i1, i2)
    sim.add_rot_bond_group("bonds", 1, 1e5, 1e5, kt, kb, 1e6, 1e6, 1e6, 1e6, True, True, 1.0)
    y0, y1 = float((pos[:, 1] - rad).min()), float((pos[:, 1] + rad).max())
    sim.add_wall("bottom", (0, y0, 0), (0, 1, 0))
    sim.add_wall("top", (0, y1, 0), (0, -1, 0))
    sim.add_wall_group("bottom_w", "bottom", 1e5)
    sim.add_wall_group("top_w", "top", 1e5)
    sim.add_damping(0, visc, 100)
    sim.add_damping(1, visc, 100)
    sim.set_wall_velocity("bottom", (0, 1.0, 0))
    sim.set_wall_velocity("top", (0, -1.0, 0))
    return sim
