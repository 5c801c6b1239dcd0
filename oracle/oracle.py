"""ctypes front end for the two CPU oracles of the DEM step (test infrastructure).

* ``backend="ref"`` loads ``oracle/_ref/libesys_ref.so``: ESyS-Particle's own
  hot-path classes compiled from the reference sources (see ``oracle/Makefile``
  and ``oracle/ref_harness.cpp``).
* ``backend="orc"`` loads ``oracle/_build/libesys_oracle.so``: the CPU
  restatement ``oracle/dem_oracle.cpp``, which also covers periodic x.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline legs and
reference arm use this module; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {
    "ref": (os.path.join(_HERE, "_ref", "libesys_ref.so"), "ref_"),
    "orc": (os.path.join(_HERE, "_build", "libesys_oracle.so"), "orc_"),
}
_loaded: dict = {}

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_P = C.c_void_p
_S = C.c_char_p


def available(backend: str) -> bool:
    return os.path.exists(_LIBS[backend][0])


def rsi_pack_ref(seed, n, bmin, bmax, periodic_x, dist, p0, p1, rmin, rmax, max_attempts):
    """The benchmarks' seeded RSI packer (``lsm_pack_rsi``, the product's packing.cpp) as
    linked into the reference library: the same packing without loading the product library.
    Returns (pos, rad) of the spheres placed."""
    lib = C.CDLL(_LIBS["ref"][0])
    f = lib.lsm_pack_rsi
    f.argtypes = [C.c_ulonglong, C.c_int, _D, _D, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                  C.c_int, _D, _D]
    f.restype = C.c_int
    pos = np.zeros((n, 3))
    rad = np.zeros(n)
    lo = np.ascontiguousarray(bmin, dtype=np.float64)
    hi = np.ascontiguousarray(bmax, dtype=np.float64)
    k = f(seed, n, lo.ctypes.data_as(_D), hi.ctypes.data_as(_D), periodic_x, dist, p0, p1, rmin, rmax, max_attempts,
          pos.ctypes.data_as(_D), rad.ctypes.data_as(_D))
    if k < 0:
        raise ValueError("lsm_pack_rsi: bad arguments")
    return pos[:k], rad[:k]


def _lib(backend: str):
    if backend in _loaded:
        return _loaded[backend]
    path, pfx = _LIBS[backend]
    lib = C.CDLL(path)
    sig = {
        "create": (C.c_int, [C.POINTER(_P), C.c_int, C.c_double, C.c_double, _D, _D, _I, C.c_double]),
        "destroy": (C.c_int, [_P]),
        "last_error": (_S, [_P]),
        "add_particles": (C.c_int, [_P, C.c_int, _I, _I, _D, _D, _D, _D, _D, _D, _I]),
        "add_connections": (C.c_int, [_P, C.c_int, _I, _I, _I]),
        "add_wall": (C.c_int, [_P, _S, _D, _D]),
        "add_elastic_group": (C.c_int, [_P, _S, C.c_double, C.c_int]),
        "add_rot_friction_group": (C.c_int, [_P, _S] + [C.c_double] * 5 + [C.c_int, C.c_int]),
        "add_rot_bond_group": (C.c_int, [_P, _S, C.c_int] + [C.c_double] * 8 + [C.c_int, C.c_int, C.c_double]),
        "add_wall_group": (C.c_int, [_P, _S, _S, C.c_double]),
        "add_gravity": (C.c_int, [_P, _S, _D]),
        "add_damping": (C.c_int, [_P, C.c_int, C.c_double, C.c_int]),
        "add_exclusion": (C.c_int, [_P, _S, _S]),
        "step": (C.c_int, [_P, C.c_int]),
        "move_wall": (C.c_int, [_P, _S, _D]),
        "set_wall_velocity": (C.c_int, [_P, _S, _D]),
        "set_group_param": (C.c_int, [_P, _S, _S, C.c_double]),
        "window_dual": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_char_p), _D, _D]),
        "apply_force_to_wall": (C.c_int, [_P, _S, _D]),
        "get_wall": (C.c_int, [_P, _S, _D, _D]),
        "num_particles": (C.c_int, [_P]),
        "get_particles": (C.c_int, [_P, _I, _D, _D, _D, _D, _D, _D]),
        "num_pairs": (C.c_int, [_P, _S]),
        "get_pairs": (C.c_int, [_P, _S, _I, _I, _D]),
        "num_breaks": (C.c_int, [_P]),
        "get_breaks": (C.c_int, [_P, _I, _I, _I]),
        "move_tagged": (C.c_int, [_P, C.c_int, C.c_int, _D]),
        "add_nrot_friction_group": (C.c_int, [_P, _S] + [C.c_double] * 4 + [C.c_int]),
        "add_local_damping": (C.c_int, [_P, _S, C.c_int, C.c_double]),
        "add_hertz_mindlin_group": (C.c_int, [_P, _S] + [C.c_double] * 4),
        "add_hertz_mindlin_visco_group": (C.c_int, [_P, _S] + [C.c_double] * 5),
        "add_brittle_beam_dzc_group": (C.c_int, [_P, _S, C.c_int] + [C.c_double] * 10),
        "add_brittle_beam_sc_group": (C.c_int, [_P, _S, C.c_int] + [C.c_double] * 7),
        "add_nrot_bond_group": (C.c_int, [_P, _S, C.c_int, C.c_double, C.c_double, C.c_int]),
        "save_checkpoint": (C.c_int, [_P, _S, C.c_int]),
        "load_checkpoint": (C.c_int, [_P, _S, C.c_longlong]),
        "timestep": (C.c_longlong, [_P]),
        "get_gross": (C.c_int, [_P, _D, _D]),
        "set_particles": (C.c_int, [_P, C.c_int, _I, _D, _D, _D, _D]),
        "search_neighbors": (C.c_int, [_P]),
        "num_rebuilds": (C.c_int, [_P]),
        "set_pair_states": (C.c_int, [_P, _S, C.c_int, _I, _I, _D]),
    }
    fns = {}
    for name, (res, args) in sig.items():
        f = getattr(lib, pfx + name, None)
        if f is None:
            continue
        f.restype = res
        f.argtypes = args
        fns[name] = f
    _loaded[backend] = fns
    return fns


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_I)


def _v3(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(3))


class OracleSim:
    """One simulated worker, driven through an oracle's C ABI."""

    def __init__(self, backend, particle_type, grid_spacing, verlet_dist, bbox_min, bbox_max, circ=(0, 0, 0), dt=1e-4):
        self.f = _lib(backend)
        self.backend = backend
        self.h = _P()
        mn, mx = _v3(bbox_min), _v3(bbox_max)
        cc = np.ascontiguousarray(np.asarray(circ, dtype=np.int32))
        pt = {"NRotSphere": 0, "RotSphere": 1}[particle_type] if isinstance(particle_type, str) else int(particle_type)
        self._chk(self.f["create"](C.byref(self.h), pt, grid_spacing, verlet_dist, _dp(mn), _dp(mx), _ip(cc), dt))
        self.rot = pt == 1

    def _chk(self, rc):
        if rc < 0:
            msg = self.f["last_error"](self.h) if self.h else b"create failed"
            raise RuntimeError((msg or b"").decode())
        return rc

    def __del__(self):
        try:
            if self.h:
                self.f["destroy"](self.h)
                self.h = _P()
        except Exception:
            pass

    def add_particles(self, id, pos, rad, mass, tag=None, vel=None, angvel=None, quat=None, flags=None):
        n = len(id)
        a = lambda x, dt: None if x is None else np.ascontiguousarray(np.asarray(x, dtype=dt))
        id, tag, flags = a(id, np.int32), a(tag, np.int32), a(flags, np.int32)
        pos, rad, mass = a(pos, np.float64), a(rad, np.float64), a(mass, np.float64)
        vel, angvel, quat = a(vel, np.float64), a(angvel, np.float64), a(quat, np.float64)
        self._chk(self.f["add_particles"](self.h, n, _ip(id), _ip(tag), _dp(pos), _dp(rad), _dp(mass), _dp(vel),
                                          _dp(angvel), _dp(quat), _ip(flags)))

    def add_connections(self, tag, id1, id2):
        t = np.ascontiguousarray(tag, dtype=np.int32)
        a = np.ascontiguousarray(id1, dtype=np.int32)
        b = np.ascontiguousarray(id2, dtype=np.int32)
        self._chk(self.f["add_connections"](self.h, len(a), _ip(t), _ip(a), _ip(b)))

    def add_wall(self, name, origin, normal):
        self._chk(self.f["add_wall"](self.h, name.encode(), _dp(_v3(origin)), _dp(_v3(normal))))

    def add_elastic_group(self, name, k, scaling=True):
        self._chk(self.f["add_elastic_group"](self.h, name.encode(), k, int(scaling)))

    def add_rot_friction_group(self, name, k, mu_s, mu_d, k_s, dt, scaling=True, meanR_scaling=True):
        self._chk(self.f["add_rot_friction_group"](self.h, name.encode(), k, mu_s, mu_d, k_s, dt, int(scaling),
                                                   int(meanR_scaling)))

    def add_rot_bond_group(self, name, tag, kr, ks, kt, kb, max_n, max_s, max_t, max_b, scaling=True,
                           meanR_scaling=True, truncated=1.0):
        self._chk(self.f["add_rot_bond_group"](self.h, name.encode(), tag, kr, ks, kt, kb, max_n, max_s, max_t,
                                               max_b, int(scaling), int(meanR_scaling), truncated))

    def add_hertz_mindlin_group(self, name, E, nu, mu, dt):
        """HertzMindlin (CHertzMindlinInteraction) group (reference backend)."""
        if "add_hertz_mindlin_group" not in self.f:
            raise NotImplementedError(f"{self.backend} has no HertzMindlin groups")
        self._chk(self.f["add_hertz_mindlin_group"](self.h, name.encode(), E, nu, mu, dt))

    def add_brittle_beam_dzc_group(self, name, tag, kr, ks, kt, kb, cohesion, tCutoff, cCutoff, fAngle, beta1, beta2):
        """BrittleBeamDZC (BrittleBeamDZCInteraction) group (reference backend)."""
        if "add_brittle_beam_dzc_group" not in self.f:
            raise NotImplementedError(f"{self.backend} has no BrittleBeamDZC groups")
        self._chk(self.f["add_brittle_beam_dzc_group"](self.h, name.encode(), int(tag), *(float(x) for x in (
            kr, ks, kt, kb, cohesion, tCutoff, cCutoff, fAngle, beta1, beta2))))

    def add_brittle_beam_sc_group(self, name, tag, kr, ks, kt, kb, cohesion, tCutoff, fAngle):
        """BrittleBeamSC (BrittleBeamSCInteraction) group (reference backend)."""
        if "add_brittle_beam_sc_group" not in self.f:
            raise NotImplementedError(f"{self.backend} has no BrittleBeamSC groups")
        self._chk(self.f["add_brittle_beam_sc_group"](self.h, name.encode(), int(tag), *(float(x) for x in (
            kr, ks, kt, kb, cohesion, tCutoff, fAngle))))

    def add_hertz_mindlin_visco_group(self, name, E, nu, mu, COR, dt):
        """HertzMindlinVisco (CHertzMindlinViscoInteraction) group (reference backend)."""
        if "add_hertz_mindlin_visco_group" not in self.f:
            raise NotImplementedError(f"{self.backend} has no HertzMindlinVisco groups")
        self._chk(self.f["add_hertz_mindlin_visco_group"](self.h, name.encode(), E, nu, mu, COR, dt))

    def add_local_damping(self, name, rot, visc):
        """LocalDamping / RotLocalDamping group (reference backend)."""
        if "add_local_damping" not in self.f:
            raise NotImplementedError(f"{self.backend} has no local damping")
        self._chk(self.f["add_local_damping"](self.h, name.encode(), int(rot), float(visc)))

    def add_nrot_friction_group(self, name, k, mu, k_s, dt, scaling=True):
        """NRotFriction (CFrictionInteraction) group (reference backend)."""
        if "add_nrot_friction_group" not in self.f:
            raise NotImplementedError(f"{self.backend} has no NRotFriction groups")
        self._chk(self.f["add_nrot_friction_group"](self.h, name.encode(), k, mu, k_s, dt, int(scaling)))

    def add_nrot_bond_group(self, name, tag, k, rbreak, scaling=True):
        """NRotBond (CBondedInteraction) group (reference backend)."""
        if "add_nrot_bond_group" not in self.f:
            raise NotImplementedError(f"{self.backend} has no NRotBond groups")
        self._chk(self.f["add_nrot_bond_group"](self.h, name.encode(), int(tag), k, rbreak, int(scaling)))

    def add_wall_group(self, name, wall, k):
        self._chk(self.f["add_wall_group"](self.h, name.encode(), wall.encode(), k))

    def add_gravity(self, name, g):
        self._chk(self.f["add_gravity"](self.h, name.encode(), _dp(_v3(g))))

    def add_damping(self, rot, visc, max_iter=100):
        self._chk(self.f["add_damping"](self.h, int(rot), visc, max_iter))

    def add_exclusion(self, bonded, dynamic):
        self._chk(self.f["add_exclusion"](self.h, bonded.encode(), dynamic.encode()))

    def step(self, n=1):
        self._chk(self.f["step"](self.h, n))

    def move_wall(self, name, d):
        self._chk(self.f["move_wall"](self.h, name.encode(), _dp(_v3(d))))

    def apply_force_to_wall(self, group, force):
        self._chk(self.f["apply_force_to_wall"](self.h, group.encode(), _dp(_v3(force))))

    def set_wall_velocity(self, name, v):
        if "set_wall_velocity" not in self.f:
            raise NotImplementedError(f"{self.backend} has no wall loader")
        self._chk(self.f["set_wall_velocity"](self.h, name.encode(), _dp(_v3(v))))
        self._loaders = getattr(self, "_loaders", set()) | {name}

    def set_group_param(self, group, key, value):
        if "set_group_param" not in self.f:
            raise NotImplementedError(f"{self.backend} cannot change group parameters")
        self._chk(self.f["set_group_param"](self.h, group.encode(), key.encode(), float(value)))

    def window_dual(self, nsteps, seeds, ngroups):
        """Forward-mode dual-number window (the restatement only): wall-group reactions
        R[nsteps, ngroups, 3] and their derivatives dR[nsteps, ngroups, 3, len(seeds)]
        with respect to the named seeds (see orc_window_dual)."""
        if "window_dual" not in self.f:
            raise NotImplementedError(f"{self.backend} has no dual window")
        ns = len(seeds)
        R = np.zeros((nsteps, ngroups, 3))
        dR = np.zeros((nsteps, ngroups, 3, max(ns, 1)))
        arr = (C.c_char_p * max(ns, 1))(*[x.encode() for x in seeds])
        self._chk(self.f["window_dual"](self.h, int(nsteps), ns, arr, _dp(R), _dp(dR)))
        return R, dR[..., :ns]

    def save_checkpoint(self, path, precision=12):
        """Restart checkpoint worker file written by the reference's own writers (reference backend)."""
        if "save_checkpoint" not in self.f:
            raise NotImplementedError(f"{self.backend} does not write checkpoints")
        self._chk(self.f["save_checkpoint"](self.h, str(path).encode(), int(precision)))

    def load_checkpoint(self, path, timestep):
        """Load a restart checkpoint worker file with the reference's own readers (reference backend)."""
        if "load_checkpoint" not in self.f:
            raise NotImplementedError(f"{self.backend} does not read checkpoints")
        self._chk(self.f["load_checkpoint"](self.h, str(path).encode(), int(timestep)))

    def move_tagged(self, tag, d, mask=-1):
        self._chk(self.f["move_tagged"](self.h, tag, mask, _dp(_v3(d))))

    def wall(self, name):
        p, f = np.zeros(3), np.zeros(3)
        self._chk(self.f["get_wall"](self.h, name.encode(), _dp(p), _dp(f)))
        return p, f

    def particles(self):
        n = self._chk(self.f["num_particles"](self.h))
        out = {"id": np.zeros(n, np.int32)}
        for k, w in (("pos", 3), ("vel", 3), ("angvel", 3), ("quat", 4), ("force", 3), ("moment", 3)):
            out[k] = np.zeros((n, w))
        self._chk(self.f["get_particles"](self.h, _ip(out["id"]), _dp(out["pos"]), _dp(out["vel"]),
                                          _dp(out["angvel"]), _dp(out["quat"]), _dp(out["force"]),
                                          _dp(out["moment"])))
        order = np.argsort(out["id"], kind="stable")
        return {k: v[order] for k, v in out.items()}

    def set_particles(self, pos=None, vel=None, angvel=None, quat=None, id=None):
        """State of the particles with these ids (restatement only); deleted ones come back."""
        if "set_particles" not in self.f:
            raise NotImplementedError(f"{self.backend} cannot set particle state")
        ids = np.ascontiguousarray(id, dtype=np.int32)
        keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (pos, vel, angvel, quat)]
        self._chk(self.f["set_particles"](self.h, len(ids), _ip(ids), *(_dp(a) for a in keep)))

    def revive_particles(self, id, pos=None, vel=None, angvel=None, quat=None):
        self.set_particles(pos=pos, vel=vel, angvel=angvel, quat=quat, id=id)

    def search_neighbors(self):
        self._chk(self.f["search_neighbors"](self.h))

    def set_pair_states(self, group, id1, id2, state):
        a = np.ascontiguousarray(id1, dtype=np.int32)
        b = np.ascontiguousarray(id2, dtype=np.int32)
        st = np.ascontiguousarray(np.asarray(state, np.float64).reshape(-1, 5))
        return self._chk(self.f["set_pair_states"](self.h, group.encode(), len(a), _ip(a), _ip(b), _dp(st)))

    def counters(self):
        """The subset of the GPU handle's counters a restatement has: neighbour searches."""
        return {"rebuilds": self._chk(self.f["num_rebuilds"](self.h))}

    def gross(self):
        """Restatement only: each particle's sum of the magnitudes of the forces and of the moments
        applied to it in the last step (rows sorted by id, like particles()): the scale a summed
        force is compared at."""
        if "get_gross" not in self.f:
            raise NotImplementedError(f"{self.backend} has no contribution sums")
        n = self._chk(self.f["num_particles"](self.h))
        ids, gf, gm = np.zeros(n, np.int32), np.zeros(n), np.zeros(n)
        self._chk(self.f["get_particles"](self.h, _ip(ids), None, None, None, None, None, None))
        self._chk(self.f["get_gross"](self.h, _dp(gf), _dp(gm)))
        order = np.argsort(ids, kind="stable")
        return gf[order], gm[order]

    def pairs(self, group):
        n = self._chk(self.f["num_pairs"](self.h, group.encode()))
        a, b = np.zeros(n, np.int32), np.zeros(n, np.int32)
        st = np.zeros((n, 5))
        self._chk(self.f["get_pairs"](self.h, group.encode(), _ip(a), _ip(b), _dp(st)))
        order = np.lexsort((b, a))
        return a[order], b[order], st[order]

    def breaks(self):
        n = self._chk(self.f["num_breaks"](self.h))
        a, b, s = (np.zeros(n, np.int32) for _ in range(3))
        self._chk(self.f["get_breaks"](self.h, _ip(a), _ip(b), _ip(s)))
        order = np.lexsort((b, a, s))
        return a[order], b[order], s[order]

    @property
    def timestep(self):
        return int(self.f["timestep"](self.h))
