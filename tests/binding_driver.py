"""ctypes front end of the ASubLattice binding's test build (tests/binding): a master that drives
TGpuSubLattice through the reference's own command and buffer protocol, with the method names
of the DemSim / OracleSim objects the scenarios use, so a scenario builds the same specimen
through the binding, the library directly and the oracle."""
import ctypes as C

import numpy as np

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)

SIGNATURES = {
    "slm_error": (C.c_char_p, []),
    "slm_start": (C.c_int, [C.c_int, C.c_double, C.c_double, _D, _D, _I, C.c_double]),
    "slm_add_particles": (C.c_int, [C.c_int, _I, _I, _D, _D, _D, _D, _D]),
    "slm_add_connections": (C.c_int, [C.c_int, _I, _I, _I]),
    "slm_add_wall": (C.c_int, [C.c_char_p, _D, _D]),
    "slm_add_wall_group": (C.c_int, [C.c_char_p, C.c_char_p, C.c_double]),
    "slm_add_elastic": (C.c_int, [C.c_char_p, C.c_double, C.c_int]),
    "slm_add_rot_friction": (C.c_int, [C.c_char_p] + [C.c_double] * 5 + [C.c_int, C.c_int]),
    "slm_add_rot_bond": (C.c_int, [C.c_char_p, C.c_int] + [C.c_double] * 8 + [C.c_int, C.c_int, C.c_double]),
    "slm_add_damping": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_int]),
    "slm_add_gravity": (C.c_int, [C.c_char_p, _D]),
    "slm_add_exclusion": (C.c_int, [C.c_char_p, C.c_char_p]),
    "slm_run": (C.c_int, [C.c_int]),
    "slm_move_wall": (C.c_int, [C.c_char_p, _D]),
    "slm_get_wall_force": (C.c_int, [C.c_char_p, _D]),
    "slm_get_wall_pos": (C.c_int, [C.c_char_p, _D]),
    "slm_num_particles": (C.c_int, []),
    "slm_get_particles": (C.c_int, [C.c_int, _I, _D, _D, _D, _D, _D, _D]),
    "slm_finish": (C.c_int, []),
}


class BindingError(RuntimeError):
    pass


def bind(lib):
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_D)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_I)


class SubLatticeMaster:
    """One master + TGpuSubLattice worker pair (one at a time per process)."""

    def __init__(self, lib, particle_type, grid_spacing, verlet_dist, bbox_min, bbox_max, circ=(0, 0, 0), dt=1e-4):
        self.lib = bind(lib)
        self.rot = particle_type == "RotSphere"
        self.dt = dt
        self._n = 0
        mn, pmn = _d(bbox_min)
        mx, pmx = _d(bbox_max)
        cc, pcc = _i(circ)
        self._chk(self.lib.slm_start(int(self.rot), grid_spacing, verlet_dist, pmn, pmx, pcc, dt))

    def _chk(self, rc):
        if rc < 0:
            raise BindingError(self.lib.slm_error().decode())
        return rc

    def close(self):
        return self._chk(self.lib.slm_finish())

    # -- set-up, with the DemSim method names --
    def add_particles(self, id, pos, rad, mass, tag=None, vel=None, angvel=None, quat=None, flags=None):
        n = len(id)
        ids, pid = _i(id)
        tags, ptag = _i(np.zeros(n) if tag is None else tag)
        p, pp = _d(np.reshape(pos, (n, 3)))
        r, pr = _d(rad)
        m, pm = _d(mass)
        v, pv = _d(np.zeros((n, 3)) if vel is None else np.reshape(vel, (n, 3)))
        w, pw = _d(np.zeros((n, 3)) if angvel is None else np.reshape(angvel, (n, 3)))
        self._chk(self.lib.slm_add_particles(n, pid, ptag, pp, pr, pm, pv, pw))
        self._n += n

    def add_connections(self, tag, id1, id2):
        t, pt = _i(tag)
        a, pa = _i(id1)
        b, pb = _i(id2)
        self._chk(self.lib.slm_add_connections(len(t), pt, pa, pb))

    def add_wall(self, name, origin, normal):
        o, po = _d(origin)
        nn, pn = _d(normal)
        self._chk(self.lib.slm_add_wall(name.encode(), po, pn))

    def add_wall_group(self, name, wall, k):
        self._chk(self.lib.slm_add_wall_group(name.encode(), wall.encode(), k))

    def add_elastic_group(self, name, k, scaling=True):
        self._chk(self.lib.slm_add_elastic(name.encode(), k, int(scaling)))

    def add_rot_friction_group(self, name, k, mu_s, mu_d, k_s, dt, scaling=True, meanR_scaling=True):
        self._chk(self.lib.slm_add_rot_friction(name.encode(), k, mu_s, mu_d, k_s, dt, int(scaling), int(meanR_scaling)))

    def add_rot_bond_group(self, name, tag, kr, ks, kt, kb, max_n, max_s, max_t, max_b, scaling=True,
                           meanR_scaling=True, truncated=1.0):
        self._chk(self.lib.slm_add_rot_bond(name.encode(), int(tag), kr, ks, kt, kb, max_n, max_s, max_t, max_b,
                                            int(scaling), int(meanR_scaling), truncated))

    def add_damping(self, rot, visc, max_iter=100):
        self._chk(self.lib.slm_add_damping(int(rot), visc, self.dt, int(max_iter)))

    def add_gravity(self, name, g):
        a, pa = _d(g)
        self._chk(self.lib.slm_add_gravity(name.encode(), pa))

    def add_exclusion(self, bonded, dynamic):
        self._chk(self.lib.slm_add_exclusion(bonded.encode(), dynamic.encode()))

    # -- running --
    def step(self, n=1):
        self._chk(self.lib.slm_run(int(n)))

    def move_wall(self, name, d):
        a, pa = _d(d)
        self._chk(self.lib.slm_move_wall(name.encode(), pa))

    def wall(self, name):
        p, pp = _d(np.zeros(3))
        f, pf = _d(np.zeros(3))
        self._chk(self.lib.slm_get_wall_pos(name.encode(), pp))
        self._chk(self.lib.slm_get_wall_force(name.encode(), pf))
        return p, f

    def num_particles(self):
        return self._chk(self.lib.slm_num_particles())

    def particles(self):
        cap = max(self._n, 1)
        ids, pid = _i(np.zeros(cap))
        arrs = [_d(np.zeros((cap, 3))) for _ in range(5)]
        q, pq = _d(np.zeros((cap, 4)))
        m = self._chk(self.lib.slm_get_particles(cap, pid, *[a[1] for a in arrs], pq))
        o = np.argsort(ids[:m], kind="stable")
        pos, vel, force, angvel, moment = (a[0][:m][o] for a in arrs)
        return {"id": ids[:m][o], "pos": pos, "vel": vel, "force": force, "angvel": angvel, "moment": moment,
                "quat": q[:m][o]}
