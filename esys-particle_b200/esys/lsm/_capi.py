"""ctypes binding of the B200 DEM library's C ABI (include/esys_dem.h).

``DemSim`` is a thin, one-to-one wrapper of the ``dem_*`` functions: one handle
is one ESyS-Particle worker sub-lattice on one GPU.  The library must have been
built (``python esys-particle_b200/build.py``); there is no CPU fallback and
loading fails loudly when the shared object or a GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.normpath(os.path.join(_HERE, "..", "..", "lib", "libesys_dem_b200.so"))

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_P = C.c_void_p
_S = C.c_char_p

# name -> (restype, argtypes); every symbol declared in include/esys_dem.h
SIGNATURES = {
    "dem_create": (C.c_int, [C.POINTER(_P), C.c_int, C.c_double, C.c_double, _D, _D, _I, C.c_double]),
    "dem_destroy": (C.c_int, [_P]),
    "dem_last_error": (_S, [_P]),
    "dem_add_particles": (C.c_int, [_P, C.c_int, _I, _I, _D, _D, _D, _D, _D, _D, _I]),
    "dem_add_connections": (C.c_int, [_P, C.c_int, _I, _I, _I]),
    "dem_add_wall": (C.c_int, [_P, _S, _D, _D]),
    "dem_add_elastic_group": (C.c_int, [_P, _S, C.c_double, C.c_int]),
    "dem_add_rot_friction_group": (C.c_int, [_P, _S] + [C.c_double] * 5 + [C.c_int, C.c_int]),
    "dem_add_rot_bond_group": (C.c_int, [_P, _S, C.c_int] + [C.c_double] * 8 + [C.c_int, C.c_int, C.c_double]),
    "dem_add_nrot_friction_group": (C.c_int, [_P, _S] + [C.c_double] * 4 + [C.c_int]),
    "dem_add_local_damping": (C.c_int, [_P, _S, C.c_int, C.c_double]),
    "dem_add_hertz_mindlin_group": (C.c_int, [_P, _S] + [C.c_double] * 4),
    "dem_add_hertz_mindlin_visco_group": (C.c_int, [_P, _S] + [C.c_double] * 5),
    "dem_add_brittle_beam_dzc_group": (C.c_int, [_P, _S, C.c_int] + [C.c_double] * 10),
    "dem_add_brittle_beam_sc_group": (C.c_int, [_P, _S, C.c_int] + [C.c_double] * 7),
    "dem_add_nrot_bond_group": (C.c_int, [_P, _S, C.c_int, C.c_double, C.c_double, C.c_int]),
    "dem_add_wall_group": (C.c_int, [_P, _S, _S, C.c_double]),
    "dem_add_gravity": (C.c_int, [_P, _S, _D]),
    "dem_add_damping": (C.c_int, [_P, C.c_int, C.c_double, C.c_int]),
    "dem_add_exclusion": (C.c_int, [_P, _S, _S]),
    "dem_set_timestep": (C.c_int, [_P, C.c_double]),
    "dem_step": (C.c_int, [_P, C.c_int]),
    "dem_move_wall": (C.c_int, [_P, _S, _D]),
    "dem_set_wall_velocity": (C.c_int, [_P, _S, _D]),
    "dem_apply_force_to_wall": (C.c_int, [_P, _S, _D]),
    "dem_get_wall": (C.c_int, [_P, _S, _D, _D]),
    "dem_num_particles": (C.c_int, [_P]),
    "dem_get_particles": (C.c_int, [_P, _I, _D, _D, _D, _D, _D, _D]),
    "dem_num_pairs": (C.c_int, [_P, _S]),
    "dem_get_pairs": (C.c_int, [_P, _S, _I, _I, _D]),
    "dem_num_breaks": (C.c_int, [_P]),
    "dem_get_breaks": (C.c_int, [_P, _I, _I, _I]),
    "dem_move_tagged": (C.c_int, [_P, C.c_int, C.c_int, _D]),
    "dem_timestep": (C.c_longlong, [_P]),
    "dem_set_option": (C.c_int, [_P, _S, C.c_double]),
    "dem_set_particles": (C.c_int, [_P, C.c_int, _I, _D, _D, _D, _D]),
    "dem_revive_particles": (C.c_int, [_P, C.c_int, _I, _D, _D, _D, _D]),
    "dem_set_pair_states": (C.c_int, [_P, _S, C.c_int, _I, _I, _D]),
    "dem_set_stream": (C.c_int, [_P, C.c_void_p]),
    "dem_get_counters": (C.c_int, [_P, C.POINTER(C.c_longlong), C.c_int]),
    "dem_precision_check": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "dem_precision_report": (C.c_int, [_P, C.POINTER(C.c_double), C.c_int]),
    "dem_wall_reactions_noalloc": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "dem_set_group_param": (C.c_int, [_P, _S, _S, C.c_double]),
    "dem_particle_scalar_field": (C.c_int, [_P, _S, _D]),
    "dem_particle_vector_field": (C.c_int, [_P, _S, _D]),
    "dem_interaction_scalar_field": (C.c_int, [_P, _S, _S, _D]),
    "dem_window_num_params": (C.c_int, [_P]),
    "dem_window_forward": (C.c_int, [_P, C.c_int, C.c_int, _D]),
    "dem_window_adjoint": (C.c_int, [_P, _D, _D, _D, _D, _D, _D]),
    "dem_window_rewind": (C.c_int, [_P]),
    "dem_ensemble_create": (C.c_int, [C.POINTER(_P), C.POINTER(_P), C.c_int]),
    "dem_ensemble_destroy": (C.c_int, [_P]),
    "dem_ensemble_last_error": (_S, [_P]),
    "dem_ensemble_step": (C.c_int, [_P, C.c_int]),
    "dem_search_neighbors": (C.c_int, [_P]),
    "dem_save_checkpoint": (C.c_int, [_P, _S, C.c_int]),
    "dem_load_checkpoint": (C.c_int, [_P, _S, C.c_longlong]),
    "dem_save_snapshot": (C.c_int, [_P, _S]),
    "dem_window_release": (C.c_int, [_P]),
    "dem_ensemble_window_forward": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(_D)]),
    "dem_ensemble_window_adjoint": (C.c_int, [_P, C.POINTER(_D), C.POINTER(_D), C.POINTER(_D), C.POINTER(_D)]),
    "dem_ensemble_set_option": (C.c_int, [_P, _S, C.c_double]),
    "dem_ensemble_get_counters": (C.c_int, [_P, C.POINTER(C.c_longlong), C.c_int]),
}

_lib = None


def load_library(path: str = LIB_PATH):
    """Load the DEM library and bind every C-ABI symbol; raise if anything is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"B200 DEM library not built: {path} (run esys-particle_b200/build.py)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)  # AttributeError if the symbol is missing
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_I)


def _v3(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(3))


# Status codes of include/esys_dem.h
DEM_OK, DEM_ERR_ARG, DEM_ERR_OVERFLOW, DEM_ERR_CUDA, DEM_ERR_INTERNAL, DEM_ERR_STATE = 0, -1, -2, -3, -4, -5


class DemError(RuntimeError):
    """A failed library call; ``status`` is its DEM_ERR_* code (None where no call failed)."""

    def __init__(self, msg, status=None):
        super().__init__(msg)
        self.status = status


class DemSim:
    """One worker sub-lattice on the GPU (a ``dem_sim`` handle)."""

    def __init__(self, particle_type, grid_spacing, verlet_dist, bbox_min, bbox_max, circ=(0, 0, 0), dt=1e-4):
        self.lib = load_library()
        self.h = _P()
        mn, mx = _v3(bbox_min), _v3(bbox_max)
        cc = np.ascontiguousarray(np.asarray(circ, dtype=np.int32))
        pt = {"NRotSphere": 0, "RotSphere": 1}[particle_type] if isinstance(particle_type, str) else int(particle_type)
        rc = self.lib.dem_create(C.byref(self.h), pt, float(grid_spacing), float(verlet_dist), _dp(mn), _dp(mx),
                                 _ip(cc), float(dt))
        if rc != 0:
            raise DemError(self.lib.dem_last_error(None).decode(), rc)
        self.rot = pt == 1
        self.wall_groups = []  # wall interaction groups, in the library's (name) order
        self._bond_prm = {}    # RotBond group -> [normalK, shearK, torsionK, bendingK]
        self._dyn_prm = {}     # dynamic group -> (kind, [normalK, shearK])
        self._damp_prm = {}    # "Damping" / "RotDamping" -> viscosity

    def _chk(self, rc):
        if rc < 0:
            raise DemError(self.lib.dem_last_error(self.h).decode(), rc)
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.lib.dem_destroy(self.h)
            self.h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_particles(self, id, pos, rad, mass, tag=None, vel=None, angvel=None, quat=None, flags=None):
        a = lambda x, dt: None if x is None else np.ascontiguousarray(np.asarray(x, dtype=dt))
        id, tag, flags = a(id, np.int32), a(tag, np.int32), a(flags, np.int32)
        pos, rad, mass = a(pos, np.float64), a(rad, np.float64), a(mass, np.float64)
        vel, angvel, quat = a(vel, np.float64), a(angvel, np.float64), a(quat, np.float64)
        self._chk(self.lib.dem_add_particles(self.h, len(id), _ip(id), _ip(tag), _dp(pos), _dp(rad), _dp(mass),
                                             _dp(vel), _dp(angvel), _dp(quat), _ip(flags)))

    def add_connections(self, tag, id1, id2):
        t = np.ascontiguousarray(tag, dtype=np.int32)
        a = np.ascontiguousarray(id1, dtype=np.int32)
        b = np.ascontiguousarray(id2, dtype=np.int32)
        self._chk(self.lib.dem_add_connections(self.h, len(a), _ip(t), _ip(a), _ip(b)))

    def add_wall(self, name, origin, normal):
        self._chk(self.lib.dem_add_wall(self.h, name.encode(), _dp(_v3(origin)), _dp(_v3(normal))))

    def add_elastic_group(self, name, k, scaling=True):
        self._chk(self.lib.dem_add_elastic_group(self.h, name.encode(), float(k), int(scaling)))
        self._dyn_prm[name] = (0, [float(k), 0.0])

    def add_rot_friction_group(self, name, k, mu_s, mu_d, k_s, dt, scaling=True, meanR_scaling=True):
        self._chk(self.lib.dem_add_rot_friction_group(self.h, name.encode(), float(k), float(mu_s), float(mu_d),
                                                      float(k_s), float(dt), int(scaling), int(meanR_scaling)))
        self._dyn_prm[name] = (1, [float(k), float(k_s)])

    def add_hertz_mindlin_group(self, name, E, nu, mu, dt):
        self._chk(self.lib.dem_add_hertz_mindlin_group(self.h, name.encode(), float(E), float(nu), float(mu), float(dt)))
        self._dyn_prm[name] = (3, [float(E), float(nu)])

    def add_brittle_beam_dzc_group(self, name, tag, kr, ks, kt, kb, cohesion, tCutoff, cCutoff, fAngle, beta1, beta2):
        self._chk(self.lib.dem_add_brittle_beam_dzc_group(self.h, name.encode(), int(tag), *(float(x) for x in (
            kr, ks, kt, kb, cohesion, tCutoff, cCutoff, fAngle, beta1, beta2))))

    def add_brittle_beam_sc_group(self, name, tag, kr, ks, kt, kb, cohesion, tCutoff, fAngle):
        self._chk(self.lib.dem_add_brittle_beam_sc_group(self.h, name.encode(), int(tag), *(float(x) for x in (
            kr, ks, kt, kb, cohesion, tCutoff, fAngle))))

    def add_hertz_mindlin_visco_group(self, name, E, nu, mu, COR, dt):
        self._chk(self.lib.dem_add_hertz_mindlin_visco_group(self.h, name.encode(), float(E), float(nu), float(mu),
                                                             float(COR), float(dt)))

    def add_local_damping(self, name, rot, visc):
        self._chk(self.lib.dem_add_local_damping(self.h, name.encode(), int(rot), float(visc)))

    def add_nrot_friction_group(self, name, k, mu, k_s, dt, scaling=True):
        self._chk(self.lib.dem_add_nrot_friction_group(self.h, name.encode(), float(k), float(mu), float(k_s),
                                                       float(dt), int(scaling)))
        self._dyn_prm[name] = (2, [float(k), float(k_s)])

    def add_nrot_bond_group(self, name, tag, k, rbreak, scaling=True):
        self._chk(self.lib.dem_add_nrot_bond_group(self.h, name.encode(), int(tag), float(k), float(rbreak),
                                                   int(scaling)))
        self._bond_prm[name] = [float(k), 0.0, 0.0, 0.0]

    def add_rot_bond_group(self, name, tag, kr, ks, kt, kb, max_n, max_s, max_t, max_b, scaling=True,
                           meanR_scaling=True, truncated=1.0):
        self._chk(self.lib.dem_add_rot_bond_group(self.h, name.encode(), int(tag), float(kr), float(ks), float(kt),
                                                  float(kb), float(max_n), float(max_s), float(max_t), float(max_b),
                                                  int(scaling), int(meanR_scaling), float(truncated)))
        self._bond_prm[name] = [float(kr), float(ks), float(kt), float(kb)]

    def add_wall_group(self, name, wall, k):
        self._chk(self.lib.dem_add_wall_group(self.h, name.encode(), wall.encode(), float(k)))
        self.wall_groups = sorted(set(self.wall_groups) | {name})

    def add_gravity(self, name, g):
        self._chk(self.lib.dem_add_gravity(self.h, name.encode(), _dp(_v3(g))))

    def add_damping(self, rot, visc, max_iter=100):
        self._chk(self.lib.dem_add_damping(self.h, int(rot), float(visc), int(max_iter)))
        self._damp_prm["RotDamping" if rot else "Damping"] = float(visc)

    def add_exclusion(self, bonded, dynamic):
        self._chk(self.lib.dem_add_exclusion(self.h, bonded.encode(), dynamic.encode()))

    def set_timestep(self, dt):
        self._chk(self.lib.dem_set_timestep(self.h, float(dt)))

    def step(self, n=1):
        self._chk(self.lib.dem_step(self.h, int(n)))

    def move_wall(self, name, d):
        self._chk(self.lib.dem_move_wall(self.h, name.encode(), _dp(_v3(d))))

    def set_wall_velocity(self, name, v):
        self._chk(self.lib.dem_set_wall_velocity(self.h, name.encode(), _dp(_v3(v))))

    def apply_force_to_wall(self, group, force):
        self._chk(self.lib.dem_apply_force_to_wall(self.h, group.encode(), _dp(_v3(force))))

    def move_tagged(self, tag, d, mask=-1):
        self._chk(self.lib.dem_move_tagged(self.h, int(tag), int(mask), _dp(_v3(d))))

    def set_option(self, key, value):
        self._chk(self.lib.dem_set_option(self.h, key.encode(), float(value)))

    def set_particles(self, pos=None, vel=None, angvel=None, quat=None, id=None, n=None):
        """Bulk state update.  Arrays may be numpy arrays or raw host pointers (int) of
        n rows; with id=None row i is particle slot i."""
        def ptr(x, t):
            if x is None:
                return None
            if isinstance(x, int):
                return C.cast(C.c_void_p(x), t)
            return np.ascontiguousarray(x).ctypes.data_as(t)
        keep = [np.ascontiguousarray(x) for x in (pos, vel, angvel, quat, id) if x is not None and not isinstance(x, int)]
        if n is None:
            n = len(keep[0]) if keep else 0
        self._chk(self.lib.dem_set_particles(self.h, int(n), ptr(id, _I), ptr(pos, _D), ptr(vel, _D),
                                             ptr(angvel, _D), ptr(quat, _D)))
        del keep

    def revive_particles(self, id, pos=None, vel=None, angvel=None, quat=None):
        """Particles deleted when they left this worker's grid come back with this state
        (dem_revive_particles; the ghosts of a slab decomposition)."""
        id = np.ascontiguousarray(id, dtype=np.int32)
        keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (pos, vel, angvel, quat)]
        self._chk(self.lib.dem_revive_particles(self.h, len(id), _ip(id), *(_dp(a) for a in keep)))

    def set_pair_states(self, group, id1, id2, state):
        """Tangential history of existing pairs of a dynamic group (dem_set_pair_states); returns
        the pairs written."""
        a = np.ascontiguousarray(id1, dtype=np.int32)
        b = np.ascontiguousarray(id2, dtype=np.int32)
        st = np.ascontiguousarray(np.asarray(state, np.float64).reshape(-1, 5))
        return self._chk(self.lib.dem_set_pair_states(self.h, group.encode(), len(a), _ip(a), _ip(b), _dp(st)))

    def set_stream(self, stream_handle: int):
        self._chk(self.lib.dem_set_stream(self.h, C.c_void_p(int(stream_handle))))

    def counters(self):
        out = (C.c_longlong * 9)()
        self._chk(self.lib.dem_get_counters(self.h, out, 9))
        keys = ("steps", "contact_updates", "rebuilds", "launches", "step_kernel_ns", "profiled_steps",
                "contacts_per_step", "threads_per_particle", "search_due")
        return dict(zip(keys, list(out)))

    def get_particles_raw(self, id_ptr, pos_ptr, vel_ptr, angvel_ptr, quat_ptr, force_ptr, moment_ptr):
        """dem_get_particles into caller-owned host buffers given as raw pointers (0 = skip)."""
        cv = lambda p, t: None if not p else C.cast(C.c_void_p(p), t)
        return self._chk(self.lib.dem_get_particles(self.h, cv(id_ptr, _I), cv(pos_ptr, _D), cv(vel_ptr, _D),
                                                    cv(angvel_ptr, _D), cv(quat_ptr, _D), cv(force_ptr, _D),
                                                    cv(moment_ptr, _D)))

    def wall(self, name):
        p, f = np.zeros(3), np.zeros(3)
        self._chk(self.lib.dem_get_wall(self.h, name.encode(), _dp(p), _dp(f)))
        return p, f

    def num_particles(self):
        return self._chk(self.lib.dem_num_particles(self.h))

    def particles(self, sort=True):
        n = self.num_particles()
        out = {"id": np.zeros(n, np.int32)}
        for k, w in (("pos", 3), ("vel", 3), ("angvel", 3), ("quat", 4), ("force", 3), ("moment", 3)):
            out[k] = np.zeros((n, w))
        self._chk(self.lib.dem_get_particles(self.h, _ip(out["id"]), _dp(out["pos"]), _dp(out["vel"]),
                                             _dp(out["angvel"]), _dp(out["quat"]), _dp(out["force"]),
                                             _dp(out["moment"])))
        if not sort:
            return out
        order = np.argsort(out["id"], kind="stable")
        return {k: v[order] for k, v in out.items()}

    def pairs(self, group):
        n = self._chk(self.lib.dem_num_pairs(self.h, group.encode()))
        a, b = np.zeros(n, np.int32), np.zeros(n, np.int32)
        st = np.zeros((n, 5))
        m = self._chk(self.lib.dem_get_pairs(self.h, group.encode(), _ip(a), _ip(b), _dp(st)))
        a, b, st = a[:m], b[:m], st[:m]
        order = np.lexsort((b, a))
        return a[order], b[order], st[order]

    def breaks(self):
        n = self._chk(self.lib.dem_num_breaks(self.h))
        a, b, s = (np.zeros(n, np.int32) for _ in range(3))
        self._chk(self.lib.dem_get_breaks(self.h, _ip(a), _ip(b), _ip(s)))
        order = np.lexsort((b, a, s))
        return a[order], b[order], s[order]

    @property
    def timestep(self):
        return int(self.lib.dem_timestep(self.h))

    def particle_scalar_field(self, field, sort=True):
        """(ids, values) of a particle scalar field (dem_particle_scalar_field), by id when sort."""
        n = self.num_particles()
        v = np.zeros(max(n, 1))
        self._chk(self.lib.dem_particle_scalar_field(self.h, field.encode(), _dp(v)))
        ids = np.zeros(max(n, 1), np.int32)
        self._chk(self.lib.dem_get_particles(self.h, _ip(ids), None, None, None, None, None, None))
        ids, v = ids[:n], v[:n]
        if sort:
            o = np.argsort(ids, kind="stable")
            return ids[o], v[o]
        return ids, v

    def particle_vector_field(self, field, sort=True):
        """(ids, values n x 3) of a particle vector field (dem_particle_vector_field), by id when sort."""
        n = self.num_particles()
        v = np.zeros((max(n, 1), 3))
        self._chk(self.lib.dem_particle_vector_field(self.h, field.encode(), _dp(v)))
        ids = np.zeros(max(n, 1), np.int32)
        self._chk(self.lib.dem_get_particles(self.h, _ip(ids), None, None, None, None, None, None))
        ids, v = ids[:n], v[:n]
        if sort:
            o = np.argsort(ids, kind="stable")
            return ids[o], v[o]
        return ids, v

    def interaction_scalar_field(self, group, field):
        """(id1, id2, values) of an interaction scalar field of one group, in the group's list
        order (dem_get_pairs order)."""
        m = self._chk(self.lib.dem_num_pairs(self.h, group.encode()))
        a, b = np.zeros(max(m, 1), np.int32), np.zeros(max(m, 1), np.int32)
        k = self._chk(self.lib.dem_get_pairs(self.h, group.encode(), _ip(a), _ip(b), None))
        v = np.zeros(max(m, 1))
        kv = self._chk(self.lib.dem_interaction_scalar_field(self.h, group.encode(), field.encode(), _dp(v)))
        if kv != k:
            raise DemError("interaction list changed between calls")
        return a[:k], b[:k], v[:k]

    def precision_report(self):
        """FP32-force error vs FP64 on the current state (dem_precision_report); run from the
        FP64 form."""
        out = (C.c_double * 7)()
        self._chk(self.lib.dem_precision_report(self.h, out, 7))
        keys = ("max_rel_force_err", "max_rel_moment_err", "median_particle_rel_err", "p99_particle_rel_err",
                "particles", "rel_to_force_scale", "worst_rel_to_own_scale")
        return dict(zip(keys, list(out)))

    # ---- parameters and the differentiable loading window ----
    def set_group_param(self, group, key, value):
        """dem_set_group_param: one unscaled parameter of an existing group."""
        self._chk(self.lib.dem_set_group_param(self.h, group.encode(), key.encode(), float(value)))
        for slot, (g, k) in enumerate(self.param_layout()):
            if g == group and k == key:
                self._set_param_value(slot, float(value))

    _BOND_KEYS = ("normalK", "shearK", "torsionK", "bendingK")

    def param_layout(self):
        """(group, key) of each dem_window_adjoint parameter gradient, in the library's
        order; key None marks a slot without a parameter (the elastic law has no shearK,
        and an absent damping group has no viscosity)."""
        out = [(g, k) for g in sorted(self._bond_prm) for k in self._BOND_KEYS]
        for g in sorted(self._dyn_prm):
            out += [(g, "normalK"), (g, "shearK" if self._dyn_prm[g][0] == 1 else None)]
        out += [("Damping", "viscosity" if "Damping" in self._damp_prm else None),
                ("RotDamping", "viscosity" if "RotDamping" in self._damp_prm else None)]
        return out

    def param_values(self):
        vals = [v for g in sorted(self._bond_prm) for v in self._bond_prm[g]]
        for g in sorted(self._dyn_prm):
            vals += list(self._dyn_prm[g][1])
        vals += [self._damp_prm.get("Damping", 0.0), self._damp_prm.get("RotDamping", 0.0)]
        return np.array(vals, dtype=np.float64)

    def _set_param_value(self, slot, value):
        nb = 4 * len(self._bond_prm)
        if slot < nb:
            self._bond_prm[sorted(self._bond_prm)[slot // 4]][slot % 4] = value
            return
        slot -= nb
        nd = 2 * len(self._dyn_prm)
        if slot < nd:
            self._dyn_prm[sorted(self._dyn_prm)[slot // 2]][1][slot % 2] = value
            return
        self._damp_prm[("Damping", "RotDamping")[slot - nd]] = value

    def set_params(self, values):
        """Apply a full parameter vector in param_layout() order."""
        for (g, k), v in zip(self.param_layout(), np.asarray(values, dtype=np.float64)):
            if k is not None:
                self.set_group_param(g, k, v)

    def window_num_params(self):
        return self._chk(self.lib.dem_window_num_params(self.h))

    def window_forward(self, nsteps, checkpoint_every=100):
        """Run a differentiable window; returns the wall-group reactions [nsteps, groups, 3]."""
        r = np.zeros((int(nsteps), len(self.wall_groups), 3))
        self._chk(self.lib.dem_window_forward(self.h, int(nsteps), int(checkpoint_every), _dp(r)))
        return r

    def window_adjoint(self, grad_reactions):
        """Reverse pass of the last window.  Returns the parameter gradients
        (dem_window_num_params values) and dLoss/d(initial pos, vel, angvel, quat) rows
        sorted by particle id, with the ids."""
        g = np.ascontiguousarray(grad_reactions, dtype=np.float64)
        n = self.num_particles()
        out = {"params": np.zeros(self.window_num_params()), "id": np.zeros(n, np.int32)}
        for k, w in (("pos", 3), ("vel", 3), ("angvel", 3), ("quat", 4)):
            out[k] = np.zeros((n, w))
        self._chk(self.lib.dem_window_adjoint(self.h, _dp(g), _dp(out["params"]), _dp(out["vel"]),
                                              _dp(out["angvel"]), _dp(out["pos"]), _dp(out["quat"])))
        self._chk(self.lib.dem_get_particles(self.h, _ip(out["id"]), None, None, None, None, None, None))
        order = np.argsort(out["id"], kind="stable")
        for k in ("id", "pos", "vel", "angvel", "quat"):
            out[k] = out[k][order]
        return out

    def window_rewind(self):
        self._chk(self.lib.dem_window_rewind(self.h))

    def window_release(self):
        """Free the last window's checkpoints and reverse-pass buffers."""
        self._chk(self.lib.dem_window_release(self.h))

    def save_checkpoint(self, path, precision=12):
        """Write the worker file of a restart checkpoint (dem_save_checkpoint)."""
        self._chk(self.lib.dem_save_checkpoint(self.h, os.fsencode(path), int(precision)))

    def save_snapshot(self, path):
        """Write the worker file of a snapshot (dem_save_snapshot)."""
        self._chk(self.lib.dem_save_snapshot(self.h, os.fsencode(path)))

    def load_checkpoint(self, path, timestep):
        """Read a worker file into this (particle-less) worker and set its step counter."""
        self._chk(self.lib.dem_load_checkpoint(self.h, os.fsencode(path), int(timestep)))

    def search_neighbors(self):
        """Neighbour search and interaction update at the head of the next step (force-neutral;
        restarts the verletDist/2 displacement budget)."""
        self._chk(self.lib.dem_search_neighbors(self.h))


class Ensemble:
    """Many independent workers advanced together (dem_ensemble_*): one kernel launch per
    timestep for all specimens, chunks replayed from a captured CUDA graph.  Each specimen
    advances exactly as its own ``step`` would advance it.  Keeps references to the member
    ``DemSim`` objects so that they outlive it."""

    def __init__(self, sims):
        self.sims = list(sims)
        if not self.sims:
            raise DemError("an ensemble needs at least one specimen")
        self.lib = self.sims[0].lib
        self.h = _P()
        arr = (_P * len(self.sims))(*[x.h for x in self.sims])
        rc = self.lib.dem_ensemble_create(C.byref(self.h), arr, len(self.sims))
        if rc != 0:
            raise DemError(f"dem_ensemble_create failed ({rc}): specimens must share particle type")

    def _chk(self, rc):
        if rc < 0:
            raise DemError(self.lib.dem_ensemble_last_error(self.h).decode(), rc)
        return rc

    def step(self, n=1):
        self._chk(self.lib.dem_ensemble_step(self.h, int(n)))

    def set_option(self, key, value):
        self._chk(self.lib.dem_ensemble_set_option(self.h, key.encode(), float(value)))

    @staticmethod
    def _ptrs(arrays):
        return (_D * len(arrays))(*[_dp(a) for a in arrays])

    def window_forward(self, nsteps, checkpoint_every=100):
        """Every specimen's differentiable window (dem_ensemble_window_forward); returns each
        specimen's wall-group reactions [nsteps, groups, 3]."""
        R = [np.zeros((int(nsteps), len(x.wall_groups), 3)) for x in self.sims]
        self._chk(self.lib.dem_ensemble_window_forward(self.h, int(nsteps), int(checkpoint_every), self._ptrs(R)))
        return R

    def window_adjoint(self, grad_reactions):
        """Batched reverse pass (dem_ensemble_window_adjoint).  Returns per specimen the
        parameter gradients and dLoss/d(initial vel, angvel), rows sorted by particle id."""
        g = [np.ascontiguousarray(x, dtype=np.float64) for x in grad_reactions]
        if len(g) != len(self.sims):
            raise DemError("one reaction gradient per specimen")
        outs = []
        for x in self.sims:
            n = x.num_particles()
            outs.append({"params": np.zeros(x.window_num_params()), "vel": np.zeros((n, 3)),
                         "angvel": np.zeros((n, 3))})
        self._chk(self.lib.dem_ensemble_window_adjoint(
            self.h, self._ptrs(g), self._ptrs([o["params"] for o in outs]), self._ptrs([o["vel"] for o in outs]),
            self._ptrs([o["angvel"] for o in outs])))
        for x, o in zip(self.sims, outs):
            ids = np.zeros(x.num_particles(), np.int32)
            x._chk(x.lib.dem_get_particles(x.h, _ip(ids), None, None, None, None, None, None))
            order = np.argsort(ids, kind="stable")
            o["id"] = ids[order]
            o["vel"] = o["vel"][order]
            o["angvel"] = o["angvel"][order]
        return outs

    def counters(self):
        out = (C.c_longlong * 8)()
        self._chk(self.lib.dem_ensemble_get_counters(self.h, out, 8))
        keys = ("specimen_steps", "contact_updates", "launches", "chunks", "step_kernel_ns", "profiled_steps",
                "threads_per_particle", "rebuild_requests")
        return dict(zip(keys, list(out)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.dem_ensemble_destroy(self.h)
            self.h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
