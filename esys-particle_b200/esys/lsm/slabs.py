"""Slab decomposition of one specimen over several workers (one per rank or GPU).

The reference splits its cell grid among MPI workers (ParallelParticleArray's domain
decomposition, ppa/src/pp_array.hpp:55-100): each worker holds its slab of cells plus one
layer of ghost cells copied from its neighbours, computes the forces on its own particles,
exchanges the ghosts' positions after every step (TSubLattice::exchangePos,
Parallel/SubLattice.hpp:2053-2060) and re-sends the ghost layers, moving particles between
workers, at every neighbour rebuild (pp_array.hpp:433-554).

Here the split is along one non-periodic axis (the longest by default) into slabs of whole
grid cells, one worker engine per slab.  A worker engine is an ordinary single-worker
simulation (the GPU library's handle, or a CPU oracle in tests) whose box is its slab: the
engine's padding layer of one cell beyond each slab face is where its ghost particles live, so
that, as in the reference, ghosts take part in the pair search and the forces of the slab's own
particles, are left out of the wall reactions (they are not in the inner region) and are
overwritten by their owners' state after every step.  A pair with a particle of the slab has its
other particle within one cell of it, hence within the ghost layer (gridSpacing is at least the
largest pair distance).

Ownership changes only at a repartition, which follows every neighbour rebuild of any worker
(a worker rebuilds once one of its particles has moved verletDist/2, so no particle moves more
than that between repartitions).  A particle that crossed a slab face is already a ghost of the
slab it entered (it was within one cell of the face), together with its pairs there; it moves
with the tangential history of its pairs from its old slab (the receiving slab may have started a
pair of two of its ghosts after it formed), as the reference moves interaction records with
particles.  A particle that newly enters a ghost layer cannot yet touch any particle of that
slab, so no other history moves.  Bonds need nothing: a bond is shorter than a cell, so a bond
across a slab face has both its particles in both slabs from the start.  The groups whose
history moves are named by `history_groups` (RotFriction and the other history laws).

The per-step exchange sends, for each slab face, the state (position, velocity, spin,
quaternion: 13 doubles) of the owner's particles in its neighbour's ghost layer.  Transports:
``TorchTransport`` over a ``torch.distributed`` process group (gloo on CPU ranks, NCCL between
GPUs: the payload goes through host arrays here), and in-process workers driven by
``SlabDomain`` for several engines in one process.
"""
from __future__ import annotations

import numpy as np

__all__ = ["SlabLayout", "SlabWorker", "SlabDomain", "TorchTransport"]

STATE_COLS = 13  # pos 3, vel 3, angvel 3, quat 4


class SlabLayout:
    """Slab bounds along `axis`: whole cells of size `grid_spacing` from bbox_min, split as
    evenly as possible among `world` slabs of at least two cells each."""

    def __init__(self, bbox_min, bbox_max, grid_spacing, world, axis=None, circ=(0, 0, 0)):
        lo, hi = np.asarray(bbox_min, float), np.asarray(bbox_max, float)
        L = hi - lo
        if axis is None:
            order = [int(a) for a in np.argsort(-L, kind="stable") if not circ[int(a)]]
            if not order:
                raise ValueError("no non-periodic axis to split along")
            axis = order[0]
        if circ[axis]:
            raise ValueError("slabs are split along a non-periodic axis")
        ncell = int(np.floor(L[axis] / grid_spacing + 1e-9))
        if ncell < 2 * world:
            raise ValueError(f"{ncell} cells along axis {axis} cannot give {world} slabs of two cells")
        counts = [ncell // world + (1 if r < ncell % world else 0) for r in range(world)]
        edges = [lo[axis]]
        for c in counts:
            edges.append(edges[-1] + c * grid_spacing)
        edges[-1] = hi[axis]  # the last slab takes the remainder of the box
        self.axis, self.world, self.gs = axis, world, float(grid_spacing)
        self.edges = np.array(edges)
        self.bbox_min, self.bbox_max = lo, hi

    def owner(self, x):
        """Slab of each coordinate along the axis (clamped to the box's slabs)."""
        r = np.searchsorted(self.edges, np.asarray(x, float), side="right") - 1
        return np.clip(r, 0, self.world - 1)

    def box(self, rank):
        lo, hi = self.bbox_min.copy(), self.bbox_max.copy()
        lo[self.axis], hi[self.axis] = self.edges[rank], self.edges[rank + 1]
        return lo, hi


class TorchTransport:
    """Neighbour exchange and reductions over a torch.distributed process group: arrays go as
    float64 tensors (on the CUDA device for NCCL, host for gloo), sizes first."""

    def __init__(self, dist, device="cpu"):
        self.dist, self.device = dist, device
        self.rank, self.world = dist.get_rank(), dist.get_world_size()

    def exchange(self, out_prev, out_next):
        """Send arrays to rank - 1 and rank + 1 (None at a domain end); returns what they sent."""
        import torch

        d = self.dist
        res = [None, None]
        for peer, out, slot in ((self.rank - 1, out_prev, 0), (self.rank + 1, out_next, 1)):
            if not (0 <= peer < self.world):
                continue
            n = torch.tensor([0 if out is None else out.size], dtype=torch.int64, device=self.device)
            m = torch.zeros(1, dtype=torch.int64, device=self.device)
            for r in d.batch_isend_irecv([d.P2POp(d.isend, n, peer), d.P2POp(d.irecv, m, peer)]):
                r.wait()
            sbuf = torch.as_tensor(np.zeros(0) if out is None else np.ascontiguousarray(out, np.float64).ravel(),
                                   device=self.device)
            rbuf = torch.zeros(int(m.item()), dtype=torch.float64, device=self.device)
            ops = []
            if sbuf.numel():
                ops.append(d.P2POp(d.isend, sbuf, peer))
            if rbuf.numel():
                ops.append(d.P2POp(d.irecv, rbuf, peer))
            if ops:
                for r in d.batch_isend_irecv(ops):
                    r.wait()
            res[slot] = rbuf.cpu().numpy()
        return res[0], res[1]

    def any(self, flag):
        import torch

        t = torch.tensor([1 if flag else 0], dtype=torch.int64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return bool(t.item())

    def sum(self, arr):
        import torch

        t = torch.as_tensor(np.asarray(arr, np.float64), device=self.device).clone()
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return t.cpu().numpy()

    def gather(self, obj):
        out = [None] * self.world
        self.dist.all_gather_object(out, obj)
        return out


def _pack(ids, st):
    """Rows (id, 13 state doubles) as one float64 array (ids are exact in float64)."""
    return np.concatenate([np.asarray(ids, np.float64)[:, None], st], axis=1).ravel()


def _unpack(buf):
    if buf is None or buf.size == 0:
        return np.zeros(0, np.int32), np.zeros((0, STATE_COLS))
    a = buf.reshape(-1, 1 + STATE_COLS)
    return a[:, 0].astype(np.int32), a[:, 1:]


class SlabWorker:
    """One slab's worker: its engine, the ids it owns and the ids it exports to each neighbour.

    make(particle_type, grid_spacing, verlet_dist, bbox_min, bbox_max, circ, dt) builds the
    engine; configure(engine) adds its groups and walls (everything but particles and
    connections), as for a single worker.  The particle and connection arrays are the whole
    specimen's (every rank keeps the static per-particle data: radius, mass, tag)."""

    def __init__(self, rank, layout, make, configure, particle_type, grid_spacing, verlet_dist, circ, dt,
                 particles, connections=None, history_groups=()):
        self.rank, self.L = rank, layout
        self.history_groups = list(history_groups)
        self._pending_states = []
        self.gs = float(grid_spacing)
        p = particles
        n = len(p["id"])
        self.static = {"id": np.asarray(p["id"], np.int32), "rad": np.asarray(p["rad"], float),
                       "mass": np.asarray(p["mass"], float),
                       "tag": np.asarray(p["tag"] if p.get("tag") is not None else np.zeros(n), np.int32)}
        self.row = {int(i): k for k, i in enumerate(self.static["id"])}
        lo, hi = layout.box(rank)
        self.engine = make(particle_type, grid_spacing, verlet_dist, lo, hi, circ, dt)
        x = np.asarray(p["pos"], float)[:, layout.axis]
        own = layout.owner(x) == rank
        e0, e1 = layout.edges[rank], layout.edges[rank + 1]
        ghost = ~own & (x >= e0 - self.gs) & (x < e1 + self.gs)
        rows = np.nonzero(own | ghost)[0]
        st = lambda k, w: None if p.get(k) is None else np.asarray(p[k], float).reshape(-1, w)[rows]
        self.engine.add_particles(self.static["id"][rows], np.asarray(p["pos"], float)[rows], self.static["rad"][rows],
                                  self.static["mass"][rows], tag=self.static["tag"][rows], vel=st("vel", 3),
                                  angvel=st("angvel", 3), quat=st("quat", 4))
        self.present = set(int(i) for i in self.static["id"][rows])
        if connections is not None and len(connections[1]):
            tags, a, b = (np.asarray(c) for c in connections)
            here = self.static["id"][rows]
            m = np.isin(a, here) & np.isin(b, here)
            if m.any():
                self.engine.add_connections(tags[m].astype(np.int32), a[m].astype(np.int32), b[m].astype(np.int32))
        configure(self.engine)
        self.owned = set(int(i) for i in self.static["id"][own])
        self.exports = [np.zeros(0, np.int32), np.zeros(0, np.int32)]

    # ---- state -------------------------------------------------------------------------
    def state(self, ids=None):
        """(ids, rows of 13 state doubles) of the alive particles, or of those of `ids` alive."""
        q = self.engine.particles()
        S = np.concatenate([q["pos"], q["vel"], q["angvel"], q["quat"]], axis=1)
        if ids is None:
            return q["id"], S
        ids = np.asarray(ids, np.int32)
        if len(q["id"]) == 0 or len(ids) == 0:
            return ids[:0], S[:0]
        pos = np.searchsorted(q["id"], ids)
        ok = (pos < len(q["id"])) & (q["id"][np.minimum(pos, len(q["id"]) - 1)] == ids)
        return ids[ok], S[pos[ok]]

    def apply(self, ids, S):
        """Ghost states from their owners: update or revive the known ones, add the others."""
        if len(ids) == 0:
            return
        new = np.array([int(i) not in self.present for i in ids], bool)
        old = ~new
        if old.any():
            self.engine.revive_particles(ids[old], pos=S[old, 0:3], vel=S[old, 3:6], angvel=S[old, 6:9],
                                         quat=S[old, 9:13])
        if new.any():
            r = np.array([self.row[int(i)] for i in ids[new]])
            self.engine.add_particles(ids[new], S[new, 0:3], self.static["rad"][r], self.static["mass"][r],
                                      tag=self.static["tag"][r], vel=S[new, 3:6], angvel=S[new, 6:9],
                                      quat=S[new, 9:13])
            self.present.update(int(i) for i in ids[new])

    def exports_for(self, ids, S):
        """Owned particles within one cell of each slab face: the neighbours' ghosts."""
        x = S[:, self.L.axis]
        mine = np.array([int(i) in self.owned for i in ids], bool)
        e0, e1 = self.L.edges[self.rank], self.L.edges[self.rank + 1]
        prev = mine & (x < e0 + self.gs) if self.rank > 0 else np.zeros(len(ids), bool)
        nxt = mine & (x >= e1 - self.gs) if self.rank < self.L.world - 1 else np.zeros(len(ids), bool)
        return ids[prev], ids[nxt]

    # ---- protocol phases -----------------------------------------------------------------
    def phase_step(self, n=1):
        before = self.engine.counters()["rebuilds"]
        self.engine.step(n)
        return self.engine.counters()["rebuilds"] != before

    def phase_export(self):
        out = []
        for ex in self.exports:
            ids, S = self.state(ex)
            out.append(_pack(ids, S) if len(ids) else None)
        return out[0], out[1]

    def phase_import(self, from_prev, from_next):
        for buf in (from_prev, from_next):
            ids, S = _unpack(buf)
            if len(ids):
                self.engine.set_particles(pos=S[:, 0:3], vel=S[:, 3:6], angvel=S[:, 6:9], quat=S[:, 9:13], id=ids)

    def phase_handover(self):
        """Owned particles that left the slab go to the neighbour slab they are in, with the
        tangential history of their pairs (this slab's copies, the exact ones: the receiving slab
        may have started a pair of two of its ghosts late)."""
        ids, S = self.state(np.array(sorted(self.owned), np.int32))
        dest = self.L.owner(S[:, self.L.axis])
        out = []
        pairs = [(gi,) + tuple(self.engine.pairs(g)) for gi, g in enumerate(self.history_groups)]
        for gone in (ids[dest < self.rank], ids[dest > self.rank]):
            self.owned.difference_update(int(i) for i in gone)
            rows = []
            for gi, a, b, st in pairs:
                m = np.isin(a, gone) | np.isin(b, gone)
                if m.any():
                    rows.append(np.concatenate([np.full((int(m.sum()), 1), gi, np.float64), a[m, None], b[m, None],
                                                st[m]], axis=1))
            rows = np.concatenate(rows) if rows else np.zeros((0, 8))
            out.append(np.concatenate([[len(gone)], np.asarray(gone, np.float64), rows.ravel()])
                       if len(gone) else None)
        return out[0], out[1]

    def phase_takeover(self, from_prev, from_next):
        for buf in (from_prev, from_next):
            if buf is None or buf.size == 0:
                continue
            k = int(buf[0])
            self.owned.update(int(i) for i in buf[1:1 + k].astype(np.int32))
            rows = buf[1 + k:].reshape(-1, 8)
            if len(rows):
                self._pending_states.append(rows)

    def phase_ghost_lists(self):
        """New export lists, sent with the particles' state (the receiver adds or revives)."""
        ids, S = self.state(np.array(sorted(self.owned), np.int32))
        prev, nxt = self.exports_for(ids, S)
        self.exports = [prev, nxt]
        out = []
        for ex in self.exports:
            i2, S2 = self.state(ex)
            out.append(_pack(i2, S2) if len(i2) else None)
        return out[0], out[1]

    def phase_ghost_apply(self, from_prev, from_next):
        for buf in (from_prev, from_next):
            ids, S = _unpack(buf)
            self.apply(ids, S)
        self.engine.search_neighbors()
        for rows in self._pending_states:  # histories of the particles taken over
            for gi, g in enumerate(self.history_groups):
                m = rows[:, 0] == gi
                if m.any():
                    self.engine.set_pair_states(g, rows[m, 1].astype(np.int32), rows[m, 2].astype(np.int32),
                                                rows[m, 3:8])
        self._pending_states = []


class SlabDomain:
    """A specimen split into `world` slabs.  With `transport` (one process per rank, e.g.
    TorchTransport) this process runs slab `transport.rank`; without, it runs every slab's
    engine itself (several engines on one device), exchanging in memory."""

    def __init__(self, make, configure, particle_type, grid_spacing, verlet_dist, bbox_min, bbox_max, circ, dt,
                 particles, connections=None, world=2, axis=None, transport=None, history_groups=()):
        self.tr = transport
        world = transport.world if transport is not None else world
        self.layout = SlabLayout(bbox_min, bbox_max, grid_spacing, world, axis, circ)
        ranks = [transport.rank] if transport is not None else range(world)
        self.workers = [SlabWorker(r, self.layout, make, configure, particle_type, grid_spacing, verlet_dist, circ,
                                   dt, particles, connections, history_groups) for r in ranks]
        self.repartitions = 0
        self._repartition()

    # exchanges: every worker's (to_prev, to_next) -> every worker's (from_prev, from_next)
    def _xchg(self, outs):
        if self.tr is not None:
            return [self.tr.exchange(*outs[0])]
        W = len(self.workers)
        return [(outs[r - 1][1] if r > 0 else None, outs[r + 1][0] if r < W - 1 else None) for r in range(W)]

    def _any(self, flags):
        return self.tr.any(any(flags)) if self.tr is not None else any(flags)

    def _repartition(self):
        ins = self._xchg([w.phase_handover() for w in self.workers])
        for w, (a, b) in zip(self.workers, ins):
            w.phase_takeover(a, b)
        ins = self._xchg([w.phase_ghost_lists() for w in self.workers])
        for w, (a, b) in zip(self.workers, ins):
            w.phase_ghost_apply(a, b)
        self.repartitions += 1

    def step(self, n=1):
        for _ in range(n):
            rebuilt = [w.phase_step(1) for w in self.workers]
            ins = self._xchg([w.phase_export() for w in self.workers])
            for w, (a, b) in zip(self.workers, ins):
                w.phase_import(a, b)
            if self._any(rebuilt):
                self._repartition()

    # ---- walls -----------------------------------------------------------------------------
    def move_wall(self, name, d):
        for w in self.workers:
            w.engine.move_wall(name, d)

    def set_wall_velocity(self, name, v):
        for w in self.workers:
            w.engine.set_wall_velocity(name, v)

    def wall_force(self, name):
        """The wall's reaction summed over slabs (each counts only its own particles)."""
        f = sum(np.asarray(w.engine.wall(name)[1], float) for w in self.workers)
        return self.tr.sum(f) if self.tr is not None else f

    def wall(self, name):
        """(origin, reaction) of a wall; the reaction summed over slabs."""
        return np.asarray(self.workers[0].engine.wall(name)[0], float), self.wall_force(name)

    # ---- results (gathered over ranks when a transport is given) ---------------------------
    def _gather(self, objs):
        if self.tr is None:
            return objs
        return [o for part in self.tr.gather(objs) for o in part]

    def particles(self):
        """The owned particles of every slab, sorted by id."""
        parts = []
        for w in self.workers:
            q = w.engine.particles()
            m = np.isin(q["id"], np.array(sorted(w.owned), np.int32))
            parts.append({k: v[m] for k, v in q.items()})
        parts = self._gather(parts)
        out = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
        o = np.argsort(out["id"], kind="stable")
        return {k: v[o] for k, v in out.items()}

    def pairs(self, group, touching_only=False):
        """Pairs with an owned first particle, each once (the copy of the slab owning it)."""
        rows = []
        for w in self.workers:
            a, b, st = w.engine.pairs(group)
            own = np.array([int(i) in w.owned for i in a], bool)
            if touching_only and len(st):
                own &= st[:, 4] > 0
            rows.append((a[own], b[own], st[own]))
        rows = self._gather(rows)
        a = np.concatenate([r[0] for r in rows])
        b = np.concatenate([r[1] for r in rows])
        st = np.concatenate([r[2] for r in rows])
        o = np.lexsort((b, a))
        return a[o], b[o], st[o]

    def breaks(self):
        """Bond-failure events (id1, id2, step), each once, in step order."""
        ev = set()
        for w in self.workers:
            ev.update(zip(*(x.tolist() for x in w.engine.breaks())))
        ev = set().union(*self._gather([ev]))
        return sorted(ev, key=lambda e: (e[2], e[0], e[1]))

    def close(self):
        for w in self.workers:
            if hasattr(w.engine, "close"):
                w.engine.close()
