"""Field savers: the reference's *FieldSaverPrms and the files they write.

Values are computed on the GPU (dem_particle_scalar_field, dem_interaction_scalar_field,
dem_get_wall) and written in the reference's formats (Fields/FieldMaster.cpp and the
ParticleFieldMaster / InteractionFieldMaster / WallFieldMaster writers):

  particle scalar    SUM, MAX: one line per save, C++ default stream format (%g);
                     RAW_SERIES: one row per save, values in particle-id order, each + two spaces;
                     RAW_WITH_POS_ID: one file per save, "id x y z radius value" lines by id
                     (ScalarParticleFieldMaster::writeAsRawWithPosID, ParticleFieldMaster.cpp:363-380)
  particle vector    SUM (component sums), MAX (the vector of largest norm), RAW_SERIES ("x y z" +
                     two spaces per particle), RAW2 (one file per save, "x y z vx vy vz" lines) and
                     RAW_WITH_ID ("id x y z vx vy vz"), all by id and in %g
                     (VectorParticleFieldMaster, ParticleFieldMaster.cpp:561-680)
  interaction scalar SUM: one line per save, scientific with 10 digits; MAX: %g
  wall vector        RAW_SERIES: one row per save, "x y z" per wall in the given order, each +
                     two spaces, scientific with 10 digits

The one-file-per-save formats name their files <fileName>.<k * timeStepIncr>.dat for the k-th
save of the saver, k counted from 0 (AFieldMaster::makeFilename, Fields/FieldMaster.cpp:100-126).
The tagged savers keep the particles whose tag satisfies (tag & mask) == (saver tag & mask)
(ParallelParticleArray::forAllInnerTaggedParticlesGetIndexed, ppa/src/pp_array.hpp:1035-1050).

A saver writes at timestep t when t >= beginTimeStep, t <= endTimeStep and
(t - beginTimeStep) % timeStepIncr == 0 (AFieldMaster::needSave), after the step's
integration, and once at t = 0 before the first step.  Sums run in the reference's
order: particles by id, interactions in list order.
"""
from __future__ import annotations

import numpy as np

__all__ = ["ParticleScalarFieldSaverPrms", "ParticleVectorFieldSaverPrms", "TaggedParticleScalarFieldSaverPrms",
           "TaggedParticleVectorFieldSaverPrms", "InteractionScalarFieldSaverPrms", "WallVectorFieldSaverPrms",
           "FieldSaver"]


class _SaverPrms:
    def __init__(self, fieldName, fileName, fileFormat, beginTimeStep, endTimeStep, timeStepIncr):
        self.fieldName, self.fileName, self.fileFormat = fieldName, fileName, fileFormat
        self.beginTimeStep, self.endTimeStep, self.timeStepIncr = int(beginTimeStep), int(endTimeStep), int(timeStepIncr)


class ParticleScalarFieldSaverPrms(_SaverPrms):  # Python/esys/lsm/ParticleFieldSaverPrmsPy.cpp
    FORMATS = ("SUM", "MAX", "RAW_SERIES", "RAW_WITH_POS_ID")


class ParticleVectorFieldSaverPrms(_SaverPrms):  # ParticleFieldSaverPrmsPy.cpp:60-77
    FORMATS = ("SUM", "MAX", "RAW_SERIES", "RAW2", "RAW_WITH_ID")


class TaggedParticleScalarFieldSaverPrms(ParticleScalarFieldSaverPrms):  # ParticleFieldSaverPrmsPy.cpp:79-97
    def __init__(self, fieldName, fileName, fileFormat, beginTimeStep, endTimeStep, timeStepIncr, tag, mask):
        super().__init__(fieldName, fileName, fileFormat, beginTimeStep, endTimeStep, timeStepIncr)
        self.tag, self.mask = int(tag), int(mask)


class TaggedParticleVectorFieldSaverPrms(ParticleVectorFieldSaverPrms):  # ParticleFieldSaverPrmsPy.cpp:99-117
    def __init__(self, fieldName, fileName, fileFormat, beginTimeStep, endTimeStep, timeStepIncr, tag, mask):
        super().__init__(fieldName, fileName, fileFormat, beginTimeStep, endTimeStep, timeStepIncr)
        self.tag, self.mask = int(tag), int(mask)


class InteractionScalarFieldSaverPrms(_SaverPrms):  # Python/esys/lsm/InteractionFieldSaverPrmsPy.cpp
    FORMATS = ("SUM", "MAX")

    def __init__(self, interactionName, fieldName, fileName, fileFormat, beginTimeStep, endTimeStep, timeStepIncr):
        super().__init__(fieldName, fileName, fileFormat, beginTimeStep, endTimeStep, timeStepIncr)
        self.interactionName = interactionName


class WallVectorFieldSaverPrms(_SaverPrms):  # Python/esys/lsm/WallFieldSaverPrmsPy.cpp
    FORMATS = ("RAW_SERIES",)

    def __init__(self, wallName, fieldName, fileName, fileFormat, beginTimeStep, endTimeStep, timeStepIncr):
        super().__init__(fieldName, fileName, fileFormat, beginTimeStep, endTimeStep, timeStepIncr)
        self.wallName = [wallName] if isinstance(wallName, str) else list(wallName)


def _g(x):
    """C++ default stream output of a double (precision 6, %g)."""
    return "%g" % x


def _v3(v):
    """Vec3's stream output: the three components in %g, one space apart."""
    return f"{_g(v[0])} {_g(v[1])} {_g(v[2])}"


def _e10(x):
    """C++ scientific output with precision 10."""
    return "%.10e" % x


class FieldSaver:
    def __init__(self, prms):
        if prms.fileFormat not in type(prms).FORMATS:
            raise NotImplementedError(f"{type(prms).__name__} format {prms.fileFormat!r} is not provided "
                                      f"(available: {', '.join(type(prms).FORMATS)})")
        if prms.timeStepIncr < 1:
            raise ValueError("timeStepIncr must be >= 1")
        self.p = prms
        self.count = 0  # saves written (AFieldMaster::m_save_count)

    def need_save(self, t):
        p = self.p
        return (t - p.beginTimeStep) % p.timeStepIncr == 0 and p.beginTimeStep <= t <= p.endTimeStep

    def next_save(self, t):
        """First save step > t, or None."""
        p = self.p
        if t < p.beginTimeStep:
            nxt = p.beginTimeStep
        else:
            nxt = p.beginTimeStep + ((t - p.beginTimeStep) // p.timeStepIncr + 1) * p.timeStepIncr
        return nxt if nxt <= p.endTimeStep else None

    def _file_name(self):
        name = f"{self.p.fileName}.{self.count * self.p.timeStepIncr}.dat"
        self.count += 1
        return name

    def _tagged(self, sim, ids):
        """Mask of the particles a tagged saver keeps (all for an untagged one), ids sorted."""
        p = self.p
        if not hasattr(p, "mask"):
            return np.ones(len(ids), bool)
        _, tags = sim.particle_scalar_field("tag", sort=True)
        tags = tags.astype(np.int64)
        return (tags & p.mask) == (p.tag & p.mask)

    def save(self, sim):
        p = self.p
        if isinstance(p, ParticleScalarFieldSaverPrms):
            ids, v = sim.particle_scalar_field(p.fieldName, sort=True)
            keep = self._tagged(sim, ids)
            ids, v = ids[keep], v[keep]
            if p.fileFormat == "RAW_WITH_POS_ID":
                _, x = sim.particle_vector_field("position", sort=True)
                _, r = sim.particle_scalar_field("radius", sort=True)
                x, r = x[keep], r[keep]
                with open(self._file_name(), "w") as f:
                    f.write("".join(f"{int(i)} {_v3(xi)} {_g(ri)} {_g(vi)}\n" for i, xi, ri, vi in zip(ids, x, r, v)))
                return
            if p.fileFormat == "SUM":
                line = _g(_ordered_sum(v))
            elif p.fileFormat == "MAX":
                line = _g(float(v.max()) if len(v) else 0.0)
            else:
                line = "".join(_g(x) + "  " for x in v)
        elif isinstance(p, ParticleVectorFieldSaverPrms):
            ids, v = sim.particle_vector_field(p.fieldName, sort=True)
            keep = self._tagged(sim, ids)
            ids, v = ids[keep], v[keep]
            if p.fileFormat in ("RAW2", "RAW_WITH_ID"):
                _, x = sim.particle_vector_field("position", sort=True)
                x = x[keep]
                pre = (lambda i: f"{int(i)} ") if p.fileFormat == "RAW_WITH_ID" else (lambda i: "")
                with open(self._file_name(), "w") as f:
                    f.write("".join(f"{pre(i)}{_v3(xi)} {_v3(vi)}\n" for i, xi, vi in zip(ids, x, v)))
                return
            if p.fileFormat == "SUM":
                line = _v3([_ordered_sum(v[:, c]) for c in range(3)])
            elif p.fileFormat == "MAX":  # the first of largest norm2 (strict >)
                best = v[0] if len(v) else np.zeros(3)
                bn = float(best @ best)
                for row in v:
                    n2 = row[0] * row[0] + row[1] * row[1] + row[2] * row[2]
                    if n2 > bn:
                        best, bn = row, n2
                line = _v3(best)
            else:
                line = "".join(_v3(x) + "  " for x in v)
        elif isinstance(p, InteractionScalarFieldSaverPrms):
            _, _, v = sim.interaction_scalar_field(p.interactionName, p.fieldName)
            if p.fileFormat == "SUM":
                line = _e10(_ordered_sum(v))
            else:
                line = _g(float(v.max()) if len(v) else 0.0)
        else:
            parts = []
            for w in p.wallName:
                pos, force = sim.wall(w)
                vec = pos if p.fieldName == "Position" else force
                if p.fieldName not in ("Position", "Force"):
                    raise NotImplementedError(f"wall field {p.fieldName!r}")
                parts.append(" ".join(_e10(x) for x in vec) + "  ")
            line = "".join(parts)
        with open(p.fileName, "a") as f:
            f.write(line + "\n")


def _ordered_sum(v):
    """Left-to-right double sum (the reference's loop order)."""
    s = 0.0
    for x in np.asarray(v, dtype=np.float64).tolist():
        s += x
    return s
