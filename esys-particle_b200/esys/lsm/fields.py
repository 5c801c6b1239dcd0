"""Field savers: the reference's *FieldSaverPrms and the files they write.

Values are computed on the GPU (dem_particle_scalar_field, dem_interaction_scalar_field,
dem_get_wall) and written in the reference's formats (Fields/FieldMaster.cpp and the
ParticleFieldMaster / InteractionFieldMaster / WallFieldMaster writers):

  particle scalar    SUM, MAX: one line per save, C++ default stream format (%g);
                     RAW_SERIES: one row per save, values in particle-id order, each + two spaces
  interaction scalar SUM: one line per save, scientific with 10 digits; MAX: %g
  wall vector        RAW_SERIES: one row per save, "x y z" per wall in the given order, each +
                     two spaces, scientific with 10 digits

A saver writes at timestep t when t >= beginTimeStep, t <= endTimeStep and
(t - beginTimeStep) % timeStepIncr == 0 (AFieldMaster::needSave), after the step's
integration, and once at t = 0 before the first step.  Sums run in the reference's
order: particles by id, interactions in list order.
"""
from __future__ import annotations

import numpy as np

__all__ = ["ParticleScalarFieldSaverPrms", "InteractionScalarFieldSaverPrms", "WallVectorFieldSaverPrms",
           "FieldSaver"]


class _SaverPrms:
    def __init__(self, fieldName, fileName, fileFormat, beginTimeStep, endTimeStep, timeStepIncr):
        self.fieldName, self.fileName, self.fileFormat = fieldName, fileName, fileFormat
        self.beginTimeStep, self.endTimeStep, self.timeStepIncr = int(beginTimeStep), int(endTimeStep), int(timeStepIncr)


class ParticleScalarFieldSaverPrms(_SaverPrms):  # Python/esys/lsm/ParticleFieldSaverPrmsPy.cpp
    FORMATS = ("SUM", "MAX", "RAW_SERIES")


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

    def save(self, sim):
        p = self.p
        if isinstance(p, ParticleScalarFieldSaverPrms):
            _, v = sim.particle_scalar_field(p.fieldName, sort=True)
            if p.fileFormat == "SUM":
                line = _g(_ordered_sum(v))
            elif p.fileFormat == "MAX":
                line = _g(float(v.max()) if len(v) else 0.0)
            else:
                line = "".join(_g(x) + "  " for x in v)
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
