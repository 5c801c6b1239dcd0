"""Vec3 and BoundingBox of esys.lsm.util (Python/esys/lsm/util/Vec3Py.cpp, BoundingBoxPy.cpp)."""
from __future__ import annotations

import math


class Vec3:
    """3-vector with the arithmetic of Foundation/vec3.h."""

    __slots__ = ("_v",)

    def __init__(self, x=0.0, y=0.0, z=0.0):
        if hasattr(x, "__len__") and not isinstance(x, str):
            x, y, z = x
        self._v = [float(x), float(y), float(z)]

    def __getitem__(self, i):
        return self._v[i]

    def __setitem__(self, i, v):
        self._v[i] = float(v)

    def __len__(self):
        return 3

    def __iter__(self):
        return iter(self._v)

    def __add__(self, o):
        return Vec3(self[0] + o[0], self[1] + o[1], self[2] + o[2])

    def __sub__(self, o):
        return Vec3(self[0] - o[0], self[1] - o[1], self[2] - o[2])

    def __neg__(self):
        return Vec3(-self[0], -self[1], -self[2])

    def __mul__(self, s):
        if isinstance(s, Vec3):
            return self[0] * s[0] + self[1] * s[1] + self[2] * s[2]
        return Vec3(self[0] * s, self[1] * s, self[2] * s)

    __rmul__ = __mul__

    def __truediv__(self, s):
        return Vec3(self[0] / s, self[1] / s, self[2] / s)

    def __eq__(self, o):
        return list(self) == list(o)

    def norm(self):
        return math.sqrt(self[0] * self[0] + self[1] * self[1] + self[2] * self[2])

    def norm2(self):
        return self[0] * self[0] + self[1] * self[1] + self[2] * self[2]

    def X(self):
        return self[0]

    def Y(self):
        return self[1]

    def Z(self):
        return self[2]

    def toList(self):
        return list(self._v)

    def __repr__(self):
        return f"Vec3({self[0]!r}, {self[1]!r}, {self[2]!r})"


class BoundingBox:
    def __init__(self, minPt=Vec3(), maxPt=Vec3()):
        self._min, self._max = Vec3(*minPt), Vec3(*maxPt)

    def getMinPt(self):
        return self._min

    def getMaxPt(self):
        return self._max

    def getSizes(self):
        return self._max - self._min

    def __repr__(self):
        return f"BoundingBox({self._min!r}, {self._max!r})"
