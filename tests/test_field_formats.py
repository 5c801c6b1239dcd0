"""The particle field savers' file formats (host logic, no GPU): a stand-in simulation hands
the savers fixed field values and the files are compared with the reference writers' output
formats, restated here line by line (ScalarParticleFieldMaster::writeAsRawWithPosID,
VectorParticleFieldMaster::writeAsSUM / MAX / RAW_SERIES / RAW2 / RAW_WITH_ID in
Fields/ParticleFieldMaster.cpp, AFieldMaster::makeFilename in Fields/FieldMaster.cpp)."""
import numpy as np
import pytest


class FakeSim:
    """Four particles stored out of id order, with tags 1, 2, 3, 1."""

    ids = np.array([7, 2, 5, 3], np.int32)
    pos = np.array([[0.5, 1.0, 1.5], [2.0, 2.25, 2.5], [3.0, 3.125, 1e-7], [4.0, -4.5, 5.0]])
    vel = np.array([[1.0, 0.0, -1.0], [0.5, 0.25, 2.0], [-3.0, 0.0, 0.0], [2.0, 2.0, 1.0]])
    rad = np.array([0.5, 0.25, 0.125, 0.75])
    tag = np.array([1, 2, 3, 1])

    def _o(self, sort):
        return np.argsort(self.ids, kind="stable") if sort else np.arange(len(self.ids))

    def particle_scalar_field(self, field, sort=True):
        o = self._o(sort)
        v = {"radius": self.rad, "tag": self.tag.astype(float), "v_abs": np.linalg.norm(self.vel, axis=1)}[field]
        return self.ids[o], v[o]

    def particle_vector_field(self, field, sort=True):
        o = self._o(sort)
        return self.ids[o], {"position": self.pos, "velocity": self.vel}[field][o]


def _saver(prms):
    from esys.lsm.fields import FieldSaver

    return FieldSaver(prms)


def test_vector_raw_formats_write_one_file_per_save(tmp_path):
    from esys.lsm import ParticleVectorFieldSaverPrms

    sim = FakeSim()
    by_id = np.argsort(sim.ids)
    for fmt, pre in (("RAW2", False), ("RAW_WITH_ID", True)):
        base = str(tmp_path / fmt)
        s = _saver(ParticleVectorFieldSaverPrms("velocity", base, fmt, 10, 100, 5))
        s.save(sim)
        s.save(sim)
        for k in (0, 1):  # <file>.<k * incr>.dat, k the save counter
            lines = open(f"{base}.{k * 5}.dat").read().splitlines()
            want = []
            for i in by_id:
                row = " ".join("%g" % x for x in sim.pos[i]) + " " + " ".join("%g" % x for x in sim.vel[i])
                want.append((f"{sim.ids[i]} " if pre else "") + row)
            assert lines == want


def test_vector_series_formats(tmp_path):
    from esys.lsm import ParticleVectorFieldSaverPrms

    sim = FakeSim()
    by_id = np.argsort(sim.ids)
    f = {k: str(tmp_path / k) for k in ("SUM", "MAX", "RAW_SERIES")}
    for k, fn in f.items():
        _saver(ParticleVectorFieldSaverPrms("velocity", fn, k, 0, 10, 1)).save(sim)
    v = sim.vel[by_id]
    s = [0.0, 0.0, 0.0]
    for row in v:
        for c in range(3):
            s[c] += row[c]
    assert open(f["SUM"]).read() == " ".join("%g" % x for x in s) + "\n"
    n2 = (v * v).sum(1)
    assert open(f["MAX"]).read() == " ".join("%g" % x for x in v[int(np.argmax(n2))]) + "\n"
    assert open(f["RAW_SERIES"]).read() == "".join(" ".join("%g" % x for x in row) + "  " for row in v) + "\n"


def test_scalar_raw_with_pos_id_and_tags(tmp_path):
    from esys.lsm import TaggedParticleScalarFieldSaverPrms, TaggedParticleVectorFieldSaverPrms

    sim = FakeSim()
    base = str(tmp_path / "vabs")
    # tag 1 under mask 3: particles 7 and 3 (tags 1, 1); tag 3 matches neither
    _saver(TaggedParticleScalarFieldSaverPrms("v_abs", base, "RAW_WITH_POS_ID", 0, 10, 2, 1, 3)).save(sim)
    lines = open(base + ".0.dat").read().splitlines()
    want = []
    for i in (3, 0):  # ids 3, 7
        want.append(f"{sim.ids[i]} " + " ".join("%g" % x for x in sim.pos[i]) + " %g %g" % (
            sim.rad[i], np.linalg.norm(sim.vel[i])))
    assert lines == want
    fn = str(tmp_path / "vsum")
    _saver(TaggedParticleVectorFieldSaverPrms("velocity", fn, "SUM", 0, 10, 1, 2, 2)).save(sim)
    # mask 2: tags 2 and 3 qualify (ids 2, 5)
    s = sim.vel[1] + sim.vel[2]
    assert open(fn).read() == " ".join("%g" % x for x in s) + "\n"


def test_unprovided_formats_are_refused():
    from esys.lsm import ParticleScalarFieldSaverPrms, ParticleVectorFieldSaverPrms

    with pytest.raises(NotImplementedError):
        _saver(ParticleVectorFieldSaverPrms("velocity", "x", "RAW_WITH_POS_ID", 0, 10, 1))
    with pytest.raises(NotImplementedError):
        _saver(ParticleScalarFieldSaverPrms("e_kin", "x", "DX", 0, 10, 1))
