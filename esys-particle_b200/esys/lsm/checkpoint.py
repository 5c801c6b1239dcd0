"""Checkpoints: the reference's CheckPointPrms / RestartCheckPointPrms and the files they write.

A checkpoint at timestep t is a set of text files named ``<prefix>_t=<t>_<rank>.txt``
(CheckPointPrmsPy::getFileName, Python/esys/lsm/CheckPointParamsPy.cpp):
  rank 0  the master's info file (CheckPointInfo::write, Parallel/CheckPointInfo.cpp:82-101):
          checkpoint version, number of timesteps, timestep size, timestep, the program
          marker, the geometry (bounding box, periodic dimensions, dimension) and the names
          of the workers' files;
  rank 1  the worker's file, written by the GPU library: TSubLattice::saveCheckPointData
          (restart checkpoints, dem_save_checkpoint) or saveSnapShotData (snapshots,
          dem_save_snapshot).

A checkpoint is taken at t when beginTimeStep <= t <= endTimeStep and
(t - beginTimeStep) % timeStepIncr == 0, or t == endTimeStep
(CheckPointController::isCheckPoint, Parallel/CheckPointController.cpp:349-363), after the
step's field savers; the initial state is checkpointed at t = 0 (LatticeMaster.cpp:2634-2640).
Before a restart checkpoint the reference forces a neighbour search (LatticeMaster.cpp:2697-2700);
here the search is scheduled for the head of the next step (force-neutral either way).
"""
from __future__ import annotations

import os

__all__ = ["CheckPointPrms", "RestartCheckPointPrms", "CheckPointer", "read_info", "write_info"]

CHECKPOINT_VERSION = 3           # lsm_version_info::CheckPointVersion (Foundation/version.h)
PROGRAM_MARKER = "ESyS-Particle_B200_rev. 0"  # read back by GeometryInfo::read as an "ESyS..." header


def file_name(prefix, t, rank):
    return f"{prefix}_t={int(t)}_{int(rank)}.txt"


class CheckPointPrms:  # Python/esys/lsm/CheckPointParamsPy.cpp:80-139
    def __init__(self, fileNamePrefix, beginTimeStep, endTimeStep, timeStepIncr):
        self.fileNamePrefix = str(fileNamePrefix)
        self.beginTimeStep, self.endTimeStep, self.timeStepIncr = int(beginTimeStep), int(endTimeStep), int(timeStepIncr)
        if self.timeStepIncr <= 0:
            raise ValueError("timeStepIncr must be positive")

    def getFileNamePrefix(self):
        return self.fileNamePrefix

    def getBeginTimeStep(self):
        return self.beginTimeStep

    def getEndTimeStep(self):
        return self.endTimeStep

    def getTimeStepIncr(self):
        return self.timeStepIncr

    def getFileName(self, timeStep, rank=0):
        return file_name(self.fileNamePrefix, timeStep, rank)

    def getFileNameList(self):
        out = [self.getFileName(t) for t in range(self.beginTimeStep, self.endTimeStep, self.timeStepIncr)]
        out.append(self.getFileName(self.endTimeStep))
        return out


class RestartCheckPointPrms(CheckPointPrms):  # CheckPointParamsPy.cpp:55-78, 141-185
    def __init__(self, fileNamePrefix, beginTimeStep, endTimeStep, timeStepIncr, Precision=12):
        super().__init__(fileNamePrefix, beginTimeStep, endTimeStep, timeStepIncr)
        self.precision = int(Precision)

    def getPrecision(self):
        return self.precision


def write_info(path, num_steps, dt, t, bbox_min, bbox_max, periodic, worker_files):
    """CheckPointInfo::write (Parallel/CheckPointInfo.cpp:82-101) with GeometryInfo's
    writeWithoutVersion (Geometry/GeometryInfo.cpp:134-155); C++ default stream format."""
    g = lambda x: format(float(x), "g")
    with open(path, "w") as f:
        f.write(f"V {CHECKPOINT_VERSION}\n{int(num_steps)}\n{g(dt)}\n{int(t)}\n{PROGRAM_MARKER}\n")
        f.write("BoundingBox " + " ".join(g(x) for x in list(bbox_min) + list(bbox_max)) + "\n")
        f.write("PeriodicBoundaries " + " ".join(str(int(bool(x))) for x in periodic) + "\n")
        f.write("Dimension 3D\n")
        f.write(" ".join(worker_files))


def read_info(path):
    """CheckPointInfo::read (Parallel/CheckPointInfo.cpp:53-78): the fields write_info writes."""
    tok = open(path).read().split()
    if not tok or tok[0] != "V":
        raise ValueError(f"{path}: not a checkpoint info file")
    k = 2
    num_steps, dt, t = int(tok[k]), float(tok[k + 1]), int(tok[k + 2])
    k += 3
    while k < len(tok) and tok[k] != "BoundingBox":   # program marker (one or two tokens)
        k += 1
    bb = [float(x) for x in tok[k + 1:k + 7]]
    k += 7
    if tok[k] != "PeriodicBoundaries":
        raise ValueError(f"{path}: expected PeriodicBoundaries")
    periodic = [bool(int(x)) for x in tok[k + 1:k + 4]]
    k += 4
    if tok[k] != "Dimension":
        raise ValueError(f"{path}: expected Dimension")
    dim = tok[k + 1]
    files = tok[k + 2:]
    return {"version": int(tok[1]), "num_steps": num_steps, "dt": dt, "t": t, "bbox_min": bb[:3], "bbox_max": bb[3:],
            "periodic": periodic, "dimension": dim, "files": files}


def worker_file(info_path, info):
    """The worker file of a loaded info file: the prefix of the first listed name with rank 1
    (CheckPointController::issueCheckPointLoadingCmd, Parallel/CheckPointController.cpp:268-300),
    opened as written or, failing that, beside the info file.  The prefix ends at the last
    "_t=" (the reference cuts at the first "_t", which a directory name can also contain)."""
    first = info["files"][0] if info["files"] else os.path.basename(info_path)
    prefix = first[:first.rfind("_t=")] if "_t=" in first else first
    name = file_name(prefix, info["t"], 1)
    if os.path.exists(name):
        return name
    alt = os.path.join(os.path.dirname(os.path.abspath(info_path)), os.path.basename(name))
    return alt


def walls_in(worker_path):
    """Wall names, origins and normals of a restart worker file (its "Walls" section)."""
    lines = open(worker_path).read().split("\n")
    for i in range(len(lines) - 1, -1, -1):
        t = lines[i].split()
        if len(t) == 2 and t[0] == "Walls":
            out, k = {}, i + 1
            for _ in range(int(t[1])):
                while not lines[k].split():
                    k += 1
                name = lines[k].split()[0]
                v = [float(x) for x in lines[k + 1].split()]
                out[name] = (v[0:3], v[6:9])
                k += 2
            return out
    return {}


class CheckPointer:
    """A checkpoint saver of LsmMpi (restart or snapshot), with the field savers' interface."""

    def __init__(self, lsm, prms, restart):
        self.lsm, self.prms, self.restart = lsm, prms, restart

    def need_save(self, t):
        p = self.prms
        return (p.beginTimeStep <= t <= p.endTimeStep and (t - p.beginTimeStep) % p.timeStepIncr == 0) or \
            t == p.endTimeStep

    def next_save(self, t):
        """The first checkpoint time after t, or None."""
        p = self.prms
        if t < p.beginTimeStep:
            return p.beginTimeStep
        if t >= p.endTimeStep:
            return None
        k = (t - p.beginTimeStep) // p.timeStepIncr + 1
        return min(p.beginTimeStep + k * p.timeStepIncr, p.endTimeStep)

    def save(self, sim, t=None):
        t = sim.timestep if t is None else t
        prefix = self.prms.fileNamePrefix
        d = os.path.dirname(prefix)
        if d:
            os.makedirs(d, exist_ok=True)
        worker = file_name(prefix, t, 1)
        if self.restart:
            sim.save_checkpoint(worker, getattr(self.prms, "precision", 12))
            sim.search_neighbors()
        else:
            sim.save_snapshot(worker)
        lsm = self.lsm
        write_info(file_name(prefix, t, 0), lsm.getNumTimeSteps(), lsm.getTimeStepSize(), t, lsm._bbox[0],
                   lsm._bbox[1], lsm._circ, [worker])
