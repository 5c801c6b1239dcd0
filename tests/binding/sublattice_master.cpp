/*
 * Test driver for TGpuSubLattice (esys-particle_b200/integration/GpuSubLattice.h): a master and a
 * worker in one process, joined by the two-party MPI stand-in of mailbox/mpi.h.
 *
 * Test infrastructure, not product code.  The worker thread runs the worker's command loop
 * for the commands the GPU path serves, as CSubLatticeControler::run dispatches them
 * (Parallel/SubLatticeControler.cpp:534-720, with makeLattice / initLattice / initLatticeCirc /
 * setTimeStepSize / getNumParticles / getIdParticleData of the same file), on a
 * TGpuSubLattice made where makeLattice makes TSubLattice.  The caller's thread is the master:
 * each slm_* function sends what CLatticeMaster sends for that operation (the file and lines
 * are cited at each), with the reference's own buffers, commands and parameter classes, and
 * reads back what the master reads.  Plain C entry points for ctypes; 0 = ok, -1 = failure
 * (slm_error() gives the text).
 */
#include "GpuSubLattice.h"

#include "Model/ElasticInteraction.h"
#include "Model/RotFricInteraction.h"
#include "Parallel/BroadCast_cmd.h"
#include "Parallel/RankAndComm.h"
#include "Parallel/mpicmdbuf.h"
#include "Parallel/sublattice_cmd.h"

#include <map>
#include <memory>
#include <string>
#include <thread>

namespace {

std::string g_err;
std::string g_worker_err;
std::thread g_worker;
int g_rot = 1;
bool g_first = true;  // CLatticeMaster::m_first_time

// ---- worker: the command loop -------------------------------------------------------------
void worker_loop() {
  mailbox::set_rank(1);
  try {
    CMPILCmdBuffer cmd_buffer(MPI_COMM_WORLD, 0);
    TML_Comm global(MPI_COMM_WORLD);
    std::unique_ptr<ASubLattice> lat;
    for (;;) {
      const int command = cmd_buffer.receive();
      switch (command) {
        case CMD_MAKELATTICE: {  // CSubLatticeControler::makeLattice (:121-150)
          CVarMPIBuffer param_buffer(MPI_COMM_WORLD);
          param_buffer.receiveBroadcast(0);
          const esys::lsm::CLatticeParam clp = esys::lsm::CLatticeParam::extractLatticeParam(&param_buffer);
          if (clp.particle_type() == "Basic")
            lat.reset(new TGpuSubLattice<CParticle>(clp, 1, MPI_COMM_WORLD, MAILBOX_WORKER_COMM));
          else if (clp.particle_type() == "Rot")
            lat.reset(new TGpuSubLattice<CRotParticle>(clp, 1, MPI_COMM_WORLD, MAILBOX_WORKER_COMM));
          else
            throw std::runtime_error("ERROR! Trying to make lattice from unknown particles: " + clp.particle_type());
          break;
        }
        case CMD_SETTIMESTEPSIZE: {  // CSubLatticeControler::setTimeStepSize
          CVarMPIBuffer buffer(MPI_COMM_WORLD);
          buffer.receiveBroadcast(0);
          lat->setTimeStepSize(buffer.pop_double());
          break;
        }
        case CMD_INITLATTICE:
        case CMD_INITLATTICECIRC: {  // CSubLatticeControler::initLattice / initLatticeCirc
          std::vector<Vec3> bbox;
          global.recv_broadcast_cont_packed(bbox, 0);
          if (command == CMD_INITLATTICE) {
            lat->initNeighborTable(bbox[0], bbox[1]);
          } else {
            std::vector<int> cv;
            global.recv_broadcast_cont(cv, 0);
            std::vector<bool> circ;
            for (int c : cv) circ.push_back(c == 1);
            lat->initNeighborTable(bbox[0], bbox[1], circ);
          }
          std::vector<int> commdims = lat->getCommDims();
          global.send_gather(commdims, 0);
          std::vector<int> commcoords = lat->getCommCoords();
          global.send_gather(commcoords, 0);
          break;
        }
        case CMD_RECEIVEPARTICLES: lat->receiveParticles(); break;
        case CMD_RECEIVECONNECTIONS: lat->receiveConnections(); break;
        case CMD_ADDWALL: lat->addWall(); break;
        case CMD_ADDEWALLIG: lat->addElasticWIG(); break;
        case CMD_ADDPIG: lat->addPairIG(); break;
        case CMD_ADDBONDEDIG: lat->addBondedIG(); break;
        case CMD_ADDROTBONDEDIG: lat->addRotBondedIG(); break;
        case CMD_ADDBRITTLEBEAMSCIG: lat->addBrittleBeamSCIG(); break;
        case CMD_ADDBRITTLEBEAMDZCIG: lat->addBrittleBeamDZCIG(); break;
        case CMD_ADDSIG: lat->addSingleIG(); break;
        case CMD_ADDDAMP: lat->addDamping(); break;
        case CMD_EXIG: lat->setExIG(); break;
        case CMD_CHECKNEIGHBORS: lat->checkNeighbors(); break;
        case CMD_NSEARCH: lat->searchNeighbors(); break;
        case CMD_UPDATE: lat->updateInteractions(); break;
        case CMD_CALC: lat->oneStep(); break;
        case CMD_XCHANGE: lat->exchangePos(); break;
        case CMD_WMOVE: lat->moveWallBy(); break;
        case CMD_WFORCE: lat->applyForceToWall(); break;
        case CMD_PMOVETAGGEDBY: lat->moveTaggedParticlesBy(); break;
        case CMD_GETWALLPOS: lat->getWallPos(); break;
        case CMD_GETWALLFORCE: lat->getWallForce(); break;
        case CMD_COUNT: lat->countParticles(); break;
        case CMD_GETNUMPARTICLES: {  // CSubLatticeControler::getNumParticles (:349-354)
          std::vector<int> v(1, lat->getNumParticles());
          global.send_gather(v, 0);
          break;
        }
        case CMD_GETIDPARTICLEDATA: {  // CSubLatticeControler::getIdParticleData (:399-415)
          ASubLattice::IdVector ids;
          global.recv_broadcast_cont(ids, 0);
          lat->getParticleData(ids);
          break;
        }
        case CMD_FINISH: return;
        default: throw std::runtime_error("worker got unknown command " + std::to_string(command));
      }
    }
  } catch (const std::exception& e) {
    g_worker_err = e.what();
    mailbox::abort_all(g_worker_err);
  }
}

// ---- master helpers --------------------------------------------------------------------------
MpiRankAndComm master_rc() { return MpiRankAndComm(0, MPI_COMM_WORLD); }

template <class F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    if (!g_worker_err.empty()) g_err += " [worker: " + g_worker_err + "]";
    return -1;
  }
}

// CLatticeMaster::searchNeighbors / checkNeighbors (Parallel/LatticeMaster.cpp:1864-1908)
void master_search(bool force) {
  CMPILCmdBuffer cmd_buffer(MPI_COMM_WORLD, 0);
  bool need = true;
  if (!force) {
    CMPISGBufferRoot buffer(MPI_COMM_WORLD, 8);
    cmd_buffer.broadcast(CMD_CHECKNEIGHBORS);
    buffer.gather();
    need = buffer.pop_int(1) == 1;
  }
  if (need) cmd_buffer.broadcast(CMD_NSEARCH);
}

void master_update() {  // CLatticeMaster::updateInteractions (:1912-1920)
  CMPILCmdBuffer cmd_buffer(MPI_COMM_WORLD, 0);
  cmd_buffer.broadcast(CMD_UPDATE);
}

Vec3 master_wall_query(int cmd_id, const char* name) {  // CLatticeMaster::getWallForce (:993-1019)
  BroadcastCommand cmd(master_rc(), cmd_id);
  cmd.append(name);
  cmd.broadcast();
  std::multimap<int, Vec3> m;
  TML_Comm(MPI_COMM_WORLD).gather(m);
  Vec3 s(0.0, 0.0, 0.0);
  for (auto& kv : m) s = s + kv.second;
  return s;
}

}  // namespace

extern "C" {

const char* slm_error() { return g_err.c_str(); }

// CLatticeMaster::makeLattice + setTimeStepSize + setSpatialDomain (Parallel/LatticeMaster.cpp:528-693)
int slm_start(int rot, double nrange, double alpha, const double* mn, const double* mx, const int* circ, double dt) {
  if (g_worker.joinable()) { g_err = "already started"; return -1; }
  mailbox::reset();
  mailbox::set_rank(0);
  g_err.clear();
  g_worker_err.clear();
  g_rot = rot;
  g_first = true;
  g_worker = std::thread(worker_loop);
  return guarded([&] {
    CMPILCmdBuffer cmd_buffer(MPI_COMM_WORLD, 0);
    TML_Comm global(MPI_COMM_WORLD);
    {
      CVarMPIBuffer buffer(MPI_COMM_WORLD);
      cmd_buffer.broadcast(CMD_MAKELATTICE);
      esys::lsm::CLatticeParam clp(rot ? "Rot" : "Basic", nrange, alpha);
      clp.packInto(&buffer);
      buffer.broadcast(0);
    }
    {
      BroadcastCommand cmd(master_rc(), CMD_SETTIMESTEPSIZE);
      cmd.append(dt);
      cmd.broadcast();
    }
    const bool periodic = circ && (circ[0] || circ[1] || circ[2]);
    cmd_buffer.broadcast(periodic ? CMD_INITLATTICECIRC : CMD_INITLATTICE);
    std::vector<Vec3> corners{Vec3(mn[0], mn[1], mn[2]), Vec3(mx[0], mx[1], mx[2])};
    global.broadcast_cont_packed(corners);
    if (periodic) {
      std::vector<int> cv{circ[0] != 0, circ[1] != 0, circ[2] != 0};
      global.broadcast_cont(cv);
    }
    std::multimap<int, int> dims, coords;  // getSlaveSpatialDomains (:697-740)
    global.gather(dims);
    global.gather(coords);
    if (dims.size() != 3) throw std::runtime_error("worker sent " + std::to_string(dims.size()) + " dims");
  });
}

// CLatticeMaster::addParticles (Parallel/LatticeMaster.hpp:260-340): one packed broadcast and
// the forced search that follows it.
int slm_add_particles(int n, const int* id, const int* tag, const double* pos, const double* rad, const double* mass,
                      const double* vel, const double* angvel) {
  return guarded([&] {
    CMPILCmdBuffer cmd_buffer(MPI_COMM_WORLD, 0);
    TML_Comm global(MPI_COMM_WORLD);
    cmd_buffer.broadcast(CMD_RECEIVEPARTICLES);
    const Vec3 zero(0.0, 0.0, 0.0);
    if (g_rot) {
      std::vector<CRotParticle> v;
      for (int i = 0; i < n; ++i) {
        Quaternion q(1.0, zero);
        CRotParticle p(rad[i], mass[i], Vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]),
                       Vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]), zero, id[i], q,
                       0.4 * mass[i] * rad[i] * rad[i], zero,
                       angvel ? Vec3(angvel[3 * i], angvel[3 * i + 1], angvel[3 * i + 2]) : zero, true, true);
        p.setTag(tag[i]);
        v.push_back(p);
      }
      global.broadcast_cont_packed(v);
    } else {
      std::vector<CParticle> v;
      for (int i = 0; i < n; ++i) {
        CParticle p(rad[i], mass[i], Vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]),
                    Vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]), zero, id[i], true);
        p.setTag(tag[i]);
        v.push_back(p);
      }
      global.broadcast_cont_packed(v);
    }
    master_search(true);
  });
}

// CLatticeMaster::addConnections (Parallel/LatticeMaster.hpp:343-392).
int slm_add_connections(int n, const int* tag, const int* id1, const int* id2) {
  return guarded([&] {
    CMPILCmdBuffer cmd_buffer(MPI_COMM_WORLD, 0);
    std::vector<int> buf;
    for (int i = 0; i < n; ++i) { buf.push_back(tag[i]); buf.push_back(id1[i]); buf.push_back(id2[i]); }
    cmd_buffer.broadcast(CMD_RECEIVECONNECTIONS);
    TML_Comm(MPI_COMM_WORLD).broadcast_cont_packed(buf);
    master_search(true);
  });
}

// CLatticeMaster::addWall (Parallel/LatticeMaster.cpp:829-845).
int slm_add_wall(const char* name, const double* o, const double* nrm) {
  return guarded([&] {
    BroadcastCommand cmd(master_rc(), CMD_ADDWALL);
    cmd.append(name);
    cmd.append(Vec3(o[0], o[1], o[2]));
    cmd.append(Vec3(nrm[0], nrm[1], nrm[2]));
    cmd.broadcast();
  });
}

// CLatticeMaster::addWallIG(const CEWallIGP&) (Parallel/LatticeMaster.cpp:851-860).
int slm_add_wall_group(const char* name, const char* wall, double k) {
  return guarded([&] {
    BroadcastCommand cmd(master_rc(), CMD_ADDEWALLIG);
    cmd.packInto(CEWallIGP(name, wall, k));
    cmd.broadcast();
  });
}

// CLatticeMaster::addPairIG(const CElasticIGP&) (Parallel/LatticeMaster.cpp:3066-3073).
int slm_add_elastic(const char* name, double k, int scaling) {
  return guarded([&] {
    CElasticIGP prms(name, k, scaling != 0);
    BroadcastCommand cmd(master_rc(), CMD_ADDPIG);
    cmd.appendTypeAndName(prms);
    cmd.append(prms.m_k);
    cmd.append(static_cast<int>(prms.m_scaling));
    cmd.broadcast();
  });
}

// CLatticeMaster::addPairIG(const CRotFrictionIGP&) (Parallel/LatticeMaster.cpp:3223-3235).
int slm_add_rot_friction(const char* name, double k, double mu_s, double mu_d, double k_s, double dt, int scaling,
                         int meanR) {
  return guarded([&] {
    CRotFrictionIGP prms(name, k, mu_d, mu_s, k_s, dt, scaling != 0, false, meanR != 0);
    BroadcastCommand cmd(master_rc(), CMD_ADDPIG);
    cmd.appendTypeAndName(prms);
    cmd.append(prms.k);
    cmd.append(prms.mu_s);
    cmd.append(prms.mu_d);
    cmd.append(prms.k_s);
    cmd.append(prms.dt);
    cmd.append(static_cast<int>(prms.scaling));
    cmd.append(static_cast<int>(prms.meanR_scaling));
    cmd.broadcast();
  });
}

// CLatticeMaster::addRotBondedIG (Parallel/LatticeMaster.cpp:2871-2913).
int slm_add_rot_bond(const char* name, int tag, double kr, double ks, double kt, double kb, double max_n, double max_s,
                     double max_t, double max_b, int scaling, int meanR, double truncated) {
  return guarded([&] {
    CMPILCmdBuffer cmd_buffer(MPI_COMM_WORLD, 0);
    CVarMPIBuffer pbuffer(MPI_COMM_WORLD, 256);
    cmd_buffer.broadcast(CMD_ADDROTBONDEDIG);
    pbuffer.append(tag);
    pbuffer.append(name);
    for (double v : {kr, ks, kt, kb, max_n, max_s, max_t, max_b}) pbuffer.append(v);
    pbuffer.append(scaling);
    pbuffer.append(meanR);
    pbuffer.append(truncated);
    pbuffer.broadcast(0);
  });
}

// CLatticeMaster::addDamping(const CDampingIGP&) (Parallel/LatticeMaster.cpp:4076-4082).
int slm_add_damping(int rot, double visc, double dt, int max_iter) {
  return guarded([&] {
    CDampingIGP prms(rot ? "RotDamping" : "Damping", rot ? "RotDamping" : "Damping", visc, dt, max_iter);
    BroadcastCommand cmd(master_rc(), CMD_ADDDAMP);
    cmd.append(prms.getTypeString().c_str());
    cmd.packInto(prms);
    cmd.broadcast();
  });
}

// CLatticeMaster::addSingleIG(const GravityIGP&) (Parallel/LatticeMaster.cpp:3970-3997).
int slm_add_gravity(const char* name, const double* g) {
  return guarded([&] {
    esys::lsm::GravityIGP prms(name, Vec3(g[0], g[1], g[2]));
    BroadcastCommand cmd(master_rc(), CMD_ADDSIG);
    cmd.append(prms.getTypeString().c_str());
    cmd.packInto(prms);
    cmd.broadcast();
  });
}

// CLatticeMaster::addExIG (Parallel/LatticeMaster.cpp:4143-4160).
int slm_add_exclusion(const char* bonded, const char* dynamic) {
  return guarded([&] {
    CVarMPIBuffer pbuffer(MPI_COMM_WORLD, 20);
    CMPILCmdBuffer cmd_buffer(MPI_COMM_WORLD, 0);
    cmd_buffer.broadcast(CMD_EXIG);
    pbuffer.append(bonded);
    pbuffer.append(dynamic);
    pbuffer.broadcast(0);
    master_update();
  });
}

// CLatticeMaster::runOneStep x nsteps (Parallel/LatticeMaster.cpp:2602-2740) without savers,
// checkpoints or runnables: the first step's forced search, then per step the neighbour check
// (and search), the interaction update and oneStep (CMD_CALC + CMD_XCHANGE, :1672-1690).
int slm_run(int nsteps) {
  return guarded([&] {
    CMPILCmdBuffer cmd_buffer(MPI_COMM_WORLD, 0);
    for (int s = 0; s < nsteps; ++s) {
      if (g_first) {
        master_search(true);
        g_first = false;
      }
      master_search(false);
      master_update();
      cmd_buffer.broadcast(CMD_CALC);
      cmd_buffer.broadcast(CMD_XCHANGE);
    }
  });
}

// CLatticeMaster::moveWallBy (Parallel/LatticeMaster.cpp:1579-1590).
int slm_move_wall(const char* name, const double* d) {
  return guarded([&] {
    CMPILCmdBuffer cmd_buffer(MPI_COMM_WORLD, 0);
    CVarMPIBuffer buffer(MPI_COMM_WORLD);
    cmd_buffer.broadcast(CMD_WMOVE);
    buffer.append(name);
    buffer.append(Vec3(d[0], d[1], d[2]));
    buffer.broadcast(0);
  });
}

int slm_get_wall_force(const char* name, double* out) {
  return guarded([&] {
    const Vec3 f = master_wall_query(CMD_GETWALLFORCE, name);
    for (int k = 0; k < 3; ++k) out[k] = f[k];
  });
}

int slm_get_wall_pos(const char* name, double* out) {
  return guarded([&] {
    const Vec3 p = master_wall_query(CMD_GETWALLPOS, name);
    for (int k = 0; k < 3; ++k) out[k] = p[k];
  });
}

// CLatticeMaster::getNumParticles (Parallel/LatticeMaster.cpp:3022-3043).
int slm_num_particles() {
  int total = -1;
  const int rc = guarded([&] {
    BroadcastCommand cmd(master_rc(), CMD_GETNUMPARTICLES);
    cmd.broadcastCommand();
    std::multimap<int, int> m;
    TML_Comm(MPI_COMM_WORLD).gather(m);
    total = 0;
    for (auto& kv : m) total += kv.second;
  });
  return rc < 0 ? -1 : total;
}

// CLatticeMaster::visitParticlesOfType (Parallel/LatticeMaster.hpp:185-215): every particle's
// id, position, velocity, force, angular velocity, moment, orientation (scalar first), up to
// cap rows.  Returns the row count.
int slm_get_particles(int cap, int* id, double* pos, double* vel, double* force, double* angvel, double* moment,
                      double* quat) {
  int rows = -1;
  const int rc = guarded([&] {
    BroadcastCommand cmd(master_rc(), CMD_GETIDPARTICLEDATA);
    cmd.broadcastCommand();
    TML_Comm global(MPI_COMM_WORLD);
    std::vector<int> ids;  // empty: all particles
    global.broadcast_cont(ids);
    rows = 0;
    auto put = [&](int k, const CParticle& p) {
      id[k] = p.getID();
      const Vec3 x = p.getPos(), v = p.getVel(), f = p.getForce();
      for (int c = 0; c < 3; ++c) { pos[3 * k + c] = x[c]; vel[3 * k + c] = v[c]; force[3 * k + c] = f[c]; }
    };
    if (g_rot) {
      std::multimap<int, CRotParticle> m;
      global.gather_packed(m);
      for (auto& kv : m) {
        if (rows >= cap) break;
        put(rows, kv.second);
        const Vec3 w = kv.second.getAngVel(), mo = kv.second.getMoment();
        const Quaternion q = kv.second.getQuat();
        for (int c = 0; c < 3; ++c) { angvel[3 * rows + c] = w[c]; moment[3 * rows + c] = mo[c]; }
        quat[4 * rows] = q.return_sca();
        for (int c = 0; c < 3; ++c) quat[4 * rows + 1 + c] = q.return_vec()[c];
        ++rows;
      }
    } else {
      std::multimap<int, CParticle> m;
      global.gather_packed(m);
      for (auto& kv : m) {
        if (rows >= cap) break;
        put(rows++, kv.second);
      }
    }
  });
  return rc < 0 ? -1 : rows;
}

// CMD_FINISH ends the worker's loop (CLatticeMaster's destructor sends it).
int slm_finish() {
  const int rc = guarded([&] {
    CMPILCmdBuffer cmd_buffer(MPI_COMM_WORLD, 0);
    cmd_buffer.broadcast(CMD_FINISH);
  });
  if (g_worker.joinable()) g_worker.join();
  if (!g_worker_err.empty() && rc == 0) {
    g_err = "worker: " + g_worker_err;
    return -1;
  }
  return rc;
}

}  // extern "C"

// BondedInteractionCpData (linked for the RotBond checkpoint records) references this accessor
// of the thermal bond, whose translation unit pulls in the whole thermal particle family.
// Thermal bonds are not on the GPU path, so the accessor is defined here and never called.
#include "Model/RotThermBondedInteraction.h"
int CRotThermBondedInteraction::getTag() const { return 0; }
