/*
 * GpuSubLattice.hpp -- method bodies of TGpuSubLattice<T> (included by GpuSubLattice.h).
 *
 * Each operation cites the TSubLattice / TRotSubLattice operation whose messages it reads:
 * the parameters are popped in the same order and the same collective calls are made, so
 * the master's side of every exchange is unchanged.
 */
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <unistd.h>

namespace esys_gpu_detail {
// The particles' dynamic / rotational switches are protected members without getters; a
// pointer to member formed in a derived class reads them from any particle.
struct ParticleFlags : CRotParticle {
  static bool dynamic(const CParticle& p) { return p.*(&ParticleFlags::m_is_dynamic); }
  static bool rotational(const CRotParticle& p) { return p.*(&ParticleFlags::m_is_rot); }
};

// A scratch file for the library's checkpoint writer / reader.
inline std::string scratch_path(const char* what) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "/tmp/esys_gpu_%s_%d_XXXXXX", what, (int)getpid());
  const int fd = mkstemp(buf);
  if (fd < 0) throw std::runtime_error("TGpuSubLattice: cannot create a scratch file");
  close(fd);
  return buf;
}
}  // namespace esys_gpu_detail

template <class T>
TGpuSubLattice<T>::TGpuSubLattice(const esys::lsm::CLatticeParam& param, int rank, MPI_Comm comm,
                                  MPI_Comm worker_comm)
    : m_h(NULL),
      m_nrange(param.nrange()),
      m_alpha(param.alpha()),
      m_dt(0.0),
      m_rank(rank),
      m_comm(comm),
      m_worker_comm(worker_comm),
      m_tml_comm(comm),
      m_pTimers(NULL) {
  int workers = 0;
  MPI_Comm_size(worker_comm, &workers);
  if (workers != 1)
    throw std::runtime_error("TGpuSubLattice: the GPU holds the whole specimen; run one worker (mpiDimList [1,1,1])");
  setParticleType(param.particle_type());
}

template <class T>
TGpuSubLattice<T>::~TGpuSubLattice() {
  if (m_h) dem_destroy(m_h);
}

template <class T>
void TGpuSubLattice<T>::check(int rc, const char* what) const {
  if (rc < 0) {
    std::stringstream msg;
    msg << "TGpuSubLattice::" << what << ": " << dem_last_error(m_h) << " (status " << rc << ")";
    throw std::runtime_error(msg.str());
  }
}

template <class T>
void TGpuSubLattice<T>::need_handle(const char* what) const {
  if (!m_h) throw std::runtime_error(std::string("TGpuSubLattice::") + what + " before initNeighborTable");
}

template <class T>
void TGpuSubLattice<T>::unsupported(const char* what) const {
  throw std::runtime_error(std::string("TGpuSubLattice::") + what + ": not on the GPU path");
}

// TSubLattice::setTimeStepSize (Parallel/SubLattice.hpp:2163-2204): the groups follow the new dt.
template <class T>
void TGpuSubLattice<T>::setTimeStepSize(double dt) {
  m_dt = dt;
  if (m_h) check(dem_set_timestep(m_h, dt), "setTimeStepSize");
}

// TSubLattice::initNeighborTable (Parallel/SubLattice.hpp:455-564): the search grid over the
// domain, x periodic when circ[0] (the library adjusts the range of a periodic x side as the
// reference does and refuses periodic y or z).
template <class T>
void TGpuSubLattice<T>::create(const Vec3& min, const Vec3& max, const int circ[3]) {
  if (m_h) throw std::runtime_error("TGpuSubLattice::initNeighborTable: called twice");
  const double mn[3] = {min.X(), min.Y(), min.Z()}, mx[3] = {max.X(), max.Y(), max.Z()};
  // the time step arrives by setTimeStepSize, before or after the table
  const int rc = dem_create(&m_h, kRot ? 1 : 0, m_nrange, m_alpha, mn, mx, circ, m_dt > 0 ? m_dt : 1.0);
  if (rc < 0) throw std::runtime_error(std::string("TGpuSubLattice::initNeighborTable: ") + dem_last_error(NULL));
}

template <class T>
void TGpuSubLattice<T>::initNeighborTable(const Vec3& min, const Vec3& max) {
  const int circ[3] = {0, 0, 0};
  create(min, max, circ);
}

template <class T>
void TGpuSubLattice<T>::initNeighborTable(const Vec3& min, const Vec3& max, const std::vector<bool>& circ) {
  const int c[3] = {circ.size() > 0 && circ[0], circ.size() > 1 && circ[1], circ.size() > 2 && circ[2]};
  create(min, max, c);
}

// TSubLattice::receiveParticles (Parallel/SubLattice.hpp:573-588): the master's packed
// particle broadcast (CLatticeMaster::addParticles, Parallel/LatticeMaster.hpp:260-330).
// Particles outside the grid are dropped, as NeighborTable::insert drops them.
template <class T>
void TGpuSubLattice<T>::receiveParticles() {
  std::vector<T> recv_buffer;
  CMPIBarrier barrier(m_comm);
  m_tml_comm.recv_broadcast_cont_packed(recv_buffer, 0);
  need_handle("receiveParticles");
  const int n = (int)recv_buffer.size();
  std::vector<int> id(n), tag(n), flags(n);
  std::vector<double> pos(3 * n), rad(n), mass(n), vel(3 * n), angvel(3 * n), quat(4 * n);
  for (int i = 0; i < n; ++i) {
    const T& p = recv_buffer[i];
    id[i] = p.getID();
    tag[i] = p.getTag();
    rad[i] = p.getRad();
    mass[i] = p.getMass();
    const Vec3 x = p.getPos(), v = p.getVel();
    for (int k = 0; k < 3; ++k) { pos[3 * i + k] = x[k]; vel[3 * i + k] = v[k]; }
    const bool dyn = esys_gpu_detail::ParticleFlags::dynamic(p);
    bool rot = false;
    quat[4 * i] = 1.0;
    if constexpr (kRot) {
      rot = esys_gpu_detail::ParticleFlags::rotational(p);
      const Vec3 w = p.getAngVel();
      const Quaternion q = p.getQuat();
      for (int k = 0; k < 3; ++k) { angvel[3 * i + k] = w[k]; quat[4 * i + 1 + k] = q.return_vec()[k]; }
      quat[4 * i] = q.return_sca();
    }
    flags[i] = (dyn ? 0 : 1) | (kRot && !rot ? 2 : 0);
    m_record[id[i]] = Record{tag[i], rad[i], mass[i], dyn, rot};
  }
  check(dem_add_particles(m_h, n, id.data(), tag.data(), pos.data(), rad.data(), mass.data(), vel.data(),
                          kRot ? angvel.data() : NULL, kRot ? quat.data() : NULL, flags.data()),
        "receiveParticles");
  barrier.wait("TSubLattice<T>::receiveParticles");
}

// TSubLattice::receiveConnections (Parallel/SubLattice.hpp:598-622): (tag, id1, id2) triples
// kept for the bonded groups created later with that tag; triples naming a particle this
// worker does not hold are skipped.
template <class T>
void TGpuSubLattice<T>::receiveConnections() {
  std::vector<int> recv_buffer;
  CMPIBarrier barrier(m_comm);
  m_tml_comm.recv_broadcast_cont_packed(recv_buffer, 0);
  need_handle("receiveConnections");
  std::vector<int> tag, id1, id2;
  for (size_t i = 0; i + 2 < recv_buffer.size(); i += 3) {
    if (!m_record.count(recv_buffer[i + 1]) || !m_record.count(recv_buffer[i + 2])) continue;
    tag.push_back(recv_buffer[i]);
    id1.push_back(recv_buffer[i + 1]);
    id2.push_back(recv_buffer[i + 2]);
  }
  check(dem_add_connections(m_h, (int)tag.size(), tag.data(), id1.data(), id2.data()), "receiveConnections");
  barrier.wait("TSubLattice<T>::receiveConnections");
}

// TSubLattice::addWall (Parallel/SubLattice.hpp:629-640): name, position, normal.
template <class T>
void TGpuSubLattice<T>::addWall() {
  CVarMPIBuffer param_buffer(m_comm);
  param_buffer.receiveBroadcast(0);
  const std::string name = param_buffer.pop_string();
  const Vec3 ipos = param_buffer.pop_vector();
  const Vec3 inorm = param_buffer.pop_vector();
  need_handle("addWall");
  const double o[3] = {ipos.X(), ipos.Y(), ipos.Z()}, nrm[3] = {inorm.X(), inorm.Y(), inorm.Z()};
  check(dem_add_wall(m_h, name.c_str(), o, nrm), "addWall");
  m_walls.insert(name);
}

// TSubLattice::addElasticWIG (Parallel/SubLattice.hpp:667-695): a CEWallIGP; an unknown wall
// is an error ("wall name '...' not found in map of walls").
template <class T>
void TGpuSubLattice<T>::addElasticWIG() {
  CVarMPIBuffer param_buffer(m_comm);
  param_buffer.receiveBroadcast(0);
  CEWallIGP* wigp = extractEWallIGP(&param_buffer);
  const std::string name = wigp->getName(), wall = wigp->getWallName();
  const double k = wigp->getSpringConst();
  delete wigp;
  need_handle("addElasticWIG");
  check(dem_add_wall_group(m_h, name.c_str(), wall.c_str(), k), "addElasticWIG");
  m_wall_groups.insert(name);
}

// TSubLattice::addPairIG + doAddPIG (Parallel/SubLattice.hpp:987-1003, 1033-1360): type and
// name, then the parameters of that type in the master's packing order
// (CLatticeMaster::addPairIG, Parallel/LatticeMaster.cpp:3066-3240).
template <class T>
void TGpuSubLattice<T>::addPairIG() {
  CVarMPIBuffer param_buffer(m_comm, 2000);
  param_buffer.receiveBroadcast(0);
  const std::string type = param_buffer.pop_string();
  const std::string name = param_buffer.pop_string();
  need_handle("addPairIG");
  int rc = DEM_OK;
  if (type == "Elastic") {
    const double k = param_buffer.pop_double();
    const int scaling = param_buffer.pop_int();
    rc = dem_add_elastic_group(m_h, name.c_str(), k, scaling);
  } else if (type == "Friction") {
    const double k = param_buffer.pop_double(), mu = param_buffer.pop_double();
    const double k_s = param_buffer.pop_double(), dt = param_buffer.pop_double();
    const int scaling = param_buffer.pop_int();
    rc = dem_add_nrot_friction_group(m_h, name.c_str(), k, mu, k_s, dt, scaling);
  } else if (type == "RotFriction" && kRot) {
    const double k = param_buffer.pop_double(), mu_s = param_buffer.pop_double();
    const double mu_d = param_buffer.pop_double(), k_s = param_buffer.pop_double();
    const double dt = param_buffer.pop_double();
    const int scaling = param_buffer.pop_int(), meanR = param_buffer.pop_int();
    rc = dem_add_rot_friction_group(m_h, name.c_str(), k, mu_s, mu_d, k_s, dt, scaling, meanR);
  } else if (type == "HertzMindlin") {
    const double E = param_buffer.pop_double(), nu = param_buffer.pop_double();
    const double mu = param_buffer.pop_double(), dt = param_buffer.pop_double();
    rc = dem_add_hertz_mindlin_group(m_h, name.c_str(), E, nu, mu, dt);
  } else if (type == "HertzMindlinVisco") {
    const double E = param_buffer.pop_double(), nu = param_buffer.pop_double();
    const double mu = param_buffer.pop_double(), cor = param_buffer.pop_double();
    const double dt = param_buffer.pop_double();
    rc = dem_add_hertz_mindlin_visco_group(m_h, name.c_str(), E, nu, mu, cor, dt);
  } else {
    throw std::runtime_error("TGpuSubLattice::addPairIG: interaction type " + type + " is not on the GPU path");
  }
  check(rc, "addPairIG");
  m_dynamic.insert(name);
}

// TSubLattice::addSingleIG (Parallel/SubLattice.hpp:1675-1715): "Gravity" (BodyForceIGP);
// any other type throws as the reference does for a type it does not know.
template <class T>
void TGpuSubLattice<T>::addSingleIG() {
  CVarMPIBuffer param_buffer(m_comm);
  param_buffer.receiveBroadcast(0);
  const std::string type = param_buffer.pop_string();
  if (type != "Gravity")
    throw std::runtime_error("Trying to setup SIG of unknown type: " + type + " (GPU path: Gravity only)");
  const esys::lsm::BodyForceIGP prms = esys::lsm::BodyForceIGP::extract(&param_buffer);
  need_handle("addSingleIG");
  const Vec3 a = prms.getAcceleration();
  const double g[3] = {a.X(), a.Y(), a.Z()};
  check(dem_add_gravity(m_h, prms.getName().c_str(), g), "addSingleIG");
}

// TSubLattice::addBondedIG (Parallel/SubLattice.hpp, CBondedIGP): tag, name, k, rbreak, scaling.
template <class T>
void TGpuSubLattice<T>::addBondedIG() {
  CVarMPIBuffer param_buffer(m_comm);
  param_buffer.receiveBroadcast(0);
  const int tag = param_buffer.pop_int();
  const std::string name = param_buffer.pop_string();
  const double k = param_buffer.pop_double(), rbreak = param_buffer.pop_double();
  const int scaling = param_buffer.pop_int();
  need_handle("addBondedIG");
  check(dem_add_nrot_bond_group(m_h, name.c_str(), tag, k, rbreak, scaling), "addBondedIG");
  m_bonded.insert(name);
}

// TRotSubLattice::addRotBondedIG (Parallel/RotSubLattice.hpp:116-186): tag, name, kr, ks, kt,
// kb, the four breaking limits, scaling, meanR_scaling, truncated; bonds from the stored
// connections of the tag.
template <class T>
void TGpuSubLattice<T>::addRotBondedIG() {
  if (!kRot) unsupported("addRotBondedIG (needs RotSphere particles)");
  CVarMPIBuffer param_buffer(m_comm);
  param_buffer.receiveBroadcast(0);
  const int tag = param_buffer.pop_int();
  const std::string name = param_buffer.pop_string();
  double v[8];
  for (int k = 0; k < 8; ++k) v[k] = param_buffer.pop_double();
  const int scaling = param_buffer.pop_int(), meanR = param_buffer.pop_int();
  const double truncated = param_buffer.pop_double();
  need_handle("addRotBondedIG");
  check(dem_add_rot_bond_group(m_h, name.c_str(), tag, v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], scaling, meanR,
                               truncated),
        "addRotBondedIG");
  m_bonded.insert(name);
}

// TRotSubLattice::addBrittleBeamSCIG (Parallel/RotSubLattice.hpp:189-225).
template <class T>
void TGpuSubLattice<T>::addBrittleBeamSCIG() {
  if (!kRot) unsupported("addBrittleBeamSCIG (needs RotSphere particles)");
  CVarMPIBuffer param_buffer(m_comm);
  param_buffer.receiveBroadcast(0);
  const int tag = param_buffer.pop_int();
  const std::string name = param_buffer.pop_string();
  double v[7];  // kr, ks, kt, kb, cohesion, tCutoff, fAngle
  for (int k = 0; k < 7; ++k) v[k] = param_buffer.pop_double();
  need_handle("addBrittleBeamSCIG");
  check(dem_add_brittle_beam_sc_group(m_h, name.c_str(), tag, v[0], v[1], v[2], v[3], v[4], v[5], v[6]),
        "addBrittleBeamSCIG");
  m_bonded.insert(name);
}

// TRotSubLattice::addBrittleBeamDZCIG (Parallel/RotSubLattice.hpp:228-270).
template <class T>
void TGpuSubLattice<T>::addBrittleBeamDZCIG() {
  if (!kRot) unsupported("addBrittleBeamDZCIG (needs RotSphere particles)");
  CVarMPIBuffer param_buffer(m_comm);
  param_buffer.receiveBroadcast(0);
  const int tag = param_buffer.pop_int();
  const std::string name = param_buffer.pop_string();
  double v[10];  // kr, ks, kt, kb, cohesion, tCutoff, cCutoff, fAngle, beta1, beta2
  for (int k = 0; k < 10; ++k) v[k] = param_buffer.pop_double();
  need_handle("addBrittleBeamDZCIG");
  check(dem_add_brittle_beam_dzc_group(m_h, name.c_str(), tag, v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8],
                                       v[9]),
        "addBrittleBeamDZCIG");
  m_bonded.insert(name);
}

// TSubLattice::addDamping / doAddDamping (Parallel/SubLattice.hpp:1725-1790) and
// TRotSubLattice::doAddDamping (Parallel/RotSubLattice.hpp:79-113).
template <class T>
void TGpuSubLattice<T>::addDamping() {
  CVarMPIBuffer param_buffer(m_comm);
  param_buffer.receiveBroadcast(0);
  const std::string type = param_buffer.pop_string();
  need_handle("addDamping");
  if (type == "Damping" || (kRot && type == "RotDamping")) {
    CDampingIGP* p = extractDampingIGP(&param_buffer);
    const double visc = p->getVisc();
    const int maxit = p->getMaxIter();
    const Vec3 vref = p->getVRef();
    delete p;
    if (vref.norm2() != 0.0) throw std::runtime_error("TGpuSubLattice::addDamping: a reference velocity is not on the GPU path");
    check(dem_add_damping(m_h, type == "RotDamping" ? 1 : 0, visc, maxit), "addDamping");
  } else if (type == "LocalDamping" || (kRot && type == "RotLocalDamping")) {
    CLocalDampingIGP* p = extractLocalDampingIGP(&param_buffer);
    const std::string name = p->getName();
    const double visc = p->getVisc();
    delete p;
    check(dem_add_local_damping(m_h, name.c_str(), type == "RotLocalDamping" ? 1 : 0, visc), "addDamping");
  } else {
    throw std::runtime_error("Trying to setup Damping of unknown type: " + type);
  }
}

// TSubLattice::setExIG (Parallel/SubLattice.hpp:1980-2009): the bonded group s1 excludes its
// pairs from the dynamic group s2; names that name no such groups are reported and ignored.
// (The reference falls back to looking s2 up as the excluding group when s1 is not a bonded
// group; that makes the dynamic group exclude itself, which the GPU path does not do: it is
// reported like a missing group.)
template <class T>
void TGpuSubLattice<T>::setExIG() {
  CVarMPIBuffer pbuffer(m_comm);
  pbuffer.receiveBroadcast(0);
  const std::string s1 = pbuffer.pop_string();
  const std::string s2 = pbuffer.pop_string();
  if (!m_h || !m_bonded.count(s1) || !m_dynamic.count(s2)) {
    console.Error() << "TSubLattice<T>::setExIG() - nonexisting interaction group \n";
    return;
  }
  check(dem_add_exclusion(m_h, s1.c_str(), s2.c_str()), "setExIG");
}

// TSubLattice::checkNeighbors (Parallel/SubLattice.hpp:2473-2520): 1 to the master when a
// particle has moved more than verletDist/2 since the last search.
template <class T>
void TGpuSubLattice<T>::checkNeighbors() {
  CMPISGBufferLeaf buffer(m_comm, 0, 8);
  int res = 0;
  if (m_h) {
    long long c[9] = {0};
    check(dem_get_counters(m_h, c, 9), "checkNeighbors");
    res = c[8] ? 1 : 0;
  }
  buffer.append(res);
  buffer.send();
}

// TSubLattice::searchNeighbors (Parallel/SubLattice.hpp:2395-2408): the search runs on the
// device at the head of the next step.
template <class T>
void TGpuSubLattice<T>::searchNeighbors() {
  CMPIBarrier barrier(getWorkerComm());
  if (m_h) check(dem_search_neighbors(m_h), "searchNeighbors");
  barrier.wait("PPA rebuild");
}

template <class T>
void TGpuSubLattice<T>::rebuildParticleArray() {
  if (m_h) check(dem_search_neighbors(m_h), "rebuildParticleArray");
}

template <class T>
void TGpuSubLattice<T>::rebuildInteractions() {
  if (m_h) check(dem_search_neighbors(m_h), "rebuildInteractions");
}

// TSubLattice::updateInteractions (Parallel/SubLattice.hpp:2415-2470): the library brings the
// bonded, dynamic and wall groups up to date at the head of every step.
template <class T>
void TGpuSubLattice<T>::updateInteractions() {}

// TSubLattice::oneStep (Parallel/SubLattice.hpp:2224-2240): forces, damping, integration.
template <class T>
void TGpuSubLattice<T>::oneStep() {
  need_handle("oneStep");
  check(dem_step(m_h, 1), "oneStep");
}

// TSubLattice::exchangePos: the ghost exchange between workers; one worker has no ghosts.
template <class T>
void TGpuSubLattice<T>::exchangePos() {}

template <class T>
Vec3 TGpuSubLattice<T>::wall_vector(const std::string& name, bool force) {
  if (!m_h || !m_walls.count(name)) return Vec3(0.0, 0.0, 0.0);
  double pos[3], f[3];
  check(dem_get_wall(m_h, name.c_str(), pos, f), force ? "getWallForce" : "getWallPos");
  return force ? Vec3(f[0], f[1], f[2]) : Vec3(pos[0], pos[1], pos[2]);
}

// TSubLattice::getWallPos (Parallel/SubLattice.hpp:835-860): the position gathered to the
// master; a name that names no wall gives (0,0,0).
template <class T>
void TGpuSubLattice<T>::getWallPos() {
  CVarMPIBuffer param_buffer(m_comm);
  param_buffer.receiveBroadcast(0);
  const std::string wname = param_buffer.pop_string();
  std::vector<Vec3> vpos(1, wall_vector(wname, false));
  m_tml_comm.send_gather(vpos, 0);
}

// TSubLattice::getWallForce (Parallel/SubLattice.hpp:897-921).
template <class T>
void TGpuSubLattice<T>::getWallForce() {
  CVarMPIBuffer param_buffer(m_comm);
  param_buffer.receiveBroadcast(0);
  const std::string wname = param_buffer.pop_string();
  std::vector<Vec3> vforce(1, wall_vector(wname, true));
  m_tml_comm.send_gather(vforce, 0);
}

// TSubLattice::moveWallBy (Parallel/SubLattice.hpp:2878-2891): an unknown wall is ignored.
template <class T>
void TGpuSubLattice<T>::moveWallBy() {
  CVarMPIBuffer buffer(m_comm);
  buffer.receiveBroadcast(0);
  const std::string wname = buffer.pop_string();
  const Vec3 mv = buffer.pop_vector();
  if (!m_h || !m_walls.count(wname)) return;
  const double d[3] = {mv.X(), mv.Y(), mv.Z()};
  check(dem_move_wall(m_h, wname.c_str(), d), "moveWallBy");
}

// TSubLattice::applyForceToWall (Parallel/SubLattice.hpp:2935-2948): by wall-group name.
template <class T>
void TGpuSubLattice<T>::applyForceToWall() {
  CVarMPIBuffer buffer(m_comm);
  buffer.receiveBroadcast(0);
  const std::string wname = buffer.pop_string();
  const Vec3 f = buffer.pop_vector();
  if (!m_h || !m_wall_groups.count(wname)) return;
  const double fv[3] = {f.X(), f.Y(), f.Z()};
  check(dem_apply_force_to_wall(m_h, wname.c_str(), fv), "applyForceToWall");
}

// TSubLattice::setVelocityOfWall (Parallel/SubLattice.hpp:2955-2968): only viscous wall groups
// take a velocity; on an elastic one it is AWallInteractionGroup::setVelocity, which only
// reports the call (Model/WallIG.h:64-68).
template <class T>
void TGpuSubLattice<T>::setVelocityOfWall() {
  CVarMPIBuffer buffer(m_comm);
  buffer.receiveBroadcast(0);
  const std::string wname = buffer.pop_string();
  buffer.pop_vector();
  if (m_wall_groups.count(wname))
    std::cerr << "calling unimplemented function AWallInteractionGroup::setVelocity" << std::endl;
}

// TSubLattice::moveTaggedParticlesBy (Parallel/SubLattice.hpp:2577-2587): tag, displacement.
template <class T>
void TGpuSubLattice<T>::moveTaggedParticlesBy() {
  CVarMPIBuffer buffer(m_comm);
  buffer.receiveBroadcast(0);
  const int tag = buffer.pop_int();
  const Vec3 dx = buffer.pop_vector();
  need_handle("moveTaggedParticlesBy");
  const double d[3] = {dx.X(), dx.Y(), dx.Z()};
  check(dem_move_tagged(m_h, tag, -1, d), "moveTaggedParticlesBy");
}

template <class T>
int TGpuSubLattice<T>::getNumParticles() {
  if (!m_h) return 0;
  const int n = dem_num_particles(m_h);
  check(n, "getNumParticles");
  return n;
}

// TSubLattice::countParticles (Parallel/SubLattice.hpp:3046-3054).
template <class T>
void TGpuSubLattice<T>::countParticles() {
  CMPIVarSGBufferLeaf buffer(m_comm, 0);
  buffer.append(getNumParticles());
  buffer.send();
}

template <class T>
std::vector<typename TGpuSubLattice<T>::Row> TGpuSubLattice<T>::rows() {
  std::vector<Row> out;
  const int n = getNumParticles();
  if (n <= 0) return out;
  std::vector<int> id(n);
  std::vector<double> pos(3 * n), vel(3 * n), angvel(3 * n), quat(4 * n), force(3 * n), moment(3 * n), disp(3 * n);
  const int m = dem_get_particles(m_h, id.data(), pos.data(), vel.data(), kRot ? angvel.data() : NULL,
                                  kRot ? quat.data() : NULL, force.data(), kRot ? moment.data() : NULL);
  check(m, "getParticleData");
  check(dem_particle_vector_field(m_h, "displacement", disp.data()), "getParticleData");
  out.resize(m);
  for (int i = 0; i < m; ++i) {
    Row& r = out[i];
    r.id = id[i];
    r.pos = Vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    r.vel = Vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    r.force = Vec3(force[3 * i], force[3 * i + 1], force[3 * i + 2]);
    r.disp = Vec3(disp[3 * i], disp[3 * i + 1], disp[3 * i + 2]);
    if (kRot) {
      r.angvel = Vec3(angvel[3 * i], angvel[3 * i + 1], angvel[3 * i + 2]);
      r.moment = Vec3(moment[3 * i], moment[3 * i + 1], moment[3 * i + 2]);
      for (int k = 0; k < 4; ++k) r.quat[k] = quat[4 * i + k];
    } else {
      r.quat[0] = 1.0;
      r.quat[1] = r.quat[2] = r.quat[3] = 0.0;
    }
  }
  return out;
}

// The particle the reference worker would hold: the library's state (position, velocity,
// force, spin, moment, orientation; initial position = position less the total displacement)
// with the record kept at receiveParticles (tag, radius, mass, switches).
template <class T>
T TGpuSubLattice<T>::make_particle(const Row& r) const {
  const Record& rec = m_record.at(r.id);
  const Vec3 initpos = r.pos - r.disp;
  if constexpr (kRot) {
    const Quaternion q(r.quat[0], Vec3(r.quat[1], r.quat[2], r.quat[3]));
    CRotParticle p(rec.rad, rec.mass, r.pos, r.pos, initpos, r.vel, r.force, r.id, q, q, 0.4 * rec.mass * rec.rad * rec.rad,
                   r.moment, r.angvel, rec.dyn, rec.rot);
    p.setTag(rec.tag);
    return p;
  } else {
    CParticle p(rec.rad, rec.mass, r.pos, r.pos, initpos, r.vel, r.force, r.id, rec.dyn);
    p.setTag(rec.tag);
    return p;
  }
}

// TSubLattice::findParticleNearestTo (Parallel/SubLattice.hpp:2691-2712).
template <class T>
std::pair<double, int> TGpuSubLattice<T>::findParticleNearestTo(const Vec3& pt) {
  double best = std::numeric_limits<double>::max();
  int id = -1;
  for (const Row& r : rows()) {
    const double d2 = (pt - r.pos).norm2();
    if (d2 < best) { best = d2; id = r.id; }
  }
  return id < 0 ? std::make_pair(std::numeric_limits<double>::max(), -1) : std::make_pair(std::sqrt(best), id);
}

// TSubLattice::getParticlePosn (Parallel/SubLattice.hpp:2724-2742).
template <class T>
std::pair<int, Vec3> TGpuSubLattice<T>::getParticlePosn(int particleId) {
  for (const Row& r : rows())
    if (r.id == particleId) return std::make_pair(particleId, r.pos);
  return std::make_pair(-1, Vec3::ZERO);
}

// TSubLattice::getParticleData (Parallel/SubLattice.hpp:2748-2780): the requested particles
// (all when the id list is empty) to the master as a packed gather.
template <class T>
void TGpuSubLattice<T>::getParticleData(const IdVector& particleIdVector) {
  std::set<int> want(particleIdVector.begin(), particleIdVector.end());
  std::vector<T> particleVector;
  for (const Row& r : rows())
    if (want.empty() || want.count(r.id)) particleVector.push_back(make_particle(r));
  m_tml_comm.send_gather_packed(particleVector, 0);
}

template <class T>
void TGpuSubLattice<T>::do2dCalculations(bool do2d) {
  if (do2d) unsupported("do2dCalculations(true)");
}

template <class T>
void TGpuSubLattice<T>::printStruct() {
  std::cout << "My Rank : " << m_rank << " (GPU sub-lattice, " << getNumParticles() << " particles)\n";
}

template <class T>
void TGpuSubLattice<T>::printData() {
  std::cout << "Data: my rank : " << m_rank << "particles : \n";
  for (const Row& r : rows()) std::cout << r.id << " " << r.pos << " " << r.vel << "\n";
}

// TSubLattice::saveCheckPointData / saveSnapShotData (Parallel/SubLattice.hpp:3552-3673): the
// library writes the worker's file; its text goes to the stream the checkpointer opened.
template <class T>
void TGpuSubLattice<T>::saveCheckPointData(std::ostream& oStream) {
  need_handle("saveCheckPointData");
  const std::string path = esys_gpu_detail::scratch_path("ckpt");
  const int rc = dem_save_checkpoint(m_h, path.c_str(), (int)oStream.precision());
  if (rc >= 0) oStream << std::ifstream(path).rdbuf();
  std::remove(path.c_str());
  check(rc, "saveCheckPointData");
}

template <class T>
void TGpuSubLattice<T>::saveSnapShotData(std::ostream& oStream) {
  need_handle("saveSnapShotData");
  const std::string path = esys_gpu_detail::scratch_path("snap");
  const int rc = dem_save_snapshot(m_h, path.c_str());
  if (rc >= 0) oStream << std::ifstream(path).rdbuf();
  std::remove(path.c_str());
  check(rc, "saveSnapShotData");
}

// TSubLattice::loadCheckPointData (Parallel/SubLattice.hpp:3675-3790) into this worker.
template <class T>
void TGpuSubLattice<T>::loadCheckPointData(std::istream& iStream) {
  need_handle("loadCheckPointData");
  const std::string path = esys_gpu_detail::scratch_path("load");
  {
    std::ofstream f(path);
    f << iStream.rdbuf();
  }
  const int rc = dem_load_checkpoint(m_h, path.c_str(), dem_timestep(m_h));
  std::remove(path.c_str());
  check(rc, "loadCheckPointData");
  // the records of the loaded particles: tag, radius and mass from the library; the switches
  // of particles this worker has not seen before are the defaults (dynamic, rotational)
  const int n = getNumParticles();
  std::vector<double> id(n), tag(n), rad(n), mass(n);
  check(dem_particle_scalar_field(m_h, "id", id.data()), "loadCheckPointData");
  check(dem_particle_scalar_field(m_h, "tag", tag.data()), "loadCheckPointData");
  check(dem_particle_scalar_field(m_h, "radius", rad.data()), "loadCheckPointData");
  check(dem_particle_scalar_field(m_h, "mass", mass.data()), "loadCheckPointData");
  for (int i = 0; i < n; ++i) {
    const int pid = (int)id[i];
    auto it = m_record.find(pid);
    const bool dyn = it == m_record.end() ? true : it->second.dyn;
    const bool rot = it == m_record.end() ? kRot : it->second.rot;
    m_record[pid] = Record{(int)tag[i], rad[i], mass[i], dyn, rot};
  }
}
