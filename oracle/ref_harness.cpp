/*
 * Reference harness: drives ESyS-Particle's OWN hot-path classes (compiled
 * from the reference sources, see oracle/Makefile) through the per-step
 * worker sequence, and exposes the result through a small C ABI so that the
 * tests can compare the CUDA path against the reference itself.
 *
 * Test infrastructure, not product code: only tests/, the smoke check and the
 * bench's CPU-baseline leg load the library this file builds into
 * oracle/_ref/libesys_ref.so.
 *
 * The driver replays, for one worker (mpirun -np 2, mpiDimList=[1,1,1]):
 *   - TSubLattice<T>::zeroForces / calcForces / integrate / oneStep
 *       (Parallel/SubLattice.hpp:2066-2236)
 *   - TSubLattice<T>::rebuildInteractions / searchNeighbors /
 *       updateInteractions / checkNeighbors / resetDisplacements
 *       (Parallel/SubLattice.hpp:2360-2536)
 *   - CLatticeMaster::runOneStep (Parallel/LatticeMaster.cpp:2602-2725):
 *       first call forces a search; then checkNeighbors -> search ->
 *       updateInteractions -> oneStep.
 *   - CLatticeMaster::addParticles / addConnections end with a forced
 *       searchNeighbors (Parallel/LatticeMaster.hpp:329,397).
 * The groups are the reference's own classes: PIS_NE<T,CElasticInteraction>,
 * PIS_ED<CRotParticle,CRotFrictionInteraction>, PIS_EB<CRotParticle,
 * CRotBondedInteraction>, CEWallInteractionGroup<T>, BodyForceGroup<T>,
 * PIS_Single<T,CDamping<T>> and PIS_Single<T,CRotDamping<T>>, kept in
 * name-ordered maps exactly as TSubLattice does (Parallel/SubLattice.h:86-96).
 */
#include <cstring>
#include <fstream>
#include <map>
#include <set>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "Foundation/console.h"
#include "Foundation/vec3.h"
#include "Foundation/Quaternion.h"
#include "Model/BodyForceGroup.h"
#include "Model/BondedInteraction.h"
#include "Model/Damping.h"
#include "Model/DampingIGP.h"
#include "Model/EWallInteractionGroup.h"
#include "Model/ElasticInteraction.h"
#include "Model/FrictionInteraction.h"
#include "Model/HertzMindlinInteraction.h"
#include "Model/HertzMindlinViscoInteraction.h"
#include "Model/BrittleBeamDZC.h"
#include "Model/BrittleBeamSC.h"
#include "Model/LocalDamping.h"
#include "Model/LocalDampingIGP.h"
#include "Model/RotLocalDamping.h"
#include "Model/Particle.h"
#include "Model/RotBondedInteraction.h"
#include "Model/RotDamping.h"
#include "Model/RotFricInteraction.h"
#include "Model/RotParticle.h"
#include "Model/Wall.h"
#include "pis/pi_storage_eb.h"
#include "pis/pi_storage_ed.h"
#include "pis/pi_storage_ne.h"
#include "pis/pi_storage_single.h"
#include "ppa/src/pp_array.h"
#include "tml/comm/comm.h"

namespace {

/* Give the harness read access to an interaction storage's list. */
template <class Base>
struct Exposed : public Base {
  template <class... A>
  explicit Exposed(A&&... a) : Base(std::forward<A>(a)...) {}
  auto& list() { return this->m_interactions; }
};

struct BreakEvent { int id1, id2, step; };

/* Read access to CFrictionInteraction's tangential force and flags (protected members), through
 * pointers to members formed in a derived class. */
/* The same for CHertzMindlinInteraction. */
struct HMAccess : CHertzMindlinInteraction {
  static Vec3 CHertzMindlinInteraction::*ffric() { return &HMAccess::m_Ffric; }
  static bool CHertzMindlinInteraction::*slipping() { return &HMAccess::m_is_slipping; }
  static bool CHertzMindlinInteraction::*touching() { return &HMAccess::m_is_touching; }
};

struct FricAccess : CFrictionInteraction {
  static Vec3 CFrictionInteraction::*ffric() { return &FricAccess::m_Ffric; }
  static bool CFrictionInteraction::*slipping() { return &FricAccess::m_is_slipping; }
  static bool CFrictionInteraction::*touching() { return &FricAccess::m_is_touching; }
};

struct ASim {
  virtual ~ASim() {}
  std::string err;
  virtual int add_particles(int n, const int* id, const int* tag, const double* pos, const double* rad,
                            const double* mass, const double* vel, const double* angvel, const double* quat,
                            const int* flags) = 0;
  virtual int add_connections(int n, const int* tag, const int* id1, const int* id2) = 0;
  virtual int add_wall(const char* name, const double* o, const double* nrm) = 0;
  virtual int add_elastic(const char* name, double k, int scaling) = 0;
  virtual int add_rot_friction(const char* name, double k, double mu_s, double mu_d, double ks, double dt,
                               int scaling, int meanR) = 0;
  virtual int add_rot_bond(const char* name, int tag, double kr, double ks, double kt, double kb, double mn,
                           double ms, double mt, double mb, int scaling, int meanR, double trunc) = 0;
  virtual int add_wall_group(const char* name, const char* wall, double k) = 0;
  virtual int add_nrot_friction(const char* name, double k, double mu, double ks, double dt, int scaling) = 0;
  virtual int add_nrot_bond(const char* name, int tag, double k, double rbreak, int scaling) = 0;
  virtual int add_hertz_mindlin(const char* name, double E, double nu, double mu, double dt) = 0;
  virtual int add_hertz_mindlin_visco(const char* name, double E, double nu, double mu, double cor, double dt) = 0;
  virtual int add_brittle_beam_dzc(const char* name, int tag, double kr, double ks, double kt, double kb, double coh,
                                   double tcut, double ccut, double fang, double b1, double b2) = 0;
  virtual int add_brittle_beam_sc(const char* name, int tag, double kr, double ks, double kt, double kb, double coh,
                                  double tcut, double fang) = 0;
  virtual int add_gravity(const char* name, const double* g) = 0;
  virtual int add_damping(int rot, double visc, int maxiter) = 0;
  virtual int add_local_damping(const char* name, int rot, double visc) = 0;
  virtual int add_exclusion(const char* b, const char* d) = 0;
  virtual int step(int n) = 0;
  virtual int move_wall(const char* name, const double* d) = 0;
  virtual int apply_force_to_wall(const char* group, const double* f) = 0;
  virtual int get_wall(const char* name, double* pos, double* force) = 0;
  virtual int num_particles() = 0;
  virtual int get_particles(int* id, double* pos, double* vel, double* angvel, double* quat, double* force,
                            double* moment) = 0;
  virtual int num_pairs(const char* group) = 0;
  virtual int get_pairs(const char* group, int* id1, int* id2, double* state) = 0;
  virtual int num_breaks() = 0;
  virtual int get_breaks(int* id1, int* id2, int* step) = 0;
  virtual int move_tagged(int tag, int mask, const double* d) = 0;
  virtual long long timestep() = 0;
  virtual int save_checkpoint(const char* path, int precision) = 0;
  virtual int load_checkpoint(const char* path, long long timestep) = 0;
};

template <class T>
struct RefSim : public ASim {
  static constexpr bool kRot = std::is_same<T, CRotParticle>::value;
  TML_Comm comm;
  ParallelParticleArray<T>* ppa = nullptr;
  double dt, nrange, alpha;
  std::map<std::string, CWall*> walls;
  std::map<std::string, AWallInteractionGroup<T>*> wig;
  std::map<std::string, AInteractionGroup<T>*> single;
  std::map<std::string, AParallelInteractionStorage*> dpis, bpis, damping;
  std::map<int, std::vector<int>> temp_conn;
  std::vector<BreakEvent> breaks;
  int last_ns = -1;
  long long t = 0;
  bool first = true;
  /* typed handles for queries */
  std::map<std::string, Exposed<ParallelInteractionStorage_NE<T, CElasticInteraction>>*> elastic;
  std::map<std::string, void*> fric, bond, dzc, bsc;
  using DzcPis = Exposed<ParallelInteractionStorage_EB<CRotParticle, BrittleBeamDZCInteraction>>;
  using ScPis = Exposed<ParallelInteractionStorage_EB<CRotParticle, BrittleBeamSCInteraction>>;
  std::map<std::string, Exposed<ParallelInteractionStorage_ED<T, CFrictionInteraction>>*> nfric;
  std::map<std::string, Exposed<ParallelInteractionStorage_EB<T, CBondedInteraction>>*> nbond;
  std::map<std::string, Exposed<ParallelInteractionStorage_NE<T, CHertzMindlinInteraction>>*> hm;
  std::map<std::string, Exposed<ParallelInteractionStorage_NE<T, CHertzMindlinViscoInteraction>>*> hmv;

  RefSim(double gs, double vd, const double* mn, const double* mx, const int* circ, double dt_)
      : comm(MPI_COMM_WORLD), dt(dt_), nrange(gs), alpha(vd) {
    /* TSubLattice::initNeighborTable (Parallel/SubLattice.hpp:455-478, 500-564) */
    Vec3 vmin(mn[0], mn[1], mn[2]), vmax(mx[0], mx[1], mx[2]);
    double size[3];
    for (int i = 0; i < 3; ++i) {
      double s = mx[i] - mn[i];
      size[i] = nrange * ceil(s / nrange);
    }
    Vec3 grow = Vec3(size[0], size[1], size[2]) - (vmax - vmin);
    Vec3 nmin = vmin - 0.5 * grow;
    Vec3 nmax = vmax + 0.5 * grow;
    std::vector<unsigned int> dims(3, 1);
    (void)circ;
    ppa = new ParallelParticleArray<T>(&comm, dims, nmin, nmax, nrange, alpha);
  }

  /* TSubLattice::rebuildInteractions + resetDisplacements (SubLattice.hpp:2360-2389, 2526-2536) */
  void searchNeighbors() {
    ppa->rebuild();
    for (auto& b : bpis) { b.second->exchange(); b.second->rebuild(); }
    for (auto& d : dpis) { d.second->exchange(); d.second->rebuild(); }
    ppa->forAllParticles(&T::resetDisplacement);
  }
  /* TSubLattice::checkNeighbors (SubLattice.hpp:2473-2519) */
  bool checkNeighbors() {
    double mdsqr = 0;
    double a = 0.5 * alpha;
    double srsqr = a * a;
    std::vector<Vec3> displ;
    ppa->forAllParticlesGet(displ, &T::getDisplacement);
    auto it = displ.begin();
    while ((it != displ.end()) && (mdsqr < srsqr)) {
      double sq = (*it) * (*it);
      mdsqr = ((mdsqr < sq) ? sq : mdsqr);
      it++;
    }
    return mdsqr > srsqr;
  }
  template <class PIS>
  void collect_ids(PIS* p, std::set<std::pair<int, int>>& s) {
    for (auto& in : p->list()) { auto v = in.getAllID(); s.insert({v[0], v[1]}); }
  }
  /* TSubLattice::updateInteractions (SubLattice.hpp:2416-2466) */
  void updateInteractions() {
    bool need_update = false;
    for (auto& b : bpis) {
      std::set<std::pair<int, int>> before, after;
      auto collect = [&](std::set<std::pair<int, int>>& s) {
        if (nbond.count(b.first)) {
          collect_ids(nbond[b.first], s);
        } else if (dzc.count(b.first)) {
          collect_ids(static_cast<DzcPis*>(dzc[b.first]), s);
        } else if (bsc.count(b.first)) {
          collect_ids(static_cast<ScPis*>(bsc[b.first]), s);
        } else if constexpr (kRot) {
          collect_ids(static_cast<Exposed<ParallelInteractionStorage_EB<T, CRotBondedInteraction>>*>(bond[b.first]), s);
        }
      };
      collect(before);
      bool n = b.second->update();
      if (n) {
        collect(after);
        for (auto& p : before)
          if (!after.count(p)) breaks.push_back({p.first, p.second, (int)t});
      }
      need_update = need_update || n;
    }
    if ((ppa->getTimeStamp() > last_ns) || need_update) {
      for (auto& d : dpis) { bool n = d.second->update(); need_update = need_update || n; }
      for (auto& w : wig) w.second->Update(ppa);
      for (auto& d : damping) d.second->update();
      last_ns = ppa->getTimeStamp();
    }
  }
  /* TSubLattice::zeroForces / calcForces / integrate (SubLattice.hpp:2066-2218) */
  void oneStep() {
    ppa->forAllParticles(&T::zeroForce);
    for (auto& w : walls) w.second->zeroForce();
    for (auto& w : wig) w.second->calcForces();
    for (auto& s : single) s.second->calcForces();
    for (auto& d : dpis) d.second->calcForces();
    for (auto& b : bpis) b.second->calcForces();
    for (auto& d : damping) d.second->calcForces();
    ppa->forAllParticles(&T::integrate, dt);
    ppa->forAllParticles(&T::rescale);
  }
  /* CLatticeMaster::runOneStep (LatticeMaster.cpp:2602-2725), without savers/runnables */
  int step(int n) override {
    for (int s = 0; s < n; ++s) {
      if (first) { searchNeighbors(); first = false; }
      t++;
      if (checkNeighbors()) searchNeighbors();
      updateInteractions();
      oneStep();
    }
    return 0;
  }

  /* TSubLattice::saveCheckPointData (Parallel/SubLattice.hpp:3600-3673): the reference's own
   * writers (particle array, bonded and saving dynamic storages, walls) in its order. */
  int save_checkpoint(const char* path, int precision) override {
    std::ofstream os(path);
    if (!os) { err = "cannot open checkpoint file"; return -1; }
    os.precision(precision);
    const std::string delim = "\n";
    ppa->saveCheckPointData(os);
    os << bpis.size() << delim;
    for (auto& b : bpis) { b.second->saveCheckPointData(os); os << delim; }
    int count_save = 0;
    for (auto& d : dpis) if (d.second->willSave()) count_save++;
    os << count_save << delim;
    for (auto& d : dpis)
      if (d.second->willSave()) { d.second->saveCheckPointData(os); os << delim; }
    os << "Walls " << walls.size() << delim;
    for (auto& w : walls) { os << w.first << delim; w.second->writeCheckPoint(os, delim); }
    os << "Spheres " << 0 << delim << "TriMesh " << 0 << delim << "Mesh2D " << 0 << delim;
    return os ? 0 : -1;
  }
  /* TSubLattice::loadCheckPointData (Parallel/SubLattice.hpp:3675-3790), then the master's
   * searchNeighbors(true) + updateInteractions (Parallel/LatticeMaster.cpp:780-820).  A wall that
   * the script created is loaded in place, so that its interaction groups keep pointing at it. */
  int load_checkpoint(const char* path, long long timestep) override {
    std::ifstream is(path);
    if (!is) { err = "cannot open checkpoint file"; return -1; }
    ppa->loadCheckPointData(is);
    ppa->rebuild();
    unsigned nb = 0, nd = 0;
    is >> nb;
    if (nb != bpis.size()) { err = "bonded group count differs"; return -1; }
    for (auto& b : bpis) b.second->loadCheckPointData(is);
    is >> nd;
    if (nd != dpis.size()) { err = "dynamic group count differs"; return -1; }
    for (auto& d : dpis) d.second->loadCheckPointData(is);
    std::string token;
    int nw = 0;
    is >> token >> nw;
    if (token != "Walls") { err = "expected Walls"; return -1; }
    for (int i = 0; i < nw; ++i) {
      std::string name;
      is >> name;
      auto it = walls.find(name);
      if (it != walls.end()) {
        it->second->loadCheckPoint(is);
      } else {
        CWall* w = new CWall();
        w->loadCheckPoint(is);
        walls[name] = w;
      }
    }
    t = timestep;
    first = false;
    searchNeighbors();
    updateInteractions();
    return is ? 0 : -1;
  }

  int add_particles(int n, const int* id, const int* tag, const double* pos, const double* rad, const double* mass,
                    const double* vel, const double* angvel, const double* quat, const int* flags) override {
    for (int i = 0; i < n; ++i) {
      Vec3 p(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
      Vec3 v = vel ? Vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]) : Vec3(0, 0, 0);
      bool dyn = !(flags && (flags[i] & 1));
      bool rot = !(flags && (flags[i] & 2));
      if constexpr (kRot) {
        Quaternion q = quat ? Quaternion(quat[4 * i], Vec3(quat[4 * i + 1], quat[4 * i + 2], quat[4 * i + 3]))
                            : Quaternion(1.0, Vec3(0, 0, 0));
        Vec3 w = angvel ? Vec3(angvel[3 * i], angvel[3 * i + 1], angvel[3 * i + 2]) : Vec3(0, 0, 0);
        double inert = 0.4 * mass[i] * rad[i] * rad[i]; /* RotParticle.cpp:34 */
        T part(rad[i], mass[i], p, v, Vec3(0, 0, 0), id[i], q, inert, Vec3(0, 0, 0), w, dyn, rot);
        part.setTag(tag ? tag[i] : 0);
        ppa->insert(part);
      } else {
        T part(rad[i], mass[i], p, v, Vec3(0, 0, 0), id[i], dyn);
        part.setTag(tag ? tag[i] : 0);
        ppa->insert(part);
      }
    }
    searchNeighbors();
    return 0;
  }
  int add_connections(int n, const int* tag, const int* id1, const int* id2) override {
    for (int i = 0; i < n; ++i) { temp_conn[tag[i]].push_back(id1[i]); temp_conn[tag[i]].push_back(id2[i]); }
    searchNeighbors();
    return 0;
  }
  int add_wall(const char* name, const double* o, const double* nrm) override {
    walls[name] = new CWall(Vec3(o[0], o[1], o[2]), Vec3(nrm[0], nrm[1], nrm[2]));
    return 0;
  }
  int add_elastic(const char* name, double k, int scaling) override {
    CElasticIGP p(name, k, scaling != 0);
    auto* s = new Exposed<ParallelInteractionStorage_NE<T, CElasticInteraction>>(ppa, p);
    dpis[name] = s;
    elastic[name] = s;
    return 0;
  }
  int add_rot_friction(const char* name, double k, double mu_s, double mu_d, double ks, double dt_, int scaling,
                       int meanR) override {
    if constexpr (kRot) {
      CRotFrictionIGP p;
      p.setName(name);
      p.k = k; p.mu_s = mu_s; p.mu_d = mu_d; p.k_s = ks; p.dt = dt_;
      p.scaling = scaling != 0; p.rigid = false; p.meanR_scaling = meanR != 0;
      auto* s = new Exposed<ParallelInteractionStorage_ED<T, CRotFrictionInteraction>>(ppa, p);
      dpis[name] = s;
      fric[name] = s;
      return 0;
    }
    err = "RotFriction needs RotSphere particles";
    return -1;
  }
  int add_rot_bond(const char* name, int tag, double kr, double ks, double kt, double kb, double mn, double ms,
                   double mt, double mb, int scaling, int meanR, double trunc) override {
    if constexpr (kRot) {
      /* TRotSubLattice::addRotBondedIG (Parallel/RotSubLattice.hpp:116-186) */
      CRotBondedIGP p;
      p.setName(name);
      p.tag = tag; p.kr = kr; p.ks = ks; p.kt = kt; p.kb = kb;
      p.max_nForce = mn; p.max_shForce = ms; p.max_tMoment = mt; p.max_bMoment = mb;
      p.scaling = scaling != 0; p.meanR_scaling = meanR != 0; p.truncated = trunc;
      auto* s = new Exposed<ParallelInteractionStorage_EB<T, CRotBondedInteraction>>(ppa, p);
      std::vector<int>& conns = temp_conn[tag];
      std::vector<int> vi(2, -1);
      for (size_t i = 0; i + 1 < conns.size(); i += 2) { vi[0] = conns[i]; vi[1] = conns[i + 1]; s->tryInsert(vi); }
      bpis[name] = s;
      bond[name] = s;
      return 0;
    }
    err = "RotBond needs RotSphere particles";
    return -1;
  }
  /* TRotSubLattice::addBrittleBeamDZCIG (Parallel/RotSubLattice.hpp:227-267) */
  int add_brittle_beam_dzc(const char* name, int tag, double kr, double ks, double kt, double kb, double coh,
                           double tcut, double ccut, double fang, double b1, double b2) override {
    if constexpr (kRot) {
      BrittleBeamDZCIGP p(name, kr, ks, kt, kb, coh, fang, tcut, ccut, b1, b2, tag);
      auto* st = new DzcPis(ppa, p);
      std::vector<int>& conns = temp_conn[tag];
      std::vector<int> vi(2, -1);
      for (size_t i = 0; i + 1 < conns.size(); i += 2) { vi[0] = conns[i]; vi[1] = conns[i + 1]; st->tryInsert(vi); }
      bpis[name] = st;
      dzc[name] = st;
      return 0;
    }
    err = "BrittleBeamDZC needs RotSphere particles";
    return -1;
  }
  /* TSubLattice::addPairIG, type "HertzMindlinVisco" (Parallel/SubLattice.hpp:1340-1356) */
  int add_hertz_mindlin_visco(const char* name, double E, double nu, double mu, double cor, double dt_) override {
    CHertzMindlinViscoIGP p(name, E, nu, mu, cor, dt_);
    auto* st = new Exposed<ParallelInteractionStorage_NE<T, CHertzMindlinViscoInteraction>>(ppa, p);
    dpis[name] = st;
    hmv[name] = st;
    return 0;
  }
  /* TRotSubLattice::addBrittleBeamSCIG (Parallel/RotSubLattice.hpp:188-225) */
  int add_brittle_beam_sc(const char* name, int tag, double kr, double ks, double kt, double kb, double coh,
                          double tcut, double fang) override {
    if constexpr (kRot) {
      BrittleBeamSCIGP p(name, kr, ks, kt, kb, coh, fang, tcut, tag);
      auto* st = new ScPis(ppa, p);
      std::vector<int>& conns = temp_conn[tag];
      std::vector<int> vi(2, -1);
      for (size_t i = 0; i + 1 < conns.size(); i += 2) { vi[0] = conns[i]; vi[1] = conns[i + 1]; st->tryInsert(vi); }
      bpis[name] = st;
      bsc[name] = st;
      return 0;
    }
    err = "BrittleBeamSC needs RotSphere particles";
    return -1;
  }
  /* TSubLattice::addPairIG, type "Friction" (Parallel/SubLattice.hpp:1055-1076) */
  int add_nrot_friction(const char* name, double k, double mu, double ks, double dt_, int scaling) override {
    CFrictionIGP p(name, k, mu, ks, dt_, scaling != 0);
    auto* s = new Exposed<ParallelInteractionStorage_ED<T, CFrictionInteraction>>(ppa, p);
    dpis[name] = s;
    nfric[name] = s;
    return 0;
  }
  /* TSubLattice::addPairIG, type "HertzMindlin" (Parallel/SubLattice.hpp:1324-1339) */
  int add_hertz_mindlin(const char* name, double E, double nu, double mu, double dt_) override {
    CHertzMindlinIGP p(name, E, nu, mu, dt_);
    auto* s = new Exposed<ParallelInteractionStorage_NE<T, CHertzMindlinInteraction>>(ppa, p);
    dpis[name] = s;
    hm[name] = s;
    return 0;
  }
  /* TSubLattice::addBondedIG (Parallel/SubLattice.hpp:1791-1831) */
  int add_nrot_bond(const char* name, int tag, double k, double rbreak, int scaling) override {
    CBondedIGP p(name, tag, k, rbreak, scaling != 0);
    auto* s = new Exposed<ParallelInteractionStorage_EB<T, CBondedInteraction>>(ppa, p);
    if (rbreak < 0) s->setUnbreakable(true);
    std::vector<int>& conns = temp_conn[tag];
    std::vector<int> vi(2, -1);
    for (size_t i = 0; i + 1 < conns.size(); i += 2) { vi[0] = conns[i]; vi[1] = conns[i + 1]; s->tryInsert(vi); }
    bpis[name] = s;
    nbond[name] = s;
    return 0;
  }
  int add_wall_group(const char* name, const char* wall, double k) override {
    auto it = walls.find(wall);
    if (it == walls.end()) { err = std::string("wall name '") + wall + "' not found in map of walls"; return -1; }
    CEWallIGP p(name, wall, k);
    auto* g = new CEWallInteractionGroup<T>(&comm, it->second, &p);
    g->Update(ppa);
    wig[name] = g;
    return 0;
  }
  int add_gravity(const char* name, const double* g) override {
    esys::lsm::BodyForceIGP p(name, Vec3(g[0], g[1], g[2]));
    single[name] = new esys::lsm::BodyForceGroup<T>(p, *ppa);
    return 0;
  }
  int add_damping(int rot, double visc, int maxiter) override {
    if (rot) {
      if constexpr (kRot) {
        CDampingIGP p("RotDamping", "RotDamping", visc, dt, maxiter);
        auto* s = new ParallelInteractionStorage_Single<T, CRotDamping<T>>(ppa, p);
        damping["RotDamping"] = s;
        s->update();
        return 0;
      }
      err = "RotDamping needs RotSphere particles";
      return -1;
    }
    CDampingIGP p("Damping", "Damping", visc, dt, maxiter);
    auto* s = new ParallelInteractionStorage_Single<T, CDamping<T>>(ppa, p);
    damping["Damping"] = s;
    s->update();
    return 0;
  }
  /* TSubLattice::doAddDamping "LocalDamping" (Parallel/SubLattice.hpp:1765-1769) and
   * TRotSubLattice::doAddDamping "RotLocalDamping" (Parallel/RotSubLattice.hpp:95-104) */
  int add_local_damping(const char* name, int rot, double visc) override {
    if (rot) {
      if constexpr (kRot) {
        CLocalDampingIGP p("RotLocalDamping", name, visc, dt);
        auto* s = new ParallelInteractionStorage_Single<T, CRotLocalDamping<T>>(ppa, p);
        damping["RotLocalDamping"] = s;
        s->update();
        return 0;
      }
      err = "RotLocalDamping needs RotSphere particles";
      return -1;
    }
    CLocalDampingIGP p("LocalDamping", name, visc, dt);
    auto* s = new ParallelInteractionStorage_Single<T, CLocalDamping<T>>(ppa, p);
    damping[name] = s;
    s->update();
    return 0;
  }
  /* TSubLattice::setExIG (Parallel/SubLattice.hpp:1980-2009) */
  int add_exclusion(const char* s1, const char* s2) override {
    auto ex = bpis.find(s1);
    if (ex == bpis.end()) { ex = dpis.find(s2); if (ex == dpis.end()) { err = "nonexisting interaction group"; return -1; } }
    auto dy = dpis.find(s2);
    if (dy == dpis.end()) { err = "nonexisting interaction group"; return -1; }
    dy->second->addExIG(ex->second);
    return 0;
  }
  int move_wall(const char* name, const double* d) override {
    auto it = walls.find(name);
    if (it == walls.end()) { err = "no such wall"; return -1; }
    it->second->moveBy(Vec3(d[0], d[1], d[2]));
    return 0;
  }
  int apply_force_to_wall(const char* group, const double* f) override {
    auto it = wig.find(group);
    if (it == wig.end()) { err = "no such wall group"; return -1; }
    it->second->applyForce(Vec3(f[0], f[1], f[2]));
    return 0;
  }
  int get_wall(const char* name, double* pos, double* force) override {
    auto it = walls.find(name);
    if (it == walls.end()) { err = "no such wall"; return -1; }
    Vec3 p = it->second->getPos(), f = it->second->getForce();
    for (int i = 0; i < 3; ++i) { if (pos) pos[i] = p[i]; if (force) force[i] = f[i]; }
    return 0;
  }
  int num_particles() override { return ppa->size(); }
  int get_particles(int* id, double* pos, double* vel, double* angvel, double* quat, double* force,
                    double* moment) override {
    auto plh = ppa->getAllParticles();
    int i = 0;
    for (auto it = plh->begin(); it != plh->end(); ++it, ++i) {
      T* p = *it;
      if (id) id[i] = p->getID();
      for (int k = 0; k < 3; ++k) {
        if (pos) pos[3 * i + k] = p->getPos()[k];
        if (vel) vel[3 * i + k] = p->getVel()[k];
        if (force) force[3 * i + k] = p->getForce()[k];
      }
      if constexpr (kRot) {
        for (int k = 0; k < 3; ++k) {
          if (angvel) angvel[3 * i + k] = p->getAngVel()[k];
          if (moment) moment[3 * i + k] = p->getMoment()[k];
        }
        if (quat) {
          Quaternion q = p->getQuat();
          quat[4 * i] = q.return_sca();
          for (int k = 0; k < 3; ++k) quat[4 * i + 1 + k] = q.return_vec()[k];
        }
      } else {
        for (int k = 0; k < 3; ++k) {
          if (angvel) angvel[3 * i + k] = 0.0;
          if (moment) moment[3 * i + k] = 0.0;
        }
        if (quat) { quat[4 * i] = 1.0; quat[4 * i + 1] = quat[4 * i + 2] = quat[4 * i + 3] = 0.0; }
      }
    }
    return i;
  }
  int num_pairs(const char* group) override {
    if (elastic.count(group)) return (int)elastic[group]->list().size();
    if (nfric.count(group)) return (int)nfric[group]->list().size();
    if (hm.count(group)) return (int)hm[group]->list().size();
    if (hmv.count(group)) return (int)hmv[group]->list().size();
    if (nbond.count(group)) return (int)nbond[group]->list().size();
    if (dzc.count(group)) return (int)static_cast<DzcPis*>(dzc[group])->list().size();
    if (bsc.count(group)) return (int)static_cast<ScPis*>(bsc[group])->list().size();
    if constexpr (kRot) {
      if (fric.count(group))
        return (int)static_cast<Exposed<ParallelInteractionStorage_ED<T, CRotFrictionInteraction>>*>(fric[group])->list().size();
      if (bond.count(group))
        return (int)static_cast<Exposed<ParallelInteractionStorage_EB<T, CRotBondedInteraction>>*>(bond[group])->list().size();
    }
    err = "no such group";
    return -1;
  }
  /* state per pair (5 doubles): friction -> tangential force (3), slipping, touching;
   * elastic -> last force on p2 (3), 0, touching; bond -> force on p1 (3), failure criterion, 0 */
  int get_pairs(const char* group, int* id1, int* id2, double* state) override {
    int i = 0;
    if (nfric.count(group)) {  /* NRotFriction: tangential force (3), slipping, touching */
      for (auto& in : nfric[group]->list()) {
        auto v = in.getAllID();
        id1[i] = v[0]; id2[i] = v[1];
        if (state) {
          const Vec3 f = in.*FricAccess::ffric();
          for (int k = 0; k < 3; ++k) state[5 * i + k] = f[k];
          state[5 * i + 3] = (in.*FricAccess::slipping()) ? 1.0 : 0.0;
          state[5 * i + 4] = (in.*FricAccess::touching()) ? 1.0 : 0.0;
        }
        ++i;
      }
      return i;
    }
    if (hm.count(group)) {  /* HertzMindlin: tangential force (3), slipping, touching */
      for (auto& in : hm[group]->list()) {
        auto v = in.getAllID();
        id1[i] = v[0]; id2[i] = v[1];
        if (state) {
          const Vec3 f = in.*HMAccess::ffric();
          for (int k = 0; k < 3; ++k) state[5 * i + k] = f[k];
          state[5 * i + 3] = (in.*HMAccess::slipping()) ? 1.0 : 0.0;
          state[5 * i + 4] = (in.*HMAccess::touching()) ? 1.0 : 0.0;
        }
        ++i;
      }
      return i;
    }
    if (hmv.count(group)) {  /* HertzMindlinVisco: 0 (3), slipping, sticking + slipping (touching) */
      for (auto& in : hmv[group]->list()) {
        auto v = in.getAllID();
        id1[i] = v[0]; id2[i] = v[1];
        if (state) {
          for (int k = 0; k < 3; ++k) state[5 * i + k] = 0.0;
          state[5 * i + 3] = in.getSlipping();
          state[5 * i + 4] = in.getSlipping() + in.getSticking();
        }
        ++i;
      }
      return i;
    }
    if (dzc.count(group)) {  /* BrittleBeamDZC: force on p1 (3), 0, 0 */
      for (auto& in : static_cast<DzcPis*>(dzc[group])->list()) {
        auto v = in.getAllID();
        id1[i] = v[0]; id2[i] = v[1];
        if (state) { Vec3 f = in.getForce(); for (int k = 0; k < 3; ++k) state[5 * i + k] = f[k]; state[5 * i + 3] = 0; state[5 * i + 4] = 0; }
        ++i;
      }
      return i;
    }
    if (bsc.count(group)) {  /* BrittleBeamSC: force on p1 (3), 0, 0 */
      for (auto& in : static_cast<ScPis*>(bsc[group])->list()) {
        auto v = in.getAllID();
        id1[i] = v[0]; id2[i] = v[1];
        if (state) { Vec3 f = in.getForce(); for (int k = 0; k < 3; ++k) state[5 * i + k] = f[k]; state[5 * i + 3] = 0; state[5 * i + 4] = 0; }
        ++i;
      }
      return i;
    }
    if (nbond.count(group)) {  /* NRotBond: force on p2 (3), failure criterion, 0 */
      for (auto& in : nbond[group]->list()) {
        auto v = in.getAllID();
        id1[i] = v[0]; id2[i] = v[1];
        if (state) { Vec3 f = in.getForce(); for (int k = 0; k < 3; ++k) state[5 * i + k] = f[k]; state[5 * i + 3] = in.getCriterion(); state[5 * i + 4] = 0; }
        ++i;
      }
      return i;
    }
    if (elastic.count(group)) {
      for (auto& in : elastic[group]->list()) {
        auto v = in.getAllID();
        id1[i] = v[0]; id2[i] = v[1];
        if (state) { Vec3 f = in.getForce(); for (int k = 0; k < 3; ++k) state[5 * i + k] = f[k]; state[5 * i + 3] = 0; state[5 * i + 4] = in.Count(); }
        ++i;
      }
      return i;
    }
    if constexpr (kRot) {
      if (fric.count(group)) {
        for (auto& in : static_cast<Exposed<ParallelInteractionStorage_ED<T, CRotFrictionInteraction>>*>(fric[group])->list()) {
          auto v = in.getAllID();
          id1[i] = v[0]; id2[i] = v[1];
          if (state) {
            Vec3 f = in.getTangentialForce();
            for (int k = 0; k < 3; ++k) state[5 * i + k] = f[k];
            state[5 * i + 3] = in.getSlipping();
            state[5 * i + 4] = in.Count();
          }
          ++i;
        }
        return i;
      }
      if (bond.count(group)) {
        for (auto& in : static_cast<Exposed<ParallelInteractionStorage_EB<T, CRotBondedInteraction>>*>(bond[group])->list()) {
          auto v = in.getAllID();
          id1[i] = v[0]; id2[i] = v[1];
          if (state) { Vec3 f = in.getForce(); for (int k = 0; k < 3; ++k) state[5 * i + k] = f[k]; state[5 * i + 3] = in.getCriterion(); state[5 * i + 4] = 0; }
          ++i;
        }
        return i;
      }
    }
    err = "no such group";
    return -1;
  }
  int num_breaks() override { return (int)breaks.size(); }
  int get_breaks(int* id1, int* id2, int* st) override {
    for (size_t i = 0; i < breaks.size(); ++i) { id1[i] = breaks[i].id1; id2[i] = breaks[i].id2; st[i] = breaks[i].step; }
    return (int)breaks.size();
  }
  /* TSubLattice::moveTaggedParticlesBy (Parallel/SubLattice.hpp:2577-2587): exact tag match */
  int move_tagged(int tag, int mask, const double* d) override {
    (void)mask;
    ppa->forParticleTag(tag, (void (T::*)(Vec3))(&T::moveBy), Vec3(d[0], d[1], d[2]));
    return 0;
  }
  long long timestep() override { return t; }
};

}  // namespace

extern "C" {
int ref_create(void** out, int ptype, double gs, double vd, const double* mn, const double* mx, const int* circ,
               double dt) {
  console.SetVerbose(0);
  if (ptype == 0) *out = new RefSim<CParticle>(gs, vd, mn, mx, circ, dt);
  else *out = new RefSim<CRotParticle>(gs, vd, mn, mx, circ, dt);
  return 0;
}
int ref_destroy(void* h) { delete static_cast<ASim*>(h); return 0; }
const char* ref_last_error(void* h) { return static_cast<ASim*>(h)->err.c_str(); }
int ref_add_particles(void* h, int n, const int* id, const int* tag, const double* pos, const double* rad,
                      const double* mass, const double* vel, const double* angvel, const double* quat,
                      const int* flags) {
  return static_cast<ASim*>(h)->add_particles(n, id, tag, pos, rad, mass, vel, angvel, quat, flags);
}
int ref_add_connections(void* h, int n, const int* tag, const int* a, const int* b) {
  return static_cast<ASim*>(h)->add_connections(n, tag, a, b);
}
int ref_add_wall(void* h, const char* name, const double* o, const double* n) { return static_cast<ASim*>(h)->add_wall(name, o, n); }
int ref_add_elastic_group(void* h, const char* name, double k, int scaling) { return static_cast<ASim*>(h)->add_elastic(name, k, scaling); }
int ref_add_rot_friction_group(void* h, const char* name, double k, double mu_s, double mu_d, double ks, double dt,
                               int scaling, int meanR) {
  return static_cast<ASim*>(h)->add_rot_friction(name, k, mu_s, mu_d, ks, dt, scaling, meanR);
}
int ref_add_rot_bond_group(void* h, const char* name, int tag, double kr, double ks, double kt, double kb, double mn,
                           double ms, double mt, double mb, int scaling, int meanR, double trunc) {
  return static_cast<ASim*>(h)->add_rot_bond(name, tag, kr, ks, kt, kb, mn, ms, mt, mb, scaling, meanR, trunc);
}
int ref_add_wall_group(void* h, const char* name, const char* wall, double k) { return static_cast<ASim*>(h)->add_wall_group(name, wall, k); }
int ref_add_hertz_mindlin_group(void* h, const char* name, double E, double nu, double mu, double dt) {
  return static_cast<ASim*>(h)->add_hertz_mindlin(name, E, nu, mu, dt);
}
int ref_add_local_damping(void* h, const char* name, int rot, double visc) {
  return static_cast<ASim*>(h)->add_local_damping(name, rot, visc);
}
int ref_add_nrot_friction_group(void* h, const char* name, double k, double mu, double ks, double dt, int scaling) {
  return static_cast<ASim*>(h)->add_nrot_friction(name, k, mu, ks, dt, scaling);
}
int ref_add_brittle_beam_dzc_group(void* h, const char* name, int tag, double kr, double ks, double kt, double kb,
                                   double coh, double tcut, double ccut, double fang, double b1, double b2) {
  return static_cast<ASim*>(h)->add_brittle_beam_dzc(name, tag, kr, ks, kt, kb, coh, tcut, ccut, fang, b1, b2);
}
int ref_add_brittle_beam_sc_group(void* h, const char* name, int tag, double kr, double ks, double kt, double kb,
                                  double coh, double tcut, double fang) {
  return static_cast<ASim*>(h)->add_brittle_beam_sc(name, tag, kr, ks, kt, kb, coh, tcut, fang);
}
int ref_add_hertz_mindlin_visco_group(void* h, const char* name, double E, double nu, double mu, double cor,
                                      double dt) {
  return static_cast<ASim*>(h)->add_hertz_mindlin_visco(name, E, nu, mu, cor, dt);
}
int ref_add_nrot_bond_group(void* h, const char* name, int tag, double k, double rbreak, int scaling) {
  return static_cast<ASim*>(h)->add_nrot_bond(name, tag, k, rbreak, scaling);
}
int ref_add_gravity(void* h, const char* name, const double* g) { return static_cast<ASim*>(h)->add_gravity(name, g); }
int ref_add_damping(void* h, int rot, double visc, int maxiter) { return static_cast<ASim*>(h)->add_damping(rot, visc, maxiter); }
int ref_add_exclusion(void* h, const char* b, const char* d) { return static_cast<ASim*>(h)->add_exclusion(b, d); }
int ref_step(void* h, int n) { return static_cast<ASim*>(h)->step(n); }
int ref_move_wall(void* h, const char* name, const double* d) { return static_cast<ASim*>(h)->move_wall(name, d); }
int ref_apply_force_to_wall(void* h, const char* g, const double* f) { return static_cast<ASim*>(h)->apply_force_to_wall(g, f); }
int ref_get_wall(void* h, const char* name, double* pos, double* force) { return static_cast<ASim*>(h)->get_wall(name, pos, force); }
int ref_num_particles(void* h) { return static_cast<ASim*>(h)->num_particles(); }
int ref_get_particles(void* h, int* id, double* pos, double* vel, double* angvel, double* quat, double* force,
                      double* moment) {
  return static_cast<ASim*>(h)->get_particles(id, pos, vel, angvel, quat, force, moment);
}
int ref_num_pairs(void* h, const char* g) { return static_cast<ASim*>(h)->num_pairs(g); }
int ref_get_pairs(void* h, const char* g, int* a, int* b, double* st) { return static_cast<ASim*>(h)->get_pairs(g, a, b, st); }
int ref_num_breaks(void* h) { return static_cast<ASim*>(h)->num_breaks(); }
int ref_get_breaks(void* h, int* a, int* b, int* s) { return static_cast<ASim*>(h)->get_breaks(a, b, s); }
int ref_move_tagged(void* h, int tag, int mask, const double* d) { return static_cast<ASim*>(h)->move_tagged(tag, mask, d); }
int ref_save_checkpoint(void* h, const char* path, int precision) { return static_cast<ASim*>(h)->save_checkpoint(path, precision); }
int ref_load_checkpoint(void* h, const char* path, long long t) { return static_cast<ASim*>(h)->load_checkpoint(path, t); }
long long ref_timestep(void* h) { return static_cast<ASim*>(h)->timestep(); }
}

/* BondedInteractionCpData (compiled above for the bond checkpoint record)
 * references this accessor of the thermal bond, whose translation unit pulls
 * in the whole thermal particle family.  Thermal bonds are not on this path,
 * so the accessor is defined here and is never called. */
#include "Model/RotThermBondedInteraction.h"
int CRotThermBondedInteraction::getTag() const { return 0; }
