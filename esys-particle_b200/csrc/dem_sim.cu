// Host side of one simulated worker on one GPU, and the C ABI (include/esys_dem.h).
//
// DemSim plays the role of TSubLattice<T> / TRotSubLattice<T>
// (Parallel/SubLattice.hpp, Parallel/RotSubLattice.hpp) for a single worker:
// it owns every particle and interaction in device memory and replays the
// per-step sequence of CLatticeMaster::runOneStep
// (Parallel/LatticeMaster.cpp:2602-2725) -- neighbour check, rebuild,
// interaction update, force + integration -- as stream-ordered kernels.  The
// force/integration kernel of several consecutive steps is launched without a
// host round trip; a step that needs host work (rebuild, bond-break update)
// raises a control flag that makes the remaining launches of the chunk
// return at once, and the host resumes from there.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/esys_dem.h"
#include "dem_device.cuh"
#include "dem_adjoint.h"
#include "dem_kernels.h"

namespace dem {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
// An operation that the simulation's current state does not allow (DEM_ERR_STATE).
struct StateError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define DEM_CUDA(x)                                                                                    \
  do {                                                                                                 \
    cudaError_t e_ = (x);                                                                              \
    if (e_ != cudaSuccess) throw ::dem::CudaError(std::string(#x) + ": " + cudaGetErrorString(e_));          \
  } while (0)

// Growable device array.
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t cap = 0;
  void reserve(size_t n, bool keep = false, cudaStream_t s = 0) {
    if (n <= cap) return;
    size_t nc = std::max<size_t>(n, cap + cap / 2 + 64);
    T* q = nullptr;
    DEM_CUDA(cudaMalloc(&q, nc * sizeof(T)));
    if (keep && p && cap) DEM_CUDA(cudaMemcpyAsync(q, p, cap * sizeof(T), cudaMemcpyDeviceToDevice, s));
    if (p) { DEM_CUDA(cudaStreamSynchronize(s)); cudaFree(p); }
    p = q;
    cap = nc;
  }
  // Growth with 25 % slack, for buffers sized by a pair count that creeps up from one neighbour
  // rebuild to the next: sized exactly, a list one pair longer than the last one reallocates, and
  // a cudaMalloc / cudaFree of tens of MB inside a rebuild measured 1 to 60 ms on B200.
  void grow(size_t n) {
    if (n > cap) reserve(n + n / 4 + 1024);
  }
  void release() { if (p) cudaFree(p); p = nullptr; cap = 0; }
};

struct Wall {
  double o[3], n[3];
  double old[3];  // CWall::m_oldpos: the origin at creation (restart checkpoints carry it)
};

struct WallGroup {
  std::string wall;
  double k;
};

struct DynGroup {
  int kind;  // 0 elastic, 1 rot friction
  double k = 0, ks = 0, mu_s = 0, mu_d = 0, dt = 0;
  int scaling = 1, meanR = 1;
  std::vector<std::string> excl;  // excluding bond groups
  int m = 0;                      // pairs
  int update_ts = 0;
  DBuf<unsigned long long> keys, keys_spare, cand;
  DBuf<double4> hist[2], hist_spare;  // hist[c]: read by the step whose particle input buffer is c
  DBuf<float4> hist32[2], hist32_spare;  // the same records in the FP32-force form
  DBuf<int> adj_start, adj_count, adj_cursor, p1_start;
  DBuf<int2> adj;
  DBuf<int> xbond;  // device bond hand-off: excluding bond of each pair
  void release() {
    keys.release(); keys_spare.release(); cand.release(); xbond.release();
    hist[0].release(); hist[1].release(); hist_spare.release();
    hist32[0].release(); hist32[1].release(); hist32_spare.release();
    adj_start.release(); adj_count.release(); adj_cursor.release(); p1_start.release(); adj.release();
  }
};

struct BondGroup {
  int kind = 0;                 // 0 RotBond, 1 NRotBond (CBondedInteraction), 2 BrittleBeamDZC, 3 BrittleBeamSC
  double knb = 0, rbreak = 0;   // NRotBond: normalK, relative breaking distance (< 0: unbreakable)
  double cohesion = 0, tan_angle = 0, t_cutoff = 0, c_cutoff = 0, beta1 = 0, beta2 = 0;  // BrittleBeamDZC
  int tag;
  double kr, ks, kt, kb, mn, ms, mt, mb, truncated;
  int scaling, meanR;
  int nb = 0;
  DBuf<unsigned long long> keys;
  DBuf<int2> ends;
  DBuf<double4> D0;
  DBuf<int> broken_step, adj_start, adj_count, adj_cursor, p1_start, events, nevents;
  DBuf<int2> adj;
  DBuf<float4> bf32;  // FP32-force form: the bond pass's FP32 records
  DBuf<double4> bf;  // bond pass results (3 records per bond)
  int cap_events = 0;
  void release() {
    bf.release(); bf32.release();
    keys.release(); ends.release(); D0.release(); broken_step.release(); adj_start.release(); adj_count.release();
    adj_cursor.release(); p1_start.release(); events.release(); nevents.release(); adj.release();
  }
};

struct DemSim {
  std::string err;
  int rot;
  double dt, nrange, alpha;
  Grid g{};
  cudaStream_t s = nullptr;
  int tpp = 0;           // 0 = choose from the mean adjacency length
  int chunk = 64;        // steps launched per host round trip
  int store_forces = 1;
  int fp32 = 0;          // 1 = FP32-force / FP64-integration form
  int split = -1;        // -1 automatic, 0 fused step kernel, 1 pair kernel + integration kernel
  int handoff = 0;       // device bond hand-off (dem_set_option "bond_handoff")
  int bond_pass = 1;     // bonds evaluated once per step by their own pass, then gathered
  int adj_tangents = 0;  // adjoint RotBond VJP: 0 hand-written reverse, else dual tangents per pass
  int adj_pair_duals = 0;  // adjoint pair-law VJPs: 0 hand-written reverse, 1 forward-mode duals
  DBuf<int> d_brk;       // [2]: last step with a bond failure, by step parity
  DBuf<int> d_servo_idx; // wall servo: candidate lists of its threads (n ints)
  DBuf<int> rows, pack_id;  // dem_get_particles: row of each alive slot, packed ids
  DBuf<double> pack;        // dem_get_particles: packed host rows of the wanted fields
  // particles
  int n = 0, cap = 0;
  Particles P{};
  std::vector<int> h_id;                 // slot -> id
  std::vector<double> h_initpos;         // slot -> CParticle::m_initpos (x, y, z), for restart checkpoints
  std::unordered_map<int, int> id2slot;  // id -> slot (of particles ever added)
  int cur = 0;
  // cells
  int ncell = 0;
  DBuf<int> cell_count, cell_start, cell_cursor, cell_list, scratch_i, scratch_j, scalars, scan_tmp;
  // groups (std::map keeps the reference's name order)
  std::map<std::string, Wall> walls;
  std::map<std::string, WallGroup> wig;
  std::map<std::string, std::vector<double>> grav;
  std::map<std::string, DynGroup> dyn;
  std::map<std::string, BondGroup> bond;
  std::map<int, std::vector<int>> temp_conn;
  int damp_lin = 0, damp_rot = 0, iter_lin = 100, iter_rot = 100;
  std::string loc_name;            // LocalDamping group present (its name orders it against "Damping")
  int damp_rotloc = 0;              // RotLocalDamping group present
  double visc_loc = 0.0, visc_rotloc = 0.0;
  double visc_lin = 0, visc_rot = 0;
  // device control
  DBuf<WallDev> d_walls;
  DBuf<double> d_wall_vel, d_wall_partial, d_wall_force;
  std::vector<double> wall_vel;  // per wall name, keyed by wig order at upload
  std::map<std::string, std::vector<double>> wall_loader;  // wall name -> velocity
  DBuf<unsigned> d_block_counter;
  DBuf<long long> d_step;
  DBuf<int> d_ctrl, d_stop;
  int* h_ctrl = nullptr;  // pinned
  long long t = 0;
  int timestamp = 0, last_ns = -1;
  bool first = true;
  int pending_ctrl = 0;   // flags raised on the device that the host has not handled yet
  bool own_stream = true;
  // counters (dem_get_counters)
  long long c_steps = 0, c_contacts = 0, c_rebuilds = 0, c_launches = 0, prof_steps = 0;
  double prof_ms = 0.0;
  bool profile = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  long long wall_cand = 0;               // wall-candidate interactions at the last update
  std::map<std::string, int> bond_alive; // intact bonds per group at the last update
  DBuf<double> stage;                    // host-state staging (dem_set_particles)
  DBuf<double> scratch_d;                // field-saver values
  DBuf<double> sig;                      // BrittleBeamSC: per-slot stress sums of the last step (9 each)
  DBuf<int> stage_slot;

  DemSim() {
    DEM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    DEM_CUDA(cudaMallocHost(&h_ctrl, 4 * sizeof(long long)));
    d_block_counter.reserve(1); d_step.reserve(1); d_ctrl.reserve(1); d_stop.reserve(1); scalars.reserve(8);
    DEM_CUDA(cudaMemsetAsync(d_block_counter.p, 0, sizeof(unsigned), s));
    DEM_CUDA(cudaMemsetAsync(d_step.p, 0, sizeof(long long), s));
    DEM_CUDA(cudaMemsetAsync(d_ctrl.p, 0, sizeof(int), s));
    DEM_CUDA(cudaMemsetAsync(d_stop.p, 0, sizeof(int), s));
    d_wall_force.reserve(kMaxWalls * 3);
    DEM_CUDA(cudaMemsetAsync(d_wall_force.p, 0, sizeof(double) * kMaxWalls * 3, s));
  }
  ~DemSim() {
    cudaStreamSynchronize(s);
    for (auto& d : dyn) d.second.release();
    for (auto& b : bond) b.second.release();
    win.release();
    void* ps[] = {P.buf[0].pr, P.buf[0].vm, P.buf[0].wi, P.buf[0].qq, P.buf[1].pr, P.buf[1].vm, P.buf[1].wi,
                  P.buf[1].qq, P.buf[0].vw, P.buf[1].vw, P.inv, P.oldpos, P.dbound, P.force, P.moment, P.force_eval,
                  P.moment_eval, P.sum_f, P.sum_m, P.pflags, P.flagged, P.id, P.tag, P.cell, P.cshift};
    for (void* p : ps) if (p) cudaFree(p);
    cell_count.release(); cell_start.release(); cell_cursor.release(); cell_list.release();
    scratch_i.release(); scratch_j.release(); scalars.release(); scan_tmp.release();
    d_walls.release(); d_wall_vel.release(); d_wall_partial.release(); d_wall_force.release();
    d_block_counter.release(); d_step.release(); d_ctrl.release(); d_stop.release();
    stage.release(); stage_slot.release(); scratch_d.release(); sig.release(); d_servo_idx.release(); d_brk.release(); rows.release(); pack_id.release();
    pack.release();
    if (h_ctrl) cudaFreeHost(h_ctrl);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (own_stream) cudaStreamDestroy(s);
  }

  void sync() { DEM_CUDA(cudaStreamSynchronize(s)); }
  // Capacity of a bonded group's failure-event log: every bond can fail once, so the
  // default never overflows; the "event_capacity" option sets a fixed size instead.
  int ev_cap = 0;
  int event_cap(int nb) const { return ev_cap > 0 ? ev_cap : std::max(1024, nb); }
  void set_event_capacity(int cap) {
    for (auto& b : bond) {
      BondGroup& B = b.second;
      const int c = cap > 0 ? cap : std::max(1024, B.nb);
      const int ne = read_int(B.nevents.p);
      if (ne > B.cap_events)  // entries past the old capacity were never written
        throw std::invalid_argument("the event log of bonded group '" + b.first + "' has overflowed; its capacity is fixed");
      if (ne > c) throw std::invalid_argument("event_capacity is below the events already logged");
    }
    ev_cap = cap;
    for (auto& b : bond) {
      BondGroup& B = b.second;
      B.cap_events = event_cap(B.nb);
      B.events.reserve(3 * (size_t)B.cap_events, true, s);
    }
    sync();
  }
  int read_int(const int* d) {
    DEM_CUDA(cudaMemcpyAsync(h_ctrl, d, sizeof(int), cudaMemcpyDeviceToHost, s));
    sync();
    return h_ctrl[0];
  }

  // TSubLattice::initNeighborTable (SubLattice.hpp:455-564) + ParallelParticleArray ctor (pp_array.hpp:55-100).
  void init_grid(const double* mn, const double* mx, const int* circ) {
    double size[3];
    bool circx = circ && circ[0];
    for (int i = 0; i < 3; ++i) {
      double sz = mx[i] - mn[i];
      if (i == 0 && circx) {
        if (std::fabs(sz / nrange - std::lrint(sz / nrange)) > 1e-6) nrange = sz / std::floor(sz / nrange);
        size[i] = sz;
      } else {
        size[i] = nrange * std::ceil(sz / nrange);
      }
    }
    double grow[3], nmin[3], nmax[3];
    for (int i = 0; i < 3; ++i) {
      grow[i] = size[i] - (mx[i] - mn[i]);
      nmin[i] = mn[i] - 0.5 * grow[i];
      nmax[i] = mx[i] + 0.5 * grow[i];
    }
    g.p0x = nmin[0]; g.p0y = nmin[1]; g.p0z = nmin[2];
    g.dim = nrange;
    g.alpha = alpha;
    int nxg = (int)std::lrint((nmax[0] - nmin[0]) / nrange);
    int nyg = (int)std::lrint((nmax[1] - nmin[1]) / nrange);
    int nzg = (int)std::lrint((nmax[2] - nmin[2]) / nrange);
    g.circx = circx;
    if (circx) {
      if (nxg < 3) throw std::invalid_argument("periodic x needs at least 3 cells");
      g.gx = 0; g.nx = nxg; g.Lx = nmax[0] - nmin[0]; g.xmin = nmin[0];
    } else {
      g.gx = -1; g.nx = nxg + 2;
    }
    g.gy = -1; g.ny = nyg + 2;
    g.gz = -1; g.nz = nzg + 2;
    ncell = g.nx * g.ny * g.nz;
    cell_count.reserve(ncell + 1); cell_start.reserve(ncell + 1); cell_cursor.reserve(ncell + 1);
  }

  template <class T>
  void grow_array(T*& p, int oldn, int newcap) {
    T* q = nullptr;
    DEM_CUDA(cudaMalloc(&q, sizeof(T) * (size_t)newcap));
    if (p) {
      if (oldn) DEM_CUDA(cudaMemcpyAsync(q, p, sizeof(T) * oldn, cudaMemcpyDeviceToDevice, s));
      sync();
      cudaFree(p);
    }
    p = q;
  }
  void ensure_capacity(int need) {
    if (need <= cap) return;
    int nc = std::max(need, cap + cap / 2 + 1024);
    for (int b = 0; b < 2; ++b) {
      grow_array(P.buf[b].pr, n, nc); grow_array(P.buf[b].vm, n, nc);
      grow_array(P.buf[b].wi, n, nc); grow_array(P.buf[b].qq, n, nc);
      grow_array(P.buf[b].vw, 2 * n, 2 * nc);
    }
    grow_array(P.sum_f, n, nc); grow_array(P.sum_m, n, nc);
    grow_array(P.inv, n, nc); grow_array(P.oldpos, n, nc); grow_array(P.dbound, n, nc); grow_array(P.force, n, nc); grow_array(P.moment, n, nc);
    grow_array(P.pflags, n, nc); grow_array(P.flagged, n, nc); grow_array(P.id, n, nc); grow_array(P.tag, n, nc);
    grow_array(P.cell, n, nc); grow_array(P.cshift, n, nc);
    cap = nc;
  }

  int add_particles(int cnt, const int* id, const int* tag, const double* pos, const double* rad, const double* mass,
                    const double* vel, const double* angvel, const double* quat, const int* flags) {
    std::vector<double4> pr, vm, wi, qq;
    std::vector<double2> inv;
    std::vector<unsigned> pf;
    std::vector<int> ids, tags;
    // Slots follow the caller's order (the reference's particle-list order).  A spatial
    // (Z-curve) slot order was measured: it raised L1 hits but mixed particle sizes
    // within warps and made the step slower on the shear-cell packing.
    for (int i = 0; i < cnt; ++i) {
      // NeighborTable::insert drops particles outside the table (ntable.hpp:243-258)
      auto cc = [&](double x, double p0, int gg) { return int(std::floor((x - p0) / g.dim)) - gg; };
      int ix = cc(pos[3 * i], g.p0x, g.gx), iy = cc(pos[3 * i + 1], g.p0y, g.gy), iz = cc(pos[3 * i + 2], g.p0z, g.gz);
      if (g.circx) ix = ((ix % g.nx) + g.nx) % g.nx;
      if (!(ix >= 0 && ix < g.nx && iy >= 0 && iy < g.ny && iz >= 0 && iz < g.nz)) continue;
      if (id2slot.count(id[i])) throw std::invalid_argument("duplicate particle id " + std::to_string(id[i]));
      if (!(rad[i] > 0) || !(mass[i] > 0)) throw std::invalid_argument("particle radius and mass must be positive");
      pr.push_back(make_double4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], rad[i]));
      vm.push_back(make_double4(vel ? vel[3 * i] : 0.0, vel ? vel[3 * i + 1] : 0.0, vel ? vel[3 * i + 2] : 0.0, mass[i]));
      const double inert = 0.4 * mass[i] * rad[i] * rad[i];  // RotParticle.cpp:34
      bool r_on = rot && !(flags && (flags[i] & 2));
      wi.push_back(make_double4(angvel && rot ? angvel[3 * i] : 0.0, angvel && rot ? angvel[3 * i + 1] : 0.0,
                                angvel && rot ? angvel[3 * i + 2] : 0.0, inert));
      qq.push_back(quat && rot ? make_double4(quat[4 * i], quat[4 * i + 1], quat[4 * i + 2], quat[4 * i + 3])
                               : make_double4(1.0, 0.0, 0.0, 0.0));
      inv.push_back(make_double2(mass[i] != 0.0 ? 1.0 / mass[i] : 0.0, 1.0 / inert));
      unsigned f = PF_ALIVE;
      if (!(flags && (flags[i] & 1))) f |= PF_DYN;
      if (r_on) f |= PF_ROT;
      pf.push_back(f);
      ids.push_back(id[i]);
      tags.push_back(tag ? tag[i] : 0);
    }
    const int add = (int)pr.size();
    ensure_capacity(n + add);
    if (add) {
      auto up = [&](void* dst, const void* src, size_t bytes) {
        DEM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
      };
      up(P.buf[cur].pr + n, pr.data(), sizeof(double4) * add);
      up(P.buf[cur].vm + n, vm.data(), sizeof(double4) * add);
      up(P.buf[cur].wi + n, wi.data(), sizeof(double4) * add);
      up(P.buf[cur].qq + n, qq.data(), sizeof(double4) * add);
      up(P.inv + n, inv.data(), sizeof(double2) * add);
      up(P.pflags + n, pf.data(), sizeof(unsigned) * add);
      up(P.id + n, ids.data(), sizeof(int) * add);
      up(P.tag + n, tags.data(), sizeof(int) * add);
      DEM_CUDA(cudaMemsetAsync(P.flagged + n, 0, add, s));
      DEM_CUDA(cudaMemsetAsync(P.force + n, 0, sizeof(double4) * add, s));
      DEM_CUDA(cudaMemsetAsync(P.moment + n, 0, sizeof(double4) * add, s));
      DEM_CUDA(cudaMemsetAsync(P.cshift + n, 0, sizeof(double) * add, s));
      for (int i = 0; i < add; ++i) {
        id2slot[ids[i]] = n + i;
        h_id.push_back(ids[i]);
        h_initpos.insert(h_initpos.end(), {pr[i].x, pr[i].y, pr[i].z});
      }
      n += add;
      P.n = n;
      sync();
    }
    search_neighbors();  // CLatticeMaster::addParticles ends with searchNeighbors(true) (LatticeMaster.hpp:329)
    resize_adjacency();
    return 0;
  }

  // Per-particle adjacency arrays are sized by the particle count: re-derive them
  // whenever particles are added or a group is created.
  void resize_adjacency() {
    for (auto& d : dyn) {
      build_adjacency(d.second.keys, d.second.m, d.second.adj_start, d.second.adj_count, d.second.adj_cursor,
                      d.second.p1_start, d.second.adj);
      if (handoff) mark_handoff(d.second);
    }
    for (auto& b : bond) build_adjacency(b.second.keys, b.second.nb, b.second.adj_start, b.second.adj_count,
                                         b.second.adj_cursor, b.second.p1_start, b.second.adj);
    sync();
  }

  // Switch between the FP64 form and the FP32-force form, converting friction history.
  void set_precision(int want) {
    want = want ? 1 : 0;
    if (want == fp32) return;
    if (want) {
      for (auto& d : dyn)
        if (d.second.kind >= 2) throw std::invalid_argument("NRotFriction and HertzMindlin groups run in the FP64 form only");
      if (has_sc()) throw std::invalid_argument("BrittleBeamSC groups run in the FP64 form only");
    }
    for (auto& d : dyn) {
      DynGroup& G = d.second;
      if (G.kind == 0 || G.m == 0) continue;
      const int m = G.m;
      for (int b = 0; b < 2; ++b) { G.hist[b].reserve(m); G.hist32[b].reserve(m); }
      launch_hist_convert(m, G.hist[cur].p, G.hist32[cur].p, want == 1, s);
    }
    sync();
    fp32 = want;
  }

  // Precision check of the FP32-force form on the current state of an FP64 run:
  // FP32 forces of this state (evaluation pass), then one FP64 step; returns
  // [0] max|dF| / max|F|, [1] max|dM| / max|M|, [2] median and [3] 99th percentile of
  // |dF_i| / |F_i| over particles with |F_i| > 1e-9 max|F|, [4] particles compared.
  void precision_check(double* out) {
    if (fp32) throw std::invalid_argument("precision check runs from the FP64 form");
    if (!prepare()) throw StateError(err);
    if (!P.force_eval) {
      DEM_CUDA(cudaMalloc(&P.force_eval, sizeof(double4) * (size_t)cap));
      DEM_CUDA(cudaMalloc(&P.moment_eval, sizeof(double4) * (size_t)cap));
    }
    const int t_pp = pick_tpp();
    d_wall_partial.reserve((size_t)step_grid(n, t_pp) * kMaxWalls * 3);
    launch_sync_vw(P, cur, s);
    StepArgs ea = make_args(cur);
    launch_step_fp32(ea, rot != 0, t_pp, true, false, s);
    const int keep = chunk;
    chunk = 1;
    step(1);
    chunk = keep;
    std::vector<double4> f(n), fe(n), m(n), me(n);
    std::vector<unsigned> pf(n);
    DEM_CUDA(cudaMemcpyAsync(f.data(), P.force, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
    DEM_CUDA(cudaMemcpyAsync(fe.data(), P.force_eval, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
    DEM_CUDA(cudaMemcpyAsync(m.data(), P.moment, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
    DEM_CUDA(cudaMemcpyAsync(me.data(), P.moment_eval, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
    DEM_CUDA(cudaMemcpyAsync(pf.data(), P.pflags, sizeof(unsigned) * n, cudaMemcpyDeviceToHost, s));
    sync();
    auto nrm = [](const double4& a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); };
    auto dif = [](const double4& a, const double4& b) {
      const double x = a.x - b.x, y = a.y - b.y, z = a.z - b.z;
      return std::sqrt(x * x + y * y + z * z);
    };
    double fmax = 0, mmax = 0, dfmax = 0, dmmax = 0;
    for (int i = 0; i < n; ++i) {
      if (!(pf[i] & PF_ALIVE)) continue;
      fmax = std::max(fmax, nrm(f[i])); mmax = std::max(mmax, nrm(m[i]));
      dfmax = std::max(dfmax, dif(f[i], fe[i])); dmmax = std::max(dmmax, dif(m[i], me[i]));
    }
    std::vector<double> rel;
    double gmax = 0.0, grel = 0.0;
    for (int i = 0; i < n; ++i) {
      if (!(pf[i] & PF_ALIVE)) continue;
      const double a = nrm(f[i]);
      if (a > 1e-9 * fmax) rel.push_back(dif(f[i], fe[i]) / a);
      gmax = std::max(gmax, fe[i].w);
    }
    for (int i = 0; i < n; ++i)
      if ((pf[i] & PF_ALIVE) && fe[i].w > 1e-9 * gmax) grel = std::max(grel, dif(f[i], fe[i]) / fe[i].w);
    std::sort(rel.begin(), rel.end());
    out[0] = fmax > 0 ? dfmax / fmax : 0.0;
    out[1] = mmax > 0 ? dmmax / mmax : 0.0;
    out[2] = rel.empty() ? 0.0 : rel[rel.size() / 2];
    out[3] = rel.empty() ? 0.0 : rel[std::min(rel.size() - 1, (size_t)(0.99 * rel.size()))];
    out[4] = (double)rel.size();
    out[5] = gmax > 0 ? dfmax / gmax : 0.0;  // relative to the largest contact-force sum
    out[6] = grel;                           // worst particle, relative to its own contact-force sum
  }

  // Bulk state update of existing particles (rows = slots when id is NULL).
  int set_particles(int cnt, const int* id, const double* pos, const double* vel, const double* angvel,
                    const double* quat) {
    if (cnt < 0 || (!id && cnt != n)) throw std::invalid_argument("without ids, rows must cover every particle slot");
    stage.reserve((size_t)cnt * 13 + 1);
    stage_slot.reserve(cnt + 1);
    double* d = stage.p;
    const size_t c3 = (size_t)cnt * 3;
    if (pos) DEM_CUDA(cudaMemcpyAsync(d, pos, sizeof(double) * c3, cudaMemcpyHostToDevice, s));
    if (vel) DEM_CUDA(cudaMemcpyAsync(d + c3, vel, sizeof(double) * c3, cudaMemcpyHostToDevice, s));
    if (angvel && rot) DEM_CUDA(cudaMemcpyAsync(d + 2 * c3, angvel, sizeof(double) * c3, cudaMemcpyHostToDevice, s));
    if (quat && rot) DEM_CUDA(cudaMemcpyAsync(d + 3 * c3, quat, sizeof(double) * 4 * cnt, cudaMemcpyHostToDevice, s));
    const int* slots = nullptr;
    if (id) {
      std::vector<int> sl(cnt);
      for (int i = 0; i < cnt; ++i) {
        auto it = id2slot.find(id[i]);
        if (it == id2slot.end()) throw std::invalid_argument("unknown particle id " + std::to_string(id[i]));
        sl[i] = it->second;
      }
      DEM_CUDA(cudaMemcpyAsync(stage_slot.p, sl.data(), sizeof(int) * cnt, cudaMemcpyHostToDevice, s));
      sync();
      slots = stage_slot.p;
    }
    launch_set_state(P, cur, cnt, slots, pos ? d : nullptr, vel ? d + c3 : nullptr,
                     (angvel && rot) ? d + 2 * c3 : nullptr, (quat && rot) ? d + 3 * c3 : nullptr, s);
    // moved particles are checked like any displacement before the next step
    launch_check_disp(P, cur, (0.5 * alpha) * (0.5 * alpha), d_ctrl.p, s);
    pending_ctrl |= read_int(d_ctrl.p);
    DEM_CUDA(cudaMemsetAsync(d_ctrl.p, 0, sizeof(int), s));
    c_launches += 2;
    return 0;
  }

  // Particles deleted when they left the local grid come back alive with the given state
  // (known ids only; alive ones are only updated).  A neighbour search is scheduled, which
  // rebuilds their cells, pairs and wall candidacy.
  int revive_particles(int cnt, const int* id, const double* pos, const double* vel, const double* angvel,
                       const double* quat) {
    if (cnt <= 0) return 0;
    if (!id) throw std::invalid_argument("revive needs particle ids");
    set_particles(cnt, id, pos, vel, angvel, quat);  // uploads the slots to stage_slot
    launch_set_alive(P, cnt, stage_slot.p, s);
    pending_ctrl |= CTRL_REBUILD;
    sync();
    c_launches += 1;
    return 0;
  }

  // The alive particles in slot order into the caller's host arrays (each may be null).  The
  // rows are packed on the device, then each wanted field is one copy into the caller's array
  // (direct DMA when the caller's memory is pinned).
  int get_particles(int* id, double* pos, double* vel, double* angvel, double* quat, double* force, double* moment) {
    if (!n) return 0;
    rows.reserve((size_t)n + 1);
    pack_id.reserve((size_t)n + 1);
    scan_tmp.reserve(scan_tmp_ints(n + 1));
    launch_alive_flags(P, pack_id.p, s);  // flags, then the scan's input is free for the ids
    launch_scan(pack_id.p, rows.p, n, scalars.p + 2, scan_tmp.p, s);
    const int k = read_int(scalars.p + 2);
    const int* rp = k == n ? nullptr : rows.p;  // every slot alive: row = slot
    pack.reserve((size_t)19 * n + 1);
    double* d = pack.p;
    const size_t n3 = (size_t)n * 3;
    double* dpos = pos ? d : nullptr;
    double* dvel = vel ? d + n3 : nullptr;
    double* dang = angvel ? d + 2 * n3 : nullptr;
    double* dfor = force ? d + 3 * n3 : nullptr;
    double* dmom = moment ? d + 4 * n3 : nullptr;
    double* dq = quat ? d + 5 * n3 : nullptr;
    launch_pack_particles(P, cur, rot, rp, id ? pack_id.p : nullptr, dpos, dvel, dang, dq, dfor, dmom, s);
    const size_t k3 = (size_t)k * 3 * sizeof(double);
    if (id) DEM_CUDA(cudaMemcpyAsync(id, pack_id.p, sizeof(int) * (size_t)k, cudaMemcpyDeviceToHost, s));
    if (pos) DEM_CUDA(cudaMemcpyAsync(pos, dpos, k3, cudaMemcpyDeviceToHost, s));
    if (vel) DEM_CUDA(cudaMemcpyAsync(vel, dvel, k3, cudaMemcpyDeviceToHost, s));
    if (angvel) DEM_CUDA(cudaMemcpyAsync(angvel, dang, k3, cudaMemcpyDeviceToHost, s));
    if (quat) DEM_CUDA(cudaMemcpyAsync(quat, dq, (size_t)k * 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (force) DEM_CUDA(cudaMemcpyAsync(force, dfor, k3, cudaMemcpyDeviceToHost, s));
    if (moment) DEM_CUDA(cudaMemcpyAsync(moment, dmom, k3, cudaMemcpyDeviceToHost, s));
    sync();
    c_launches += 3;
    return k;
  }

  // ---- neighbour search (TSubLattice::searchNeighbors, SubLattice.hpp:2395-2408) ----
  void search_neighbors() {
    DEM_CUDA(cudaMemsetAsync(cell_count.p, 0, sizeof(int) * (ncell + 1), s));
    launch_bin(g, P, cur, cell_count.p, s);
    scan_tmp.reserve(scan_tmp_ints(std::max(ncell + 1, n + 2)));
    launch_scan(cell_count.p, cell_start.p, ncell + 1, scalars.p, scan_tmp.p, s);
    DEM_CUDA(cudaMemsetAsync(cell_cursor.p, 0, sizeof(int) * (ncell + 1), s));
    cell_list.reserve(std::max(n, 1));
    launch_scatter_cells(P, cell_start.p, cell_cursor.p, cell_list.p, s);
    launch_sort_cells(ncell, cell_start.p, cell_list.p, s);
    for (auto& b : bond) launch_bonds_rebuild(b.second.nb, b.second.ends.p, P.pflags, b.second.broken_step.p, s);
    timestamp++;
    c_rebuilds++;
    c_launches += 4 + (long long)bond.size();
  }

  ExclDev excl_of(const DynGroup& G) {
    ExclDev ex{};
    for (auto& nm : G.excl) {
      auto it = bond.find(nm);
      if (it == bond.end() || ex.n >= kMaxBond) continue;
      ex.keys[ex.n] = it->second.keys.p;
      ex.broken_step[ex.n] = it->second.broken_step.p;
      ex.count[ex.n] = it->second.nb;
      ex.group[ex.n] = (int)std::distance(bond.begin(), it);
      ex.n++;
    }
    return ex;
  }

  void build_adjacency(DBuf<unsigned long long>& keys, int m, DBuf<int>& adj_start, DBuf<int>& adj_count,
                       DBuf<int>& adj_cursor, DBuf<int>& p1_start, DBuf<int2>& adj) {
    adj_start.reserve(n + 2); adj_count.reserve(n + 2); adj_cursor.reserve(n + 2); p1_start.reserve(n + 2);
    adj.grow(std::max(2 * m, 1));
    scan_tmp.reserve(scan_tmp_ints(n + 2));
    launch_adj(keys.p, m, n, adj_count.p, p1_start.p, adj_start.p, adj_cursor.p, adj.p, scalars.p + 1, scan_tmp.p, s);
    c_launches += 5;
  }

  // PIS_NE::update / PIS_ED::update after a rebuild: the full pair list with history carried
  // for persistent RotFriction interactions (pi_storage_ne.hpp:49-80, pi_storage_ed.hpp:84-129).
  void dyn_full_update(DynGroup& G) {
    // with the device hand-off the list keeps the bond-excluded pairs (marked by mark_handoff)
    const ExclDev ex = handoff ? ExclDev{} : excl_of(G);
    scratch_i.reserve(n + 1); scratch_j.reserve(n + 1);
    launch_pairs_count(g, P, cur, cell_start.p, cell_list.p, ex, scratch_i.p, s);
    scan_tmp.reserve(scan_tmp_ints(n + 2));
    launch_scan(scratch_i.p, scratch_j.p, n, scalars.p, scan_tmp.p, s);
    const int m = read_int(scalars.p);
    c_launches += 3;
    check_list_size(m);
    G.keys_spare.grow(std::max(m, 1));
    if (G.kind != 0) G.hist_spare.grow(std::max(m, 1));
    if (fp32) {
      if (G.kind != 0) G.hist32_spare.grow(std::max(m, 1));
      launch_pairs_write<float4>(g, P, cur, cell_start.p, cell_list.p, ex, scratch_j.p, G.keys_spare.p, hist_mode(G),
                                 G.keys.p, G.m, G.hist32[cur].p, G.hist32_spare.p, s);
    } else {
      launch_pairs_write<double4>(g, P, cur, cell_start.p, cell_list.p, ex, scratch_j.p, G.keys_spare.p, hist_mode(G),
                                  G.keys.p, G.m, G.hist[cur].p, G.hist_spare.p, s);
    }
    std::swap(G.keys, G.keys_spare);
    if (G.kind != 0) {
      if (fp32) {
        std::swap(G.hist32[cur], G.hist32_spare);
        G.hist32[cur ^ 1].grow(std::max(m, 1));
      } else {
        std::swap(G.hist[cur], G.hist_spare);
        G.hist[cur ^ 1].grow(std::max(m, 1));
      }
    }
    G.m = m;
    build_adjacency(G.keys, m, G.adj_start, G.adj_count, G.adj_cursor, G.p1_start, G.adj);
    if (handoff) mark_handoff(G);
  }

  // A dynamic group's adjacency entries hold the pair index in 30 bits (kAdjIndex).
  static void check_list_size(long long m) {
    if (m > (long long)kAdjIndex + 1) throw StateError("a dynamic interaction group would hold more than 2^30 pairs");
  }

  // Device bond hand-off: per pair of the list the intact bond that excludes it (xbond) and
  // kAdjHeld on the pair's two adjacency entries.  Run after every build of the group's
  // adjacency while the hand-off is on.
  void mark_handoff(DynGroup& G) {
    G.xbond.grow(std::max(G.m, 1));
    launch_pairs_xbond(G.keys.p, G.m, excl_of(G), G.xbond.p, s);
    launch_adj_mark_held(2 * G.m, G.xbond.p, G.adj.p, s);
    c_launches += 2;
  }

  // PIS_NE / PIS_ED::update without a rebuild: append the "new list" of flagged pairs
  // (ntable.hpp:628-664; pi_storage_ne.hpp:80-98, pi_storage_ed.hpp:130-155).
  void dyn_new_update(DynGroup& G) {
    ExclDev ex = excl_of(G);
    const int check_in = G.kind == 1 || G.kind == 2;  // PIS_ED tests isIn; PIS_NE appends without it
    scratch_i.reserve(n + 1); scratch_j.reserve(n + 1);
    launch_newlist_count(g, P, cell_start.p, cell_list.p, ex, G.keys.p, G.m, check_in, scratch_i.p, s);
    scan_tmp.reserve(scan_tmp_ints(n + 2));
    launch_scan(scratch_i.p, scratch_j.p, n, scalars.p, scan_tmp.p, s);
    const int nb = read_int(scalars.p);
    c_launches += 3;
    if (nb > 0) {
      c_launches += 2;
      G.cand.grow(nb);
      launch_newlist_write(g, P, cell_start.p, cell_list.p, ex, G.keys.p, G.m, check_in, scratch_j.p, G.cand.p, s);
      check_list_size((long long)G.m + nb);
      const int m2 = G.m + nb;
      G.keys_spare.grow(m2);
      if (fp32) {
        if (G.kind != 0) G.hist32_spare.grow(m2);
        launch_merge<float4>(G.keys.p, G.hist32[cur].p, G.m, G.cand.p, nb, G.keys_spare.p, G.hist32_spare.p, G.kind != 0 ? 1 : 0, s);
      } else {
        if (G.kind != 0) G.hist_spare.grow(m2);
        launch_merge<double4>(G.keys.p, G.hist[cur].p, G.m, G.cand.p, nb, G.keys_spare.p, G.hist_spare.p, G.kind != 0 ? 1 : 0, s);
      }
      std::swap(G.keys, G.keys_spare);
      if (G.kind != 0) {
        if (fp32) {
          std::swap(G.hist32[cur], G.hist32_spare);
          G.hist32[cur ^ 1].grow(m2);
        } else {
          std::swap(G.hist[cur], G.hist_spare);
          G.hist[cur ^ 1].grow(m2);
        }
      }
      G.m = m2;
      build_adjacency(G.keys, G.m, G.adj_start, G.adj_count, G.adj_cursor, G.p1_start, G.adj);
    }
    launch_clear_flags(n, P.flagged, s);  // getNewList clears every flag (ntable.hpp:658-662)
  }

  void upload_walls() {
    std::vector<WallDev> w;
    std::vector<double> v;
    for (auto& it : wig) {
      const Wall& W = walls.at(it.second.wall);
      w.push_back(WallDev{W.o[0], W.o[1], W.o[2], W.n[0], W.n[1], W.n[2], it.second.k});
      auto lv = wall_loader.find(it.second.wall);
      for (int k = 0; k < 3; ++k) v.push_back(lv == wall_loader.end() ? 0.0 : lv->second[k]);
    }
    d_walls.reserve(kMaxWalls);
    d_wall_vel.reserve(kMaxWalls * 3);
    if (!w.empty()) {
      DEM_CUDA(cudaMemcpyAsync(d_walls.p, w.data(), sizeof(WallDev) * w.size(), cudaMemcpyHostToDevice, s));
      DEM_CUDA(cudaMemcpyAsync(d_wall_vel.p, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice, s));
    }
    sync();
  }
  // device wall origins are authoritative once groups exist: bring them back to the host
  void download_walls() {
    if (wig.empty()) return;
    std::vector<WallDev> w(wig.size());
    DEM_CUDA(cudaMemcpyAsync(w.data(), d_walls.p, sizeof(WallDev) * w.size(), cudaMemcpyDeviceToHost, s));
    sync();
    int k = 0;
    for (auto& it : wig) {
      Wall& W = walls.at(it.second.wall);
      W.o[0] = w[k].ox; W.o[1] = w[k].oy; W.o[2] = w[k].oz;
      ++k;
    }
  }

  // TSubLattice::updateInteractions (SubLattice.hpp:2416-2466)
  void update_interactions(bool need) {
    if (timestamp > last_ns || need) {
      bool flags_consumed = false;
      for (auto& d : dyn) {
        DynGroup& G = d.second;
        if (G.update_ts != timestamp) dyn_full_update(G);
        else if (!flags_consumed) { dyn_new_update(G); flags_consumed = true; }
        G.update_ts = timestamp;
      }
      if (!wig.empty()) {
        DEM_CUDA(cudaMemsetAsync(scalars.p + 2, 0, sizeof(int), s));
        launch_wall_update(g, P, cur, (int)wig.size(), d_walls.p, scalars.p + 2, s);
        wall_cand = read_int(scalars.p + 2);
        c_launches += 1;
      }
      for (auto& b : bond) {
        int ne = read_int(b.second.nevents.p);
        bond_alive[b.first] = b.second.nb - ne;
      }
      last_ns = timestamp;
    }
  }

  // With the device hand-off a bond failure needs no host update: only the interaction
  // counters (wall candidates, intact bonds) are brought up to date, in one read.
  void refresh_counts() {
    DEM_CUDA(cudaMemsetAsync(scalars.p + 2, 0, sizeof(int), s));
    launch_count_candidates(n, P.pflags, scalars.p + 2, s);
    int k = 3;
    for (auto& b : bond) {
      if (k >= 8) break;
      DEM_CUDA(cudaMemcpyAsync(scalars.p + k, b.second.nevents.p, sizeof(int), cudaMemcpyDeviceToDevice, s));
      ++k;
    }
    int host[8] = {0};
    DEM_CUDA(cudaMemcpyAsync(host, scalars.p, sizeof(int) * k, cudaMemcpyDeviceToHost, s));
    sync();
    wall_cand = host[2];
    k = 3;
    for (auto& b : bond) {
      if (k >= 8) break;
      bond_alive[b.first] = b.second.nb - host[k++];
    }
    c_launches += 1;
  }

  void set_handoff(bool on) {
    if (on == (handoff != 0)) return;
    if (on)
      for (auto& d : dyn)
        if (d.second.kind == 0 || d.second.kind >= 3)
          throw std::invalid_argument("the device bond hand-off needs every dynamic group to be RotFriction or NRotFriction");
    handoff = on;
    if (!d_brk.p) {
      d_brk.reserve(2);
    }
    DEM_CUDA(cudaMemsetAsync(d_brk.p, 0xff, sizeof(int) * 2, s));
    launch_clear_flags(n, P.flagged, s);
    // the dynamic lists are rebuilt in the new form before the next step
    if (!first) pending_ctrl |= CTRL_REBUILD;
  }

  // NRotFriction groups or NRotBond groups present: the FP64 general instances run the step
  // (bonds through the bond pass); the FP32 form, the batched ensemble and differentiable
  // windows are not built for them.
  // History handling of a dynamic group's list at a rebuild: 0 none (NRotElastic), 1 carried for
  // persistent pairs (PIS_ED groups: RotFriction, NRotFriction), 2 reset (HertzMindlin, whose
  // history lives in a PIS_NE storage that rebuilds its list from scratch).
  static int hist_mode(const DynGroup& G) { return G.kind == 0 ? 0 : (G.kind >= 3 ? 2 : 1); }

  bool widened() const {
    for (auto& d : dyn) if (d.second.kind >= 2) return true;
    for (auto& b : bond) if (b.second.kind != 0) return true;
    return false;
  }

  // interactions evaluated per step: Verlet pairs + intact bonds + wall candidates
  long long contacts_per_step() const {
    long long c = wall_cand;
    for (auto& d : dyn) c += d.second.m;
    for (auto& b : bond) {
      auto it = bond_alive.find(b.first);
      c += it == bond_alive.end() ? b.second.nb : it->second;
    }
    return c;
  }

  bool has_sc() const {
    for (auto& b : bond) if (b.second.kind == 3) return true;
    return false;
  }
  // The stress sums BrittleBeamSC groups read: zero until a step has written them (the particles'
  // m_sigma starts at zero), kept when the particle storage grows.
  double* ensure_sig() {
    const size_t need = 9 * (size_t)std::max(n, 1);
    if (sig.cap < need) {
      const size_t old = sig.cap;
      sig.reserve(need, true, s);
      DEM_CUDA(cudaMemsetAsync(sig.p + old, 0, sizeof(double) * (sig.cap - old), s));
    }
    return sig.p;
  }

  StepArgs make_args(int c) {
    StepArgs a{};
    if (has_sc()) a.sig = ensure_sig();
    a.g = g;
    a.P = P;
    a.cur = c;
    a.dt = dt;
    a.half_alpha_sq = (0.5 * alpha) * (0.5 * alpha);
    a.nwall = (int)wig.size();
    a.walls = d_walls.p;
    a.wall_vel = d_wall_vel.p;
    a.ngrav = 0;
    for (auto& gr : grav) {
      if (a.ngrav >= kMaxGrav) break;
      for (int k = 0; k < 3; ++k) a.grav[a.ngrav][k] = gr.second[k];
      a.ngrav++;
    }
    a.ndyn = 0;
    for (auto& d : dyn) {
      DynGroup& G = d.second;
      DynDev& D = a.dyn[a.ndyn++];
      D.kind = G.kind; D.k = G.k; D.ks = G.ks; D.mu_s = G.mu_s; D.mu_d = G.mu_d; D.dt = G.dt;
      D.scaling = G.scaling; D.meanR = G.meanR;
      D.adj_start = G.adj_start.p; D.adj = G.adj.p;
      D.hist_in = G.hist[c].p; D.hist_out = G.hist[c ^ 1].p;
      D.hist32_in = G.hist32[c].p; D.hist32_out = G.hist32[c ^ 1].p;
      D.xbond = handoff ? G.xbond.p : nullptr;
    }
    a.nbond = 0;
    for (auto& b : bond) {
      BondGroup& B = b.second;
      BondDev& D = a.bond[a.nbond++];
      D.kind = B.kind; D.knb = B.knb; D.rbreak = B.rbreak;
      D.cohesion = B.cohesion; D.tan_angle = B.tan_angle; D.t_cutoff = B.t_cutoff; D.c_cutoff = B.c_cutoff;
      D.beta1 = B.beta1; D.beta2 = B.beta2;
      D.kr = B.kr; D.ks = B.ks; D.kt = B.kt; D.kb = B.kb; D.mn = B.mn; D.ms = B.ms; D.mt = B.mt; D.mb = B.mb;
      D.truncated = B.truncated; D.scaling = B.scaling; D.meanR = B.meanR;
      D.adj_start = B.adj_start.p; D.adj = B.adj.p; D.D0 = B.D0.p; D.broken_step = B.broken_step.p;
      D.events = B.events.p; D.nevents = B.nevents.p; D.cap_events = B.cap_events;
      D.nb_launch = B.nb;
      D.ends = B.ends.p;
      // the FP32 form and the widened laws always take their bonds from the FP64 bond pass
      if (bond_pass || fp32 || widened()) {
        B.bf.reserve((size_t)3 * std::max(B.nb, 1));
        D.bf = B.bf.p;
      }
      if (fp32) {  // the FP32 form gathers its bonds' forces from FP32 records of the same pass
        B.bf32.reserve((size_t)4 * std::max(B.nb, 1));
        D.bf32 = B.bf32.p;
      }
    }
    a.damp_lin = damp_lin; a.damp_rot = damp_rot;
    a.damp_loc = !loc_name.empty(); a.damp_rotloc = damp_rotloc; a.visc_loc = visc_loc; a.visc_rotloc = visc_rotloc;
    a.loc_before_lin = !loc_name.empty() && loc_name < std::string("Damping");
    a.visc_lin = visc_lin; a.visc_rot = visc_rot; a.dt_lin = dt; a.dt_rot = dt;
    a.iter_lin = iter_lin; a.iter_rot = iter_rot;
    a.store_forces = store_forces;
    a.force_step = -1;
    a.handoff = handoff;
    a.brk_step = d_brk.p;
    a.stop_skip = handoff ? CTRL_BROKE : 0;
    a.wall_partial = d_wall_partial.p;
    a.wall_force = d_wall_force.p;
    a.block_counter = d_block_counter.p;
    a.step_counter = d_step.p;
    a.ctrl = d_ctrl.p;
    a.stop = d_stop.p;
    return a;
  }

  // Groups the tiled step kernels cover: the core pair laws, and bonds through the bond pass.
  bool tiled_ok() const {
    for (auto& d : dyn) if (d.second.kind >= 2) return false;
    for (auto& b : bond) if (b.second.kind == 1 || b.second.kind == 3) return false;
    return bond.empty() || bond_pass || fp32;
  }

  // Lanes per particle when none is set.  A specimen with at least as many particles as the
  // GPU keeps step threads resident (3 blocks of 256 per SM) already fills it at one lane per
  // particle, which measured fastest on the 250k shear cell and the 1M bonded block; a smaller
  // one spreads each particle's adjacency over lanes by its mean length.  The tiled kernels
  // (kTiled) are chosen explicitly or by the ensemble autotuner.
  int pick_tpp() {
    if (tpp) return tpp == kTiled && !tiled_ok() ? 1 : tpp;
    static const long long resident = [] {
      int dev = 0, sms = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      return 768LL * (sms > 0 ? sms : 148);
    }();
    if (n >= resident) return 1;
    long long e = 0;
    for (auto& d : dyn) e += 2LL * d.second.m;
    for (auto& b : bond) e += 2LL * b.second.nb;
    double mean = n ? (double)e / n : 0.0;
    if (mean >= 12) return 8;
    if (mean >= 6) return 4;
    if (mean >= 2.5) return 2;
    return 1;
  }

  // CLatticeMaster::runOneStep x nsteps (LatticeMaster.cpp:2602-2740), without savers and runnables.
  // The head of one runOneStep: the first step's forced search, checkNeighbors +
  // searchNeighbors (LatticeMaster.cpp:1864-1908) and updateInteractions.
  bool prepare() {
    if (first) { search_neighbors(); first = false; }
    if (pending_ctrl & CTRL_REBUILD) search_neighbors();
    if (handoff && (pending_ctrl & CTRL_BROKE) && timestamp == last_ns) refresh_counts();
    else update_interactions((pending_ctrl & CTRL_BROKE) != 0);
    pending_ctrl = 0;
    return true;
  }

  // A full event log loses entries only: the failures themselves are in each bond's state.
  // The call in which the log filled reports it; later calls go on.
  bool take_overflow() {
    const bool o = (pending_ctrl & CTRL_OVERFLOW) != 0;
    pending_ctrl &= ~CTRL_OVERFLOW;
    return o;
  }
  static constexpr const char* kOverflowText =
      "bond-break event log overflowed (failures past its capacity are not logged; the bond states are exact)";

  int step(int nsteps) {
    int done = 0;
    bool overflowed = false;
    // the forces a caller can observe are the last step's: only that step stores them
    const long long t_last = t + nsteps;
    while (done < nsteps) {
      if (!prepare()) return -2;
      // launch a chunk of force + integration steps
      const int k = std::min(chunk, nsteps - done);
      const int t_pp = pick_tpp();
      const int grid = step_grid(n, t_pp);
      d_wall_partial.reserve((size_t)grid * kMaxWalls * 3);
      DEM_CUDA(cudaMemsetAsync(d_ctrl.p, 0, sizeof(int), s));
      DEM_CUDA(cudaMemsetAsync(d_stop.p, 0, sizeof(int), s));
      const long long t0 = t;
      const long long cps = contacts_per_step();
      if (profile) {
        if (!ev0) { DEM_CUDA(cudaEventCreate(&ev0)); DEM_CUDA(cudaEventCreate(&ev1)); }
        DEM_CUDA(cudaEventRecord(ev0, s));
      }
      if (fp32 && t_pp == kTiled) launch_sync_vw(P, cur, s);  // only the tiled kernels read the shadow
      const bool two = split == 1;  // automatic = fused: measured faster on the 250k shear cell
      for (int j = 0; j < k; ++j) {
        StepArgs a = make_args((cur + j) & 1);
        a.force_step = t_last;
        a.skip_vw = t_pp != kTiled;  // only the tiled kernels read the FP32 velocity shadow
        if (fp32) launch_step_fp32(a, rot != 0, t_pp, false, two, s);
        else launch_step(a, rot != 0, t_pp, two, s);
      }
      DEM_CUDA(cudaGetLastError());
      if (profile) DEM_CUDA(cudaEventRecord(ev1, s));
      c_launches += two ? 2LL * k : k;
      DEM_CUDA(cudaMemcpyAsync(h_ctrl, d_step.p, sizeof(long long), cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(h_ctrl + 2, d_ctrl.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      sync();
      long long dev_t;
      std::memcpy(&dev_t, h_ctrl, sizeof(long long));
      const int ran = (int)(dev_t - t0);
      pending_ctrl = h_ctrl[2];
      overflowed |= take_overflow();
      // a BrittleBeamSC failure at the head of the chunk's first step stops it before any step
      if (ran < 0 || ran > k || (ran == 0 && !(pending_ctrl & CTRL_BROKE))) {
        err = "device step counter out of sequence";
        return -3;
      }
      t = dev_t;
      cur = (cur + ran) & 1;
      done += ran;
      c_steps += ran;
      c_contacts += (long long)ran * cps;
      if (profile) {
        float ms = 0.f;
        DEM_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        prof_ms += ms;
        prof_steps += ran;
      }
    }
    if (overflowed) { err = kOverflowText; return -2; }
    return 0;
  }

  // ---- differentiable loading window -------------------------------------
  // Forward: T FP64 steps from the current state with the topology frozen
  // (no neighbour rebuild may fall inside the window; a bond failure may only
  // with the device bond hand-off, and is then a fixed event of the window),
  // checkpoints of the particle state, friction histories and wall planes every
  // K steps, and the reaction of every wall group after every step.
  // Adjoint: the reverse pass over the stored window, segment by segment from
  // the last, each segment's forward states recomputed from its checkpoint.
  // With failures inside the window the recompute replays them: the bonds'
  // failure steps are already recorded (a bond is evaluated while its failure
  // step lies ahead, exactly as in the forward), the wall candidacy and the
  // last-failure record are restored per segment, and nothing is logged again.
  struct Window {
    bool valid = false;
    bool brk = false;  // bond failures may fall inside the window (device hand-off)
    long long tcv = 0;  // step counter at the start of the segment being recomputed (copy source)
    int T = 0, K = 0, nseg = 0, n = 0, ts = 0, cur0 = 0;
    long long t0 = 0;
    int m[kMaxDyn] = {0, 0};
    DBuf<double4> ck, ck_hist[kMaxDyn], st, st_hist[kMaxDyn], st_f, st_m, lam, gb[kMaxBond], lH[kMaxDyn],
        gpair[kMaxDyn];
    DBuf<WallDev> ck_walls, st_walls, save_walls;
    DBuf<unsigned char> st_it;
    DBuf<double> R, gR, gvisc, gpar_b[kMaxBond], gpar_d[kMaxDyn], acc, save_wf;
    DBuf<long long> ck_step;
    DBuf<unsigned> ck_pf, st_pf, save_pf;  // wall candidacy: per checkpoint, per recomputed step, live
    DBuf<int> ck_brk, save_brk, bs0[kMaxBond], nev0;
    DBuf<unsigned char> flag0, gact[kMaxDyn];
    DBuf<float4> st_vw, st_hist32[kMaxDyn];  // FP32 form: velocity shadows and histories of the recompute
    bool fp32 = false;
    void release() {
      st_vw.release();
      for (int d = 0; d < kMaxDyn; ++d) st_hist32[d].release();
      ck_pf.release(); st_pf.release(); save_pf.release(); ck_brk.release(); save_brk.release(); nev0.release();
      flag0.release();
      for (int d = 0; d < kMaxDyn; ++d) gact[d].release();
      for (int b = 0; b < kMaxBond; ++b) bs0[b].release();
      ck.release(); st.release(); st_f.release(); st_m.release(); lam.release();
      for (int d = 0; d < kMaxDyn; ++d) {
        ck_hist[d].release(); st_hist[d].release(); lH[d].release(); gpair[d].release(); gpar_d[d].release();
      }
      for (int b = 0; b < kMaxBond; ++b) { gb[b].release(); gpar_b[b].release(); }
      ck_walls.release(); st_walls.release(); save_walls.release(); st_it.release();
      R.release(); gR.release(); gvisc.release(); acc.release(); save_wf.release(); ck_step.release();
      valid = false;
    }
  } win;

  static ParticleBuf view4(double4* base, int n) { return ParticleBuf{base, base + n, base + 2 * (size_t)n, base + 3 * (size_t)n, nullptr}; }
  // state j of the segment being recomputed (with its FP32 velocity shadow in the FP32 form)
  ParticleBuf st_view(int j) {
    ParticleBuf b = view4(win.st.p + (size_t)j * 4 * n, n);
    if (win.fp32) b.vw = win.st_vw.p + (size_t)j * 2 * std::max(n, 1);
    return b;
  }
  void copy_state(const ParticleBuf& dst, const ParticleBuf& src) {
    const size_t b = sizeof(double4) * (size_t)n;
    DEM_CUDA(cudaMemcpyAsync(dst.pr, src.pr, b, cudaMemcpyDeviceToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(dst.vm, src.vm, b, cudaMemcpyDeviceToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(dst.wi, src.wi, b, cudaMemcpyDeviceToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(dst.qq, src.qq, b, cudaMemcpyDeviceToDevice, s));
  }
  std::vector<DynGroup*> dyn_list() { std::vector<DynGroup*> v; for (auto& d : dyn) v.push_back(&d.second); return v; }
  std::vector<BondGroup*> bond_list() { std::vector<BondGroup*> v; for (auto& b : bond) v.push_back(&b.second); return v; }
  int window_num_params() const { return 4 * (int)bond.size() + 2 * (int)dyn.size() + 2; }

  void window_check_ctrl(int ctrl, bool last) {
    if ((ctrl & CTRL_BROKE) && !handoff)
      throw StateError("a bond broke inside the differentiable window (enable the device bond hand-off to keep it)");
    if (ctrl & CTRL_OVERFLOW) throw StateError("bond-break event log overflowed inside the differentiable window");
    if ((ctrl & CTRL_REBUILD) && !last)
      throw StateError("a neighbour rebuild fell inside the differentiable window (shorten it or enlarge verletDist)");
  }

  // Forward, in parts shared with the batched ensemble.  Prologue: the runOneStep head, the
  // checkpoint buffers and what a rewind must put back.  False: the head failed (err is set).
  bool win_begin(int T, int K) {
    if (T < 1 || K < 1) throw std::invalid_argument("window length and checkpoint interval must be >= 1");
    if (iter_lin > 255 || iter_rot > 255) throw std::invalid_argument("window damping needs maxIterations <= 255");
    if (widened()) throw std::invalid_argument("the differentiable window covers NRotElastic, RotFriction and RotBond groups");
    if (!loc_name.empty() || damp_rotloc)
      throw std::invalid_argument("the differentiable window covers the viscous damping groups, not local damping");
    win.valid = false;
    if (!prepare()) return false;
    const int nd = (int)dyn.size();
    auto dl = dyn_list();
    win.T = T; win.K = std::min(K, T); win.nseg = (T + win.K - 1) / win.K; win.n = n; win.t0 = t;
    win.ts = timestamp; win.cur0 = cur;
    win.brk = handoff != 0;
    win.fp32 = fp32 != 0;
    win.ck.reserve((size_t)win.nseg * 4 * std::max(n, 1));
    if (win.brk) {  // what a rewind must put back: failure records, event counts, flags
      win.ck_pf.reserve((size_t)win.nseg * std::max(n, 1));
      win.ck_brk.reserve((size_t)win.nseg * 2);
      win.nev0.reserve(kMaxBond);
      win.flag0.reserve(std::max(n, 1));
      int b = 0;
      for (auto& bg : bond) {
        BondGroup& B = bg.second;
        win.bs0[b].reserve(std::max(B.nb, 1));
        if (B.nb)
          DEM_CUDA(cudaMemcpyAsync(win.bs0[b].p, B.broken_step.p, sizeof(int) * B.nb, cudaMemcpyDeviceToDevice, s));
        DEM_CUDA(cudaMemcpyAsync(win.nev0.p + b, B.nevents.p, sizeof(int), cudaMemcpyDeviceToDevice, s));
        ++b;
      }
      if (n) DEM_CUDA(cudaMemcpyAsync(win.flag0.p, P.flagged, n, cudaMemcpyDeviceToDevice, s));
    }
    win.ck_walls.reserve((size_t)win.nseg * kMaxWalls);
    win.R.reserve((size_t)T * kMaxWalls * 3);
    for (int d = 0; d < nd; ++d) {
      win.m[d] = dl[d]->m;
      if (dl[d]->kind == 1) win.ck_hist[d].reserve((size_t)win.nseg * std::max(win.m[d], 1));
    }
    DEM_CUDA(cudaMemsetAsync(win.R.p, 0, sizeof(double) * T * kMaxWalls * 3, s));
    if (fp32) launch_sync_vw(P, cur, s);
    return true;
  }

  // Checkpoint c: particle records, friction histories, wall planes, and under the hand-off
  // the wall candidacy and the last-failure record.
  void win_checkpoint(int c) {
    const int nd = (int)dyn.size();
    auto dl = dyn_list();
    copy_state(view4(win.ck.p + (size_t)c * 4 * n, n), P.buf[cur]);
    if (win.brk) {
      if (n) DEM_CUDA(cudaMemcpyAsync(win.ck_pf.p + (size_t)c * n, P.pflags, sizeof(unsigned) * n,
                                      cudaMemcpyDeviceToDevice, s));
      DEM_CUDA(cudaMemcpyAsync(win.ck_brk.p + 2 * c, d_brk.p, 2 * sizeof(int), cudaMemcpyDeviceToDevice, s));
    }
    for (int d = 0; d < nd; ++d)
      if (dl[d]->kind == 1 && win.m[d]) {
        if (fp32)  // FP32 records widened exactly
          launch_hist_convert(win.m[d], win.ck_hist[d].p + (size_t)c * win.m[d], dl[d]->hist32[cur].p, false, s);
        else
          DEM_CUDA(cudaMemcpyAsync(win.ck_hist[d].p + (size_t)c * win.m[d], dl[d]->hist[cur].p,
                                   sizeof(double4) * win.m[d], cudaMemcpyDeviceToDevice, s));
      }
    if (!wig.empty())
      DEM_CUDA(cudaMemcpyAsync(win.ck_walls.p + (size_t)c * kMaxWalls, d_walls.p, sizeof(WallDev) * wig.size(),
                               cudaMemcpyDeviceToDevice, s));
  }

  // Segment c of len steps ended with the device counter at dev_t and control bits ctrl.
  // The steps that ran are real steps of the simulation, whether the window stands or not.
  void win_segment_done(int c, int len, long long dev_t, int ctrl, long long cps) {
    const long long ran = dev_t - t;
    if (ran < 0 || ran > len) throw StateError("device step counter out of sequence in the window");
    t = dev_t;
    cur = (int)((cur + ran) & 1);
    c_steps += ran;
    c_contacts += ran * cps;
    pending_ctrl = ctrl;
    window_check_ctrl(ctrl, c == win.nseg - 1 && ran == len);
    if (ran != len) throw StateError("device step counter out of sequence in the window");
  }

  void win_finish(double* R_host) {
    if (R_host) {
      std::vector<double> r((size_t)win.T * kMaxWalls * 3);
      DEM_CUDA(cudaMemcpyAsync(r.data(), win.R.p, sizeof(double) * r.size(), cudaMemcpyDeviceToHost, s));
      sync();
      const int nw = (int)wig.size();
      for (int k = 0; k < win.T; ++k)
        for (int w = 0; w < nw; ++w)
          for (int c = 0; c < 3; ++c) R_host[((size_t)k * nw + w) * 3 + c] = r[((size_t)k * kMaxWalls + w) * 3 + c];
    }
    win.valid = true;
  }

  int window_forward(int T, int K, double* R_host) {
    if (!win_begin(T, K)) return DEM_ERR_OVERFLOW;
    const int t_pp = pick_tpp();
    d_wall_partial.reserve((size_t)step_grid(n, t_pp) * kMaxWalls * 3);
    const bool two = split == 1;
    const long long cps = contacts_per_step();
    for (int c = 0; c < win.nseg; ++c) {
      const int len = std::min(win.K, win.T - c * win.K);
      win_checkpoint(c);
      DEM_CUDA(cudaMemsetAsync(d_ctrl.p, 0, sizeof(int), s));
      DEM_CUDA(cudaMemsetAsync(d_stop.p, 0, sizeof(int), s));
      for (int j = 0; j < len; ++j) {
        StepArgs a = make_args((cur + j) & 1);
        a.wall_hist = win.R.p;
        a.wall_hist_t0 = win.t0;
        if (fp32) launch_step_fp32(a, rot != 0, t_pp, false, two, s);
        else launch_step(a, rot != 0, t_pp, two, s);
      }
      DEM_CUDA(cudaGetLastError());
      c_launches += two ? 2LL * len : len;
      DEM_CUDA(cudaMemcpyAsync(h_ctrl, d_step.p, sizeof(long long), cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(h_ctrl + 2, d_ctrl.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      sync();
      long long dev_t;
      std::memcpy(&dev_t, h_ctrl, sizeof(long long));
      win_segment_done(c, len, dev_t, h_ctrl[2], cps);
    }
    win_finish(R_host);
    return 0;
  }

  void window_require() {
    if (!win.valid) throw StateError("no differentiable window has been run");
    if (t != win.t0 + win.T || timestamp != win.ts || n != win.n)
      throw StateError("the simulation moved on since the window was run");
  }

  // Reverse, in parts shared with the batched ensemble.  Prologue: buffers, the loss gradient
  // gR_host [T][nwall][3], the live device state the recompute touches, and the reverse
  // arguments that do not depend on the step.
  AdjArgs adj_begin(const double* gR_host) {
    window_require();
    if (!gR_host) throw std::invalid_argument("null reaction gradient");
    const int T = win.T, K = win.K, nw = (int)wig.size();
    auto dl = dyn_list();
    auto bl = bond_list();
    const int nd = (int)dl.size(), nbg = (int)bl.size();
    const int nn = std::max(n, 1);
    win.st.reserve((size_t)(K + 1) * 4 * nn);
    if (win.fp32) win.st_vw.reserve((size_t)(K + 1) * 2 * nn);
    win.st_f.reserve((size_t)K * nn);
    win.st_m.reserve((size_t)K * nn);
    win.st_it.reserve((size_t)K * 2 * nn);
    win.st_walls.reserve((size_t)K * kMaxWalls);
    win.lam.reserve((size_t)6 * nn);
    win.gvisc.reserve((size_t)2 * nn);
    win.gR.reserve((size_t)T * kMaxWalls * 3);
    win.acc.reserve(64);
    win.save_walls.reserve(kMaxWalls);
    win.save_wf.reserve(kMaxWalls * 3);
    if (win.brk) {
      win.st_pf.reserve((size_t)K * nn);
      win.save_pf.reserve(nn);
      win.save_brk.reserve(2);
      if (n) DEM_CUDA(cudaMemcpyAsync(win.save_pf.p, P.pflags, sizeof(unsigned) * n, cudaMemcpyDeviceToDevice, s));
      DEM_CUDA(cudaMemcpyAsync(win.save_brk.p, d_brk.p, 2 * sizeof(int), cudaMemcpyDeviceToDevice, s));
    }
    for (int d = 0; d < nd; ++d) {
      const int m = std::max(win.m[d], 1);
      if (dl[d]->kind == 1) {
        if (win.fp32) win.st_hist32[d].reserve((size_t)(K + 1) * m);
        else win.st_hist[d].reserve((size_t)(K + 1) * m);
      }
      win.lH[d].reserve(m);
      win.gpair[d].reserve((size_t)3 * m);
      win.gact[d].reserve(m);
      win.gpar_d[d].reserve((size_t)2 * m);
      DEM_CUDA(cudaMemsetAsync(win.lH[d].p, 0, sizeof(double4) * m, s));
      DEM_CUDA(cudaMemsetAsync(win.gpar_d[d].p, 0, sizeof(double) * 2 * m, s));
    }
    for (int b = 0; b < nbg; ++b) {
      const int m = std::max(bl[b]->nb, 1);
      win.gb[b].reserve((size_t)3 * m);
      win.gpar_b[b].reserve((size_t)4 * m);
      DEM_CUDA(cudaMemsetAsync(win.gpar_b[b].p, 0, sizeof(double) * 4 * m, s));
    }
    DEM_CUDA(cudaMemsetAsync(win.lam.p, 0, sizeof(double4) * 6 * nn, s));
    DEM_CUDA(cudaMemsetAsync(win.gvisc.p, 0, sizeof(double) * 2 * nn, s));
    DEM_CUDA(cudaMemsetAsync(win.acc.p, 0, sizeof(double) * 64, s));
    {
      std::vector<double> g((size_t)T * kMaxWalls * 3, 0.0);
      for (int k = 0; k < T; ++k)
        for (int w = 0; w < nw; ++w)
          for (int c = 0; c < 3; ++c) g[((size_t)k * kMaxWalls + w) * 3 + c] = gR_host[((size_t)k * nw + w) * 3 + c];
      DEM_CUDA(cudaMemcpyAsync(win.gR.p, g.data(), sizeof(double) * g.size(), cudaMemcpyHostToDevice, s));
      sync();
    }
    if (nw) DEM_CUDA(cudaMemcpyAsync(win.save_walls.p, d_walls.p, sizeof(WallDev) * nw, cudaMemcpyDeviceToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(win.save_wf.p, d_wall_force.p, sizeof(double) * kMaxWalls * 3, cudaMemcpyDeviceToDevice, s));
    double4* lam = win.lam.p;
    AdjArgs A{};
    A.g = g; A.n = n; A.rot = rot; A.dt = dt; A.pflags = P.pflags;
    A.damp_lin = damp_lin; A.damp_rot = damp_rot; A.iter_lin = iter_lin; A.iter_rot = iter_rot;
    A.visc_lin = visc_lin; A.visc_rot = visc_rot; A.dt_lin = dt; A.dt_rot = dt;
    A.nwall = nw;
    A.bond_tangents = adj_tangents;
    A.pair_duals = adj_pair_duals;
    A.lx = lam; A.lv = lam + nn; A.lw = lam + 2 * (size_t)nn; A.lq = lam + 3 * (size_t)nn;
    A.lF = lam + 4 * (size_t)nn; A.lM = lam + 5 * (size_t)nn;
    A.gvisc = win.gvisc.p;
    A.ndyn = nd;
    for (int d = 0; d < nd; ++d) {
      DynGroup& G = *dl[d];
      AdjDyn& D = A.dyn[d];
      D.kind = G.kind; D.k = G.k; D.ks = G.ks; D.mu_s = G.mu_s; D.mu_d = G.mu_d; D.dt = G.dt;
      D.scaling = G.scaling; D.meanR = G.meanR; D.m = win.m[d];
      D.keys = G.keys.p; D.adj_start = G.adj_start.p; D.adj = G.adj.p;
      D.lH = win.lH[d].p; D.gpair = win.gpair[d].p; D.gact = win.gact[d].p; D.gpar = win.gpar_d[d].p;
      D.xbond = handoff ? G.xbond.p : nullptr;
    }
    A.nbond = nbg;
    for (int b = 0; b < nbg; ++b) {
      BondGroup& B = *bl[b];
      AdjBond& D = A.bond[b];
      D.kr = B.kr; D.ks = B.ks; D.kt = B.kt; D.kb = B.kb; D.mn = B.mn; D.ms = B.ms; D.mt = B.mt; D.mb = B.mb;
      D.scaling = B.scaling; D.meanR = B.meanR; D.nb = B.nb;
      D.ends = B.ends.p; D.D0 = B.D0.p; D.broken_step = B.broken_step.p;
      D.adj_start = B.adj_start.p; D.adj = B.adj.p;
      D.gb = win.gb[b].p; D.gpar = win.gpar_b[b].p;
    }
    return A;
  }

  // Segment c's start state from its checkpoint, into the recompute buffers; the device
  // step counter at the segment's first step.
  void adj_restore(int c) {
    const int nd = (int)dyn.size(), nw = (int)wig.size();
    auto dl = dyn_list();
    copy_state(view4(win.st.p, n), view4(win.ck.p + (size_t)c * 4 * n, n));
    if (win.fp32) {  // the velocity shadow of the checkpoint, as the forward kept it
      Particles Q = P;
      Q.buf[0] = st_view(0);
      launch_sync_vw(Q, 0, s);
    }
    for (int d = 0; d < nd; ++d)
      if (dl[d]->kind == 1 && win.m[d]) {
        if (win.fp32)
          launch_hist_convert(win.m[d], win.ck_hist[d].p + (size_t)c * win.m[d], win.st_hist32[d].p, true, s);
        else
          DEM_CUDA(cudaMemcpyAsync(win.st_hist[d].p, win.ck_hist[d].p + (size_t)c * win.m[d],
                                   sizeof(double4) * win.m[d], cudaMemcpyDeviceToDevice, s));
      }
    if (nw)
      DEM_CUDA(cudaMemcpyAsync(d_walls.p, win.ck_walls.p + (size_t)c * kMaxWalls, sizeof(WallDev) * nw,
                               cudaMemcpyDeviceToDevice, s));
    if (win.brk) {
      if (n) DEM_CUDA(cudaMemcpyAsync(P.pflags, win.ck_pf.p + (size_t)c * n, sizeof(unsigned) * n,
                                      cudaMemcpyDeviceToDevice, s));
      DEM_CUDA(cudaMemcpyAsync(d_brk.p, win.ck_brk.p + 2 * c, 2 * sizeof(int), cudaMemcpyDeviceToDevice, s));
    }
    win.tcv = win.t0 + (long long)c * win.K;
    DEM_CUDA(cudaMemcpyAsync(d_step.p, &win.tcv, sizeof(long long), cudaMemcpyHostToDevice, s));
    DEM_CUDA(cudaMemsetAsync(d_ctrl.p, 0, sizeof(int), s));
    DEM_CUDA(cudaMemsetAsync(d_stop.p, 0, sizeof(int), s));
  }

  // Step arguments of recomputed step j of a segment: state j -> j + 1 in the recompute
  // buffers, the pre-damping sums and damping iterations stored, nothing logged again.
  StepArgs adj_recompute_args(int j) {
    const int nd = (int)dyn.size();
    auto dl = dyn_list();
    StepArgs a = make_args(0);
    a.P.buf[0] = st_view(j);
    a.P.buf[1] = st_view(j + 1);
    a.cur = 0;
    for (int d = 0; d < nd; ++d)
      if (dl[d]->kind == 1) {
        const size_t m = std::max(win.m[d], 1);
        if (win.fp32) {
          a.dyn[d].hist32_in = win.st_hist32[d].p + j * m;
          a.dyn[d].hist32_out = win.st_hist32[d].p + (j + 1) * m;
        } else {
          a.dyn[d].hist_in = win.st_hist[d].p + j * m;
          a.dyn[d].hist_out = win.st_hist[d].p + (j + 1) * m;
        }
      }
    a.f_int = win.st_f.p + (size_t)j * n;
    a.m_int = win.st_m.p + (size_t)j * n;
    a.damp_iters = win.st_it.p + (size_t)j * 2 * n;
    a.store_forces = 0;
    a.replay = 1;
    if (win.brk) a.pf_log = win.st_pf.p + (size_t)j * n;  // the wall candidacy this step used
    return a;
  }

  // The step-dependent reverse arguments of step j of segment c.
  void adj_fill(AdjArgs& A, int c, int j) {
    const int nd = (int)dyn.size();
    auto dl = dyn_list();
    A.step = win.t0 + (long long)c * win.K + j + 1;
    A.s0 = st_view(j);
    A.s1 = st_view(j + 1);
    A.f_int = win.st_f.p + (size_t)j * n;
    A.m_int = win.st_m.p + (size_t)j * n;
    A.iters = win.st_it.p + (size_t)j * 2 * n;
    A.walls = win.st_walls.p + (size_t)j * kMaxWalls;
    A.pflags = win.brk ? win.st_pf.p + (size_t)j * n : P.pflags;
    A.gR = win.gR.p + (size_t)(c * win.K + j) * kMaxWalls * 3;
    for (int d = 0; d < nd; ++d)
      if (dl[d]->kind == 1) {
        const size_t m = std::max(win.m[d], 1);
        A.dyn[d].hist_in = win.fp32 ? nullptr : win.st_hist[d].p + j * m;
        A.dyn[d].hist32_in = win.fp32 ? win.st_hist32[d].p + j * m : nullptr;
      }
  }

  // The window's buffers as the batched ensemble's expansion kernels index them.
  WinSpec win_spec() const {
    WinSpec w{};
    w.n = n;
    w.K = win.K;
    w.t0 = win.t0;
    w.st = win.st.p;
    w.st_vw = win.fp32 ? win.st_vw.p : nullptr;
    w.st_f = win.st_f.p;
    w.st_m = win.st_m.p;
    w.st_it = win.st_it.p;
    w.st_walls = win.st_walls.p;
    w.st_pf = win.brk ? win.st_pf.p : nullptr;
    w.gR = win.gR.p;
    w.walls = d_walls.p;
    w.nwall = (int)wig.size();
    int d = 0;
    for (auto& g : dyn) {
      w.hstride[d] = std::max(win.m[d], 1);
      if (g.second.kind == 1) {
        w.st_hist[d] = win.fp32 ? nullptr : win.st_hist[d].p;
        w.st_hist32[d] = win.fp32 ? win.st_hist32[d].p : nullptr;
      }
      ++d;
    }
    return w;
  }

  // Parameter reductions, the live device state put back, the gradients to the host.
  void adj_finish(double* grad_params, double* gvel, double* gang, double* gpos, double* gquat) {
    auto dl = dyn_list();
    auto bl = bond_list();
    const int nd = (int)dl.size(), nbg = (int)bl.size(), nw = (int)wig.size();
    const int nn = std::max(n, 1);
    double4* lam = win.lam.p;
    int off = 0;
    for (int b = 0; b < nbg; ++b, off += 4) launch_reduce_cols(win.gpar_b[b].p, bl[b]->nb, 4, win.acc.p + off, s);
    for (int d = 0; d < nd; ++d, off += 2) launch_reduce_cols(win.gpar_d[d].p, win.m[d], 2, win.acc.p + off, s);
    launch_reduce_cols(win.gvisc.p, n, 2, win.acc.p + off, s);
    off += 2;
    DEM_CUDA(cudaGetLastError());
    if (win.brk) {
      if (n) DEM_CUDA(cudaMemcpyAsync(P.pflags, win.save_pf.p, sizeof(unsigned) * n, cudaMemcpyDeviceToDevice, s));
      DEM_CUDA(cudaMemcpyAsync(d_brk.p, win.save_brk.p, 2 * sizeof(int), cudaMemcpyDeviceToDevice, s));
    }
    if (nw) DEM_CUDA(cudaMemcpyAsync(d_walls.p, win.save_walls.p, sizeof(WallDev) * nw, cudaMemcpyDeviceToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(d_wall_force.p, win.save_wf.p, sizeof(double) * kMaxWalls * 3, cudaMemcpyDeviceToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(d_step.p, &t, sizeof(long long), cudaMemcpyHostToDevice, s));
    DEM_CUDA(cudaMemsetAsync(d_ctrl.p, 0, sizeof(int), s));
    DEM_CUDA(cudaMemsetAsync(d_stop.p, 0, sizeof(int), s));
    std::vector<double> acc(off);
    std::vector<double4> lh((size_t)4 * n);
    std::vector<unsigned> pf(n);
    DEM_CUDA(cudaMemcpyAsync(acc.data(), win.acc.p, sizeof(double) * off, cudaMemcpyDeviceToHost, s));
    if (n) {
      DEM_CUDA(cudaMemcpyAsync(lh.data(), lam, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(lh.data() + n, lam + nn, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(lh.data() + 2 * (size_t)n, lam + 2 * (size_t)nn, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(lh.data() + 3 * (size_t)n, lam + 3 * (size_t)nn, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(pf.data(), P.pflags, sizeof(unsigned) * n, cudaMemcpyDeviceToHost, s));
    }
    sync();
    if (grad_params) for (int k = 0; k < off; ++k) grad_params[k] = acc[k];
    int k = 0;
    for (int i = 0; i < n; ++i) {
      if (!(pf[i] & PF_ALIVE)) continue;
      const double4 x = lh[i], v = lh[n + i], w = lh[2 * (size_t)n + i], q = lh[3 * (size_t)n + i];
      if (gpos) { gpos[3 * k] = x.x; gpos[3 * k + 1] = x.y; gpos[3 * k + 2] = x.z; }
      if (gvel) { gvel[3 * k] = v.x; gvel[3 * k + 1] = v.y; gvel[3 * k + 2] = v.z; }
      if (gang) {
        gang[3 * k] = rot ? w.x : 0.0; gang[3 * k + 1] = rot ? w.y : 0.0; gang[3 * k + 2] = rot ? w.z : 0.0;
      }
      if (gquat) {
        gquat[4 * k] = rot ? q.x : 0.0; gquat[4 * k + 1] = rot ? q.y : 0.0;
        gquat[4 * k + 2] = rot ? q.z : 0.0; gquat[4 * k + 3] = rot ? q.w : 0.0;
      }
      ++k;
    }
  }

  // Reverse pass.  gR_host: [T][nwall][3] dLoss/dReaction; grad_params: window_num_params()
  // values (bond groups x (kr, ks, kt, kb), dynamic groups x (k, ks), linear and rotational
  // viscosity); per-particle outputs in dem_get_particles order (any may be null).
  void window_adjoint(const double* gR_host, double* grad_params, double* gvel, double* gang, double* gpos,
                      double* gquat) {
    AdjArgs A = adj_begin(gR_host);
    const int K = win.K, T = win.T, nw = (int)wig.size();
    const int t_pp = pick_tpp();
    d_wall_partial.reserve((size_t)step_grid(n, t_pp) * kMaxWalls * 3);
    const bool two = split == 1;
    for (int c = win.nseg - 1; c >= 0; --c) {
      const int len = std::min(K, T - c * K);
      adj_restore(c);  // recompute the segment's forward states from its checkpoint
      for (int j = 0; j < len; ++j) {
        if (nw)
          DEM_CUDA(cudaMemcpyAsync(win.st_walls.p + (size_t)j * kMaxWalls, d_walls.p, sizeof(WallDev) * nw,
                                   cudaMemcpyDeviceToDevice, s));
        const StepArgs a = adj_recompute_args(j);
        if (win.fp32) launch_step_fp32(a, rot != 0, t_pp, false, two, s);
        else launch_step(a, rot != 0, t_pp, two, s);
      }
      DEM_CUDA(cudaGetLastError());
      c_launches += two ? 2LL * len : len;
      for (int j = len - 1; j >= 0; --j) {  // reverse the segment
        adj_fill(A, c, j);
        launch_adjoint_step(A, s);
      }
      DEM_CUDA(cudaGetLastError());
    }
    adj_finish(grad_params, gvel, gang, gpos, gquat);
  }

  // ---- restart checkpoints: the worker's file of TSubLattice::saveCheckPointData /
  // loadCheckPointData (Parallel/SubLattice.hpp:3600-3790), written and read with the same
  // iostream formatting (the caller sets the precision, 12 digits by default).
  //
  // Scaled RotBond constants as CRotBondedInteraction's constructor forms them
  // (Model/RotBondedInteraction.cpp:122-161); the restart record carries them.
  static void bond_scaled(const BondGroup& B, double dist0, double r1, double r2, double* k) {
    double effR = 1.0, effL = 1.0, effA = 1.0, J = 1.0, I = 1.0;
    if (B.scaling) {
      effR = B.meanR ? 0.5 * dist0 : std::min(r1, r2);
      effL = dist0;
      effA = effR * effR;
      J = 0.5 * effR * effR * effR * effR;
      I = 0.5 * J;
    }
    k[0] = B.kr * effA / effL;  // kr
    k[1] = B.ks * effA / effL;  // ks
    k[2] = B.kb * I / effL;     // kb
    k[3] = B.kt * J / effL;     // kt
    k[4] = B.mn * effA;         // max_nForce
    k[5] = B.ms * effA;         // max_shForce
    k[6] = B.mt * J / effR;     // max_tMoment
    k[7] = B.mb * I / effR;     // max_bMoment
  }

  void save_checkpoint(std::ostream& os) {
    for (auto& b : bond)
      if (b.second.kind >= 2) throw std::invalid_argument("restart checkpoints of BrittleBeam groups are not built");
    download_walls();
    std::vector<double4> pr(n), vm(n), wi(n), qq(n), op(n), fo(n);
    std::vector<unsigned> pf(n);
    std::vector<int> tg(n);
    std::vector<double> csh(n);
    if (n) {
      const ParticleBuf& b = P.buf[cur];
      DEM_CUDA(cudaMemcpyAsync(pr.data(), b.pr, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(vm.data(), b.vm, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(wi.data(), b.wi, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(qq.data(), b.qq, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(op.data(), P.oldpos, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      if (store_forces) DEM_CUDA(cudaMemcpyAsync(fo.data(), P.force, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(pf.data(), P.pflags, sizeof(unsigned) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(tg.data(), P.tag, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(csh.data(), P.cshift, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    }
    sync();
    const char d = ' ';
    // ParallelParticleArray::saveCheckPointData (ppa/src/pp_array.hpp:1217-1236)
    os << g.p0x << d << g.p0y << d << g.p0z << "\n";
    os << g.gx << " " << g.gy << " " << g.gz << "\n";
    int alive = 0;
    for (int i = 0; i < n; ++i) alive += (pf[i] & PF_ALIVE) ? 1 : 0;
    os << alive << "\n";
    for (int i = 0; i < n; ++i) {
      if (!(pf[i] & PF_ALIVE)) continue;
      // CParticle::saveCheckPointData (Model/Particle.cpp:461-475): the initial position less the
      // circular shift, and the shift
      os << pr[i].x << d << pr[i].y << d << pr[i].z << d << pr[i].w << d << h_id[i] << d << tg[i] << d << vm[i].w << d
         << h_initpos[3 * (size_t)i] << d << h_initpos[3 * (size_t)i + 1] << d << h_initpos[3 * (size_t)i + 2] << d
         << op[i].x << d << op[i].y << d << op[i].z << d << vm[i].x << d << vm[i].y << d << vm[i].z << d
         << fo[i].x << d << fo[i].y << d << fo[i].z << d << csh[i] << d << 0.0 << d << 0.0 << d
         << ((pf[i] & PF_DYN) ? 1 : 0);
      if (rot)  // CRotParticle::saveCheckPointData (Model/RotParticle.cpp:510-519)
        os << d << wi[i].w << d << qq[i].x << d << qq[i].y << d << qq[i].z << d << qq[i].w << d << wi[i].x << d
           << wi[i].y << d << wi[i].z << d << ((pf[i] & PF_ROT) ? 1 : 0);
      os << "\n";
    }
    // bonded groups: PIS_EB::saveCheckPointData (pis/pi_storage_eb.hpp:79-97) per group, name order
    os << bond.size() << "\n";
    for (auto& it : bond) {
      BondGroup& B = it.second;
      std::vector<int2> ends(B.nb);
      std::vector<double4> D0(B.nb);
      std::vector<int> bs(B.nb);
      if (B.nb) {
        DEM_CUDA(cudaMemcpyAsync(ends.data(), B.ends.p, sizeof(int2) * B.nb, cudaMemcpyDeviceToHost, s));
        DEM_CUDA(cudaMemcpyAsync(D0.data(), B.D0.p, sizeof(double4) * B.nb, cudaMemcpyDeviceToHost, s));
        DEM_CUDA(cudaMemcpyAsync(bs.data(), B.broken_step.p, sizeof(int) * B.nb, cudaMemcpyDeviceToHost, s));
      }
      sync();
      // a bond that failed in the last step stays listed until the next update, as in the reference
      int intact = 0;
      for (int k = 0; k < B.nb; ++k) intact += bs[k] > t ? 1 : 0;
      if (B.kind == 1) {
        // CBondedInteraction::saveRestartData (Model/BondedInteraction.cpp:283-293); m_dist is the
        // distance of the last force evaluation, whose positions are the other particle buffer
        std::vector<double4> pl(n);
        if (n) DEM_CUDA(cudaMemcpyAsync(pl.data(), P.buf[cur ^ 1].pr, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
        sync();
        os << "Bonded" << "\n" << intact;
        for (int k = 0; k < B.nb; ++k) {
          if (!(bs[k] > t)) continue;
          const int i = ends[k].x, j = ends[k].y;
          const double r0 = pr[i].w + pr[j].w;
          double effR = 1.0, effA = 1.0, effL = 1.0;
          if (B.scaling) { effR = 0.5 * r0; effL = r0; effA = effR * effR; }
          double dx = pl[i].x - pl[j].x, dy = pl[i].y - pl[j].y, dz = pl[i].z - pl[j].z;
          if (g.circx) {  // minimum image, as the step kernel forms the pair
            if (dx > 0.5 * g.Lx) dx -= g.Lx; else if (dx < -0.5 * g.Lx) dx += g.Lx;
          }
          os << "\n" << B.knb * effA / effL << " " << r0 << " " << std::sqrt(dx * dx + dy * dy + dz * dz) << " "
             << r0 * B.rbreak << " " << (B.scaling ? 1 : 0) << " " << h_id[i] << " " << h_id[j] << " " << B.tag << "\n";
        }
        os << "\n";
        continue;
      }
      os << "RotBonded" << "\n";
      os << intact;
      for (int k = 0; k < B.nb; ++k) {
        if (!(bs[k] > t)) continue;
        const int i = ends[k].x, j = ends[k].y;
        const double dist0 = std::sqrt(D0[k].x * D0[k].x + D0[k].y * D0[k].y + D0[k].z * D0[k].z);
        double c[8];
        bond_scaled(B, dist0, pr[i].w, pr[j].w, c);
        // CRotBondedInteraction::saveRestartData (Model/RotBondedInteraction.cpp:379-399)
        os << "\n" << h_id[i] << " " << h_id[j] << " " << 1 << " " << c[0] << " " << c[1] << " " << c[2] << " " << c[3]
           << " " << (B.scaling ? 1 : 0) << " " << (B.meanR ? 1 : 0) << " " << B.truncated << " " << 1.0 << " " << 1.0
           << " " << c[4] << " " << c[5] << " " << c[6] << " " << c[7] << " " << D0[k].x << d << D0[k].y << d
           << D0[k].z << " " << B.tag << "\n";
      }
      os << "\n";
    }
    // dynamic groups that save (PIS_ED; PIS_NE saves nothing): PIS_ED::saveCheckPointData
    // (pis/pi_storage_ed.hpp:202-214).  The reference writes the record count and the first record
    // with no separator; a newline is written here so that the count can be read back.
    int nsave = 0;
    for (auto& it : dyn) nsave += (it.second.kind == 1 || it.second.kind == 2) ? 1 : 0;
    os << nsave << "\n";
    for (auto& it : dyn) {
      DynGroup& G = it.second;
      if (G.kind == 0 || G.kind >= 3) continue;  // PIS_NE storages do not save
      std::vector<unsigned long long> keys(G.m);
      std::vector<double4> h(G.m);
      std::vector<int> xb(handoff ? G.m : 0);
      if (G.m) {
        DEM_CUDA(cudaMemcpyAsync(keys.data(), G.keys.p, sizeof(unsigned long long) * G.m, cudaMemcpyDeviceToHost, s));
        if (fp32) {
          std::vector<float4> h32(G.m);
          DEM_CUDA(cudaMemcpyAsync(h32.data(), G.hist32[cur].p, sizeof(float4) * G.m, cudaMemcpyDeviceToHost, s));
          sync();
          for (int k = 0; k < G.m; ++k) h[k] = make_double4(h32[k].x, h32[k].y, h32[k].z, h32[k].w);
        } else {
          DEM_CUDA(cudaMemcpyAsync(h.data(), G.hist[cur].p, sizeof(double4) * G.m, cudaMemcpyDeviceToHost, s));
        }
        if (handoff) DEM_CUDA(cudaMemcpyAsync(xb.data(), G.xbond.p, sizeof(int) * G.m, cudaMemcpyDeviceToHost, s));
      }
      std::vector<std::vector<int>> bsteps;
      if (handoff)
        for (auto& b : bond) {
          bsteps.emplace_back(b.second.nb);
          if (b.second.nb)
            DEM_CUDA(cudaMemcpyAsync(bsteps.back().data(), b.second.broken_step.p, sizeof(int) * b.second.nb,
                                     cudaMemcpyDeviceToHost, s));
        }
      sync();
      std::vector<int> listed;
      for (int k = 0; k < G.m; ++k) {
        // the device bond hand-off keeps bond-held pairs that the reference's list does not have
        if (handoff && xb[k] >= 0 && bsteps[xb[k] >> 28][xb[k] & 0x0fffffff] > t) continue;
        listed.push_back(k);
      }
      os << (G.kind == 1 ? "RotFriction" : "Friction") << "\n";
      os << listed.size() << "\n";
      for (int k : listed) {
        const int i = (int)(keys[k] >> 32), j = (int)(keys[k] & 0xffffffffu);
        const double r1 = pr[i].w, r2 = pr[j].w;
        if (G.kind == 2) {  // CFrictionInteraction::saveRestartData (Model/FrictionInteraction.cpp:628-643)
          const double f = G.scaling ? 0.5 * (r1 + r2) : 1.0;
          const int fl = (int)h[k].w;
          os << f * G.k << " " << r1 + r2 << " " << G.mu_s << " " << f * G.ks << " " << G.dt << " "
             << (G.scaling ? 1 : 0) << " " << h_id[i] << " " << h_id[j] << " " << (fl & 1) << " " << ((fl >> 1) & 1)
             << " " << h[k].x << " " << h[k].y << " " << h[k].z << "\n";
          continue;
        }
        // scaled stiffnesses as CRotFrictionInteraction's constructor forms them (Model/RotFricInteraction.cpp:103-146)
        double effR = 1.0, effL = 1.0, effA = 1.0;
        const double r0 = r1 + r2;
        if (G.scaling) {
          effR = G.meanR ? 0.5 * r0 : std::min(r1, r2);
          effL = r0;
          effA = effR * effR;
        }
        const int flags = (int)h[k].w;
        // CRotFrictionInteraction::saveRestartData (Model/RotFricInteraction.cpp:597-614)
        os << G.k * effA / effL << " " << r0 << " " << G.mu_d << " " << G.mu_s << " " << G.ks * effA / effL << " "
           << G.dt << " " << (G.scaling ? 1 : 0) << " " << (G.meanR ? 1 : 0) << " " << h_id[i] << " " << h_id[j] << " "
           << (flags & 1) << " " << ((flags >> 1) & 1) << " " << h[k].x << " " << h[k].y << " " << h[k].z << "\n";
      }
      os << "\n";
    }
    // walls (name, CWall::writeCheckPoint, Model/Wall.cpp:118-121), then the empty body and mesh sections
    os << "Walls " << walls.size() << "\n";
    for (auto& w : walls) {
      const Wall& W = w.second;
      os << w.first << "\n";
      os << W.o[0] << d << W.o[1] << d << W.o[2] << " " << W.old[0] << d << W.old[1] << d << W.old[2] << " "
         << W.n[0] << d << W.n[1] << d << W.n[2] << "\n";
    }
    os << "Spheres " << 0 << "\n";
    os << "TriMesh " << 0 << "\n";
    os << "Mesh2D " << 0 << "\n";
  }

  // Snapshot (visualisation / post-processing) file of TSubLattice::saveSnapShotData
  // (Parallel/SubLattice.hpp:3552-3594): 9 significant digits, CParticle / CRotParticle
  // snapshot records (Model/Particle.cpp:443-456, Model/RotParticle.cpp:494-503), then each bonded
  // group's (id1, id2, tag) records (pis/pi_storage_eb.hpp:54-71, BondedInteractionCpData).
  void save_snapshot(std::ostream& os) {
    const std::streamsize oldprec = os.precision(9);
    std::vector<double4> pr(n), vm(n), wi(n), qq(n), op(n), fo(n);
    std::vector<unsigned> pf(n);
    std::vector<int> tg(n);
    std::vector<double> csh(n);
    if (n) {
      const ParticleBuf& b = P.buf[cur];
      DEM_CUDA(cudaMemcpyAsync(pr.data(), b.pr, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(vm.data(), b.vm, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(wi.data(), b.wi, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(qq.data(), b.qq, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(op.data(), P.oldpos, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      if (store_forces) DEM_CUDA(cudaMemcpyAsync(fo.data(), P.force, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(pf.data(), P.pflags, sizeof(unsigned) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(tg.data(), P.tag, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
      DEM_CUDA(cudaMemcpyAsync(csh.data(), P.cshift, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    }
    sync();
    const char d = ' ';
    int alive = 0;
    for (int i = 0; i < n; ++i) alive += (pf[i] & PF_ALIVE) ? 1 : 0;
    os << alive << "\n";
    for (int i = 0; i < n; ++i) {
      if (!(pf[i] & PF_ALIVE)) continue;
      os << pr[i].x << d << pr[i].y << d << pr[i].z << d << pr[i].w << d << h_id[i] << d << tg[i] << d << vm[i].w << d
         << h_initpos[3 * (size_t)i] << d << h_initpos[3 * (size_t)i + 1] << d << h_initpos[3 * (size_t)i + 2] << d
         << op[i].x << d << op[i].y << d << op[i].z << d << vm[i].x << d << vm[i].y << d << vm[i].z << d
         << fo[i].x << d << fo[i].y << d << fo[i].z << d << csh[i] << d << 0.0 << d << 0.0;
      if (rot)
        os << d << qq[i].x << d << qq[i].y << d << qq[i].z << d << qq[i].w << d << wi[i].x << d << wi[i].y << d
           << wi[i].z;
      os << "\n";
    }
    os << bond.size() << "\n";
    for (auto& it : bond) {
      BondGroup& B = it.second;
      std::vector<int2> ends(B.nb);
      std::vector<int> bs(B.nb);
      if (B.nb) {
        DEM_CUDA(cudaMemcpyAsync(ends.data(), B.ends.p, sizeof(int2) * B.nb, cudaMemcpyDeviceToHost, s));
        DEM_CUDA(cudaMemcpyAsync(bs.data(), B.broken_step.p, sizeof(int) * B.nb, cudaMemcpyDeviceToHost, s));
      }
      sync();
      int intact = 0;
      for (int k = 0; k < B.nb; ++k) intact += bs[k] > t ? 1 : 0;
      os << "RotBonded" << "\n" << intact;
      for (int k = 0; k < B.nb; ++k)
        if (bs[k] > t) os << "\n" << h_id[ends[k].x] << d << h_id[ends[k].y] << d << B.tag;
      os << "\n";
    }
    os << "TMIG " << 0 << "\n";
    os.precision(oldprec);
  }

  // Reads a worker file into this worker: particles (into an empty worker), each bonded group's
  // bonds with their creation vectors, each RotFriction group's pairs with their tangential
  // history (carried through the neighbour search that follows, for the pairs still touching, as
  // PIS_ED::update keeps them), and the walls.  The groups themselves come from the script, as in
  // the reference; the per-interaction constants in the file are not read back (they follow from
  // the groups' parameters).  timestep: the master's step counter (CheckPointInfo).
  void load_checkpoint(std::istream& is, long long timestep) {
    if (n) throw StateError("a checkpoint is loaded into a worker without particles");
    for (auto& b : bond)
      if (b.second.kind >= 2) throw std::invalid_argument("restart checkpoints of BrittleBeam groups are not built");
    auto fail = [&](const std::string& what) { throw std::invalid_argument("checkpoint: " + what); };
    double bp[3];
    int bi[3];
    is >> bp[0] >> bp[1] >> bp[2] >> bi[0] >> bi[1] >> bi[2];
    int np = 0;
    is >> np;
    if (!is || np < 0) fail("bad particle block header");
    std::vector<int> ids(np), tags(np), flags(np);
    std::vector<double> pos(3 * (size_t)np), rad(np), mass(np), vel(3 * (size_t)np), angvel(3 * (size_t)np),
        quat(4 * (size_t)np), initpos(3 * (size_t)np), shx(np);
    for (int i = 0; i < np; ++i) {
      double op[3], f[3], sh[3];
      int dynb = 1, rotb = 1;
      is >> pos[3 * i] >> pos[3 * i + 1] >> pos[3 * i + 2] >> rad[i] >> ids[i] >> tags[i] >> mass[i] >> initpos[3 * i]
         >> initpos[3 * i + 1] >> initpos[3 * i + 2] >> op[0] >> op[1] >> op[2] >> vel[3 * i] >> vel[3 * i + 1]
         >> vel[3 * i + 2] >> f[0] >> f[1] >> f[2] >> sh[0] >> sh[1] >> sh[2] >> dynb;
      shx[i] = sh[0];  // x: the circular shift, carried on the device
      for (int k = 1; k < 3; ++k) initpos[3 * i + k] += sh[k];
      quat[4 * i] = 1.0;
      if (rot) {
        double inert;
        is >> inert >> quat[4 * i] >> quat[4 * i + 1] >> quat[4 * i + 2] >> quat[4 * i + 3] >> angvel[3 * i]
           >> angvel[3 * i + 1] >> angvel[3 * i + 2] >> rotb;
      }
      if (!is) fail("bad particle record " + std::to_string(i));
      flags[i] = (dynb ? 0 : 1) | (rotb ? 0 : 2);
    }
    add_particles(np, ids.data(), tags.data(), pos.data(), rad.data(), mass.data(), vel.data(),
                  rot ? angvel.data() : nullptr, rot ? quat.data() : nullptr, flags.data());
    std::vector<double> csh(n, 0.0);
    for (int i = 0; i < np; ++i) {
      auto sl = id2slot.find(ids[i]);
      if (sl == id2slot.end()) continue;
      for (int k = 0; k < 3; ++k) h_initpos[3 * (size_t)sl->second + k] = initpos[3 * i + k];
      csh[sl->second] = shx[i];
    }
    if (n) DEM_CUDA(cudaMemcpyAsync(P.cshift, csh.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
    std::vector<double4> pr(n);
    if (n) DEM_CUDA(cudaMemcpyAsync(pr.data(), P.buf[cur].pr, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
    sync();
    // bonded groups, name order (the reference's map order)
    unsigned nbg = 0;
    is >> nbg;
    if (!is || nbg != bond.size()) fail("the number of bonded groups differs from the script's");
    for (auto& it : bond) {
      BondGroup& B = it.second;
      std::string type;
      int nconn = 0;
      is >> type >> nconn;
      const std::string want_type = B.kind == 1 ? "Bonded" : "RotBonded";
      if (!is || type != want_type) fail("expected " + want_type + " interactions, got " + type);
      std::vector<std::pair<unsigned long long, double4>> rec;
      for (int q = 0; q < nconn && B.kind == 1; ++q) {  // CBondedInteraction::loadRestartData (:300-312)
        double k, r0, dist, brk;
        int scl, a, b, tag;
        is >> k >> r0 >> dist >> brk >> scl >> a >> b >> tag;
        if (!is) fail("bad Bonded record " + std::to_string(q));
        if (a > b) std::swap(a, b);
        auto ia = id2slot.find(a), ib = id2slot.find(b);
        if (ia == id2slot.end() || ib == id2slot.end()) continue;
        rec.push_back({((unsigned long long)(unsigned)ia->second << 32) | (unsigned)ib->second, make_double4(0, 0, 0, 0)});
      }
      for (int q = 0; q < nconn && B.kind == 0; ++q) {
        int a, b, init, scl, mr, tag;
        double kr, ks, kb, kt, tr, b1, b2, mn, ms, mt, mb, Dx, Dy, Dz;
        is >> a >> b >> init >> kr >> ks >> kb >> kt >> scl >> mr >> tr >> b1 >> b2 >> mn >> ms >> mt >> mb >> Dx >> Dy
           >> Dz >> tag;
        if (!is) fail("bad RotBonded record " + std::to_string(q));
        if (a > b) { std::swap(a, b); Dx = -Dx; Dy = -Dy; Dz = -Dz; }  // p1 is the lower id
        auto ia = id2slot.find(a), ib = id2slot.find(b);
        if (ia == id2slot.end() || ib == id2slot.end()) continue;  // "particles ... not present"
        rec.push_back({((unsigned long long)(unsigned)ia->second << 32) | (unsigned)ib->second,
                       make_double4(Dx, Dy, Dz, 0.0)});
      }
      std::sort(rec.begin(), rec.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
      rec.erase(std::unique(rec.begin(), rec.end(), [](const auto& x, const auto& y) { return x.first == y.first; }),
                rec.end());
      B.nb = (int)rec.size();
      const int nb = std::max(B.nb, 1);
      B.keys.reserve(nb); B.ends.reserve(nb); B.D0.reserve(nb); B.broken_step.reserve(nb);
      B.cap_events = event_cap(B.nb);
      B.events.reserve(3 * B.cap_events); B.nevents.reserve(1);
      std::vector<unsigned long long> keys(B.nb);
      std::vector<int2> ends(B.nb);
      std::vector<double4> D0(B.nb);
      std::vector<int> alive(B.nb, kBondAlive);
      for (int k = 0; k < B.nb; ++k) {
        keys[k] = rec[k].first;
        ends[k] = make_int2((int)(keys[k] >> 32), (int)(keys[k] & 0xffffffffu));
        D0[k] = rec[k].second;
      }
      if (B.nb) {
        DEM_CUDA(cudaMemcpyAsync(B.keys.p, keys.data(), sizeof(unsigned long long) * B.nb, cudaMemcpyHostToDevice, s));
        DEM_CUDA(cudaMemcpyAsync(B.ends.p, ends.data(), sizeof(int2) * B.nb, cudaMemcpyHostToDevice, s));
        DEM_CUDA(cudaMemcpyAsync(B.D0.p, D0.data(), sizeof(double4) * B.nb, cudaMemcpyHostToDevice, s));
        DEM_CUDA(cudaMemcpyAsync(B.broken_step.p, alive.data(), sizeof(int) * B.nb, cudaMemcpyHostToDevice, s));
      }
      DEM_CUDA(cudaMemsetAsync(B.nevents.p, 0, sizeof(int), s));
      build_adjacency(B.keys, B.nb, B.adj_start, B.adj_count, B.adj_cursor, B.p1_start, B.adj);
      sync();
    }
    // RotFriction groups: the pairs and histories become the list the next search updates
    unsigned nsave = 0;
    is >> nsave;
    unsigned want = 0;
    for (auto& it : dyn) want += (it.second.kind == 1 || it.second.kind == 2) ? 1 : 0;
    if (!is || nsave != want) fail("the number of friction groups differs from the script's");
    for (auto& it : dyn) {
      DynGroup& G = it.second;
      if (G.kind == 0 || G.kind >= 3) continue;
      std::string type;
      is >> type;
      const std::string want_type = G.kind == 1 ? "RotFriction" : "Friction";
      if (!is || type != want_type) fail("expected " + want_type + " interactions, got " + type);
      // One record per line up to the group's blank line.  The first line is the record count
      // (this library's files) or, in the reference's files, the count run together with the
      // first record's scaled normal stiffness, which is not read back.
      std::string line;
      std::getline(is, line);  // the rest of the type line
      std::vector<std::string> lines;
      long long count = -1;
      while (std::getline(is, line)) {
        if (line.find_first_not_of(" \t\r") == std::string::npos) {
          if (count >= 0 || !lines.empty()) break;
          continue;
        }
        std::istringstream ls(line);
        std::vector<std::string> tok;
        for (std::string w; ls >> w;) tok.push_back(w);
        if (count < 0 && lines.empty() && tok.size() == 1) { count = std::stoll(tok[0]); if (count == 0) break; continue; }
        lines.push_back(line);
        if (count >= 0 && (long long)lines.size() == count) break;
      }
      std::vector<std::pair<unsigned long long, double4>> rec;
      for (size_t q = 0; q < lines.size(); ++q) {
        std::istringstream ls(lines[q]);
        std::string k;  // scaled normal stiffness (or the count run together with it): not read back
        double r0, mud, mus, ks, dtg, fx, fy, fz;
        int scl, mr = 0, a, b, slip, touch;
        if (G.kind == 1)
          ls >> k >> r0 >> mud >> mus >> ks >> dtg >> scl >> mr >> a >> b >> slip >> touch >> fx >> fy >> fz;
        else  // CFrictionInteraction::loadRestartData (Model/FrictionInteraction.cpp:651-666)
          ls >> k >> r0 >> mud >> ks >> dtg >> scl >> a >> b >> slip >> touch >> fx >> fy >> fz;
        if (!ls) fail("bad " + want_type + " record " + std::to_string(q));
        if (a > b) { std::swap(a, b); fx = -fx; fy = -fy; fz = -fz; }  // the history is the force on p1
        auto ia = id2slot.find(a), ib = id2slot.find(b);
        if (ia == id2slot.end() || ib == id2slot.end()) continue;
        rec.push_back({((unsigned long long)(unsigned)ia->second << 32) | (unsigned)ib->second,
                       make_double4(fx, fy, fz, (double)((slip ? 1 : 0) + (touch ? 2 : 0)))});
      }
      std::sort(rec.begin(), rec.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
      rec.erase(std::unique(rec.begin(), rec.end(), [](const auto& x, const auto& y) { return x.first == y.first; }),
                rec.end());
      G.m = (int)rec.size();
      const int m = std::max(G.m, 1);
      G.keys.reserve(m);
      for (int c = 0; c < 2; ++c) G.hist[c].reserve(m);
      if (fp32) for (int c = 0; c < 2; ++c) G.hist32[c].reserve(m);
      std::vector<unsigned long long> keys(G.m);
      std::vector<double4> h(G.m);
      for (int q = 0; q < G.m; ++q) { keys[q] = rec[q].first; h[q] = rec[q].second; }
      if (G.m) {
        DEM_CUDA(cudaMemcpyAsync(G.keys.p, keys.data(), sizeof(unsigned long long) * G.m, cudaMemcpyHostToDevice, s));
        DEM_CUDA(cudaMemcpyAsync(G.hist[cur].p, h.data(), sizeof(double4) * G.m, cudaMemcpyHostToDevice, s));
        if (fp32) launch_hist_convert(G.m, G.hist[cur].p, G.hist32[cur].p, true, s);
      }
      sync();
    }
    // walls
    std::string token;
    int nw = 0;
    is >> token >> nw;
    if (!is || token != "Walls") fail("expected Walls, got " + token);
    download_walls();
    for (int k = 0; k < nw; ++k) {
      std::string name;
      Wall W;
      is >> name >> W.o[0] >> W.o[1] >> W.o[2] >> W.old[0] >> W.old[1] >> W.old[2] >> W.n[0] >> W.n[1] >> W.n[2];
      if (!is) fail("bad wall record");
      walls[name] = W;
    }
    upload_walls();
    for (const char* sec : {"Spheres", "TriMesh", "Mesh2D"}) {
      int cnt = 0;
      is >> token >> cnt;
      if (!is || token != sec) fail(std::string("expected ") + sec + ", got " + token);
      if (cnt != 0) fail(std::string(sec) + " are not part of this worker");
    }
    // CLatticeMaster::loadCheckPointData (Parallel/LatticeMaster.cpp:780-820): the step counter,
    // then searchNeighbors(true) and updateInteractions
    t = timestep;
    DEM_CUDA(cudaMemcpyAsync(d_step.p, &t, sizeof(long long), cudaMemcpyHostToDevice, s));
    sync();
    search_neighbors();
    resize_adjacency();
    pending_ctrl = 0;
  }

  void set_group_param(const std::string& group, const std::string& key, double v) {
    auto b = bond.find(group);
    if (b != bond.end()) {
      BondGroup& B = b->second;
      if (key == "normalK") B.kr = v;
      else if (key == "shearK") B.ks = v;
      else if (key == "torsionK") B.kt = v;
      else if (key == "bendingK") B.kb = v;
      else throw std::invalid_argument("unknown RotBond parameter " + key);
      return;
    }
    auto d = dyn.find(group);
    if (d != dyn.end()) {
      DynGroup& G = d->second;
      if (key == "normalK") G.k = v;
      else if (key == "shearK" && G.kind != 0) G.ks = v;
      else if (key == "dynamicMu" && G.kind != 0) G.mu_d = v;
      else if (key == "staticMu" && G.kind != 0) G.mu_s = v;
      else throw std::invalid_argument("unknown parameter " + key + " of group " + group);
      return;
    }
    if (group == "Damping" && damp_lin && key == "viscosity") { visc_lin = v; return; }
    if (group == "RotDamping" && damp_rot && key == "viscosity") { visc_rot = v; return; }
    throw std::invalid_argument("unknown group " + group);
  }

  // Put the simulation back to the state at the start of the window.
  void window_rewind() {
    if (!win.valid) throw StateError("no differentiable window has been run");
    if (timestamp != win.ts || n != win.n) throw StateError("the topology changed since the window was run");
    auto dl = dyn_list();
    cur = win.cur0;
    copy_state(P.buf[cur], view4(win.ck.p, n));
    if (fp32) launch_sync_vw(P, cur, s);
    for (int d = 0; d < (int)dl.size(); ++d)
      if (dl[d]->kind == 1 && win.m[d]) {
        if (fp32)
          launch_hist_convert(win.m[d], win.ck_hist[d].p, dl[d]->hist32[cur].p, true, s);
        else
          DEM_CUDA(cudaMemcpyAsync(dl[d]->hist[cur].p, win.ck_hist[d].p, sizeof(double4) * win.m[d],
                                   cudaMemcpyDeviceToDevice, s));
      }
    if (!wig.empty())
      DEM_CUDA(cudaMemcpyAsync(d_walls.p, win.ck_walls.p, sizeof(WallDev) * wig.size(), cudaMemcpyDeviceToDevice, s));
    if (win.brk) {  // undo the window's bond failures
      int b = 0;
      for (auto& bg : bond) {
        BondGroup& B = bg.second;
        if (B.nb)
          DEM_CUDA(cudaMemcpyAsync(B.broken_step.p, win.bs0[b].p, sizeof(int) * B.nb, cudaMemcpyDeviceToDevice, s));
        DEM_CUDA(cudaMemcpyAsync(B.nevents.p, win.nev0.p + b, sizeof(int), cudaMemcpyDeviceToDevice, s));
        ++b;
      }
      if (n) {
        DEM_CUDA(cudaMemcpyAsync(P.flagged, win.flag0.p, n, cudaMemcpyDeviceToDevice, s));
        DEM_CUDA(cudaMemcpyAsync(P.pflags, win.ck_pf.p, sizeof(unsigned) * n, cudaMemcpyDeviceToDevice, s));
      }
      DEM_CUDA(cudaMemcpyAsync(d_brk.p, win.ck_brk.p, 2 * sizeof(int), cudaMemcpyDeviceToDevice, s));
    }
    t = win.t0;
    DEM_CUDA(cudaMemcpyAsync(d_step.p, &t, sizeof(long long), cudaMemcpyHostToDevice, s));
    pending_ctrl = 0;
    sync();
    if (win.brk) refresh_counts();
    download_walls();
  }
};

// ---- batched ensemble (many independent workers, one launch per timestep) ----
// Each specimen is a complete DemSim: its rebuilds, interaction updates, bond
// failures and step counter stay its own, so each advances exactly as it would
// alone.  Between chunks the host runs every specimen's runOneStep head
// (prepare); within a chunk one k_step_batch launch per timestep advances every
// specimen that has not stopped or reached its target.  Chunks are replayed from
// a captured CUDA graph (the kernels read everything through a fixed device
// table, so one graph per chunk length serves every chunk).
struct Ensemble {
  std::string err;
  std::vector<DemSim*> sims;
  std::vector<cudaStream_t> saved;
  cudaStream_t s = nullptr;
  int tpp = 0, chunk = 64, use_graph = 1, profile = 0;
  int rot = 0, fp32 = 0;
  bool el = false, fr = false, bd = false, gather = false;
  DBuf<StepArgs> d_args;
  DBuf<int> d_tile_start, d_btile_start, d_base_cur, d_status_ctrl;
  DBuf<long long> d_base_t, d_target, d_status_t;
  StepArgs* h_args = nullptr;   // pinned staging of the table
  long long* h_t = nullptr;     // pinned status
  int* h_ctrl = nullptr;
  std::map<int, cudaGraphExec_t> graphs;  // chunk length -> instantiated graph
  int graph_tpp = -1, graph_tiles = -1, graph_gather = -1;
  long long c_steps = 0, c_contacts = 0, c_launches = 0, c_chunks = 0, c_rebuild_calls = 0;
  double prof_ms = 0.0;
  long long prof_steps = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  Ensemble(DemSim* const* list, int n) {
    if (n < 1) throw std::invalid_argument("an ensemble needs at least one specimen");
    for (int k = 0; k < n; ++k) {
      if (!list[k]) throw std::invalid_argument("null specimen handle");
      for (int j = 0; j < k; ++j)
        if (list[j] == list[k]) throw std::invalid_argument("a specimen appears twice in the ensemble");
      sims.push_back(list[k]);
    }
    rot = sims[0]->rot;
    for (DemSim* d : sims) {
      if (d->rot != rot) throw std::invalid_argument("ensemble specimens must share the particle type");
      if (d->widened()) throw std::invalid_argument("the batched ensemble covers NRotElastic, RotFriction and RotBond groups");
    }
    DEM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    const int ns = (int)sims.size();
    d_args.reserve((size_t)2 * ns);
    d_tile_start.reserve(ns + 1);
    d_btile_start.reserve((size_t)ns * kMaxBond + 1);
    d_base_cur.reserve(ns);
    d_base_t.reserve(ns);
    d_target.reserve(ns);
    d_status_t.reserve(ns);
    d_status_ctrl.reserve(ns);
    DEM_CUDA(cudaMallocHost(&h_args, sizeof(StepArgs) * 2 * ns));
    DEM_CUDA(cudaMallocHost(&h_t, sizeof(long long) * ns));
    DEM_CUDA(cudaMallocHost(&h_ctrl, sizeof(int) * ns));
  }
  ~Ensemble() {
    if (s) cudaStreamSynchronize(s);
    d_wbase.release(); d_wtab.release(); d_abase.release(); d_atab.release(); d_wspec.release();
    d_ptile.release(); d_bptile.release(); d_dtile.release();
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    d_args.release(); d_tile_start.release(); d_btile_start.release(); d_base_cur.release(); d_status_ctrl.release();
    d_base_t.release(); d_target.release(); d_status_t.release();
    if (h_args) cudaFreeHost(h_args);
    if (h_t) cudaFreeHost(h_t);
    if (h_ctrl) cudaFreeHost(h_ctrl);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (s) cudaStreamDestroy(s);
  }

  // Work of the specimens runs on the ensemble's stream for the duration of a call.
  void borrow() {
    saved.clear();
    for (DemSim* d : sims) {
      d->sync();
      saved.push_back(d->s);
      d->s = s;
    }
  }
  void give_back() {
    cudaStreamSynchronize(s);
    for (size_t k = 0; k < sims.size() && k < saved.size(); ++k) sims[k]->s = saved[k];
    saved.clear();
  }

  int pick_tpp() const {
    if (tpp == kTiled) {
      bool tiled = true;
      for (DemSim* d : sims) tiled = tiled && d->tiled_ok() && (d->bond.empty() || d->bond_pass);
      return tiled ? kTiled : 1;
    }
    if (tpp) return tpp;
    long long e = 0, np = 0;
    for (DemSim* d : sims) {
      for (auto& g : d->dyn) e += 2LL * g.second.m;
      for (auto& b : d->bond) e += 2LL * b.second.nb;
      np += d->n;
    }
    const double mean = np ? (double)e / np : 0.0;
    if (mean >= 12) return 8;
    if (mean >= 6) return 4;
    if (mean >= 2.5) return 2;
    return 1;
  }

  void launch_chunk(const BatchArgs& B, int k, int t_pp) {
    auto one = [&]() {
      if (fp32) launch_batch_step_fp32(B, rot != 0, el, fr, bd, gather, t_pp, s);
      else launch_batch_step(B, rot != 0, el, fr, bd, gather, t_pp, s);
    };
    if (!use_graph) {
      for (int j = 0; j < k; ++j) one();
      DEM_CUDA(cudaGetLastError());
      return;
    }
    if (graph_tpp != t_pp || graph_tiles != B.total_tiles || graph_gather != (int)gather) {
      // a new launch shape runs once uncaptured first (it sets up the per-instance occupancy
      // query), then later chunks are captured and replayed
      for (auto& g : graphs) cudaGraphExecDestroy(g.second);
      graphs.clear();
      graph_tpp = t_pp;
      graph_tiles = B.total_tiles;
      graph_gather = gather;
      for (int j = 0; j < k; ++j) one();
      DEM_CUDA(cudaGetLastError());
      return;
    }
    auto it = graphs.find(k);
    if (it == graphs.end()) {
      cudaGraph_t g = nullptr;
      DEM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      for (int j = 0; j < k; ++j) one();
      const cudaError_t le = cudaGetLastError();
      const cudaError_t ce = cudaStreamEndCapture(s, &g);
      DEM_CUDA(le);
      DEM_CUDA(ce);
      cudaGraphExec_t ex = nullptr;
      const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      DEM_CUDA(ie);
      it = graphs.emplace(k, ex).first;
    }
    DEM_CUDA(cudaGraphLaunch(it->second, s));
  }

  // Families present over the specimens (the batch instance to launch).
  void scan_families() {
    el = fr = bd = false;
    gather = true;
    for (DemSim* d : sims) {
      for (auto& g : d->dyn) (g.second.kind == 0 ? el : fr) = true;
      if (!d->bond.empty()) {
        bd = true;
        if (!d->bond_pass) gather = false;
      }
    }
    gather = gather && bd;
  }

  // Bond-pass tiles per (specimen, bond group) and step tiles per specimen, uploaded.
  int upload_tiles(int t_pp, std::vector<int>& tile_start) {
    const int ns = (int)sims.size();
    tile_start.assign(ns + 1, 0);
    std::vector<int> btile_start((size_t)ns * kMaxBond + 1, 0);
    for (int k = 0; k < ns; ++k) {
      DemSim& d = *sims[k];
      int q = 0;
      for (auto& b : d.bond) {
        if (q >= kMaxBond) break;
        btile_start[(size_t)k * kMaxBond + q + 1] = (b.second.nb + kBondPassThreads - 1) / kBondPassThreads;
        ++q;
      }
      tile_start[k + 1] = tile_start[k] + step_grid(d.n, t_pp);
      d.d_wall_partial.reserve((size_t)step_grid(d.n, t_pp) * kMaxWalls * 3);
    }
    for (size_t it = 0; it < (size_t)ns * kMaxBond; ++it) btile_start[it + 1] += btile_start[it];
    DEM_CUDA(cudaMemcpyAsync(d_btile_start.p, btile_start.data(), sizeof(int) * btile_start.size(),
                             cudaMemcpyHostToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(d_tile_start.p, tile_start.data(), sizeof(int) * (ns + 1), cudaMemcpyHostToDevice, s));
    return btile_start[(size_t)ns * kMaxBond];
  }

  // One chunk of up to k steps for every specimen below its target: the step table (with the
  // window's reaction record when `window`), a graph replay, and every specimen's counter and
  // control word read back into h_t / h_ctrl.  `head`: run each unfinished specimen's
  // runOneStep head first.  Returns false if a head failed (err is set).
  bool run_chunk(const std::vector<long long>& target, int k, int t_pp, bool head, bool window, std::vector<long long>& cps) {
    const int ns = (int)sims.size();
    std::vector<int> base_cur(ns);
    std::vector<long long> base_t(ns);
    cps.assign(ns, 0);
    if (head)
      for (int q = 0; q < ns; ++q) {
        DemSim& d = *sims[q];
        if (d.t < target[q] && !d.prepare()) { err = "specimen " + std::to_string(q) + ": " + d.err; return false; }
      }
    // tiles after the heads (bond counts may change), step arguments after the tiles (the
    // wall-partial scratch they point to is sized there)
    scan_families();
    std::vector<int> tile_start;
    const int total_btiles = upload_tiles(t_pp, tile_start);
    for (int q = 0; q < ns; ++q) {
      DemSim& d = *sims[q];
      h_args[2 * q] = d.make_args(0);
      h_args[2 * q + 1] = d.make_args(1);
      h_args[2 * q].store_forces = h_args[2 * q + 1].store_forces = d.store_forces;
      h_args[2 * q].force_step = h_args[2 * q + 1].force_step = target[q];
      if (window) {
        for (int c = 0; c < 2; ++c) {
          h_args[2 * q + c].wall_hist = d.win.R.p;
          h_args[2 * q + c].wall_hist_t0 = d.win.t0;
        }
      }
      base_cur[q] = d.cur;
      base_t[q] = d.t;
      cps[q] = d.contacts_per_step();
    }
    DEM_CUDA(cudaMemcpyAsync(d_args.p, h_args, sizeof(StepArgs) * 2 * ns, cudaMemcpyHostToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(d_base_cur.p, base_cur.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(d_base_t.p, base_t.data(), sizeof(long long) * ns, cudaMemcpyHostToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(d_target.p, target.data(), sizeof(long long) * ns, cudaMemcpyHostToDevice, s));
    launch_batch_reset(d_args.p, ns, s);
    if (fp32) launch_batch_sync_vw(d_args.p, d_base_cur.p, ns, s);
    BatchArgs B{};
    B.nspec = ns;
    B.total_tiles = tile_start[ns];
    B.args = d_args.p;
    B.tile_start = d_tile_start.p;
    B.base_t = d_base_t.p;
    B.base_cur = d_base_cur.p;
    B.target = d_target.p;
    B.btile_start = d_btile_start.p;
    B.total_btiles = total_btiles;
    if (profile) {
      if (!ev0) { DEM_CUDA(cudaEventCreate(&ev0)); DEM_CUDA(cudaEventCreate(&ev1)); }
      DEM_CUDA(cudaEventRecord(ev0, s));
    }
    launch_chunk(B, k, t_pp);
    if (profile) DEM_CUDA(cudaEventRecord(ev1, s));
    launch_batch_status(d_args.p, ns, d_status_t.p, d_status_ctrl.p, s);
    DEM_CUDA(cudaMemcpyAsync(h_t, d_status_t.p, sizeof(long long) * ns, cudaMemcpyDeviceToHost, s));
    DEM_CUDA(cudaMemcpyAsync(h_ctrl, d_status_ctrl.p, sizeof(int) * ns, cudaMemcpyDeviceToHost, s));
    DEM_CUDA(cudaStreamSynchronize(s));
    c_launches += k + 3 + (fp32 ? 1 : 0);
    ++c_chunks;
    if (profile) {
      float ms = 0.f;
      DEM_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
      prof_ms += ms;
      prof_steps += k;
    }
    return true;
  }

  void check_form() {
    fp32 = sims[0]->fp32;
    for (DemSim* d : sims)
      if (d->fp32 != fp32) throw std::invalid_argument("ensemble specimens must share the precision form");
  }

  int step(int nsteps) {
    if (nsteps < 0) throw std::invalid_argument("negative step count");
    const int ns = (int)sims.size();
    check_form();
    borrow();
    struct Back { Ensemble* e; ~Back() { e->give_back(); } } back{this};
    std::vector<long long> target(ns);
    for (int k = 0; k < ns; ++k) target[k] = sims[k]->t + nsteps;
    const int t_pp = pick_tpp();
    std::vector<long long> cps;
    int overflow_at = -1;
    while (true) {
      long long remaining = 0;
      for (int k = 0; k < ns; ++k) remaining = std::max(remaining, target[k] - sims[k]->t);
      if (remaining <= 0) break;
      const int k = (int)std::min<long long>(chunk, remaining);
      if (!run_chunk(target, k, t_pp, true, false, cps)) return DEM_ERR_OVERFLOW;
      long long ran_total = 0;
      for (int j = 0; j < ns; ++j) {
        DemSim& d = *sims[j];
        const long long ran = h_t[j] - d.t;
        if (ran < 0 || ran > k) { err = "specimen " + std::to_string(j) + ": step counter out of sequence"; return -3; }
        d.t = h_t[j];
        d.cur = (int)((d.cur + ran) & 1);
        d.c_steps += ran;
        d.c_contacts += ran * cps[j];
        d.pending_ctrl = h_ctrl[j];
        if (d.take_overflow() && overflow_at < 0) overflow_at = j;
        c_steps += ran;
        c_contacts += ran * cps[j];
        ran_total += ran;
        if (h_ctrl[j] & CTRL_REBUILD) ++c_rebuild_calls;
      }
      if (ran_total == 0) { err = "no specimen advanced in a chunk"; return -3; }
    }
    if (overflow_at >= 0) {
      err = "specimen " + std::to_string(overflow_at) + ": " + DemSim::kOverflowText;
      return DEM_ERR_OVERFLOW;
    }
    return 0;
  }

  // ---- batched differentiable windows --------------------------------------------------
  // Every specimen runs the same window (nsteps from its own current step, checkpoints every
  // K) as DemSim::window_forward would alone: the forward in batched chunks, one per
  // checkpoint segment; the reverse with one launch per kernel and step for all specimens,
  // the per-step arguments expanded on the device from each specimen's base.
  DBuf<StepArgs> d_wbase, d_wtab;
  DBuf<AdjArgs> d_abase, d_atab;
  DBuf<WinSpec> d_wspec;
  DBuf<int> d_ptile, d_bptile, d_dtile;

  static std::string where(int k, const std::string& what) { return "specimen " + std::to_string(k) + ": " + what; }

  int window_forward(int T, int K, double* const* R) {
    const int ns = (int)sims.size();
    check_form();
    borrow();
    struct Back { Ensemble* e; ~Back() { e->give_back(); } } back{this};
    for (int k = 0; k < ns; ++k) {
      try {
        if (!sims[k]->win_begin(T, K)) { err = where(k, sims[k]->err); return DEM_ERR_OVERFLOW; }
      } catch (const StateError& e) { throw StateError(where(k, e.what())); }
    }
    const int Kc = sims[0]->win.K, nseg = sims[0]->win.nseg;
    const int t_pp = pick_tpp();
    std::vector<long long> target(ns), cps;
    for (int c = 0; c < nseg; ++c) {
      const int len = std::min(Kc, T - c * Kc);
      for (int k = 0; k < ns; ++k) {
        sims[k]->win_checkpoint(c);
        target[k] = sims[k]->t + len;
      }
      run_chunk(target, len, t_pp, false, true, cps);
      for (int k = 0; k < ns; ++k) {
        try {
          sims[k]->win_segment_done(c, len, h_t[k], h_ctrl[k], cps[k]);
        } catch (const StateError& e) { throw StateError(where(k, e.what())); }
        c_steps += len;
        c_contacts += len * cps[k];
      }
    }
    for (int k = 0; k < ns; ++k) sims[k]->win_finish(R ? R[k] : nullptr);
    return 0;
  }

  int window_adjoint(const double* const* gR, double* const* grad_params, double* const* gvel,
                     double* const* gang) {
    const int ns = (int)sims.size();
    if (!gR) throw std::invalid_argument("null reaction gradients");
    check_form();
    for (int k = 0; k < ns; ++k) {
      sims[k]->window_require();
      if (sims[k]->win.T != sims[0]->win.T || sims[k]->win.K != sims[0]->win.K)
        throw StateError(where(k, "its window differs from the other specimens'"));
    }
    borrow();
    struct Back { Ensemble* e; ~Back() { e->give_back(); } } back{this};
    const int T = sims[0]->win.T, K = sims[0]->win.K, nseg = sims[0]->win.nseg;
    const int t_pp = pick_tpp();
    std::vector<AdjArgs> abase(ns);
    std::vector<WinSpec> spec(ns);
    std::vector<int> ptile(ns + 1, 0), bptile((size_t)ns * kMaxBond + 1, 0), dtile((size_t)ns * kMaxDyn + 1, 0);
    bool bonds = false, pairs = false;
    scan_families();
    std::vector<int> tile_start;
    const int total_btiles = upload_tiles(t_pp, tile_start);  // sizes the wall-partial scratch make_args points to
    for (int k = 0; k < ns; ++k) {
      DemSim& d = *sims[k];
      abase[k] = d.adj_begin(gR[k]);
      spec[k] = d.win_spec();
      h_args[k] = d.make_args(0);  // the recompute's base: live groups, walls, counters
      ptile[k + 1] = ptile[k] + (d.n + 255) / 256;
      for (int b = 0; b < abase[k].nbond; ++b) {
        bptile[(size_t)k * kMaxBond + b + 1] = (abase[k].bond[b].nb + 127) / 128;
        bonds = bonds || abase[k].bond[b].nb > 0;
      }
      for (int g = 0; g < abase[k].ndyn; ++g) {
        dtile[(size_t)k * kMaxDyn + g + 1] = (abase[k].dyn[g].m + 127) / 128;
        pairs = pairs || abase[k].dyn[g].m > 0;
      }
    }
    for (size_t it = 0; it < (size_t)ns * kMaxBond; ++it) bptile[it + 1] += bptile[it];
    for (size_t it = 0; it < (size_t)ns * kMaxDyn; ++it) dtile[it + 1] += dtile[it];
    d_wbase.reserve(ns); d_wtab.reserve((size_t)2 * ns); d_abase.reserve(ns); d_atab.reserve(ns); d_wspec.reserve(ns);
    d_ptile.reserve(ns + 1); d_bptile.reserve((size_t)ns * kMaxBond + 1); d_dtile.reserve((size_t)ns * kMaxDyn + 1);
    DEM_CUDA(cudaMemcpyAsync(d_wbase.p, h_args, sizeof(StepArgs) * ns, cudaMemcpyHostToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(d_abase.p, abase.data(), sizeof(AdjArgs) * ns, cudaMemcpyHostToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(d_wspec.p, spec.data(), sizeof(WinSpec) * ns, cudaMemcpyHostToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(d_ptile.p, ptile.data(), sizeof(int) * ptile.size(), cudaMemcpyHostToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(d_bptile.p, bptile.data(), sizeof(int) * bptile.size(), cudaMemcpyHostToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(d_dtile.p, dtile.data(), sizeof(int) * dtile.size(), cudaMemcpyHostToDevice, s));
    std::vector<int> zeros(ns, 0);
    std::vector<long long> zt(ns, 0), target(ns);
    DEM_CUDA(cudaMemcpyAsync(d_base_cur.p, zeros.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, s));
    DEM_CUDA(cudaMemcpyAsync(d_base_t.p, zt.data(), sizeof(long long) * ns, cudaMemcpyHostToDevice, s));
    BatchArgs B{};
    B.nspec = ns;
    B.total_tiles = tile_start[ns];
    B.args = d_wtab.p;
    B.tile_start = d_tile_start.p;
    B.base_t = d_base_t.p;
    B.base_cur = d_base_cur.p;
    B.target = d_target.p;
    B.btile_start = d_btile_start.p;
    B.total_btiles = total_btiles;
    AdjBatch AB{};
    AB.nspec = ns;
    AB.args = d_atab.p;
    AB.ptile_start = d_ptile.p;
    AB.total_ptiles = ptile[ns];
    AB.btile_start = d_bptile.p;
    AB.total_btiles = bptile[(size_t)ns * kMaxBond];
    AB.dtile_start = d_dtile.p;
    AB.total_dtiles = dtile[(size_t)ns * kMaxDyn];
    AB.pair_duals = abase[0].pair_duals;
    for (int k = 1; k < ns; ++k)
      if (abase[k].pair_duals != AB.pair_duals)
        throw std::invalid_argument("ensemble specimens must share the adjoint_pair_duals option");
    for (int c = nseg - 1; c >= 0; --c) {
      const int len = std::min(K, T - c * K);
      for (int k = 0; k < ns; ++k) {
        sims[k]->adj_restore(c);
        target[k] = sims[k]->win.t0 + (long long)c * K + len;
      }
      DEM_CUDA(cudaMemcpyAsync(d_target.p, target.data(), sizeof(long long) * ns, cudaMemcpyHostToDevice, s));
      for (int j = 0; j < len; ++j) {  // recompute every specimen's segment, one step at a time
        launch_window_step_expand(d_wbase.p, d_wtab.p, d_wspec.p, ns, j, s);
        if (fp32) launch_batch_step_fp32(B, rot != 0, el, fr, bd, gather, t_pp, s);
        else launch_batch_step(B, rot != 0, el, fr, bd, gather, t_pp, s);
      }
      for (int j = len - 1; j >= 0; --j) {  // and reverse it
        launch_window_adj_expand(d_abase.p, d_atab.p, d_wspec.p, ns, c, j, s);
        launch_adjoint_step_batch(AB, bonds, pairs, s);
      }
      DEM_CUDA(cudaGetLastError());
      c_launches += (long long)len * (3 + (gather ? 1 : 0)) + (long long)len * (2 + (bonds ? 1 : 0) + (pairs ? 1 : 0) + ((bonds || pairs) ? 1 : 0));
    }
    for (int k = 0; k < ns; ++k)
      sims[k]->adj_finish(grad_params ? grad_params[k] : nullptr, gvel ? gvel[k] : nullptr,
                          gang ? gang[k] : nullptr, nullptr, nullptr);
    return 0;
  }
};

}  // namespace dem

using dem::DemSim;

namespace {
// Text of this thread's last failed dem_create (there is no handle to keep it in).
thread_local std::string g_create_err;

int create_fail(int rc, const std::string& why) {
  g_create_err = "dem_create: " + why;
  return rc;
}

// The checks of TSubLattice::initNeighborTable and the ParallelParticleArray ctor
// (Parallel/SubLattice.hpp:455-564, ppa/src/pp_array.hpp:72-88) made before any device
// work: the reference throws "size doesn't fit range" where the grown domain is not a
// whole number of cells.  Here the grid is grown the same way (non-periodic sides to
// whole cells, the range of a periodic x side adjusted to divide it), so what remains
// is a domain that is empty, not finite, periodic in y or z, or too small or too large
// for the cell grid.  Returns "" when the domain is usable.
std::string check_domain(double range, double alpha, const double* mn, const double* mx, const int* circ) {
  if (!(range > 0) || !std::isfinite(range)) return "grid spacing must be positive";
  if (!(alpha >= 0) || !std::isfinite(alpha)) return "verlet distance must be non-negative";
  if (!mn || !mx) return "null bounding box";
  for (int i = 0; i < 3; ++i) {
    if (!std::isfinite(mn[i]) || !std::isfinite(mx[i])) return "bounding box is not finite";
    if (!(mx[i] > mn[i])) return "bounding box max must exceed min in every dimension";
  }
  if (circ && (circ[1] || circ[2])) return "only x may be periodic (circDimList y and z must be false)";
  double cells = 1.0;
  for (int i = 0; i < 3; ++i) {
    const double sz = mx[i] - mn[i];
    double n = std::ceil(sz / range);
    if (i == 0 && circ && circ[0]) {
      n = std::floor(sz / range);
      if (std::fabs(sz / range - std::lrint(sz / range)) <= 1e-6) n = (double)std::lrint(sz / range);
      if (n < 3) return "periodic x needs at least 3 cells of the grid spacing";
    } else {
      n += 2;  // the padding layer on both sides
    }
    cells *= n;
  }
  if (!(cells < 2147483647.0)) return "the cell grid has more than 2^31 - 1 cells";
  return "";
}

template <class F>
int guard(dem_sim* h, F&& f) {
  DemSim* s = reinterpret_cast<DemSim*>(h);
  if (!s) return DEM_ERR_ARG;
  (void)cudaGetLastError();  // every runtime call is checked where it is made; drop a reported, non-sticky error
  try {
    return f(*s);
  } catch (const dem::CudaError& e) {
    s->err = e.what();
    return DEM_ERR_CUDA;
  } catch (const std::invalid_argument& e) {
    s->err = e.what();
    return DEM_ERR_ARG;
  } catch (const dem::StateError& e) {
    s->err = e.what();
    return DEM_ERR_STATE;
  } catch (const std::exception& e) {
    s->err = e.what();
    return DEM_ERR_INTERNAL;
  }
}
}  // namespace

// The bonds of a new bonded group from the connections of its tag, p1 the lower id
// (PIS_E::tryInsert, pi_storage_e.hpp:222-263); `set` fills the group's parameters.
template <class F>
static void add_bond_group(DemSim& s, const char* name, int tag, F&& set) {
    if ((int)s.bond.size() >= dem::kMaxBond) throw std::invalid_argument("too many bonded interaction groups");
    std::vector<unsigned> pf(s.n);
    if (s.n) {
      DEM_CUDA(cudaMemcpyAsync(pf.data(), s.P.pflags, sizeof(unsigned) * s.n, cudaMemcpyDeviceToHost, s.s));
      s.sync();
    }
    std::set<std::pair<int, int>> seen;
    std::vector<unsigned long long> keys;
    const std::vector<int>& c = s.temp_conn[tag];
    for (size_t i = 0; i + 1 < c.size(); i += 2) {
      int a = std::min(c[i], c[i + 1]), b = std::max(c[i], c[i + 1]);
      if (!seen.insert({a, b}).second) continue;
      auto ia = s.id2slot.find(a), ib = s.id2slot.find(b);
      if (ia == s.id2slot.end() || ib == s.id2slot.end()) continue;
      if (!(pf[ia->second] & dem::PF_ALIVE) || !(pf[ib->second] & dem::PF_ALIVE)) continue;
      keys.push_back(((unsigned long long)(unsigned)ia->second << 32) | (unsigned)ib->second);
    }
    std::sort(keys.begin(), keys.end());
    dem::BondGroup& B = s.bond[name];
    B.tag = tag;
    set(B);
    B.nb = (int)keys.size();
    const int nb = std::max(B.nb, 1);
    B.keys.reserve(nb); B.ends.reserve(nb); B.D0.reserve(nb); B.broken_step.reserve(nb);
    B.cap_events = s.event_cap(B.nb);
    B.events.reserve(3 * B.cap_events); B.nevents.reserve(1);
    std::vector<int2> ends(B.nb);
    for (int i = 0; i < B.nb; ++i) ends[i] = make_int2((int)(keys[i] >> 32), (int)(keys[i] & 0xffffffffu));
    std::vector<int> alive(B.nb, dem::kBondAlive);
    if (B.nb) {
      DEM_CUDA(cudaMemcpyAsync(B.keys.p, keys.data(), sizeof(unsigned long long) * B.nb, cudaMemcpyHostToDevice, s.s));
      DEM_CUDA(cudaMemcpyAsync(B.ends.p, ends.data(), sizeof(int2) * B.nb, cudaMemcpyHostToDevice, s.s));
      DEM_CUDA(cudaMemcpyAsync(B.broken_step.p, alive.data(), sizeof(int) * B.nb, cudaMemcpyHostToDevice, s.s));
    }
    DEM_CUDA(cudaMemsetAsync(B.nevents.p, 0, sizeof(int), s.s));
    dem::launch_bonds_init(B.nb, B.ends.p, s.P.buf[s.cur].pr, B.D0.p, s.s);
    s.build_adjacency(B.keys, B.nb, B.adj_start, B.adj_count, B.adj_cursor, B.p1_start, B.adj);
    s.sync();
}

extern "C" {

int dem_create(dem_sim** out, int particle_type, double grid_spacing, double verlet_dist, const double* bbox_min,
               const double* bbox_max, const int* circ, double dt) {
  if (!out) return create_fail(DEM_ERR_ARG, "null output handle");
  *out = nullptr;
  // the domain is checked on the host before any device is touched
  if (particle_type != 0 && particle_type != 1) return create_fail(DEM_ERR_ARG, "particle type must be 0 or 1");
  if (!(dt > 0) || !std::isfinite(dt)) return create_fail(DEM_ERR_ARG, "time step must be positive");
  const std::string bad = check_domain(grid_spacing, verlet_dist, bbox_min, bbox_max, circ);
  if (!bad.empty()) return create_fail(DEM_ERR_ARG, bad);
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) return create_fail(DEM_ERR_CUDA, "no usable GPU");
  DemSim* s = nullptr;
  try {
    s = new DemSim();
    s->rot = particle_type ? 1 : 0;
    s->dt = dt; s->nrange = grid_spacing; s->alpha = verlet_dist;
    s->init_grid(bbox_min, bbox_max, circ);
  } catch (const dem::CudaError& e) {
    delete s;
    return create_fail(DEM_ERR_CUDA, e.what());
  } catch (const std::exception& e) {
    delete s;
    return create_fail(DEM_ERR_ARG, e.what());
  }
  g_create_err.clear();
  *out = reinterpret_cast<dem_sim*>(s);
  return DEM_OK;
}

int dem_destroy(dem_sim* h) {
  delete reinterpret_cast<DemSim*>(h);
  return DEM_OK;
}

const char* dem_last_error(dem_sim* h) {
  if (h) return reinterpret_cast<DemSim*>(h)->err.c_str();
  return g_create_err.empty() ? "null handle" : g_create_err.c_str();
}

int dem_add_particles(dem_sim* h, int n, const int* id, const int* tag, const double* pos, const double* rad,
                      const double* mass, const double* vel, const double* angvel, const double* quat,
                      const int* flags) {
  return guard(h, [&](DemSim& s) {
    if (n < 0 || (n && (!id || !pos || !rad || !mass))) throw std::invalid_argument("bad particle arrays");
    return s.add_particles(n, id, tag, pos, rad, mass, vel, angvel, quat, flags);
  });
}

int dem_add_connections(dem_sim* h, int n, const int* tag, const int* id1, const int* id2) {
  return guard(h, [&](DemSim& s) {
    for (int i = 0; i < n; ++i) { s.temp_conn[tag[i]].push_back(id1[i]); s.temp_conn[tag[i]].push_back(id2[i]); }
    s.search_neighbors();  // LatticeMaster.hpp:397
    return DEM_OK;
  });
}

int dem_add_wall(dem_sim* h, const char* name, const double* o, const double* nrm) {
  return guard(h, [&](DemSim& s) {
    s.download_walls();
    dem::Wall w;
    for (int k = 0; k < 3; ++k) { w.o[k] = o[k]; w.n[k] = nrm[k]; w.old[k] = o[k]; }
    s.walls[name] = w;
    s.upload_walls();
    return DEM_OK;
  });
}

int dem_add_elastic_group(dem_sim* h, const char* name, double k, int scaling) {
  return guard(h, [&](DemSim& s) {
    if ((int)s.dyn.size() >= dem::kMaxDyn) throw std::invalid_argument("too many dynamic interaction groups");
    dem::DynGroup& G = s.dyn[name];
    G.kind = 0; G.k = k; G.scaling = scaling != 0;
    s.resize_adjacency();
    return DEM_OK;
  });
}

int dem_add_rot_friction_group(dem_sim* h, const char* name, double k, double mu_s, double mu_d, double ks, double dt,
                               int scaling, int meanR) {
  return guard(h, [&](DemSim& s) {
    if (!s.rot) throw std::invalid_argument("RotFriction needs RotSphere particles");
    if ((int)s.dyn.size() >= dem::kMaxDyn) throw std::invalid_argument("too many dynamic interaction groups");
    dem::DynGroup& G = s.dyn[name];
    G.kind = 1; G.k = k; G.mu_s = mu_s; G.mu_d = mu_d; G.ks = ks; G.dt = dt; G.scaling = scaling != 0;
    G.meanR = meanR != 0;
    s.resize_adjacency();
    return DEM_OK;
  });
}

// TSubLattice::addPairIG, type "Friction" (Parallel/SubLattice.hpp:1055-1076): CFrictionIGP in its
// packing order (k, mu, k_s, dt, scaling).
int dem_add_nrot_friction_group(dem_sim* h, const char* name, double k, double mu, double ks, double dt, int scaling) {
  return guard(h, [&](DemSim& s) {
    if ((int)s.dyn.size() >= dem::kMaxDyn) throw std::invalid_argument("too many dynamic interaction groups");
    if (s.fp32) throw std::invalid_argument("NRotFriction groups run in the FP64 form only");
    dem::DynGroup& G = s.dyn[name];
    G.kind = 2; G.k = k; G.mu_s = mu; G.mu_d = mu; G.ks = ks; G.dt = dt; G.scaling = scaling != 0; G.meanR = 0;
    s.resize_adjacency();
    return DEM_OK;
  });
}

// TSubLattice::addPairIG, type "HertzMindlin" (Parallel/SubLattice.hpp:1324-1339): CHertzMindlinIGP in
// its packing order (E, nu, mu, dt), a PIS_NE storage.
int dem_add_hertz_mindlin_group(dem_sim* h, const char* name, double E, double nu, double mu, double dt) {
  return guard(h, [&](DemSim& s) {
    if ((int)s.dyn.size() >= dem::kMaxDyn) throw std::invalid_argument("too many dynamic interaction groups");
    if (s.fp32) throw std::invalid_argument("HertzMindlin groups run in the FP64 form only");
    if (s.handoff) throw std::invalid_argument("the device bond hand-off needs RotFriction or NRotFriction groups");
    dem::DynGroup& G = s.dyn[name];
    G.kind = 3; G.k = E; G.ks = nu; G.mu_s = mu; G.mu_d = mu; G.dt = dt; G.scaling = 0; G.meanR = 0;
    s.resize_adjacency();
    return DEM_OK;
  });
}

// TRotSubLattice::addRotBondedIG (RotSubLattice.hpp:116-186) with PIS_E::tryInsert (pi_storage_e.hpp:222-263).
int dem_add_rot_bond_group(dem_sim* h, const char* name, int tag, double kr, double ks, double kt, double kb,
                           double mn, double ms, double mt, double mb, int scaling, int meanR, double truncated) {
  return guard(h, [&](DemSim& s) {
    if (!s.rot) throw std::invalid_argument("RotBond needs RotSphere particles");
    add_bond_group(s, name, tag, [&](dem::BondGroup& B) {
      B.kind = 0;
      B.kr = kr; B.ks = ks; B.kt = kt; B.kb = kb; B.mn = mn; B.ms = ms; B.mt = mt; B.mb = mb;
      B.scaling = scaling != 0; B.meanR = meanR != 0; B.truncated = truncated;
    });
    return DEM_OK;
  });
}

// TSubLattice::addPairIG, type "HertzMindlinVisco" (Parallel/SubLattice.hpp:1340-1356): CHertzMindlinViscoIGP
// packing order E, nu, mu, COR, dt; PIS_NE storage like HertzMindlin.
int dem_add_hertz_mindlin_visco_group(dem_sim* h, const char* name, double E, double nu, double mu, double COR,
                                      double dt) {
  return guard(h, [&](DemSim& s) {
    if ((int)s.dyn.size() >= dem::kMaxDyn && !s.dyn.count(name)) throw std::invalid_argument("too many dynamic groups");
    if (s.fp32) throw std::invalid_argument("HertzMindlinVisco groups run in the FP64 form only");
    if (s.handoff) throw std::invalid_argument("the device bond hand-off needs RotFriction or NRotFriction groups");
    dem::DynGroup& G = s.dyn[name];
    G.kind = 4; G.k = E; G.ks = nu; G.mu_s = mu; G.mu_d = COR; G.dt = dt; G.scaling = 0; G.meanR = 0;
    s.resize_adjacency();
    return DEM_OK;
  });
}

// TRotSubLattice::addBrittleBeamDZCIG (Parallel/RotSubLattice.hpp:227-267): BrittleBeamDZCIGP from raw
// stiffnesses, which ARotBondedIGP scales with the bond's half length (scaling on); the failure
// criterion's friction angle is in degrees, its tangent taken as the interaction's constructor does
// (Model/BrittleBeamDZC.cpp:90-103).
int dem_add_brittle_beam_dzc_group(dem_sim* h, const char* name, int tag, double kr, double ks, double kt, double kb,
                                   double cohesion, double tCutoff, double cCutoff, double fAngle, double beta1,
                                   double beta2) {
  return guard(h, [&](DemSim& s) {
    if (!s.rot) throw std::invalid_argument("BrittleBeamDZC needs RotSphere particles");
    add_bond_group(s, name, tag, [&](dem::BondGroup& B) {
      B.kind = 2;
      B.kr = kr; B.ks = ks; B.kt = kt; B.kb = kb;
      B.mn = B.ms = B.mt = B.mb = 1.0;  // no force strengths: the criterion is the beam's
      B.scaling = 1; B.meanR = 1; B.truncated = 1.0;
      B.cohesion = cohesion; B.tan_angle = std::tan(fAngle / 57.2957795); B.t_cutoff = tCutoff;
      B.c_cutoff = cCutoff; B.beta1 = beta1; B.beta2 = beta2;
    });
    return DEM_OK;
  });
}

// TRotSubLattice::addBrittleBeamSCIG (Parallel/RotSubLattice.hpp:188-225): BrittleBeamSCIGP from raw
// stiffnesses (scaled as for BrittleBeamDZC); the failure test reads the particles' stress sums, which
// the step then accumulates (BrittleBeamSCInteraction ctor and broken, Model/BrittleBeamSC.cpp).
int dem_add_brittle_beam_sc_group(dem_sim* h, const char* name, int tag, double kr, double ks, double kt, double kb,
                                  double cohesion, double tCutoff, double fAngle) {
  return guard(h, [&](DemSim& s) {
    if (!s.rot) throw std::invalid_argument("BrittleBeamSC needs RotSphere particles");
    if (s.fp32) throw std::invalid_argument("BrittleBeamSC groups run in the FP64 form only");
    add_bond_group(s, name, tag, [&](dem::BondGroup& B) {
      B.kind = 3;
      B.kr = kr; B.ks = ks; B.kt = kt; B.kb = kb;
      B.mn = B.ms = B.mt = B.mb = 1.0;
      B.scaling = 1; B.meanR = 1; B.truncated = 1.0;
      B.cohesion = cohesion; B.tan_angle = std::tan(fAngle / 57.2957795); B.t_cutoff = tCutoff;
    });
    return DEM_OK;
  });
}

// TSubLattice::addBondedIG (Parallel/SubLattice.hpp:1791-1831): CBondedIGP (tag, k, rbreak, scaling);
// rbreak < 0 makes the group unbreakable.
int dem_add_nrot_bond_group(dem_sim* h, const char* name, int tag, double k, double rbreak, int scaling) {
  return guard(h, [&](DemSim& s) {
    add_bond_group(s, name, tag, [&](dem::BondGroup& B) {
      B.kind = 1;
      B.knb = k; B.rbreak = rbreak; B.scaling = scaling != 0; B.meanR = 0;
      B.kr = B.ks = B.kt = B.kb = B.mn = B.ms = B.mt = B.mb = 0.0; B.truncated = 1.0;
    });
    return DEM_OK;
  });
}

int dem_add_wall_group(dem_sim* h, const char* name, const char* wall, double k) {
  return guard(h, [&](DemSim& s) {
    if (!s.walls.count(wall)) throw std::invalid_argument(std::string("wall name '") + wall + "' not found in map of walls");
    if (!s.wig.count(name) && (int)s.wig.size() >= dem::kMaxWalls) throw std::invalid_argument("too many wall groups");
    s.download_walls();
    s.wig[name] = dem::WallGroup{wall, k};
    s.upload_walls();
    DEM_CUDA(cudaMemsetAsync(s.scalars.p + 2, 0, sizeof(int), s.s));
    dem::launch_wall_update(s.g, s.P, s.cur, (int)s.wig.size(), s.d_walls.p, s.scalars.p + 2, s.s);  // CEWallInteractionGroup::Update
    s.wall_cand = s.read_int(s.scalars.p + 2);
    s.sync();
    return DEM_OK;
  });
}

int dem_add_gravity(dem_sim* h, const char* name, const double* gv) {
  return guard(h, [&](DemSim& s) {
    if (!s.grav.count(name) && (int)s.grav.size() >= dem::kMaxGrav) throw std::invalid_argument("too many body forces");
    s.grav[name] = {gv[0], gv[1], gv[2]};
    return DEM_OK;
  });
}

int dem_add_damping(dem_sim* h, int rot, double visc, int max_iter) {
  return guard(h, [&](DemSim& s) {
    if (rot) {
      if (!s.rot) throw std::invalid_argument("RotDamping needs RotSphere particles");
      s.damp_rot = 1; s.visc_rot = visc; s.iter_rot = max_iter;
    } else {
      s.damp_lin = 1; s.visc_lin = visc; s.iter_lin = max_iter;
    }
    return DEM_OK;
  });
}

// TSubLattice::doAddDamping "LocalDamping" (Parallel/SubLattice.hpp:1765-1769) and
// TRotSubLattice::doAddDamping "RotLocalDamping" (Parallel/RotSubLattice.hpp:95-104).
int dem_add_local_damping(dem_sim* h, const char* name, int rot, double visc) {
  return guard(h, [&](DemSim& s) {
    if (rot) {
      if (!s.rot) throw std::invalid_argument("RotLocalDamping needs RotSphere particles");
      s.damp_rotloc = 1; s.visc_rotloc = visc;
    } else {
      const std::string n = name ? name : "";
      if (n.empty() || n == "Damping" || n == "RotDamping" || n == "RotLocalDamping")
        throw std::invalid_argument("a LocalDamping group needs a name of its own");
      s.loc_name = n; s.visc_loc = visc;
    }
    return DEM_OK;
  });
}

// TSubLattice::setExIG (SubLattice.hpp:1980-2009) + PIS_ED::addExIG (pi_storage_ed.hpp:20-40).
int dem_add_exclusion(dem_sim* h, const char* bonded, const char* dynamic) {
  return guard(h, [&](DemSim& s) {
    auto dy = s.dyn.find(dynamic);
    if (dy == s.dyn.end() || !s.bond.count(bonded))
      throw std::invalid_argument("nonexisting interaction group");
    dem::DynGroup& G = dy->second;
    G.excl.push_back(bonded);
    if (G.m > 0 && s.handoff) {  // the hand-off keeps excluded pairs in the list, marked
      s.mark_handoff(G);
      s.sync();
    } else if (G.m > 0) {  // clean out pairs that are now excluded, keeping the others' history
      dem::BondGroup& B = s.bond[bonded];
      std::vector<unsigned long long> keys(G.m), bk(B.nb);
      std::vector<double4> hist(G.kind != 0 ? G.m : 0);
      std::vector<int> bs(B.nb);
      DEM_CUDA(cudaMemcpyAsync(keys.data(), G.keys.p, sizeof(unsigned long long) * G.m, cudaMemcpyDeviceToHost, s.s));
      if (G.kind != 0) DEM_CUDA(cudaMemcpyAsync(hist.data(), G.hist[s.cur].p, sizeof(double4) * G.m, cudaMemcpyDeviceToHost, s.s));
      if (B.nb) {
        DEM_CUDA(cudaMemcpyAsync(bk.data(), B.keys.p, sizeof(unsigned long long) * B.nb, cudaMemcpyDeviceToHost, s.s));
        DEM_CUDA(cudaMemcpyAsync(bs.data(), B.broken_step.p, sizeof(int) * B.nb, cudaMemcpyDeviceToHost, s.s));
      }
      s.sync();
      std::vector<unsigned long long> k2;
      std::vector<double4> h2;
      for (int i = 0; i < G.m; ++i) {
        auto p = std::lower_bound(bk.begin(), bk.end(), keys[i]);
        bool ex = p != bk.end() && *p == keys[i] && bs[p - bk.begin()] == dem::kBondAlive;
        if (!ex) { k2.push_back(keys[i]); if (G.kind != 0) h2.push_back(hist[i]); }
      }
      G.m = (int)k2.size();
      if (G.m) {
        DEM_CUDA(cudaMemcpyAsync(G.keys.p, k2.data(), sizeof(unsigned long long) * G.m, cudaMemcpyHostToDevice, s.s));
        if (G.kind != 0) DEM_CUDA(cudaMemcpyAsync(G.hist[s.cur].p, h2.data(), sizeof(double4) * G.m, cudaMemcpyHostToDevice, s.s));
      }
      s.build_adjacency(G.keys, G.m, G.adj_start, G.adj_count, G.adj_cursor, G.p1_start, G.adj);
      s.sync();
    }
    return DEM_OK;
  });
}

int dem_set_timestep(dem_sim* h, double dt) {
  return guard(h, [&](DemSim& s) {
    if (!(dt > 0)) throw std::invalid_argument("time step must be positive");
    s.dt = dt;  // TSubLattice::setTimeStepSize (SubLattice.hpp:2163-2204) propagates to the groups
    for (auto& d : s.dyn) d.second.dt = dt;
    return DEM_OK;
  });
}

int dem_step(dem_sim* h, int nsteps) {
  return guard(h, [&](DemSim& s) {
    if (nsteps < 0) throw std::invalid_argument("negative step count");
    return s.step(nsteps);
  });
}

int dem_move_wall(dem_sim* h, const char* name, const double* d) {
  return guard(h, [&](DemSim& s) {
    if (!s.walls.count(name)) throw std::invalid_argument("no such wall");
    s.download_walls();
    dem::Wall& W = s.walls[name];
    for (int k = 0; k < 3; ++k) W.o[k] += d[k];  // CWall::moveBy (Model/Wall.h:53-60)
    s.upload_walls();
    return DEM_OK;
  });
}

int dem_set_wall_velocity(dem_sim* h, const char* name, const double* v) {
  return guard(h, [&](DemSim& s) {
    if (!s.walls.count(name)) throw std::invalid_argument("no such wall");
    s.download_walls();
    s.wall_loader[name] = {v[0], v[1], v[2]};
    s.upload_walls();
    return DEM_OK;
  });
}

int dem_apply_force_to_wall(dem_sim* h, const char* group, const double* f) {
  return guard(h, [&](DemSim& s) {
    auto it = s.wig.find(group);
    if (it == s.wig.end()) throw std::invalid_argument("no such wall group");
    int w = (int)std::distance(s.wig.begin(), it);
    s.d_servo_idx.reserve(std::max(s.n, 1));
    dem::launch_wall_servo(s.P, s.cur, w, s.d_walls.p, f, s.d_servo_idx.p, s.s);
    // the servo moves the group's copy of the wall: propagate to groups sharing the wall (the
    // read follows the servo on the stream, so one wait covers both)
    std::vector<dem::WallDev> wd(s.wig.size());
    DEM_CUDA(cudaMemcpyAsync(wd.data(), s.d_walls.p, sizeof(dem::WallDev) * wd.size(), cudaMemcpyDeviceToHost, s.s));
    s.sync();
    dem::Wall& W = s.walls.at(it->second.wall);
    W.o[0] = wd[w].ox; W.o[1] = wd[w].oy; W.o[2] = wd[w].oz;
    s.upload_walls();
    return DEM_OK;
  });
}

int dem_get_wall(dem_sim* h, const char* name, double* pos, double* force) {
  return guard(h, [&](DemSim& s) {
    if (!s.walls.count(name)) throw std::invalid_argument("no such wall");
    s.download_walls();
    double wf[dem::kMaxWalls * 3];
    DEM_CUDA(cudaMemcpyAsync(wf, s.d_wall_force.p, sizeof(wf), cudaMemcpyDeviceToHost, s.s));
    s.sync();
    double F[3] = {0, 0, 0};
    int k = 0;
    for (auto& it : s.wig) {
      if (it.second.wall == name) for (int c = 0; c < 3; ++c) F[c] += wf[3 * k + c];
      ++k;
    }
    for (int c = 0; c < 3; ++c) { if (pos) pos[c] = s.walls[name].o[c]; if (force) force[c] = F[c]; }
    return DEM_OK;
  });
}

int dem_num_particles(dem_sim* h) {
  return guard(h, [&](DemSim& s) {
    std::vector<unsigned> pf(s.n);
    if (s.n) DEM_CUDA(cudaMemcpyAsync(pf.data(), s.P.pflags, sizeof(unsigned) * s.n, cudaMemcpyDeviceToHost, s.s));
    s.sync();
    int c = 0;
    for (unsigned f : pf) c += (f & dem::PF_ALIVE) ? 1 : 0;
    return c;
  });
}

int dem_get_particles(dem_sim* h, int* id, double* pos, double* vel, double* angvel, double* quat, double* force,
                      double* moment) {
  return guard(h, [&](DemSim& s) { return s.get_particles(id, pos, vel, angvel, quat, force, moment); });
}

int dem_num_pairs(dem_sim* h, const char* group) {
  return guard(h, [&](DemSim& s) {
    auto d = s.dyn.find(group);
    if (d != s.dyn.end()) return d->second.m;
    auto b = s.bond.find(group);
    if (b == s.bond.end()) throw std::invalid_argument("no such group");
    std::vector<int> bs(b->second.nb);
    if (b->second.nb) DEM_CUDA(cudaMemcpyAsync(bs.data(), b->second.broken_step.p, sizeof(int) * bs.size(), cudaMemcpyDeviceToHost, s.s));
    s.sync();
    int c = 0;
    for (int v : bs) c += v > s.t ? 1 : 0;
    return c;
  });
}

int dem_set_pair_states(dem_sim* h, const char* group, int n, const int* id1, const int* id2, const double* state) {
  return guard(h, [&](DemSim& s) {
    auto d = s.dyn.find(group);
    if (d == s.dyn.end()) throw std::invalid_argument("no such dynamic group");
    dem::DynGroup& G = d->second;
    if (n < 0 || (n && (!id1 || !id2 || !state))) throw std::invalid_argument("null pair arrays");
    if (G.kind == 0 || !G.m || !n) return 0;  // the elastic law keeps no history
    std::vector<unsigned long long> keys(G.m);
    DEM_CUDA(cudaMemcpyAsync(keys.data(), G.keys.p, sizeof(unsigned long long) * G.m, cudaMemcpyDeviceToHost, s.s));
    s.sync();
    int done = 0;
    for (int r = 0; r < n; ++r) {
      auto ia = s.id2slot.find(std::min(id1[r], id2[r])), ib = s.id2slot.find(std::max(id1[r], id2[r]));
      if (ia == s.id2slot.end() || ib == s.id2slot.end()) continue;
      const unsigned long long key = ((unsigned long long)(unsigned)ia->second << 32) | (unsigned)ib->second;
      auto it = std::lower_bound(keys.begin(), keys.end(), key);
      if (it == keys.end() || *it != key) continue;
      const size_t q = (size_t)(it - keys.begin());
      const double* st = state + 5 * (size_t)r;
      const double w = (st[3] != 0.0 ? 1.0 : 0.0) + (st[4] != 0.0 ? 2.0 : 0.0);
      if (s.fp32) {
        const float4 v = make_float4((float)st[0], (float)st[1], (float)st[2], (float)w);
        DEM_CUDA(cudaMemcpyAsync(G.hist32[s.cur].p + q, &v, sizeof(float4), cudaMemcpyHostToDevice, s.s));
        s.sync();
      } else {
        const double4 v = make_double4(st[0], st[1], st[2], w);
        DEM_CUDA(cudaMemcpyAsync(G.hist[s.cur].p + q, &v, sizeof(double4), cudaMemcpyHostToDevice, s.s));
        s.sync();
      }
      ++done;
    }
    return done;
  });
}

int dem_get_pairs(dem_sim* h, const char* group, int* id1, int* id2, double* state) {
  return guard(h, [&](DemSim& s) {
    auto d = s.dyn.find(group);
    if (d != s.dyn.end()) {
      dem::DynGroup& G = d->second;
      std::vector<unsigned long long> keys(G.m);
      std::vector<int> xb(s.handoff ? G.m : 0);
      std::vector<std::vector<int>> bsteps;
      if (s.handoff) {
        if (G.m) DEM_CUDA(cudaMemcpyAsync(xb.data(), G.xbond.p, sizeof(int) * G.m, cudaMemcpyDeviceToHost, s.s));
        for (auto& b : s.bond) {
          bsteps.emplace_back(b.second.nb);
          if (b.second.nb)
            DEM_CUDA(cudaMemcpyAsync(bsteps.back().data(), b.second.broken_step.p, sizeof(int) * b.second.nb,
                                     cudaMemcpyDeviceToHost, s.s));
        }
      }
      std::vector<double4> hist(G.kind != 0 ? G.m : 0);
      std::vector<float4> hist32(G.kind != 0 && s.fp32 ? G.m : 0);
      if (G.m) DEM_CUDA(cudaMemcpyAsync(keys.data(), G.keys.p, sizeof(unsigned long long) * G.m, cudaMemcpyDeviceToHost, s.s));
      if (G.kind != 0 && G.m) {
        if (s.fp32) DEM_CUDA(cudaMemcpyAsync(hist32.data(), G.hist32[s.cur].p, sizeof(float4) * G.m, cudaMemcpyDeviceToHost, s.s));
        else DEM_CUDA(cudaMemcpyAsync(hist.data(), G.hist[s.cur].p, sizeof(double4) * G.m, cudaMemcpyDeviceToHost, s.s));
      }
      s.sync();
      for (size_t q = 0; q < hist32.size(); ++q) hist[q] = make_double4(hist32[q].x, hist32[q].y, hist32[q].z, hist32[q].w);
      int o = 0;
      for (int i = 0; i < G.m; ++i) {
        // device hand-off: a pair whose excluding bond still holds is not in the reference's list
        if (s.handoff && xb[i] >= 0 && bsteps[xb[i] >> 28][xb[i] & 0x0fffffff] > s.t) continue;
        id1[o] = s.h_id[(int)(keys[i] >> 32)];
        id2[o] = s.h_id[(int)(keys[i] & 0xffffffffu)];
        if (state) {
          for (int c = 0; c < 5; ++c) state[5 * o + c] = 0.0;
          if (G.kind != 0) {
            const int fl = (int)hist[i].w;
            const bool touching = (fl & 2) != 0;
            if (touching) { state[5 * o] = hist[i].x; state[5 * o + 1] = hist[i].y; state[5 * o + 2] = hist[i].z; }
            state[5 * o + 3] = (fl & 1) ? 1.0 : 0.0;
            state[5 * o + 4] = touching ? 1.0 : 0.0;
          }
        }
        ++o;
      }
      return o;
    }
    auto b = s.bond.find(group);
    if (b == s.bond.end()) throw std::invalid_argument("no such group");
    dem::BondGroup& B = b->second;
    std::vector<int2> ends(B.nb);
    std::vector<int> bs(B.nb);
    if (B.nb) {
      DEM_CUDA(cudaMemcpyAsync(ends.data(), B.ends.p, sizeof(int2) * B.nb, cudaMemcpyDeviceToHost, s.s));
      DEM_CUDA(cudaMemcpyAsync(bs.data(), B.broken_step.p, sizeof(int) * B.nb, cudaMemcpyDeviceToHost, s.s));
    }
    s.sync();
    int k = 0;
    for (int i = 0; i < B.nb; ++i) {
      if (bs[i] <= s.t) continue;
      id1[k] = s.h_id[ends[i].x];
      id2[k] = s.h_id[ends[i].y];
      if (state) for (int c = 0; c < 5; ++c) state[5 * k + c] = 0.0;
      ++k;
    }
    return k;
  });
}

int dem_num_breaks(dem_sim* h) {
  return guard(h, [&](DemSim& s) {
    int tot = 0;
    for (auto& b : s.bond) tot += std::min(s.read_int(b.second.nevents.p), b.second.cap_events);
    return tot;
  });
}

int dem_get_breaks(dem_sim* h, int* id1, int* id2, int* step) {
  return guard(h, [&](DemSim& s) {
    int k = 0;
    for (auto& b : s.bond) {
      int ne = std::min(s.read_int(b.second.nevents.p), b.second.cap_events);
      std::vector<int> ev(3 * (size_t)ne);
      if (ne) DEM_CUDA(cudaMemcpyAsync(ev.data(), b.second.events.p, sizeof(int) * ev.size(), cudaMemcpyDeviceToHost, s.s));
      s.sync();
      for (int i = 0; i < ne; ++i) { id1[k] = ev[3 * i]; id2[k] = ev[3 * i + 1]; step[k] = ev[3 * i + 2]; ++k; }
    }
    return k;
  });
}

int dem_move_tagged(dem_sim* h, int tag, int mask, const double* d) {
  (void)mask;
  return guard(h, [&](DemSim& s) {
    dem::launch_move_tagged(s.P, s.cur, tag, d, s.s);
    // a host-side move is checked like any displacement (checkNeighbors runs after pre-runnables)
    dem::launch_check_disp(s.P, s.cur, (0.5 * s.alpha) * (0.5 * s.alpha), s.d_ctrl.p, s.s);
    s.pending_ctrl |= s.read_int(s.d_ctrl.p);
    return DEM_OK;
  });
}

long long dem_timestep(dem_sim* h) { return h ? reinterpret_cast<DemSim*>(h)->t : -1; }

int dem_set_stream(dem_sim* h, void* stream) {
  return guard(h, [&](DemSim& s) {
    s.sync();
    if (s.own_stream) DEM_CUDA(cudaStreamDestroy(s.s));
    s.s = reinterpret_cast<cudaStream_t>(stream);
    s.own_stream = false;
    return DEM_OK;
  });
}

int dem_get_counters(dem_sim* h, long long* out, int n) {
  return guard(h, [&](DemSim& s) {
    const long long search_due = (s.first || (s.pending_ctrl & dem::CTRL_REBUILD)) ? 1 : 0;
    long long v[9] = {s.c_steps, s.c_contacts, s.c_rebuilds, s.c_launches,
                      (long long)(s.prof_ms * 1e6), s.prof_steps, s.contacts_per_step(), (long long)s.pick_tpp(),
                      search_due};
    for (int i = 0; i < n && i < 9; ++i) out[i] = v[i];
    return std::min(n, 9);
  });
}

int dem_set_particles(dem_sim* h, int n, const int* id, const double* pos, const double* vel, const double* angvel,
                      const double* quat) {
  return guard(h, [&](DemSim& s) { return s.set_particles(n, id, pos, vel, angvel, quat); });
}

int dem_revive_particles(dem_sim* h, int n, const int* id, const double* pos, const double* vel, const double* angvel,
                         const double* quat) {
  return guard(h, [&](DemSim& s) { return s.revive_particles(n, id, pos, vel, angvel, quat); });
}

int dem_precision_check(dem_sim* h, double* out) {
  return guard(h, [&](DemSim& s) {
    if (!out) throw std::invalid_argument("null output");
    double v[7];
    s.precision_check(v);
    for (int k = 0; k < 5; ++k) out[k] = v[k];
    return DEM_OK;
  });
}

int dem_precision_report(dem_sim* h, double* out, int n) {
  return guard(h, [&](DemSim& s) {
    if (!out || n < 0) throw std::invalid_argument("null output");
    double v[7];
    s.precision_check(v);
    for (int k = 0; k < n && k < 7; ++k) out[k] = v[k];
    return std::min(n, 7);
  });
}

int dem_set_option(dem_sim* h, const char* key, double value) {
  return guard(h, [&](DemSim& s) {
    std::string k = key ? key : "";
    if (k == "threads_per_particle") {
      int v = (int)value;
      if (v != 0 && v != 1 && v != 2 && v != 4 && v != 8 && v != dem::kTiled && v != dem::kWarpCoop)
        throw std::invalid_argument("threads_per_particle must be 0,1,2,4,8, 16 (tiled) or 32 (warp-cooperative)");
      s.tpp = v;
    } else if (k == "chunk") {
      if (value < 1) throw std::invalid_argument("chunk must be >= 1");
      s.chunk = (int)value;
    } else if (k == "store_forces") {
      s.store_forces = value != 0;
    } else if (k == "split") {
      if (value != -1 && value != 0 && value != 1) throw std::invalid_argument("split must be -1, 0 or 1");
      s.split = (int)value;
    } else if (k == "profile") {
      s.profile = value != 0;
    } else if (k == "bond_handoff") {
      s.set_handoff(value != 0);
    } else if (k == "bond_pass") {
      s.bond_pass = value != 0;
    } else if (k == "adjoint_bond_tangents") {
      const int v = (int)value;
      if (v != 0 && v != 3 && v != 6 && v != 9 && v != 18)
        throw std::invalid_argument("adjoint_bond_tangents must be 0 (hand-written reverse), 3, 6, 9 or 18");
      s.adj_tangents = v;
    } else if (k == "adjoint_pair_duals") {
      s.adj_pair_duals = value != 0;
    } else if (k == "event_capacity") {
      if (!(value >= 0 && value <= 1 << 30) || value != std::floor(value))
        throw std::invalid_argument("event_capacity must be a whole number in [0, 2^30] (0 = one entry per bond)");
      s.set_event_capacity((int)value);
    } else if (k == "precision") {
      if (value != 32 && value != 64) throw std::invalid_argument("precision must be 64 or 32");
      s.set_precision(value == 32);
    } else {
      throw std::invalid_argument("unknown option " + k);
    }
    return DEM_OK;
  });
}

int dem_particle_scalar_field(dem_sim* h, const char* field, double* values) {
  return guard(h, [&](DemSim& s) {
    static const char* names[] = {"e_kin", "e_kin_linear", "e_kin_rot", "v_abs", "radius", "id", "tag", "mass"};
    const std::string f = field ? field : "";
    int code = -1;
    for (int k = 0; k < 8; ++k)
      if (f == names[k]) code = k;
    if (code < 0) throw std::invalid_argument("unknown particle scalar field " + f);
    if (!values) throw std::invalid_argument("null output");
    const int n = s.n;
    s.scratch_d.reserve(std::max(n, 1));
    launch_particle_field(s.P, s.cur, s.rot, code, s.scratch_d.p, s.s);
    std::vector<double> v(n);
    std::vector<unsigned> pf(n);
    if (n) {
      DEM_CUDA(cudaMemcpyAsync(v.data(), s.scratch_d.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s.s));
      DEM_CUDA(cudaMemcpyAsync(pf.data(), s.P.pflags, sizeof(unsigned) * n, cudaMemcpyDeviceToHost, s.s));
    }
    s.sync();
    int k = 0;
    for (int i = 0; i < n; ++i)
      if (pf[i] & dem::PF_ALIVE) values[k++] = v[i];
    return k;
  });
}

int dem_particle_vector_field(dem_sim* h, const char* field, double* values) {
  return guard(h, [&](DemSim& s) {
    static const char* names[] = {"position", "velocity", "force", "ang_velocity", "displacement"};
    const std::string f = field ? field : "";
    int code = -1;
    for (int k = 0; k < 5; ++k)
      if (f == names[k]) code = k;
    if (code < 0 || (code == 3 && !s.rot)) throw std::invalid_argument("unknown particle vector field " + f);
    if (!values) throw std::invalid_argument("null output");
    const int n = s.n;
    s.scratch_d.reserve(std::max(6 * n, 1));
    if (code == 4 && n)
      DEM_CUDA(cudaMemcpyAsync(s.scratch_d.p + 3 * (size_t)n, s.h_initpos.data(), sizeof(double) * 3 * n,
                               cudaMemcpyHostToDevice, s.s));
    launch_particle_vector_field(s.P, s.cur, code, s.scratch_d.p + 3 * (size_t)n, s.scratch_d.p, s.s);
    std::vector<double> v(3 * (size_t)n);
    std::vector<unsigned> pf(n);
    if (n) {
      DEM_CUDA(cudaMemcpyAsync(v.data(), s.scratch_d.p, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s.s));
      DEM_CUDA(cudaMemcpyAsync(pf.data(), s.P.pflags, sizeof(unsigned) * n, cudaMemcpyDeviceToHost, s.s));
    }
    s.sync();
    int k = 0;
    for (int i = 0; i < n; ++i)
      if (pf[i] & dem::PF_ALIVE) {
        for (int c = 0; c < 3; ++c) values[3 * k + c] = v[3 * (size_t)i + c];
        ++k;
      }
    return k;
  });
}

int dem_interaction_scalar_field(dem_sim* h, const char* group, const char* field, double* values) {
  return guard(h, [&](DemSim& s) {
    const std::string gname = group ? group : "", f = field ? field : "";
    if (!values) throw std::invalid_argument("null output");
    const int prev = s.cur ^ 1;  // the particle buffer the last force evaluation read
    auto d = s.dyn.find(gname);
    if (d != s.dyn.end()) {
      dem::DynGroup& G = d->second;
      int code = f == "count" ? 0 : f == "potential_energy" ? 1 : -1;
      if (G.kind != 0 && f == "slipping") code = 2;
      if (G.kind != 0 && f == "sticking") code = 3;
      if (code < 0) throw std::invalid_argument("unknown interaction scalar field " + f + " of group " + gname);
      std::vector<double> v(G.m, 0.0);
      if (s.t > 0 && G.m) {
        s.scratch_d.reserve(G.m);
        launch_pair_field(s.g, s.P, prev, G.keys.p, G.m, G.kind, G.k, G.ks, G.scaling, G.meanR,
                          G.kind != 0 && !s.fp32 ? G.hist[s.cur].p : nullptr,
                          G.kind != 0 && s.fp32 ? G.hist32[s.cur].p : nullptr, code, s.scratch_d.p, s.s);
        DEM_CUDA(cudaMemcpyAsync(v.data(), s.scratch_d.p, sizeof(double) * G.m, cudaMemcpyDeviceToHost, s.s));
      }
      // the pairs dem_get_pairs reports (the device hand-off keeps bond-held pairs it does not report)
      std::vector<int> xb(s.handoff ? G.m : 0);
      std::vector<std::vector<int>> bsteps;
      if (s.handoff) {
        if (G.m) DEM_CUDA(cudaMemcpyAsync(xb.data(), G.xbond.p, sizeof(int) * G.m, cudaMemcpyDeviceToHost, s.s));
        for (auto& b : s.bond) {
          bsteps.emplace_back(b.second.nb);
          if (b.second.nb)
            DEM_CUDA(cudaMemcpyAsync(bsteps.back().data(), b.second.broken_step.p, sizeof(int) * b.second.nb,
                                     cudaMemcpyDeviceToHost, s.s));
        }
      }
      s.sync();
      int k = 0;
      for (int q = 0; q < G.m; ++q) {
        if (s.handoff && xb[q] >= 0 && bsteps[xb[q] >> 28][xb[q] & 0x0fffffff] > s.t) continue;
        values[k++] = v[q];
      }
      return k;
    }
    auto b = s.bond.find(gname);
    if (b == s.bond.end()) throw std::invalid_argument("no such group " + gname);
    if (b->second.kind == 1) throw std::invalid_argument("interaction fields of NRotBond groups are not built");
    if (b->second.kind >= 2 && f == "breaking_criterion")
      throw std::invalid_argument("BrittleBeam groups have no breaking_criterion field");
    static const char* names[] = {"count", "potential_energy", "e_pot_normal", "e_pot_shear", "e_pot_twist",
                                  "e_pot_bend", "breaking_criterion"};
    int code = -1;
    for (int k = 0; k < 7; ++k)
      if (f == names[k]) code = k;
    if (code < 0) throw std::invalid_argument("unknown RotBond scalar field " + f);
    dem::BondGroup& B = b->second;
    std::vector<double> v(B.nb, 0.0);
    std::vector<int> bs(B.nb);
    if (B.nb) {
      DEM_CUDA(cudaMemcpyAsync(bs.data(), B.broken_step.p, sizeof(int) * B.nb, cudaMemcpyDeviceToHost, s.s));
      if (s.t > 0 || code == 0) {
        s.scratch_d.reserve(B.nb);
        const dem::StepArgs a = s.make_args(s.cur);
        int gi = 0;
        for (auto& it : s.bond) {
          if (it.first == gname) break;
          ++gi;
        }
        launch_bond_field(s.g, s.P, prev, s.t, a.bond[gi], B.nb, code, s.scratch_d.p, s.s);
        DEM_CUDA(cudaMemcpyAsync(v.data(), s.scratch_d.p, sizeof(double) * B.nb, cudaMemcpyDeviceToHost, s.s));
      }
    }
    s.sync();
    int k = 0;
    for (int i = 0; i < B.nb; ++i)
      if (bs[i] > s.t) values[k++] = v[i];
    return k;
  });
}

int dem_set_group_param(dem_sim* h, const char* group, const char* key, double value) {
  return guard(h, [&](DemSim& s) {
    if (!group || !key) throw std::invalid_argument("null group or key");
    s.set_group_param(group, key, value);
    return DEM_OK;
  });
}

int dem_window_num_params(dem_sim* h) {
  return guard(h, [&](DemSim& s) { return s.window_num_params(); });
}

int dem_window_forward(dem_sim* h, int nsteps, int checkpoint_every, double* reactions) {
  return guard(h, [&](DemSim& s) { return s.window_forward(nsteps, checkpoint_every, reactions); });
}

int dem_window_adjoint(dem_sim* h, const double* grad_reactions, double* grad_params, double* grad_vel,
                       double* grad_angvel, double* grad_pos, double* grad_quat) {
  return guard(h, [&](DemSim& s) {
    s.window_adjoint(grad_reactions, grad_params, grad_vel, grad_angvel, grad_pos, grad_quat);
    return DEM_OK;
  });
}

int dem_window_rewind(dem_sim* h) {
  return guard(h, [&](DemSim& s) {
    s.window_rewind();
    return DEM_OK;
  });
}

int dem_save_checkpoint(dem_sim* h, const char* path, int precision) {
  return guard(h, [&](DemSim& s) {
    if (!path) throw std::invalid_argument("null path");
    std::ofstream os(path);
    if (!os) throw std::invalid_argument(std::string("cannot open ") + path + " for writing");
    os.precision(precision > 0 ? precision : 12);  // CheckPointer::saveRestartable (Parallel/CheckPointer.cpp:48-66)
    s.save_checkpoint(os);
    os.close();
    if (!os) throw std::runtime_error(std::string("writing ") + path + " failed");
    return DEM_OK;
  });
}

int dem_save_snapshot(dem_sim* h, const char* path) {
  return guard(h, [&](DemSim& s) {
    if (!path) throw std::invalid_argument("null path");
    std::ofstream os(path);
    if (!os) throw std::invalid_argument(std::string("cannot open ") + path + " for writing");
    s.save_snapshot(os);
    os.close();
    if (!os) throw std::runtime_error(std::string("writing ") + path + " failed");
    return DEM_OK;
  });
}

int dem_load_checkpoint(dem_sim* h, const char* path, long long timestep) {
  return guard(h, [&](DemSim& s) {
    if (!path) throw std::invalid_argument("null path");
    std::ifstream is(path);
    if (!is) throw std::invalid_argument(std::string("cannot open ") + path);
    s.load_checkpoint(is, timestep);
    return DEM_OK;
  });
}

int dem_window_release(dem_sim* h) {
  return guard(h, [&](DemSim& s) {
    s.sync();
    s.win.release();
    return DEM_OK;
  });
}

int dem_search_neighbors(dem_sim* h) {
  return guard(h, [&](DemSim& s) {
    s.pending_ctrl |= dem::CTRL_REBUILD;
    return DEM_OK;
  });
}

int dem_ensemble_create(dem_ensemble** out, dem_sim* const* sims, int n) {
  if (!out) return DEM_ERR_ARG;
  *out = nullptr;
  try {
    std::vector<DemSim*> v;
    for (int k = 0; k < n; ++k) v.push_back(reinterpret_cast<DemSim*>(sims ? sims[k] : nullptr));
    *out = reinterpret_cast<dem_ensemble*>(new dem::Ensemble(v.data(), n));
    return DEM_OK;
  } catch (const dem::CudaError&) {
    return DEM_ERR_CUDA;
  } catch (const std::invalid_argument&) {
    return DEM_ERR_ARG;
  } catch (const std::exception&) {
    return DEM_ERR_INTERNAL;
  }
}

int dem_ensemble_destroy(dem_ensemble* e) {
  delete reinterpret_cast<dem::Ensemble*>(e);
  return DEM_OK;
}

const char* dem_ensemble_last_error(dem_ensemble* e) {
  return e ? reinterpret_cast<dem::Ensemble*>(e)->err.c_str() : "null ensemble";
}

}  // extern "C"

namespace {
template <class F>
int eguard(dem_ensemble* h, F&& f) {
  dem::Ensemble* e = reinterpret_cast<dem::Ensemble*>(h);
  if (!e) return DEM_ERR_ARG;
  try {
    cudaGetLastError();
    return f(*e);
  } catch (const dem::CudaError& x) {
    e->err = x.what();
    return DEM_ERR_CUDA;
  } catch (const std::invalid_argument& x) {
    e->err = x.what();
    return DEM_ERR_ARG;
  } catch (const dem::StateError& x) {
    e->err = x.what();
    return DEM_ERR_STATE;
  } catch (const std::exception& x) {
    e->err = x.what();
    return DEM_ERR_INTERNAL;
  }
}
}  // namespace

extern "C" {

int dem_ensemble_step(dem_ensemble* h, int nsteps) {
  return eguard(h, [&](dem::Ensemble& e) { return e.step(nsteps); });
}

int dem_ensemble_window_forward(dem_ensemble* h, int nsteps, int checkpoint_every, double* const* reactions) {
  return eguard(h, [&](dem::Ensemble& e) { return e.window_forward(nsteps, checkpoint_every, reactions); });
}

int dem_ensemble_window_adjoint(dem_ensemble* h, const double* const* grad_reactions, double* const* grad_params,
                                double* const* grad_vel, double* const* grad_angvel) {
  return eguard(h, [&](dem::Ensemble& e) { return e.window_adjoint(grad_reactions, grad_params, grad_vel, grad_angvel); });
}

int dem_ensemble_set_option(dem_ensemble* h, const char* key, double value) {
  return eguard(h, [&](dem::Ensemble& e) {
    const std::string k = key ? key : "";
    if (k == "threads_per_particle") {
      const int v = (int)value;
      if (v != 0 && v != 1 && v != 2 && v != 4 && v != 8 && v != dem::kTiled)
        throw std::invalid_argument("threads_per_particle must be 0,1,2,4,8 or 16 (tiled)");
      e.tpp = v;
    } else if (k == "chunk") {
      if (value < 1) throw std::invalid_argument("chunk must be >= 1");
      e.chunk = (int)value;
    } else if (k == "graph") {
      e.use_graph = value != 0;
    } else if (k == "profile") {
      e.profile = value != 0;
    } else {
      throw std::invalid_argument("unknown ensemble option " + k);
    }
    return DEM_OK;
  });
}

int dem_ensemble_get_counters(dem_ensemble* h, long long* out, int n) {
  return eguard(h, [&](dem::Ensemble& e) {
    if (!out) throw std::invalid_argument("null output");
    const long long v[8] = {e.c_steps, e.c_contacts, e.c_launches, e.c_chunks, (long long)(e.prof_ms * 1e6),
                            e.prof_steps, (long long)e.pick_tpp(), e.c_rebuild_calls};
    for (int i = 0; i < n && i < 8; ++i) out[i] = v[i];
    return std::min(n, 8);
  });
}

}  // extern "C"
