/*
 * CPU restatement (FP64) of ESyS-Particle's per-timestep DEM hot path on one
 * worker.  TEST INFRASTRUCTURE: the oracle that the CUDA path is checked
 * against.  Only tests/, the smoke check and bench.py's CPU-baseline leg load
 * the library built from this file (oracle/_build/libesys_oracle.so).
 *
 * Parity pinning: on non-periodic inputs this restatement follows the
 * reference's interaction-list order and operation order, so its results are
 * compared bit-for-bit with the reference's own classes built into
 * oracle/_ref (tests/test_oracle_pin.py).  Periodic x, which the reference
 * only reaches with >= 2 MPI workers, is restated as the minimum-image
 * equivalent of the ghost-copy exchange (ppa/src/pp_array.hpp:465-503,
 * Model/Particle.cpp:305-342): a pair across the x boundary is evaluated once
 * with the image of p2 nearest p1, and each particle gets its share.
 *
 * Every function names the reference file:line it restates.  Vector algebra
 * follows Foundation/vec3.hpp, Foundation/Quaternion.hpp and
 * Foundation/Matrix3.hpp operation by operation; build with
 * -ffp-contract=off.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <vector>

namespace orc {

/* ---- Foundation/vec3.hpp restated (operation order preserved) ---------- */
struct V3 {
  double x = 0, y = 0, z = 0;
  V3() {}
  V3(double a, double b, double c) : x(a), y(b), z(c) {}
  double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
static inline V3 operator+(const V3& a, const V3& b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 operator-(const V3& a, const V3& b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 operator-(const V3& a) { return V3(-a.x, -a.y, -a.z); }
static inline V3 operator*(const V3& a, double s) { return V3(a.x * s, a.y * s, a.z * s); }   /* vec3.hpp:117 */
static inline V3 operator*(double f, const V3& a) { return V3(f * a.x, f * a.y, f * a.z); }   /* vec3.hpp:219 */
static inline V3 operator/(const V3& a, double s) { return V3(a.x / s, a.y / s, a.z / s); }
static inline double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; } /* vec3.hpp:112,211 */
static inline V3& operator+=(V3& a, const V3& b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
static inline V3& operator-=(V3& a, const V3& b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
static inline V3 cross(const V3& l, const V3& r) {                                             /* vec3.hpp:203 */
  return V3(l.y * r.z - l.z * r.y, l.z * r.x - l.x * r.z, l.x * r.y - l.y * r.x);
}
static inline double norm2(const V3& a) { return a.x * a.x + a.y * a.y + a.z * a.z; }        /* vec3.hpp:234 */
static inline double norm(const V3& a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); } /* vec3.hpp:227 */

/* ---- Foundation/Quaternion.hpp, Matrix3.hpp restated -------------------- */
struct Q { double s = 1; V3 v; Q() {} Q(double a, const V3& b) : s(a), v(b) {} };
static inline Q qmul(const Q& a, const Q& b) {                                                 /* Quaternion.hpp operator* */
  return Q(a.s * b.s - dot(a.v, b.v), a.s * b.v + b.s * a.v + cross(a.v, b.v));
}
static inline Q qinv(const Q& a) { return Q(a.s, -a.v); }
struct M3 { double m[3][3]; };
static inline M3 to_matrix(const Q& q) {                                                       /* Quaternion.hpp to_matrix */
  M3 r; const double s = q.s, x = q.v.x, y = q.v.y, z = q.v.z;
  r.m[0][0] = s * s + x * x - y * y - z * z;
  r.m[0][1] = 2 * (x * y + s * z);
  r.m[0][2] = 2 * (x * z - s * y);
  r.m[1][0] = 2 * (x * y - s * z);
  r.m[1][1] = s * s - x * x + y * y - z * z;
  r.m[1][2] = 2 * (y * z + s * x);
  r.m[2][0] = 2 * (x * z + s * y);
  r.m[2][1] = 2 * (y * z - s * x);
  r.m[2][2] = s * s - x * x - y * y + z * z;
  return r;
}
static inline M3 trans(const M3& a) { M3 r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[j][i]; return r; }
static inline V3 mul(const M3& a, const V3& v) {                                               /* Matrix3.hpp:126 */
  return V3(a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z,
            a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
            a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z);
}

/* ---- particle store: slots in insertion order (the reference's m_list order) */
struct Particles {
  std::vector<int> id, tag;
  std::vector<V3> pos, vel, force, oldpos, angvel, moment;
  std::vector<Q> quat;
  std::vector<double> rad, mass, invmass, inert, invinert;
  std::vector<double> gross_f, gross_m;  /* checker diagnostic: sum of |each force / moment| of the last step */
  std::vector<char> dyn, rot, flag, alive;
  int n() const { return (int)id.size(); }
};

struct Elastic { int p1, p2; double k; V3 force; bool touching = false; };
struct Fric {
  int p1, p2; double k, ks, mu_d, mu_s, dt; V3 Ffric; bool slipping = false, touching = false;
};
struct Bond {
  int p1, p2; V3 D; double kr, ks, kb, kt, max_n, max_s, max_b, max_t, truncated, beta1 = 1.0, beta2 = 1.0;
  double nF = 0, shF = 0, tM = 0, bM = 0; V3 force;
};
struct WallI { int p; double k; bool inner; };

struct PairGroup {            /* one dynamic (NE or ED) or bonded (EB) interaction storage */
  int kind;                   /* 0 elastic (NE), 1 rot friction (ED), 2 rot bond (EB) */
  std::string name;
  double k = 0; bool scaling = true;                            /* elastic prms */
  double fk = 0, mu_s = 0, mu_d = 0, fks = 0, fdt = 0; bool meanR = true; /* friction prms */
  int tag = 0; double kr = 0, ks = 0, kt = 0, kb = 0, mn = 0, ms = 0, mt = 0, mb = 0, trunc = 1.0;
  std::vector<Elastic> el; std::vector<Fric> fr; std::vector<Bond> bd;
  std::set<std::pair<int, int>> idset;                          /* m_set, by particle id */
  std::vector<PairGroup*> exig;                                 /* excluding groups */
  int update_ts = 0;
};
struct Wall { V3 o, n, F; V3 vel; bool loader = false; };
struct WallGroup { std::string wall; double k; std::vector<WallI> its; };
struct Damp { double visc; int maxiter; double dt; };

struct Sim {
  int rotmode;  /* 0 NRotSphere (CParticle), 1 RotSphere (CRotParticle) */
  double dt, nrange, alpha;
  V3 p0;                       /* global grid origin (nmin) */
  int nxg, nyg, nzg;           /* global cells */
  int nx, ny, nz;              /* local table incl. padding */
  int gx, gy, gz;              /* local origin index (-1 for padded dims) */
  bool circx = false; double Lx = 0, xmin = 0;
  Particles P;
  std::map<int, int> id2slot;
  std::vector<std::vector<int>> cells;
  std::map<std::string, Wall> walls;
  std::map<std::string, WallGroup> wig;
  std::map<std::string, V3> gravity;
  std::map<std::string, PairGroup*> dpis, bpis;
  std::map<std::string, Damp> damping;   /* keys "Damping", "RotDamping" */
  std::vector<int> damp_list;            /* particle slots at last damping update */
  std::map<int, std::vector<int>> temp_conn;
  std::vector<int> brk1, brk2, brkstep;
  int timestamp = 0, last_ns = -1;
  long long t = 0;
  bool first = true;
  std::string err;
};

/* ---- neighbour table (ntable/src/ntable.hpp) ----------------------------- */
/* NeighborTable::index (ntable.hpp:128-140); with periodic x the x index wraps. */
static int cell_index(const Sim& s, const V3& p) {
  if (!(std::isfinite(p.x) && std::isfinite(p.y) && std::isfinite(p.z))) return -1;
  int ix = int(std::floor((p.x - s.p0.x) / s.nrange)) - s.gx;
  int iy = int(std::floor((p.y - s.p0.y) / s.nrange)) - s.gy;
  int iz = int(std::floor((p.z - s.p0.z) / s.nrange)) - s.gz;
  if (s.circx) ix = ((ix % s.nx) + s.nx) % s.nx;
  if (ix >= 0 && ix < s.nx && iy >= 0 && iy < s.ny && iz >= 0 && iz < s.nz) return s.ny * s.nz * ix + s.nz * iy + iz;
  return -1;
}
/* NeighborTable::isInInner (ntable.hpp:212-233) */
static bool is_inner(const Sim& s, const V3& p) {
  int ix = int(std::floor((p.x - s.p0.x) / s.nrange)) - s.gx;
  int iy = int(std::floor((p.y - s.p0.y) / s.nrange)) - s.gy;
  int iz = int(std::floor((p.z - s.p0.z) / s.nrange)) - s.gz;
  bool inx = s.circx ? true : (ix > 0 && ix < s.nx - 1);
  if (s.nz < 3) return inx && iy > 0 && iy < s.ny - 1;
  return inx && iy > 0 && iy < s.ny - 1 && iz > 0 && iz < s.nz - 1;
}
/* position of p2 as seen from p1: the nearest periodic image in x */
static inline V3 image_of(const Sim& s, const V3& p1, V3 p2) {
  if (s.circx) {
    double dx = p1.x - p2.x;
    if (dx > 0.5 * s.Lx) p2.x += s.Lx;
    else if (dx < -0.5 * s.Lx) p2.x -= s.Lx;
  }
  return p2;
}
/* NeighborTable::build (ntable.hpp:262-288): rebin in list order, drop particles outside the grid.
 * Periodic x: positions are wrapped into the box first (the circular shift of pp_array.hpp:465-503). */
static void ntable_build(Sim& s) {
  for (auto& c : s.cells) c.clear();
  s.id2slot.clear();
  for (int i = 0; i < s.P.n(); ++i) {
    if (!s.P.alive[i]) continue;
    if (s.circx && std::isfinite(s.P.pos[i].x)) {
      V3& p = s.P.pos[i];
      if (p.x >= s.xmin + s.Lx || p.x < s.xmin) {
        p.x -= s.Lx * std::floor((p.x - s.xmin) / s.Lx);
        if (p.x >= s.xmin + s.Lx) p.x -= s.Lx;
      }
    }
    int idx = cell_index(s, s.P.pos[i]);
    if (idx != -1) { s.cells[idx].push_back(i); s.id2slot[s.P.id[i]] = i; }
    else s.P.alive[i] = 0;
  }
}
/* addPairsToList / addPairsToListLocal (ntable.hpp:471-521), with periodic minimum image */
static void add_pair_if_near(const Sim& s, int a, int b, std::vector<std::pair<int, int>>& out) {
  V3 pb = image_of(s, s.P.pos[a], s.P.pos[b]);
  double dist2 = norm2(s.P.pos[a] - pb);
  double dmax = s.P.rad[a] + s.P.rad[b] + s.alpha;
  if (dist2 <= (dmax * dmax)) {
    if (s.P.id[a] < s.P.id[b]) out.push_back({a, b}); else out.push_back({b, a});
  }
}
static void add_pair_flagged(const Sim& s, int a, int b, std::vector<std::pair<int, int>>& out) {
  if (s.P.flag[a] && s.P.flag[b]) {
    if (s.P.id[a] < s.P.id[b]) out.push_back({a, b}); else out.push_back({b, a});
  }
}
/* NeighborTable::getFullList / getNewList traversal (ntable.hpp:590-664).  Non-periodic: the
 * reference's cell order (ix,iy,iz) with idx2 > idx1.  Periodic x: the 13-cell forward
 * half stencil with x wrapping, which visits every unordered neighbour-cell pair once. */
template <class F>
static void traverse(const Sim& s, F pairfn, std::vector<std::pair<int, int>>& out) {
  auto idx = [&](int x, int y, int z) { return s.ny * s.nz * x + s.nz * y + z; };
  for (int ix = 0; ix < s.nx; ix++)
    for (int iy = 0; iy < s.ny; iy++)
      for (int iz = 0; iz < s.nz; iz++) {
        const std::vector<int>& c1 = s.cells[idx(ix, iy, iz)];
        if (c1.size() >= 2)
          for (size_t a = 0; a + 1 < c1.size(); ++a)
            for (size_t b = a + 1; b < c1.size(); ++b) pairfn(s, c1[a], c1[b], out);
        if (!s.circx) {
          int xmax = (ix < s.nx - 1) ? ix + 1 : ix, ymax = (iy < s.ny - 1) ? iy + 1 : iy, zmax = (iz < s.nz - 1) ? iz + 1 : iz;
          int xmin = (ix > 0) ? ix - 1 : ix, ymin = (iy > 0) ? iy - 1 : iy, zmin = (iz > 0) ? iz - 1 : iz;
          for (int i = xmin; i <= xmax; i++)
            for (int j = ymin; j <= ymax; j++)
              for (int k = zmin; k <= zmax; k++) {
                int i1 = idx(ix, iy, iz), i2 = idx(i, j, k);
                if (i2 > i1)
                  for (int a : s.cells[i1]) for (int b : s.cells[i2]) pairfn(s, a, b, out);
              }
        } else {
          for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
              for (int dz = -1; dz <= 1; ++dz) {
                /* forward half: (dx,dy,dz) lexicographically positive */
                if (dx < 0 || (dx == 0 && (dy < 0 || (dy == 0 && dz <= 0)))) continue;
                int jx = ((ix + dx) % s.nx + s.nx) % s.nx, jy = iy + dy, jz = iz + dz;
                if (jy < 0 || jy >= s.ny || jz < 0 || jz >= s.nz) continue;
                for (int a : c1) for (int b : s.cells[idx(jx, jy, jz)]) pairfn(s, a, b, out);
              }
        }
      }
}
static std::vector<std::pair<int, int>> full_list(const Sim& s) {
  std::vector<std::pair<int, int>> out;
  traverse(s, add_pair_if_near, out);
  return out;
}
static std::vector<std::pair<int, int>> new_list(Sim& s) {
  std::vector<std::pair<int, int>> out;
  traverse(s, add_pair_flagged, out);
  for (int i = 0; i < s.P.n(); ++i) s.P.flag[i] = 0;   /* ntable.hpp:658-662 */
  return out;
}

/* ---- interaction constructors (scaling) ---------------------------------- */
/* CElasticInteraction ctor (Model/ElasticInteraction.cpp:25-49) */
static Elastic make_elastic(const Sim& s, const PairGroup& g, int a, int b) {
  double effR = 1.0, effA = 1.0, effL = 1.0;
  double r0 = s.P.rad[a] + s.P.rad[b];
  if (g.scaling) { effR = 0.5 * r0; effL = r0; effA = effR * effR; }
  Elastic e; e.p1 = a; e.p2 = b; e.k = g.k * effA / effL;
  return e;
}
/* CRotFrictionInteraction ctor (Model/RotFricInteraction.cpp:103-146) */
static Fric make_fric(const Sim& s, const PairGroup& g, int a, int b) {
  double effR = 1.0, effL = 1.0, effA = 1.0;
  double r0 = s.P.rad[a] + s.P.rad[b];
  if (g.scaling) {
    if (g.meanR) effR = 0.5 * r0; else effR = std::fmin(s.P.rad[a], s.P.rad[b]);
    effL = r0; effA = effR * effR;
  }
  Fric f; f.p1 = a; f.p2 = b;
  f.k = g.fk * effA / effL; f.ks = g.fks * effA / effL;
  f.mu_d = g.mu_d; f.mu_s = g.mu_s; f.dt = g.fdt;
  return f;
}
/* ARotBondedInteraction ctor (ARotBondedInteraction.cpp:141-180) + CRotBondedInteraction ctor
 * (Model/RotBondedInteraction.cpp:122-161); p1 is the lower id (pi_storage_e.hpp:222-263). */
static Bond make_bond(const Sim& s, const PairGroup& g, int a, int b) {
  Bond d; d.p1 = a; d.p2 = b;
  d.D = s.P.pos[b] - s.P.pos[a];
  double dist = std::sqrt(dot(d.D, d.D));
  double effR = 1.0, effL = 1.0, effA = 1.0, J = 1.0, I = 1.0;
  if (g.scaling) {
    if (g.meanR) effR = 0.5 * dist; else effR = std::fmin(s.P.rad[a], s.P.rad[b]);
    effL = dist; effA = effR * effR;
    J = 0.5 * effR * effR * effR * effR; I = 0.5 * J;
  }
  d.kr = g.kr * effA / effL; d.ks = g.ks * effA / effL; d.kb = g.kb * I / effL; d.kt = g.kt * J / effL;
  d.max_n = g.mn * effA; d.max_s = g.ms * effA; d.max_b = g.mb * I / effR; d.max_t = g.mt * J / effR;
  d.truncated = g.trunc;
  return d;
}

/* ---- force laws ------------------------------------------------------------ */
/* CParticle::applyForce (Model/Particle.cpp:391-400), without the stress tensor */
static inline void apply_force(Sim& s, int i, const V3& f) {
  s.P.force[i] += f;
  if (i < (int)s.P.gross_f.size()) s.P.gross_f[i] += norm(f);  /* the checker's force scale, not a force */
}
static inline void apply_moment(Sim& s, int i, const V3& m) {
  s.P.moment[i] += m;
  if (i < (int)s.P.gross_m.size()) s.P.gross_m[i] += norm(m);
}

/* CElasticInteraction::calcForces (Model/ElasticInteraction.cpp:54-71) */
static void calc_elastic(Sim& s, Elastic& e) {
  const V3 x1 = s.P.pos[e.p1], x2 = image_of(s, x1, s.P.pos[e.p2]);
  V3 D = x1 - x2;
  double dist = dot(D, D);
  double eq_dist = s.P.rad[e.p1] + s.P.rad[e.p2];
  if (dist < (eq_dist * eq_dist)) {
    dist = std::sqrt(dist);
    V3 F = D * (e.k * (dist - eq_dist) / dist);
    apply_force(s, e.p2, F);
    apply_force(s, e.p1, -1.0 * F);
    e.force = F;
    e.touching = true;
  } else {
    e.touching = false;
  }
}
/* CRotFrictionInteraction::calcSimpleForces (Model/RotFricInteraction.cpp:171-231) */
static void calc_fric(Sim& s, Fric& f) {
  double mu_current = f.slipping ? f.mu_d : f.mu_s;
  const V3 x1 = s.P.pos[f.p1], x2 = image_of(s, x1, s.P.pos[f.p2]);
  const V3 D = x1 - x2;
  double dist = dot(D, D);
  const double r1 = s.P.rad[f.p1], r2 = s.P.rad[f.p2];
  const double eq_dist = r1 + r2;
  if (dist < (eq_dist * eq_dist)) {
    dist = std::sqrt(dist);
    const V3 force(D * (f.k * (dist - eq_dist) / dist));
    const V3 pos(x2 + (r2 / eq_dist) * D);
    apply_force(s, f.p2, force);
    apply_force(s, f.p1, -1.0 * force);
    const V3 vp1 = s.P.vel[f.p1] + cross(s.P.angvel[f.p1], pos - x1);
    const V3 vp2 = s.P.vel[f.p2] + cross(s.P.angvel[f.p2], pos - x2);
    V3 ds((vp2 - vp1) * f.dt);
    ds -= ((dot(ds, D)) / (norm2(D))) * D;
    f.Ffric += f.ks * ds;
    const double FfricNorm = norm(f.Ffric);
    const double forceNorm = norm(force);
    if (FfricNorm > forceNorm * mu_current) {
      f.Ffric = f.Ffric * ((f.mu_d * forceNorm) / FfricNorm);
      f.slipping = true;
    } else {
      f.slipping = false;
    }
    const V3 Moment1(cross(pos - x1, f.Ffric));
    const V3 Moment2(cross(pos - x2, -f.Ffric));
    apply_moment(s, f.p1, Moment1);
    apply_moment(s, f.p2, Moment2);
    apply_force(s, f.p1, f.Ffric);
    apply_force(s, f.p2, -1.0 * f.Ffric);
    f.touching = true;
  } else {
    f.Ffric = V3(0, 0, 0);
    f.slipping = false;
    f.touching = false;
  }
}
/* calc_angle (Model/ARotBondedInteraction.cpp:22-51) */
static double calc_angle(double s_in, double c_os) {
  if (s_in > 0.0) return (c_os >= 1.0 || c_os <= -1.0) ? 0.0 : std::acos(c_os);
  if (s_in == 0.0) return 0.0;
  return (c_os >= 1.0 || c_os <= -1.0) ? 0.0 : -std::acos(c_os);
}
/* ARotBondedInteraction::calcForces (Model/ARotBondedInteraction.cpp:307-448) */
static void calc_bond(Sim& s, Bond& b) {
  const double HALF_SQRT_2 = 0.5 * std::sqrt(2.0);
  double s_fai = 0.0, c_fai = 0.0, c_pasi2 = 0.0, s_pasi2 = 0.0, sita = 0.0, pasi = 0.0;
  const Q q1 = s.P.quat[b.p1], q2 = s.P.quat[b.p2];
  const V3 x1 = s.P.pos[b.p1], x2 = image_of(s, x1, s.P.pos[b.p2]);
  const double r1 = s.P.rad[b.p1], r2 = s.P.rad[b.p2];
  const M3 mat0 = to_matrix(q1);
  const V3 rbp = x2 - x1;
  const double rbpNorm = norm(rbp);
  const V3 rb = mul(mat0, x2 - x1);
  const double rbNorm = norm(rb);
  const double r_0Norm = r1 + r2;
  const V3 delta_r = (rbNorm - r_0Norm) * rb / rbNorm;
  const V3 Fr = b.kr * delta_r;
  const double gama_cos = dot(rb, b.D) / (rbNorm * norm(b.D));
  double gama = 0.0;
  if (gama_cos < 1.0 && gama_cos > -1.0) gama = std::acos(gama_cos);
  const V3 rb_0 = cross(rb, b.D);
  const V3 rb_b0 = cross(rb, rb_0);
  const double rb_b0Norm = norm(rb_b0);
  V3 Fst(0, 0, 0);
  if (rb_b0Norm != 0) Fst = b.ks * r_0Norm * gama * rb_b0 / rb_b0Norm;
  V3 Mst(0, 0, 0);
  const double rb_0Norm = norm(rb_0);
  if (rb_0Norm != 0) Mst = -norm(Fst) * rb_0 / rb_0Norm;
  const double m0 = HALF_SQRT_2 * std::sqrt((rbNorm + rb.z) / rbNorm);
  double m1 = -HALF_SQRT_2 * std::sqrt((rbNorm - rb.z) / rbNorm);
  double m2 = -m1;
  const double m3 = 0.0;
  const double rbX2PlusRbY2 = rb.x * rb.x + rb.y * rb.y;
  if (rbX2PlusRbY2 != 0.0) {
    const double denomSqrt = std::sqrt(rbX2PlusRbY2);
    m1 = m1 * rb.y / denomSqrt;
    m2 = m2 * rb.x / denomSqrt;
  }
  const Q qm(m0, V3(m1, m2, m3));
  const M3 mat = to_matrix(qm);
  const M3 matTrans = trans(mat);
  const Q rp = qmul(qinv(q1), q2);
  const Q r = qmul(qmul(qinv(qm), rp), qm);
  const double temp0 = r.s * r.s + r.v.z * r.v.z;
  if (temp0 == 0.0) {
    pasi = 0.0;
  } else {
    const double sqrtTemp0 = std::sqrt(temp0);
    c_pasi2 = r.s / sqrtTemp0;
    s_pasi2 = r.v.z / sqrtTemp0;
    pasi = 2.0 * calc_angle(s_pasi2, c_pasi2);
  }
  const V3 Mtp(0.0, 0.0, b.kt * pasi);
  const V3 Mtr = mul(matTrans, Mtp);
  const double temp2 = r.v.x * r.v.x + r.v.y * r.v.y;
  const double temp3 = r.v.x * r.v.z + r.s * r.v.y;
  const double temp4 = r.v.y * r.v.z - r.s * r.v.x;
  V3 Mbr(0, 0, 0), Fsr(0, 0, 0), Msr(0, 0, 0);
  if (temp2 != 0.0) {
    const double temp1 = temp0 - temp2;
    if (temp1 >= 1.0 || temp1 <= -1.0) sita = 0.0; else sita = std::acos(temp1);
    if (temp0 == 0.0) {
      const double sqrtDenom = std::sqrt(temp2);
      c_fai = r.v.y / sqrtDenom;
      s_fai = -r.v.x / sqrtDenom;
    } else {
      const double sqrtDenom = std::sqrt(temp0 * temp2);
      c_fai = temp3 / sqrtDenom;
      s_fai = temp4 / sqrtDenom;
    }
    const V3 Mbp(-0.5 * b.kb * sita * s_fai, 0.5 * b.kb * sita * c_fai, 0.0);
    Mbr = mul(matTrans, Mbp);
    const V3 Fsp(-0.5 * b.ks * c_fai * sita * r_0Norm, -0.5 * b.ks * s_fai * sita * r_0Norm, 0.0);
    Fsr = mul(matTrans, Fsp);
    const V3 Msp(0.5 * b.ks * s_fai * sita * r_0Norm, -0.5 * b.ks * c_fai * sita * r_0Norm, 0.0);
    Msr = mul(matTrans, Msp);
  }
  const double eq_rad1 = r1 / (r1 + r2);
  const double eq_rad2 = r2 / (r1 + r2);
  const M3 mat0Trans = trans(mat0);
  const V3 force = mul(mat0Trans, Fr + Fst + Fsr);
  const V3 moment = mul(mat0Trans, Mbr + Mtr + Msr * eq_rad1 * rbpNorm + Mst * eq_rad1 * rbpNorm);
  const V3 moment2 = mul(mat0Trans, Msr * eq_rad2 * rbpNorm + Mst * eq_rad2 * rbpNorm - Mbr - Mtr);
  b.shF = norm(Fst + Fsr);
  b.tM = norm(Mtr);
  b.bM = norm(Mbr);
  const double r0 = r1 + r2;
  const V3 D = x1 - x2;
  const double dist = std::sqrt(dot(D, D));
  b.nF = ((dist < r0) ? -1.0 : 1.0) * norm(Fr);
  b.force = force;
  apply_force(s, b.p2, -1.0 * force);
  apply_force(s, b.p1, force);
  apply_moment(s, b.p1, moment);
  apply_moment(s, b.p2, moment2);
}
/* CRotBondedInteraction::broken (Model/RotBondedInteraction.cpp:175-219) */
static bool bond_broken(Sim& s, const Bond& b) {
  double shearStress = b.shF / b.max_s + b.beta2 * b.tM / b.max_t;
  double normalStress = b.nF / b.max_n + b.beta1 * b.bM / b.max_b;
  if ((normalStress > b.truncated) || (shearStress > (1.0 - normalStress))) {
    s.P.flag[b.p1] = 1; s.P.flag[b.p2] = 1;
    return true;
  }
  return false;
}
/* CElasticWallInteraction<T>::calcForces (Model/EWallInteraction.hpp:42-78) */
static void calc_wall(Sim& s, Wall& w, const WallI& wi) {
  double dist = dot(s.P.pos[wi.p] - w.o, w.n);
  const double r = s.P.rad[wi.p];
  if (dist < r) {
    V3 force = wi.k * (r - dist) * w.n;
    apply_force(s, wi.p, force);
    if (wi.inner) w.F -= -1.0 * force;   /* CWall::addForce(-F): m_force -= (-F) (Model/Wall.h:68) */
  }
}
/* CDamping<T>::calcForces (Model/Damping.hpp:99-124); vref = 0 (DampingIGP.cpp:28-42) */
static void calc_damping(Sim& s, int i, const Damp& d) {
  const double s_limit2 = 1e-12;
  V3 v = s.P.vel[i], v_rel(0, 0, 0), frc = s.P.force[i], vref(0, 0, 0);
  double sm = s.P.invmass[i], mass = s.P.mass[i], error = 1.0;
  int count = 0;
  while ((error * error > s_limit2) & (count < d.maxiter)) {
    count++;
    V3 v_old = v_rel;
    v_rel = v - vref + sm * d.dt * (frc - v_rel * d.visc * mass);
    error = norm2(v_rel - v_old);
  }
  if (count >= d.maxiter) v_rel = V3(0, 0, 0);
  V3 F = -1.0 * d.visc * v_rel * mass;
  apply_force(s, i, F);
}
/* CRotDamping<T>::calcForces (Model/RotDamping.hpp:58-84) */
static void calc_rot_damping(Sim& s, int i, const Damp& d) {
  const double s_limit2 = 1e-12;
  V3 v = s.P.angvel[i], v_rel(0, 0, 0), frc = s.P.moment[i], vref(0, 0, 0);
  double sm = 1.0 / s.P.inert[i], in = s.P.inert[i], error = 1.0;
  int count = 0;
  while ((error * error > s_limit2) & (count < d.maxiter)) {
    count++;
    V3 v_old = v_rel;
    v_rel = v - vref + sm * d.dt * (frc - v_rel * d.visc * in);
    error = norm2(v_rel - v_old);
  }
  if (count >= d.maxiter) v_rel = V3(0, 0, 0);
  apply_moment(s, i, -1.0 * d.visc * v_rel * in);
}
/* CParticle::integrate / CRotParticle::integrate + rescale
 * (Model/Particle.cpp:257-274, Model/RotParticle.cpp:277-321) */
static void integrate(Sim& s, int i) {
  double dt = s.dt;
  if (s.rotmode) {
    if (s.P.rot[i]) {
      s.P.angvel[i] += (dt * s.P.invinert[i]) * s.P.moment[i];
      Q w(0, s.P.angvel[i]);
      Q dq = qmul(w, s.P.quat[i]);
      double c = dt / 2.0;
      s.P.quat[i].s += c * dq.s;
      s.P.quat[i].v += c * dq.v;
    } else {
      s.P.angvel[i] = V3(0, 0, 0);
    }
  }
  if (s.P.dyn[i]) {
    s.P.vel[i] += s.P.force[i] * s.P.invmass[i] * dt;
    s.P.pos[i] += s.P.vel[i] * dt;
  }
}
static void rescale(Sim& s, int i) {
  if (!s.rotmode) return;
  Q& q = s.P.quat[i];
  const double module = std::sqrt(q.s * q.s + q.v.x * q.v.x + q.v.y * q.v.y + q.v.z * q.v.z);
  if (module != 0.0) {
    const double inverse = 1.0 / module;
    q = Q(inverse * q.s, inverse * q.v);
  }
}

/* ---- interaction storages -------------------------------------------------- */
static bool is_excluded(PairGroup& g, int id1, int id2) {     /* pi_storage_ed.hpp:49-61 */
  for (auto* e : g.exig) if (e->idset.count({id1, id2})) return true;
  return false;
}
/* PIS_E::rebuild (pi_storage_e.hpp:111-155): drop interactions whose particles vanished */
template <class V>
static void pis_rebuild(Sim& s, PairGroup& g, V& v) {
  V keep;
  for (auto& it : v) {
    if (s.P.alive[it.p1] && s.P.alive[it.p2]) keep.push_back(it);
    else g.idset.erase({s.P.id[it.p1], s.P.id[it.p2]});
  }
  v.swap(keep);
}
static void group_rebuild(Sim& s, PairGroup& g) {
  if (g.kind == 0) pis_rebuild(s, g, g.el);
  else if (g.kind == 1) pis_rebuild(s, g, g.fr);
  else pis_rebuild(s, g, g.bd);
}
/* PIS_NE::update (pi_storage_ne.hpp:49-102) and PIS_ED::update (pi_storage_ed.hpp:84-161) */
static void dyn_update(Sim& s, PairGroup& g) {
  if (g.update_ts != s.timestamp) {
    std::vector<std::pair<int, int>> pl = full_list(s);
    if (g.kind == 0) {
      g.el.clear(); g.idset.clear();
      for (auto& p : pl) {
        int a = s.P.id[p.first], b = s.P.id[p.second];
        if (!is_excluded(g, a, b)) { g.el.push_back(make_elastic(s, g, p.first, p.second)); g.idset.insert({a, b}); }
      }
    } else {
      std::vector<Fric> keep;
      for (auto& f : g.fr) {
        /* CRotFrictionInteraction::isPersistent (RotFricInteraction.cpp:345-351) */
        const V3 x1 = s.P.pos[f.p1], x2 = image_of(s, x1, s.P.pos[f.p2]);
        V3 D = x1 - x2;
        double dist = dot(D, D), eq = s.P.rad[f.p1] + s.P.rad[f.p2];
        if (dist <= (eq * eq)) keep.push_back(f);
        else g.idset.erase({s.P.id[f.p1], s.P.id[f.p2]});
      }
      g.fr.swap(keep);
      for (auto& p : pl) {
        int a = s.P.id[p.first], b = s.P.id[p.second];
        if (!is_excluded(g, a, b) && !g.idset.count({a, b})) {
          g.fr.push_back(make_fric(s, g, p.first, p.second));
          g.idset.insert({a, b});
        }
      }
    }
  } else {
    std::vector<std::pair<int, int>> pl = new_list(s);
    for (auto& p : pl) {
      int a = s.P.id[p.first], b = s.P.id[p.second];
      if (g.kind == 0) {
        if (!is_excluded(g, a, b)) { g.el.push_back(make_elastic(s, g, p.first, p.second)); g.idset.insert({a, b}); }
      } else if (!is_excluded(g, a, b) && !g.idset.count({a, b})) {
        g.fr.push_back(make_fric(s, g, p.first, p.second));
        g.idset.insert({a, b});
      }
    }
  }
  g.update_ts = s.timestamp;
}
/* PIS_EB::update (pi_storage_eb.hpp:23-49) */
static bool bond_update(Sim& s, PairGroup& g) {
  bool res = false;
  std::vector<Bond> keep;
  for (auto& b : g.bd) {
    if (bond_broken(s, b)) {
      res = true;
      int a = s.P.id[b.p1], c = s.P.id[b.p2];
      g.idset.erase({a, c});
      s.brk1.push_back(a); s.brk2.push_back(c); s.brkstep.push_back((int)s.t);
    } else keep.push_back(b);
  }
  g.bd.swap(keep);
  return res;
}
/* CEWallInteractionGroup::Update (EWallInteractionGroup.hpp:57-82) via getParticlesAtPlane (ntable.hpp:674-690) */
static void wall_update(Sim& s, WallGroup& wg) {
  wg.its.clear();
  Wall& w = s.walls[wg.wall];
  for (int i = 0; i < s.P.n(); ++i) {
    if (!s.P.alive[i]) continue;
    double dist = dot(s.P.pos[i] - w.o, w.n);
    if (std::fabs(dist) < s.nrange) {
      double f = 1.0;
      f *= 3.141592654 * s.P.rad[i];   /* EWallInteraction.hpp:26-36 */
      wg.its.push_back(WallI{i, f * wg.k, is_inner(s, s.P.pos[i])});
    }
  }
}
/* PIS_Single::update (pi_storage_single.hpp:22-43) */
static void damping_update(Sim& s) {
  s.damp_list.clear();
  for (int i = 0; i < s.P.n(); ++i) if (s.P.alive[i]) s.damp_list.push_back(i);
}

/* ---- TSubLattice step sequence ------------------------------------------- */
/* searchNeighbors = ppa rebuild + rebuildInteractions + resetDisplacements (SubLattice.hpp:2360-2408) */
static void search_neighbors(Sim& s) {
  ntable_build(s);
  s.timestamp++;
  for (auto& b : s.bpis) group_rebuild(s, *b.second);
  for (auto& d : s.dpis) group_rebuild(s, *d.second);
  for (int i = 0; i < s.P.n(); ++i) s.P.oldpos[i] = s.P.pos[i];
}
/* TSubLattice::checkNeighbors (SubLattice.hpp:2473-2519), early exit in list order */
static bool check_neighbors(Sim& s) {
  double mdsqr = 0, a = 0.5 * s.alpha, srsqr = a * a;
  for (int i = 0; i < s.P.n() && mdsqr < srsqr; ++i) {
    if (!s.P.alive[i]) continue;
    V3 d = s.P.pos[i] - s.P.oldpos[i];
    double sq = dot(d, d);
    mdsqr = (mdsqr < sq) ? sq : mdsqr;
  }
  return mdsqr > srsqr;
}
/* TSubLattice::updateInteractions (SubLattice.hpp:2416-2466) */
static void update_interactions(Sim& s) {
  bool need = false;
  for (auto& b : s.bpis) need = bond_update(s, *b.second) || need;
  if (s.timestamp > s.last_ns || need) {
    for (auto& d : s.dpis) dyn_update(s, *d.second);
    for (auto& w : s.wig) wall_update(s, w.second);
    if (!s.damping.empty()) damping_update(s);
    s.last_ns = s.timestamp;
  }
}
/* TSubLattice::oneStep (SubLattice.hpp:2066-2236): zero, calcForces in group order, integrate, rescale */
static void one_step(Sim& s) {
  for (int i = 0; i < s.P.n(); ++i) { s.P.force[i] = V3(0, 0, 0); s.P.moment[i] = V3(0, 0, 0); }
  s.P.gross_f.assign(s.P.n(), 0.0);
  s.P.gross_m.assign(s.P.n(), 0.0);
  for (auto& w : s.walls) w.second.F = V3(0, 0, 0);
  for (auto& wg : s.wig) { Wall& w = s.walls[wg.second.wall]; for (auto& wi : wg.second.its) calc_wall(s, w, wi); }
  for (auto& g : s.gravity)   /* BodyForceGroup::calcForces (BodyForceGroup.hpp:54-65) */
    for (int i = 0; i < s.P.n(); ++i) if (s.P.alive[i]) apply_force(s, i, g.second * s.P.mass[i]);
  for (auto& d : s.dpis) {
    if (d.second->kind == 0) for (auto& e : d.second->el) calc_elastic(s, e);
    else for (auto& f : d.second->fr) calc_fric(s, f);
  }
  for (auto& b : s.bpis) for (auto& bd : b.second->bd) calc_bond(s, bd);
  for (auto& d : s.damping) {
    if (d.first == "Damping") for (int i : s.damp_list) calc_damping(s, i, d.second);
    else for (int i : s.damp_list) calc_rot_damping(s, i, d.second);
  }
  for (int i = 0; i < s.P.n(); ++i) if (s.P.alive[i]) integrate(s, i);
  for (int i = 0; i < s.P.n(); ++i) if (s.P.alive[i]) rescale(s, i);
}

static void move_loaded_walls(Sim& s) {
  for (auto& w : s.walls)
    if (w.second.loader) {
      w.second.o.x += w.second.vel.x * s.dt;
      w.second.o.y += w.second.vel.y * s.dt;
      w.second.o.z += w.second.vel.z * s.dt;
    }
}

}  // namespace orc

using namespace orc;

extern "C" {

/* TSubLattice::initNeighborTable (Parallel/SubLattice.hpp:455-564) + ParallelParticleArray ctor
 * (ppa/src/pp_array.hpp:55-100) for one worker: one padding cell on each non-periodic side. */
int orc_create(void** out, int ptype, double gs, double vd, const double* mn, const double* mx, const int* circ, double dt) {
  Sim* s = new Sim();
  s->rotmode = ptype ? 1 : 0;
  s->dt = dt; s->nrange = gs; s->alpha = vd;
  s->circx = circ && circ[0];
  double size[3];
  for (int i = 0; i < 3; ++i) {
    double sz = mx[i] - mn[i];
    if (i == 0 && s->circx) {
      if (std::fabs(sz / s->nrange - std::lrint(sz / s->nrange)) > 1e-6) s->nrange = sz / std::floor(sz / s->nrange);
      size[i] = sz;
    } else {
      size[i] = s->nrange * std::ceil(sz / s->nrange);
    }
  }
  V3 vmin(mn[0], mn[1], mn[2]), vmax(mx[0], mx[1], mx[2]);
  V3 grow = V3(size[0], size[1], size[2]) - (vmax - vmin);
  V3 nmin = vmin - 0.5 * grow, nmax = vmax + 0.5 * grow;
  s->p0 = nmin;
  s->nxg = (int)std::lrint((nmax.x - nmin.x) / s->nrange);
  s->nyg = (int)std::lrint((nmax.y - nmin.y) / s->nrange);
  s->nzg = (int)std::lrint((nmax.z - nmin.z) / s->nrange);
  if (s->circx) { s->gx = 0; s->nx = s->nxg; s->Lx = nmax.x - nmin.x; s->xmin = nmin.x; }
  else { s->gx = -1; s->nx = s->nxg + 2; }
  s->gy = -1; s->ny = s->nyg + 2;
  s->gz = -1; s->nz = s->nzg + 2;
  if (s->circx && s->nx < 3) { s->err = "periodic x needs at least 3 cells"; *out = s; return -1; }
  s->cells.assign((size_t)s->nx * s->ny * s->nz, {});
  *out = s;
  return 0;
}
int orc_destroy(void* h) {
  Sim* s = (Sim*)h;
  for (auto& d : s->dpis) delete d.second;
  for (auto& b : s->bpis) delete b.second;
  delete s;
  return 0;
}
const char* orc_last_error(void* h) { return ((Sim*)h)->err.c_str(); }

int orc_add_particles(void* h, int n, const int* id, const int* tag, const double* pos, const double* rad,
                      const double* mass, const double* vel, const double* angvel, const double* quat, const int* flags) {
  Sim& s = *(Sim*)h;
  Particles& P = s.P;
  for (int i = 0; i < n; ++i) {
    V3 p(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    if (cell_index(s, p) == -1) continue;   /* NeighborTable::insert deletes outside particles (ntable.hpp:243-258) */
    P.id.push_back(id[i]); P.tag.push_back(tag ? tag[i] : 0);
    P.pos.push_back(p); P.oldpos.push_back(p);
    P.vel.push_back(vel ? V3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]) : V3());
    P.angvel.push_back(angvel && s.rotmode ? V3(angvel[3 * i], angvel[3 * i + 1], angvel[3 * i + 2]) : V3());
    P.quat.push_back(quat && s.rotmode ? Q(quat[4 * i], V3(quat[4 * i + 1], quat[4 * i + 2], quat[4 * i + 3])) : Q(1.0, V3()));
    P.force.push_back(V3()); P.moment.push_back(V3());
    P.rad.push_back(rad[i]); P.mass.push_back(mass[i]);
    P.invmass.push_back(mass[i] != 0.0 ? 1.0 / mass[i] : 0.0);
    double inert = 0.4 * mass[i] * rad[i] * rad[i];   /* RotParticle.cpp:34 */
    P.inert.push_back(inert); P.invinert.push_back(1.0 / inert);
    P.dyn.push_back(!(flags && (flags[i] & 1)));
    P.rot.push_back(s.rotmode && !(flags && (flags[i] & 2)));
    P.flag.push_back(0); P.alive.push_back(1);
  }
  search_neighbors(s);   /* LatticeMaster.hpp:329 */
  return 0;
}
int orc_add_connections(void* h, int n, const int* tag, const int* a, const int* b) {
  Sim& s = *(Sim*)h;
  for (int i = 0; i < n; ++i) { s.temp_conn[tag[i]].push_back(a[i]); s.temp_conn[tag[i]].push_back(b[i]); }
  search_neighbors(s);   /* LatticeMaster.hpp:397 */
  return 0;
}
int orc_add_wall(void* h, const char* name, const double* o, const double* n) {
  Sim& s = *(Sim*)h;
  s.walls[name] = Wall{V3(o[0], o[1], o[2]), V3(n[0], n[1], n[2]), V3()};
  return 0;
}
int orc_add_elastic_group(void* h, const char* name, double k, int scaling) {
  Sim& s = *(Sim*)h;
  PairGroup* g = new PairGroup(); g->kind = 0; g->name = name; g->k = k; g->scaling = scaling != 0;
  s.dpis[name] = g;
  return 0;
}
int orc_add_rot_friction_group(void* h, const char* name, double k, double mu_s, double mu_d, double ks, double dt,
                               int scaling, int meanR) {
  Sim& s = *(Sim*)h;
  if (!s.rotmode) { s.err = "RotFriction needs RotSphere particles"; return -1; }
  PairGroup* g = new PairGroup(); g->kind = 1; g->name = name;
  g->fk = k; g->mu_s = mu_s; g->mu_d = mu_d; g->fks = ks; g->fdt = dt; g->scaling = scaling != 0; g->meanR = meanR != 0;
  s.dpis[name] = g;
  return 0;
}
/* TRotSubLattice::addRotBondedIG (RotSubLattice.hpp:116-186) -> PIS_E::tryInsert(vector<int>) (pi_storage_e.hpp:222-263) */
int orc_add_rot_bond_group(void* h, const char* name, int tag, double kr, double ks, double kt, double kb, double mn,
                           double ms, double mt, double mb, int scaling, int meanR, double trunc) {
  Sim& s = *(Sim*)h;
  if (!s.rotmode) { s.err = "RotBond needs RotSphere particles"; return -1; }
  PairGroup* g = new PairGroup(); g->kind = 2; g->name = name; g->tag = tag;
  g->kr = kr; g->ks = ks; g->kt = kt; g->kb = kb; g->mn = mn; g->ms = ms; g->mt = mt; g->mb = mb;
  g->scaling = scaling != 0; g->meanR = meanR != 0; g->trunc = trunc;
  std::vector<int>& c = s.temp_conn[tag];
  for (size_t i = 0; i + 1 < c.size(); i += 2) {
    int a = std::min(c[i], c[i + 1]), b = std::max(c[i], c[i + 1]);
    if (g->idset.count({a, b})) continue;
    auto ia = s.id2slot.find(a), ib = s.id2slot.find(b);
    if (ia == s.id2slot.end() || ib == s.id2slot.end()) continue;
    g->bd.push_back(make_bond(s, *g, ia->second, ib->second));
    g->idset.insert({a, b});
  }
  s.bpis[name] = g;
  return 0;
}
int orc_add_wall_group(void* h, const char* name, const char* wall, double k) {
  Sim& s = *(Sim*)h;
  if (!s.walls.count(wall)) { s.err = std::string("wall name '") + wall + "' not found in map of walls"; return -1; }
  WallGroup wg; wg.wall = wall; wg.k = k;
  s.wig[name] = wg;
  wall_update(s, s.wig[name]);
  return 0;
}
int orc_add_gravity(void* h, const char* name, const double* g) {
  Sim& s = *(Sim*)h;
  s.gravity[name] = V3(g[0], g[1], g[2]);
  return 0;
}
int orc_add_damping(void* h, int rot, double visc, int maxiter) {
  Sim& s = *(Sim*)h;
  if (rot && !s.rotmode) { s.err = "RotDamping needs RotSphere particles"; return -1; }
  s.damping[rot ? "RotDamping" : "Damping"] = Damp{visc, maxiter, s.dt};
  damping_update(s);
  return 0;
}
/* TSubLattice::setExIG (SubLattice.hpp:1980-2009) + PIS_ED::addExIG (pi_storage_ed.hpp:20-40) */
int orc_add_exclusion(void* h, const char* s1, const char* s2) {
  Sim& s = *(Sim*)h;
  auto ex = s.bpis.find(s1);
  PairGroup* exg = nullptr;
  if (ex != s.bpis.end()) exg = ex->second;
  else { auto e2 = s.dpis.find(s2); if (e2 == s.dpis.end()) { s.err = "nonexisting interaction group"; return -1; } exg = e2->second; }
  auto dy = s.dpis.find(s2);
  if (dy == s.dpis.end()) { s.err = "nonexisting interaction group"; return -1; }
  PairGroup& g = *dy->second;
  g.exig.push_back(exg);
  if (g.kind == 1) {
    std::vector<Fric> keep;
    for (auto& f : g.fr) {
      std::pair<int, int> k{s.P.id[f.p1], s.P.id[f.p2]};
      if (exg->idset.count(k)) g.idset.erase(k); else keep.push_back(f);
    }
    g.fr.swap(keep);
  }
  return 0;
}
/* CLatticeMaster::runOneStep (LatticeMaster.cpp:2602-2725) */
int orc_step(void* h, int n) {
  Sim& s = *(Sim*)h;
  for (int k = 0; k < n; ++k) {
    if (s.first) { search_neighbors(s); s.first = false; }
    s.t++;
    if (check_neighbors(s)) search_neighbors(s);
    update_interactions(s);
    one_step(s);
    move_loaded_walls(s);
  }
  return 0;
}
/* State of the particles with these ids (rows; any array may be null); a particle deleted when it
   left the grid comes back alive (the ghost copies of a slab decomposition, which the reference
   re-sends at every rebuild, pp_array.hpp:450-504); then a neighbour search, as after an insert. */
int orc_set_particles(void* h, int n, const int* id, const double* pos, const double* vel, const double* angvel,
                      const double* quat) {
  Sim& s = *(Sim*)h;
  std::map<int, int> slot;
  for (int i = 0; i < s.P.n(); ++i) slot[s.P.id[i]] = i;
  bool revived = false;
  for (int r = 0; r < n; ++r) {
    auto it = slot.find(id[r]);
    if (it == slot.end()) return -1;
    const int i = it->second;
    if (pos) s.P.pos[i] = V3(pos[3 * r], pos[3 * r + 1], pos[3 * r + 2]);
    if (vel) s.P.vel[i] = V3(vel[3 * r], vel[3 * r + 1], vel[3 * r + 2]);
    if (angvel && s.rotmode) s.P.angvel[i] = V3(angvel[3 * r], angvel[3 * r + 1], angvel[3 * r + 2]);
    if (quat && s.rotmode) s.P.quat[i] = Q(quat[4 * r], V3(quat[4 * r + 1], quat[4 * r + 2], quat[4 * r + 3]));
    if (!s.P.alive[i]) { s.P.alive[i] = 1; revived = true; }
  }
  if (revived) search_neighbors(s);
  return 0;
}
/* The neighbour search of the next step, now (force-neutral). */
int orc_search_neighbors(void* h) {
  Sim& s = *(Sim*)h;
  s.first = false;
  search_neighbors(s);
  update_interactions(s);
  return 0;
}
/* Neighbour searches so far (the neighbour table's timestamp). */
int orc_num_rebuilds(void* h) { return ((Sim*)h)->timestamp; }
/* Tangential history of existing pairs of a RotFriction group (rows Fx, Fy, Fz, slipping,
   touching); returns the pairs written. */
int orc_set_pair_states(void* h, const char* group, int n, const int* a, const int* b, const double* st) {
  Sim& s = *(Sim*)h;
  auto it = s.dpis.find(group);
  if (it == s.dpis.end()) return -1;
  PairGroup& g = *it->second;
  if (g.kind != 1) return 0;
  std::map<std::pair<int, int>, int> row;
  for (int r = 0; r < n; ++r) row[{std::min(a[r], b[r]), std::max(a[r], b[r])}] = r;
  int done = 0;
  for (auto& f : g.fr) {
    const int i1 = s.P.id[f.p1], i2 = s.P.id[f.p2];
    auto r = row.find({std::min(i1, i2), std::max(i1, i2)});
    if (r == row.end()) continue;
    const double* v = st + 5 * r->second;
    f.Ffric = V3(v[0], v[1], v[2]);
    f.slipping = v[3] != 0.0;
    f.touching = v[4] != 0.0;
    ++done;
  }
  return done;
}
/* LsmMpi.setInteractionParameter -> forAllInteractionsSet (LatticeMaster.cpp:4290-4301,
 * pi_storage.hpp:277-292), widened to the parameters the differentiable window uses: a group's
 * unscaled parameter is replaced and every existing interaction's scaled constant is recomputed
 * with its constructor's formula (new interactions pick the new value up by themselves). */
int orc_set_group_param(void* h, const char* group, const char* key, double v) {
  Sim& s = *(Sim*)h;
  const std::string g = group, k = key;
  if ((g == "Damping" || g == "RotDamping") && k == "viscosity" && s.damping.count(g)) { s.damping[g].visc = v; return 0; }
  auto b = s.bpis.find(g);
  if (b != s.bpis.end()) {
    PairGroup& G = *b->second;
    if (k == "normalK") G.kr = v; else if (k == "shearK") G.ks = v;
    else if (k == "torsionK") G.kt = v; else if (k == "bendingK") G.kb = v;
    else { s.err = "unknown RotBond parameter " + k; return -1; }
    for (auto& bd : G.bd) {
      const double dist = std::sqrt(dot(bd.D, bd.D));
      double effR = 1.0, effL = 1.0, effA = 1.0, J = 1.0, I = 1.0;
      if (G.scaling) {
        if (G.meanR) effR = 0.5 * dist; else effR = std::fmin(s.P.rad[bd.p1], s.P.rad[bd.p2]);
        effL = dist; effA = effR * effR;
        J = 0.5 * effR * effR * effR * effR; I = 0.5 * J;
      }
      bd.kr = G.kr * effA / effL; bd.ks = G.ks * effA / effL; bd.kb = G.kb * I / effL; bd.kt = G.kt * J / effL;
    }
    return 0;
  }
  auto d = s.dpis.find(g);
  if (d != s.dpis.end()) {
    PairGroup& G = *d->second;
    if (G.kind == 0 && k == "normalK") {
      G.k = v;
      for (auto& e : G.el) e = [&] { Elastic n = make_elastic(s, G, e.p1, e.p2); n.force = e.force; n.touching = e.touching; return n; }();
      return 0;
    }
    if (G.kind == 1 && (k == "normalK" || k == "shearK")) {
      (k == "normalK" ? G.fk : G.fks) = v;
      for (auto& f : G.fr) {
        Fric n = make_fric(s, G, f.p1, f.p2);
        f.k = n.k; f.ks = n.ks;
      }
      return 0;
    }
  }
  s.err = "unknown group or parameter " + g + "." + k;
  return -1;
}
/* Wall loader: the wall moves by v*dt after every step (the constant-speed phase of
 * WallLoaderRunnable, Doc/Tutorial/examples/WallLoader.py.tex, run as a post-step hook). */
int orc_set_wall_velocity(void* h, const char* name, const double* v) {
  Sim& s = *(Sim*)h;
  auto it = s.walls.find(name);
  if (it == s.walls.end()) { s.err = "no such wall"; return -1; }
  it->second.vel = V3(v[0], v[1], v[2]);
  it->second.loader = v[0] != 0.0 || v[1] != 0.0 || v[2] != 0.0;
  return 0;
}
int orc_move_wall(void* h, const char* name, const double* d) {
  Sim& s = *(Sim*)h;
  auto it = s.walls.find(name);
  if (it == s.walls.end()) { s.err = "no such wall"; return -1; }
  it->second.o += V3(d[0], d[1], d[2]);
  return 0;
}
/* CEWallInteractionGroup::applyForce (EWallInteractionGroup.hpp:93-164), one worker */
int orc_apply_force_to_wall(void* h, const char* group, const double* fp) {
  Sim& s = *(Sim*)h;
  auto it = s.wig.find(group);
  if (it == s.wig.end()) { s.err = "no such wall group"; return -1; }
  WallGroup& wg = it->second;
  Wall& w = s.walls[wg.wall];
  V3 F(fp[0], fp[1], fp[2]);
  int iter = 0; double d, df, ef;
  V3 O_f = F / norm(F);
  do {
    double k_local = 0.0;
    for (auto& wi : wg.its) {   /* CElasticWallInteraction::getStiffness: k if touching else 0 */
      double dist = dot(s.P.pos[wi.p] - w.o, w.n);
      k_local += (dist < s.P.rad[wi.p]) ? wi.k : 0.0;
    }
    if (k_local > 0) {
      V3 F_local(0, 0, 0);
      for (auto& wi : wg.its) {
        if (!wi.inner) continue;
        double dist = dot(s.P.pos[wi.p] - w.o, w.n);
        /* CElasticWallInteraction::getForce (EWallInteraction.hpp:83-93): minus the contact force */
        V3 fc(0, 0, 0);
        if (dist < s.P.rad[wi.p]) fc = wi.k * (s.P.rad[wi.p] - dist) * w.n;
        V3 f_i = -1.0 * fc;
        F_local += dot(f_i, O_f) * O_f;
      }
      df = dot(F + F_local, O_f);
      d = df / k_local;
      ef = df / norm(F);
      w.o += d * O_f;
      iter++;
    } else {
      d = 1e-5; ef = 1;
      w.o += d * O_f;
      iter++;
    }
  } while ((iter < 50) && (ef > 1e-3));
  return 0;
}
int orc_get_wall(void* h, const char* name, double* pos, double* force) {
  Sim& s = *(Sim*)h;
  auto it = s.walls.find(name);
  if (it == s.walls.end()) { s.err = "no such wall"; return -1; }
  for (int i = 0; i < 3; ++i) { if (pos) pos[i] = it->second.o[i]; if (force) force[i] = it->second.F[i]; }
  return 0;
}
int orc_num_particles(void* h) {
  Sim& s = *(Sim*)h;
  int c = 0;
  for (int i = 0; i < s.P.n(); ++i) c += s.P.alive[i];
  return c;
}
int orc_get_particles(void* h, int* id, double* pos, double* vel, double* angvel, double* quat, double* force, double* moment) {
  Sim& s = *(Sim*)h;
  int k = 0;
  for (int i = 0; i < s.P.n(); ++i) {
    if (!s.P.alive[i]) continue;
    if (id) id[k] = s.P.id[i];
    for (int c = 0; c < 3; ++c) {
      if (pos) pos[3 * k + c] = s.P.pos[i][c];
      if (vel) vel[3 * k + c] = s.P.vel[i][c];
      if (angvel) angvel[3 * k + c] = s.P.angvel[i][c];
      if (force) force[3 * k + c] = s.P.force[i][c];
      if (moment) moment[3 * k + c] = s.P.moment[i][c];
    }
    if (quat) { quat[4 * k] = s.P.quat[i].s; for (int c = 0; c < 3; ++c) quat[4 * k + 1 + c] = s.P.quat[i].v[c]; }
    ++k;
  }
  return k;
}
/* Checker diagnostic: each alive particle's sum of the magnitudes of the forces and moments
   applied to it in the last step (the scale its summed force is compared at), in
   orc_get_particles order. */
int orc_get_gross(void* h, double* gf, double* gm) {
  Sim& s = *(Sim*)h;
  int k = 0;
  for (int i = 0; i < s.P.n(); ++i) {
    if (!s.P.alive[i]) continue;
    if (gf) gf[k] = i < (int)s.P.gross_f.size() ? s.P.gross_f[i] : 0.0;
    if (gm) gm[k] = i < (int)s.P.gross_m.size() ? s.P.gross_m[i] : 0.0;
    ++k;
  }
  return k;
}
static PairGroup* find_group(Sim& s, const char* g) {
  auto a = s.dpis.find(g); if (a != s.dpis.end()) return a->second;
  auto b = s.bpis.find(g); if (b != s.bpis.end()) return b->second;
  return nullptr;
}
int orc_num_pairs(void* h, const char* g) {
  Sim& s = *(Sim*)h;
  PairGroup* p = find_group(s, g);
  if (!p) { s.err = "no such group"; return -1; }
  return (int)(p->kind == 0 ? p->el.size() : (p->kind == 1 ? p->fr.size() : p->bd.size()));
}
int orc_get_pairs(void* h, const char* g, int* a, int* b, double* st) {
  Sim& s = *(Sim*)h;
  PairGroup* p = find_group(s, g);
  if (!p) { s.err = "no such group"; return -1; }
  int i = 0;
  if (p->kind == 0) for (auto& e : p->el) {
    a[i] = s.P.id[e.p1]; b[i] = s.P.id[e.p2];
    if (st) { for (int c = 0; c < 3; ++c) st[5 * i + c] = e.force[c]; st[5 * i + 3] = 0; st[5 * i + 4] = e.touching ? 1.0 : 0.0; }
    ++i;
  }
  else if (p->kind == 1) for (auto& f : p->fr) {
    a[i] = s.P.id[f.p1]; b[i] = s.P.id[f.p2];
    if (st) { V3 t = f.touching ? f.Ffric : V3(); for (int c = 0; c < 3; ++c) st[5 * i + c] = t[c]; st[5 * i + 3] = f.slipping ? 1.0 : 0.0; st[5 * i + 4] = f.touching ? 1.0 : 0.0; }
    ++i;
  }
  else for (auto& d : p->bd) {
    a[i] = s.P.id[d.p1]; b[i] = s.P.id[d.p2];
    if (st) { for (int c = 0; c < 3; ++c) st[5 * i + c] = d.force[c]; st[5 * i + 3] = d.nF / d.max_n + d.shF / d.max_s + d.tM / d.max_t + d.bM / d.max_b; st[5 * i + 4] = 0; }
    ++i;
  }
  return i;
}
int orc_num_breaks(void* h) { return (int)((Sim*)h)->brk1.size(); }
int orc_get_breaks(void* h, int* a, int* b, int* st) {
  Sim& s = *(Sim*)h;
  for (size_t i = 0; i < s.brk1.size(); ++i) { a[i] = s.brk1[i]; b[i] = s.brk2[i]; st[i] = s.brkstep[i]; }
  return (int)s.brk1.size();
}
int orc_move_tagged(void* h, int tag, int mask, const double* d) {
  (void)mask;
  Sim& s = *(Sim*)h;
  for (int i = 0; i < s.P.n(); ++i) if (s.P.alive[i] && s.P.tag[i] == tag) s.P.pos[i] += V3(d[0], d[1], d[2]);
  return 0;
}
long long orc_timestep(void* h) { return ((Sim*)h)->t; }
}

/* ==== Forward-mode dual-number window ==========================================
 * Checker of the differentiable window: the step above restated on FP64 dual
 * numbers (a value and kSeeds tangents) over a window of steps with the
 * interaction lists, wall candidates and bond set frozen, as the GPU window
 * freezes them.  Seeded on group parameters or initial velocities, it gives the
 * exact derivative of every wall-group reaction along the branch the values
 * take.  The primal arithmetic is the FP64 restatement's, operation by
 * operation, so the values equal orc_step's.  Each law cites the same reference
 * lines as its FP64 form above.
 */
namespace orc {
namespace dual {

constexpr int kSeeds = 8;

struct Du {
  double v = 0.0;
  double d[kSeeds] = {};
  Du() {}
  Du(double x) : v(x) {}
};
static inline Du operator+(const Du& a, const Du& b) { Du r(a.v + b.v); for (int k = 0; k < kSeeds; ++k) r.d[k] = a.d[k] + b.d[k]; return r; }
static inline Du operator-(const Du& a, const Du& b) { Du r(a.v - b.v); for (int k = 0; k < kSeeds; ++k) r.d[k] = a.d[k] - b.d[k]; return r; }
static inline Du operator-(const Du& a) { Du r(-a.v); for (int k = 0; k < kSeeds; ++k) r.d[k] = -a.d[k]; return r; }
static inline Du operator*(const Du& a, const Du& b) {
  Du r(a.v * b.v);
  for (int k = 0; k < kSeeds; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
static inline Du operator/(const Du& a, const Du& b) {
  Du r(a.v / b.v);
  for (int k = 0; k < kSeeds; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
  return r;
}
static inline Du& operator+=(Du& a, const Du& b) { a = a + b; return a; }
static inline bool operator<(const Du& a, const Du& b) { return a.v < b.v; }
static inline bool operator>(const Du& a, const Du& b) { return a.v > b.v; }
static inline bool operator<=(const Du& a, const Du& b) { return a.v <= b.v; }
static inline bool operator>=(const Du& a, const Du& b) { return a.v >= b.v; }
static inline bool operator==(const Du& a, const Du& b) { return a.v == b.v; }
static inline bool operator!=(const Du& a, const Du& b) { return a.v != b.v; }
static inline Du dsqrt(const Du& a) {
  Du r(std::sqrt(a.v));
  const double g = r.v > 0.0 ? 0.5 / r.v : 0.0;
  for (int k = 0; k < kSeeds; ++k) r.d[k] = a.d[k] * g;
  return r;
}
static inline Du dacos(const Du& a) {
  Du r(std::acos(a.v));
  const double g = -1.0 / std::sqrt(1.0 - a.v * a.v);
  for (int k = 0; k < kSeeds; ++k) r.d[k] = a.d[k] * g;
  return r;
}

/* vec3.hpp / Quaternion.hpp / Matrix3.hpp on dual scalars (same operation order as V3, Q, M3) */
struct DV {
  Du x, y, z;
  DV() {}
  DV(const Du& a, const Du& b, const Du& c) : x(a), y(b), z(c) {}
  explicit DV(const V3& a) : x(a.x), y(a.y), z(a.z) {}
};
static inline DV operator+(const DV& a, const DV& b) { return DV(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline DV operator-(const DV& a, const DV& b) { return DV(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline DV operator-(const DV& a) { return DV(-a.x, -a.y, -a.z); }
static inline DV operator*(const DV& a, const Du& s) { return DV(a.x * s, a.y * s, a.z * s); }
static inline DV operator*(const Du& f, const DV& a) { return DV(f * a.x, f * a.y, f * a.z); }
static inline DV operator/(const DV& a, const Du& s) { return DV(a.x / s, a.y / s, a.z / s); }
static inline DV& operator+=(DV& a, const DV& b) { a.x = a.x + b.x; a.y = a.y + b.y; a.z = a.z + b.z; return a; }
static inline DV& operator-=(DV& a, const DV& b) { a.x = a.x - b.x; a.y = a.y - b.y; a.z = a.z - b.z; return a; }
static inline Du ddot(const DV& a, const DV& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline DV dcross(const DV& l, const DV& r) {
  return DV(l.y * r.z - l.z * r.y, l.z * r.x - l.x * r.z, l.x * r.y - l.y * r.x);
}
static inline Du dnorm2(const DV& a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static inline Du dnorm(const DV& a) { return dsqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
struct DQ { Du s = 1.0; DV v; DQ() {} DQ(const Du& a, const DV& b) : s(a), v(b) {} };
static inline DQ dqmul(const DQ& a, const DQ& b) {
  return DQ(a.s * b.s - ddot(a.v, b.v), a.s * b.v + b.s * a.v + dcross(a.v, b.v));
}
static inline DQ dqinv(const DQ& a) { return DQ(a.s, -a.v); }
struct DM { Du m[3][3]; };
static inline DM dto_matrix(const DQ& q) {
  DM r; const Du s = q.s, x = q.v.x, y = q.v.y, z = q.v.z;
  r.m[0][0] = s * s + x * x - y * y - z * z;
  r.m[0][1] = 2.0 * (x * y + s * z);
  r.m[0][2] = 2.0 * (x * z - s * y);
  r.m[1][0] = 2.0 * (x * y - s * z);
  r.m[1][1] = s * s - x * x + y * y - z * z;
  r.m[1][2] = 2.0 * (y * z + s * x);
  r.m[2][0] = 2.0 * (x * z + s * y);
  r.m[2][1] = 2.0 * (y * z - s * x);
  r.m[2][2] = s * s - x * x - y * y + z * z;
  return r;
}
static inline DM dtrans(const DM& a) { DM r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[j][i]; return r; }
static inline DV dmul(const DM& a, const DV& v) {
  return DV(a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z,
            a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
            a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z);
}

struct DState {
  std::vector<DV> pos, vel, angvel, force, moment;
  std::vector<DQ> quat;
};

struct Params {  /* seeded group parameters */
  std::map<std::string, Du> k, ks, kt, kb;   /* per group: normalK, shearK, torsionK, bendingK */
  Du visc_lin, visc_rot;
};

static DV dimage_of(const Sim& s, const DV& p1, DV p2) {
  if (s.circx) {
    const double dx = p1.x.v - p2.x.v;
    if (dx > 0.5 * s.Lx) p2.x = p2.x + s.Lx;
    else if (dx < -0.5 * s.Lx) p2.x = p2.x - s.Lx;
  }
  return p2;
}

/* CElasticInteraction ctor scaling + calcForces (Model/ElasticInteraction.cpp:25-71) */
static void d_elastic(const Sim& s, const PairGroup& g, const Elastic& e, const Du& k, DState& st) {
  double effR = 1.0, effA = 1.0, effL = 1.0;
  const double r0 = s.P.rad[e.p1] + s.P.rad[e.p2];
  if (g.scaling) { effR = 0.5 * r0; effL = r0; effA = effR * effR; }
  const Du keff = k * effA / effL;
  const DV x1 = st.pos[e.p1], x2 = dimage_of(s, x1, st.pos[e.p2]);
  DV D = x1 - x2;
  Du dist = ddot(D, D);
  const double eq_dist = r0;
  if (dist < (eq_dist * eq_dist)) {
    dist = dsqrt(dist);
    DV F = D * (keff * (dist - eq_dist) / dist);
    st.force[e.p2] += F;
    st.force[e.p1] += -1.0 * F;
  }
}

struct DFric { DV Ffric; bool slipping, touching; };

/* CRotFrictionInteraction ctor scaling + calcSimpleForces (Model/RotFricInteraction.cpp:103-231) */
static void d_fric(const Sim& s, const PairGroup& g, const Fric& f0, DFric& f, const Du& k, const Du& ks, DState& st) {
  double effR = 1.0, effL = 1.0, effA = 1.0;
  const double r1 = s.P.rad[f0.p1], r2 = s.P.rad[f0.p2];
  const double r0 = r1 + r2;
  if (g.scaling) {
    if (g.meanR) effR = 0.5 * r0; else effR = std::fmin(r1, r2);
    effL = r0; effA = effR * effR;
  }
  const Du fk = k * effA / effL, fks = ks * effA / effL;
  const double mu_current = f.slipping ? f0.mu_d : f0.mu_s;
  const DV x1 = st.pos[f0.p1], x2 = dimage_of(s, x1, st.pos[f0.p2]);
  const DV D = x1 - x2;
  Du dist = ddot(D, D);
  const double eq_dist = r1 + r2;
  if (dist < (eq_dist * eq_dist)) {
    dist = dsqrt(dist);
    const DV force(D * (fk * (dist - eq_dist) / dist));
    const DV pos(x2 + (r2 / eq_dist) * D);
    st.force[f0.p2] += force;
    st.force[f0.p1] += -1.0 * force;
    const DV vp1 = st.vel[f0.p1] + dcross(st.angvel[f0.p1], pos - x1);
    const DV vp2 = st.vel[f0.p2] + dcross(st.angvel[f0.p2], pos - x2);
    DV ds((vp2 - vp1) * f0.dt);
    ds -= ((ddot(ds, D)) / (dnorm2(D))) * D;
    f.Ffric += fks * ds;
    const Du FfricNorm = dnorm(f.Ffric);
    const Du forceNorm = dnorm(force);
    if (FfricNorm > forceNorm * mu_current) {
      f.Ffric = f.Ffric * ((f0.mu_d * forceNorm) / FfricNorm);
      f.slipping = true;
    } else {
      f.slipping = false;
    }
    const DV Moment1(dcross(pos - x1, f.Ffric));
    const DV Moment2(dcross(pos - x2, -f.Ffric));
    st.moment[f0.p1] += Moment1;
    st.moment[f0.p2] += Moment2;
    st.force[f0.p1] += f.Ffric;
    st.force[f0.p2] += -1.0 * f.Ffric;
    f.touching = true;
  } else {
    f.Ffric = DV(V3(0, 0, 0));
    f.slipping = false;
    f.touching = false;
  }
}

static Du d_calc_angle(const Du& s_in, const Du& c_os) {   /* ARotBondedInteraction.cpp:22-51 */
  if (s_in > 0.0) return (c_os >= 1.0 || c_os <= -1.0) ? Du(0.0) : dacos(c_os);
  if (s_in == 0.0) return Du(0.0);
  return (c_os >= 1.0 || c_os <= -1.0) ? Du(0.0) : -dacos(c_os);
}

/* Bond ctor scaling (RotBondedInteraction.cpp:122-161) + ARotBondedInteraction::calcForces
 * (ARotBondedInteraction.cpp:307-448) + CRotBondedInteraction::broken (:175-219).
 * Returns true when the bond would break. */
static bool d_bond(const Sim& s, const PairGroup& g, const Bond& b, const Du& gkr, const Du& gks, const Du& gkt,
                   const Du& gkb, DState& st) {
  const double dist0 = std::sqrt(dot(b.D, b.D));
  double effR = 1.0, effL = 1.0, effA = 1.0, J = 1.0, I = 1.0;
  if (g.scaling) {
    if (g.meanR) effR = 0.5 * dist0; else effR = std::fmin(s.P.rad[b.p1], s.P.rad[b.p2]);
    effL = dist0; effA = effR * effR;
    J = 0.5 * effR * effR * effR * effR; I = 0.5 * J;
  }
  const Du kr = gkr * effA / effL, ks = gks * effA / effL, kb = gkb * I / effL, kt = gkt * J / effL;
  const double HALF_SQRT_2 = 0.5 * std::sqrt(2.0);
  Du s_fai = 0.0, c_fai = 0.0, c_pasi2 = 0.0, s_pasi2 = 0.0, sita = 0.0, pasi = 0.0;
  const DQ q1 = st.quat[b.p1], q2 = st.quat[b.p2];
  const DV x1 = st.pos[b.p1], x2 = dimage_of(s, x1, st.pos[b.p2]);
  const double r1 = s.P.rad[b.p1], r2 = s.P.rad[b.p2];
  const DV mD(b.D);
  const DM mat0 = dto_matrix(q1);
  const DV rbp = x2 - x1;
  const Du rbpNorm = dnorm(rbp);
  const DV rb = dmul(mat0, x2 - x1);
  const Du rbNorm = dnorm(rb);
  const double r_0Norm = r1 + r2;
  const DV delta_r = (rbNorm - r_0Norm) * rb / rbNorm;
  const DV Fr = kr * delta_r;
  const Du gama_cos = ddot(rb, mD) / (rbNorm * dnorm(mD));
  Du gama = 0.0;
  if (gama_cos < 1.0 && gama_cos > -1.0) gama = dacos(gama_cos);
  const DV rb_0 = dcross(rb, mD);
  const DV rb_b0 = dcross(rb, rb_0);
  const Du rb_b0Norm = dnorm(rb_b0);
  DV Fst(V3(0, 0, 0));
  if (rb_b0Norm != 0.0) Fst = ks * r_0Norm * gama * rb_b0 / rb_b0Norm;
  DV Mst(V3(0, 0, 0));
  const Du rb_0Norm = dnorm(rb_0);
  if (rb_0Norm != 0.0) Mst = -dnorm(Fst) * rb_0 / rb_0Norm;
  const Du m0 = HALF_SQRT_2 * dsqrt((rbNorm + rb.z) / rbNorm);
  Du m1 = -HALF_SQRT_2 * dsqrt((rbNorm - rb.z) / rbNorm);
  Du m2 = -m1;
  const Du m3 = 0.0;
  const Du rbX2PlusRbY2 = rb.x * rb.x + rb.y * rb.y;
  if (rbX2PlusRbY2 != 0.0) {
    const Du denomSqrt = dsqrt(rbX2PlusRbY2);
    m1 = m1 * rb.y / denomSqrt;
    m2 = m2 * rb.x / denomSqrt;
  }
  const DQ qm(m0, DV(m1, m2, m3));
  const DM mat = dto_matrix(qm);
  const DM matTrans = dtrans(mat);
  const DQ rp = dqmul(dqinv(q1), q2);
  const DQ r = dqmul(dqmul(dqinv(qm), rp), qm);
  const Du temp0 = r.s * r.s + r.v.z * r.v.z;
  if (temp0 == 0.0) {
    pasi = 0.0;
  } else {
    const Du sqrtTemp0 = dsqrt(temp0);
    c_pasi2 = r.s / sqrtTemp0;
    s_pasi2 = r.v.z / sqrtTemp0;
    pasi = 2.0 * d_calc_angle(s_pasi2, c_pasi2);
  }
  const DV Mtp(Du(0.0), Du(0.0), kt * pasi);
  const DV Mtr = dmul(matTrans, Mtp);
  const Du temp2 = r.v.x * r.v.x + r.v.y * r.v.y;
  const Du temp3 = r.v.x * r.v.z + r.s * r.v.y;
  const Du temp4 = r.v.y * r.v.z - r.s * r.v.x;
  DV Mbr(V3(0, 0, 0)), Fsr(V3(0, 0, 0)), Msr(V3(0, 0, 0));
  if (temp2 != 0.0) {
    const Du temp1 = temp0 - temp2;
    if (temp1 >= 1.0 || temp1 <= -1.0) sita = 0.0; else sita = dacos(temp1);
    if (temp0 == 0.0) {
      const Du sqrtDenom = dsqrt(temp2);
      c_fai = r.v.y / sqrtDenom;
      s_fai = -r.v.x / sqrtDenom;
    } else {
      const Du sqrtDenom = dsqrt(temp0 * temp2);
      c_fai = temp3 / sqrtDenom;
      s_fai = temp4 / sqrtDenom;
    }
    const DV Mbp(-0.5 * kb * sita * s_fai, 0.5 * kb * sita * c_fai, Du(0.0));
    Mbr = dmul(matTrans, Mbp);
    const DV Fsp(-0.5 * ks * c_fai * sita * r_0Norm, -0.5 * ks * s_fai * sita * r_0Norm, Du(0.0));
    Fsr = dmul(matTrans, Fsp);
    const DV Msp(0.5 * ks * s_fai * sita * r_0Norm, -0.5 * ks * c_fai * sita * r_0Norm, Du(0.0));
    Msr = dmul(matTrans, Msp);
  }
  const double eq_rad1 = r1 / (r1 + r2);
  const double eq_rad2 = r2 / (r1 + r2);
  const DM mat0Trans = dtrans(mat0);
  const DV force = dmul(mat0Trans, Fr + Fst + Fsr);
  const DV moment = dmul(mat0Trans, Mbr + Mtr + Msr * eq_rad1 * rbpNorm + Mst * eq_rad1 * rbpNorm);
  const DV moment2 = dmul(mat0Trans, Msr * eq_rad2 * rbpNorm + Mst * eq_rad2 * rbpNorm - Mbr - Mtr);
  const double shF = dnorm(Fst + Fsr).v, tM = dnorm(Mtr).v, bM = dnorm(Mbr).v;
  const double r0 = r1 + r2;
  const DV D = x1 - x2;
  const double dist = std::sqrt(ddot(D, D).v);
  const double nF = ((dist < r0) ? -1.0 : 1.0) * dnorm(Fr).v;
  st.force[b.p2] += -1.0 * force;
  st.force[b.p1] += force;
  st.moment[b.p1] += moment;
  st.moment[b.p2] += moment2;
  const double shearStress = shF / b.max_s + b.beta2 * tM / b.max_t;
  const double normalStress = nF / b.max_n + b.beta1 * bM / b.max_b;
  return (normalStress > b.truncated) || (shearStress > (1.0 - normalStress));
}

/* CDamping / CRotDamping::calcForces (Model/Damping.hpp:99-124, Model/RotDamping.hpp:58-84), vref = 0 */
static DV d_damping(const DV& v, const DV& frc, const Du& sm, const Du& mass, const Du& visc, double dt, int maxiter) {
  const double s_limit2 = 1e-12;
  DV v_rel(V3(0, 0, 0));
  double error = 1.0;
  int count = 0;
  while ((error * error > s_limit2) & (count < maxiter)) {
    count++;
    DV v_old = v_rel;
    v_rel = v + sm * dt * (frc - v_rel * visc * mass);
    error = dnorm2(v_rel - v_old).v;
  }
  if (count >= maxiter) v_rel = DV(V3(0, 0, 0));
  return -1.0 * visc * v_rel * mass;
}

}  // namespace dual
}  // namespace orc

extern "C" {

/* Dual-number window of nsteps steps from the current state.  seeds[k] names the k-th tangent:
 * "param:<group>:<key>" (RotBond normalK / shearK / torsionK / bendingK, dynamic-group normalK /
 * shearK, "Damping" or "RotDamping" viscosity), "vel:<id>:<c>", "angvel:<id>:<c>" or
 * "pos:<id>:<c>".  R[nsteps][wall groups][3] receives the reaction of each wall group (name
 * order) after each step, dR[nsteps][wall groups][3][nseed] its derivatives.  The simulation
 * itself is not advanced (only the head of its next step, the pending neighbour search and
 * interaction update, is done).  A bond failure inside the window is followed as the reference
 * handles it (erase, flags, new list to the RotFriction groups, wall candidates refreshed); the
 * derivatives are those of the branch taken.  Returns -5 if a rebuild falls inside the window
 * or a failure would feed new-list pairs to an elastic group. */
int orc_window_dual(void* h, int nsteps, int nseed, const char* const* seeds, double* R, double* dR) {
  using namespace orc::dual;
  Sim& s = *(Sim*)h;
  if (nsteps < 1 || nseed < 0 || nseed > kSeeds) { s.err = "bad window size or seed count"; return -1; }
  if (s.first) { search_neighbors(s); s.first = false; }
  if (check_neighbors(s)) search_neighbors(s);
  update_interactions(s);
  const int n = s.P.n();
  DState st;
  st.pos.resize(n); st.vel.resize(n); st.angvel.resize(n); st.force.resize(n); st.moment.resize(n); st.quat.resize(n);
  for (int i = 0; i < n; ++i) {
    st.pos[i] = DV(s.P.pos[i]); st.vel[i] = DV(s.P.vel[i]); st.angvel[i] = DV(s.P.angvel[i]);
    st.quat[i] = DQ(Du(s.P.quat[i].s), DV(s.P.quat[i].v));
  }
  Params prm;
  for (auto& b : s.bpis) { prm.k[b.first] = b.second->kr; prm.ks[b.first] = b.second->ks; prm.kt[b.first] = b.second->kt; prm.kb[b.first] = b.second->kb; }
  for (auto& d : s.dpis) {
    if (d.second->kind == 0) prm.k[d.first] = d.second->k;
    else { prm.k[d.first] = d.second->fk; prm.ks[d.first] = d.second->fks; }
  }
  if (s.damping.count("Damping")) prm.visc_lin = s.damping["Damping"].visc;
  if (s.damping.count("RotDamping")) prm.visc_rot = s.damping["RotDamping"].visc;
  for (int k = 0; k < nseed; ++k) {
    std::string sd = seeds[k];
    size_t a = sd.find(':'), b = sd.rfind(':');
    if (a == std::string::npos || b == a) { s.err = "bad seed " + sd; return -1; }
    std::string kind = sd.substr(0, a), mid = sd.substr(a + 1, b - a - 1), last = sd.substr(b + 1);
    if (kind == "param") {
      Du* p = nullptr;
      if ((mid == "Damping" || mid == "RotDamping") && last == "viscosity") p = mid == "Damping" ? &prm.visc_lin : &prm.visc_rot;
      else if (last == "normalK" && prm.k.count(mid)) p = &prm.k[mid];
      else if (last == "shearK" && prm.ks.count(mid)) p = &prm.ks[mid];
      else if (last == "torsionK" && prm.kt.count(mid)) p = &prm.kt[mid];
      else if (last == "bendingK" && prm.kb.count(mid)) p = &prm.kb[mid];
      if (!p) { s.err = "unknown parameter seed " + sd; return -1; }
      p->d[k] = 1.0;
    } else {
      auto it = s.id2slot.find(std::atoi(mid.c_str()));
      const int c = std::atoi(last.c_str());
      if (it == s.id2slot.end() || c < 0 || c > 2) { s.err = "bad particle seed " + sd; return -1; }
      DV* v = kind == "vel" ? &st.vel[it->second] : kind == "angvel" ? &st.angvel[it->second]
                             : kind == "pos" ? &st.pos[it->second] : nullptr;
      if (!v) { s.err = "bad seed kind " + sd; return -1; }
      (c == 0 ? v->x : c == 1 ? v->y : v->z).d[k] = 1.0;
    }
  }
  std::map<std::string, std::vector<DFric>> hist;
  for (auto& d : s.dpis)
    if (d.second->kind == 1)
      for (auto& f : d.second->fr) hist[d.first].push_back(DFric{DV(f.Ffric), f.slipping, f.touching});
  std::map<std::string, V3> wo;
  for (auto& w : s.walls) wo[w.first] = w.second.o;
  const int ng = (int)s.wig.size();
  const double half = 0.5 * s.alpha, srsqr = half * half;
  /* Bond failures inside the window are taken as the forward's events: the failed bond leaves
   * its storage at the head of the next step and the "new list" of pairs between flagged
   * particles joins the dynamic groups (TSubLattice::updateInteractions, SubLattice.hpp:2416-2466),
   * all held in window-local copies so the simulation itself is left as it was. */
  std::map<std::string, std::vector<char>> gone;        /* bond erased inside the window */
  std::map<std::string, std::vector<int>> failed;       /* bonds that failed in the last step */
  std::map<std::string, std::vector<Fric>> extra;       /* new-list pairs appended inside the window */
  std::set<std::pair<int, int>> released, added;        /* failed bonds' ids; appended pairs' ids */
  std::map<std::string, std::vector<WallI>> wits;       /* wall candidates, refreshed after a failure */
  for (auto& b : s.bpis) gone[b.first].assign(b.second->bd.size(), 0);
  for (auto& wg : s.wig) wits[wg.first] = wg.second.its;
  for (int j = 0; j < nsteps; ++j) {
    if (j > 0) {  /* checkNeighbors at the head of step j: a rebuild would unfreeze the topology */
      double mdsqr = 0;
      for (int i = 0; i < n && mdsqr < srsqr; ++i) {
        if (!s.P.alive[i]) continue;
        V3 d(st.pos[i].x.v - s.P.oldpos[i].x, st.pos[i].y.v - s.P.oldpos[i].y, st.pos[i].z.v - s.P.oldpos[i].z);
        double sq = dot(d, d);
        mdsqr = (mdsqr < sq) ? sq : mdsqr;
      }
      if (mdsqr > srsqr) { s.err = "a neighbour rebuild falls inside the window"; return -5; }
    }
    bool changed = false;
    for (auto& f : failed) {   /* PIS_EB::update (pi_storage_eb.hpp:23-49) */
      for (int q : f.second) {
        const Bond& b = s.bpis[f.first]->bd[q];
        gone[f.first][q] = 1;
        released.insert({s.P.id[b.p1], s.P.id[b.p2]});
        s.P.flag[b.p1] = 1;
        s.P.flag[b.p2] = 1;
        changed = true;
      }
      f.second.clear();
    }
    if (changed) {
      for (auto& d : s.dpis) {   /* PIS_ED::update without a rebuild: the new list (pi_storage_ed.hpp:84-161) */
        const std::vector<std::pair<int, int>> pl = new_list(s);
        for (auto& p : pl) {
          const int a = s.P.id[p.first], b = s.P.id[p.second];
          bool excl = false;
          for (auto* e : d.second->exig) excl = excl || (e->idset.count({a, b}) && !released.count({a, b}));
          if (excl || d.second->idset.count({a, b}) || added.count({a, b})) continue;
          if (d.second->kind != 1) { s.err = "a bond failure inside the window feeds an elastic group"; return -5; }
          extra[d.first].push_back(make_fric(s, *d.second, p.first, p.second));
          hist[d.first].push_back(DFric{DV(V3(0, 0, 0)), false, false});
          added.insert({a, b});
        }
      }
      for (auto& wg : s.wig) {   /* CEWallInteractionGroup::Update at the current positions */
        std::vector<WallI>& its = wits[wg.first];
        its.clear();
        const Wall& w = s.walls[wg.second.wall];
        const V3 o = wo[wg.second.wall];
        for (int i = 0; i < n; ++i) {
          if (!s.P.alive[i]) continue;
          const V3 x(st.pos[i].x.v, st.pos[i].y.v, st.pos[i].z.v);
          if (std::fabs(dot(x - o, w.n)) < s.nrange) {
            double f = 1.0;
            f *= 3.141592654 * s.P.rad[i];
            its.push_back(WallI{i, f * wg.second.k, is_inner(s, x)});
          }
        }
      }
    }
    for (int i = 0; i < n; ++i) { st.force[i] = DV(V3(0, 0, 0)); st.moment[i] = DV(V3(0, 0, 0)); }
    int gi = 0;
    for (auto& wg : s.wig) {   /* walls (EWallInteraction.hpp:42-78), reaction per group */
      const Wall& w = s.walls[wg.second.wall];
      const DV o(wo[wg.second.wall]), nn(w.n);
      DV acc(V3(0, 0, 0));
      for (auto& wi : wits[wg.first]) {
        const Du dist = ddot(st.pos[wi.p] - o, nn);
        const double r = s.P.rad[wi.p];
        if (dist < r) {
          const DV force = Du(wi.k) * (r - dist) * nn;
          st.force[wi.p] += force;
          if (wi.inner) acc -= -1.0 * force;
        }
      }
      for (int c = 0; c < 3; ++c) {
        const Du& v = c == 0 ? acc.x : c == 1 ? acc.y : acc.z;
        const size_t o3 = ((size_t)j * ng + gi) * 3 + c;
        R[o3] = v.v;
        for (int k = 0; k < nseed; ++k) dR[o3 * nseed + k] = v.d[k];
      }
      ++gi;
    }
    for (auto& g : s.gravity)
      for (int i = 0; i < n; ++i) if (s.P.alive[i]) st.force[i] += DV(g.second) * Du(s.P.mass[i]);
    for (auto& d : s.dpis) {
      if (d.second->kind == 0) {
        for (auto& e : d.second->el) d_elastic(s, *d.second, e, prm.k[d.first], st);
      } else {
        auto& hv = hist[d.first];
        const size_t m0 = d.second->fr.size();
        for (size_t q = 0; q < m0; ++q)
          d_fric(s, *d.second, d.second->fr[q], hv[q], prm.k[d.first], prm.ks[d.first], st);
        auto ex = extra.find(d.first);
        if (ex != extra.end())
          for (size_t q = 0; q < ex->second.size(); ++q)
            d_fric(s, *d.second, ex->second[q], hv[m0 + q], prm.k[d.first], prm.ks[d.first], st);
      }
    }
    for (auto& b : s.bpis) {
      const std::vector<char>& gb = gone[b.first];
      for (size_t q = 0; q < b.second->bd.size(); ++q)
        if (!gb[q] && d_bond(s, *b.second, b.second->bd[q], prm.k[b.first], prm.ks[b.first], prm.kt[b.first],
                             prm.kb[b.first], st))
          failed[b.first].push_back((int)q);
    }
    for (auto& d : s.damping) {
      if (d.first == "Damping") {
        for (int i : s.damp_list)
          st.force[i] += d_damping(st.vel[i], st.force[i], Du(s.P.invmass[i]), Du(s.P.mass[i]), prm.visc_lin,
                                   d.second.dt, d.second.maxiter);
      } else {
        for (int i : s.damp_list)
          st.moment[i] += d_damping(st.angvel[i], st.moment[i], Du(1.0 / s.P.inert[i]), Du(s.P.inert[i]),
                                    prm.visc_rot, d.second.dt, d.second.maxiter);
      }
    }
    const double dt = s.dt;
    for (int i = 0; i < n; ++i) {   /* integrate (Particle.cpp:257-274, RotParticle.cpp:277-293) */
      if (!s.P.alive[i]) continue;
      if (s.rotmode) {
        if (s.P.rot[i]) {
          st.angvel[i] += Du(dt * s.P.invinert[i]) * st.moment[i];
          const DQ w(Du(0.0), st.angvel[i]);
          const DQ dq = dqmul(w, st.quat[i]);
          const double c = dt / 2.0;
          st.quat[i].s = st.quat[i].s + c * dq.s;
          st.quat[i].v += Du(c) * dq.v;
        } else {
          st.angvel[i] = DV(V3(0, 0, 0));
        }
      }
      if (s.P.dyn[i]) {
        st.vel[i] += st.force[i] * Du(s.P.invmass[i]) * Du(dt);
        st.pos[i] += st.vel[i] * Du(dt);
      }
    }
    if (s.rotmode)   /* rescale (RotParticle.cpp:305-321) */
      for (int i = 0; i < n; ++i) {
        if (!s.P.alive[i]) continue;
        DQ& q = st.quat[i];
        const Du module = dsqrt(q.s * q.s + q.v.x * q.v.x + q.v.y * q.v.y + q.v.z * q.v.z);
        if (module != 0.0) {
          const Du inverse = Du(1.0) / module;
          q = DQ(inverse * q.s, inverse * q.v);
        }
      }
    for (auto& w : s.walls)   /* wall loaders move after the step */
      if (w.second.loader) {
        V3& o = wo[w.first];
        o.x += w.second.vel.x * dt;
        o.y += w.second.vel.y * dt;
        o.z += w.second.vel.z * dt;
      }
  }
  return 0;
}

}  // extern "C"
