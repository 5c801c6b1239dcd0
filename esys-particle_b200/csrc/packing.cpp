// Seeded random sequential insertion (RSI) of spheres into a box, used to
// generate the synthetic input packings of the benchmarks and tests.
//
// Plays the role of the reference's set-up packers (Geometry/RandomBoxPacker.hpp);
// the algorithm is plain RSI: radii are drawn first and inserted largest
// first, each at up to max_attempts uniform random centres, rejected on any
// overlap (|d| < r1 + r2, minimum image in x when periodic).  Host code only.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <random>
#include <vector>

#include "../../include/esys_geometry.h"

extern "C" int lsm_pack_rsi(unsigned long long seed, int n, const double* bmin, const double* bmax, int periodic_x,
                            int dist, double p0, double p1, double rmin, double rmax, int max_attempts,
                            double* pos, double* rad) {
  if (n <= 0 || !bmin || !bmax || !pos || !rad || !(rmax >= rmin) || !(rmin > 0)) return -1;
  std::mt19937_64 rng(seed);
  std::vector<double> r(n);
  if (dist == 0) {  // uniform in [p0, p1]
    std::uniform_real_distribution<double> u(p0, p1);
    for (auto& x : r) x = std::min(std::max(u(rng), rmin), rmax);
  } else {          // lognormal with median p0 and log-sigma p1
    std::normal_distribution<double> g(std::log(p0), p1);
    for (auto& x : r) x = std::min(std::max(std::exp(g(rng)), rmin), rmax);
  }
  std::sort(r.begin(), r.end(), [](double a, double b) { return a > b; });
  const double L[3] = {bmax[0] - bmin[0], bmax[1] - bmin[1], bmax[2] - bmin[2]};
  const double cs = 2.0 * rmax;
  int nc[3];
  for (int k = 0; k < 3; ++k) nc[k] = std::max(1, (int)std::floor(L[k] / cs));
  const double cl[3] = {L[0] / nc[0], L[1] / nc[1], L[2] / nc[2]};
  std::vector<std::vector<int>> cells((size_t)nc[0] * nc[1] * nc[2]);
  std::uniform_real_distribution<double> u01(0.0, 1.0);
  int placed = 0;
  for (int i = 0; i < n; ++i) {
    const double ri = r[i];
    bool ok = false;
    double c[3];
    for (int a = 0; a < max_attempts && !ok; ++a) {
      c[0] = periodic_x ? bmin[0] + u01(rng) * L[0] : bmin[0] + ri + u01(rng) * (L[0] - 2 * ri);
      c[1] = bmin[1] + ri + u01(rng) * (L[1] - 2 * ri);
      c[2] = bmin[2] + ri + u01(rng) * (L[2] - 2 * ri);
      int ic[3];
      for (int k = 0; k < 3; ++k) ic[k] = std::min(nc[k] - 1, std::max(0, (int)((c[k] - bmin[k]) / cl[k])));
      ok = true;
      for (int dx = -1; dx <= 1 && ok; ++dx)
        for (int dy = -1; dy <= 1 && ok; ++dy)
          for (int dz = -1; dz <= 1 && ok; ++dz) {
            int jx = ic[0] + dx, jy = ic[1] + dy, jz = ic[2] + dz;
            if (periodic_x) jx = (jx + nc[0]) % nc[0];
            else if (jx < 0 || jx >= nc[0]) continue;
            if (jy < 0 || jy >= nc[1] || jz < 0 || jz >= nc[2]) continue;
            if (periodic_x && nc[0] < 3 && dx != 0) continue;
            for (int j : cells[((size_t)jx * nc[1] + jy) * nc[2] + jz]) {
              double d0 = c[0] - pos[3 * j], d1 = c[1] - pos[3 * j + 1], d2 = c[2] - pos[3 * j + 2];
              if (periodic_x) { if (d0 > 0.5 * L[0]) d0 -= L[0]; else if (d0 < -0.5 * L[0]) d0 += L[0]; }
              const double rr = ri + rad[j];
              if (d0 * d0 + d1 * d1 + d2 * d2 < rr * rr) { ok = false; break; }
            }
          }
    }
    if (!ok) continue;
    pos[3 * placed] = c[0]; pos[3 * placed + 1] = c[1]; pos[3 * placed + 2] = c[2];
    rad[placed] = ri;
    int ic[3];
    for (int k = 0; k < 3; ++k) ic[k] = std::min(nc[k] - 1, std::max(0, (int)((c[k] - bmin[k]) / cl[k])));
    cells[((size_t)ic[0] * nc[1] + ic[1]) * nc[2] + ic[2]].push_back(placed);
    ++placed;
  }
  return placed;
}

// ---- fitting packer -------------------------------------------------------
// Dense random packing by gap filling, in the manner of the reference's
// RandomBoxPacker (Geometry/RandomBoxPacker.hpp: a seed packing, then
// FittedParticleIterator::generateNext inserting spheres that touch their
// closest neighbours and, near the box, a face).  Each trial takes a uniform
// random point, its four nearest spheres (by surface distance) and the nearest
// box face, and solves for the sphere tangent to the four spheres, or to three
// of them and the face; it is kept when its radius lies in [rmin, rmax], it
// stays inside the box and it overlaps nothing.  Filling stops after
// max_failures consecutive rejected trials or at n spheres.
namespace {

struct FitGrid {
  double bmin[3], L[3], cl[3];
  int nc[3];
  std::vector<std::vector<int>> cells;
  FitGrid(const double* mn, const double* mx, double cs) {
    for (int k = 0; k < 3; ++k) {
      bmin[k] = mn[k];
      L[k] = mx[k] - mn[k];
      nc[k] = std::max(1, (int)std::floor(L[k] / cs));
      cl[k] = L[k] / nc[k];
    }
    cells.resize((size_t)nc[0] * nc[1] * nc[2]);
  }
  void cell_of(const double* c, int* ic) const {
    for (int k = 0; k < 3; ++k) ic[k] = std::min(nc[k] - 1, std::max(0, (int)((c[k] - bmin[k]) / cl[k])));
  }
  std::vector<int>& at(int x, int y, int z) { return cells[((size_t)x * nc[1] + y) * nc[2] + z]; }
};

double det3(const double A[3][3]) {
  return A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
         A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
}

// Solves M z = b for 3x3 M by Cramer's rule; false when nearly singular.
bool solve3(const double M[3][3], const double* b, double* z) {
  const double det = det3(M);
  double scale = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) scale = std::max(scale, std::fabs(M[i][j]));
  if (!(std::fabs(det) > 1e-12 * scale * scale * scale)) return false;
  for (int c = 0; c < 3; ++c) {
    double A[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) A[i][j] = j == c ? b[i] : M[i][j];
    z[c] = det3(A) / det;
  }
  return true;
}

// Given three linear equations R . (c, r) = rhs in the unknowns (c, r), writes
// c = u + v r, then solves |c - x1|^2 = (r + r1)^2 for the smallest positive r.
bool tangent_from_linear(const double R[3][4], const double* rhs, const double* x1, double r1, double* c, double* r) {
  double M[3][3], d[3], u[3], v[3];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) M[i][j] = R[i][j];
    d[i] = -R[i][3];
  }
  if (!solve3(M, rhs, u) || !solve3(M, d, v)) return false;
  const double w[3] = {u[0] - x1[0], u[1] - x1[1], u[2] - x1[2]};
  const double a = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] - 1.0;
  const double b = 2.0 * (w[0] * v[0] + w[1] * v[1] + w[2] * v[2] - r1);
  const double cc = w[0] * w[0] + w[1] * w[1] + w[2] * w[2] - r1 * r1;
  double best = -1.0;
  if (std::fabs(a) < 1e-14) {
    if (std::fabs(b) > 1e-300) best = -cc / b;
  } else {
    const double disc = b * b - 4.0 * a * cc;
    if (disc < 0.0) return false;
    const double s = std::sqrt(disc);
    const double q1 = (-b - s) / (2.0 * a), q2 = (-b + s) / (2.0 * a);
    const double lo = std::min(q1, q2), hi = std::max(q1, q2);
    best = lo > 0.0 ? lo : hi;
  }
  if (!(best > 0.0)) return false;
  *r = best;
  for (int k = 0; k < 3; ++k) c[k] = u[k] + v[k] * best;
  return true;
}

}  // namespace

extern "C" int lsm_pack_fit(unsigned long long seed, int n, const double* bmin, const double* bmax, double rmin,
                            double rmax, int max_failures, double* pos, double* rad) {
  if (n <= 0 || !bmin || !bmax || !pos || !rad || !(rmax >= rmin) || !(rmin > 0) || max_failures < 1) return -1;
  for (int k = 0; k < 3; ++k)
    if (!(bmax[k] - bmin[k] > 2 * rmax)) return -1;
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> u01(0.0, 1.0);
  FitGrid G(bmin, bmax, 2.0 * rmax);
  int placed = 0;
  auto insert = [&](const double* c, double r) {
    for (int k = 0; k < 3; ++k) pos[3 * placed + k] = c[k];
    rad[placed] = r;
    int ic[3];
    G.cell_of(c, ic);
    G.at(ic[0], ic[1], ic[2]).push_back(placed);
    ++placed;
  };
  auto overlaps = [&](const double* c, double r) {
    int ic[3];
    G.cell_of(c, ic);
    const int reach = (int)std::ceil((r + rmax) / std::min(G.cl[0], std::min(G.cl[1], G.cl[2])));
    for (int x = std::max(0, ic[0] - reach); x <= std::min(G.nc[0] - 1, ic[0] + reach); ++x)
      for (int y = std::max(0, ic[1] - reach); y <= std::min(G.nc[1] - 1, ic[1] + reach); ++y)
        for (int z = std::max(0, ic[2] - reach); z <= std::min(G.nc[2] - 1, ic[2] + reach); ++z)
          for (int j : G.at(x, y, z)) {
            const double d0 = c[0] - pos[3 * j], d1 = c[1] - pos[3 * j + 1], d2 = c[2] - pos[3 * j + 2];
            const double rr = r + rad[j] - 1e-9 * (r + rad[j]);
            if (d0 * d0 + d1 * d1 + d2 * d2 < rr * rr) return true;
          }
    return false;
  };
  // seed layer: sparse random insertion of radii uniform in [rmin, rmax] (~5% solid fraction)
  {
    const double vol = (bmax[0] - bmin[0]) * (bmax[1] - bmin[1]) * (bmax[2] - bmin[2]);
    const double rm = 0.5 * (rmin + rmax);
    const int nseed = std::min(n, std::max(4, (int)(0.05 * vol / (4.18879 * rm * rm * rm))));
    std::uniform_real_distribution<double> ur(rmin, rmax);
    for (int i = 0, tries = 0; i < nseed && tries < 100 * nseed; ++tries) {
      const double r = ur(rng);
      double c[3];
      for (int k = 0; k < 3; ++k) c[k] = bmin[k] + r + u01(rng) * (bmax[k] - bmin[k] - 2 * r);
      if (!overlaps(c, r)) { insert(c, r); ++i; }
    }
  }
  // gap filling
  std::vector<std::pair<double, int>> near;
  int fails = 0;
  while (placed < n && fails < max_failures) {
    double p[3];
    for (int k = 0; k < 3; ++k) p[k] = bmin[k] + u01(rng) * (bmax[k] - bmin[k]);
    int ic[3];
    G.cell_of(p, ic);
    for (int reach = 1; reach <= 3; ++reach) {
      near.clear();
      for (int x = std::max(0, ic[0] - reach); x <= std::min(G.nc[0] - 1, ic[0] + reach); ++x)
        for (int y = std::max(0, ic[1] - reach); y <= std::min(G.nc[1] - 1, ic[1] + reach); ++y)
          for (int z = std::max(0, ic[2] - reach); z <= std::min(G.nc[2] - 1, ic[2] + reach); ++z)
            for (int j : G.at(x, y, z)) {
              const double d0 = p[0] - pos[3 * j], d1 = p[1] - pos[3 * j + 1], d2 = p[2] - pos[3 * j + 2];
              near.push_back({std::sqrt(d0 * d0 + d1 * d1 + d2 * d2) - rad[j], j});
            }
      if (near.size() >= 4) break;
    }
    bool ok = false;
    double c[3], r = 0.0;
    if (near.size() >= 3) {
      std::partial_sort(near.begin(), near.begin() + std::min<size_t>(4, near.size()), near.end());
      const int id[4] = {near[0].second, near[1].second, near[2].second, near.size() >= 4 ? near[3].second : -1};
      const double* x1 = pos + 3 * id[0];
      const double r1 = rad[id[0]];
      auto lin_row = [&](int j, double* row, double& rhs) {  // sphere j minus sphere 1
        const double* xj = pos + 3 * j;
        for (int k = 0; k < 3; ++k) row[k] = 2.0 * (xj[k] - x1[k]);
        row[3] = 2.0 * (rad[j] - r1);
        rhs = (xj[0] * xj[0] + xj[1] * xj[1] + xj[2] * xj[2]) - (x1[0] * x1[0] + x1[1] * x1[1] + x1[2] * x1[2]) -
              rad[j] * rad[j] + r1 * r1;
      };
      int fk = 0, fs = 0;  // nearest box face to the point
      double fd = 1e300;
      for (int k = 0; k < 3; ++k) {
        if (p[k] - bmin[k] < fd) { fd = p[k] - bmin[k]; fk = k; fs = 0; }
        if (bmax[k] - p[k] < fd) { fd = bmax[k] - p[k]; fk = k; fs = 1; }
      }
      for (int mode = 0; mode < 2 && !ok; ++mode) {
        double R[3][4], rhs[3];
        if (mode == 0) {  // four spheres
          if (id[3] < 0) continue;
          for (int q = 0; q < 3; ++q) lin_row(id[q + 1], R[q], rhs[q]);
        } else {          // three spheres and the nearest face: n.c - r = face offset (inward normal)
          lin_row(id[1], R[0], rhs[0]);
          lin_row(id[2], R[1], rhs[1]);
          for (int k = 0; k < 3; ++k) R[2][k] = 0.0;
          R[2][fk] = fs == 0 ? 1.0 : -1.0;
          R[2][3] = -1.0;
          rhs[2] = fs == 0 ? bmin[fk] : -bmax[fk];
        }
        double cc[3], rr;
        if (!tangent_from_linear(R, rhs, x1, r1, cc, &rr)) continue;
        if (rr < rmin || rr > rmax) continue;
        bool inside = true;
        for (int k = 0; k < 3; ++k) inside = inside && cc[k] - rr >= bmin[k] - 1e-9 && cc[k] + rr <= bmax[k] + 1e-9;
        if (!inside || overlaps(cc, rr)) continue;
        for (int k = 0; k < 3; ++k) c[k] = cc[k];
        r = rr;
        ok = true;
      }
    }
    if (ok) { insert(c, r); fails = 0; } else { ++fails; }
  }
  return placed;
}

// Pairs (i, j), i < j, whose gap |x_i - x_j| - r_i - r_j is at most max_gap (the rule of
// Geometry/DistConnections.hpp), found through a cell grid of size 2 r_max + max_gap.  Writes
// up to cap pairs in (i, j) order and returns the total count (call again with a larger cap
// when it exceeds cap), or -1 on bad arguments.
extern "C" long long lsm_dist_connections(int n, const double* pos, const double* rad, double max_gap,
                                          long long cap, int* out_i, int* out_j) {
  if (n < 0 || (n > 0 && (!pos || !rad)) || max_gap < 0 || cap < 0 || (cap > 0 && (!out_i || !out_j))) return -1;
  if (n < 2) return 0;
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300}, rmax = 0.0;
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) { mn[k] = std::min(mn[k], pos[3 * i + k]); mx[k] = std::max(mx[k], pos[3 * i + k]); }
    rmax = std::max(rmax, rad[i]);
  }
  const double cs = 2.0 * rmax + max_gap;
  long long nc[3];
  for (int k = 0; k < 3; ++k) nc[k] = std::max(1LL, (long long)std::floor((mx[k] - mn[k]) / cs) + 1);
  std::vector<long long> key(n);
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) {
    long long c[3];
    for (int k = 0; k < 3; ++k) c[k] = std::min(nc[k] - 1, (long long)((pos[3 * i + k] - mn[k]) / cs));
    key[i] = (c[0] * nc[1] + c[1]) * nc[2] + c[2];
    order[i] = i;
  }
  std::sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b] || (key[a] == key[b] && a < b); });
  std::vector<long long> skey(n);
  for (int i = 0; i < n; ++i) skey[i] = key[order[i]];
  std::vector<std::pair<int, int>> found;
  for (int i = 0; i < n; ++i) {
    const long long k0 = key[i];
    const long long cx = k0 / (nc[1] * nc[2]), cy = (k0 / nc[2]) % nc[1], cz = k0 % nc[2];
    for (long long dx = -1; dx <= 1; ++dx)
      for (long long dy = -1; dy <= 1; ++dy)
        for (long long dz = -1; dz <= 1; ++dz) {
          const long long x = cx + dx, y = cy + dy, z = cz + dz;
          if (x < 0 || y < 0 || z < 0 || x >= nc[0] || y >= nc[1] || z >= nc[2]) continue;
          const long long kk = (x * nc[1] + y) * nc[2] + z;
          auto lo = std::lower_bound(skey.begin(), skey.end(), kk);
          for (auto it = lo; it != skey.end() && *it == kk; ++it) {
            const int j = order[it - skey.begin()];
            if (j <= i) continue;
            const double d0 = pos[3 * i] - pos[3 * j], d1 = pos[3 * i + 1] - pos[3 * j + 1],
                         d2 = pos[3 * i + 2] - pos[3 * j + 2];
            if (std::sqrt(d0 * d0 + d1 * d1 + d2 * d2) - rad[i] - rad[j] <= max_gap) found.push_back({i, j});
          }
        }
  }
  std::sort(found.begin(), found.end());
  const long long m = (long long)found.size();
  for (long long k = 0; k < m && k < cap; ++k) { out_i[k] = found[k].first; out_j[k] = found[k].second; }
  return m;
}
