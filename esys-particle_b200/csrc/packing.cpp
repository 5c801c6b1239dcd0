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
