/*
 * esys_geometry.h -- seeded synthetic packings for the DEM benchmarks and tests.
 * Stands in for the reference's set-up packers (Geometry/RandomBoxPacker.hpp,
 * Python RandomBoxPacker) that generate particle inputs; not part of the
 * per-step hot path.
 */
#ifndef ESYS_GEOMETRY_H
#define ESYS_GEOMETRY_H
#ifdef __cplusplus
extern "C" {
#endif

/* Random sequential insertion of up to n spheres into [bmin, bmax] (x periodic when
 * periodic_x != 0): radii uniform in [p0, p1] (dist = 0) or lognormal with median p0 and
 * log-sigma p1 (dist = 1), clipped to [rmin, rmax], inserted largest first with up to
 * max_attempts trials each.  Writes pos (3 per sphere) and rad; returns the number placed
 * (<= n) or -1 on bad arguments. */
int lsm_pack_rsi(unsigned long long seed, int n, const double* bmin, const double* bmax, int periodic_x, int dist,
                 double p0, double p1, double rmin, double rmax, int max_attempts, double* pos, double* rad);

/* Dense random packing by gap filling (the role of Geometry/RandomBoxPacker.hpp: a seed
 * packing, then spheres fitted to touch their four nearest neighbours, or three and the nearest
 * box face, FittedParticleIterator::generateNext).  Radii of fitted spheres lie in
 * [rmin, rmax]; stops at n spheres or after max_failures consecutive rejected trials.  Returns
 * the number placed or -1 on bad arguments. */
int lsm_pack_fit(unsigned long long seed, int n, const double* bmin, const double* bmax, double rmin, double rmax,
                 int max_failures, double* pos, double* rad);

/* Pairs (i, j), i < j, with gap |x_i - x_j| - r_i - r_j <= max_gap (Geometry/DistConnections.hpp,
 * the Python ConnectionFinder); writes up to cap pairs sorted by (i, j) and returns the total
 * number found (call again with a larger cap if it exceeds cap), or -1 on bad arguments. */
long long lsm_dist_connections(int n, const double* pos, const double* rad, double max_gap, long long cap, int* out_i,
                               int* out_j);

#ifdef __cplusplus
}
#endif
#endif
