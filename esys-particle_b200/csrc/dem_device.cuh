// Device-side data layout of one simulated worker (shared by kernels and host).
//
// Particles live in slots in insertion order (the reference's particle-list
// order, ntable/src/ntable.h:85); a slot is never reused, a particle that
// leaves the grid is only marked dead.  State is structure-of-arrays of
// 32-byte double4 records so that a neighbour gather touches one sector per
// field, and it is double-buffered: a step reads buffer `cur` and writes
// buffer `cur ^ 1`, which lets one kernel do forces and integration without a
// grid-wide barrier.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dem {

enum : unsigned {
  PF_DYN = 1u,          // linear dynamics on (CParticle::m_is_dynamic)
  PF_ROT = 2u,          // rotational dynamics on (CRotParticle::m_is_rot)
  PF_ALIVE = 8u,        // still in the neighbour table
  PF_WALL_SHIFT = 8,    // bits 8..15: candidate of wall group w (getParticlesAtPlane)
  PF_INNER_SHIFT = 16,  // bits 16..23: candidate w is in the inner region (isInInner)
};

enum : int {
  CTRL_REBUILD = 1,     // some particle moved further than verletDist/2
  CTRL_BROKE = 2,       // at least one bond broke in the last force evaluation
  CTRL_OVERFLOW = 4,    // an event buffer overflowed
};

constexpr int kMaxWalls = 8;
constexpr int kMaxGrav = 4;
constexpr int kMaxDyn = 2;
constexpr int kMaxBond = 2;
constexpr int kBondAlive = 0x7fffffff;
// Dynamic-group adjacency entry .y: the pair index in the low 30 bits, bit 30 set under the
// device bond hand-off when an intact bond excluded the pair as the list was built, bit 31
// set when the entry's own particle is the pair's p1.
constexpr int kAdjIndex = 0x3fffffff;
constexpr int kAdjHeld = 0x40000000;
constexpr int kBondPassThreads = 128;  // bonds per block of the bond pass
constexpr int kTiled = 16;             // threads_per_particle setting of the tiled step kernels (dem_tiled.cuh)
constexpr int kWarpCoop = 32;          // threads_per_particle setting of the warp-cooperative pair sums (dem_step.cuh)
#ifndef DEM_TILE_THREADS
#define DEM_TILE_THREADS 256
#endif
constexpr int kTileThreads = DEM_TILE_THREADS;  // threads (= particles) per tile of the tiled step kernels

struct Grid {
  double p0x, p0y, p0z;  // origin of the global grid (the grown bounding box minimum)
  double dim;            // cell size = gridSpacing
  int gx, gy, gz;        // local-table offset of each dimension (-1: one padding layer)
  int nx, ny, nz;        // cells of the local table, padding included
  int circx;             // periodic in x
  double Lx, xmin;       // periodic box length and minimum
  double alpha;          // verletDist
};

struct ParticleBuf {
  double4* pr;  // x, y, z, radius
  double4* vm;  // vx, vy, vz, mass
  double4* wi;  // wx, wy, wz, rotational inertia
  double4* qq;  // quaternion scalar, x, y, z
  float4* vw;   // FP32 form: 2 per particle, (vx, vy, vz, wx), (wy, wz, 0, 0): one 32-byte sector
};

struct Particles {
  int n;                 // slots in use
  ParticleBuf buf[2];
  double2* inv;          // 1/mass, 1/inertia
  double4* oldpos;       // position at the last neighbour search
  float* dbound;         // upper bound of |position - oldpos| (FP32, rounded up): the step displacements
                         // summed since the last search, or the exact distance after a host-side move
  double* cshift;        // accumulated circular shift in x (CParticle::m_circular_shift)
  double4* force;        // last accumulated force  (w unused)
  double4* moment;       // last accumulated moment (w unused)
  double4* force_eval;   // FP32 forces of an evaluation-only pass (precision check)
  double4* moment_eval;
  double4* sum_f;        // split step: pair + bond force sums between the two kernels
  double4* sum_m;
  unsigned* pflags;      // PF_* bits
  unsigned char* flagged;// set on both particles of a broken bond (CParticle::flag)
  int* id;
  int* tag;
  int* cell;             // cell of each slot at the last neighbour search
};

struct WallDev {
  double ox, oy, oz, nx, ny, nz;  // plane origin and normal (CWall)
  double k;                       // NRotElasticWall normalK
};

// One dynamic interaction group (PIS_NE elastic or PIS_ED rot friction) as
// seen by the step kernel: a per-particle adjacency over the group's pairs.
struct DynDev {
  int kind;             // 0 NRotElastic, 1 RotFriction, 2 NRotFriction (CFrictionInteraction; mu in mu_s)
  double k, ks, mu_s, mu_d, dt;
  int scaling, meanR;
  const int* adj_start; // n+1
  const int2* adj;      // (partner slot, pair index | kAdjHeld | 0x80000000 when this particle is p1)
  const double4* hist_in;   // RotFriction: Ffric xyz, w = slipping + 2*touching
  double4* hist_out;
  const float4* hist32_in;  // the same in the FP32 form
  float4* hist32_out;
  // device bond hand-off only (else null): per pair, the bond that excluded it when the list
  // was built, (bond group << 28) | bond index, or -1.  Such a pair is skipped while that
  // bond is intact and becomes an ordinary pair at the step after the bond fails.  Its
  // adjacency entries carry kAdjHeld.
  const int* xbond;
};

struct BondDev {
  int kind;                 // 0 RotBond (ARotBondedInteraction), 1 NRotBond (CBondedInteraction),
                            // 2 BrittleBeamDZC (RotBond forces, BrittleBeamDZCInteraction::broken),
                            // 3 BrittleBeamSC (RotBond forces, BrittleBeamSCInteraction::broken at the update)
  double knb, rbreak;       // NRotBond: normal stiffness (unscaled), relative breaking distance (< 0: unbreakable)
  double cohesion, tan_angle, t_cutoff, c_cutoff, beta1, beta2;  // BrittleBeamDZC / SC failure criteria
  double kr, ks, kt, kb, mn, ms, mt, mb, truncated;
  int scaling, meanR;
  const int* adj_start;
  const int2* adj;          // (partner slot, bond index | 0x80000000 when this particle is p1)
  const double4* D0;        // m_D: p2 - p1 at creation (w unused)
  int* broken_step;         // kBondAlive while intact; else the step of the update that removes it
  int* events;              // (id1, id2, step) triples
  int* nevents;
  int cap_events;
  double4* bf;              // bond pass (else null): per bond the force on p1, the moment on p1 and on p2
  float4* bf32;             // FP32-force form (else null; takes the place of bf): per bond two 32-byte
                            // records, p1's then p2's, each (Fx, Fy, Fz, Mx), (My, Mz, 0, 0) of the
                            // force and moment on that particle
  int nb_launch;            // bonds in the group (the bond pass's extent)
  const int2* ends;         // (p1 slot, p2 slot) of each bond, p1 = lower id
};

// Intact bonds of the groups that exclude pairs from a dynamic group
// (TSubLattice::setExIG, Parallel/SubLattice.hpp:1980-2009).  Bond arrays are
// stored in (p1 slot, p2 slot) key order, so a key's position is its bond index.
struct ExclDev {
  int n;
  const unsigned long long* keys[kMaxBond];
  const int* broken_step[kMaxBond];
  int count[kMaxBond];
  int group[kMaxBond];  // the bond group's index in StepArgs::bond
};

struct StepArgs {
  Grid g;
  Particles P;
  int cur;                 // input buffer index
  double dt;
  double half_alpha_sq;    // (verletDist/2)^2
  long long step;          // timestep number being computed (1-based, like CLatticeMaster::m_t)
  int nwall;
  WallDev* walls;           // [nwall] in group-name order; origins move on the device
  const double* wall_vel;   // [nwall][3] native wall loader velocity (0 = static)
  int ngrav;
  double grav[kMaxGrav][3];
  int ndyn;
  DynDev dyn[kMaxDyn];
  int nbond;
  BondDev bond[kMaxBond];
  int damp_lin, damp_rot;   // damping groups present
  double visc_lin, visc_rot, dt_lin, dt_rot;
  int iter_lin, iter_rot;
  // local damping groups (CLocalDamping / CRotLocalDamping): present, viscosity, and whether the
  // LocalDamping group's name sorts before "Damping" (the damping map's order)
  int damp_loc, damp_rotloc, loc_before_lin;
  double visc_loc, visc_rotloc;
  int store_forces;
  long long force_step;     // forces are stored by this step only (-1: by every step)
  bool skip_vw;             // FP32 form: do not keep the FP32 velocity shadow (vw) up to date; set only
                            // where no kernel of the chunk reads it (the lane kernels read vm / wi)
  // device bond hand-off: a bond failure does not stop the chunk; the pairs it excluded turn
  // into ordinary pairs (DynDev::xbond) and every particle refreshes its wall candidacy at the
  // step after a failure (brk_step: last step with a failure)
  int handoff;
  int* brk_step;
  int stop_skip;            // CTRL_* bits that do not stop the chunk (0: every raised bit stops it)
  int replay;               // recompute of steps already taken: bond failures are not logged again
  double* sig;              // BrittleBeamSC present: each particle's stress sum of the last step (9 per slot)
  unsigned* pf_log;         // window recompute (else null): the PF_* bits each particle used in this step
  // adjoint recompute pass only (null otherwise): the pair + bond + wall + body force
  // sums before damping, and the damping iterations (lin, rot) of every particle
  double4* f_int;
  double4* m_int;
  unsigned char* damp_iters;
  double* wall_partial;     // [gridDim.x][kMaxWalls][3]
  double* wall_force;       // [kMaxWalls][3]: reaction of each wall group (adds into CWall::m_force)
  double* wall_hist;        // differentiable window only: [step - wall_hist_t0 - 1][kMaxWalls][3] reactions
  long long wall_hist_t0;
  unsigned* block_counter;  // last-block detection (wraps to 0 by itself)
  long long* step_counter;  // timesteps completed on the device
  int* ctrl;                // CTRL_* bits raised by this chunk of steps
  int* stop;                // set by the last block when ctrl != 0: later steps of the chunk skip
};

// Batched ensemble step (dem_batch.cuh): the specimens' step arguments in a device table.
struct BatchArgs {
  int nspec;
  int total_tiles;
  const StepArgs* args;     // [nspec][2]: step arguments for input buffer 0 and 1
  const int* tile_start;    // [nspec + 1]: prefix of step_tiles(n, TPP)
  const long long* base_t;  // [nspec]: the specimen's step counter when the table was written
  const int* base_cur;      // [nspec]: its input buffer then
  const long long* target;  // [nspec]: last timestep to compute in this call
  int total_btiles;         // bond pass: tiles of kBondPassThreads bonds over (specimen, bond group)
  const int* btile_start;   // [nspec * kMaxBond + 1]
};

}  // namespace dem
