/*
 * esys_dem.h -- C ABI of the B200 DEM step (libesys_dem_b200.so).
 *
 * One dem_sim handle is one ESyS-Particle worker sub-lattice living on one GPU:
 * the state and operations of TSubLattice<T> / TRotSubLattice<T>
 * (Parallel/SubLattice.h:77-302, Parallel/RotSubLattice.h), behind the
 * ASubLattice operations the master drives over MPI
 * (Parallel/ASubLattice.h:36-197, Parallel/SubLatticeControler.cpp:534-600).
 * Plain pointers and sizes only; all arrays are host memory owned by the
 * caller; the library owns all device memory.
 *
 * Every function returns a status (DEM_OK = 0, negative on failure) or a
 * non-negative count; dem_last_error() gives the message of the last failure.
 * The reference throws std::runtime_error for the same conditions
 * (SubLattice.hpp:688-692, 1709-1714; pp_array.hpp:77-88).
 * A handle is single-threaded: calls on one handle must not overlap.
 */
#ifndef ESYS_DEM_H
#define ESYS_DEM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dem_sim dem_sim;
typedef struct dem_ensemble dem_ensemble;

enum {
  DEM_OK = 0,
  DEM_ERR_ARG = -1,      /* invalid argument (unknown group or wall, bad sizes, wrong particle type) */
  DEM_ERR_OVERFLOW = -2, /* a device-side log ran out of room */
  DEM_ERR_CUDA = -3,     /* CUDA error or no GPU */
  DEM_ERR_INTERNAL = -4,
  DEM_ERR_STATE = -5     /* not allowed in the current state (e.g. a bond broke inside a differentiable window) */
};

/* Particle types: 0 = "NRotSphere" (CParticle), 1 = "RotSphere" (CRotParticle). */

/* CLatticeMaster::makeLattice + setTimeStepSize + setSpatialDomain
 * (Parallel/LatticeMaster.cpp:528-553, 574-583, 613-693) -> TSubLattice ctor and
 * initNeighborTable(min, max[, circ]) (Parallel/SubLattice.hpp:455-564).
 * grid_spacing / verlet_dist are initNeighbourSearch's gridSpacing and
 * verletDist; circ[0] != 0 makes x periodic (circDimList).  The domain is checked on the host
 * before any device is touched, so a bad one returns DEM_ERR_ARG with or without a GPU:
 * bbox_max <= bbox_min or a non-finite corner, grid_spacing <= 0, verlet_dist < 0, dt <= 0,
 * circ[1] or circ[2] set, a periodic x side shorter than 3 grid spacings, more than 2^31 - 1
 * cells.  Without a usable GPU a valid domain returns DEM_ERR_CUDA.  Failing, *out is NULL and
 * dem_last_error(NULL) gives this thread's last dem_create failure. */
int dem_create(dem_sim** out, int particle_type, double grid_spacing, double verlet_dist, const double* bbox_min,
               const double* bbox_max, const int* circ, double dt);
int dem_destroy(dem_sim* h);
const char* dem_last_error(dem_sim* h);

/* TSubLattice::receiveParticles + searchNeighbors(true) (Parallel/SubLattice.hpp:573-588,
 * Parallel/LatticeMaster.hpp:260-330).  pos/vel/angvel are n x 3, quat n x 4 (scalar first),
 * vel/angvel/quat/tag/flags may be NULL.  flags bit0: non-dynamic, bit1: non-rotational.
 * Rotational inertia is 0.4 m r^2 (Model/RotParticle.cpp:34).  Particles outside the
 * search grid are dropped (ntable/src/ntable.hpp:243-258). */
int dem_add_particles(dem_sim* h, int n, const int* id, const int* tag, const double* pos, const double* rad,
                      const double* mass, const double* vel, const double* angvel, const double* quat,
                      const int* flags);

/* TSubLattice::receiveConnections (Parallel/SubLattice.hpp:598-622): (tag, id1, id2) triples
 * stored for a later bonded group with that tag. */
int dem_add_connections(dem_sim* h, int n, const int* tag, const int* id1, const int* id2);

/* TSubLattice::addWall (Parallel/SubLattice.hpp:629-642): plane through origin o with normal n. */
int dem_add_wall(dem_sim* h, const char* name, const double* o, const double* n);

/* addPairIG "Elastic" -> PIS_NE<T,CElasticInteraction> (Parallel/SubLattice.hpp:1038-1054);
 * parameters of CElasticIGP (Model/ElasticInteraction.h:24-41). */
int dem_add_elastic_group(dem_sim* h, const char* name, double k, int scaling);

/* addPairIG "RotFriction" -> PIS_ED<CRotParticle,CRotFrictionInteraction>
 * (Parallel/SubLattice.hpp:1202-1227), parameters in CRotFrictionIGP packing order
 * k, mu_s, mu_d, k_s, dt, scaling, meanR_scaling (Parallel/LatticeMaster.cpp:3223-3235). */
int dem_add_rot_friction_group(dem_sim* h, const char* name, double k, double mu_s, double mu_d, double ks,
                               double dt, int scaling, int meanR_scaling);

/* TSubLattice::addPairIG, type "Friction" (NRotFrictionPrms; Parallel/SubLattice.hpp:1055-1076):
 * CFrictionInteraction (Model/FrictionInteraction.cpp:57-149) with CFrictionIGP's packing order
 * k, mu, k_s, dt, scaling.  Elastic normal force and tangential friction from the relative
 * translation, forces only.  FP64 form; no differentiable window or batched ensemble. */
int dem_add_nrot_friction_group(dem_sim* h, const char* name, double k, double mu, double ks, double dt, int scaling);

/* TSubLattice::addPairIG, type "HertzMindlin" (HertzMindlinPrms; Parallel/SubLattice.hpp:1324-1339):
 * CHertzMindlinInteraction (Model/HertzMindlinInteraction.cpp:108-172) with CHertzMindlinIGP's packing
 * order E, nu, mu, dt: Hertz normal force, Mindlin tangential stiffness, forces only.  Its storage is
 * PIS_NE: the tangential history restarts at every neighbour rebuild, and checkpoints do not save it.
 * FP64 form; no device bond hand-off, differentiable window or batched ensemble. */
int dem_add_hertz_mindlin_group(dem_sim* h, const char* name, double E, double nu, double mu, double dt);

/* TSubLattice::addPairIG, type "HertzMindlinVisco" (HertzMindlinViscoPrms; Parallel/SubLattice.hpp:
 * 1340-1356): CHertzMindlinViscoInteraction (Model/HertzMindlinViscoInteraction.cpp:119-200), packing
 * order E, nu, mu, COR (restitution), dt: HertzMindlin with normal and tangential damping from the
 * restitution coefficient and a tangential force without history.  PIS_NE; FP64 form; fields "count",
 * "slipping", "sticking". */
int dem_add_hertz_mindlin_visco_group(dem_sim* h, const char* name, double E, double nu, double mu, double COR,
                                      double dt);

/* TRotSubLattice::addBrittleBeamDZCIG (BrittleBeamDZCPrms; Parallel/RotSubLattice.hpp:227-267):
 * BrittleBeamDZCInteraction (Model/BrittleBeamDZC.cpp) between the tagged connections, with the
 * master's packing order kr, ks, kt, kb, cohesion, tCutoff, cCutoff, fAngle (degrees), beta1,
 * beta2.  Forces and moments are RotBond's (ARotBondedInteraction::calcForces, stiffnesses scaled by
 * the half bond length); failure when the beam's normal stress falls below -tCutoff, its shear
 * stress exceeds cCutoff, or exceeds cohesion + normal stress * tan(fAngle).  RotSpheres; no
 * restart checkpoint, differentiable window or batched ensemble. */
int dem_add_brittle_beam_dzc_group(dem_sim* h, const char* name, int tag, double kr, double ks, double kt, double kb,
                                   double cohesion, double tCutoff, double cCutoff, double fAngle, double beta1,
                                   double beta2);

/* TRotSubLattice::addBrittleBeamSCIG (BrittleBeamSCPrms; Parallel/RotSubLattice.hpp:188-225):
 * BrittleBeamSCInteraction (Model/BrittleBeamSC.cpp) with the master's packing order kr, ks, kt, kb,
 * cohesion, tCutoff, fAngle (degrees).  RotBond forces and moments; the bond fails at the update that
 * opens a step when the symmetric part of its two particles' mean stress (each particle's sum of
 * -f (x) (contact point - centre) over the last step's forces, over its volume), in the frame of the bond
 * axis, has a normal component below -tCutoff or a shear magnitude above cohesion + normal * tan(fAngle).
 * RotSpheres; FP64 form; no restart checkpoint, differentiable window or batched ensemble. */
int dem_add_brittle_beam_sc_group(dem_sim* h, const char* name, int tag, double kr, double ks, double kt, double kb,
                                  double cohesion, double tCutoff, double fAngle);

/* TSubLattice::addBondedIG (NRotBondPrms; Parallel/SubLattice.hpp:1791-1831): CBondedInteraction
 * (Model/BondedInteraction.cpp:43-140) between connections of `tag`; rest length r1 + r2, failure
 * when the extension exceeds (r1 + r2) * rbreak; rbreak < 0: unbreakable.  Forces only.  No
 * differentiable window or batched ensemble. */
int dem_add_nrot_bond_group(dem_sim* h, const char* name, int tag, double k, double rbreak, int scaling);

/* TRotSubLattice::addRotBondedIG (Parallel/RotSubLattice.hpp:116-186): bonds from the stored
 * connections with this tag, CRotBondedIGP fields in packing order; beta1 = beta2 = 1. */
int dem_add_rot_bond_group(dem_sim* h, const char* name, int tag, double kr, double ks, double kt, double kb,
                           double max_nForce, double max_shForce, double max_tMoment, double max_bMoment,
                           int scaling, int meanR_scaling, double truncated);

/* TSubLattice::addElasticWIG (Parallel/SubLattice.hpp:667-696): CEWallInteractionGroup<T>. */
int dem_add_wall_group(dem_sim* h, const char* name, const char* wall, double k);

/* TSubLattice::addSingleIG "Gravity" -> BodyForceGroup<T> (Parallel/SubLattice.hpp:1687-1697). */
int dem_add_gravity(dem_sim* h, const char* name, const double* g);

/* TSubLattice::doAddDamping "Damping" / TRotSubLattice::doAddDamping "RotDamping"
 * (Parallel/SubLattice.hpp:1748-1784, Parallel/RotSubLattice.hpp:79-109); v_ref = 0. */
int dem_add_damping(dem_sim* h, int rotational, double viscosity, int max_iterations);

/* TSubLattice::doAddDamping "LocalDamping" / TRotSubLattice::doAddDamping "RotLocalDamping"
 * (Parallel/SubLattice.hpp:1765-1769, Parallel/RotSubLattice.hpp:95-104): CLocalDamping /
 * CRotLocalDamping (Model/LocalDamping.hpp:82-118, Model/RotLocalDamping.hpp:82-117) with this
 * viscosity.  Applied with the other damping groups in their name order ("Damping" and the
 * LocalDamping group's own name on the force; "RotDamping" then "RotLocalDamping" on the moment).
 * Not part of the differentiable window. */
int dem_add_local_damping(dem_sim* h, const char* name, int rot, double visc);

/* TSubLattice::setExIG (Parallel/SubLattice.hpp:1980-2009): pairs bonded in `bonded` are
 * excluded from the dynamic group `dynamic` while the bond is intact. */
int dem_add_exclusion(dem_sim* h, const char* bonded, const char* dynamic);

/* TSubLattice::setTimeStepSize (Parallel/SubLattice.hpp:2163-2204). */
int dem_set_timestep(dem_sim* h, double dt);

/* nsteps x CLatticeMaster::runOneStep (Parallel/LatticeMaster.cpp:2602-2725) on this worker:
 * checkNeighbors -> searchNeighbors -> updateInteractions -> oneStep (zeroForces, calcForces,
 * integrate).  Field savers and Python runnables are the caller's. */
int dem_step(dem_sim* h, int nsteps);

/* ASubLattice::searchNeighbors (Parallel/ASubLattice.h; TSubLattice::searchNeighbors,
 * Parallel/SubLattice.hpp:2360-2408) on demand: the neighbour search and interaction update
 * that a displacement beyond verletDist/2 triggers, run at the head of the next step.  It
 * changes no force (pairs that leave the lists are not touching; pairs that join start with
 * the zero history they would have); it restarts the displacement budget, e.g. before a
 * differentiable window. */
int dem_search_neighbors(dem_sim* h);

/* TSubLattice::moveWallBy (Parallel/SubLattice.hpp:2878-2895) -> CWall::moveBy (Model/Wall.h:54-60). */
int dem_move_wall(dem_sim* h, const char* name, const double* d);

/* Device-side wall loader: moves the wall by v*dt after every step, the constant-speed phase of
 * WallLoaderRunnable (Doc/Tutorial/examples/WallLoader.py.tex) without a host call per step. */
int dem_set_wall_velocity(dem_sim* h, const char* name, const double* v);

/* TSubLattice::applyForceToWall (Parallel/SubLattice.hpp:2935-2950) -> CEWallInteractionGroup::applyForce
 * (Model/EWallInteractionGroup.hpp:93-164). */
int dem_apply_force_to_wall(dem_sim* h, const char* group, const double* f);

/* getWallPosition / getWallForce (Python/esys/lsm/LsmMpiPy.cpp:2767-2786); either output may be NULL. */
int dem_get_wall(dem_sim* h, const char* name, double* pos, double* force);

/* TSubLattice::getNumParticles (Parallel/SubLattice.hpp:486-490): particles in the table. */
int dem_num_particles(dem_sim* h);

/* Particle state (the fields CParticle / CRotParticle expose to savers), one row per particle
 * in table order; any output may be NULL.  Returns the number of rows written. */
int dem_get_particles(dem_sim* h, int* id, double* pos, double* vel, double* angvel, double* quat, double* force,
                      double* moment);

/* Interactions of a group as (id1 < id2) pairs (CLatticeMaster::getBondGroupIdPairs, Parallel/LatticeMaster.cpp:2742-2766);
 * state is n x 5 or NULL: RotFriction -> tangential force (3), slipping, touching.
 * Returns the number of pairs. */
int dem_num_pairs(dem_sim* h, const char* group);
int dem_get_pairs(dem_sim* h, const char* group, int* id1, int* id2, double* state);

/* Bond failures so far (PIS_EB::update, pis/pi_storage_eb.hpp:23-49): (id1, id2, step) per
 * broken bond, step = the time step whose interaction update removed it. */
int dem_num_breaks(dem_sim* h);
int dem_get_breaks(dem_sim* h, int* id1, int* id2, int* step);

/* TSubLattice::moveTaggedParticlesBy (Parallel/SubLattice.hpp:2577-2587). */
int dem_move_tagged(dem_sim* h, int tag, int mask, const double* d);

/* Time steps completed (CLatticeMaster::m_t). */
long long dem_timestep(dem_sim* h);

/* Bulk update of existing particles' state (pos/vel n x 3, angvel n x 3, quat n x 4; any may be
 * NULL), like setParticleVelocity / moveParticleTo over many particles
 * (Python/esys/lsm/LsmMpiPy.cpp:3054-3136).  With id == NULL, row i is particle slot i (the
 * order of dem_get_particles while no particle has left the grid).  A move is checked against
 * verletDist/2 before the next step, as checkNeighbors would. */
int dem_set_particles(dem_sim* h, int n, const int* id, const double* pos, const double* vel, const double* angvel,
                      const double* quat);

/* Ghost particles of a slab decomposition (esys.lsm.slabs): the particles with these ids, deleted
 * when they left this worker's grid, come back alive with the given state (pos, vel, angvel: 3 per
 * row; quat: 4 per row; any may be null); alive ones are only updated.  Replaces the reference's
 * re-sending of the ghost layer at a rebuild (ParallelParticleArray::rebuild, the circular cell
 * shifts of ppa/src/pp_array.hpp:450-504).  Schedules a neighbour search. */
int dem_revive_particles(dem_sim* h, int n, const int* id, const double* pos, const double* vel, const double* angvel,
                         const double* quat);

/* Ghost particles of a slab decomposition: the tangential history of pairs of a dynamic group
 * (rows of dem_get_pairs' state: Fx, Fy, Fz, slipping, touching), written into the pairs of this
 * worker's current list (pairs not in it are skipped; the elastic law keeps no history).  Returns
 * the pairs written.  Replaces the interaction records the reference moves with the particles it
 * moves between workers at a rebuild (ParallelInteractionStorage_ED::update,
 * pis/pi_storage_ed.hpp:84-161, after pp_array.hpp:450-504). */
int dem_set_pair_states(dem_sim* h, const char* group, int n, const int* id1, const int* id2, const double* state);

/* Run all device work of this handle on the caller's CUDA stream (a cudaStream_t); the caller
 * keeps ownership.  No reference counterpart (the reference has no device). */
int dem_set_stream(dem_sim* h, void* stream);

/* Counters, no reference counterpart (the reference's MpiWTimers, Foundation/Timer.h:28-102, time
 * phases instead): out[0] steps, [1] interactions evaluated (Verlet pairs + intact bonds + wall
 * candidates, summed over steps), [2] neighbour searches, [3] kernel launches, [4] device time of
 * the force/integration kernels in ns (with option "profile"), [5] steps timed by [4],
 * [6] interactions evaluated per step now, [7] threads per particle in use, [8] 1 when a neighbour
 * search is due at the head of the next step (a particle moved more than verletDist/2 since the
 * last search, dem_search_neighbors was called, or no step has run yet: what
 * TSubLattice::checkNeighbors reports, Parallel/SubLattice.hpp:2473-2520).  Returns entries written. */
int dem_get_counters(dem_sim* h, long long* out, int n);

/* Precision check of the FP32-force form, no reference counterpart: from the FP64 form, evaluates
 * the FP32-form forces of the current state, then advances one FP64 step and compares.
 * out[0] = max|dF|/max|F|, out[1] = max|dM|/max|M|, out[2] / out[3] = median / 99th percentile of
 * |dF_i|/|F_i| over particles with |F_i| > 1e-9 max|F|, out[4] = particles compared. */
int dem_precision_check(dem_sim* h, double* out);

/* dem_precision_check with two more figures, out[0..n-1] (n <= 7): out[0..4] as above; out[5] =
 * max |dF| / the largest per-particle contact-force sum (sum of |f| over the particle's pair and
 * bond contributions: the system's force scale, which stays meaningful where net forces cancel);
 * out[6] = max over particles of |dF| / that particle's own contact-force sum.  Returns the count. */
int dem_precision_report(dem_sim* h, double* out, int n);

/* Allocation-free per-wall reaction forces, for callers that cannot call cudaMalloc: code that
 * runs during CUDA graph capture, hosts that hand the library only memory from their own pool,
 * real-time loops that forbid allocation.  No counterpart in the reference.
 * Computes, for each wall, the sum over the given particles of the elastic wall contact force.
 * Every given particle counts, wherever it lies; the reaction the step accumulates into
 * CWall::m_force (what dem_get_wall reports) counts only the wall's candidates (within one grid
 * spacing of the plane, in the grid interior), so pass those particles to get that quantity.
 * particles: device, n rows of 4 doubles (x, y, z, radius), 16-byte aligned; walls: device, nwall
 * rows of 7 doubles (origin xyz, normal xyz, normalK), 8-byte aligned; reactions: device, nwall x 3
 * doubles, 8-byte aligned; stream: a cudaStream_t (NULL = default stream).  Limits:
 * 1 <= nwall <= 8, 0 <= n <= 16777216; larger sizes or misaligned buffers return DEM_ERR_ARG.  No
 * memory is allocated: block partial sums live in a fixed 111 KiB (113,672-byte) __device__ array that every GPU loading the library keeps until exit.  The first call on
 * each device looks up that array's address (make it before any stream capture).  All calls on a
 * device share the array, so calls that overlap on the GPU race; the result of each call is
 * written asynchronously on `stream`. */
int dem_wall_reactions_noalloc(int n, const double* particles, int nwall, const double* walls, double* reactions,
                               void* stream);

/* Tuning knobs with no reference counterpart: "threads_per_particle" (0 = automatic: one lane for
 * a specimen with at least 768 particles per SM, else by the mean adjacency length; 1, 2, 4, 8;
 * 16 = block-cooperative tiles; 32 = warp-cooperative pair sums),
 * "chunk" (steps launched per host round trip), "store_forces" (keep per-particle F/M),
 * "profile" (time the force/integration kernels with CUDA events), "precision" (64 = FP64 form,
 * 32 = FP32 pair forces with Kahan-compensated accumulation, FP64 positions / contact detection /
 * integration), "split" (1: pair kernel + integration kernel), "bond_pass" (1: each bond
 * evaluated once per step and gathered), "bond_handoff" (1: bond failures handed to the friction
 * lists on the device), "adjoint_bond_tangents" (0: hand-written RotBond reverse; 3, 6, 9, 18:
 * forward-mode dual tangents per pass), "adjoint_pair_duals" (0: hand-written pair-law
 * reverses; 1: forward-mode duals), "event_capacity" (entries of each bonded group's failure-event
 * log, existing groups and later ones; 0 = one per bond, the default, which cannot overflow; a
 * smaller log that fills makes the dem_step or dem_ensemble_step call in which it filled return
 * DEM_ERR_OVERFLOW after running all its steps; the bond states stay exact, dem_get_breaks holds
 * the events logged before it filled, later calls go on, and the capacity of a group whose log
 * overflowed can no longer change). */
int dem_set_option(dem_sim* h, const char* key, double value);

/* ---- Field savers ----------------------------------------------------------------------- */

/* Per-particle scalar field, computed on the device in the reference's accessor arithmetic
 * (CParticle / CRotParticle::getScalarFieldFunction, Model/Particle.cpp:140-160,
 * Model/RotParticle.cpp:422-456): "e_kin", "e_kin_linear", "e_kin_rot", "v_abs", "radius",
 * "id", "tag", and "mass" (no reference field: CParticle::getMass).  values[] in
 * dem_get_particles order; returns the count. */
int dem_particle_scalar_field(dem_sim* h, const char* field, double* values);

/* Per-particle vector field (CParticle::getVectorFieldFunction, Model/Particle.cpp:166-184;
 * CRotParticle::getVectorFieldFunction, Model/RotParticle.cpp:459-480): "position", "velocity",
 * "force", "displacement" (getTotalDisplacement: position less the position at creation, which
 * follows the circular shifts) and, for RotSpheres, "ang_velocity".  values[] is n x 3 in
 * dem_get_particles order; returns the count. */
int dem_particle_vector_field(dem_sim* h, const char* field, double* values);

/* Per-interaction scalar field of one group, from the state its last force evaluation read:
 * NRotElastic "count", "potential_energy"; RotFriction "count", "potential_energy", "slipping",
 * "sticking" (Model/RotFricInteraction.cpp:384-452, 486-508); RotBond "count",
 * "potential_energy", "e_pot_normal", "e_pot_shear", "e_pot_twist", "e_pot_bend",
 * "breaking_criterion" (Model/ARotBondedInteraction.cpp:456-485, RotBondedInteraction.cpp:
 * 221-256); NRotFriction and HertzMindlin "count", "potential_energy", "slipping", "sticking"
 * (Model/FrictionInteraction.cpp:336-400, HertzMindlinInteraction.cpp:371-400).  BrittleBeam groups
 * as RotBond without "breaking_criterion".  values[] in dem_get_pairs order; returns the count.  NRotElastic's
 * potential_energy is 0 for a pair not touching at that evaluation (the reference keeps the
 * last contact force of such a pair until the next rebuild). */
int dem_interaction_scalar_field(dem_sim* h, const char* group, const char* field, double* values);

/* ---- Parameters and the differentiable loading window -------------------------------- */

/* Sets one parameter of an existing group for every interaction in it, like
 * LsmMpi.setInteractionParameter -> TParallelInteractionStorage::forAllInteractionsSet
 * (Parallel/LatticeMaster.cpp:4290-4301, pis/pi_storage.hpp:277-292).  The reference only
 * binds "k" of CElasticInteraction (Model/ElasticInteraction.cpp:169-180); here the keys are
 * the *Prms attribute names: RotBond "normalK", "shearK", "torsionK", "bendingK"; RotFriction
 * "normalK", "shearK", "staticMu", "dynamicMu"; NRotElastic "normalK"; the damping groups
 * "Damping" / "RotDamping" take "viscosity".  Values are unscaled group parameters: the
 * per-interaction scaling of each law's constructor is applied to them at every step. */
int dem_set_group_param(dem_sim* h, const char* group, const char* key, double value);

/* Number of parameter gradients dem_window_adjoint writes: 4 per RotBond group (normalK,
 * shearK, torsionK, bendingK), 2 per dynamic group (normalK, shearK; elastic: normalK, 0) in
 * group-name order, then the linear and rotational damping viscosities. */
int dem_window_num_params(dem_sim* h);

/* Runs nsteps FP64 steps (the dem_step sequence) as a differentiable window: the neighbour
 * lists are frozen (DEM_ERR_STATE if a rebuild falls inside the window).  A bond failure
 * inside the window needs the device bond hand-off (dem_set_option "bond_handoff"; else
 * DEM_ERR_STATE): the failures are then events of the window, the same in the forward run
 * and in the adjoint's recompute, and the gradient is that of the branch taken.  The state
 * is checkpointed every checkpoint_every steps, and the
 * reaction of every wall group after every step (CWall::m_force, EWallInteractionGroup.hpp:
 * 47-53) is written to reactions[nsteps][wall groups in name order][3] (may be null). */
int dem_window_forward(dem_sim* h, int nsteps, int checkpoint_every, double* reactions);

/* Reverse pass of the last window: grad_reactions[nsteps][wall groups][3] is dLoss/dReaction;
 * grad_params receives dem_window_num_params values; grad_vel / grad_angvel / grad_pos (n x 3)
 * and grad_quat (n x 4) receive dLoss/d(initial state) in dem_get_particles order.  Any output
 * may be null.  The simulation must not have stepped since dem_window_forward. */
int dem_window_adjoint(dem_sim* h, const double* grad_reactions, double* grad_params, double* grad_vel,
                       double* grad_angvel, double* grad_pos, double* grad_quat);

/* Restores the state at the start of the last window (particles, friction histories, wall
 * planes, timestep, and the bond failures, event log and wall candidacy the window changed),
 * so that the window can be run again with other parameters. */
int dem_window_rewind(dem_sim* h);

/* Restart checkpoints: the worker's file of TSubLattice::saveCheckPointData
 * (Parallel/SubLattice.hpp:3600-3673), in its text layout and iostream formatting with
 * `precision` significant digits (CheckPointer::saveRestartable, Parallel/CheckPointer.cpp:48-66;
 * 12 if <= 0): the particle block (ParallelParticleArray::saveCheckPointData, CRotParticle
 * records), each RotBond group's restart records, each RotFriction group's pair records with
 * their tangential history, the walls.  The master's info file (CheckPointInfo) is the caller's
 * (esys.lsm.LsmMpi.createRestartCheckPointer writes both).  One difference: the reference writes
 * a RotFriction group's record count and first record with no separator between them; a newline
 * is written here so that the count reads back. */
int dem_save_checkpoint(dem_sim* h, const char* path, int precision);

/* Snapshot (visualisation) file of TSubLattice::saveSnapShotData (Parallel/SubLattice.hpp:3552-3594):
 * 9 significant digits; particle snapshot records, then each RotBond group's (id1, id2, tag) records.
 * The master's info file is the caller's (esys.lsm.LsmMpi.createCheckPointer writes both). */
int dem_save_snapshot(dem_sim* h, const char* path);

/* TSubLattice::loadCheckPointData (Parallel/SubLattice.hpp:3675-3790) into a worker without
 * particles whose groups the script has created (as in the reference): particles, the bonds of
 * each RotBond group with their creation vectors, each RotFriction group's pairs and histories,
 * the walls (created or replaced); then, as CLatticeMaster::loadCheckPointData
 * (Parallel/LatticeMaster.cpp:780-820), the step counter is set to `timestep` and the neighbour
 * search and interaction update run.  Pair histories survive for the pairs still touching, as
 * PIS_ED::update keeps them.  The per-interaction constants in the file are not read back: they
 * follow from the groups' parameters. */
int dem_load_checkpoint(dem_sim* h, const char* path, long long timestep);

/* Frees the last window's checkpoints and reverse-pass buffers (no rewind or adjoint after). */
int dem_window_release(dem_sim* h);

/* ---- Batched ensemble --------------------------------------------------------------------
 * No counterpart in the reference, where each specimen is its own MPI job.  An ensemble advances
 * n independent workers (each a dem_sim set up as usual, all RotSphere or all NRotSphere, all in
 * the same precision form) together: one kernel launch per timestep covers every specimen's
 * particles, and chunks of launches are replayed from a captured CUDA graph.  Each specimen keeps
 * its own rebuilds, interaction updates, bond failures, walls and timestep, so it advances
 * exactly as dem_step would advance it alone.  The ensemble borrows the handles: destroy it
 * before any of them, and do not call a member handle while an ensemble call runs. */
int dem_ensemble_create(dem_ensemble** out, dem_sim* const* sims, int n);
int dem_ensemble_destroy(dem_ensemble* e);
const char* dem_ensemble_last_error(dem_ensemble* e);

/* nsteps timesteps of every specimen (each runs its own runOneStep sequence). */
int dem_ensemble_step(dem_ensemble* e, int nsteps);

/* Batched differentiable windows: every specimen runs dem_window_forward(nsteps,
 * checkpoint_every) from its own current step, the forward in batched launches; reactions[k]
 * (may be null, as may the array) receives specimen k's [nsteps][wall groups][3] reactions.
 * A failure of any specimen (a rebuild inside the window, ...) fails the call with the
 * specimen's index in the message. */
int dem_ensemble_window_forward(dem_ensemble* e, int nsteps, int checkpoint_every, double* const* reactions);

/* The reverse pass of every specimen's last window together: one launch per reverse kernel
 * and timestep covers all specimens (recompute included).  Per specimen k, grad_reactions[k]
 * is its dLoss/dReaction as in dem_window_adjoint; grad_params[k] (dem_window_num_params
 * values), grad_vel[k] and grad_angvel[k] (n x 3) receive its gradients (any may be null).
 * Results equal each specimen's own dem_window_adjoint. */
int dem_ensemble_window_adjoint(dem_ensemble* e, const double* const* grad_reactions, double* const* grad_params,
                                double* const* grad_vel, double* const* grad_angvel);

/* "threads_per_particle" (0 automatic, 1, 2, 4, 8), "chunk" (timesteps per graph replay),
 * "graph" (1 replay captured graphs, 0 plain launches), "profile" (CUDA-event timing). */
int dem_ensemble_set_option(dem_ensemble* e, const char* key, double value);

/* out[0..7] = specimen-timesteps, contact updates, kernel launches, chunks, batched-step device ns,
 * profiled timesteps, threads per particle in use, rebuild requests. */
int dem_ensemble_get_counters(dem_ensemble* e, long long* out, int n);

#ifdef __cplusplus
}
#endif
#endif
