/*
 * GpuSubLattice.h -- TGpuSubLattice<T>: an ESyS-Particle worker sub-lattice whose particles and
 * interactions live on one GPU, behind the C ABI of include/esys_dem.h.
 *
 * It implements the ASubLattice operations (Parallel/ASubLattice.h:36-197) that the worker's
 * command loop calls (CSubLatticeControler::run, Parallel/SubLatticeControler.cpp:534-720), so a
 * master (CLatticeMaster) drives it exactly as it drives TSubLattice<T> / TRotSubLattice<T>:
 * each operation receives its parameters from the master in the reference's own buffers and
 * packing order (CVarMPIBuffer, TML_Comm packed broadcasts), takes part in the same barriers and
 * gathers, and hands the work to the GPU library.  To use it, CSubLatticeControler::makeLattice
 * (Parallel/SubLatticeControler.cpp:121-150) constructs TGpuSubLattice<CParticle> for "Basic"
 * and TGpuSubLattice<CRotParticle> for "Rot" in place of TSubLattice / TRotSubLattice; this
 * file is compiled inside the reference tree against its headers and linked with
 * libesys_dem_b200.so.
 *
 * One worker holds the whole specimen (the worker communicator has one rank): the GPU library
 * keeps every particle, so there is no ghost exchange (exchangePos has nothing to do) and the
 * neighbour check, search and interaction update that the master orders at the head of each
 * step run inside dem_step.  Operations outside the GPU path (meshes, sphere bodies, fluid,
 * thermal groups, tagged pair groups, field savers) throw std::runtime_error, as TSubLattice
 * does for interaction types it does not know (Parallel/SubLattice.hpp:1709-1714).
 */
#ifndef ESYS_GPU_SUBLATTICE_H
#define ESYS_GPU_SUBLATTICE_H

#include "Parallel/ASubLattice.h"
#include "Parallel/LatticeParam.h"
#include "Parallel/mpibarrier.h"
#include "Parallel/mpisgbuf.h"
#include "Parallel/mpisgvbuf.h"
#include "Parallel/mpivbuf.h"
#include "Model/BodyForceGroup.h"
#include "Model/DampingIGP.h"
#include "Model/EWallInteractionGroup.h"
#include "Model/LocalDampingIGP.h"
#include "Model/Particle.h"
#include "Model/RotParticle.h"
#include "Foundation/console.h"
#include "tml/comm/comm.h"

#include "esys_dem.h"

#include <map>
#include <set>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

class MpiWTimers;

template <class T>
class TGpuSubLattice : public ASubLattice {
 public:
  TGpuSubLattice(const esys::lsm::CLatticeParam& param, int rank, MPI_Comm comm, MPI_Comm worker_comm);
  virtual ~TGpuSubLattice();

  // the GPU handle (NULL before initNeighborTable)
  dem_sim* handle() const { return m_h; }

  // -- set-up --
  virtual void setTimeStepSize(double dt);
  virtual std::vector<int> getCommCoords() const { return std::vector<int>(3, 0); }
  virtual std::vector<int> getCommDims() const { return std::vector<int>(3, 1); }
  virtual void initNeighborTable(const Vec3& min, const Vec3& max);
  virtual void initNeighborTable(const Vec3& min, const Vec3& max, const std::vector<bool>& circ);
  virtual void receiveParticles();
  virtual void receiveConnections();
  virtual void addWall();
  virtual void addElasticWIG();
  virtual void addPairIG();
  virtual void addSingleIG();
  virtual void addBondedIG();
  virtual void addRotBondedIG();
  virtual void addBrittleBeamSCIG();
  virtual void addBrittleBeamDZCIG();
  virtual void addDamping();
  virtual void setExIG();

  // -- per step (CLatticeMaster::runOneStep, Parallel/LatticeMaster.cpp:2602-2740) --
  virtual void checkNeighbors();
  virtual void searchNeighbors();
  virtual void rebuildParticleArray();
  virtual void rebuildInteractions();
  virtual void updateInteractions();
  virtual void oneStep();
  virtual void exchangePos();

  // -- walls and particles during the run --
  virtual void getWallPos();
  virtual void getWallForce();
  virtual void moveWallBy();
  virtual void applyForceToWall();
  virtual void setVelocityOfWall();
  virtual void moveTaggedParticlesBy();
  virtual int getNumParticles();
  virtual void countParticles();
  virtual std::pair<double, int> findParticleNearestTo(const Vec3& pt);
  virtual std::pair<int, Vec3> getParticlePosn(int particleId);
  virtual void getParticleData(const IdVector& particleIdVector);

  // -- checkpoints (the reference's worker file layout, written by the GPU library) --
  virtual void saveCheckPointData(std::ostream& oStream);
  virtual void saveSnapShotData(std::ostream& oStream);
  virtual void loadCheckPointData(std::istream& iStream);

  // -- housekeeping --
  virtual const MPI_Comm& getWorkerComm() const { return m_worker_comm; }
  virtual void setTimer(MpiWTimers& timers) { m_pTimers = &timers; }
  virtual void do2dCalculations(bool do2d);
  virtual void printStruct();
  virtual void printData();
  virtual void printTimes() {}

  // -- not on the GPU path: each throws std::runtime_error naming itself --
  virtual void addFluidInteraction() { unsupported("addFluidInteraction"); }
  virtual void updateFluid() { unsupported("updateFluid"); }
  virtual void exchangeCells() { unsupported("exchangeCells"); }
  virtual void sendCoeffi() { unsupported("sendCoeffi"); }
  virtual void recvPressure() { unsupported("recvPressure"); }
  virtual void solveMatrix() { unsupported("solveMatrix"); }
  virtual void addBondedWIG() { unsupported("addBondedWIG"); }
  virtual void addDirBondedWIG() { unsupported("addDirBondedWIG"); }
  virtual void addViscWIG() { unsupported("addViscWIG"); }
  virtual void addTaggedElasticWIG() { unsupported("addTaggedElasticWIG"); }
  virtual void addTaggedPairIG() { unsupported("addTaggedPairIG"); }
  virtual void addTriMesh() { unsupported("addTriMesh"); }
  virtual void addTriMeshIG() { unsupported("addTriMeshIG"); }
  virtual void addBondedTriMeshIG() { unsupported("addBondedTriMeshIG"); }
  virtual void addMesh2D() { unsupported("addMesh2D"); }
  virtual void addMesh2DIG() { unsupported("addMesh2DIG"); }
  virtual void addBondedMesh2DIG() { unsupported("addBondedMesh2DIG"); }
  virtual void addCappedBondedIG() { unsupported("addCappedBondedIG"); }
  virtual void addShortBondedIG() { unsupported("addShortBondedIG"); }
  virtual void addRotThermBondedIG() { unsupported("addRotThermBondedIG"); }
  virtual void removeIG() { unsupported("removeIG"); }
  virtual void addSphereBody() { unsupported("addSphereBody"); }
  virtual void addESphereBodyIG() { unsupported("addESphereBodyIG"); }
  virtual void getSphereBodyPos() { unsupported("getSphereBodyPos"); }
  virtual void getSphereBodyForce() { unsupported("getSphereBodyForce"); }
  virtual void moveParticleTo() { unsupported("moveParticleTo"); }
  virtual void changeRadiusBy() { unsupported("changeRadiusBy"); }
  virtual void moveSingleParticleTo(int, const Vec3&) { unsupported("moveSingleParticleTo"); }
  virtual void moveSphereBodyBy() { unsupported("moveSphereBodyBy"); }
  virtual void setWallNormal() { unsupported("setWallNormal"); }
  virtual void setParticleVelocity() { unsupported("setParticleVelocity"); }
  virtual void setParticleDensity() { unsupported("setParticleDensity"); }
  virtual void resetParticleRotation() { unsupported("resetParticleRotation"); }
  virtual void setTaggedParticleVel() { unsupported("setTaggedParticleVel"); }
  virtual void setParticleNonDynamic() { unsupported("setParticleNonDynamic"); }
  virtual void setParticleNonRot() { unsupported("setParticleNonRot"); }
  virtual void tagParticleNearestTo() { unsupported("tagParticleNearestTo"); }
  virtual void moveSingleNode() { unsupported("moveSingleNode"); }
  virtual void moveTaggedNodes() { unsupported("moveTaggedNodes"); }
  virtual void translateMeshBy(const std::string&, const Vec3&) { unsupported("translateMeshBy"); }
  virtual void rotateMeshBy(const std::string&, const Vec3&, const Vec3&, double) { unsupported("rotateMeshBy"); }
  virtual void setInteractionParameter() { unsupported("setInteractionParameter"); }
  virtual void addScalarParticleField() { unsupported("addScalarParticleField"); }
  virtual void addVectorParticleField() { unsupported("addVectorParticleField"); }
  virtual void addScalarInteractionField() { unsupported("addScalarInteractionField"); }
  virtual void addScalarHistoryInteractionField() { unsupported("addScalarHistoryInteractionField"); }
  virtual void addVectorInteractionField() { unsupported("addVectorInteractionField"); }
  virtual void addVectorTriangleField() { unsupported("addVectorTriangleField"); }
  virtual void addScalarTriangleField() { unsupported("addScalarTriangleField"); }
  virtual void sendFieldData() { unsupported("sendFieldData"); }
  virtual void addVectorWallField() { unsupported("addVectorWallField"); }
  virtual void addScalarFluidField() { unsupported("addScalarFluidField"); }
  virtual void addVectorFluidField() { unsupported("addVectorFluidField"); }
  virtual void addScalarFluidInteractionField() { unsupported("addScalarFluidInteractionField"); }
  virtual void addVectorFluidInteractionField() { unsupported("addVectorFluidInteractionField"); }
  virtual void getMeshNodeRef() { unsupported("getMeshNodeRef"); }
  virtual void getMeshFaceRef() { unsupported("getMeshFaceRef"); }
  virtual void getMesh2DStress() { unsupported("getMesh2DStress"); }
  virtual void getTriMeshForce() { unsupported("getTriMeshForce"); }

 private:
  static constexpr bool kRot = std::is_same<T, CRotParticle>::value;

  // what the GPU library does not keep for a particle: the reference's record of it
  struct Record {
    int tag;
    double rad, mass;
    bool dyn, rot;
  };
  struct Row {  // one particle's state as the library reports it
    int id;
    Vec3 pos, vel, angvel, force, moment, disp;
    double quat[4];
  };

  void create(const Vec3& min, const Vec3& max, const int circ[3]);
  void need_handle(const char* what) const;
  void check(int rc, const char* what) const;
  [[noreturn]] void unsupported(const char* what) const;
  std::vector<Row> rows();
  T make_particle(const Row& r) const;
  Vec3 wall_vector(const std::string& name, bool force);

  dem_sim* m_h;
  double m_nrange, m_alpha, m_dt;
  int m_rank;
  MPI_Comm m_comm, m_worker_comm;
  TML_Comm m_tml_comm;
  MpiWTimers* m_pTimers;
  std::map<int, Record> m_record;             // by particle id
  std::set<std::string> m_walls, m_wall_groups, m_bonded, m_dynamic;
};

#include "GpuSubLattice.hpp"

#endif
