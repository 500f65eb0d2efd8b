// Integrators: Langevin thermostat, Nose-Hoover and leapfrog, with SETTLE
// (TIP3 water) and SHAKE (X-H clusters) in FP64.
//
// Mirror the reference's CudaIntegrator hierarchy (src/CudaIntegrator.cu,
// src/CudaLangevinThermostatIntegrator.cu, src/CudaNoseHooverIntegrator.cu,
// src/CudaLeapFrogIntegrator.cu, constraints src/CudaHolonomicConstraint.cu):
// same position-Verlet "delta" formulation, same thermostat algebra, same
// Philox stream per atom (curand_init(seed, atom, 0) + skipahead(4*step) +
// curand_normal4), same 20-step list cadence and 1000-step centre-of-mass
// removal.  Differences by design:
//   * one thread owns a whole constraint group (a water, an X-H cluster or a
//     run of free atoms), so the position update, the constraint, the
//     velocity update, the kinetic-energy partial sums and the refresh of the
//     sorted single-precision coordinates are one kernel;
//   * reductions finish in the last block of the grid (fixed summation order,
//     no host round trip), and the step counter and RNG position live on the
//     device;
//   * `propagate` runs whole list-update segments (rebuild + 20 steps) as
//     captured CUDA graphs.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "engine.h"
#include "restart.h"
#include "subscribers.h"

namespace apo {

struct IntegratorState;  // device buffers, defined in integrators.cu

class CudaIntegrator : public std::enable_shared_from_this<CudaIntegrator> {
 public:
  explicit CudaIntegrator(double timeStepPs);
  virtual ~CudaIntegrator();

  double getTimeStep() const { return m_Dt * kTimfac; }
  void setTimeStep(double ps);
  void setCharmmContext(std::shared_ptr<CharmmContext> ctx);
  std::shared_ptr<CharmmContext> getCharmmContext() const { return m_Ctx; }
  void setNonbondedListUpdateFrequency(int f);
  // 0 switches the removal off (always off for a multi-system context)
  void setRemoveCenterOfMassFrequency(int f) { m_ComFreq = f < 0 ? 0 : f; clearGraphs(); }
  void setUseGraphs(bool g) { m_UseGraphs = g; }
  void subscribe(std::shared_ptr<Subscriber> sub);
  // stops the reports of one subscriber (src/CudaIntegrator.cu unsubscribe);
  // true when it was subscribed
  bool unsubscribe(const std::shared_ptr<Subscriber> &sub);
  virtual void propagate(int numSteps);
  long long getCurrentPropagatedStep() const { return m_Step; }
  double getInstantaneousTemperature();  // "Jung" estimate of the last step
  double getAverageTemperature();
  void resetAverageTemperature();
  cudaStream_t stream() const;
  // number of kernels one step and one list update launch (for accounting)
  int kernelsPerStep() const { return m_KernelsPerStep; }
  int kernelsPerRebuild() const;
  // position-Verlet state: the last displacement of every atom (device)
  double4 *deltaState() const;
  // several systems (Langevin): every system's noise position at the start
  // of this integrator and its step limit from then on; a system past its
  // limit is not advanced (its forces are still evaluated)
  void setSystemLimits(const std::vector<unsigned long long> &rng0,
                       const std::vector<long long> &stop);
  // steps taken by this integrator, read from the device counter
  long long deviceStep();
  // the state a restart file carries (Langevin thermostat and Nose-Hoover
  // only, as in src/RestartSubscriber.cu:53-68; one system)
  RestartRecord restartRecord();
  // continue the run a restart file describes: coordinates, velocities,
  // the position-Verlet delta, the step counters and the thermostat seed
  // and RNG position (Langevin) or piston velocity and force (Nose-Hoover)
  // (src/CudaLangevinThermostatIntegrator.cu:264-545,
  // src/CudaNoseHooverIntegrator.cu:337-615).  The context must already
  // hold the box of the file.
  void initializeFromRestartFile(const std::string &path);

 protected:
  virtual void initialize() = 0;
  virtual void stepKernels(cudaStream_t s) = 0;  // the integration after forces
  void segment(int nsteps, cudaStream_t s);      // rebuild + nsteps steps
  void launchSegment(int nsteps, cudaStream_t s);  // as a captured graph (cached) or eagerly
  virtual void forcesForStep(cudaStream_t s);
  virtual void beforeReport() {}  // host state the subscribers read, after a synchronisation
  double m_Dt;  // AKMA
  int m_ListFreq = 20, m_ComFreq = 1000;
  bool m_UseGraphs = true;
  bool m_Initialized = false;
  long long m_Step = 0;
  int m_KernelsPerStep = 0;
  int m_PluginGen = -1;  // plug-in set the graphs were captured with
  std::shared_ptr<CharmmContext> m_Ctx;
  std::unique_ptr<IntegratorState> m_S;
  std::map<int, cudaGraphExec_t> m_Graphs;
  std::vector<std::shared_ptr<Subscriber>> m_Subscribers;
  void buildGroups();
  void clearGraphs();
};

class CudaLangevinThermostatIntegrator : public CudaIntegrator {
 public:
  explicit CudaLangevinThermostatIntegrator(double timeStepPs);
  void setThermostatFriction(double frictionPerPs);
  double getThermostatFriction() const { return m_Friction; }
  // a setting change drops the captured segments, which hold the old value
  void setReferenceTemperature(double t) { m_RefT = t; clearGraphs(); }
  double getReferenceTemperature() const { return m_RefT; }
  void setThermostatRngSeed(uint64_t seed) { m_Seed = seed; clearGraphs(); }
  uint64_t getThermostatRngSeed() const { return m_Seed; }
  unsigned long long getRngSequencePos();

 protected:
  void initialize() override;
  void stepKernels(cudaStream_t s) override;
  double m_Friction = 0.0, m_RefT = 300.0;
  uint64_t m_Seed;
};

class CudaNoseHooverIntegrator : public CudaIntegrator {
 public:
  explicit CudaNoseHooverIntegrator(double timeStepPs);
  void setReferenceTemperature(double t) { m_RefT = t; clearGraphs(); }
  double getReferenceTemperature() const { return m_RefT; }
  void setNoseHooverPistonMass(double m);
  void useOldTemperature(bool f) { m_OldT = f; clearGraphs(); }

 protected:
  void initialize() override;
  void stepKernels(cudaStream_t s) override;
  double m_RefT = 300.0, m_PistonMass = -9999.9999;
  bool m_OldT = false;
};

// Constant pressure: Langevin piston on the box edges (Feller, Zhang, Pastor
// & Brooks, J. Chem. Phys. 103, 4613 (1995)) with an optional Nose-Hoover
// thermostat, after src/CudaLangevinPistonIntegrator.cu:1705-2060: a half
// step, the constraint forces and their virial, the pressure tensor from
// the half-step kinetic terms and the virial, then predictor-corrector
// passes that move the piston (one Philox normal per piston degree of
// freedom and pass, curand_init(seed, dof, 0) + skipahead), the thermostat
// and the atoms together, the constraints applied to the new and the scaled
// reference positions, and the on-step velocities.  Cubic, tetragonal and
// orthorhombic cells.  The box lives in device memory (the force manager's
// device box, its direct-space set-up and its list dims, all rewritten by
// the last kernel of the step; the list's periodic shifts follow the box
// between builds), so piston steps run as captured 20-step segments like
// the other integrators; the host copies are brought up to date after
// every segment a subscriber reports on and at the end of propagate.
enum class Crystal : int { None = 0, Cubic = 1, Orthorhombic = 2, Tetragonal = 3 };

struct PistonState;  // device scalars, defined in integrators.cu

class CudaLangevinPistonIntegrator : public CudaIntegrator {
 public:
  explicit CudaLangevinPistonIntegrator(double timeStepPs);
  ~CudaLangevinPistonIntegrator() override;
  void setCrystalType(Crystal c);
  Crystal getCrystalType() const { return m_Crystal; }
  int getPistonDegreesOfFreedom() const { return m_Dof; }
  // reference pressure tensor (atm), row-major XX XY XZ YX YY YZ ZX ZY ZZ
  void setPressure(const std::vector<double> &p);
  std::vector<double> getReferencePressureTensor() const { return m_Pref; }
  void setConstantSurfaceTension(bool f) { m_ConstST = f; clearGraphs(); }
  void setSurfaceTension(double dyneCm) { m_SurfaceTension = dyneCm; clearGraphs(); }
  // amu, one per piston degree of freedom; default 0.02 x total mass
  void setLangevinPistonMass(const std::vector<double> &m);
  std::vector<double> getLangevinPistonMass() const { return m_PMass; }
  void setLangevinPistonFriction(double perPs) { m_PGamma = perPs; clearGraphs(); }
  double getLangevinPistonFriction() const { return m_PGamma; }
  void setLangevinPistonFrictionSeed(uint64_t seed);
  uint64_t getLangevinPistonFrictionSeed() const { return m_Seed; }
  void setRngSequencePos(unsigned long long pos);
  unsigned long long getRngSequencePos();
  void setReferenceTemperature(double t) { m_RefT = t; clearGraphs(); }
  double getReferenceTemperature() const { return m_RefT; }
  void useNoseHooverThermostat(bool f) { m_UseNH = f; clearGraphs(); }
  void setNoseHooverPistonMass(double m);
  double getNoseHooverPistonMass() const { return m_NHMass; }
  void useOldTemperature(bool f) { m_OldT = f; clearGraphs(); }
  void setMaxPredictorCorrectorIterations(int n);
  int getMaxPredictorCorrectorIterations() const { return m_MaxPC; }
  void resetAverages();
  // pressure tensor (atm) of the last step and its running average
  std::vector<double> getInstantaneousPressureTensor();
  double getInstantaneousPressureScalar();
  std::vector<double> getAveragePressureTensor();
  double getAveragePressureScalar();
  // piston positions (box edges, A) and their last displacement
  std::vector<double> getLangevinPistonOnStepPosition();
  std::vector<double> getLangevinPistonDeltaPosition();
  std::vector<double> getLangevinPistonHalfStepPosition();
  std::vector<double> getLangevinPistonOnStepVelocity();
  std::vector<double> getLangevinPistonDeltaPressure();
  // surface tension of the last step, dyne/cm (getInstantaneousSurfaceTension)
  double getInstantaneousSurfaceTension();
  // the thermostat piston: velocity, its value one step back, the velocity
  // change ("force") and its value one step back
  // (set/getNoseHooverPiston{Velocity,VelocityPrevious,Force,ForcePrevious})
  std::vector<double> getNoseHooverPistonState();
  void setNoseHooverPistonState(double v, double v_prev, double f, double f_prev);
  void propagate(int numSteps) override;
  // the piston part of a restart record (crystal tag, HDOT, box, seed and
  // RNG position), after the base class has restored the atoms and the
  // thermostat (src/CudaLangevinPistonIntegrator.cu:706-1020)
  void applyRestartRecord(const RestartRecord &r);

 protected:
  void initialize() override;
  void stepKernels(cudaStream_t s) override;
  void forcesForStep(cudaStream_t s) override;  // with the virial
  void beforeReport() override;
  void adoptBox();  // the device's box into the force manager's host copies
  Crystal m_Crystal = Crystal::None;
  int m_Dof = -1, m_MaxPC = 3;
  std::vector<double> m_Pref{1, 0, 0, 0, 1, 0, 0, 0, 1};
  std::vector<double> m_PMass;
  double m_PGamma = 0.0, m_RefT = 300.0, m_NHMass = -9999.9999, m_SurfaceTension = 0.0;
  bool m_UseNH = true, m_OldT = false, m_ConstST = false;
  uint64_t m_Seed;
  unsigned long long m_RngPos = 0;
  bool m_RngDirty = true;
  std::unique_ptr<PistonState> m_P;
};

class CudaLeapFrogIntegrator : public CudaIntegrator {
 public:
  explicit CudaLeapFrogIntegrator(double timeStepPs);

 protected:
  void initialize() override;
  void stepKernels(cudaStream_t s) override;
};

}  // namespace apo
