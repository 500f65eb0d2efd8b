// Many independent systems advanced together on one GPU.
//
// A Batch owns one multi-system ForceManager, one CharmmContext over the
// concatenated atoms and one Langevin integrator: every stage of a step
// (direct space, the five PME stages, bonded terms, the integrator) is one
// launch for all systems, and a whole list-update segment (rebuild + 20
// steps) is one captured CUDA graph.  Each system keeps its own box,
// cutoffs, PME grid, LJ tables, velocity seed and noise stream, so its
// trajectory is the same alone and in any batch.  The tiles per direct-space
// work item are chosen by a measured sweep (autotune).
//
// No counterpart class in the reference (it runs one system per
// CharmmContext); the per-system physics is the reference's.
#pragma once

#include <memory>
#include <vector>

#include "engine.h"
#include "integrators.h"

namespace apo {

class Batch {
 public:
  Batch(int order = 4, int tilesPerWork = 8, bool precise = false);
  int addSystem(const SystemSpec &spec);  // returns the system index
  void initialize();
  bool isInitialized() const { return (bool)m_Ctx; }
  int numSystems() const { return (int)m_Specs.size(); }
  int numAtoms(int sys) const;            // sys < 0: all systems
  int atomOffset(int sys) const;

  void setCoordinates(int sys, const double *xyz);
  void getCoordinates(int sys, double *xyz);
  void setVelocities(int sys, const double *v);
  void getVelocities(int sys, double *v);
  // a system's state kept on the device: coordinates, velocities and the
  // integrator's position-Verlet delta, 3 x numAtoms(sys) double4 at dst
  // (the delta part is zero while no integrator exists); loadState puts all
  // three back (the delta only when an integrator exists).  Synchronous.
  void saveState(int sys, double4 *dst);
  void loadState(int sys, const double4 *src);
  void assignVelocities(double temperature);
  void setLangevin(double dtPs, double frictionPerPs, double temperature, uint64_t seed);
  // create the Langevin integrator now (it is otherwise created by the first
  // propagate); it initialises every system's delta state from its velocities
  void createIntegrator();
  void propagate(int steps);
  void calculateForces(bool energy, bool virial);
  std::map<std::string, double> energyComponents(int sys);
  void getForces(int sys, double *xyz);
  std::vector<double> temperatures();
  // time `steps` steps for each direct-space kernel form and each candidate
  // tiles-per-work-item value and keep the fastest pair; returns the tiles
  // per work item (the state is restored afterwards)
  int autotune(int steps, const std::vector<int> &candidates);
  int tilesPerWork() const { return m_Tpw; }
  int directKernel() const { return m_Form; }
  std::shared_ptr<CharmmContext> context() const { return m_Ctx; }
  std::shared_ptr<ForceManager> forceManager() const { return m_Fm; }
  std::shared_ptr<CudaLangevinThermostatIntegrator> integrator() const { return m_Integ; }

 private:
  void requireInit() const;
  void requireSys(int sys) const;
  int m_Order, m_Tpw, m_Form = kNbTileBatches;
  bool m_Precise;
  std::vector<SystemSpec> m_Specs;
  std::shared_ptr<ForceManager> m_Fm;
  std::shared_ptr<CharmmContext> m_Ctx;
  std::shared_ptr<CudaLangevinThermostatIntegrator> m_Integ;
  double m_Dt = 0.002, m_Friction = 1.0, m_Temp = 300.0;
  uint64_t m_Seed = 1;
  std::vector<double> m_Forces;
};

}  // namespace apo
