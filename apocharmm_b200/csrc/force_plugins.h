// Extra force terms that a ForceManager evaluates with every force call:
// the reference's ForceView plug-in point (include/ForceManager.h:37-105,
// ForceManager::subscribe/unsubscribe :420-475; evaluated in
// src/ForceManager.cu:530-540, 596-620, 678-740), and the harmonic
// positional restraint that plugs into it (include/HarmonicRestraintForce.h,
// src/HarmonicRestraintForce.cu).
//
// The reference gives every plug-in its own stream, force buffer and energy
// table and adds them into the total on the host.  Here a plug-in adds its
// gradient straight into the manager's fixed-point buffer (gradient slots
// in neighbour-list order) and its energy into a fixed-point slot of its
// own, on the manager's stream, so it is part of every captured MD segment
// and the total stays independent of the order of the additions.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <string>
#include <vector>

namespace apo {

struct ForcePluginArgs {
  int natom;
  const double4 *coords;  // FP64 state (x, y, z, q), atom order
  const float4 *xyzq;     // single-precision copy, atom order
  const int *glo2loc;     // atom -> gradient slot
  long long *force;       // fixed-point gradient (2^40), x/y/z planes of `stride`
  int stride;
  long long *energy;      // this plug-in's fixed-point energy slot (2^32)
  double box[3];          // orthorhombic cell edges
};

class ForcePlugin {
 public:
  virtual ~ForcePlugin() = default;
  // called when the plug-in joins an initialised manager, and again when the
  // manager is (re)initialised
  virtual void initialize(int natom, const std::array<double, 3> &box) = 0;
  // adds the gradient (and the energy when calcEnergy) on stream s; must not
  // synchronise or allocate (it runs inside captured CUDA graphs)
  virtual void calcForce(const ForcePluginArgs &a, bool calcEnergy, bool calcVirial,
                         cudaStream_t s) = 0;
};

// E = sum_i k_i m_i |r_i - r0_i|^2 over the selected atoms, gradient
// 2 k_i m_i (r_i - r0_i), masses 1 unless set
// (src/HarmonicRestraintForce.cu:242-290).  r_i - r0_i is taken as its
// nearest periodic image: the integrator wraps molecules back into the box
// at every list update, and the reference's plain difference would then
// turn into a box length; for displacements below half a box edge both are
// the same.  An absolute restraint has no internal virial (the reference
// leaves it out for the same reason).
class HarmonicRestraintForce : public ForcePlugin {
 public:
  explicit HarmonicRestraintForce(int natom);
  ~HarmonicRestraintForce() override;
  int getNumAtoms() const { return m_N; }
  // atoms outside the selection get force constant 0 (as the reference's
  // setSelection); the selection starts empty
  void setSelection(const std::vector<int> &atoms);
  // k for every selected atom, 0 elsewhere
  void setForceConstant(double k);
  // k_i for the selected atoms (one value per atom), 0 elsewhere
  void setForceConstants(const std::vector<double> &k);
  void setReferenceCoordinates(const std::vector<double> &xyz);  // N x 3
  void setMasses(const std::vector<double> &m);
  // scales the reference positions with a change of box (as the reference)
  void setBoxDimensions(const std::array<double, 3> &box);

  void initialize(int natom, const std::array<double, 3> &box) override;
  void calcForce(const ForcePluginArgs &a, bool calcEnergy, bool calcVirial,
                 cudaStream_t s) override;

 private:
  // the compact list of restrained atoms, rewritten in place whenever a
  // setter runs after initialize(): the buffers never move and the count
  // lives on the device, so captured graphs see every change
  void upload();
  int m_N;
  std::vector<char> m_Selected;
  std::vector<double> m_K;
  std::vector<double> m_Ref;   // x, y, z, mass per atom
  std::array<double, 3> m_Box{{0.0, 0.0, 0.0}};
  int *m_Count = nullptr;      // device: number of restrained atoms
  int *m_Atoms = nullptr;      // device: restrained atoms (capacity N)
  double4 *m_Target = nullptr; // device: (x0, y0, z0, k m) per restrained atom
};

// A force term evaluated by the caller's own code, reached through a table
// of plain functions: the reference's ForceView type erasure
// (include/ForceManager.h:37-105) across the C ABI.  Each call forks the
// caller's stream from the manager's, lets the caller clear and evaluate
// its term there, joins back, and adds the caller's atom-order fixed-point
// gradient (2^40, x/y/z planes) and the sum of its FP64 energies into the
// manager's buffers (src/ForceManager.cu:596-620 and 678-690 do the same
// through per-force streams and a host-side total).  The caller's virial is
// not added: the reference computes it from the force buffers only for the
// pressure, which no integrator here reads from plug-ins.
struct ExternalForceOps {
  void *object = nullptr;
  void (*initialize)(void *object, int num_atoms, const double *box3) = nullptr;
  void (*clear)(void *object) = nullptr;
  void (*calc_force)(void *object, const float *d_xyzq, int calc_energy, int calc_virial) = nullptr;
  const long long *(*get_force)(void *object, int *stride) = nullptr;
  const double *(*get_energies)(void *object, int *count) = nullptr;
  cudaStream_t stream = nullptr;
};

class ExternalForce : public ForcePlugin {
 public:
  explicit ExternalForce(const ExternalForceOps &ops);
  ~ExternalForce() override;
  void initialize(int natom, const std::array<double, 3> &box) override;
  void calcForce(const ForcePluginArgs &a, bool calcEnergy, bool calcVirial,
                 cudaStream_t s) override;
  const void *object() const { return m_Ops.object; }

 private:
  ExternalForceOps m_Ops;
  cudaEvent_t m_Fork = nullptr, m_Join = nullptr;
};

}  // namespace apo
