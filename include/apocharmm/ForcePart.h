// One part of a ForceManager's force field as a force object of its own:
// the base of CudaBondedForce, CudaPMEDirectForce and CudaPMEReciprocalForce.
//
// The reference builds each part as a separate object with its own force
// buffer, stream and energy table (src/ForceManager.cu:430-545).  Here the
// parts share the manager's topology, list and buffers; a part's
// calc_force evaluates only its own terms through the manager and copies
// the gradient into the part's Force<long long int> (2^40 fixed point, atom
// order) and its energies (and virial) into the part's CudaEnergyVirial.
// The manager's own results then hold that part alone.  A part has the
// ForceView members, so it can also be subscribed to another manager.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "apocharmm/CudaEnergyVirial.h"
#include "apocharmm/Force.h"
#include "apocharmm/ForceManager.h"

class ForcePart {
 public:
  ForcePart(std::shared_ptr<ForceManager> fm, int components, std::vector<std::string> terms)
      : m_Fm(std::move(fm)), m_Components(components), m_Terms(std::move(terms)) {
    if (!m_Fm) throw std::invalid_argument("force part: null ForceManager");
    m_Force = std::make_shared<Force<long long int>>(m_Fm->getNumAtoms());
    m_EnergyVirial = std::make_shared<CudaEnergyVirial>();
    for (auto &t : m_Terms) m_EnergyVirial->insert(t);
  }
  virtual ~ForcePart() = default;

  // (numAtoms, box): the manager's box, then its initialisation
  void initialize(const int numAtoms, const std::vector<double> &boxDimensions) {
    if (numAtoms != m_Fm->getNumAtoms())
      throw std::invalid_argument("force part: atom count differs from the ForceManager's");
    m_Fm->setBoxDimensions(boxDimensions);
    m_Fm->initialize();
    if (m_Force->size() != numAtoms) m_Force->realloc(numAtoms);
  }
  void setBoxDimensions(const std::vector<double> &boxDimensions) {
    m_Fm->setBoxDimensions(boxDimensions);
  }
  void clear(void) {
    m_Force->clear(*m_Fm->getForceManagerStream());
    m_EnergyVirial->clear(*m_Fm->getForceManagerStream());
  }
  void calc_force(const float4 *xyzq, bool calcEnergy, bool calcVirial) {
    m_Fm->evaluate(xyzq, false, calcEnergy || calcVirial, calcVirial, m_Components);
    m_Fm->getForceValues(*m_Force);
    if (calcEnergy || calcVirial) {
      std::vector<double> w;
      if (calcVirial) w = m_Fm->getVirial();
      m_EnergyVirial->set(m_Fm->getEnergyComponents(), calcVirial ? w.data() : nullptr);
    }
  }
  void calcForce(const float4 *xyzq, bool calcEnergy, bool calcVirial) {
    calc_force(xyzq, calcEnergy, calcVirial);
  }
  // rebuilds the manager's tile list from these coordinates
  void resetNeighborList(const float4 *xyzq) { m_Fm->resetNeighborList(xyzq); }

  std::shared_ptr<Force<long long int>> getForce(void) { return m_Force; }
  std::shared_ptr<CudaEnergyVirial> getEnergyVirial(void) { return m_EnergyVirial; }
  std::shared_ptr<ForceManager> getForceManager(void) { return m_Fm; }
  int getComponents() const { return m_Components; }

 private:
  std::shared_ptr<ForceManager> m_Fm;
  int m_Components;
  std::vector<std::string> m_Terms;
  std::shared_ptr<Force<long long int>> m_Force;
  std::shared_ptr<CudaEnergyVirial> m_EnergyVirial;
};
