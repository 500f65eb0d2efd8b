// CharmmCrd and CharmmContext: coordinates files and the simulation state
// of one system (the reference's include/CharmmCrd.h and
// include/CharmmContext.h:69-366: setCoordinates, getCoordinates,
// assignVelocitiesAtTemperature, setRandomSeedForVelocities,
// useHolonomicConstraints, computeTemperature, calculatePotentialEnergy,
// getForces, getDegreesOfFreedom, getForceManager), header-only over the
// C ABI.  The context keeps the ForceManager it is built on alive.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "apocharmm/Check.h"
#include "apocharmm/Force.h"
#include "apocharmm/ForceManager.h"
#include "apocharmm_c/CharmmContext.h"
#include "apocharmm_c/CharmmCrd.h"
#include "apocharmm_c/ForceView.h"

class CharmmCrd {
 public:
  explicit CharmmCrd(const std::string &fileName) {
    apocharmm_detail::check(apo_charmm_crd_create(&m_H, fileName.c_str()));
  }
  ~CharmmCrd() { apo_charmm_crd_destroy(m_H); }
  CharmmCrd(const CharmmCrd &) = delete;
  CharmmCrd &operator=(const CharmmCrd &) = delete;
  int getNumAtoms() const {
    size_t n = 0;
    apocharmm_detail::check(apo_charmm_crd_get_num_atoms(&n, m_H));
    return (int)n;
  }
  // one (x, y, z) per atom
  std::vector<std::vector<double>> getCoordinates() const {
    const int n = getNumAtoms();
    std::vector<double> flat(3 * (size_t)n);
    apocharmm_detail::check(apo_charmm_crd_get_coordinates(flat.data(), flat.size(), m_H));
    std::vector<std::vector<double>> out(n);
    for (int i = 0; i < n; ++i) out[i] = {flat[3 * i], flat[3 * i + 1], flat[3 * i + 2]};
    return out;
  }
  const apo_charmm_crd *handle() const { return m_H; }

 private:
  apo_charmm_crd *m_H = nullptr;
};

class CharmmContext {
 public:
  explicit CharmmContext(std::shared_ptr<ForceManager> fmIn) : m_Fm(std::move(fmIn)) {
    if (!m_Fm) throw std::invalid_argument("CharmmContext: null ForceManager");
    apocharmm_detail::check(apo_charmm_context_create(&m_H, m_Fm->handle()));
  }
  ~CharmmContext() { apo_charmm_context_destroy(m_H); }
  CharmmContext(const CharmmContext &) = delete;
  CharmmContext &operator=(const CharmmContext &) = delete;

  void setCoordinates(const std::shared_ptr<CharmmCrd> crd) {
    if (!crd) throw std::invalid_argument("setCoordinates: null coordinates");
    apocharmm_detail::check(apo_charmm_context_set_coordinates(m_H, crd->handle()));
  }
  // (x, y, z, w) per atom; w is not used (the charges are the PSF's)
  void setCoordinates(const std::vector<double4> &coords) {
    std::vector<double> flat(3 * coords.size());
    for (size_t i = 0; i < coords.size(); ++i) {
      flat[3 * i] = coords[i].x;
      flat[3 * i + 1] = coords[i].y;
      flat[3 * i + 2] = coords[i].z;
    }
    apocharmm_detail::check(apo_charmm_context_set_coordinates_xyz(m_H, flat.data(), flat.size()));
  }
  std::vector<std::vector<double>> getCoordinates() {
    const int n = getNumAtoms();
    std::vector<double> flat(3 * (size_t)n);
    apocharmm_detail::check(apo_charmm_context_get_coordinates(flat.data(), flat.size(), m_H));
    std::vector<std::vector<double>> out(n);
    for (int i = 0; i < n; ++i) out[i] = {flat[3 * i], flat[3 * i + 1], flat[3 * i + 2]};
    return out;
  }
  // (vx, vy, vz) per atom, A/ps
  void assignVelocities(const std::vector<double> &velIn) {
    apocharmm_detail::check(apo_charmm_context_set_velocities(m_H, velIn.data(), velIn.size()));
  }
  std::vector<double> getVelocities() {
    std::vector<double> v(3 * (size_t)getNumAtoms());
    apocharmm_detail::check(apo_charmm_context_get_velocities(v.data(), v.size(), m_H));
    return v;
  }
  void setRandomSeedForVelocities(uint64_t seed) {
    apocharmm_detail::check(apo_charmm_context_set_random_seed_for_velocities(m_H, seed));
  }
  void assignVelocitiesAtTemperature(float temp) {
    apocharmm_detail::check(apo_charmm_context_assign_velocities_at_temperature(m_H, temp));
  }
  void useHolonomicConstraints(bool flag) {
    apocharmm_detail::check(apo_charmm_context_use_holonomic_constraints(m_H, flag));
  }
  float computeTemperature() {
    double t = 0.0;
    apocharmm_detail::check(apo_charmm_context_compute_temperature(&t, m_H));
    return (float)t;
  }
  int getNumAtoms() const {
    size_t n = 0;
    apocharmm_detail::check(apo_charmm_context_get_num_atoms(&n, m_H));
    return (int)n;
  }
  int getDegreesOfFreedom() const {
    int n = 0;
    apocharmm_detail::check(apo_charmm_context_get_degrees_of_freedom(&n, m_H));
    return n;
  }
  void resetNeighborList() { apocharmm_detail::check(apo_charmm_context_reset_neighbor_list(m_H)); }
  // energies and virial at the current coordinates (reset: rebuild the list)
  void calculatePotentialEnergy(bool reset = false, bool print = false) {
    apocharmm_detail::check(apo_charmm_context_calculate_forces(m_H, reset, true, true));
    if (print) {
      for (auto &kv : getEnergyComponents())
        std::printf("%-8s %16.6f\n", kv.first.c_str(), kv.second);
    }
  }
  float getPotentialEnergies() {
    double e = 0.0;
    apocharmm_detail::check(apo_charmm_context_get_potential_energy(&e, m_H));
    return (float)e;
  }
  std::map<std::string, double> getEnergyComponents() {
    const auto &names = ForceManager::energyTermNames();
    std::vector<double> e(names.size());
    apocharmm_detail::check(apo_charmm_context_get_energy_components(e.data(), e.size(), m_H));
    std::map<std::string, double> m;
    for (size_t k = 0; k < names.size(); ++k) m[names[k]] = e[k];
    return m;
  }
  // gradient of the last evaluation (device planes, atom order)
  std::shared_ptr<Force<double>> getForces() {
    if (!m_Forces) m_Forces = std::make_shared<Force<double>>();
    const int n = getNumAtoms();
    if (m_Forces->size() != n) m_Forces->realloc(n);
    void *s = nullptr;
    apocharmm_detail::check(apo_charmm_context_get_stream(&s, m_H));
    apocharmm_detail::check(
        apo_force_manager_get_forces_device(m_Forces->xyz(), m_Forces->stride(), m_Fm->handle(), s));
    apocharmm_detail::cuda_check(cudaStreamSynchronize((cudaStream_t)s), "CharmmContext::getForces");
    return m_Forces;
  }
  std::vector<double> &getBoxDimensions(void) { return m_Fm->getBoxDimensions(); }
  std::shared_ptr<ForceManager> getForceManager() { return m_Fm; }
  apo_charmm_context *handle() { return m_H; }

 private:
  std::shared_ptr<ForceManager> m_Fm;
  apo_charmm_context *m_H = nullptr;
  std::shared_ptr<Force<double>> m_Forces;
};
