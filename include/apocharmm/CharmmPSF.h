// CharmmPSF and CharmmParameters: the topology and the force-field files a
// ForceManager is built from (the reference's include/CharmmPSF.h and
// include/CharmmParameters.h constructors and counts), over the C handles.
#pragma once

#include <cstddef>
#include <string>
#include <vector>

#include "apocharmm/Check.h"
#include "apocharmm_c/CharmmParameters.h"
#include "apocharmm_c/CharmmPsf.h"

class CharmmPSF {
 public:
  explicit CharmmPSF(const std::string &fileName) {
    apocharmm_detail::check(apo_charmm_psf_create(&m_H, fileName.c_str()));
  }
  ~CharmmPSF() { apo_charmm_psf_destroy(m_H); }
  CharmmPSF(const CharmmPSF &) = delete;
  CharmmPSF &operator=(const CharmmPSF &) = delete;

  int getNumAtoms() const { return (int)count(apo_charmm_psf_get_num_atoms); }
  int getNumBonds() const { return (int)count(apo_charmm_psf_get_num_bonds); }
  int getNumAngles() const { return (int)count(apo_charmm_psf_get_num_angles); }
  int getNumDihedrals() const { return (int)count(apo_charmm_psf_get_num_dihedrals); }
  int getNumImpropers() const { return (int)count(apo_charmm_psf_get_num_impropers); }
  std::vector<double> getCharges() const {
    std::vector<double> q(getNumAtoms());
    apocharmm_detail::check(apo_charmm_psf_get_charges(q.data(), q.size(), m_H));
    return q;
  }
  std::vector<double> getMasses() const {
    std::vector<double> m(getNumAtoms());
    apocharmm_detail::check(apo_charmm_psf_get_masses(m.data(), m.size(), m_H));
    return m;
  }
  const apo_charmm_psf *handle() const { return m_H; }

 private:
  size_t count(apo_status (*f)(size_t *, const apo_charmm_psf *)) const {
    size_t n = 0;
    apocharmm_detail::check(f(&n, m_H));
    return n;
  }
  apo_charmm_psf *m_H = nullptr;
};

class CharmmParameters {
 public:
  explicit CharmmParameters(const std::string &fileName) {
    apocharmm_detail::check(apo_charmm_parameters_create(&m_H, fileName.c_str()));
  }
  explicit CharmmParameters(const std::vector<std::string> &fileNames) {
    std::vector<const char *> p;
    for (auto &f : fileNames) p.push_back(f.c_str());
    apocharmm_detail::check(apo_charmm_parameters_create_from_files(&m_H, p.data(), p.size()));
  }
  ~CharmmParameters() { apo_charmm_parameters_destroy(m_H); }
  CharmmParameters(const CharmmParameters &) = delete;
  CharmmParameters &operator=(const CharmmParameters &) = delete;
  const apo_charmm_parameters *handle() const { return m_H; }

 private:
  apo_charmm_parameters *m_H = nullptr;
};
