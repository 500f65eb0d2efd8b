// CudaEnergyVirial: named energy terms and a 3x3 virial, in device memory
// with a host copy (the reference's CudaEnergyVirial, include/CudaEnergyVirial.h:29-150,
// and its EnergyVirial base, include/EnergyVirial.h).
//
// Terms are inserted by name; the device array holds one double per term,
// followed by the 9 virial doubles (row major).  A ForceView's
// getEnergyVirial() returns one of these; the force manager adds the sum of
// its energies to the energy named by the subscription tag.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "apocharmm/Check.h"

class CudaEnergyVirial {
 public:
  CudaEnergyVirial() = default;
  ~CudaEnergyVirial() {
    if (m_Dev) cudaFree(m_Dev);
  }
  CudaEnergyVirial(const CudaEnergyVirial &) = delete;
  CudaEnergyVirial &operator=(const CudaEnergyVirial &) = delete;

  // adds a term (the device array is re-allocated and cleared)
  void insert(const std::string &name) {
    if (m_Index.count(name)) return;
    m_Index[name] = (int)m_Names.size();
    m_Names.push_back(name);
    m_Host.assign(m_Names.size() + 9, 0.0);
    if (m_Dev) cudaFree(m_Dev);
    m_Dev = nullptr;
    apocharmm_detail::cuda_check(cudaMalloc(&m_Dev, m_Host.size() * sizeof(double)),
                                 "CudaEnergyVirial::insert");
    apocharmm_detail::cuda_check(cudaMemset(m_Dev, 0, m_Host.size() * sizeof(double)),
                                 "CudaEnergyVirial::insert");
  }
  void insert(const char *name) { insert(std::string(name)); }
  int getN() const { return (int)m_Names.size(); }
  const std::vector<std::string> &getNames() const { return m_Names; }

  void clear(cudaStream_t stream = 0) { clearRange(0, (int)m_Host.size(), stream); }
  void clearEnergy(cudaStream_t stream = 0) { clearRange(0, getN(), stream); }
  void clearVirial(cudaStream_t stream = 0) { clearRange(getN(), 9, stream); }
  void clearEtermDevice(const std::string &name, cudaStream_t stream = 0) {
    clearRange(index(name), 1, stream);
  }

  // device pointers
  double *getEnergyPointer(const int idx = 0) { return m_Dev + checked(idx); }
  double *getEnergyPointer(const std::string &name) { return m_Dev + index(name); }
  double *getVirialPointer() { return m_Dev + getN(); }
  const double *deviceData() const { return m_Dev; }

  // device -> host copy, then the getters below read the host copy
  void copyToHost(cudaStream_t stream = 0) {
    if (!m_Dev) return;
    apocharmm_detail::cuda_check(cudaMemcpyAsync(m_Host.data(), m_Dev,
                                                 m_Host.size() * sizeof(double),
                                                 cudaMemcpyDeviceToHost, stream),
                                 "CudaEnergyVirial::copyToHost");
    apocharmm_detail::cuda_check(cudaStreamSynchronize(stream), "CudaEnergyVirial::copyToHost");
  }
  double getEnergy(const int idx = 0) const { return m_Host[checked(idx)]; }
  double getEnergy(const std::string &name) const { return m_Host[index(name)]; }
  double getEnergy(const char *name) const { return getEnergy(std::string(name)); }
  void getVirial(double *virmat) const {
    for (int k = 0; k < 9; ++k) virmat[k] = m_Host[getN() + k];
  }

  // sets host and device values at once (used by the part views)
  void set(const std::map<std::string, double> &energies, const double *virial9) {
    for (auto &kv : energies)
      if (m_Index.count(kv.first)) m_Host[m_Index[kv.first]] = kv.second;
    if (virial9)
      for (int k = 0; k < 9; ++k) m_Host[getN() + k] = virial9[k];
    if (m_Dev)
      apocharmm_detail::cuda_check(cudaMemcpy(m_Dev, m_Host.data(), m_Host.size() * sizeof(double),
                                              cudaMemcpyHostToDevice),
                                   "CudaEnergyVirial::set");
  }

 private:
  int index(const std::string &name) const {
    auto it = m_Index.find(name);
    if (it == m_Index.end())
      throw std::invalid_argument("CudaEnergyVirial: no energy term named '" + name + "'");
    return it->second;
  }
  int checked(int idx) const {
    if (idx < 0 || idx >= getN())
      throw std::invalid_argument("CudaEnergyVirial: energy index out of range");
    return idx;
  }
  void clearRange(int first, int count, cudaStream_t stream) {
    if (!m_Dev || count <= 0) return;
    apocharmm_detail::cuda_check(
        cudaMemsetAsync(m_Dev + first, 0, (size_t)count * sizeof(double), stream),
        "CudaEnergyVirial::clear");
    for (int k = first; k < first + count; ++k) m_Host[k] = 0.0;
  }

  std::vector<std::string> m_Names;
  std::map<std::string, int> m_Index;
  std::vector<double> m_Host;
  double *m_Dev = nullptr;
};
