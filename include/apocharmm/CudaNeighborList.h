// CudaNeighborList<32>: a ForceManager's tile neighbour list (the
// reference's include/CudaNeighborList.h:32-170: build, get_glo2loc,
// get_ind_sorted, getNumList, analyze).
//
// The list sorts atoms into 32-atom clusters by x-y column and z, and keeps
// every cluster pair whose bounding boxes come within the list radius
// (cutnb) under one of the 27 periodic images, with a 32x32 exclusion mask
// for the tiles that hold a topological exclusion.  There is one list per
// manager (getNumList() == 1: no domain-decomposition zones).
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdio>
#include <memory>
#include <vector>

#include "apocharmm/ForceManager.h"

template <int tilesize>
class CudaNeighborList {
  static_assert(tilesize == 32, "CudaNeighborList: the library builds 32-atom tiles");

 public:
  explicit CudaNeighborList(std::shared_ptr<ForceManager> fm) : m_Fm(std::move(fm)) {
    if (!m_Fm) throw std::invalid_argument("CudaNeighborList: null ForceManager");
  }

  // rebuilds the list from device coordinates (float4 x, y, z, q; atom order)
  void build(const float4 *xyzq) { m_Fm->resetNeighborList(xyzq); }
  int getNumList() const { return 1; }

  // device arrays, valid until the next build: atom -> sorted slot, and
  // sorted slot -> atom (-1 for the padding slots of a cluster)
  const int *get_glo2loc() { return arrays().first; }
  const int *get_ind_sorted() { return arrays().second; }

  // sizes of the last build
  int getNumSlots() { return counts()[0]; }
  int getNumTiles() { return counts()[1]; }
  int getNumWorkItems() { return counts()[2]; }

  // every list pair whose distance is below `radius`: (atom i, atom j,
  // excluded), each unordered pair once
  std::vector<std::array<int, 3>> getPairs(double radius) {
    size_t n = 0;
    auto s = *m_Fm->getForceManagerStream();
    apocharmm_detail::check(apo_force_manager_get_list_pairs(nullptr, 0, &n, radius, m_Fm->handle(), s));
    std::vector<int> flat(3 * n);
    apocharmm_detail::check(
        apo_force_manager_get_list_pairs(flat.data(), flat.size(), &n, radius, m_Fm->handle(), s));
    std::vector<std::array<int, 3>> out(n);
    for (size_t k = 0; k < n; ++k) out[k] = {flat[3 * k], flat[3 * k + 1], flat[3 * k + 2]};
    return out;
  }

  void analyze() {
    const auto c = counts();
    std::printf("CudaNeighborList<32>: %d sorted slots (%d clusters), %d tiles, %d work items\n",
                c[0], c[0] / 32, c[1], c[2]);
  }

 private:
  std::array<int, 3> counts() {
    std::array<int, 3> c{{0, 0, 0}};
    apocharmm_detail::check(apo_force_manager_get_list_counts(
        &c[0], &c[1], &c[2], m_Fm->handle(), *m_Fm->getForceManagerStream()));
    return c;
  }
  std::pair<const int *, const int *> arrays() {
    const int *g = nullptr, *p = nullptr;
    apocharmm_detail::check(apo_force_manager_get_list_arrays(&g, &p, m_Fm->handle()));
    return {g, p};
  }
  std::shared_ptr<ForceManager> m_Fm;
};
