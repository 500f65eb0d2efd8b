// Device-ready topology assembled from a PSF and a parameter set.
//
// Restates the reference's host-side assembly:
//   exclusions / 1-4 lists   CharmmPSF::buildTopologicalExclusions and
//                            getInclusionExclusionLists (src/CharmmPSF.cu:235-385)
//   LJ tables                CharmmParameters::getVdwParamsAndTypes
//                            (src/CharmmParameters.cu:718-844)
//   bonded terms             CharmmParameters::getBondedParamsAndLists
//                            (src/CharmmParameters.cu:357-700)
//   SHAKE clusters           ForceManager::initializeHolonomicConstraintsVariables
//                            (src/ForceManager.cu:844-921)
//   degrees of freedom       CharmmContext::useHolonomicConstraints
//                            (src/CharmmContext.cu:919-946)
// Unlike the reference, bonded parameters are resolved per term (one record
// per bond/angle/...) instead of through a shared type table, so each bonded
// thread reads one contiguous record.
#pragma once

#include <vector_types.h>

#include <string>
#include <vector>

#include "charmm_io.h"

namespace apo {

struct Topology {
  int natom = 0;
  std::vector<double> charge, mass;
  std::vector<std::string> types;       // sorted unique LJ types
  std::vector<int> vdwtype;             // per atom, index into `types`
  // full ntype x ntype tables of (6*c6, 12*c12): the r*dU/dr coefficients
  std::vector<float2> vdw, vdw14;
  // symmetric CSR of all topological exclusions (1-2, 1-3, 1-4), sorted
  std::vector<int> excl_ptr, excl_idx;
  std::vector<int2> in14, ex14;
  // bonded terms, one record per term
  std::vector<int2> bond_ij;    std::vector<float2> bond_p;    // (kb, b0)
  std::vector<int2> ub_ij;      std::vector<float2> ub_p;      // (kub, s0)
  std::vector<int4> angle_ijk;  std::vector<float2> angle_p;   // (k, theta0 rad)
  std::vector<int4> dihe_ijkl;  std::vector<int2> dihe_terms;  // (first, count)
  std::vector<float4> dihe_coef;  // (k, n, cos delta, sin delta)
  std::vector<int4> imp_ijkl;   std::vector<float2> imp_p;     // (k, psi0 rad)
  // constraints
  std::vector<int4> waters;       // (O, H1, H2, 0)
  std::vector<int4> shake_atoms;  // (heavy, h1, h2|-1, h3|-1)
  std::vector<float4> shake_p;    // (1/m_heavy, unused, b0^2, 1/m_H)
  // bonded components for image centering, [first, last]
  std::vector<int2> groups;

  int num_shake_constraints() const;
  int degrees_of_freedom(bool holonomic) const;
};

Topology build_topology(const CharmmPSF &psf, const CharmmParameters &prm);

}  // namespace apo
