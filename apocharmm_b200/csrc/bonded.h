// Bonded terms, 1-4 inclusions and 1-2/1-3 exclusion corrections in one
// launch.
//
// Replaces CudaBondedForce::calc_force (src/CudaBondedForce.cu:1642-1808,
// bond/UB :85-220, angle :223-345, dihedral :387-700) and
// CudaPMEDirectForce::calc_14_force (src/CudaPMEDirectForce.cu:1072,
// body include/CudaDirectForce14_util.h, pair code
// src/CudaDirectForceKernels.cu:643-870).  One thread per term over the
// concatenated term lists; every gradient contribution is rounded to 64-bit
// fixed point and added with integer atomics (order independent).
#pragma once

#include <cuda_runtime.h>

#include "nonbonded.h"

namespace apo {

struct BondedArgs {
  const double4 *coords;  // global atom order: x, y, z, charge (FP64 state)
  const int *glo2loc;     // atom -> force slot
  long long *force;
  int stride;
  long long *energy;
  int nbond; const int2 *bond_ij; const float2 *bond_p;
  int nub; const int2 *ub_ij; const float2 *ub_p;
  int nangle; const int4 *angle_ijk; const float2 *angle_p;
  int ndihe; const int4 *dihe_ijkl; const int2 *dihe_terms; const float4 *dihe_coef;
  int nimp; const int4 *imp_ijkl; const float2 *imp_p;
  int nin14; const int2 *in14;
  int nex14; const int2 *ex14;
  const int *vdwtype; const float2 *vdw14; int ntype;
  NbSetup nb;             // kappa and the VFSW constants for the 1-4 LJ
  long long *virial = nullptr;  // 3x3 internal virial, 2^32 fixed point (virial launches)
  // multi-system launches: atom -> system, per-system set-ups (kappa, VFSW,
  // 1-4 table offset and type count), energies of system s at
  // energy + s * energy_stride (virial at + kNumEnergyTerms)
  const int *sys_of_atom = nullptr;
  const NbSetup *setups = nullptr;
  int energy_stride = 0;
};

// virial: also accumulate W = -sum over terms of (r_k - r_ref) (x) dU/dr_k
// into a.virial (implies energy)
void launch_bonded(const BondedArgs &a, bool energy, cudaStream_t s, bool virial = false);
void launch_bonded_multi(const BondedArgs &a, bool energy, cudaStream_t s, bool virial = false);

}  // namespace apo
