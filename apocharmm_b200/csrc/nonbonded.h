// Direct-space erfc-Ewald + CHARMM force-switched LJ over neighbour tiles.
//
// Replaces the reference's calcForceKernel (include/CudaDirectForce_util.h:18-333,
// pair functions src/CudaDirectForceKernels.cu:209-489; VDW_VFSW, EWALD).
#pragma once

#include <cuda_runtime.h>

namespace apo {

struct NbSetup {
  double Lxd, Lyd, Lzd;   // box, full precision
  float Lx, Ly, Lz;
  float Lx_lo, Ly_lo, Lz_lo;  // L - (float)L: the box as a two-float sum
  float roff2, ron2;
  float kappa, kappa2, two_kappa_sqrtpi;
  float ewald_e2;             // -kappa^2 log2(e): exp(-kappa^2 r^2) = 2^(ewald_e2 r^2)
  float k6, k12, dv6, dv12, roffinv3, roffinv6;
  // LJ tables of this system (multi-system launches): ntype x ntype entries
  // at vdw + vdw_off (and vdw14 + vdw14_off for the 1-4 pairs)
  int vdw_off = 0, vdw14_off = 0, ntype = 0;
};

// largest LJ type count of one system in a multi-system launch (the
// direct-space kernel keeps one ntype^2 table per warp in shared memory)
constexpr int kMaxMultiTypes = 16;

NbSetup make_nb_setup(double Lx, double Ly, double Lz, double kappa, double roff,
                      double ron);

struct NbArgs {
  const float4 *xyzq_s;   // cluster-local coordinates (NeighborList::xyzq_s)
  const float4 *origin;   // per cluster origin (NeighborList::cl_origin)
  const int *perm;        // slot -> atom, -1 for padding
  const int *type_s;
  const int2 *tiles;
  const unsigned *masks;
  const int4 *work;
  const int *counts;      // [2] = number of work items
  const float2 *vdw;      // ntype x ntype (6 c6, 12 c12)
  int ntype;
  long long *force;       // SoA fixed point in sorted slot order
  int stride;
  long long *energy;      // energy slots (elec, vdw used)
  const NbSetup *setups;  // per system (indexed by work item .w)
  long long *virial = nullptr;  // 3x3 internal virial, 2^32 fixed point (virial launches)
  // multi-system launches: energies (and virial) of system s at
  // energy + s * energy_stride (virial at + kNumEnergyTerms); 0 = one system
  int energy_stride = 0;
  int variant = 0;        // kernel form, below
  // dynamic schedule: [0] work items handed out, [1] warps retired; both
  // zero between launches (the last warp to retire resets them)
  int *sched = nullptr;
  // at most this many work items per warp (0: no bound, a persistent grid);
  // with a bound the grid covers work_cap items, so blocks retire while the
  // reciprocal-space kernels of the other stream wait for SMs
  int items_per_warp = 0;
  int work_cap = 0;
};

// direct-space kernel forms: one j-list per tile for all 32 i-atoms, or one
// queue per 8-atom i-group carried across tiles
constexpr int kNbTileBatches = 0;
constexpr int kNbGroupedQueues = 1;
constexpr int kNbOctetLists = 2;

// per_pair: round every pair contribution to 64-bit fixed point before it is
// summed (order-independent, the reference's accumulation,
// include/gpu_utils.h:281-312); otherwise FP32 sums per atom and tile are
// rounded once (deterministic for a given tile list).
// virial: also accumulate W = -sum over pairs of d (x) dU/dd into a.virial
// (implies energy).
void launch_nonbonded(const NbArgs &a, bool energy, bool per_pair, cudaStream_t s,
                      bool virial = false);
// every work item's system from its .w, with per-system LJ tables
void launch_nonbonded_multi(const NbArgs &a, bool energy, bool per_pair, cudaStream_t s,
                            bool virial = false);

// the octet-list form (nonbonded_lists.cu)
void launch_nonbonded_octets(const NbArgs &a, bool energy, bool per_pair, bool virial, bool multi,
                             cudaStream_t s);

}  // namespace apo
