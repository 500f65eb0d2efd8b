// Small device helpers shared by the kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "common.h"

namespace apo {

__device__ __forceinline__ long long to_fixed_force(float v) {
  return __float2ll_rn(v * (float)kForceScale);
}
__device__ __forceinline__ long long to_fixed_force_d(double v) {
  return __double2ll_rn(v * kForceScale);
}
__device__ __forceinline__ void add_fixed(long long *p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long *>(p), (unsigned long long)v);
}
// Energy accumulation: every partial sum is rounded to fixed point before it
// is combined, so the total does not depend on the order of the atomics.
__device__ __forceinline__ void add_energy(long long *slot, double e) {
  add_fixed(slot, __double2ll_rn(e * kEnergyScale));
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Image shift code 0..26 -> integer image offsets (-1, 0, 1) per axis, the
// reference's ish convention (include/gpu_utils.h:363-372): code 13 = no shift.
__device__ __forceinline__ void shift_code(int sc, float Lx, float Ly, float Lz,
                                           float &sx, float &sy, float &sz) {
  sz = (float)(sc / 9 - 1) * Lz;
  sc -= (sc / 9) * 9;
  sy = (float)(sc / 3 - 1) * Ly;
  sx = (float)(sc - (sc / 3) * 3 - 1) * Lx;
}

}  // namespace apo
