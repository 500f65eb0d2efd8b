// Pair arithmetic and warp helpers shared by the direct-space kernel forms
// (nonbonded.cu: tile batches and grouped queues; nonbonded_lists.cu: octet
// lists).
#pragma once

#include <cuda_runtime.h>

#include "common.h"
#include "device_util.cuh"
#include "nblist.h"
#include "nonbonded.h"

namespace apo {
namespace nbdetail {

// sum of v[jj] over the 32 lanes; on return lane L holds the total of
// jj = L >> 2 (every lane of a quad holds the same value)
template <typename T>
__device__ __forceinline__ T transpose_reduce8(T (&v)[8], int lane) {
  const bool b16 = lane & 16, b8 = lane & 8, b4 = lane & 4;
  T u[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    T send = b16 ? v[k] : v[k + 4];
    T keep = b16 ? v[k + 4] : v[k];
    u[k] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
  T w[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    T send = b8 ? u[k] : u[k + 2];
    T keep = b8 ? u[k + 2] : u[k];
    w[k] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  T send = b4 ? w[0] : w[1];
  T z = (b4 ? w[1] : w[0]) + __shfl_xor_sync(0xffffffffu, send, 4);
  z += __shfl_xor_sync(0xffffffffu, z, 2);
  z += __shfl_xor_sync(0xffffffffu, z, 1);
  return z;
}

// erfc(x) = exp(-x^2) t P(t), t = 1/(1 + p x): the form of Hastings'
// approximation (Abramowitz & Stegun 7.1.26) with p = 0.365 and the nine
// coefficients of P refitted here by linear least squares on the relative
// error of erfc over 0 <= x <= 6 (the range kappa r takes inside the
// cutoff); max relative error 1.3e-8 in FP64, 1.3e-7 with the coefficients
// rounded to single precision.  The exponential is the one the Ewald force
// needs anyway.
__device__ __forceinline__ float rcp_approx(float v) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
}
__device__ __forceinline__ float rsqrt_approx(float v) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
}
__device__ __forceinline__ float ex2_approx(float v) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
}

__device__ __forceinline__ float erfc_from_exp(float x, float expv) {
  const float t = rcp_approx(fmaf(0.365f, x, 1.f));
  float p = 6.816177070e-02f;
  p = fmaf(p, t, -3.500733972e-01f);
  p = fmaf(p, t, 6.125112772e-01f);
  p = fmaf(p, t, -4.309675097e-01f);
  p = fmaf(p, t, 4.153276980e-01f);
  p = fmaf(p, t, 6.009365246e-02f);
  p = fmaf(p, t, 2.160071135e-01f);
  p = fmaf(p, t, 2.028342783e-01f);
  p = fmaf(p, t, 2.061051130e-01f);
  return expv * t * p;
}

// warp-wide sum of a double, rounded to fixed point, added to *dst by lane 0
__device__ __forceinline__ void warp_flush(double v, long long *dst, int lane) {
  long long iv = __double2ll_rn(v * kEnergyScale);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) iv += __shfl_xor_sync(0xffffffffu, iv, o);
  if (lane == 0 && iv) add_fixed(dst, iv);
}

// The pairs of i-lane `lane` that a tile skips, as a bit per j-lane: its
// topological exclusions (only tiles that hold one carry a mask) and, for a
// cluster's tile with itself, the pairs j <= i.
__device__ __forceinline__ unsigned tile_excl_word(const NbArgs &a, int2 tl, int code, int icl,
                                                   int lane) {
  const int midx = tile_mask(tl.y);
  unsigned w = midx >= 0 ? a.masks[(size_t)midx * kTile + lane] : 0u;
  if (tl.x == icl && code == 13) w |= self_tile_word(lane);
  return w;
}

// Work items are handed out one at a time from a counter, so warps that
// start late (SMs still busy with the reciprocal-space kernels of the other
// stream) or draw cheap items simply take more of them.
__device__ __forceinline__ int next_work(int *sched, int lane) {
  int v = 0;
  if (lane == 0) v = atomicAdd(sched, 1);
  return __shfl_sync(0xffffffffu, v, 0);
}
__device__ __forceinline__ void retire_warp(int *sched, int lane) {
  if (lane == 0 && atomicAdd(sched + 1, 1) == (int)(gridDim.x * (blockDim.x >> 5)) - 1) {
    sched[0] = 0;
    sched[1] = 0;
  }
}

// One pair: erfc-Ewald (src/CudaDirectForceKernels.cu:479-489) plus VDW_VFSW
// (src/CudaDirectForceKernels.cu:263-286).  Returns f with gradient on i =
// f (x_i - x_j); `in` = inside the cutoff and not excluded, anything else
// gives 0 (r2raw may then be anything finite, including 0).  With ENERGY the
// two energies of the pair are added to e_el / e_vdw.
template <bool ENERGY>
__device__ __forceinline__ float pair_force(const NbSetup &st, float r2raw, bool in, float qi,
                                            float qj, float2 cc, double &e_el, double &e_vdw) {
  const float r2 = in ? r2raw : 1.f;
  const float rinv = rsqrt_approx(r2);  // r2 >= 1e-2 inside the cutoff: never denormal
  const float rr = r2 * rinv;
  const float rinv2 = rinv * rinv;
  const float qq = qi * qj;
  const float exp_v = ex2_approx(st.ewald_e2 * r2);
  const float erfc_v = erfc_from_exp(st.kappa * rr, exp_v);
  const float el = qq * erfc_v * rinv;
  const float fr_el = fmaf(-qq * st.two_kappa_sqrtpi, exp_v, -el);
  const float rinv3 = rinv * rinv2, rinv6 = rinv3 * rinv3;
  const bool sw = r2 > st.ron2;
  const float A6 = sw ? st.k6 : 1.f, B6 = sw ? st.roffinv3 : 0.f;
  const float A12 = sw ? st.k12 : 1.f, B12 = sw ? st.roffinv6 : 0.f;
  const float t6 = rinv3 - B6, t12 = rinv6 - B12;
  const float fr_vdw = (cc.x * A6) * t6 * rinv3 - (cc.y * A12) * t12 * rinv6;
  if (ENERGY && in) {
    const float C6 = sw ? 0.f : st.dv6, C12 = sw ? 0.f : st.dv12;
    e_el += (double)el;
    e_vdw += (double)((1.f / 12.f) * cc.y * (A12 * t12 * t12 + C12) -
                      (1.f / 6.f) * cc.x * (A6 * t6 * t6 + C6));
  }
  return in ? (fr_vdw + fr_el) * rinv2 : 0.f;
}

// Two single-precision values in one 64-bit register pair, for the packed
// arithmetic of sm_100 (add / sub / mul / fma .rn.f32x2: one instruction
// does the operation on both halves, each half rounded exactly as the
// scalar instruction would round it).
struct F2 {
  unsigned long long v;
};
__device__ __forceinline__ F2 f2(float lo, float hi) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ F2 f2(float both) { return f2(both, both); }
__device__ __forceinline__ float f2lo(F2 a) {
  float x;
  asm("{\n\t.reg .f32 t;\n\tmov.b64 {%0, t}, %1;\n\t}" : "=f"(x) : "l"(a.v));
  return x;
}
__device__ __forceinline__ float f2hi(F2 a) {
  float y;
  asm("{\n\t.reg .f32 t;\n\tmov.b64 {t, %0}, %1;\n\t}" : "=f"(y) : "l"(a.v));
  return y;
}
__device__ __forceinline__ F2 operator+(F2 a, F2 b) {
  F2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
  F2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b) {
  F2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) {
  F2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}

// pair_force for two j-atoms of one i-atom at once (halves lo and hi), on
// packed arithmetic: the same terms, with the electrostatic part summed as
// s = qq (2 kappa / sqrt(pi)) exp + el and subtracted at the end, which is
// the scalar form's fma(-qq 2 kappa / sqrt(pi), exp, -el) negated (IEEE
// rounding is symmetric, so that part is bit for bit the same).  Returns
// the two values f with gradient on i = f (x_i - x_j); a half that is not
// `in` gives 0 (its r2raw may be anything finite).
template <bool ENERGY>
__device__ __forceinline__ F2 pair_force2(const NbSetup &st, F2 r2raw, bool in0, bool in1, F2 qq,
                                          float2 cc0, float2 cc1, double &e_el,
                                          double &e_vdw) {
  const float r2a = in0 ? f2lo(r2raw) : 1.f, r2b = in1 ? f2hi(r2raw) : 1.f;
  const F2 r2 = f2(r2a, r2b);
  const F2 rinv = f2(rsqrt_approx(r2a), rsqrt_approx(r2b));
  const F2 rr = r2 * rinv;
  const F2 rinv2 = rinv * rinv;
  const F2 arg = f2(st.ewald_e2) * r2;
  const F2 ex = f2(ex2_approx(f2lo(arg)), ex2_approx(f2hi(arg)));
  const F2 den = fma2(f2(0.365f), f2(st.kappa) * rr, f2(1.f));
  const F2 t = f2(rcp_approx(f2lo(den)), rcp_approx(f2hi(den)));
  F2 p = f2(6.816177070e-02f);
  p = fma2(p, t, f2(-3.500733972e-01f));
  p = fma2(p, t, f2(6.125112772e-01f));
  p = fma2(p, t, f2(-4.309675097e-01f));
  p = fma2(p, t, f2(4.153276980e-01f));
  p = fma2(p, t, f2(6.009365246e-02f));
  p = fma2(p, t, f2(2.160071135e-01f));
  p = fma2(p, t, f2(2.028342783e-01f));
  p = fma2(p, t, f2(2.061051130e-01f));
  const F2 erfc_v = ex * t * p;
  const F2 el = qq * erfc_v * rinv;
  const F2 s_el = fma2(qq * f2(st.two_kappa_sqrtpi), ex, el);
  const F2 rinv3 = rinv * rinv2, rinv6 = rinv3 * rinv3;
  const bool swa = r2a > st.ron2, swb = r2b > st.ron2;
  const F2 A6 = f2(swa ? st.k6 : 1.f, swb ? st.k6 : 1.f);
  const F2 B6 = f2(swa ? st.roffinv3 : 0.f, swb ? st.roffinv3 : 0.f);
  const F2 A12 = f2(swa ? st.k12 : 1.f, swb ? st.k12 : 1.f);
  const F2 B12 = f2(swa ? st.roffinv6 : 0.f, swb ? st.roffinv6 : 0.f);
  const F2 t6 = rinv3 - B6, t12 = rinv6 - B12;
  const F2 m6 = f2(cc0.x, cc1.x) * A6 * t6 * rinv3;
  const F2 m12 = f2(cc0.y, cc1.y) * A12 * t12 * rinv6;
  const F2 f = (m6 - m12 - s_el) * rinv2;
  if (ENERGY) {
    if (in0) {
      const float C6 = swa ? 0.f : st.dv6, C12 = swa ? 0.f : st.dv12;
      const float t6a = f2lo(t6), t12a = f2lo(t12);
      e_el += (double)f2lo(el);
      e_vdw += (double)((1.f / 12.f) * cc0.y * (f2lo(A12) * t12a * t12a + C12) -
                        (1.f / 6.f) * cc0.x * (f2lo(A6) * t6a * t6a + C6));
    }
    if (in1) {
      const float C6 = swb ? 0.f : st.dv6, C12 = swb ? 0.f : st.dv12;
      const float t6b = f2hi(t6), t12b = f2hi(t12);
      e_el += (double)f2hi(el);
      e_vdw += (double)((1.f / 12.f) * cc1.y * (f2hi(A12) * t12b * t12b + C12) -
                        (1.f / 6.f) * cc1.x * (f2hi(A6) * t6b * t6b + C6));
    }
  }
  return f2(in0 ? f2lo(f) : 0.f, in1 ? f2hi(f) : 0.f);
}

// sum of v[k] over the 8 lanes of a group; lane l of the group returns the
// total of entry l
template <typename T>
__device__ __forceinline__ T group_reduce8(T (&v)[8], int lane) {
  const bool b4 = lane & 4, b2 = lane & 2, b1 = lane & 1;
  T u[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const T send = b4 ? v[k] : v[k + 4];
    const T keep = b4 ? v[k + 4] : v[k];
    u[k] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  T w[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const T send = b2 ? u[k] : u[k + 2];
    const T keep = b2 ? u[k + 2] : u[k];
    w[k] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
  }
  const T send = b1 ? w[0] : w[1];
  return (b1 ? w[1] : w[0]) + __shfl_xor_sync(0xffffffffu, send, 1);
}

}  // namespace nbdetail
}  // namespace apo
