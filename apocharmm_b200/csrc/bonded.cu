// Fused bonded / 1-4 / exclusion-correction kernel; see bonded.h.
#include "bonded.h"

#include <algorithm>
#include <stdexcept>

#include "device_util.cuh"

namespace apo {
namespace {

constexpr int kThreads = 256;
enum Seg { kSBond = 0, kSUb, kSAngle, kSDihe, kSImp, kSIn14, kSEx14, kNumSeg };

// difference of two atom positions, formed from the FP64 state coordinates
// so that stiff terms are not limited by single-precision absolute positions
__device__ __forceinline__ float3 diff(const BondedArgs &a, int i, int j) {
  const double4 xi = a.coords[i], xj = a.coords[j];
  return make_float3((float)(xi.x - xj.x), (float)(xi.y - xj.y), (float)(xi.z - xj.z));
}

__device__ __forceinline__ void push(const BondedArgs &a, int atom, float gx, float gy,
                                     float gz) {
  const int s = a.glo2loc[atom];
  add_fixed(a.force + s, to_fixed_force(gx));
  add_fixed(a.force + a.stride + s, to_fixed_force(gy));
  add_fixed(a.force + 2 * a.stride + s, to_fixed_force(gz));
}

// w -= d (x) g  (one atom's contribution to the internal virial, d its
// position relative to the term's reference atom)
__device__ __forceinline__ void vir_sub(float *w, float dx, float dy, float dz, float gx, float gy,
                                        float gz) {
  w[0] -= dx * gx; w[1] -= dx * gy; w[2] -= dx * gz;
  w[3] -= dy * gx; w[4] -= dy * gy; w[5] -= dy * gz;
  w[6] -= dz * gx; w[7] -= dz * gy; w[8] -= dz * gz;
}

// E = k (r - r0)^2, reference src/CudaBondedForce.cu:85-120
template <bool VIR>
__device__ float bond_term(const BondedArgs &a, int i, int j, float2 p, float *w) {
  const float3 d = diff(a, i, j);
  const float dx = d.x, dy = d.y, dz = d.z;
  const float r = sqrtf(dx * dx + dy * dy + dz * dz);
  const float db = r - p.y;
  const float f = 2.f * p.x * db / r;
  push(a, i, f * dx, f * dy, f * dz);
  push(a, j, -f * dx, -f * dy, -f * dz);
  if (VIR) vir_sub(w, dx, dy, dz, f * dx, f * dy, f * dz);
  return p.x * db * db;
}

// E = k (theta - theta0)^2 with cos(theta) clamped to +-0.999
// (src/CudaBondedForce.cu:223-300)
template <bool VIR>
__device__ float angle_term(const BondedArgs &a, int4 t, float2 p, float *w) {
  const float3 dv1 = diff(a, t.x, t.y), dv2 = diff(a, t.z, t.y);
  const float ax = dv1.x, ay = dv1.y, az = dv1.z;
  const float bx = dv2.x, by = dv2.y, bz = dv2.z;
  const float rai = rsqrtf(ax * ax + ay * ay + az * az);
  const float rbi = rsqrtf(bx * bx + by * by + bz * bz);
  const float uax = ax * rai, uay = ay * rai, uaz = az * rai;
  const float ubx = bx * rbi, uby = by * rbi, ubz = bz * rbi;
  float cst = uax * ubx + uay * uby + uaz * ubz;
  cst = fminf(0.999f, fmaxf(-0.999f, cst));
  const float th = acosf(cst);
  const float da = th - p.y;
  const float df = -2.f * p.x * da * rsqrtf(1.f - cst * cst);
  const float gix = df * rai * (ubx - cst * uax), giy = df * rai * (uby - cst * uay),
              giz = df * rai * (ubz - cst * uaz);
  const float gkx = df * rbi * (uax - cst * ubx), gky = df * rbi * (uay - cst * uby),
              gkz = df * rbi * (uaz - cst * ubz);
  push(a, t.x, gix, giy, giz);
  push(a, t.z, gkx, gky, gkz);
  push(a, t.y, -gix - gkx, -giy - gky, -giz - gkz);
  if (VIR) {
    vir_sub(w, ax, ay, az, gix, giy, giz);
    vir_sub(w, bx, by, bz, gkx, gky, gkz);
  }
  return p.x * da * da;
}

// proper (HARM = false: sum k (1 + cos(n phi - delta))) and improper
// (HARM = true: k (phi - psi0)^2) dihedrals; gradient expressions of the
// reference (src/CudaBondedForce.cu:517-640)
template <bool HARM, bool VIR>
__device__ float dihedral_term(const BondedArgs &a, int4 t, int2 terms, float2 hp, float *w) {
  const float3 F = diff(a, t.x, t.y), G = diff(a, t.y, t.z), H = diff(a, t.w, t.z);
  const float fx = F.x, fy = F.y, fz = F.z;
  const float gx = G.x, gy = G.y, gz = G.z;
  const float hx = H.x, hy = H.y, hz = H.z;
  const float ax = fy * gz - fz * gy, ay = fz * gx - fx * gz, az = fx * gy - fy * gx;
  const float bx = hy * gz - hz * gy, by = hz * gx - hx * gz, bz = hx * gy - hy * gx;
  const float ra2 = ax * ax + ay * ay + az * az, rb2 = bx * bx + by * by + bz * bz;
  const float rg = sqrtf(gx * gx + gy * gy + gz * gz);
  const float rgr = 1.f / rg, ra2r = 1.f / ra2, rb2r = 1.f / rb2;
  const float rabr = sqrtf(ra2r * rb2r);
  const float ct = (ax * bx + ay * by + az * bz) * rabr;
  const float st = rg * rabr * (ax * hx + ay * hy + az * hz);
  float e = 0.f, df = 0.f;
  if (HARM) {
    const float c0 = cosf(hp.y), s0 = sinf(hp.y);
    const float ca = ct * c0 + st * s0, sa = st * c0 - ct * s0;
    const float ap = atan2f(sa, ca);
    e = hp.x * ap * ap;
    df = 2.f * hp.x * ap;
  } else {
    for (int q = terms.x; q < terms.x + terms.y; ++q) {
      const float4 c = a.dihe_coef[q];  // (k, n, cos delta, sin delta)
      const int n = (int)c.y;
      // cos(n phi), sin(n phi) by recursion
      float cn = 1.f, sn = 0.f;
      for (int m = 0; m < n; ++m) {
        const float c2 = cn * ct - sn * st;
        sn = cn * st + sn * ct;
        cn = c2;
      }
      e += c.x * (1.f + cn * c.z + sn * c.w);
      df += -c.x * (float)n * (sn * c.z - cn * c.w);
    }
  }
  const float fg = fx * gx + fy * gy + fz * gz, hg = hx * gx + hy * gy + hz * gz;
  const float ra2d = ra2r * df, rb2d = rb2r * df;
  const float fga = fg * ra2d * rgr, hgb = hg * rb2d * rgr;
  const float gaa = ra2d * rg, gbb = rb2d * rg;
  const float dfx = -gaa * ax, dfy = -gaa * ay, dfz = -gaa * az;
  const float dgx = fga * ax - hgb * bx, dgy = fga * ay - hgb * by, dgz = fga * az - hgb * bz;
  const float dhx = gbb * bx, dhy = gbb * by, dhz = gbb * bz;
  push(a, t.x, dfx, dfy, dfz);
  push(a, t.y, dgx - dfx, dgy - dfy, dgz - dfz);
  push(a, t.z, -dhx - dgx, -dhy - dgy, -dhz - dgz);
  push(a, t.w, dhx, dhy, dhz);
  if (VIR) {
    // positions relative to atom k: i - k = F + G, j - k = G, l - k = H
    vir_sub(w, fx + gx, fy + gy, fz + gz, dfx, dfy, dfz);
    vir_sub(w, gx, gy, gz, dgx - dfx, dgy - dfy, dgz - dfz);
    vir_sub(w, hx, hy, hz, dhx, dhy, dhz);
  }
  return e;
}

// 1-4 inclusion (LJ14 with VFSW + qq erfc/r) or exclusion correction
// (qq (erfc - 1)/r = -qq erf/r); src/CudaDirectForceKernels.cu:643-870
template <bool INCL, bool VIR, bool MULTI>
__device__ void pair14_term(const BondedArgs &a, const NbSetup &st, int2 p, float &e_el,
                            float &e_vdw, float *w) {
  const float3 d = diff(a, p.x, p.y);
  const float dx = d.x, dy = d.y, dz = d.z;
  const float r2 = dx * dx + dy * dy + dz * dz;
  const float rinv = rsqrtf(r2), r = r2 * rinv, rinv2 = rinv * rinv;
  const float qq = (float)kCcelec * (float)a.coords[p.x].w * (float)a.coords[p.y].w;
  const float expv = __expf(-st.kappa2 * r2);
  float fr;
  if (INCL) {
    const float ev = qq * erfcf(st.kappa * r) * rinv;
    fr = -qq * st.two_kappa_sqrtpi * expv - ev;
    e_el = ev;
    const int T = MULTI ? st.ntype : a.ntype;
    const float2 cc = a.vdw14[(MULTI ? st.vdw14_off : 0) + a.vdwtype[p.x] * T + a.vdwtype[p.y]];
    const float rinv3 = rinv * rinv2, rinv6 = rinv3 * rinv3;
    const bool sw = r2 > st.ron2;
    const float A6 = sw ? st.k6 : 1.f, B6 = sw ? st.roffinv3 : 0.f;
    const float A12 = sw ? st.k12 : 1.f, B12 = sw ? st.roffinv6 : 0.f;
    const float C6 = sw ? 0.f : st.dv6, C12 = sw ? 0.f : st.dv12;
    const float t6 = rinv3 - B6, t12 = rinv6 - B12;
    fr += cc.x * A6 * t6 * rinv3 - cc.y * A12 * t12 * rinv6;
    e_vdw = (1.f / 12.f) * cc.y * (A12 * t12 * t12 + C12) - (1.f / 6.f) * cc.x * (A6 * t6 * t6 + C6);
  } else {
    const float ev = -qq * erff(st.kappa * r) * rinv;
    fr = -qq * st.two_kappa_sqrtpi * expv - ev;
    e_el = ev;
    e_vdw = 0.f;
  }
  const float f = fr * rinv2;
  push(a, p.x, f * dx, f * dy, f * dz);
  push(a, p.y, -f * dx, -f * dy, -f * dz);
  if (VIR) vir_sub(w, dx, dy, dz, f * dx, f * dy, f * dz);
}

template <bool ENERGY, bool VIRIAL, bool MULTI = false>
__global__ void __launch_bounds__(kThreads) bonded_kernel(BondedArgs a) {
  __shared__ unsigned long long sh_e[kNumEnergyTerms];
  __shared__ unsigned long long sh_v[9];
  if (ENERGY && !MULTI) {
    if (threadIdx.x < kNumEnergyTerms) sh_e[threadIdx.x] = 0ull;
    if (VIRIAL && threadIdx.x < 9) sh_v[threadIdx.x] = 0ull;
    __syncthreads();
  }
  const int b1 = a.nbond, b2 = b1 + a.nub, b3 = b2 + a.nangle, b4 = b3 + a.ndihe,
            b5 = b4 + a.nimp, b6 = b5 + a.nin14, b7 = b6 + a.nex14;
  // the loop runs in whole warps (t0 is the same in every lane), so the
  // virial can be summed across the warp before it reaches shared memory
  for (int t0 = blockIdx.x * blockDim.x; t0 < b7; t0 += gridDim.x * blockDim.x) {
    const int t = t0 + threadIdx.x;
    float e = 0.f, e2 = 0.f;
    float w[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int slot = -1, slot2 = -1;
    if (t >= b7) {
      // past the last term: contributes nothing
    } else if (t < b1) {
      e = bond_term<VIRIAL>(a, a.bond_ij[t].x, a.bond_ij[t].y, a.bond_p[t], w);
      slot = kEBond;
    } else if (t < b2) {
      const int k = t - b1;
      e = bond_term<VIRIAL>(a, a.ub_ij[k].x, a.ub_ij[k].y, a.ub_p[k], w);
      slot = kEUreyb;
    } else if (t < b3) {
      const int k = t - b2;
      e = angle_term<VIRIAL>(a, a.angle_ijk[k], a.angle_p[k], w);
      slot = kEAngle;
    } else if (t < b4) {
      const int k = t - b3;
      e = dihedral_term<false, VIRIAL>(a, a.dihe_ijkl[k], a.dihe_terms[k], make_float2(0.f, 0.f),
                                       w);
      slot = kEDihe;
    } else if (t < b5) {
      const int k = t - b4;
      e = dihedral_term<true, VIRIAL>(a, a.imp_ijkl[k], make_int2(0, 0), a.imp_p[k], w);
      slot = kEImdihe;
    } else if (t < b6) {
      const int2 pr = a.in14[t - b5];
      pair14_term<true, VIRIAL, MULTI>(a, MULTI ? a.setups[a.sys_of_atom[pr.x]] : a.nb, pr, e, e2,
                                       w);
      slot = kEElec;
      slot2 = kEVdw;
    } else {
      const int2 pr = a.ex14[t - b6];
      pair14_term<false, VIRIAL, MULTI>(a, MULTI ? a.setups[a.sys_of_atom[pr.x]] : a.nb, pr, e,
                                        e2, w);
      slot = kEEwex;
    }
    if (MULTI) {
      if (ENERGY && t < b7) {  // straight to this term's system
        int first;
        if (t < b1) first = a.bond_ij[t].x;
        else if (t < b2) first = a.ub_ij[t - b1].x;
        else if (t < b3) first = a.angle_ijk[t - b2].x;
        else if (t < b4) first = a.dihe_ijkl[t - b3].x;
        else if (t < b5) first = a.imp_ijkl[t - b4].x;
        else if (t < b6) first = a.in14[t - b5].x;
        else first = a.ex14[t - b6].x;
        long long *es = a.energy + (size_t)a.sys_of_atom[first] * a.energy_stride;
        add_fixed(es + slot, __double2ll_rn((double)e * kEnergyScale));
        if (slot2 >= 0) add_fixed(es + slot2, __double2ll_rn((double)e2 * kEnergyScale));
        if (VIRIAL) {
#pragma unroll
          for (int k = 0; k < 9; ++k)
            add_fixed(es + kNumEnergyTerms + k, __double2ll_rn((double)w[k] * kEnergyScale));
        }
      }
      continue;
    }
    if (ENERGY && slot >= 0) {
      atomicAdd(&sh_e[slot], (unsigned long long)__double2ll_rn((double)e * kEnergyScale));
      if (slot2 >= 0)
        atomicAdd(&sh_e[slot2], (unsigned long long)__double2ll_rn((double)e2 * kEnergyScale));
    }
    if (VIRIAL) {
      // fixed-point sums: the same integers in any order
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        long long v = __double2ll_rn((double)w[k] * kEnergyScale);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&sh_v[k], (unsigned long long)v);
      }
    }
  }
  if (ENERGY && !MULTI) {
    __syncthreads();
    if (threadIdx.x < kNumEnergyTerms && sh_e[threadIdx.x])
      add_fixed(a.energy + threadIdx.x, (long long)sh_e[threadIdx.x]);
    if (VIRIAL && threadIdx.x < 9 && sh_v[threadIdx.x])
      add_fixed(a.virial + threadIdx.x, (long long)sh_v[threadIdx.x]);
  }
}

}  // namespace

void launch_bonded(const BondedArgs &a, bool energy, cudaStream_t s, bool virial) {
  const long long total = (long long)a.nbond + a.nub + a.nangle + a.ndihe + a.nimp + a.nin14 + a.nex14;
  if (total == 0) return;
  int blocks = (int)std::min<long long>((total + kThreads - 1) / kThreads, 148 * 16);
  if (virial) {
    if (!a.virial) throw std::invalid_argument("bonded: virial requested without a buffer");
    bonded_kernel<true, true><<<blocks, kThreads, 0, s>>>(a);
  } else if (energy) {
    bonded_kernel<true, false><<<blocks, kThreads, 0, s>>>(a);
  } else {
    bonded_kernel<false, false><<<blocks, kThreads, 0, s>>>(a);
  }
  APO_LAUNCH_CHECK();
}

void launch_bonded_multi(const BondedArgs &a, bool energy, cudaStream_t s, bool virial) {
  const long long total = (long long)a.nbond + a.nub + a.nangle + a.ndihe + a.nimp + a.nin14 + a.nex14;
  if (total == 0) return;
  if (!a.sys_of_atom || !a.setups || ((energy || virial) && a.energy_stride <= 0))
    throw std::invalid_argument("bonded: multi-system launch without system tables");
  int blocks = (int)std::min<long long>((total + kThreads - 1) / kThreads, 148 * 16);
  if (virial) bonded_kernel<true, true, true><<<blocks, kThreads, 0, s>>>(a);
  else if (energy) bonded_kernel<true, false, true><<<blocks, kThreads, 0, s>>>(a);
  else bonded_kernel<false, false, true><<<blocks, kThreads, 0, s>>>(a);
  APO_LAUNCH_CHECK();
}

}  // namespace apo
