// Direct-space tile kernel; see nonbonded.h.
//
// One warp per work item (an i-cluster and a run of up to tiles_per_work of
// its j-tiles), persistent grid.  Lane l owns i-atom l for the whole work
// item: its force lives in registers.  For each tile the 32 j-atoms are
// staged in shared memory and read back as warp-wide broadcasts, so the pair
// loop costs one LDS.128 + one LDS.32 + one table LDS.64 per pair and no
// shuffles.  The j-forces of a tile are combined across the warp with a
// transpose reduction: 9 shuffles per component for every 8 j-atoms, after
// which lane L holds the full force of j-atom (L&3)*8 + (L>>2).
#include "nonbonded.h"

#include <algorithm>
#include <cmath>
#include <type_traits>

#include "device_util.cuh"
#include "nblist.h"
#include "nonbonded_pair.cuh"

namespace apo {

NbSetup make_nb_setup(double Lx, double Ly, double Lz, double kappa, double roff,
                      double ron) {
  NbSetup s;
  s.Lxd = Lx;
  s.Lyd = Ly;
  s.Lzd = Lz;
  s.Lx_lo = (float)(Lx - (double)(float)Lx);
  s.Ly_lo = (float)(Ly - (double)(float)Ly);
  s.Lz_lo = (float)(Lz - (double)(float)Lz);
  s.Lx = (float)Lx;
  s.Ly = (float)Ly;
  s.Lz = (float)Lz;
  s.roff2 = (float)(roff * roff);
  s.ron2 = (float)(ron * ron);
  s.kappa = (float)kappa;
  s.kappa2 = (float)(kappa * kappa);
  s.two_kappa_sqrtpi = (float)(2.0 * kappa / std::sqrt(M_PI));
  s.ewald_e2 = (float)(-kappa * kappa / std::log(2.0));
  // VDW_VFSW constants (src/CudaPMEDirectForce.cu:318-330)
  double roff3 = roff * roff * roff, ron3 = ron * ron * ron;
  double roff6 = roff3 * roff3, ron6 = ron3 * ron3;
  s.roffinv3 = (float)(1.0 / roff3);
  s.roffinv6 = (float)(1.0 / roff6);
  if (ron < roff) {
    s.k6 = (float)(roff3 / (roff3 - ron3));
    s.k12 = (float)(roff6 / (roff6 - ron6));
    s.dv6 = (float)(-1.0 / (ron3 * roff3));
    s.dv12 = (float)(-1.0 / (ron6 * roff6));
  } else {
    s.k6 = 1.f;
    s.k12 = 1.f;
    s.dv6 = (float)(-1.0 / roff6);
    s.dv12 = (float)(-1.0 / (roff6 * roff6));
  }
  return s;
}

namespace {

using namespace nbdetail;

constexpr int kWarps = 4;
constexpr int kThreads = kWarps * 32;

template <bool ENERGY, bool PER_PAIR, bool VIRIAL = false, bool MULTI = false>
__global__ void __launch_bounds__(kThreads) nb_kernel(NbArgs a) {
  // the j-atoms of a tile that pass the box test, compacted: position and
  // charge, and (LJ type | tile lane << 16)
  // (PER_PAIR) or, for the packed arithmetic, as pairs of j-atoms: {x0 x1
  // y0 y1} and {z0 z1 q0 q1} per pair
  __shared__ float4 sh_xq[kWarps][32];
  __shared__ __align__(16) int sh_tj[kWarps][32];
  extern __shared__ float2 sh_vdw[];
  int T = a.ntype;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  // one system: the whole table once per block; several systems: one
  // ntype^2 slice per warp, reloaded when the warp's system changes
  const int tab_off = MULTI ? wib * kMaxMultiTypes * kMaxMultiTypes : 0;
  int cur_sys = -1;
  if (!MULTI) {
    for (int k = threadIdx.x; k < T * T; k += blockDim.x) sh_vdw[k] = a.vdw[k];
    __syncthreads();
  }
  const unsigned lt_mask = (1u << lane) - 1u;
  const int nwork = a.counts[2];
  const int stride = a.stride;
  double e_elec = 0.0, e_vdw = 0.0;
  double dv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  // one system: per-lane fixed-point sums of every work item's energies and
  // virial (integer sums: the total does not depend on which warp took
  // which item)
  long long ie_el = 0, ie_vdw = 0;
  long long ivir[6] = {0, 0, 0, 0, 0, 0};  // xx xy xz yy yz zz (VIRIAL)
  using Acc = typename std::conditional<PER_PAIR, long long, float>::type;

  int taken = 0;  // warp-uniform
  auto next = [&]() -> int {
    if (a.items_per_warp > 0 && taken >= a.items_per_warp) return nwork;
    ++taken;
    return next_work(a.sched, lane);
  };
  for (int w = next(); w < nwork; w = next()) {
    // work items are taken in a scattered order, w -> (w * 7919) mod nwork
    // (one to one unless nwork is a multiple of 7919): warps working at the
    // same time then add their j-forces to distant parts of the buffer
    // (chain23k: 116.7 -> 114.8 us a launch); the results do not depend on
    // the order
    const int wp = (nwork % 7919) ? (int)(((long long)w * 7919) % nwork) : w;
    const int4 wk = a.work[wp];
    const NbSetup st = a.setups[wk.w];
    if (MULTI && wk.w != cur_sys) {  // warp-uniform
      __syncwarp();
      T = st.ntype;
      for (int k = lane; k < T * T; k += 32) sh_vdw[tab_off + k] = a.vdw[st.vdw_off + k];
      __syncwarp();
      cur_sys = wk.w;
    }
    const float4 oi = a.origin[wk.x];
    const int islot = wk.x * kTile + lane;
    const float4 xi = a.xyzq_s[islot];
    const bool ivalid = a.perm[islot] >= 0;
    const float qi = xi.w * (float)kCcelec;
    // this lane's row of the LJ table
    const float2 *vrow = sh_vdw + tab_off + a.type_s[islot] * T;
    // box around the current positions of the i-cluster
    float lo_x = ivalid ? xi.x : INFINITY, lo_y = ivalid ? xi.y : INFINITY,
          lo_z = ivalid ? xi.z : INFINITY;
    float hi_x = ivalid ? xi.x : -INFINITY, hi_y = ivalid ? xi.y : -INFINITY,
          hi_z = ivalid ? xi.z : -INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo_x = fminf(lo_x, __shfl_xor_sync(0xffffffffu, lo_x, o));
      lo_y = fminf(lo_y, __shfl_xor_sync(0xffffffffu, lo_y, o));
      lo_z = fminf(lo_z, __shfl_xor_sync(0xffffffffu, lo_z, o));
      hi_x = fmaxf(hi_x, __shfl_xor_sync(0xffffffffu, hi_x, o));
      hi_y = fmaxf(hi_y, __shfl_xor_sync(0xffffffffu, hi_y, o));
      hi_z = fmaxf(hi_z, __shfl_xor_sync(0xffffffffu, hi_z, o));
    }
    Acc fix = 0, fiy = 0, fiz = 0;
    float vw[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    // packed form: i-atom values in both halves, two partial sums per sum;
    // a padding slot sits 1e18 A away, so none of its pairs is inside the
    // cutoff (its differences stay finite: their force factor is exactly 0)
    const F2 xi2x = f2(ivalid ? xi.x : 1e18f), xi2y = f2(ivalid ? xi.y : 1e18f),
             xi2z = f2(ivalid ? xi.z : 1e18f), qi2 = f2(qi);
    F2 fi2x = f2(0.f), fi2y = f2(0.f), fi2z = f2(0.f);
    F2 vw2[6] = {f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(0.f)};

    for (int t = wk.y; t < wk.z; ++t) {
      const int2 tl = a.tiles[t];
      const int code = tile_image(tl.y);
      // j cluster frame -> i cluster frame: origin difference (exact: both
      // origins are multiples of 1/64 A) plus the periodic image k L with L
      // as a two-float sum, so |offset| < rlist + 2 cluster edges carries
      // about one rounding
      const float4 oj = a.origin[tl.x];
      const int ic = code / 9, ib = (code - 9 * ic) / 3, ia = code - 9 * ic - 3 * ib;
      const float kx = (float)(ia - 1), ky = (float)(ib - 1), kz = (float)(ic - 1);
      const float sx = fmaf(kx, st.Lx, oj.x - oi.x) + kx * st.Lx_lo;
      const float sy = fmaf(ky, st.Ly, oj.y - oi.y) + ky * st.Ly_lo;
      const float sz = fmaf(kz, st.Lz, oj.z - oi.z) + kz * st.Lz_lo;
      const int jslot = tl.x * kTile + lane;
      float4 xj = a.xyzq_s[jslot];
      xj.x += sx;
      xj.y += sy;
      xj.z += sz;
      // j-atoms that can reach the cutoff of some i-atom
      const float bx = fmaxf(0.f, fmaxf(lo_x - xj.x, xj.x - hi_x));
      const float by = fmaxf(0.f, fmaxf(lo_y - xj.y, xj.y - hi_y));
      const float bz = fmaxf(0.f, fmaxf(lo_z - xj.z, xj.z - hi_z));
      const bool jnear = a.perm[jslot] >= 0 && bx * bx + by * by + bz * bz < st.roff2;
      const unsigned jmask = __ballot_sync(0xffffffffu, jnear);
      if (jmask == 0u) continue;
      const unsigned excl = tile_excl_word(a, tl, code, wk.x, lane);
      const int nj = __popc(jmask);
      const int tj_own = a.type_s[jslot] | (lane << 16);
      __syncwarp();
      if (jnear) {
        const int pos = __popc(jmask & lt_mask);
        if (PER_PAIR) {
          sh_xq[wib][pos] = xj;
        } else {
          float *pa = reinterpret_cast<float *>(&sh_xq[wib][pos & ~1]);
          const int h = pos & 1;
          pa[h] = xj.x;
          pa[2 + h] = xj.y;
          pa[4 + h] = xj.z;
          pa[6 + h] = xj.w;
        }
        sh_tj[wib][pos] = tj_own;
      }
      if (!PER_PAIR && (nj & 1) && lane == 0) {  // an odd count: a finite filler, never `in`
        float *pa = reinterpret_cast<float *>(&sh_xq[wib][nj - 1]);
        pa[1] = 0.f;
        pa[3] = 0.f;
        pa[5] = 0.f;
        pa[7] = 0.f;
        sh_tj[wib][nj] = 0;
      }
      __syncwarp();

      Acc fjx = 0, fjy = 0, fjz = 0;  // force of compacted j (lane&3)*8 + (lane>>2)
      const int nbatch = (nj + 7) >> 3;
      if constexpr (!PER_PAIR) {
        // tiles without a topological exclusion and other than a cluster's
        // tile with itself (most of them) skip the exclusion test
        auto batches = [&](auto with_excl) {
          constexpr bool EXCL = decltype(with_excl)::value;
          for (int b = 0; b < nbatch; ++b) {
            float fx[8], fy[8], fz[8];
#pragma unroll
            for (int pp = 0; pp < 4; ++pp) {
              const int r = b * 8 + 2 * pp;
              fx[2 * pp] = fx[2 * pp + 1] = 0.f;
              fy[2 * pp] = fy[2 * pp + 1] = 0.f;
              fz[2 * pp] = fz[2 * pp + 1] = 0.f;
              if (r < nj) {  // uniform across the warp
                const float4 A = sh_xq[wib][r];      // x0 x1 y0 y1
                const float4 B = sh_xq[wib][r + 1];  // z0 z1 q0 q1
                const int2 tj = *reinterpret_cast<const int2 *>(&sh_tj[wib][r]);
                const F2 dx = xi2x - f2(A.x, A.y), dy = xi2y - f2(A.z, A.w),
                         dz = xi2z - f2(B.x, B.y);
                const F2 r2raw = fma2(dz, dz, fma2(dy, dy, dx * dx));
                bool in0 = f2lo(r2raw) < st.roff2;
                bool in1 = r + 1 < nj && f2hi(r2raw) < st.roff2;
                if (EXCL) {
                  in0 = in0 && !((excl >> (tj.x >> 16)) & 1u);
                  in1 = in1 && !((excl >> (tj.y >> 16)) & 1u);
                }
                const float2 cc0 = vrow[tj.x & 0xffff], cc1 = vrow[tj.y & 0xffff];
                const F2 f = pair_force2<ENERGY>(st, r2raw, in0, in1, qi2 * f2(B.z, B.w), cc0,
                                                 cc1, e_elec, e_vdw);
                const F2 gx = f * dx, gy = f * dy, gz = f * dz;
                if (VIRIAL) {
                  vw2[0] = fma2(gx, dx, vw2[0]);
                  vw2[1] = fma2(gx, dy, vw2[1]);
                  vw2[2] = fma2(gx, dz, vw2[2]);
                  vw2[3] = fma2(gy, dy, vw2[3]);
                  vw2[4] = fma2(gy, dz, vw2[4]);
                  vw2[5] = fma2(gz, dz, vw2[5]);
                }
                fi2x = fi2x + gx;
                fi2y = fi2y + gy;
                fi2z = fi2z + gz;
                fx[2 * pp] = f2lo(gx);
                fx[2 * pp + 1] = f2hi(gx);
                fy[2 * pp] = f2lo(gy);
                fy[2 * pp + 1] = f2hi(gy);
                fz[2 * pp] = f2lo(gz);
                fz[2 * pp + 1] = f2hi(gz);
              }
            }
            // the sums hold the gradient on i of each pair: the j-atom's is minus it
            const float rx = transpose_reduce8(fx, lane);
            const float ry = transpose_reduce8(fy, lane);
            const float rz = transpose_reduce8(fz, lane);
            if ((lane & 3) == b) {
              fjx = -rx;
              fjy = -ry;
              fjz = -rz;
            }
          }
        };
        if (__any_sync(0xffffffffu, excl != 0u)) batches(std::true_type{});
        else batches(std::false_type{});
      } else for (int b = 0; b < nbatch; ++b) {
        Acc fx[8], fy[8], fz[8];
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
          const int r = b * 8 + jj;
          fx[jj] = 0;
          fy[jj] = 0;
          fz[jj] = 0;
          if (r < nj) {  // uniform across the warp
            const float4 pj = sh_xq[wib][r];
            const int tj = sh_tj[wib][r];
            const float dx = xi.x - pj.x, dy = xi.y - pj.y, dz = xi.z - pj.z;
            const float r2raw = dx * dx + dy * dy + dz * dz;
            const bool in = ivalid && !((excl >> (tj >> 16)) & 1u) && r2raw < st.roff2;
            const float2 cc = vrow[tj & 0xffff];
            const float fij = pair_force<ENERGY>(st, r2raw, in, qi, pj.w, cc, e_elec, e_vdw);
            if (VIRIAL) {
              const float gx = fij * dx, gy = fij * dy, gz = fij * dz;
              vw[0] -= gx * dx;
              vw[1] -= gx * dy;
              vw[2] -= gx * dz;
              vw[3] -= gy * dy;
              vw[4] -= gy * dz;
              vw[5] -= gz * dz;
            }
            if (PER_PAIR) {
              const long long gx = to_fixed_force(fij * dx);
              const long long gy = to_fixed_force(fij * dy);
              const long long gz = to_fixed_force(fij * dz);
              fix += gx;
              fiy += gy;
              fiz += gz;
              fx[jj] = -gx;
              fy[jj] = -gy;
              fz[jj] = -gz;
            } else {
              fix += fij * dx;
              fiy += fij * dy;
              fiz += fij * dz;
              fx[jj] = -fij * dx;
              fy[jj] = -fij * dy;
              fz[jj] = -fij * dz;
            }
          }
        }
        const Acc rx = transpose_reduce8(fx, lane);
        const Acc ry = transpose_reduce8(fy, lane);
        const Acc rz = transpose_reduce8(fz, lane);
        if ((lane & 3) == b) {
          fjx = rx;
          fjy = ry;
          fjz = rz;
        }
      }
      const int rown = (lane & 3) * 8 + (lane >> 2);
      if (rown < nj) {
        const int jown = tl.x * kTile + (sh_tj[wib][rown] >> 16);
        if (PER_PAIR) {
          add_fixed(a.force + jown, (long long)fjx);
          add_fixed(a.force + stride + jown, (long long)fjy);
          add_fixed(a.force + 2 * stride + jown, (long long)fjz);
        } else {
          add_fixed(a.force + jown, to_fixed_force((float)fjx));
          add_fixed(a.force + stride + jown, to_fixed_force((float)fjy));
          add_fixed(a.force + 2 * stride + jown, to_fixed_force((float)fjz));
        }
      }
    }
    if (!PER_PAIR) {
      fix = f2lo(fi2x) + f2hi(fi2x);
      fiy = f2lo(fi2y) + f2hi(fi2y);
      fiz = f2lo(fi2z) + f2hi(fi2z);
      if (VIRIAL) {
#pragma unroll
        for (int k = 0; k < 6; ++k) vw[k] = -(f2lo(vw2[k]) + f2hi(vw2[k]));
      }
    }
    if (VIRIAL) {
#pragma unroll
      for (int k = 0; k < 6; ++k) dv[k] += (double)vw[k];
    }
    if (MULTI && ENERGY) {  // energies (and virial) belong to this work item's system
      long long *es = a.energy + (size_t)wk.w * a.energy_stride;
      warp_flush(e_elec, es + kEElec, lane);
      warp_flush(e_vdw, es + kEVdw, lane);
      e_elec = 0.0;
      e_vdw = 0.0;
      if (VIRIAL) {
        constexpr int kSlotM[6][2] = {{0, 0}, {1, 3}, {2, 6}, {4, 4}, {5, 7}, {8, 8}};
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          long long iw = __double2ll_rn(dv[k] * kEnergyScale);
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) iw += __shfl_xor_sync(0xffffffffu, iw, o);
          if (lane == 0 && iw) {
            add_fixed(es + kNumEnergyTerms + kSlotM[k][0], iw);
            if (kSlotM[k][1] != kSlotM[k][0]) add_fixed(es + kNumEnergyTerms + kSlotM[k][1], iw);
          }
          dv[k] = 0.0;
        }
      }
    }
    if (ENERGY && !MULTI) {
      ie_el += __double2ll_rn(e_elec * kEnergyScale);
      ie_vdw += __double2ll_rn(e_vdw * kEnergyScale);
      e_elec = 0.0;
      e_vdw = 0.0;
      if (VIRIAL) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          ivir[k] += __double2ll_rn(dv[k] * kEnergyScale);
          dv[k] = 0.0;
        }
      }
    }
    if (ivalid) {
      if (PER_PAIR) {
        add_fixed(a.force + islot, (long long)fix);
        add_fixed(a.force + stride + islot, (long long)fiy);
        add_fixed(a.force + 2 * stride + islot, (long long)fiz);
      } else {
        add_fixed(a.force + islot, to_fixed_force((float)fix));
        add_fixed(a.force + stride + islot, to_fixed_force((float)fiy));
        add_fixed(a.force + 2 * stride + islot, to_fixed_force((float)fiz));
      }
    }
  }
  retire_warp(a.sched, lane);
  if (ENERGY && !MULTI) {
    long long ie = ie_el, iv = ie_vdw;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ie += __shfl_xor_sync(0xffffffffu, ie, o);
      iv += __shfl_xor_sync(0xffffffffu, iv, o);
    }
    if (lane == 0) {
      add_fixed(a.energy + kEElec, ie);
      add_fixed(a.energy + kEVdw, iv);
    }
  }
  if (VIRIAL && !MULTI) {
    // xx xy xz yy yz zz -> row-major 3x3 (symmetric)
    constexpr int kSlot[6][2] = {{0, 0}, {1, 3}, {2, 6}, {4, 4}, {5, 7}, {8, 8}};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      long long iw = ivir[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) iw += __shfl_xor_sync(0xffffffffu, iw, o);
      if (lane == 0) {
        add_fixed(a.virial + kSlot[k][0], iw);
        if (kSlot[k][1] != kSlot[k][0]) add_fixed(a.virial + kSlot[k][1], iw);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Grouped-queue variant.  The i-cluster is split into four 8-atom groups
// (the neighbour list orders each cluster as two z-halves of two x-halves,
// so a group is a compact 3.5 x 3.5 x 7 A block).  Every j-atom of a tile
// is tested against each group's live box and appended to that group's
// queue in shared memory (a 64-entry ring per group) with its position
// already in the i-cluster frame; the queues are consumed in batches of 8
// entries per group across tile boundaries.  Lane (g, l) computes the pairs
// of its i-atom with 8 entries of queue g, and the j-forces are combined
// over the group's 8 lanes (3 shuffle levels) before one atomic add per j.
// Fewer wasted pairs than testing all 32 i-atoms against a j that is only
// near part of the cluster, and no padding to 8 pairs per tile.
// ---------------------------------------------------------------------------

constexpr int kQ = 64;  // ring entries per group

__device__ __forceinline__ int sel4(int g, int a0, int a1, int a2, int a3) {
  return g == 0 ? a0 : g == 1 ? a1 : g == 2 ? a2 : a3;
}

// bits [start, start + n) of a 64-bit ring (n <= 64)
__device__ __forceinline__ unsigned long long ring_mask(int start, int n) {
  if (n <= 0) return 0ull;
  const unsigned long long m = n >= 64 ? ~0ull : ((1ull << n) - 1ull);
  const int s = start & 63;
  return s == 0 ? m : ((m << s) | (m >> (64 - s)));
}

template <bool ENERGY, bool PER_PAIR, bool VIRIAL, bool MULTI>
__global__ void __launch_bounds__(kThreads, 5) nbq_kernel(NbArgs a) {
  __shared__ float4 q_pos[kWarps][4][kQ];   // j position in the i frame, charge
  __shared__ int2 q_inf[kWarps][4][kQ];     // j slot, LJ type
  __shared__ float sh_box[kWarps][4][6];    // group boxes: lo xyz, hi xyz
  extern __shared__ float2 sh_vdw[];
  int T = a.ntype;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int g = lane >> 3;
  const int tab_off = MULTI ? wib * kMaxMultiTypes * kMaxMultiTypes : 0;
  int cur_sys = -1;
  if (!MULTI) {
    for (int k = threadIdx.x; k < T * T; k += blockDim.x) sh_vdw[k] = a.vdw[k];
    __syncthreads();
  }
  const unsigned lt_mask = (1u << lane) - 1u;
  const int nwork = a.counts[2];
  const int stride = a.stride;
  double e_elec = 0.0, e_vdw = 0.0;
  double dv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  // one system: per-lane fixed-point sums of every work item's energies and
  // virial (integer sums: the total does not depend on which warp took
  // which item)
  long long ie_el = 0, ie_vdw = 0;
  long long ivir[6] = {0, 0, 0, 0, 0, 0};
  using Acc = typename std::conditional<PER_PAIR, long long, float>::type;

  int taken = 0;  // warp-uniform
  auto next = [&]() -> int {
    if (a.items_per_warp > 0 && taken >= a.items_per_warp) return nwork;
    ++taken;
    return next_work(a.sched, lane);
  };
  for (int w = next(); w < nwork; w = next()) {
    const int4 wk = a.work[w];
    const NbSetup st = a.setups[wk.w];
    if (MULTI && wk.w != cur_sys) {  // warp-uniform
      __syncwarp();
      T = st.ntype;
      for (int k = lane; k < T * T; k += 32) sh_vdw[tab_off + k] = a.vdw[st.vdw_off + k];
      __syncwarp();
      cur_sys = wk.w;
    }
    const float4 oi = a.origin[wk.x];
    const int islot = wk.x * kTile + lane;
    const float4 xi = a.xyzq_s[islot];
    const bool ivalid = a.perm[islot] >= 0;
    const float qi = xi.w * (float)kCcelec;
    const int ti = a.type_s[islot] * T;
    // live box of this lane's group
    float lo_x = ivalid ? xi.x : INFINITY, lo_y = ivalid ? xi.y : INFINITY,
          lo_z = ivalid ? xi.z : INFINITY;
    float hi_x = ivalid ? xi.x : -INFINITY, hi_y = ivalid ? xi.y : -INFINITY,
          hi_z = ivalid ? xi.z : -INFINITY;
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      lo_x = fminf(lo_x, __shfl_xor_sync(0xffffffffu, lo_x, o));
      lo_y = fminf(lo_y, __shfl_xor_sync(0xffffffffu, lo_y, o));
      lo_z = fminf(lo_z, __shfl_xor_sync(0xffffffffu, lo_z, o));
      hi_x = fmaxf(hi_x, __shfl_xor_sync(0xffffffffu, hi_x, o));
      hi_y = fmaxf(hi_y, __shfl_xor_sync(0xffffffffu, hi_y, o));
      hi_z = fmaxf(hi_z, __shfl_xor_sync(0xffffffffu, hi_z, o));
    }
    __syncwarp();
    if ((lane & 7) == 0) {
      sh_box[wib][g][0] = lo_x;
      sh_box[wib][g][1] = lo_y;
      sh_box[wib][g][2] = lo_z;
      sh_box[wib][g][3] = hi_x;
      sh_box[wib][g][4] = hi_y;
      sh_box[wib][g][5] = hi_z;
    }
    __syncwarp();
    Acc fix = 0, fiy = 0, fiz = 0;
    float vw[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int h0 = 0, h1 = 0, h2 = 0, h3 = 0;   // ring heads (uniform)
    int t0 = 0, t1 = 0, t2 = 0, t3 = 0;   // ring tails (uniform)
    unsigned long long xmask = 0ull;      // excluded entries of my group, by ring position

    // consume up to 8 entries of every group
    auto batch = [&]() {
      const int head = sel4(g, h0, h1, h2, h3);
      const int cnt = min(8, sel4(g, t0, t1, t2, t3) - head);
      Acc fx[8], fy[8], fz[8];
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) {
        const int pos = (head + jj) & (kQ - 1);
        // entries past this group's count are stale ring contents (possibly
        // not even finite): they are masked and their differences zeroed
        const float4 pj = q_pos[wib][g][pos];
        const int tj = q_inf[wib][g][pos].y;
        float dx = xi.x - pj.x, dy = xi.y - pj.y, dz = xi.z - pj.z;
        const float r2raw = dx * dx + dy * dy + dz * dz;
        const bool in = jj < cnt && ivalid && !((xmask >> pos) & 1ull) && r2raw < st.roff2;
        dx = in ? dx : 0.f;
        dy = in ? dy : 0.f;
        dz = in ? dz : 0.f;
        // stale entries: an in-range table index and a finite charge
        const float2 cc = sh_vdw[tab_off + ti + (in ? tj : 0)];
        const float fij = pair_force<ENERGY>(st, r2raw, in, qi, in ? pj.w : 0.f, cc, e_elec, e_vdw);
        if (VIRIAL) {
          const float gx = fij * dx, gy = fij * dy, gz = fij * dz;
          vw[0] -= gx * dx;
          vw[1] -= gx * dy;
          vw[2] -= gx * dz;
          vw[3] -= gy * dy;
          vw[4] -= gy * dz;
          vw[5] -= gz * dz;
        }
        if (PER_PAIR) {
          const long long gx = to_fixed_force(fij * dx);
          const long long gy = to_fixed_force(fij * dy);
          const long long gz = to_fixed_force(fij * dz);
          fix += gx;
          fiy += gy;
          fiz += gz;
          fx[jj] = -gx;
          fy[jj] = -gy;
          fz[jj] = -gz;
        } else {
          fix += fij * dx;
          fiy += fij * dy;
          fiz += fij * dz;
          fx[jj] = -fij * dx;
          fy[jj] = -fij * dy;
          fz[jj] = -fij * dz;
        }
      }
      const Acc rx = group_reduce8(fx, lane);
      const Acc ry = group_reduce8(fy, lane);
      const Acc rz = group_reduce8(fz, lane);
      const int own = lane & 7;
      if (own < cnt) {
        const int js = q_inf[wib][g][(head + own) & (kQ - 1)].x;
        if (PER_PAIR) {
          add_fixed(a.force + js, (long long)rx);
          add_fixed(a.force + stride + js, (long long)ry);
          add_fixed(a.force + 2 * stride + js, (long long)rz);
        } else {
          add_fixed(a.force + js, to_fixed_force((float)rx));
          add_fixed(a.force + stride + js, to_fixed_force((float)ry));
          add_fixed(a.force + 2 * stride + js, to_fixed_force((float)rz));
        }
      }
      xmask &= ~ring_mask(head, cnt > 0 ? cnt : 0);
      h0 += min(8, t0 - h0);
      h1 += min(8, t1 - h1);
      h2 += min(8, t2 - h2);
      h3 += min(8, t3 - h3);
      __syncwarp();
    };

    // one call site for the batch and one for the enqueue (code size: the
    // batch is an unrolled 8-pair loop): full batches while every group has
    // 8 waiting; before a tile, at most 32 waiting per group so that the tile
    // fits the rings; after the last tile, until the rings are empty
    int t = wk.y;
    for (;;) {
      const int fmin = min(min(t0 - h0, t1 - h1), min(t2 - h2, t3 - h3));
      const int fmax = max(max(t0 - h0, t1 - h1), max(t2 - h2, t3 - h3));
      if (fmin >= 8 || fmax > kQ - 32 || (t >= wk.z && fmax > 0)) {
        batch();
        continue;
      }
      if (t >= wk.z) break;
      const int2 tl = a.tiles[t];
      const int code = tile_image(tl.y);
      const float4 oj = a.origin[tl.x];
      const int ic = code / 9, ib = (code - 9 * ic) / 3, ia = code - 9 * ic - 3 * ib;
      const float kx = (float)(ia - 1), ky = (float)(ib - 1), kz = (float)(ic - 1);
      const float sx = fmaf(kx, st.Lx, oj.x - oi.x) + kx * st.Lx_lo;
      const float sy = fmaf(ky, st.Ly, oj.y - oi.y) + ky * st.Ly_lo;
      const float sz = fmaf(kz, st.Lz, oj.z - oi.z) + kz * st.Lz_lo;
      const int jslot = tl.x * kTile + lane;
      float4 xj = a.xyzq_s[jslot];
      xj.x += sx;
      xj.y += sy;
      xj.z += sz;
      const bool jvalid = a.perm[jslot] >= 0;
      const int tj = a.type_s[jslot];
      const unsigned excl = tile_excl_word(a, tl, code, wk.x, lane);
      const bool any_excl = __any_sync(0xffffffffu, ivalid && excl != 0u);
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const float *bb = sh_box[wib][h];
        const float bx = fmaxf(0.f, fmaxf(bb[0] - xj.x, xj.x - bb[3]));
        const float by = fmaxf(0.f, fmaxf(bb[1] - xj.y, xj.y - bb[4]));
        const float bz = fmaxf(0.f, fmaxf(bb[2] - xj.z, xj.z - bb[5]));
        const bool near = jvalid && bx * bx + by * by + bz * bz < st.roff2;
        const unsigned m = __ballot_sync(0xffffffffu, near);
        const int tail = h == 0 ? t0 : h == 1 ? t1 : h == 2 ? t2 : t3;
        if (near) {
          const int pos = (tail + __popc(m & lt_mask)) & (kQ - 1);
          q_pos[wib][h][pos] = xj;
          q_inf[wib][h][pos] = make_int2(jslot, tj);
        }
        if (any_excl && g == h && ivalid && excl != 0u) {
          unsigned mm = m & excl;   // excluded among the new entries, in order
          while (mm) {
            const int k = __ffs(mm) - 1;
            mm &= mm - 1u;
            xmask |= 1ull << ((tail + __popc(m & ((1u << k) - 1u))) & (kQ - 1));
          }
        }
        const int n = __popc(m);
        if (h == 0) t0 += n;
        else if (h == 1) t1 += n;
        else if (h == 2) t2 += n;
        else t3 += n;
      }
      __syncwarp();
      ++t;
    }

    if (VIRIAL) {
#pragma unroll
      for (int k = 0; k < 6; ++k) dv[k] += (double)vw[k];
    }
    if (MULTI && ENERGY) {
      long long *es = a.energy + (size_t)wk.w * a.energy_stride;
      warp_flush(e_elec, es + kEElec, lane);
      warp_flush(e_vdw, es + kEVdw, lane);
      e_elec = 0.0;
      e_vdw = 0.0;
      if (VIRIAL) {
        constexpr int kSlotM[6][2] = {{0, 0}, {1, 3}, {2, 6}, {4, 4}, {5, 7}, {8, 8}};
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          long long iw = __double2ll_rn(dv[k] * kEnergyScale);
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) iw += __shfl_xor_sync(0xffffffffu, iw, o);
          if (lane == 0 && iw) {
            add_fixed(es + kNumEnergyTerms + kSlotM[k][0], iw);
            if (kSlotM[k][1] != kSlotM[k][0]) add_fixed(es + kNumEnergyTerms + kSlotM[k][1], iw);
          }
          dv[k] = 0.0;
        }
      }
    }
    if (ENERGY && !MULTI) {
      ie_el += __double2ll_rn(e_elec * kEnergyScale);
      ie_vdw += __double2ll_rn(e_vdw * kEnergyScale);
      e_elec = 0.0;
      e_vdw = 0.0;
      if (VIRIAL) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          ivir[k] += __double2ll_rn(dv[k] * kEnergyScale);
          dv[k] = 0.0;
        }
      }
    }
    if (ivalid) {
      if (PER_PAIR) {
        add_fixed(a.force + islot, (long long)fix);
        add_fixed(a.force + stride + islot, (long long)fiy);
        add_fixed(a.force + 2 * stride + islot, (long long)fiz);
      } else {
        add_fixed(a.force + islot, to_fixed_force((float)fix));
        add_fixed(a.force + stride + islot, to_fixed_force((float)fiy));
        add_fixed(a.force + 2 * stride + islot, to_fixed_force((float)fiz));
      }
    }
  }
  retire_warp(a.sched, lane);
  if (ENERGY && !MULTI) {
    long long ie = ie_el, iv = ie_vdw;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ie += __shfl_xor_sync(0xffffffffu, ie, o);
      iv += __shfl_xor_sync(0xffffffffu, iv, o);
    }
    if (lane == 0) {
      add_fixed(a.energy + kEElec, ie);
      add_fixed(a.energy + kEVdw, iv);
    }
  }
  if (VIRIAL && !MULTI) {
    constexpr int kSlot[6][2] = {{0, 0}, {1, 3}, {2, 6}, {4, 4}, {5, 7}, {8, 8}};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      long long iw = ivir[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) iw += __shfl_xor_sync(0xffffffffu, iw, o);
      if (lane == 0) {
        add_fixed(a.virial + kSlot[k][0], iw);
        if (kSlot[k][1] != kSlot[k][0]) add_fixed(a.virial + kSlot[k][1], iw);
      }
    }
  }
}

// persistent grid (resident blocks) or, with a bound on the items per warp,
// enough blocks for every work item the list can hold
int launch_grid(int resident, const NbArgs &a) {
  if (a.items_per_warp <= 0) return resident;
  const long long per_block = (long long)kWarps * a.items_per_warp;
  const long long need = ((long long)a.work_cap + per_block - 1) / per_block;
  return (int)std::max<long long>(resident, std::min<long long>(need, 1ll << 30));
}

template <bool E, bool P, bool V, bool M>
void launch_q(const NbArgs &a, cudaStream_t s) {
  static int grid = 0;
  size_t sm = M ? (size_t)kWarps * kMaxMultiTypes * kMaxMultiTypes * sizeof(float2)
                : (size_t)a.ntype * a.ntype * sizeof(float2);
  if (!grid) {
    int dev, nsm, per = 0;
    APO_CUDA(cudaGetDevice(&dev));
    APO_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    APO_CUDA(cudaFuncSetAttribute(nbq_kernel<E, P, V, M>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    APO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, nbq_kernel<E, P, V, M>, kThreads,
                                                           64 * 1024 > sm ? sm : 64 * 1024));
    grid = nsm * (per > 0 ? per : 1);
  }
  nbq_kernel<E, P, V, M><<<launch_grid(grid, a), kThreads, sm, s>>>(a);
  APO_LAUNCH_CHECK();
}

template <bool M>
void dispatch_q(const NbArgs &a, bool energy, bool per_pair, bool virial, cudaStream_t s) {
  if (virial) {
    if (per_pair) launch_q<true, true, true, M>(a, s);
    else launch_q<true, false, true, M>(a, s);
  } else if (energy) {
    if (per_pair) launch_q<true, true, false, M>(a, s);
    else launch_q<true, false, false, M>(a, s);
  } else {
    if (per_pair) launch_q<false, true, false, M>(a, s);
    else launch_q<false, false, false, M>(a, s);
  }
}

template <bool E, bool P, bool V = false, bool M = false>
void launch_t(const NbArgs &a, cudaStream_t s) {
  static int grid = 0;
  size_t sm = M ? (size_t)kWarps * kMaxMultiTypes * kMaxMultiTypes * sizeof(float2)
                : (size_t)a.ntype * a.ntype * sizeof(float2);
  if (!grid) {
    int dev, nsm, per = 0;
    APO_CUDA(cudaGetDevice(&dev));
    APO_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    APO_CUDA(cudaFuncSetAttribute(nb_kernel<E, P, V, M>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    APO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, nb_kernel<E, P, V, M>, kThreads,
                                                           64 * 1024 > sm ? sm : 64 * 1024));
    grid = nsm * (per > 0 ? per : 1);
  }
  nb_kernel<E, P, V, M><<<launch_grid(grid, a), kThreads, sm, s>>>(a);
  APO_LAUNCH_CHECK();
}

}  // namespace

void launch_nonbonded(const NbArgs &a, bool energy, bool per_pair, cudaStream_t s, bool virial) {
  if (!a.sched) throw std::invalid_argument("nonbonded: no schedule counters");
  if (a.ntype * a.ntype * sizeof(float2) > 64 * 1024)
    throw std::invalid_argument("nonbonded: too many LJ types for the shared table");
  if (virial && !a.virial) throw std::invalid_argument("nonbonded: virial requested without a buffer");
  if (a.variant == kNbGroupedQueues) return dispatch_q<false>(a, energy, per_pair, virial, s);
  if (a.variant == kNbOctetLists) return launch_nonbonded_octets(a, energy, per_pair, virial, false, s);
  if (virial) {
    if (!a.virial) throw std::invalid_argument("nonbonded: virial requested without a buffer");
    if (per_pair) launch_t<true, true, true>(a, s);
    else launch_t<true, false, true>(a, s);
    return;
  }
  if (per_pair) {
    if (energy) launch_t<true, true>(a, s);
    else launch_t<false, true>(a, s);
  } else {
    if (energy) launch_t<true, false>(a, s);
    else launch_t<false, false>(a, s);
  }
}

void launch_nonbonded_multi(const NbArgs &a, bool energy, bool per_pair, cudaStream_t s,
                            bool virial) {
  if (!a.sched) throw std::invalid_argument("nonbonded: no schedule counters");
  if (a.energy_stride <= 0 && (energy || virial))
    throw std::invalid_argument("nonbonded: multi-system energies need an energy stride");
  if (a.variant == kNbGroupedQueues) return dispatch_q<true>(a, energy, per_pair, virial, s);
  if (a.variant == kNbOctetLists) return launch_nonbonded_octets(a, energy, per_pair, virial, true, s);
  if (virial) {
    if (per_pair) launch_t<true, true, true, true>(a, s);
    else launch_t<true, false, true, true>(a, s);
  } else if (energy) {
    if (per_pair) launch_t<true, true, false, true>(a, s);
    else launch_t<true, false, false, true>(a, s);
  } else {
    if (per_pair) launch_t<false, true, false, true>(a, s);
    else launch_t<false, false, false, true>(a, s);
  }
}

}  // namespace apo
