// Direct-space kernel, octet-list form; see nonbonded.h.
//
// One warp per work item (an i-cluster and a run of its j-tiles), as the
// tile-batch form, but the 32 lanes are four octets: lane (g, l) owns i-atom
// 8g + l of the cluster (the neighbour list orders every cluster as
// x-ordered z-halves, so an octet is a compact 8-atom block) and keeps its
// force in registers.  The work item's j-atoms are staged once in shared
// memory: every j that passes the cluster's live box is stored with its
// position already in the i-cluster frame, and appended to the list of each
// octet whose own box it reaches.  The four lists cover the whole work item
// (up to kJCap staged atoms), so their lengths even out over the tiles.
// Octet g then walks its own list, eight entries per batch, computing the
// pairs of its 8 i-atoms with one j each: a pair slot is spent only on a j
// near the octet, about 1.4x fewer slots than testing all 32 i-atoms against
// every j near the cluster.  The j-forces of a batch are summed over the
// octet's 8 lanes by a shuffle transpose and added to the staged atom's
// accumulator in shared memory, octet by octet in a fixed order (the float
// sums do not depend on the schedule); at the end of the chunk every staged
// atom's force goes to the fixed-point force buffer with one atomic per
// component.  Exclusions: a tile with a topological exclusion (or a
// cluster's tile with itself) transposes its mask words across the warp, so
// each list entry carries the 8 exclusion bits of its octet.
#include "nonbonded.h"

#include <algorithm>
#include <type_traits>

#include "device_util.cuh"
#include "nblist.h"
#include "nonbonded_pair.cuh"

namespace apo {
namespace {

using namespace nbdetail;

constexpr int kOWarps = 4;
constexpr int kOThreads = kOWarps * 32;
constexpr int kJCap = 160;  // staged j-atoms per warp and chunk (list entries hold 8 bits)

static_assert(kJCap <= 256, "list entries store the staged index in 8 bits");

// 32 x 32 bit transpose across the warp: on entry bit j of lane i is element
// (i, j), on return bit i of lane j is element (i, j) (block swaps of 16,
// 8, 4, 2 and 1 bits)
__device__ __forceinline__ unsigned bit_transpose(unsigned x, int lane) {
  unsigned y = __shfl_xor_sync(0xffffffffu, x, 16);
  x = (lane & 16) ? ((x & 0xFFFF0000u) | (y >> 16)) : ((x & 0x0000FFFFu) | (y << 16));
  y = __shfl_xor_sync(0xffffffffu, x, 8);
  x = (lane & 8) ? ((x & 0xFF00FF00u) | ((y >> 8) & 0x00FF00FFu))
                 : ((x & 0x00FF00FFu) | ((y << 8) & 0xFF00FF00u));
  y = __shfl_xor_sync(0xffffffffu, x, 4);
  x = (lane & 4) ? ((x & 0xF0F0F0F0u) | ((y >> 4) & 0x0F0F0F0Fu))
                 : ((x & 0x0F0F0F0Fu) | ((y << 4) & 0xF0F0F0F0u));
  y = __shfl_xor_sync(0xffffffffu, x, 2);
  x = (lane & 2) ? ((x & 0xCCCCCCCCu) | ((y >> 2) & 0x33333333u))
                 : ((x & 0x33333333u) | ((y << 2) & 0xCCCCCCCCu));
  y = __shfl_xor_sync(0xffffffffu, x, 1);
  x = (lane & 1) ? ((x & 0xAAAAAAAAu) | ((y >> 1) & 0x55555555u))
                 : ((x & 0x55555555u) | ((y << 1) & 0xAAAAAAAAu));
  return x;
}

__device__ __forceinline__ int sel4i(int g, int a0, int a1, int a2, int a3) {
  return g == 0 ? a0 : g == 1 ? a1 : g == 2 ? a2 : a3;
}

// squared distance from a point to an axis-aligned box (0 inside)
__device__ __forceinline__ float box_d2(const float4 &lo, const float4 &hi, const float4 &p) {
  const float bx = fmaxf(0.f, fmaxf(lo.x - p.x, p.x - hi.x));
  const float by = fmaxf(0.f, fmaxf(lo.y - p.y, p.y - hi.y));
  const float bz = fmaxf(0.f, fmaxf(lo.z - p.z, p.z - hi.z));
  return bx * bx + by * by + bz * bz;
}

template <bool ENERGY, bool PER_PAIR, bool VIRIAL, bool MULTI>
__global__ void __launch_bounds__(kOThreads, 5) nbo_kernel(NbArgs a) {
  using Acc = typename std::conditional<PER_PAIR, long long, float>::type;
  __shared__ float4 s_pos[kOWarps][kJCap];           // j position in the i frame, charge
  __shared__ int s_slot[kOWarps][kJCap];             // j sorted slot
  __shared__ Acc s_f[kOWarps][3][kJCap];             // j force of the chunk
  __shared__ unsigned s_list[kOWarps][4][kJCap];     // k | LJ type << 8 | octet exclusions << 16
  __shared__ float4 s_box[kOWarps][4][2];            // octet boxes (lo, hi)
  extern __shared__ float2 sh_vdw[];
  int T = a.ntype;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int g = lane >> 3, l = lane & 7;
  const int tab_off = MULTI ? wib * kMaxMultiTypes * kMaxMultiTypes : 0;
  int cur_sys = -1;
  if (!MULTI) {
    for (int k = threadIdx.x; k < T * T; k += blockDim.x) sh_vdw[k] = a.vdw[k];
  }
  for (int k = lane; k < kJCap; k += 32) {
    s_f[wib][0][k] = 0;
    s_f[wib][1][k] = 0;
    s_f[wib][2][k] = 0;
  }
  __syncthreads();
  const unsigned lt_mask = (1u << lane) - 1u;
  const int nwork = a.counts[2];
  const int stride = a.stride;
  double e_elec = 0.0, e_vdw = 0.0;
  double dv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  long long ie_el = 0, ie_vdw = 0;
  long long ivir[6] = {0, 0, 0, 0, 0, 0};

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
    // live boxes: this lane's octet, then the whole cluster
    float lo_x = ivalid ? xi.x : INFINITY, lo_y = ivalid ? xi.y : INFINITY,
          lo_z = ivalid ? xi.z : INFINITY;
    float hi_x = ivalid ? xi.x : -INFINITY, hi_y = ivalid ? xi.y : -INFINITY,
          hi_z = ivalid ? xi.z : -INFINITY;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      lo_x = fminf(lo_x, __shfl_xor_sync(0xffffffffu, lo_x, o));
      lo_y = fminf(lo_y, __shfl_xor_sync(0xffffffffu, lo_y, o));
      lo_z = fminf(lo_z, __shfl_xor_sync(0xffffffffu, lo_z, o));
      hi_x = fmaxf(hi_x, __shfl_xor_sync(0xffffffffu, hi_x, o));
      hi_y = fmaxf(hi_y, __shfl_xor_sync(0xffffffffu, hi_y, o));
      hi_z = fmaxf(hi_z, __shfl_xor_sync(0xffffffffu, hi_z, o));
      if (o == 4 && l == 0) {  // the octet's box is complete after xor 1, 2, 4
        s_box[wib][g][0] = make_float4(lo_x, lo_y, lo_z, 0.f);
        s_box[wib][g][1] = make_float4(hi_x, hi_y, hi_z, 0.f);
      }
    }
    const float4 clo = make_float4(lo_x, lo_y, lo_z, 0.f), chi = make_float4(hi_x, hi_y, hi_z, 0.f);
    __syncwarp();
    Acc fix = 0, fiy = 0, fiz = 0;
    float vw[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int c0 = 0, c1 = 0, c2 = 0, c3 = 0;  // list lengths (uniform)
    int base = 0;                        // staged atoms (uniform)

    // the pairs of every octet with its list, then the staged j-forces out
    auto run_lists = [&]() {
      __syncwarp();
      const int mycnt = sel4i(g, c0, c1, c2, c3);
      const int steps = max(max(c0, c1), max(c2, c3));
      for (int s0 = 0; s0 < steps; s0 += 8) {
        Acc fx[8], fy[8], fz[8];
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
          const int s = s0 + jj;
          const bool valid = s < mycnt;
          // entries past this octet's list are never read: index 0, type 0, out
          const unsigned e = valid ? s_list[wib][g][s] : 0u;
          const float4 pj = s_pos[wib][e & 0xffu];
          const float dx = xi.x - pj.x, dy = xi.y - pj.y, dz = xi.z - pj.z;
          const float r2raw = dx * dx + dy * dy + dz * dz;
          const bool in = valid && ivalid && !((e >> (16 + l)) & 1u) && r2raw < st.roff2;
          const float2 cc = sh_vdw[tab_off + ti + ((e >> 8) & 0xffu)];
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
        // lane (g, l) now holds the octet's total on entry s0 + l
        const Acc rx = group_reduce8(fx, lane);
        const Acc ry = group_reduce8(fy, lane);
        const Acc rz = group_reduce8(fz, lane);
        const int so = s0 + l;
        const int own = so < mycnt ? (int)(s_list[wib][g][so] & 0xffu) : -1;
        // octet by octet: an atom in two octets' lists is summed in a fixed order
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          if (g == h && own >= 0) {
            s_f[wib][0][own] += rx;
            s_f[wib][1][own] += ry;
            s_f[wib][2][own] += rz;
          }
          __syncwarp();
        }
      }
      for (int k = lane; k < base; k += 32) {
        const Acc vx = s_f[wib][0][k], vy = s_f[wib][1][k], vz = s_f[wib][2][k];
        const int js = s_slot[wib][k];
        if (PER_PAIR) {
          if (vx) add_fixed(a.force + js, (long long)vx);
          if (vy) add_fixed(a.force + stride + js, (long long)vy);
          if (vz) add_fixed(a.force + 2 * stride + js, (long long)vz);
        } else {
          if (vx != 0) add_fixed(a.force + js, to_fixed_force((float)vx));
          if (vy != 0) add_fixed(a.force + stride + js, to_fixed_force((float)vy));
          if (vz != 0) add_fixed(a.force + 2 * stride + js, to_fixed_force((float)vz));
        }
        s_f[wib][0][k] = 0;
        s_f[wib][1][k] = 0;
        s_f[wib][2][k] = 0;
      }
      __syncwarp();
      c0 = c1 = c2 = c3 = 0;
      base = 0;
    };

    for (int t = wk.y; t < wk.z; ++t) {
      const int2 tl = a.tiles[t];
      const int code = tile_image(tl.y);
      // j cluster frame -> i cluster frame (exact origin difference plus the
      // periodic image with L as a two-float sum)
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
      const bool near_c = a.perm[jslot] >= 0 && box_d2(clo, chi, xj) < st.roff2;
      const unsigned cmask = __ballot_sync(0xffffffffu, near_c);
      if (cmask == 0u) continue;
      const int nj = __popc(cmask);
      if (base + nj > kJCap) run_lists();
      const unsigned excl = tile_excl_word(a, tl, code, wk.x, lane);
      // lane (as a j-atom of the tile): bit i = pair (i, this j) excluded
      const unsigned col = __any_sync(0xffffffffu, excl != 0u) ? bit_transpose(excl, lane) : 0u;
      const int k = base + __popc(cmask & lt_mask);
      const unsigned tj = (unsigned)a.type_s[jslot];
      if (near_c) {
        s_pos[wib][k] = xj;
        s_slot[wib][k] = jslot;
      }
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const bool near = near_c && box_d2(s_box[wib][h][0], s_box[wib][h][1], xj) < st.roff2;
        const unsigned m = __ballot_sync(0xffffffffu, near);
        const int cnt = h == 0 ? c0 : h == 1 ? c1 : h == 2 ? c2 : c3;
        if (near)
          s_list[wib][h][cnt + __popc(m & lt_mask)] =
              (unsigned)k | (tj << 8) | (((col >> (8 * h)) & 0xffu) << 16);
        const int n = __popc(m);
        if (h == 0) c0 += n;
        else if (h == 1) c1 += n;
        else if (h == 2) c2 += n;
        else c3 += n;
      }
      base += nj;
    }
    if (base) run_lists();

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
int grid_for(int resident, const NbArgs &a) {
  if (a.items_per_warp <= 0) return resident;
  const long long per_block = (long long)kOWarps * a.items_per_warp;
  const long long need = ((long long)a.work_cap + per_block - 1) / per_block;
  return (int)std::max<long long>(resident, std::min<long long>(need, 1ll << 30));
}

template <bool E, bool P, bool V, bool M>
void launch_o(const NbArgs &a, cudaStream_t s) {
  static int grid = 0;
  const size_t sm = M ? (size_t)kOWarps * kMaxMultiTypes * kMaxMultiTypes * sizeof(float2)
                      : (size_t)a.ntype * a.ntype * sizeof(float2);
  if (!grid) {
    int dev, nsm, per = 0;
    APO_CUDA(cudaGetDevice(&dev));
    APO_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    APO_CUDA(cudaFuncSetAttribute(nbo_kernel<E, P, V, M>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    APO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, nbo_kernel<E, P, V, M>, kOThreads,
                                                           64 * 1024 > sm ? sm : 64 * 1024));
    grid = nsm * (per > 0 ? per : 1);
  }
  nbo_kernel<E, P, V, M><<<grid_for(grid, a), kOThreads, sm, s>>>(a);
  APO_LAUNCH_CHECK();
}

}  // namespace

void launch_nonbonded_octets(const NbArgs &a, bool energy, bool per_pair, bool virial, bool multi,
                             cudaStream_t s) {
  if (multi) {
    if (virial) {
      if (per_pair) launch_o<true, true, true, true>(a, s);
      else launch_o<true, false, true, true>(a, s);
    } else if (energy) {
      if (per_pair) launch_o<true, true, false, true>(a, s);
      else launch_o<true, false, false, true>(a, s);
    } else {
      if (per_pair) launch_o<false, true, false, true>(a, s);
      else launch_o<false, false, false, true>(a, s);
    }
    return;
  }
  if (virial) {
    if (per_pair) launch_o<true, true, true, false>(a, s);
    else launch_o<true, false, true, false>(a, s);
  } else if (energy) {
    if (per_pair) launch_o<true, true, false, false>(a, s);
    else launch_o<true, false, false, false>(a, s);
  } else {
    if (per_pair) launch_o<false, true, false, false>(a, s);
    else launch_o<false, false, false, false>(a, s);
  }
}

}  // namespace apo
