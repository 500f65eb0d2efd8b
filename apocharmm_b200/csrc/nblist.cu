// Neighbour-list kernels; see nblist.h.
#include "nblist.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "device_util.cuh"

namespace apo {
namespace {

constexpr int kScanThreads = 1024;

__device__ __forceinline__ int floor_div(int a, int b) {
  return a >= 0 ? a / b : -((-a + b - 1) / b);
}

// (1) bin atoms into x-y columns; record wrapped z key and image shift
__global__ void bin_kernel(int n, const float4 *__restrict__ xyzq,
                           const int *__restrict__ sys_of_atom,
                           const NbSysDims *__restrict__ sysd,
                           int *__restrict__ col_count, int *__restrict__ atom_col,
                           int *__restrict__ atom_rank, float4 *__restrict__ atom_shift,
                           float *__restrict__ zkey, unsigned *__restrict__ err) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const NbSysDims d = sysd[sys_of_atom[g]];
  float4 p = xyzq[g];
  float sx = 0.f, sy = 0.f, sz = 0.f;
  int col = 0;
  float zw = 0.f;
  if (isfinite(p.x) && isfinite(p.y) && isfinite(p.z)) {
    float ix = floorf(p.x / d.Lx + 0.5f), iy = floorf(p.y / d.Ly + 0.5f),
          iz = floorf(p.z / d.Lz + 0.5f);
    sx = -ix * d.Lx;
    sy = -iy * d.Ly;
    sz = -iz * d.Lz;
    float xw = p.x + sx, yw = p.y + sy;
    zw = p.z + sz;
    int cx = (int)((xw + 0.5f * d.Lx) * ((float)d.ncx / d.Lx));
    int cy = (int)((yw + 0.5f * d.Ly) * ((float)d.ncy / d.Ly));
    cx = min(max(cx, 0), d.ncx - 1);
    cy = min(max(cy, 0), d.ncy - 1);
    col = d.col_off + cx + d.ncx * cy;
  } else {
    atomicOr(err, (unsigned)kErrNaN);
    col = d.col_off;
  }
  atom_col[g] = col;
  atom_rank[g] = atomicAdd(&col_count[col], 1);
  atom_shift[g] = make_float4(sx, sy, sz, 0.f);
  zkey[g] = zw;
}

// block-wide exclusive scan helper (kScanThreads threads)
__device__ int block_exclusive_scan(int v, int *sh, int &total) {
  int t = threadIdx.x;
  sh[t] = v;
  __syncthreads();
  for (int o = 1; o < kScanThreads; o <<= 1) {
    int a = t >= o ? sh[t - o] : 0;
    __syncthreads();
    sh[t] += a;
    __syncthreads();
  }
  total = sh[kScanThreads - 1];
  int r = sh[t] - v;
  __syncthreads();
  return r;
}

// (2) padded column offsets; slot totals
__global__ void col_scan_kernel(int ncol, const int *__restrict__ col_count,
                                int *__restrict__ col_start, int *__restrict__ counts,
                                int slot_cap, int sort_cap, unsigned *__restrict__ err) {
  __shared__ int sh[kScanThreads];
  int carry = 0;
  bool over = false;
  for (int base = 0; base < ncol; base += kScanThreads) {
    int c = base + threadIdx.x;
    int cnt = c < ncol ? col_count[c] : 0;
    if (cnt > sort_cap) over = true;
    int padded = (cnt + kTile - 1) / kTile * kTile;
    int tot;
    int ex = block_exclusive_scan(padded, sh, tot);
    if (c < ncol) col_start[c] = carry + ex;
    carry += tot;
  }
  if (over) atomicOr(err, (unsigned)kErrColumnOverflow);
  if (threadIdx.x == 0) {
    col_start[ncol] = carry;
    if (carry > slot_cap) {
      atomicOr(err, (unsigned)kErrColumnOverflow);
      carry = 0;
    }
    counts[0] = carry;
  }
}

// (3) scatter atoms to their column's slot range (order inside a column is
// fixed afterwards by the column sort)
__global__ void scatter_kernel(int n, const int *__restrict__ atom_col,
                               const int *__restrict__ atom_rank,
                               const int *__restrict__ col_start,
                               const float *__restrict__ zkey, float *__restrict__ tkey,
                               int *__restrict__ tidx, const int *__restrict__ counts) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n || counts[0] == 0) return;
  int s = col_start[atom_col[g]] + atom_rank[g];
  tkey[s] = zkey[g];
  tidx[s] = g;
}

// (4) one block per column: bitonic sort by (z, atom index); write the
// permutation, its inverse, shifts, types and the cluster -> column map
__global__ void col_sort_kernel(int ncol, const int *__restrict__ col_count,
                                const int *__restrict__ col_start,
                                const float *__restrict__ tkey, const int *__restrict__ tidx,
                                const float4 *__restrict__ atom_shift,
                                const int *__restrict__ vdwtype, int *__restrict__ perm,
                                int *__restrict__ glo2loc, float4 *__restrict__ slot_shift,
                                int *__restrict__ type_s, int *__restrict__ cl_col,
                                const int *__restrict__ col_sys, int *__restrict__ cl_sys,
                                const int *__restrict__ counts, int sort_cap,
                                const float4 *__restrict__ xyzq) {
  extern __shared__ unsigned char smem[];
  float *sk = reinterpret_cast<float *>(smem);
  int *si = reinterpret_cast<int *>(smem + sizeof(float) * sort_cap);
  int *so = si + sort_cap;
  int col = blockIdx.x;
  if (col >= ncol || counts[0] == 0) return;
  int cnt = col_count[col];
  int start = col_start[col];
  int padded = col_start[col + 1] - start;
  if (cnt > sort_cap) return;
  int P = 1;
  while (P < cnt) P <<= 1;
  for (int k = threadIdx.x; k < P; k += blockDim.x) {
    if (k < cnt) {
      sk[k] = tkey[start + k];
      si[k] = tidx[start + k];
    } else {
      sk[k] = INFINITY;
      si[k] = 0x7fffffff;
    }
  }
  __syncthreads();
  for (int size = 2; size <= P; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int k = threadIdx.x; k < P; k += blockDim.x) {
        int l = k ^ stride;
        if (l > k) {
          bool up = (k & size) == 0;
          float ka = sk[k], kb = sk[l];
          int ia = si[k], ib = si[l];
          bool gt = (ka > kb) || (ka == kb && ia > ib);
          if (gt == up) {
            sk[k] = kb;
            sk[l] = ka;
            si[k] = ib;
            si[l] = ia;
          }
        }
      }
      __syncthreads();
    }
  }
  // inside every 32-atom cluster: the lower and the upper z-half, each
  // ordered by x, so that slots 8m..8m+7 form compact 8-atom blocks (the
  // direct-space kernel's i-groups); ties by atom index
  for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
    const int g = si[k];
    sk[k] = xyzq[g].x + atom_shift[g].x;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
    const int c0 = k & ~15, n16 = min(16, cnt - c0);
    const float xk = sk[k];
    const int gk = si[k];
    int rank = 0;
    for (int m = c0; m < c0 + n16; ++m) {
      const float xm = sk[m];
      rank += (xm < xk || (xm == xk && si[m] < gk)) ? 1 : 0;
    }
    so[c0 + rank] = gk;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < padded; k += blockDim.x) {
    int s = start + k;
    if (k < cnt) {
      int g = so[k];
      perm[s] = g;
      glo2loc[g] = s;
      slot_shift[s] = atom_shift[g];
      type_s[s] = vdwtype[g];
    } else {
      perm[s] = -1;
      slot_shift[s] = make_float4(0.f, 0.f, 0.f, 0.f);
      type_s[s] = 0;
    }
    if ((k & (kTile - 1)) == 0) {
      cl_col[s / kTile] = col;
      cl_sys[s / kTile] = col_sys[col];
    }
  }
}

// (4b) cluster origins, one warp per cluster: the centre of the wrapped
// positions rounded to a multiple of 1/64 A (exact in single precision for
// any box below 2^17 A), and per slot the FP64 offset image shift - origin
__global__ void origin_kernel(const float4 *__restrict__ xyzq, const int *__restrict__ perm,
                              const float4 *__restrict__ slot_shift,
                              const NbSysDims *__restrict__ sysd, const int *__restrict__ cl_sys,
                              float4 *__restrict__ cl_origin, double4 *__restrict__ slot_off,
                              const int *__restrict__ counts) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= counts[0] / kTile) return;
  const NbSysDims d = sysd[cl_sys[w]];
  const int s = w * kTile + lane;
  const int g = perm[s];
  float4 p = make_float4(0.f, 0.f, 0.f, 0.f), sh = slot_shift[s];
  if (g >= 0) p = xyzq[g];
  const bool valid = g >= 0;
  float mnx = valid ? p.x + sh.x : INFINITY, mny = valid ? p.y + sh.y : INFINITY,
        mnz = valid ? p.z + sh.z : INFINITY;
  float mxx = valid ? p.x + sh.x : -INFINITY, mxy = valid ? p.y + sh.y : -INFINITY,
        mxz = valid ? p.z + sh.z : -INFINITY;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
    mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
    mnz = fminf(mnz, __shfl_xor_sync(0xffffffffu, mnz, o));
    mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
    mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
    mxz = fmaxf(mxz, __shfl_xor_sync(0xffffffffu, mxz, o));
  }
  float ox = 0.f, oy = 0.f, oz = 0.f;
  if (mnx <= mxx) {  // at least one atom
    ox = rintf(0.5f * (mnx + mxx) * 64.f) * (1.f / 64.f);
    oy = rintf(0.5f * (mny + mxy) * 64.f) * (1.f / 64.f);
    oz = rintf(0.5f * (mnz + mxz) * 64.f) * (1.f / 64.f);
  }
  if (lane == 0) cl_origin[w] = make_float4(ox, oy, oz, 0.f);
  // the wrap shift is k * L with a small integer k
  const double kx = rint((double)sh.x / (double)d.Lx), ky = rint((double)sh.y / (double)d.Ly),
               kz = rint((double)sh.z / (double)d.Lz);
  slot_off[s] = make_double4(kx * d.Lxd - (double)ox, ky * d.Lyd - (double)oy,
                             kz * d.Lzd - (double)oz, 0.0);
}

// a new box for the built list: slot_off = k L - origin becomes k L' - origin
// (k recovered from the old box; the origins stay)
__global__ void rescale_dev_kernel(double4 *__restrict__ slot_off,
                                   const float4 *__restrict__ cl_origin,
                                   const double *__restrict__ L0, const double *__restrict__ L1,
                                   const unsigned *__restrict__ err, const int *__restrict__ counts) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (*err || s >= counts[0]) return;
  const float4 o = cl_origin[s / kTile];
  double4 v = slot_off[s];
  const double kx = rint((v.x + (double)o.x) / L0[0]), ky = rint((v.y + (double)o.y) / L0[1]),
               kz = rint((v.z + (double)o.z) / L0[2]);
  v.x = kx * L1[0] - (double)o.x;
  v.y = ky * L1[1] - (double)o.y;
  v.z = kz * L1[2] - (double)o.z;
  slot_off[s] = v;
}

// sorted, cluster-local coordinates (runs after every coordinate update)
__global__ void refresh_kernel(const double4 *__restrict__ coords, const int *__restrict__ perm,
                               const double4 *__restrict__ slot_off,
                               float4 *__restrict__ xyzq_s, const int *__restrict__ counts) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= counts[0]) return;
  int g = perm[s];
  float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
  if (g >= 0) {
    const double4 c = coords[g], o = slot_off[s];
    out = make_float4((float)(c.x + o.x), (float)(c.y + o.y), (float)(c.z + o.z), (float)c.w);
  }
  xyzq_s[s] = out;
}

// (5) cluster bounding boxes, one warp per cluster
__global__ void bbox_kernel(const float4 *__restrict__ xyzq_s, const int *__restrict__ perm,
                            const float4 *__restrict__ cl_origin,
                            float4 *__restrict__ bb_c, float4 *__restrict__ bb_h,
                            const int *__restrict__ counts) {
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (w >= counts[0] / kTile) return;
  int s = w * kTile + lane;
  float4 p = xyzq_s[s];
  bool valid = perm[s] >= 0;
  float mnx = valid ? p.x : INFINITY, mny = valid ? p.y : INFINITY,
        mnz = valid ? p.z : INFINITY;
  float mxx = valid ? p.x : -INFINITY, mxy = valid ? p.y : -INFINITY,
        mxz = valid ? p.z : -INFINITY;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
    mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
    mnz = fminf(mnz, __shfl_xor_sync(0xffffffffu, mnz, o));
    mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
    mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
    mxz = fmaxf(mxz, __shfl_xor_sync(0xffffffffu, mxz, o));
  }
  if (lane == 0) {
    const float4 o = cl_origin[w];
    bb_c[w] = make_float4(0.5f * (mnx + mxx) + o.x, 0.5f * (mny + mxy) + o.y,
                          0.5f * (mnz + mxz) + o.z, 0.f);
    bb_h[w] = make_float4(0.5f * (mxx - mnx), 0.5f * (mxy - mny), 0.5f * (mxz - mnz), 0.f);
  }
}

// (6) tile search.  One warp per i-cluster; lanes test (j-cluster, z-image)
// candidates of every column within reach, and a ballot compacts the hits in
// candidate order, so the list is deterministic.  With FILL the tiles, their
// exclusion masks and the work items are written at the offsets of the scan.
template <bool FILL>
__global__ void tiles_kernel(const NbSysDims *__restrict__ sysd, const int *__restrict__ cl_sys,
                             int tiles_per_work, const int *__restrict__ cl_col,
                             const int *__restrict__ col_start,
                             const float4 *__restrict__ bb_c, const float4 *__restrict__ bb_h,
                             const int *__restrict__ perm, const int *__restrict__ glo2loc,
                             const int *__restrict__ excl_ptr, const int *__restrict__ excl_idx,
                             int *__restrict__ tile_count, const int *__restrict__ tile_start,
                             const int *__restrict__ work_start, int2 *__restrict__ tiles,
                             unsigned *__restrict__ masks, int4 *__restrict__ work,
                             int *__restrict__ counts, int mask_cap,
                             unsigned *__restrict__ err) {
  const int ic = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (ic >= counts[0] / kTile) return;
  if (FILL && counts[1] == 0) return;  // overflow: nothing to write
  const int sys = cl_sys[ic];
  const NbSysDims d = sysd[sys];
  const int c = cl_col[ic] - d.col_off;
  const int cx = c % d.ncx, cy = c / d.ncx;
  const float4 ci = bb_c[ic], hi = bb_h[ic];
  const float cwx = d.Lx / d.ncx, cwy = d.Ly / d.ncy;
  const int Rx = (int)ceilf(d.rlist / cwx), Ry = (int)ceilf(d.rlist / cwy);
  const float rl2 = d.rlist * d.rlist;
  int gi = 0;
  int nexcl_begin = 0, nexcl_end = 0;
  // the slots of this lane's first kExclSlots exclusion partners, loaded once
  // for all tiles (the rest, if any, are read again for every tile)
  constexpr int kExclSlots = 16;
  int ex_slot[kExclSlots];
#pragma unroll
  for (int q = 0; q < kExclSlots; ++q) ex_slot[q] = -1;
  if (FILL) {
    gi = perm[ic * kTile + lane];
    if (gi >= 0) {
      nexcl_begin = excl_ptr[gi];
      nexcl_end = excl_ptr[gi + 1];
    }
    int eidx[kExclSlots];
#pragma unroll
    for (int q = 0; q < kExclSlots; ++q)
      eidx[q] = nexcl_begin + q < nexcl_end ? excl_idx[nexcl_begin + q] : -1;
#pragma unroll
    for (int q = 0; q < kExclSlots; ++q)
      if (eidx[q] >= 0) ex_slot[q] = glo2loc[eidx[q]];
  }
  int count = 0;
  const int base_tile = FILL ? tile_start[ic] : 0;
  // the cluster ranges of the columns in reach, loaded at once by the lanes
  // (column q of the (2 Rx + 1) x (2 Ry + 1) window by lane q mod 32) and
  // handed out by shuffles in the loop below; wider windows read them there
  const int wxn = 2 * Rx + 1, ncols = wxn * (2 * Ry + 1);
  const bool pre = ncols <= 64;
  int pre_js[2] = {0, 0}, pre_je[2] = {0, 0};
  if (pre) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int q = lane + 32 * h;
      if (q < ncols) {
        const int yy = cy + q / wxn - Ry, xx = cx + q % wxn - Rx;
        const int iy = floor_div(yy, d.ncy), ix = floor_div(xx, d.ncx);
        if (iy >= -1 && iy <= 1 && ix >= -1 && ix <= 1) {
          const int col = d.col_off + (xx - ix * d.ncx) + d.ncx * (yy - iy * d.ncy);
          pre_js[h] = col_start[col] / kTile;
          pre_je[h] = col_start[col + 1] / kTile;
        }
      }
    }
  }
  for (int dy = -Ry; dy <= Ry; ++dy) {
    int yy = cy + dy;
    int iy = floor_div(yy, d.ncy);
    if (iy < -1 || iy > 1) continue;
    int wy = yy - iy * d.ncy;
    for (int dx = -Rx; dx <= Rx; ++dx) {
      int xx = cx + dx;
      int ix = floor_div(xx, d.ncx);
      if (ix < -1 || ix > 1) continue;
      int wx = xx - ix * d.ncx;
      int col = d.col_off + wx + d.ncx * wy;
      int js, je;
      if (pre) {
        const int q = (dy + Ry) * wxn + (dx + Rx);
        js = __shfl_sync(0xffffffffu, q < 32 ? pre_js[0] : pre_js[1], q & 31);
        je = __shfl_sync(0xffffffffu, q < 32 ? pre_je[0] : pre_je[1], q & 31);
      } else {
        js = col_start[col] / kTile;
        je = col_start[col + 1] / kTile;
      }
      int ncand = (je - js) * 3;
      for (int b0 = 0; b0 < ncand; b0 += 32) {
        int cand = b0 + lane;
        bool ok = false;
        int jc = 0, sc = 13;
        if (cand < ncand) {
          jc = js + cand / 3;
          int iz = cand % 3 - 1;
          sc = (ix + 1) + 3 * (iy + 1) + 9 * (iz + 1);
          if (jc > ic || (jc == ic && sc >= 13)) {
            float4 cj = bb_c[jc], hj = bb_h[jc];
            float ddx = fmaxf(0.f, fabsf(ci.x - cj.x - ix * d.Lx) - hi.x - hj.x);
            float ddy = fmaxf(0.f, fabsf(ci.y - cj.y - iy * d.Ly) - hi.y - hj.y);
            float ddz = fmaxf(0.f, fabsf(ci.z - cj.z - iz * d.Lz) - hi.z - hj.z);
            ok = ddx * ddx + ddy * ddy + ddz * ddz < rl2;
          }
        }
        unsigned hits = __ballot_sync(0xffffffffu, ok);
        if (FILL) {
          while (hits) {
            int src = __ffs(hits) - 1;
            hits &= hits - 1;
            int tjc = __shfl_sync(0xffffffffu, jc, src);
            int tsc = __shfl_sync(0xffffffffu, sc, src);
            int t = base_tile + count;
            ++count;
            // topological exclusions of i-lane `lane` against this j-cluster
            unsigned word = 0u;
#pragma unroll
            for (int q = 0; q < kExclSlots; ++q)
              if (ex_slot[q] >= 0 && (ex_slot[q] >> 5) == tjc) word |= 1u << (ex_slot[q] & 31);
            for (int e = nexcl_begin + kExclSlots; e < nexcl_end; ++e) {
              int lp = glo2loc[excl_idx[e]];
              if ((lp >> 5) == tjc) word |= 1u << (lp & 31);
            }
            int midx = -1;
            if (__any_sync(0xffffffffu, word != 0u)) {
              if (lane == 0) midx = atomicAdd(&counts[5], 1);
              midx = __shfl_sync(0xffffffffu, midx, 0);
              if (midx < mask_cap) {
                masks[(size_t)midx * kTile + lane] = word;
              } else {  // more masked tiles than allocated: the build is void
                if (lane == 0) atomicOr(err, (unsigned)kErrTileOverflow);
                midx = -1;
              }
            }
            if (lane == 0) tiles[t] = make_int2(tjc, tsc | ((midx + 1) << 5));
          }
        } else {
          count += __popc(hits);
        }
      }
    }
  }
  if (!FILL) {
    if (lane == 0) tile_count[ic] = count;
  } else if (lane == 0) {
    int w0 = work_start[ic];
    int tpw = tiles_per_work;
    for (int k = 0; k * tpw < count; ++k)
      work[w0 + k] = make_int4(ic, base_tile + k * tpw, base_tile + min(count, (k + 1) * tpw), sys);
  }
}

// (7) offsets of tiles and work items per i-cluster
__global__ void tile_scan_kernel(const int *__restrict__ tile_count, int *__restrict__ tile_start,
                                 int *__restrict__ work_start, int *__restrict__ counts,
                                 int tile_cap, int work_cap, int tpw, unsigned *__restrict__ err) {
  __shared__ int sh[kScanThreads];
  int ncl = counts[0] / kTile;
  int carry_t = 0, carry_w = 0;
  for (int base = 0; base < ncl; base += kScanThreads) {
    int c = base + threadIdx.x;
    int nt = c < ncl ? tile_count[c] : 0;
    int nw = (nt + tpw - 1) / tpw;
    int tot;
    int ex = block_exclusive_scan(nt, sh, tot);
    if (c < ncl) tile_start[c] = carry_t + ex;
    carry_t += tot;
    ex = block_exclusive_scan(nw, sh, tot);
    if (c < ncl) work_start[c] = carry_w + ex;
    carry_w += tot;
  }
  if (threadIdx.x == 0) {
    if (carry_t > tile_cap || carry_w > work_cap) {
      atomicOr(err, (unsigned)(carry_t > tile_cap ? kErrTileOverflow : kErrWorkOverflow));
      // record the demand so the host can grow the buffers, but publish empty
      // lists so nothing is written out of bounds
      counts[3] = carry_t;
      counts[4] = carry_w;
      carry_t = carry_w = 0;
    } else {
      counts[3] = carry_t;
      counts[4] = carry_w;
    }
    counts[1] = carry_t;
    counts[2] = carry_w;
    counts[5] = 0;  // masked tiles, counted by the fill pass
  }
}

template <typename T>
void dalloc(T *&p, size_t n) {
  if (p) APO_CUDA(cudaFree(p));
  p = nullptr;
  if (n) APO_CUDA(cudaMalloc(&p, n * sizeof(T)));
}
template <typename T>
void dfree(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

}  // namespace

NeighborList::~NeighborList() { release(); }

void NeighborList::release() {
  dfree(perm); dfree(glo2loc); dfree(slot_shift); dfree(xyzq_s); dfree(type_s);
  dfree(slot_off); dfree(cl_origin); dfree(cl_sys); dfree(sys_of_atom);
  dfree(tiles); dfree(masks); dfree(work); dfree(counts); dfree(error);
  dfree(m_excl_ptr); dfree(m_excl_idx); dfree(m_col_count); dfree(m_col_start);
  dfree(m_atom_col); dfree(m_atom_rank); dfree(m_atom_shift); dfree(m_atom_z); dfree(m_tmp_key);
  dfree(m_tmp_idx); dfree(m_cl_col); dfree(m_bb_c); dfree(m_bb_h);
  dfree(m_tile_count); dfree(m_tile_start); dfree(m_work_start);
  dfree(m_sys); dfree(m_col_sys);
}

void NeighborList::setup(int natom, double Lx, double Ly, double Lz, float rlist,
                         const std::vector<int> &excl_ptr, const std::vector<int> &excl_idx,
                         const int *d_vdwtype, int tiles_per_work) {
  setup(std::vector<NbListSystem>{NbListSystem{natom, Lx, Ly, Lz, rlist}}, excl_ptr, excl_idx,
        d_vdwtype, tiles_per_work);
}

void NeighborList::setup(const std::vector<NbListSystem> &systems,
                         const std::vector<int> &excl_ptr, const std::vector<int> &excl_idx,
                         const int *d_vdwtype, int tiles_per_work) {
  if (systems.empty()) throw std::invalid_argument("NeighborList: no systems");
  {
    static bool attr = false;
    if (!attr) {
      APO_CUDA(cudaFuncSetAttribute(col_sort_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
      attr = true;
    }
  }
  release();
  m_sys_h.clear();
  m_d = NbListDims{};
  m_d.nsys = (int)systems.size();
  m_d.tiles_per_work = std::max(1, tiles_per_work);
  m_d.sort_cap = 1024;
  long long slots = 0;
  double tiles = 0.0;
  int natom = 0, ncol = 0;
  std::vector<int> col_sys, atom_sys;
  for (size_t k = 0; k < systems.size(); ++k) {
    const NbListSystem &y = systems[k];
    if (y.natom <= 0) throw std::invalid_argument("NeighborList: a system has no atoms");
    if (!(y.Lx > 0.0 && y.Ly > 0.0 && y.Lz > 0.0) || y.Lx > 65536.0 || y.Ly > 65536.0 ||
        y.Lz > 65536.0)
      throw std::invalid_argument("NeighborList: box lengths must be in (0, 65536] A");
    NbSysDims d;
    d.Lx = (float)y.Lx;
    d.Ly = (float)y.Ly;
    d.Lz = (float)y.Lz;
    d.Lxd = y.Lx;
    d.Lyd = y.Ly;
    d.Lzd = y.Lz;
    d.rlist = y.rlist;
    d.atom_off = natom;
    d.natom = y.natom;
    // columns whose cross-section holds ~32 atoms per z-slab of equal height:
    // clusters come out close to cubic
    const double rho = y.natom / (y.Lx * y.Ly * y.Lz);
    const double edge = std::cbrt(32.0 / rho);
    d.ncx = std::max(1, (int)std::floor(y.Lx / edge));
    d.ncy = std::max(1, (int)std::floor(y.Ly / edge));
    d.col_off = ncol;
    const int nc = d.ncx * d.ncy;
    const double per_col = y.natom / (double)nc;
    while (m_d.sort_cap < 1.6 * per_col + 64) m_d.sort_cap *= 2;
    slots += y.natom + (long long)kTile * nc;
    // tile estimate: clusters within rlist + two cluster edges, half list
    const double reach = y.rlist + 2.0 * edge;
    const double ncl_s = (y.natom + (double)kTile * nc) / kTile;
    tiles += ncl_s * (rho * 4.18879 * reach * reach * reach / 32.0 * 0.5 + 16.0);
    for (int c = 0; c < nc; ++c) col_sys.push_back((int)k);
    for (int a = 0; a < y.natom; ++a) atom_sys.push_back((int)k);
    ncol += nc;
    natom += y.natom;
    m_sys_h.push_back(d);
  }
  if ((size_t)m_d.sort_cap * (sizeof(float) + 2 * sizeof(int)) > 96 * 1024)
    throw std::invalid_argument("NeighborList: a cell column would hold more atoms than the "
                                "column sort supports (box too elongated for its density)");
  m_d.natom = natom;
  m_d.ncol = ncol;
  m_d.slot_cap = (int)((slots + kTile - 1) / kTile * kTile);
  const int ncl = m_d.slot_cap / kTile;
  m_d.tile_cap = (int)std::min<double>(tiles, 2.0e9 / 128.0);
  m_d.work_cap = m_d.tile_cap / m_d.tiles_per_work + ncl + 16;
  // masked tiles: a cluster's tile with itself and with its neighbours along
  // the column usually hold its molecules' exclusions
  m_d.mask_cap = 4 * ncl + 1024;
  if ((int)excl_ptr.size() != natom + 1)
    throw std::invalid_argument("NeighborList: exclusion pointer array must have natom + 1 entries");
  m_vdwtype = d_vdwtype;
  alloc();
  dalloc(m_sys, m_sys_h.size());
  APO_CUDA(cudaMemcpy(m_sys, m_sys_h.data(), m_sys_h.size() * sizeof(NbSysDims),
                      cudaMemcpyHostToDevice));
  dalloc(m_col_sys, col_sys.size());
  APO_CUDA(cudaMemcpy(m_col_sys, col_sys.data(), col_sys.size() * sizeof(int),
                      cudaMemcpyHostToDevice));
  APO_CUDA(cudaMemcpy(sys_of_atom, atom_sys.data(), atom_sys.size() * sizeof(int),
                      cudaMemcpyHostToDevice));
  dalloc(m_excl_ptr, excl_ptr.size());
  dalloc(m_excl_idx, std::max<size_t>(1, excl_idx.size()));
  APO_CUDA(cudaMemcpy(m_excl_ptr, excl_ptr.data(), excl_ptr.size() * sizeof(int),
                      cudaMemcpyHostToDevice));
  if (!excl_idx.empty())
    APO_CUDA(cudaMemcpy(m_excl_idx, excl_idx.data(), excl_idx.size() * sizeof(int),
                        cudaMemcpyHostToDevice));
}

void NeighborList::set_tiles_per_work(int tpw) {
  tpw = std::max(1, tpw);
  if (tpw == m_d.tiles_per_work) return;
  const int ncl = m_d.slot_cap / kTile;
  m_d.tiles_per_work = tpw;
  const int need = m_d.tile_cap / tpw + ncl + 16;
  if (need > m_d.work_cap) {
    m_d.work_cap = need;
    dalloc(work, m_d.work_cap);
  }
}

void NeighborList::alloc() {
  const int n = m_d.natom, S = m_d.slot_cap, ncl = S / kTile;
  dalloc(perm, S); dalloc(glo2loc, n); dalloc(slot_shift, S); dalloc(xyzq_s, S);
  dalloc(slot_off, S); dalloc(cl_origin, ncl); dalloc(cl_sys, ncl); dalloc(sys_of_atom, n);
  APO_CUDA(cudaMemset(slot_off, 0, (size_t)S * sizeof(double4)));
  APO_CUDA(cudaMemset(cl_origin, 0, (size_t)ncl * sizeof(float4)));
  APO_CUDA(cudaMemset(cl_sys, 0, (size_t)ncl * sizeof(int)));
  dalloc(type_s, S); dalloc(tiles, m_d.tile_cap); dalloc(masks, (size_t)m_d.mask_cap * kTile);
  dalloc(work, m_d.work_cap); dalloc(counts, 8); dalloc(error, 1);
  dalloc(m_col_count, m_d.ncol); dalloc(m_col_start, m_d.ncol + 1); dalloc(m_atom_col, n);
  dalloc(m_atom_rank, n); dalloc(m_atom_shift, n); dalloc(m_atom_z, n);
  dalloc(m_tmp_key, S); dalloc(m_tmp_idx, S);
  dalloc(m_cl_col, ncl); dalloc(m_bb_c, ncl); dalloc(m_bb_h, ncl);
  dalloc(m_tile_count, ncl); dalloc(m_tile_start, ncl); dalloc(m_work_start, ncl);
  APO_CUDA(cudaMemset(counts, 0, 8 * sizeof(int)));
  APO_CUDA(cudaMemset(error, 0, sizeof(unsigned)));
  APO_CUDA(cudaMemset(xyzq_s, 0, (size_t)S * sizeof(float4)));
  APO_CUDA(cudaMemset(perm, 0xff, (size_t)S * sizeof(int)));
  APO_CUDA(cudaMemset(type_s, 0, (size_t)S * sizeof(int)));
}

void NeighborList::build(const float4 *d_xyzq, cudaStream_t s) {
  const int n = m_d.natom;
  const int S = m_d.slot_cap;
  const int ncl = S / kTile;
  APO_CUDA(cudaMemsetAsync(m_col_count, 0, m_d.ncol * sizeof(int), s));
  bin_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, d_xyzq, sys_of_atom, m_sys, m_col_count,
                                              m_atom_col, m_atom_rank, m_atom_shift, m_atom_z,
                                              error);
  APO_LAUNCH_CHECK();
  col_scan_kernel<<<1, kScanThreads, 0, s>>>(m_d.ncol, m_col_count, m_col_start, counts, S,
                                             m_d.sort_cap, error);
  APO_LAUNCH_CHECK();
  scatter_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, m_atom_col, m_atom_rank, m_col_start,
                                                  m_atom_z, m_tmp_key, m_tmp_idx, counts);
  APO_LAUNCH_CHECK();
  size_t sm = (size_t)m_d.sort_cap * (sizeof(float) + 2 * sizeof(int));
  col_sort_kernel<<<m_d.ncol, 512, sm, s>>>(m_d.ncol, m_col_count, m_col_start, m_tmp_key,
                                            m_tmp_idx, m_atom_shift, m_vdwtype, perm, glo2loc,
                                            slot_shift, type_s, m_cl_col, m_col_sys, cl_sys,
                                            counts, m_d.sort_cap, d_xyzq);
  APO_LAUNCH_CHECK();
  origin_kernel<<<(ncl * 32 + 255) / 256, 256, 0, s>>>(d_xyzq, perm, slot_shift, m_sys, cl_sys,
                                                        cl_origin, slot_off, counts);
  APO_LAUNCH_CHECK();
  refresh(s);
  bbox_kernel<<<(ncl * 32 + 255) / 256, 256, 0, s>>>(xyzq_s, perm, cl_origin, m_bb_c, m_bb_h,
                                                      counts);
  APO_LAUNCH_CHECK();
  tiles_kernel<false><<<(ncl * 32 + 127) / 128, 128, 0, s>>>(
      m_sys, cl_sys, m_d.tiles_per_work, m_cl_col, m_col_start, m_bb_c, m_bb_h, perm, glo2loc,
      m_excl_ptr, m_excl_idx, m_tile_count, m_tile_start, m_work_start, tiles, masks, work,
      counts, m_d.mask_cap, error);
  APO_LAUNCH_CHECK();
  tile_scan_kernel<<<1, kScanThreads, 0, s>>>(m_tile_count, m_tile_start, m_work_start,
                                              counts, m_d.tile_cap, m_d.work_cap,
                                              m_d.tiles_per_work, error);
  APO_LAUNCH_CHECK();
  tiles_kernel<true><<<(ncl * 32 + 127) / 128, 128, 0, s>>>(
      m_sys, cl_sys, m_d.tiles_per_work, m_cl_col, m_col_start, m_bb_c, m_bb_h, perm, glo2loc,
      m_excl_ptr, m_excl_idx, m_tile_count, m_tile_start, m_work_start, tiles, masks, work,
      counts, m_d.mask_cap, error);
  APO_LAUNCH_CHECK();
}

void NeighborList::refresh(cudaStream_t s) {
  if (!m_coords) throw std::runtime_error("NeighborList: no state coordinates attached");
  refresh_kernel<<<(m_d.slot_cap + 255) / 256, 256, 0, s>>>(m_coords, perm, slot_off, xyzq_s,
                                                             counts);
  APO_LAUNCH_CHECK();
}

void NeighborList::set_box(int sys, double Lx, double Ly, double Lz) {
  if (sys < 0 || sys >= (int)m_sys_h.size()) throw std::invalid_argument("NeighborList: no such system");
  if (!(Lx > 0.0 && Ly > 0.0 && Lz > 0.0) || Lx > 65536.0 || Ly > 65536.0 || Lz > 65536.0)
    throw std::invalid_argument("NeighborList: box lengths must be in (0, 65536] A");
  NbSysDims &d = m_sys_h[sys];
  d.Lx = (float)Lx;
  d.Ly = (float)Ly;
  d.Lz = (float)Lz;
  d.Lxd = Lx;
  d.Lyd = Ly;
  d.Lzd = Lz;
  APO_CUDA(cudaMemcpy(m_sys + sys, &d, sizeof(NbSysDims), cudaMemcpyHostToDevice));
}

void NeighborList::rescale_box_device(const double *old_box, const double *new_box,
                                      const unsigned *err, cudaStream_t s) {
  if (m_sys_h.size() != 1) throw std::invalid_argument("NeighborList: one system only");
  rescale_dev_kernel<<<(m_d.slot_cap + 255) / 256, 256, 0, s>>>(slot_off, cl_origin, old_box,
                                                                new_box, err, counts);
  APO_LAUNCH_CHECK();
}

void NeighborList::set_box_host(int sys, double Lx, double Ly, double Lz) {
  if (sys < 0 || sys >= (int)m_sys_h.size()) throw std::invalid_argument("NeighborList: no such system");
  NbSysDims &d = m_sys_h[sys];
  d.Lx = (float)Lx;
  d.Ly = (float)Ly;
  d.Lz = (float)Lz;
  d.Lxd = Lx;
  d.Lyd = Ly;
  d.Lzd = Lz;
}

void NeighborList::set_capacity(int tile_cap, int work_cap) {
  if (tile_cap < 1 || work_cap < 1) throw std::invalid_argument("NeighborList: capacities must be positive");
  m_d.tile_cap = tile_cap;
  m_d.work_cap = work_cap;
  dalloc(tiles, m_d.tile_cap);
  dalloc(work, m_d.work_cap);
}

void NeighborList::clear_error(cudaStream_t s) {
  APO_CUDA(cudaMemsetAsync(error, 0, sizeof(unsigned), s));
}

void NeighborList::sync_counts(cudaStream_t s) {
  int c[8];
  APO_CUDA(cudaMemcpyAsync(c, counts, sizeof(c), cudaMemcpyDeviceToHost, s));
  APO_CUDA(cudaStreamSynchronize(s));
  h_counts[0] = c[0];
  h_counts[1] = c[1];
  h_counts[2] = c[2];
}

unsigned NeighborList::read_error(cudaStream_t s) {
  unsigned e = 0;
  APO_CUDA(cudaMemcpyAsync(&e, error, sizeof(e), cudaMemcpyDeviceToHost, s));
  APO_CUDA(cudaStreamSynchronize(s));
  return e;
}

bool NeighborList::ensure_capacity(const float4 *d_xyzq, cudaStream_t s, double fill) {
  build(d_xyzq, s);
  int c[8];
  APO_CUDA(cudaMemcpyAsync(c, counts, sizeof(c), cudaMemcpyDeviceToHost, s));
  APO_CUDA(cudaStreamSynchronize(s));
  unsigned e = read_error(s);
  if (e & (kErrColumnOverflow | kErrNaN))
    throw std::runtime_error("neighbour list: column overflow or non-finite coordinates");
  bool grew = false;
  const bool tiles_short = c[3] > fill * m_d.tile_cap || c[4] > fill * m_d.work_cap;
  const bool masks_short = c[5] > fill * m_d.mask_cap;
  if (tiles_short || masks_short) {
    if (tiles_short) {
      m_d.tile_cap = (int)(std::max<double>(c[3], 1) / fill * 1.25) + 1024;
      m_d.work_cap = (int)(std::max<double>(c[4], 1) / fill * 1.25) + 1024;
      dalloc(tiles, m_d.tile_cap);
      dalloc(work, m_d.work_cap);
    }
    if (masks_short) {
      m_d.mask_cap = (int)(std::max<double>(c[5], 1) / fill * 1.25) + 1024;
      dalloc(masks, (size_t)m_d.mask_cap * kTile);
    }
    APO_CUDA(cudaMemsetAsync(error, 0, sizeof(unsigned), s));
    build(d_xyzq, s);
    APO_CUDA(cudaStreamSynchronize(s));
    grew = true;
  }
  sync_counts(s);
  return grew;
}

}  // namespace apo
