// PME reciprocal-space kernels; see pme.h.
#include "pme.h"

#include <cuda.h>  // CUtensorMap (the encoder is fetched through the runtime)

#include <algorithm>
#include <atomic>
#include <cmath>
#include <functional>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <vector>

#include "common.h"
#include "device_util.cuh"

namespace apo {
namespace {

constexpr int kPlaneThreads = 512;
// dynamic shared memory a plane transform may use: the SM's 227 KB per
// block less the kernels' static digit-reversal table
constexpr size_t kPlaneSmemMax = 227 * 1024 - 1024;
// the tensor-map argument of launches that move their slabs with plain loads
const CUtensorMap kNoTensorMap{};
constexpr int kPencilThreads = 256;
constexpr int kPencilTX = 16;

// ------------------------------------------------------------------------
// B-spline weights (Essmann et al. recursion, the reference's calc_one_theta,
// src/CudaPMERecip.cu:438-470)
// ------------------------------------------------------------------------
template <int ORDER>
__device__ __forceinline__ void bspline(float w, float (&th)[ORDER], float (&dth)[ORDER]) {
  th[ORDER - 1] = 0.f;
  th[1] = w;
  th[0] = 1.f - w;
#pragma unroll
  for (int k = 3; k <= ORDER - 1; ++k) {
    const float div = 1.f / (float)(k - 1);
    th[k - 1] = div * w * th[k - 2];
#pragma unroll
    for (int j = 1; j <= k - 2; ++j)
      th[k - j - 1] = div * ((w + j) * th[k - j - 2] + (k - j - w) * th[k - j - 1]);
    th[0] = div * (1.f - w) * th[0];
  }
  dth[0] = -th[0];
#pragma unroll
  for (int j = 1; j < ORDER; ++j) dth[j] = th[j - 1] - th[j];
  const float div = 1.f / (float)(ORDER - 1);
  th[ORDER - 1] = div * w * th[ORDER - 2];
#pragma unroll
  for (int j = 1; j <= ORDER - 2; ++j)
    th[ORDER - j - 1] =
        div * ((w + j) * th[ORDER - j - 2] + (ORDER - j - w) * th[ORDER - j - 1]);
  th[0] = div * (1.f - w) * th[0];
}

// grid anchoring of the reference (include/cuda_pme_spread.h:64-81):
// w = x/L + 2, fr = n (w - (floor(w+0.5) - 0.5)), points floor(fr)+0..p-1.
// Evaluated in FP64 from the exact global position (cluster origin + local
// offset): in FP32 the rounding of w near 2 (1.2e-7) times n shifts the
// B-spline fraction by up to n * 1.2e-7 grid units, which at a 216-point
// axis is the largest error of the reciprocal force.  The fraction itself
// is returned in FP32 for the spline recursion.
__device__ __forceinline__ void anchor(double x, double recip, int n, int &i0, float &w) {
  const double t = x * recip + 2.0;
  const double fr = (double)n * (t - (floor(t + 0.5) - 0.5));
  // non-finite or exploded coordinates must not index outside the grid
  if (!(fr >= 0.0 && fr < (double)n)) {
    i0 = fr >= (double)n ? n - 1 : 0;
    w = 0.f;
    return;
  }
  i0 = (int)fr;
  w = (float)(fr - (double)i0);
  if (i0 > n - 1) i0 = n - 1;
}

// global position of a sorted slot: the cluster origin (a multiple of
// 1/64 A, exact in FP32) plus the local offset, summed without rounding
__device__ __forceinline__ double3 global_pos(const float4 &p, const float4 *origin, int s) {
  if (!origin) return make_double3(p.x, p.y, p.z);
  const float4 o = origin[s >> 5];
  return make_double3((double)o.x + (double)p.x, (double)o.y + (double)p.y,
                      (double)o.z + (double)p.z);
}

// ------------------------------------------------------------------------
// small DFTs
// ------------------------------------------------------------------------
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// cos / sin of 2*pi*k/R for the radices used (exact mathematical constants)
__device__ __forceinline__ constexpr float rcos(int R, int k) {
  return R == 3 ? (k == 0 ? 1.f : -0.5f)
       : R == 5 ? (k == 0 ? 1.f : (k == 1 || k == 4) ? 0.30901699437494745f : -0.8090169943749475f)
       : R == 6 ? (k == 0 ? 1.f : (k == 1 || k == 5) ? 0.5f : (k == 2 || k == 4) ? -0.5f : -1.f)
       : R == 7 ? (k == 0 ? 1.f : (k == 1 || k == 6) ? 0.6234898018587336f
                              : (k == 2 || k == 5) ? -0.22252093395631434f : -0.9009688679024191f)
       : R == 8 ? (k == 0 ? 1.f : (k == 1 || k == 7) ? 0.7071067811865476f
                              : (k == 2 || k == 6) ? 0.f : (k == 3 || k == 5) ? -0.7071067811865476f : -1.f)
       : 1.f;
}
__device__ __forceinline__ constexpr float rsin(int R, int k) {
  return R == 3 ? (k == 0 ? 0.f : k == 1 ? 0.8660254037844386f : -0.8660254037844386f)
       : R == 5 ? (k == 0 ? 0.f : k == 1 ? 0.9510565162951535f : k == 2 ? 0.5877852522924731f
                  : k == 3 ? -0.5877852522924731f : -0.9510565162951535f)
       : R == 6 ? (k == 0 || k == 3 ? 0.f : (k == 1 || k == 2) ? 0.8660254037844386f : -0.8660254037844386f)
       : R == 7 ? (k == 0 ? 0.f : k == 1 ? 0.7818314824680298f : k == 2 ? 0.9749279121818236f
                  : k == 3 ? 0.4338837391175582f : k == 4 ? -0.4338837391175582f
                  : k == 5 ? -0.9749279121818236f : -0.7818314824680298f)
       : R == 8 ? (k == 0 || k == 4 ? 0.f : (k == 1 || k == 3) ? 0.7071067811865476f
                  : k == 2 ? 1.f : (k == 5 || k == 7) ? -0.7071067811865476f : -1.f)
       : 0.f;
}

// y_k = sum_q x_q exp(sign * 2 pi i q k / R)
template <int R>
__device__ __forceinline__ void dft(float2 (&x)[R], float sign) {
  if (R == 2) {
    float2 a = x[0], b = x[1];
    x[0] = make_float2(a.x + b.x, a.y + b.y);
    x[1] = make_float2(a.x - b.x, a.y - b.y);
  } else if (R == 4) {
    float2 s02 = make_float2(x[0].x + x[2].x, x[0].y + x[2].y);
    float2 d02 = make_float2(x[0].x - x[2].x, x[0].y - x[2].y);
    float2 s13 = make_float2(x[1].x + x[3].x, x[1].y + x[3].y);
    float2 d13 = make_float2(x[1].x - x[3].x, x[1].y - x[3].y);
    // sign * i * d13
    float2 id13 = make_float2(-sign * d13.y, sign * d13.x);
    x[0] = make_float2(s02.x + s13.x, s02.y + s13.y);
    x[2] = make_float2(s02.x - s13.x, s02.y - s13.y);
    x[1] = make_float2(d02.x + id13.x, d02.y + id13.y);
    x[3] = make_float2(d02.x - id13.x, d02.y - id13.y);
  } else {
    float2 y[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      float re = 0.f, im = 0.f;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int idx = (q * k) % R;
        const float c = rcos(R, idx), s = sign * rsin(R, idx);
        re += x[q].x * c - x[q].y * s;
        im += x[q].x * s + x[q].y * c;
      }
      y[k] = make_float2(re, im);
    }
#pragma unroll
    for (int k = 0; k < R; ++k) x[k] = y[k];
  }
}

__device__ __forceinline__ float2 twiddle(const float2 *tw, int idx, float sign) {
  float2 w = tw[idx];
  if (sign > 0.f) w.y = -w.y;
  return w;
}

// One decimation-in-frequency stage (butterfly, then twiddle) on sub-blocks
// of length m of every line.  Lines start at buf + line*lstride; element e of
// a line is at e*estride.  The twiddle index j k n/m stays below n.
template <int R>
__device__ void dif_stage(float2 *buf, int nlines, int lstride, int estride, int n, int m,
                          FastDiv fpl, FastDiv fmr, const float2 *tw, float sign) {
  const int mr = m / R, per_line = n / R, total = nlines * per_line, nm = n / m;
  for (int b = threadIdx.x; b < total; b += blockDim.x) {
    const int line = (int)fdiv((unsigned)b, fpl), rem = b - line * per_line;
    const int blk = (int)fdiv((unsigned)rem, fmr), j = rem - blk * mr;
    float2 *p = buf + line * lstride + (blk * m + j) * estride;
    float2 x[R];
#pragma unroll
    for (int q = 0; q < R; ++q) x[q] = p[q * mr * estride];
    dft<R>(x, sign);
    if (j > 0) {
#pragma unroll
      for (int k = 1; k < R; ++k) x[k] = cmul(x[k], twiddle(tw, j * k * nm, sign));
    }
#pragma unroll
    for (int k = 0; k < R; ++k) p[k * mr * estride] = x[k];
  }
}

// One decimation-in-time stage (twiddle, then butterfly).
template <int R>
__device__ void dit_stage(float2 *buf, int nlines, int lstride, int estride, int n, int m,
                          FastDiv fpl, FastDiv fmr, const float2 *tw, float sign) {
  const int mr = m / R, per_line = n / R, total = nlines * per_line, nm = n / m;
  for (int b = threadIdx.x; b < total; b += blockDim.x) {
    const int line = (int)fdiv((unsigned)b, fpl), rem = b - line * per_line;
    const int blk = (int)fdiv((unsigned)rem, fmr), j = rem - blk * mr;
    float2 *p = buf + line * lstride + (blk * m + j) * estride;
    float2 x[R];
#pragma unroll
    for (int k = 0; k < R; ++k) x[k] = p[k * mr * estride];
    if (j > 0) {
#pragma unroll
      for (int k = 1; k < R; ++k) x[k] = cmul(x[k], twiddle(tw, j * k * nm, sign));
    }
    dft<R>(x, sign);
#pragma unroll
    for (int q = 0; q < R; ++q) p[q * mr * estride] = x[q];
  }
}

template <bool DIF>
__device__ __forceinline__ void stage(int R, float2 *buf, int nl, int ls, int es, int n, int m,
                                      FastDiv fpl, FastDiv fmr, const float2 *tw, float sign) {
  switch (R) {
    case 2: DIF ? dif_stage<2>(buf, nl, ls, es, n, m, fpl, fmr, tw, sign) : dit_stage<2>(buf, nl, ls, es, n, m, fpl, fmr, tw, sign); break;
    case 3: DIF ? dif_stage<3>(buf, nl, ls, es, n, m, fpl, fmr, tw, sign) : dit_stage<3>(buf, nl, ls, es, n, m, fpl, fmr, tw, sign); break;
    case 4: DIF ? dif_stage<4>(buf, nl, ls, es, n, m, fpl, fmr, tw, sign) : dit_stage<4>(buf, nl, ls, es, n, m, fpl, fmr, tw, sign); break;
    case 5: DIF ? dif_stage<5>(buf, nl, ls, es, n, m, fpl, fmr, tw, sign) : dit_stage<5>(buf, nl, ls, es, n, m, fpl, fmr, tw, sign); break;
    case 6: DIF ? dif_stage<6>(buf, nl, ls, es, n, m, fpl, fmr, tw, sign) : dit_stage<6>(buf, nl, ls, es, n, m, fpl, fmr, tw, sign); break;
    case 7: DIF ? dif_stage<7>(buf, nl, ls, es, n, m, fpl, fmr, tw, sign) : dit_stage<7>(buf, nl, ls, es, n, m, fpl, fmr, tw, sign); break;
    case 8: DIF ? dif_stage<8>(buf, nl, ls, es, n, m, fpl, fmr, tw, sign) : dit_stage<8>(buf, nl, ls, es, n, m, fpl, fmr, tw, sign); break;
    default: break;
  }
}

// natural order in, digit-reversed out
__device__ void fft_dif(float2 *buf, int nl, int ls, int es, const FftAxis &a, const float2 *tw,
                        float sign) {
  int m = a.n;
  for (int s = 0; s < a.nrad; ++s) {
    stage<true>(a.radix[s], buf, nl, ls, es, a.n, m, a.per_line[s], a.dif_mr[s], tw, sign);
    __syncthreads();
    m /= a.radix[s];
  }
}
// digit-reversed in, natural order out
__device__ void fft_dit(float2 *buf, int nl, int ls, int es, const FftAxis &a, const float2 *tw,
                        float sign) {
  int m = 1;
  for (int s = a.nrad - 1; s >= 0; --s) {
    m *= a.radix[s];
    stage<false>(a.radix[s], buf, nl, ls, es, a.n, m, a.per_line[s], a.dit_mr[s], tw, sign);
    __syncthreads();
  }
}

// digit-reversal table of an axis (positions of fft_dif's output, or their
// inverse) in shared memory, built by the whole block
__device__ __forceinline__ void fill_rev_table(short *tab, const FftAxis &a, bool inverse);

// natural index -> position in the output of fft_dif
__device__ __forceinline__ int dig_rev(int x, const FftAxis &a) {
  int p = 0, m = a.n;
  for (int s = 0; s < a.nrad; ++s) {
    const int R = a.radix[s];
    m /= R;
    p += (x % R) * m;
    x /= R;
  }
  return p;
}
// position in the output of fft_dif -> natural index
__device__ __forceinline__ int dig_unrev(int p, const FftAxis &a) {
  int k = 0, mult = 1, m = a.n;
  for (int s = 0; s < a.nrad; ++s) {
    const int R = a.radix[s];
    m /= R;
    const int d = p / m;
    p -= d * m;
    k += d * mult;
    mult *= R;
  }
  return k;
}

__device__ __forceinline__ void fill_rev_table(short *tab, const FftAxis &a, bool inverse) {
  for (int x = threadIdx.x; x < a.n; x += blockDim.x)
    tab[x] = (short)(inverse ? dig_unrev(x, a) : dig_rev(x, a));
}

// ------------------------------------------------------------------------
// tensor-memory-access (TMA) copies of pencil slabs: one thread issues a
// tiled bulk copy between global memory and shared memory; the load's
// completion is counted on an mbarrier (transaction bytes), waited for with
// a bounded number of polls
// ------------------------------------------------------------------------
constexpr int kTmaPollLimit = 1 << 22;

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// true once the phase `parity` has completed; false after kTmaPollLimit polls
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
  for (int i = 0; i < kTmaPollLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, int x, int y, int z,
                                             const void *src) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
          reinterpret_cast<unsigned long long>(map)),
      "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
      : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// shared-memory writes of this thread become visible to the async proxy
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// the box held in device memory (a box that changes every step under
// pressure control): the same conversions as Pme::setup / set_box
__device__ __forceinline__ void box_from_device(PmeDims &d, const double4 b) {
  d.Lx = (float)b.x;
  d.Ly = (float)b.y;
  d.Lz = (float)b.z;
  d.rLx = 1.0 / b.x;
  d.rLy = 1.0 / b.y;
  d.rLz = 1.0 / b.z;
}

// ------------------------------------------------------------------------
// spread
// ------------------------------------------------------------------------
template <int ORDER>
__global__ void __launch_bounds__(128) spread_kernel(const float4 *__restrict__ xyzq,
                                                     const int *__restrict__ counts, PmeDims d,
                                                     int *__restrict__ qgrid,
                                                     const float4 *__restrict__ origin,
                                                     const PmeSysArgs *__restrict__ multi = nullptr,
                                                     const int *__restrict__ cl_sys = nullptr,
                                                     const double4 *__restrict__ dbox = nullptr) {
  if (multi) {  // one block = one 32-slot cluster of one system
    const PmeSysArgs &A = multi[cl_sys[blockIdx.x]];
    d = A.d;
    qgrid = A.qgrid;
  }
  if (dbox) box_from_device(d, *dbox);
  constexpr int P3 = ORDER * ORDER * ORDER;
  __shared__ int sh_i[3][32];
  __shared__ float sh_q[32];
  __shared__ float sh_th[3][32][ORDER];
  const int nslot = counts ? counts[0] : 0;
  const int s0 = blockIdx.x * 32;
  if (s0 >= nslot) return;
  // the splines of the 32 atoms, one thread per (dimension, atom)
  if (threadIdx.x < 96) {
    const int dim = threadIdx.x >> 5, a = threadIdx.x & 31;
    const int s = s0 + a;
    float q = 0.f, w = 0.f;
    int i0 = 0;
    if (s < nslot) {
      const float4 p = xyzq[s];
      const double3 g = global_pos(p, origin, s);
      q = p.w;
      if (dim == 0) anchor(g.x, d.rLx, d.nx, i0, w);
      else if (dim == 1) anchor(g.y, d.rLy, d.ny, i0, w);
      else anchor(g.z, d.rLz, d.nz, i0, w);
    }
    float th[ORDER], dth[ORDER];
    bspline<ORDER>(w, th, dth);
    sh_i[dim][a] = i0;
#pragma unroll
    for (int k = 0; k < ORDER; ++k) sh_th[dim][a][k] = th[k];
    if (dim == 0) sh_q[a] = q;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < 32 * P3; k += blockDim.x) {
    const int a = k / P3, pt = k - a * P3;
    const float q = sh_q[a];
    if (q == 0.f) continue;
    const int xa = pt % ORDER, yb = (pt / ORDER) % ORDER, zc = pt / (ORDER * ORDER);
    int x = sh_i[0][a] + xa, y = sh_i[1][a] + yb, z = sh_i[2][a] + zc;
    if (x >= d.nx) x -= d.nx;
    if (y >= d.ny) y -= d.ny;
    if (z >= d.nz) z -= d.nz;
    const float v = q * sh_th[0][a][xa] * sh_th[1][a][yb] * sh_th[2][a][zc];
    atomicAdd(&qgrid[x + d.nx * (y + d.ny * z)], __float2int_rn(v * kGridScale));
  }
}

// ------------------------------------------------------------------------
// plane transforms
// ------------------------------------------------------------------------
// The grid dimensions are read through a pointer (to the kernel parameter or
// to the system's entry of the multi-system table), never copied: the FFT
// stages index their per-stage divisors at run time.
__global__ void __launch_bounds__(kPlaneThreads) plane_fwd_kernel(const __grid_constant__ PmeDims d0, int *__restrict__ qgrid,
                                                                  float2 *__restrict__ cgrid,
                                                                  const float2 *__restrict__ twx,
                                                                  const float2 *__restrict__ twy,
                                                                  const PmeSysArgs *__restrict__ multi = nullptr,
                                                                  const int *__restrict__ plane_sys = nullptr) {
  extern __shared__ float2 buf[];
  int z = blockIdx.x;
  const PmeDims *dp = &d0;
  if (multi) {
    const PmeSysArgs &A = multi[plane_sys[blockIdx.x]];
    dp = &A.d;
    qgrid = A.qgrid;
    cgrid = A.cgrid;
    twx = A.tw;
    twy = A.tw + A.d.nx;
    z = blockIdx.x - A.plane0;
  }
  const PmeDims &d = *dp;
  __shared__ short s_rev[256];  // x -> position in the digit-reversed row
  const int nx = d.nx, ny = d.ny, nxc = d.nxc, nxcp = d.nxcp, rowp = nx + 2, h = nx / 2;
  int *plane = qgrid + (size_t)z * nx * ny;
  fill_rev_table(s_rev, d.ax, false);
  __syncthreads();
  // four loads in flight per thread before any store (latency-bound loop)
  const int total = nx * ny;
  for (int base = threadIdx.x; base < total; base += 4 * blockDim.x) {
    int v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int idx = base + u * blockDim.x;
      v[u] = idx < total ? plane[idx] : 0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int idx = base + u * blockDim.x;
      if (idx < total) {
        plane[idx] = 0;  // ready for the next spread
        const int y = (int)fdiv((unsigned)idx, d.ax.by_n), x = idx - y * nx;
        float *slot = reinterpret_cast<float *>(&buf[(y >> 1) * rowp + s_rev[x]]);
        slot[y & 1] = (float)v[u] * kInvGridScale;
      }
    }
  }
  __syncthreads();
  fft_dit(buf, ny / 2, rowp, 1, d.ax, twx, -1.f);
  // split the packed rows into the two half spectra, in place
  const int ngrp = (h + 1) / 2 + 1;
  for (int idx = threadIdx.x; idx < (ny / 2) * ngrp; idx += blockDim.x) {
    const int r = (int)fdiv((unsigned)idx, d.ax.by_ngrp), g = idx - r * ngrp;
    float2 *b = buf + r * rowp;
    if (g == ngrp - 1) {
      const float2 Z = b[h];
      b[h] = make_float2(Z.x, 0.f);
      b[nxc + h] = make_float2(Z.y, 0.f);
    } else {
      const int k1 = g, k2 = h - 1 - g;
      const float2 Z1 = b[k1], M1 = b[(nx - k1) % nx];
      const float2 Z2 = b[k2], M2 = b[nx - k2];
      const float2 A1 = make_float2(0.5f * (Z1.x + M1.x), 0.5f * (Z1.y - M1.y));
      const float2 B1 = make_float2(0.5f * (Z1.y + M1.y), -0.5f * (Z1.x - M1.x));
      const float2 A2 = make_float2(0.5f * (Z2.x + M2.x), 0.5f * (Z2.y - M2.y));
      const float2 B2 = make_float2(0.5f * (Z2.y + M2.y), -0.5f * (Z2.x - M2.x));
      b[k1] = A1;
      b[nxc + k1] = B1;
      if (k2 != k1) {
        b[k2] = A2;
        b[nxc + k2] = B2;
      }
    }
  }
  __syncthreads();
  // the in-place split leaves row y at y*nxc (rowp = 2 nxc: row 2r+1 starts
  // right after row 2r); in global memory rows have the even pitch nxcp
  fft_dif(buf, nxc, 1, nxc, d.ay, twy, -1.f);
  float2 *out = cgrid + (size_t)z * ny * nxcp;
  for (int idx = threadIdx.x; idx < ny * nxcp; idx += blockDim.x) {
    const int y = (int)fdiv((unsigned)idx, d.ax.by_nxcp), kx = idx - y * nxcp;
    out[idx] = kx < nxc ? buf[y * nxc + kx] : make_float2(0.f, 0.f);
  }
}

__global__ void __launch_bounds__(kPlaneThreads) plane_inv_kernel(const __grid_constant__ PmeDims d0,
                                                                  const float2 *__restrict__ cgrid,
                                                                  float *__restrict__ phi,
                                                                  const float2 *__restrict__ twx,
                                                                  const float2 *__restrict__ twy,
                                                                  const PmeSysArgs *__restrict__ multi = nullptr,
                                                                  const int *__restrict__ plane_sys = nullptr) {
  extern __shared__ float2 buf[];
  int z = blockIdx.x;
  const PmeDims *dp = &d0;
  if (multi) {
    const PmeSysArgs &A = multi[plane_sys[blockIdx.x]];
    dp = &A.d;
    cgrid = A.cgrid;
    phi = A.phi;
    twx = A.tw;
    twy = A.tw + A.d.nx;
    z = blockIdx.x - A.plane0;
  }
  const PmeDims &d = *dp;
  __shared__ short s_unrev[256];  // position in the digit-reversed row -> x
  const int nx = d.nx, ny = d.ny, nxc = d.nxc, nxcp = d.nxcp, rowp = nx + 2, h = nx / 2;
  const float2 *in = cgrid + (size_t)z * ny * nxcp;
  fill_rev_table(s_unrev, d.ax, true);
  for (int idx = threadIdx.x; idx < ny * nxc; idx += blockDim.x) {
    const int y = (int)fdiv((unsigned)idx, d.ax.by_nxc), kx = idx - y * nxc;
    buf[idx] = in[y * nxcp + kx];
  }
  __syncthreads();
  fft_dit(buf, nxc, 1, nxc, d.ay, twy, 1.f);
  // pack pairs of half spectra into one complex row, in place
  const int ngrp = (h + 1) / 2 + 1;
  for (int idx = threadIdx.x; idx < (ny / 2) * ngrp; idx += blockDim.x) {
    const int r = (int)fdiv((unsigned)idx, d.ax.by_ngrp), g = idx - r * ngrp;
    float2 *b = buf + r * rowp;
    if (g == ngrp - 1) {
      const float2 A = b[h], B = b[nxc + h];
      b[h] = make_float2(A.x - B.y, A.y + B.x);
    } else {
      const int k1 = g, k2 = h - 1 - g;
      const float2 A1 = b[k1], B1 = b[nxc + k1], A2 = b[k2], B2 = b[nxc + k2];
      b[k1] = make_float2(A1.x - B1.y, A1.y + B1.x);
      if (k1 > 0) b[nx - k1] = make_float2(A1.x + B1.y, -A1.y + B1.x);
      if (k2 != k1) {
        b[k2] = make_float2(A2.x - B2.y, A2.y + B2.x);
        if (k2 > 0) b[nx - k2] = make_float2(A2.x + B2.y, -A2.y + B2.x);
      }
    }
  }
  __syncthreads();
  fft_dif(buf, ny / 2, rowp, 1, d.ax, twx, 1.f);
  float *out = phi + (size_t)z * nx * ny;
  for (int idx = threadIdx.x; idx < (ny / 2) * nx; idx += blockDim.x) {
    const int r = (int)fdiv((unsigned)idx, d.ax.by_n), p = idx - r * nx;
    const int x = s_unrev[p];
    const float2 v = buf[r * rowp + p];
    out[(2 * r) * nx + x] = v.x;
    out[(2 * r + 1) * nx + x] = v.y;
  }
}

// ------------------------------------------------------------------------
// z pencils: FFT, influence function, inverse FFT
// ------------------------------------------------------------------------
template <bool ENERGY, typename FT, bool VIRIAL = false, bool TMA = false>
__global__ void __launch_bounds__(kPencilThreads) pencil_kernel(const __grid_constant__ PmeDims d0, float2 *__restrict__ cgrid,
                                                                const float2 *__restrict__ twz,
                                                                const float *__restrict__ prefac,
                                                                const double *__restrict__ prefac_d,
                                                                long long *__restrict__ energy,
                                                                long long *__restrict__ virial,
                                                                const PmeSysArgs *__restrict__ multi,
                                                                const int *__restrict__ pencil_sys,
                                                                const __grid_constant__ CUtensorMap tmap,
                                                                unsigned *__restrict__ err,
                                                                const double4 *__restrict__ dbox = nullptr) {
  // TMA: the slab of 16 complex columns x nz arrives in (and leaves from)
  // buf as one tiled copy of the padded complex grid
  __shared__ __align__(128) float2 buf[256 * kPencilTX];
  __shared__ __align__(8) unsigned long long s_bar;
  __shared__ short s_unrev_z[256];
  __shared__ double sh_e[kPencilThreads / 32];
  __shared__ double sh_v[6][kPencilThreads / 32];
  int blk = blockIdx.x;
  const PmeDims *dp = &d0;
  if (multi) {
    const PmeSysArgs &A = multi[pencil_sys[blockIdx.x]];
    dp = &A.d;
    cgrid = A.cgrid;
    twz = A.tw + A.d.nx + A.d.ny;
    prefac = A.prefac;
    prefac_d = A.prefac_d;
    energy = A.energy;
    virial = A.virial;
    blk = blockIdx.x - A.pencil0;
  }
  const PmeDims &d = *dp;
  const int nx = d.nx, ny = d.ny, nz = d.nz, nxc = d.nxc;
  float Lx = d.Lx, Ly = d.Ly, Lz = d.Lz;  // the box, or the device's copy of it
  if (dbox) {
    const double4 b = *dbox;
    Lx = (float)b.x;
    Ly = (float)b.y;
    Lz = (float)b.z;
  }
  const int tiles_x = (nxc + kPencilTX - 1) / kPencilTX;
  const int py = blk / tiles_x, x0 = (blk - py * tiles_x) * kPencilTX;
  if (TMA) {
    if (threadIdx.x == 0) mbar_init(&s_bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
      mbar_expect_tx(&s_bar, (unsigned)(nz * kPencilTX * sizeof(float2)));
      tma_load_3d(buf, &tmap, 2 * x0, py, 0, &s_bar);
    }
    fill_rev_table(s_unrev_z, d.az, true);
    if (!mbar_wait(&s_bar, 0u)) {
      // the copy did not land: report it, give it a second bounded wait so
      // no write into this block's shared memory is left in flight, and leave
      // the slab untouched
      if (threadIdx.x == 0) atomicOr(err, (unsigned)kErrCopyTimeout);
      mbar_wait(&s_bar, 0u);
      return;
    }
  } else {
    fill_rev_table(s_unrev_z, d.az, true);
    for (int idx = threadIdx.x; idx < nz * kPencilTX; idx += blockDim.x) {
      const int zz = idx / kPencilTX, xt = idx - zz * kPencilTX, kx = x0 + xt;
      buf[idx] = kx < nxc ? cgrid[((size_t)zz * ny + py) * d.nxcp + kx] : make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
  fft_dif(buf, kPencilTX, 1, kPencilTX, d.az, twz, -1.f);
  const int ky = dig_unrev(py, d.ay);
  const int nf1 = nx / 2 + (nx & 1), nf2 = ny / 2 + (ny & 1), nf3 = nz / 2 + (nz & 1);
  const FT m2 = (FT)(ky >= nf2 ? ky - ny : ky) / (FT)Ly;
  const FT pi = (FT)3.14159265358979323846;
  const FT fac = pi * pi / ((FT)d.kappa * (FT)d.kappa);
  const FT piv_inv = (FT)1 / ((FT)Lx * (FT)Ly * (FT)Lz * pi);
  const FT *pf = sizeof(FT) == 8 ? reinterpret_cast<const FT *>(prefac_d)
                                 : reinterpret_cast<const FT *>(prefac);
  const FT pyv = pf[nx + ky];
  double e = 0.0;
  double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int idx = threadIdx.x; idx < nz * kPencilTX; idx += blockDim.x) {
    const int pz = idx / kPencilTX, xt = idx - pz * kPencilTX, kx = x0 + xt;
    if (kx >= nxc) continue;
    const int kz = s_unrev_z[pz];
    FT eterm = 0;
    const FT m1 = (FT)(kx >= nf1 ? kx - nx : kx) / (FT)Lx;
    const FT m3 = (FT)(kz >= nf3 ? kz - nz : kz) / (FT)Lz;
    const FT msq = m1 * m1 + m2 * m2 + m3 * m3;
    if (kx != 0 || ky != 0 || kz != 0)
      eterm = exp(-fac * msq) * piv_inv * pf[kx] * pyv * pf[nx + ny + kz] / msq;
    const float2 q = buf[idx];
    if (ENERGY) {
      const FT mult = kx >= 1 ? (FT)2 : (FT)1;
      const FT t1 = mult * eterm * ((FT)q.x * q.x + (FT)q.y * q.y);
      e += (double)t1;
      if (VIRIAL && eterm != (FT)0) {
        // reference scalar_sum (src/CudaPMERecip.cu:770-790): t1 (vterm m_a m_b - delta_ab)
        const FT vt = (FT)2 * (fac + (FT)1 / msq);
        v[0] += (double)(t1 * (vt * m1 * m1 - (FT)1));
        v[1] += (double)(t1 * vt * m1 * m2);
        v[2] += (double)(t1 * vt * m1 * m3);
        v[3] += (double)(t1 * (vt * m2 * m2 - (FT)1));
        v[4] += (double)(t1 * vt * m2 * m3);
        v[5] += (double)(t1 * (vt * m3 * m3 - (FT)1));
      }
    }
    buf[idx] = make_float2((float)(q.x * eterm), (float)(q.y * eterm));
  }
  __syncthreads();
  fft_dit(buf, kPencilTX, 1, kPencilTX, d.az, twz, 1.f);
  if (TMA) {
    // columns past the grid's padded width are clipped by the copy
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) tma_store_3d(&tmap, 2 * x0, py, 0, buf);
  } else {
    for (int idx = threadIdx.x; idx < nz * kPencilTX; idx += blockDim.x) {
      const int zz = idx / kPencilTX, xt = idx - zz * kPencilTX, kx = x0 + xt;
      if (kx < nxc) cgrid[((size_t)zz * ny + py) * d.nxcp + kx] = buf[idx];
    }
  }
  if (ENERGY) {
    e = warp_sum(e);
    if ((threadIdx.x & 31) == 0) sh_e[threadIdx.x >> 5] = e;
    if (VIRIAL) {
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double t = warp_sum(v[k]);
        if ((threadIdx.x & 31) == 0) sh_v[k][threadIdx.x >> 5] = t;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kPencilThreads / 32; ++w) t += sh_e[w];
      add_energy(energy + kEEwks, 0.5 * kCcelec * t);
    }
    if (VIRIAL && threadIdx.x < 6) {
      double t = 0.0;
      for (int w = 0; w < kPencilThreads / 32; ++w) t += sh_v[threadIdx.x][w];
      // xx xy xz yy yz zz -> row-major 3x3, W = -ccelec/2 * sum
      constexpr int kA[6] = {0, 1, 2, 4, 5, 8}, kB[6] = {0, 3, 6, 4, 7, 8};
      const long long iw = __double2ll_rn(-0.5 * kCcelec * t * kEnergyScale);
      add_fixed(virial + kA[threadIdx.x], iw);
      if (kB[threadIdx.x] != kA[threadIdx.x]) add_fixed(virial + kB[threadIdx.x], iw);
    }
  }
}

// ------------------------------------------------------------------------
// gather: 8 threads per atom, (y,z) pairs split across the 8, x loop inside
// ------------------------------------------------------------------------
template <int ORDER>
__global__ void __launch_bounds__(256) gather_kernel(const float4 *__restrict__ xyzq,
                                                     const int *__restrict__ counts, PmeDims d,
                                                     const float *__restrict__ phi,
                                                     long long *__restrict__ force, int stride,
                                                     const float4 *__restrict__ origin,
                                                     const PmeSysArgs *__restrict__ multi = nullptr,
                                                     const int *__restrict__ cl_sys = nullptr,
                                                     const double4 *__restrict__ dbox = nullptr) {
  if (multi) {  // one block = one 32-slot cluster of one system
    const PmeSysArgs &A = multi[cl_sys[blockIdx.x]];
    d = A.d;
    phi = A.phi;
  }
  if (dbox) box_from_device(d, *dbox);
  const int nslot = counts[0];
  const int s = blockIdx.x * 32 + (threadIdx.x >> 3);
  const int sub = threadIdx.x & 7;
  float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
  double3 g = make_double3(0.0, 0.0, 0.0);
  if (s < nslot) {
    p = xyzq[s];
    g = global_pos(p, origin, s);
  }
  float thx[ORDER], thy[ORDER], thz[ORDER], dx[ORDER], dy[ORDER], dz[ORDER], w;
  int ix, iy, iz;
  anchor(g.x, d.rLx, d.nx, ix, w);
  bspline<ORDER>(w, thx, dx);
  anchor(g.y, d.rLy, d.ny, iy, w);
  bspline<ORDER>(w, thy, dy);
  anchor(g.z, d.rLz, d.nz, iz, w);
  bspline<ORDER>(w, thz, dz);
  float f1 = 0.f, f2 = 0.f, f3 = 0.f;
  if (s < nslot && p.w != 0.f) {
    for (int k = sub; k < ORDER * ORDER; k += 8) {
      const int b = k % ORDER, c = k / ORDER;
      int y = iy + b, z = iz + c;
      if (y >= d.ny) y -= d.ny;
      if (z >= d.nz) z -= d.nz;
      const float *row = phi + ((size_t)z * d.ny + y) * d.nx;
      float tyb = 0.f, dyb = 0.f, tzc = 0.f, dzc = 0.f;
#pragma unroll
      for (int t = 0; t < ORDER; ++t) {
        if (t == b) { tyb = thy[t]; dyb = dy[t]; }
        if (t == c) { tzc = thz[t]; dzc = dz[t]; }
      }
      float sx = 0.f, sdx = 0.f;
#pragma unroll
      for (int a = 0; a < ORDER; ++a) {
        int x = ix + a;
        if (x >= d.nx) x -= d.nx;
        const float v = __ldg(row + x);
        sx += thx[a] * v;
        sdx += dx[a] * v;
      }
      f1 += sdx * tyb * tzc;
      f2 += sx * dyb * tzc;
      f3 += sx * tyb * dzc;
    }
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    f1 += __shfl_xor_sync(0xffffffffu, f1, o);
    f2 += __shfl_xor_sync(0xffffffffu, f2, o);
    f3 += __shfl_xor_sync(0xffffffffu, f3, o);
  }
  if (sub == 0 && s < nslot && p.w != 0.f) {
    const float qc = p.w * (float)kCcelec;
    add_fixed(force + s, to_fixed_force(qc * (float)d.nx / d.Lx * f1));
    add_fixed(force + stride + s, to_fixed_force(qc * (float)d.ny / d.Ly * f2));
    add_fixed(force + 2 * stride + s, to_fixed_force(qc * (float)d.nz / d.Lz * f3));
  }
}

// B-spline moduli as the reference's dftmod (src/CudaPMERecip.cu:2656-2678)
void bspline_moduli(int n, int order, std::vector<double> &out) {
  std::vector<double> th(order), arr(n + order + 2, 0.0);
  // weights at w = 0
  th[order - 1] = 0.0;
  th[1] = 0.0;
  th[0] = 1.0;
  for (int k = 3; k <= order - 1; ++k) {
    double div = 1.0 / (k - 1);
    th[k - 1] = 0.0;
    for (int j = 1; j <= k - 2; ++j) th[k - j - 1] = div * (j * th[k - j - 2] + (k - j) * th[k - j - 1]);
    th[0] = div * th[0];
  }
  {
    double div = 1.0 / (order - 1);
    th[order - 1] = 0.0;
    for (int j = 1; j <= order - 2; ++j)
      th[order - j - 1] = div * (j * th[order - j - 2] + (order - j) * th[order - j - 1]);
    th[0] = div * th[0];
  }
  for (int i = 2; i <= order + 1; ++i) arr[i - 1] = th[i - 2];
  out.assign(n, 0.0);
  for (int k = 0; k < n; ++k) {
    double s1 = 0, s2 = 0;
    for (int j = 0; j < n - 1; ++j) {
      double a = 2.0 * M_PI * k * j / n;
      s1 += arr[j] * std::cos(a);
      s2 += arr[j] * std::sin(a);
    }
    out[k] = s1 * s1 + s2 * s2;
  }
  for (int k = 0; k < n; ++k)
    if (out[k] < 1e-10) out[k] = 0.5 * (out[(k - 1 + n) % n] + out[(k + 1) % n]);
  for (int k = 0; k < n; ++k) out[k] = 1.0 / out[k];
}

template <typename T>
void dalloc(T *&p, size_t n) {
  if (p) cudaFree(p);
  p = nullptr;
  if (n) APO_CUDA(cudaMalloc(&p, n * sizeof(T)));
}

}  // namespace

// The tensor map of the pencil slabs: the padded complex grid viewed as
// floats [nz][ny][2 nxcp], a box of 16 complex columns x 1 row x nz planes.
// The encoder is the driver's, fetched through the runtime (no link to the
// driver library).
bool encode_pencil_map(CUtensorMap *map, float2 *cgrid, const PmeDims &d) {
  using Encode = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                              const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                              const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static Encode fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<Encode>(p);
    else
      cudaGetLastError();
  }
  // a row at least one box wide, at most 256 planes, rows of 16-byte multiples
  if (!fn || d.nz > 256 || (d.nxcp & 1) || 2 * d.nxcp < 2 * kPencilTX) return false;
  const cuuint64_t dims[3] = {2ull * d.nxcp, (cuuint64_t)d.ny, (cuuint64_t)d.nz};
  const cuuint64_t strides[2] = {2ull * d.nxcp * sizeof(float),
                                 2ull * d.nxcp * d.ny * sizeof(float)};
  const cuuint32_t box[3] = {2u * kPencilTX, 1u, (cuuint32_t)d.nz};
  const cuuint32_t es[3] = {1u, 1u, 1u};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, cgrid, dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// shared memory of one plane transform: ny/2 packed rows of nx + 2 complex
static size_t plane_smem_bytes(int nx, int ny) {
  return (size_t)(ny / 2) * (nx + 2) * sizeof(float2);
}

FastDiv make_fastdiv(unsigned d) {
  FastDiv f{0u, 0u};
  if (d <= 1) return f;
  unsigned l = 0;  // ceil(log2 d)
  while ((1u << l) < d) ++l;
  f.mul = (unsigned)(((1ull << (31 + l)) + d - 1) / d);
  f.shift = l - 1;
  return f;
}

void fill_axis_divisors(FftAxis &a) {
  int prod = 1;
  for (int s = 0; s < a.nrad; ++s) {
    prod *= a.radix[s];
    a.per_line[s] = make_fastdiv((unsigned)(a.n / a.radix[s]));
    a.dif_mr[s] = make_fastdiv((unsigned)(a.n / prod));
  }
  int tail = 1;
  for (int s = a.nrad - 1; s >= 0; --s) {
    a.dit_mr[s] = make_fastdiv((unsigned)tail);
    tail *= a.radix[s];
  }
  a.by_n = make_fastdiv((unsigned)a.n);
  a.by_nxc = make_fastdiv((unsigned)(a.n / 2 + 1));
  a.by_nxcp = make_fastdiv((unsigned)((a.n / 2 + 2) & ~1));
  a.by_ngrp = make_fastdiv((unsigned)((a.n / 2 + 1) / 2 + 1));
}

FftAxis Pme::plan_axis(int n) {
  // fewest stages, then smallest total radix
  std::vector<int> best;
  std::vector<int> cur;
  std::function<void(int)> rec = [&](int m) {
    if (m == 1) {
      if (best.empty() || cur.size() < best.size() ||
          (cur.size() == best.size() &&
           std::accumulate(cur.begin(), cur.end(), 0) < std::accumulate(best.begin(), best.end(), 0)))
        best = cur;
      return;
    }
    if (!best.empty() && cur.size() + 1 > best.size()) return;
    for (int R : {8, 7, 6, 5, 4, 3, 2}) {
      if (m % R == 0) {
        cur.push_back(R);
        rec(m / R);
        cur.pop_back();
      }
    }
  };
  rec(n);
  if (best.empty() || best.size() > 8)
    throw std::invalid_argument("PME grid size " + std::to_string(n) +
                                " must factor into 2, 3, 5 and 7");
  FftAxis a{};
  a.n = n;
  a.nrad = (int)best.size();
  for (size_t i = 0; i < best.size(); ++i) a.radix[i] = best[i];
  fill_axis_divisors(a);
  return a;
}

Pme::~Pme() { release(); }

void Pme::release() {
  if (qgrid) cudaFree(qgrid);
  if (cgrid) cudaFree(cgrid);
  if (phi) cudaFree(phi);
  if (m_tw) cudaFree(m_tw);
  if (m_prefac) cudaFree(m_prefac);
  if (m_prefac_d) cudaFree(m_prefac_d);
  qgrid = nullptr;
  cgrid = nullptr;
  phi = nullptr;
  m_tw = nullptr;
  m_prefac = nullptr;
  m_prefac_d = nullptr;
}

void Pme::setup(int nx, int ny, int nz, int order, double kappa, double Lx, double Ly,
                double Lz) {
  if (nx % 2 || ny % 2 || nz % 2)
    throw std::invalid_argument("PME grid dimensions must be even");
  if (nx > 256 || ny > 256 || nz > 256)
    throw std::invalid_argument("PME grid dimensions above 256 are not supported");
  if (order != 4 && order != 6 && order != 8)
    throw std::invalid_argument("PME spline order must be 4, 6 or 8");
  // a spline's p points wrap the grid at most once only when n >= p
  if (nx < order || ny < order || nz < order)
    throw std::invalid_argument("PME grid dimensions must be at least the spline order");
  const size_t plane_bytes = plane_smem_bytes(nx, ny);
  if (plane_bytes > kPlaneSmemMax)
    throw std::invalid_argument("PME plane does not fit in shared memory");
  release();
  m_d.nx = nx;
  m_d.ny = ny;
  m_d.nz = nz;
  m_d.nxc = nx / 2 + 1;
  m_d.nxcp = (m_d.nxc + 1) & ~1;
  m_d.order = order;
  m_d.Lx = (float)Lx;
  m_d.Ly = (float)Ly;
  m_d.Lz = (float)Lz;
  m_d.rLx = 1.0 / Lx;
  m_d.rLy = 1.0 / Ly;
  m_d.rLz = 1.0 / Lz;
  m_d.kappa = (float)kappa;
  m_d.ax = plan_axis(nx);
  m_d.ay = plan_axis(ny);
  m_d.az = plan_axis(nz);
  const size_t G = (size_t)nx * ny * nz;
  dalloc(qgrid, G);
  dalloc(cgrid, (size_t)nz * ny * m_d.nxcp);
  APO_CUDA(cudaMemset(cgrid, 0, (size_t)nz * ny * m_d.nxcp * sizeof(float2)));
  m_tma = encode_pencil_map(&m_tmap, cgrid, m_d);
  dalloc(phi, G);
  APO_CUDA(cudaMemset(qgrid, 0, G * sizeof(int)));
  std::vector<float2> tw;
  for (int n : {nx, ny, nz})
    for (int k = 0; k < n; ++k) {
      double a = 2.0 * M_PI * k / n;
      tw.push_back(make_float2((float)std::cos(a), (float)-std::sin(a)));
    }
  dalloc(m_tw, tw.size());
  APO_CUDA(cudaMemcpy(m_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice));
  std::vector<double> pd, tmp;
  for (int n : {nx, ny, nz}) {
    bspline_moduli(n, order, tmp);
    pd.insert(pd.end(), tmp.begin(), tmp.end());
  }
  std::vector<float> pf(pd.begin(), pd.end());
  dalloc(m_prefac, pf.size());
  dalloc(m_prefac_d, pd.size());
  APO_CUDA(cudaMemcpy(m_prefac, pf.data(), pf.size() * sizeof(float), cudaMemcpyHostToDevice));
  APO_CUDA(cudaMemcpy(m_prefac_d, pd.data(), pd.size() * sizeof(double), cudaMemcpyHostToDevice));
  static bool attr = false;
  if (!attr) {
    APO_CUDA(cudaFuncSetAttribute(plane_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kPlaneSmemMax));
    APO_CUDA(cudaFuncSetAttribute(plane_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kPlaneSmemMax));
    attr = true;
  }
}

void Pme::spread(const float4 *xyzq_s, const int *counts, cudaStream_t s,
                 const float4 *origin) {
  const int blocks = (max_slots + 31) / 32;
  switch (m_d.order) {
    case 4: spread_kernel<4><<<blocks, 128, 0, s>>>(xyzq_s, counts, m_d, qgrid, origin, nullptr, nullptr, m_dbox); break;
    case 6: spread_kernel<6><<<blocks, 128, 0, s>>>(xyzq_s, counts, m_d, qgrid, origin, nullptr, nullptr, m_dbox); break;
    case 8: spread_kernel<8><<<blocks, 128, 0, s>>>(xyzq_s, counts, m_d, qgrid, origin, nullptr, nullptr, m_dbox); break;
  }
  APO_LAUNCH_CHECK();
}

void Pme::forward(cudaStream_t s) {
  const size_t sm = plane_smem_bytes(m_d.nx, m_d.ny);
  plane_fwd_kernel<<<m_d.nz, kPlaneThreads, sm, s>>>(m_d, qgrid, cgrid, m_tw, m_tw + m_d.nx);
  APO_LAUNCH_CHECK();
}

void Pme::convolve(long long *energy, bool calc_energy, bool fp64, cudaStream_t s,
                   long long *virial) {
  const int tiles_x = (m_d.nxc + kPencilTX - 1) / kPencilTX;
  const int grid = tiles_x * m_d.ny;
  const float2 *twz = m_tw + m_d.nx + m_d.ny;
  const bool tma = tensor_copies() && m_err;
#define APO_PENCIL(E, FT, V)                                                                   \
  do {                                                                                         \
    if (tma)                                                                                   \
      pencil_kernel<E, FT, V, true><<<grid, kPencilThreads, 0, s>>>(                           \
          m_d, cgrid, twz, m_prefac, m_prefac_d, energy, virial, nullptr, nullptr, m_tmap, m_err, \
          m_dbox);                                                                             \
    else                                                                                       \
      pencil_kernel<E, FT, V, false><<<grid, kPencilThreads, 0, s>>>(                          \
          m_d, cgrid, twz, m_prefac, m_prefac_d, energy, virial, nullptr, nullptr, m_tmap, m_err, \
          m_dbox);                                                                             \
  } while (0)
  if (virial) {
    if (fp64) APO_PENCIL(true, double, true);
    else APO_PENCIL(true, float, true);
  } else if (fp64) {
    if (calc_energy) APO_PENCIL(true, double, false);
    else APO_PENCIL(false, double, false);
  } else {
    if (calc_energy) APO_PENCIL(true, float, false);
    else APO_PENCIL(false, float, false);
  }
#undef APO_PENCIL
  APO_LAUNCH_CHECK();
}

void Pme::backward(cudaStream_t s) {
  const size_t sm = plane_smem_bytes(m_d.nx, m_d.ny);
  plane_inv_kernel<<<m_d.nz, kPlaneThreads, sm, s>>>(m_d, cgrid, phi, m_tw, m_tw + m_d.nx);
  APO_LAUNCH_CHECK();
}

void Pme::gather(const float4 *xyzq_s, const int *counts, long long *force, int stride,
                 cudaStream_t s, const float4 *origin) {
  const int blocks = (max_slots + 31) / 32;
  switch (m_d.order) {
    case 4: gather_kernel<4><<<blocks, 256, 0, s>>>(xyzq_s, counts, m_d, phi, force, stride, origin, nullptr, nullptr, m_dbox); break;
    case 6: gather_kernel<6><<<blocks, 256, 0, s>>>(xyzq_s, counts, m_d, phi, force, stride, origin, nullptr, nullptr, m_dbox); break;
    case 8: gather_kernel<8><<<blocks, 256, 0, s>>>(xyzq_s, counts, m_d, phi, force, stride, origin, nullptr, nullptr, m_dbox); break;
  }
  APO_LAUNCH_CHECK();
}

void Pme::compute(const float4 *xyzq_s, const int *counts, long long *force, int stride,
                  long long *energy, bool calc_energy, bool fp64, cudaStream_t s,
                  long long *virial, const float4 *origin) {
  spread(xyzq_s, counts, s, origin);
  forward(s);
  convolve(energy, calc_energy, fp64, s, virial);
  backward(s);
  gather(xyzq_s, counts, force, stride, s, origin);
}

}  // namespace apo

// ---------------------------------------------------------------------------
// Many systems
// ---------------------------------------------------------------------------

namespace apo {

PmeMulti::~PmeMulti() { release(); }

void PmeMulti::release() {
  for (void *p : {(void *)m_args, (void *)m_plane_sys, (void *)m_pencil_sys, (void *)m_q,
                  (void *)m_c, (void *)m_phi, (void *)m_tw, (void *)m_pf, (void *)m_pfd})
    if (p) cudaFree(p);
  m_args = nullptr;
  m_plane_sys = m_pencil_sys = nullptr;
  m_q = nullptr;
  m_c = nullptr;
  m_phi = nullptr;
  m_tw = nullptr;
  m_pf = nullptr;
  m_pfd = nullptr;
}

void PmeMulti::setup(const std::vector<PmeSystemSpec> &systems, int order, long long *energy,
                     int energy_stride, int max_slots) {
  if (systems.empty()) throw std::invalid_argument("PmeMulti: no systems");
  if (order != 4 && order != 6 && order != 8)
    throw std::invalid_argument("PME spline order must be 4, 6 or 8");
  release();
  m_host.clear();
  m_order = order;
  m_max_slots = max_slots;
  size_t q = 0, c = 0, t = 0;
  std::vector<int> plane_sys, pencil_sys;
  std::vector<float2> tw;
  std::vector<double> pd;
  m_plane_smem = 0;
  for (size_t k = 0; k < systems.size(); ++k) {
    const PmeSystemSpec &y = systems[k];
    if (y.nx % 2 || y.ny % 2 || y.nz % 2 || y.nx <= 0 || y.ny <= 0 || y.nz <= 0)
      throw std::invalid_argument("PME grid dimensions must be even");
    if (y.nx > 256 || y.ny > 256 || y.nz > 256)
      throw std::invalid_argument("PME grid dimensions above 256 are not supported");
    if (y.nx < order || y.ny < order || y.nz < order)
      throw std::invalid_argument("PME grid dimensions must be at least the spline order");
    const size_t plane_bytes = plane_smem_bytes(y.nx, y.ny);
    if (plane_bytes > kPlaneSmemMax) throw std::invalid_argument("PME plane does not fit in shared memory");
    m_plane_smem = std::max(m_plane_smem, plane_bytes);
    PmeSysArgs A{};
    A.d.nx = y.nx;
    A.d.ny = y.ny;
    A.d.nz = y.nz;
    A.d.nxc = y.nx / 2 + 1;
    A.d.nxcp = (A.d.nxc + 1) & ~1;
    A.d.order = order;
    A.d.Lx = (float)y.Lx;
    A.d.Ly = (float)y.Ly;
    A.d.Lz = (float)y.Lz;
    A.d.rLx = 1.0 / y.Lx;
    A.d.rLy = 1.0 / y.Ly;
    A.d.rLz = 1.0 / y.Lz;
    A.d.kappa = (float)y.kappa;
    A.d.ax = Pme::plan_axis(y.nx);
    A.d.ay = Pme::plan_axis(y.ny);
    A.d.az = Pme::plan_axis(y.nz);
    // offsets for now; turned into pointers once the buffers exist
    A.qgrid = reinterpret_cast<int *>(q);
    A.phi = reinterpret_cast<float *>(q);
    A.cgrid = reinterpret_cast<float2 *>(c);
    A.tw = reinterpret_cast<const float2 *>(t);
    A.prefac = reinterpret_cast<const float *>(t);
    A.prefac_d = reinterpret_cast<const double *>(t);
    A.energy = energy + k * (size_t)energy_stride;
    A.virial = A.energy + kNumEnergyTerms;
    A.plane0 = m_planes;
    A.pencil0 = m_pencils;
    const int tiles_x = (A.d.nxc + kPencilTX - 1) / kPencilTX;
    for (int z = 0; z < y.nz; ++z) plane_sys.push_back((int)k);
    for (int b = 0; b < tiles_x * y.ny; ++b) pencil_sys.push_back((int)k);
    m_planes += y.nz;
    m_pencils += tiles_x * y.ny;
    q += (size_t)y.nx * y.ny * y.nz;
    c += (size_t)y.nz * y.ny * A.d.nxcp;
    t += (size_t)y.nx + y.ny + y.nz;
    for (int n : {y.nx, y.ny, y.nz})
      for (int j = 0; j < n; ++j) {
        const double a = 2.0 * M_PI * j / n;
        tw.push_back(make_float2((float)std::cos(a), (float)-std::sin(a)));
      }
    std::vector<double> tmp;
    for (int n : {y.nx, y.ny, y.nz}) {
      bspline_moduli(n, order, tmp);
      pd.insert(pd.end(), tmp.begin(), tmp.end());
    }
    m_host.push_back(A);
  }
  APO_CUDA(cudaMalloc(&m_q, q * sizeof(int)));
  APO_CUDA(cudaMalloc(&m_phi, q * sizeof(float)));
  APO_CUDA(cudaMalloc(&m_c, c * sizeof(float2)));
  APO_CUDA(cudaMalloc(&m_tw, t * sizeof(float2)));
  APO_CUDA(cudaMalloc(&m_pf, t * sizeof(float)));
  APO_CUDA(cudaMalloc(&m_pfd, t * sizeof(double)));
  APO_CUDA(cudaMemset(m_q, 0, q * sizeof(int)));
  std::vector<float> pf(pd.begin(), pd.end());
  APO_CUDA(cudaMemcpy(m_tw, tw.data(), t * sizeof(float2), cudaMemcpyHostToDevice));
  APO_CUDA(cudaMemcpy(m_pf, pf.data(), t * sizeof(float), cudaMemcpyHostToDevice));
  APO_CUDA(cudaMemcpy(m_pfd, pd.data(), t * sizeof(double), cudaMemcpyHostToDevice));
  for (PmeSysArgs &A : m_host) {
    const size_t qo = reinterpret_cast<size_t>(A.qgrid), co = reinterpret_cast<size_t>(A.cgrid),
                 to = reinterpret_cast<size_t>(A.tw);
    A.qgrid = m_q + qo;
    A.phi = m_phi + qo;
    A.cgrid = m_c + co;
    A.tw = m_tw + to;
    A.prefac = m_pf + to;
    A.prefac_d = m_pfd + to;
  }
  APO_CUDA(cudaMalloc(&m_args, m_host.size() * sizeof(PmeSysArgs)));
  APO_CUDA(cudaMemcpy(m_args, m_host.data(), m_host.size() * sizeof(PmeSysArgs),
                      cudaMemcpyHostToDevice));
  APO_CUDA(cudaMalloc(&m_plane_sys, plane_sys.size() * sizeof(int)));
  APO_CUDA(cudaMemcpy(m_plane_sys, plane_sys.data(), plane_sys.size() * sizeof(int),
                      cudaMemcpyHostToDevice));
  APO_CUDA(cudaMalloc(&m_pencil_sys, pencil_sys.size() * sizeof(int)));
  APO_CUDA(cudaMemcpy(m_pencil_sys, pencil_sys.data(), pencil_sys.size() * sizeof(int),
                      cudaMemcpyHostToDevice));
  APO_CUDA(cudaFuncSetAttribute(plane_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kPlaneSmemMax));
  APO_CUDA(cudaFuncSetAttribute(plane_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kPlaneSmemMax));
}

void PmeMulti::compute(const float4 *xyzq_s, const float4 *origin, const int *cl_sys,
                       const int *counts, long long *force, int stride, bool calc_energy,
                       bool calc_virial, bool fp64, cudaStream_t s) {
  const PmeDims &d0 = m_host[0].d;
  const int blocks = (m_max_slots + 31) / 32;
  switch (m_order) {
    case 4: spread_kernel<4><<<blocks, 128, 0, s>>>(xyzq_s, counts, d0, nullptr, origin, m_args, cl_sys); break;
    case 6: spread_kernel<6><<<blocks, 128, 0, s>>>(xyzq_s, counts, d0, nullptr, origin, m_args, cl_sys); break;
    case 8: spread_kernel<8><<<blocks, 128, 0, s>>>(xyzq_s, counts, d0, nullptr, origin, m_args, cl_sys); break;
  }
  APO_LAUNCH_CHECK();
  plane_fwd_kernel<<<m_planes, kPlaneThreads, m_plane_smem, s>>>(d0, nullptr, nullptr, nullptr,
                                                                  nullptr, m_args, m_plane_sys);
  APO_LAUNCH_CHECK();
  if (calc_virial) {
    if (fp64)
      pencil_kernel<true, double, true><<<m_pencils, kPencilThreads, 0, s>>>(d0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, m_args, m_pencil_sys, kNoTensorMap, nullptr);
    else
      pencil_kernel<true, float, true><<<m_pencils, kPencilThreads, 0, s>>>(d0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, m_args, m_pencil_sys, kNoTensorMap, nullptr);
  } else if (calc_energy) {
    if (fp64)
      pencil_kernel<true, double><<<m_pencils, kPencilThreads, 0, s>>>(d0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, m_args, m_pencil_sys, kNoTensorMap, nullptr);
    else
      pencil_kernel<true, float><<<m_pencils, kPencilThreads, 0, s>>>(d0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, m_args, m_pencil_sys, kNoTensorMap, nullptr);
  } else {
    if (fp64)
      pencil_kernel<false, double><<<m_pencils, kPencilThreads, 0, s>>>(d0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, m_args, m_pencil_sys, kNoTensorMap, nullptr);
    else
      pencil_kernel<false, float><<<m_pencils, kPencilThreads, 0, s>>>(d0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, m_args, m_pencil_sys, kNoTensorMap, nullptr);
  }
  APO_LAUNCH_CHECK();
  plane_inv_kernel<<<m_planes, kPlaneThreads, m_plane_smem, s>>>(d0, nullptr, nullptr, nullptr,
                                                                  nullptr, m_args, m_plane_sys);
  APO_LAUNCH_CHECK();
  switch (m_order) {
    case 4: gather_kernel<4><<<blocks, 256, 0, s>>>(xyzq_s, counts, d0, nullptr, force, stride, origin, m_args, cl_sys); break;
    case 6: gather_kernel<6><<<blocks, 256, 0, s>>>(xyzq_s, counts, d0, nullptr, force, stride, origin, m_args, cl_sys); break;
    case 8: gather_kernel<8><<<blocks, 256, 0, s>>>(xyzq_s, counts, d0, nullptr, force, stride, origin, m_args, cl_sys); break;
  }
  APO_LAUNCH_CHECK();
}

}  // namespace apo

// ---------------------------------------------------------------------------
// Reciprocal space from a static scratch area (no allocation of its own)
// ---------------------------------------------------------------------------
//
// The charge grid, complex grid, potential grid, twiddles, B-spline moduli,
// atom count and energy accumulator live in g_pme_static, a file-scope
// device array.  Its address is looked up once per device with
// cudaGetSymbolAddress (that first call also sets the plane kernels'
// shared-memory attribute, so it belongs before any stream capture).  What
// must be zero when a call's spread starts: the charge grid and the energy
// accumulator.  The array is zero at module load, every call clears both
// with cudaMemsetAsync before its first kernel, and plane_fwd leaves the
// charge grid zeroed again as it reads it.  The tables are recomputed on
// the device by every call, so nothing else carries over between calls;
// calls that overlap in time (two streams, two host threads) race on the
// area.

namespace apo {
namespace {

__device__ __align__(256) unsigned char g_pme_static[kPmeStaticScratchBytes];

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mu;
std::atomic<unsigned char *> g_static_base[kStaticMaxDevices];

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

struct StaticLayout {
  size_t energy, counts, tw, prefac, prefac_d, qgrid, cgrid, phi, total;
};

StaticLayout static_layout(int nx, int ny, int nz) {
  StaticLayout l{};
  const size_t n3 = (size_t)nx + ny + nz;
  const size_t G = (size_t)nx * ny * nz;
  const size_t Gc = (size_t)nz * ny * ((nx / 2 + 2) & ~1);  // padded rows
  size_t o = 0;
  l.energy = o;   o += align256(kNumEnergyTerms * sizeof(long long));
  l.counts = o;   o += align256(4 * sizeof(int));
  l.tw = o;       o += align256(n3 * sizeof(float2));
  l.prefac = o;   o += align256(n3 * sizeof(float));
  l.prefac_d = o; o += align256(n3 * sizeof(double));
  l.qgrid = o;    o += align256(G * sizeof(int));
  l.cgrid = o;    o += align256(Gc * sizeof(float2));
  l.phi = o;      o += align256(G * sizeof(float));
  l.total = o;
  return l;
}

// The plan search of Pme::plan_axis (fewest stages, then the smallest sum
// of radices, radices tried from 8 down to 2) on fixed arrays.
struct FixedPlan {
  int cur[8], best[8], ncur = 0, nbest = -1, sbest = 0;
  void rec(int m) {
    if (m == 1) {
      int s = 0;
      for (int i = 0; i < ncur; ++i) s += cur[i];
      if (nbest < 0 || ncur < nbest || (ncur == nbest && s < sbest)) {
        for (int i = 0; i < ncur; ++i) best[i] = cur[i];
        nbest = ncur;
        sbest = s;
      }
      return;
    }
    if (ncur == 8 || (nbest >= 0 && ncur + 1 > nbest)) return;
    for (int R : {8, 7, 6, 5, 4, 3, 2}) {
      if (m % R == 0) {
        cur[ncur++] = R;
        rec(m / R);
        --ncur;
      }
    }
  }
};

bool fixed_plan_axis(int n, FftAxis &a) {
  FixedPlan p;
  p.rec(n);
  if (p.nbest < 0) return false;
  a = FftAxis{};
  a.n = n;
  a.nrad = p.nbest;
  for (int i = 0; i < p.nbest; ++i) a.radix[i] = p.best[i];
  fill_axis_divisors(a);
  return true;
}

// |b(k)|^2 of the order-p B-spline for grid size n, as bspline_moduli
__device__ double static_modulus(int n, int order, int k) {
  double th[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  th[0] = 1.0;
  for (int kk = 3; kk <= order; ++kk) {
    const double div = 1.0 / (kk - 1);
    th[kk - 1] = 0.0;
    for (int j = 1; j <= kk - 2; ++j) th[kk - j - 1] = div * (j * th[kk - j - 2] + (kk - j) * th[kk - j - 1]);
    th[0] = div * th[0];
  }
  // arr[i - 1] = th[i - 2] for i = 2..order+1: arr[j] = th[j - 1] for j = 1..order
  double s1 = 0.0, s2 = 0.0;
  for (int j = 1; j <= order && j < n - 1; ++j) {
    double sv, cv;
    sincospi(2.0 * (double)(((long long)k * j) % n) / n, &sv, &cv);
    s1 += th[j - 1] * cv;
    s2 += th[j - 1] * sv;
  }
  return s1 * s1 + s2 * s2;
}

__global__ void static_tables_kernel(PmeDims d, float2 *__restrict__ tw, float *__restrict__ prefac,
                                     double *__restrict__ prefac_d, int *__restrict__ counts,
                                     int natom) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) counts[0] = natom;
  int n, k;
  if (t < d.nx) { n = d.nx; k = t; }
  else if (t < d.nx + d.ny) { n = d.ny; k = t - d.nx; }
  else if (t < d.nx + d.ny + d.nz) { n = d.nz; k = t - d.nx - d.ny; }
  else return;
  double sv, cv;
  sincospi(2.0 * k / n, &sv, &cv);
  tw[t] = make_float2((float)cv, (float)-sv);
  double m = static_modulus(n, d.order, k);
  if (m < 1e-10)
    m = 0.5 * (static_modulus(n, d.order, (k - 1 + n) % n) + static_modulus(n, d.order, (k + 1) % n));
  prefac_d[t] = 1.0 / m;
  prefac[t] = (float)(1.0 / m);
}

__global__ void static_finish_kernel(const long long *__restrict__ acc, double *__restrict__ energy) {
  if (threadIdx.x == 0 && blockIdx.x == 0) energy[0] = (double)acc[kEEwks] / kEnergyScale;
}

unsigned char *static_base() {
  int dev = 0;
  APO_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kStaticMaxDevices)
    throw std::invalid_argument("pme_reciprocal_static: device ordinal out of range");
  unsigned char *b = g_static_base[dev].load(std::memory_order_acquire);
  if (b) return b;
  std::lock_guard<std::mutex> lock(g_static_mu);
  b = g_static_base[dev].load(std::memory_order_relaxed);
  if (!b) {
    void *p = nullptr;
    APO_CUDA(cudaGetSymbolAddress(&p, g_pme_static));
    APO_CUDA(cudaFuncSetAttribute(plane_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kPlaneSmemMax));
    APO_CUDA(cudaFuncSetAttribute(plane_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kPlaneSmemMax));
    b = static_cast<unsigned char *>(p);
    g_static_base[dev].store(b, std::memory_order_release);
  }
  return b;
}

}  // namespace

size_t pme_static_scratch_bytes(int nx, int ny, int nz) { return static_layout(nx, ny, nz).total; }

void pme_reciprocal_static(const float4 *xyzq, int n, double Lx, double Ly, double Lz, int nx,
                           int ny, int nz, int order, double kappa, long long *grad, int stride,
                           double *energy, bool fp64, cudaStream_t s) {
  if (n < 0) throw std::invalid_argument("pme_reciprocal_static: negative atom count");
  if (n > 0 && (xyzq == nullptr || grad == nullptr))
    throw std::invalid_argument("pme_reciprocal_static: coordinate or gradient pointer is NULL");
  if (n > 0 && stride < n) throw std::invalid_argument("pme_reciprocal_static: stride < atom count");
  if (!(Lx > 0.0 && Ly > 0.0 && Lz > 0.0 && kappa > 0.0))
    throw std::invalid_argument("pme_reciprocal_static: box lengths and kappa must be positive");
  if (nx <= 0 || ny <= 0 || nz <= 0 || nx % 2 || ny % 2 || nz % 2 || nx > 256 || ny > 256 ||
      nz > 256)
    throw std::invalid_argument("pme_reciprocal_static: grid dimensions must be even, 2..256");
  if (order != 4 && order != 6 && order != 8)
    throw std::invalid_argument("pme_reciprocal_static: spline order must be 4, 6 or 8");
  if (nx < order || ny < order || nz < order)
    throw std::invalid_argument(
        "pme_reciprocal_static: grid dimensions must be at least the spline order");
  if (plane_smem_bytes(nx, ny) > kPlaneSmemMax)
    throw std::invalid_argument("pme_reciprocal_static: grid plane does not fit in shared memory");
  const StaticLayout l = static_layout(nx, ny, nz);
  if (l.total > kPmeStaticScratchBytes)
    throw std::invalid_argument(
        "pme_reciprocal_static: grid needs more scratch than the static area holds "
        "(8 MiB: about 5.5e5 grid points)");
  PmeDims d{};
  d.nx = nx;
  d.ny = ny;
  d.nz = nz;
  d.nxc = nx / 2 + 1;
  d.nxcp = (d.nxc + 1) & ~1;
  d.order = order;
  d.Lx = (float)Lx;
  d.Ly = (float)Ly;
  d.Lz = (float)Lz;
  d.rLx = 1.0 / Lx;
  d.rLy = 1.0 / Ly;
  d.rLz = 1.0 / Lz;
  d.kappa = (float)kappa;
  if (!fixed_plan_axis(nx, d.ax) || !fixed_plan_axis(ny, d.ay) || !fixed_plan_axis(nz, d.az))
    throw std::invalid_argument("pme_reciprocal_static: grid sizes must factor into 2, 3, 5 and 7");

  unsigned char *b = static_base();
  long long *acc = reinterpret_cast<long long *>(b + l.energy);
  int *counts = reinterpret_cast<int *>(b + l.counts);
  float2 *tw = reinterpret_cast<float2 *>(b + l.tw);
  float *prefac = reinterpret_cast<float *>(b + l.prefac);
  double *prefac_d = reinterpret_cast<double *>(b + l.prefac_d);
  int *qgrid = reinterpret_cast<int *>(b + l.qgrid);
  float2 *cgrid = reinterpret_cast<float2 *>(b + l.cgrid);
  float *phi = reinterpret_cast<float *>(b + l.phi);
  const size_t G = (size_t)nx * ny * nz;

  APO_CUDA(cudaMemsetAsync(acc, 0, kNumEnergyTerms * sizeof(long long), s));
  if (n == 0) {
    if (energy) APO_CUDA(cudaMemsetAsync(energy, 0, sizeof(double), s));
    return;
  }
  APO_CUDA(cudaMemsetAsync(qgrid, 0, G * sizeof(int), s));
  const int n3 = nx + ny + nz;
  static_tables_kernel<<<(n3 + 127) / 128, 128, 0, s>>>(d, tw, prefac, prefac_d, counts, n);
  APO_LAUNCH_CHECK();
  const int blocks = (n + 31) / 32;
  switch (order) {
    case 4: spread_kernel<4><<<blocks, 128, 0, s>>>(xyzq, counts, d, qgrid, nullptr); break;
    case 6: spread_kernel<6><<<blocks, 128, 0, s>>>(xyzq, counts, d, qgrid, nullptr); break;
    case 8: spread_kernel<8><<<blocks, 128, 0, s>>>(xyzq, counts, d, qgrid, nullptr); break;
  }
  APO_LAUNCH_CHECK();
  const size_t sm = plane_smem_bytes(nx, ny);
  plane_fwd_kernel<<<nz, kPlaneThreads, sm, s>>>(d, qgrid, cgrid, tw, tw + nx);
  APO_LAUNCH_CHECK();
  const int pgrid = ((d.nxc + kPencilTX - 1) / kPencilTX) * ny;
  const float2 *twz = tw + nx + ny;
  if (fp64)
    pencil_kernel<true, double><<<pgrid, kPencilThreads, 0, s>>>(d, cgrid, twz, prefac, prefac_d, acc, nullptr, nullptr, nullptr, kNoTensorMap, nullptr);
  else
    pencil_kernel<true, float><<<pgrid, kPencilThreads, 0, s>>>(d, cgrid, twz, prefac, prefac_d, acc, nullptr, nullptr, nullptr, kNoTensorMap, nullptr);
  APO_LAUNCH_CHECK();
  plane_inv_kernel<<<nz, kPlaneThreads, sm, s>>>(d, cgrid, phi, tw, tw + nx);
  APO_LAUNCH_CHECK();
  switch (order) {
    case 4: gather_kernel<4><<<blocks, 256, 0, s>>>(xyzq, counts, d, phi, grad, stride, nullptr); break;
    case 6: gather_kernel<6><<<blocks, 256, 0, s>>>(xyzq, counts, d, phi, grad, stride, nullptr); break;
    case 8: gather_kernel<8><<<blocks, 256, 0, s>>>(xyzq, counts, d, phi, grad, stride, nullptr); break;
  }
  APO_LAUNCH_CHECK();
  if (energy) {
    static_finish_kernel<<<1, 32, 0, s>>>(acc, energy);
    APO_LAUNCH_CHECK();
  }
}

}  // namespace apo
