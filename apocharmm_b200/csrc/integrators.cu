// Integrators; see integrators.h.
#include "integrators.h"

#include <curand_kernel.h>

#include <algorithm>
#include <cstddef>
#include <cmath>
#include <random>
#include <stdexcept>
#include <vector>

#include "device_util.cuh"

namespace apo {

namespace {

constexpr int kThreads = 128;
constexpr int kMaxBlocks = 4096;

// constraint group kinds
enum GroupKind : int { kFree = 0, kSettle = 1, kShake = 2 };

struct Scalars {
  double ke[2];              // [0] average of half/on/half-step KE, [1] on-step KE
  double avgT[2];
  double piston_v, piston_v_prev, piston_f, piston_f_prev, piston_mass;
  double com[4];             // mass-weighted delta sum + total mass
  unsigned long long rngpos;
  long long step;
  long long window;
  unsigned counter;
  unsigned pad;
};

struct SettleConst {
  double wo, wh, ra, rb, rc;
};

// TIP3 geometry and masses of SETTLE (src/CudaHolonomicConstraint.cu:18-33)
SettleConst make_settle() {
  const double mO = 15.99940, mH = 1.00800, mH2O = 18.0154;
  const double rOHsq = 0.91623184, rHHsq = 2.29189321;
  SettleConst s;
  s.wo = mO / mH2O;
  s.wh = mH / mH2O;
  s.ra = s.wh * std::sqrt(4.0 * rOHsq - rHHsq);
  s.rb = s.ra * mO / (2.0 * mH);
  s.rc = std::sqrt(rHHsq) / 2.0;
  return s;
}

// ------------------------------------------------------------ vector math
struct d3 {
  double x, y, z;
};
__device__ __forceinline__ d3 mk(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 operator*(double s, d3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 cross(d3 a, d3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ d3 xyz(double4 v) { return {v.x, v.y, v.z}; }

// Analytic SETTLE (Miyamoto & Kollman, J. Comput. Chem. 13, 952 (1992)):
// moves the unconstrained positions n[0..2] (O, H, H) onto the rigid TIP3
// geometry, keeping the centre of mass, using the constrained positions
// o[0..2] of the previous step to fix the frame.
__device__ void settle(const d3 o[3], d3 n[3], const SettleConst &k) {
  const d3 com = k.wo * n[0] + k.wh * (n[1] + n[2]);
  const d3 a1 = n[0] - com, b1 = n[1] - com, c1 = n[2] - com;
  const d3 b0 = o[1] - o[0], c0 = o[2] - o[0];
  d3 ez = cross(b0, c0);
  d3 ex = cross(a1, ez);
  d3 ey = cross(ez, ex);
  ex = (1.0 / sqrt(dot(ex, ex))) * ex;
  ey = (1.0 / sqrt(dot(ey, ey))) * ey;
  ez = (1.0 / sqrt(dot(ez, ez))) * ez;
  const double xb0 = dot(ex, b0), yb0 = dot(ey, b0), xc0 = dot(ex, c0), yc0 = dot(ey, c0);
  const double za1 = dot(ez, a1);
  const double xb1 = dot(ex, b1), yb1 = dot(ey, b1), zb1 = dot(ez, b1);
  const double xc1 = dot(ex, c1), yc1 = dot(ey, c1), zc1 = dot(ez, c1);
  const double sinphi = za1 / k.ra;
  const double cosphi = sqrt(fmax(0.0, 1.0 - sinphi * sinphi));
  const double sinpsi = (zb1 - zc1) / (2.0 * k.rc * cosphi);
  const double cospsi = sqrt(fmax(0.0, 1.0 - sinpsi * sinpsi));
  const double ya2 = k.ra * cosphi;
  const double xb2 = -k.rc * cospsi;
  const double yb2 = -k.rb * cosphi - k.rc * sinpsi * sinphi;
  const double yc2 = -k.rb * cosphi + k.rc * sinpsi * sinphi;
  const double alpha = xb2 * (xb0 - xc0) + yb0 * yb2 + yc0 * yc2;
  const double beta = xb2 * (yc0 - yb0) + xb0 * yb2 + xc0 * yc2;
  const double gamma = xb0 * yb1 - xb1 * yb0 + xc0 * yc1 - xc1 * yc0;
  const double ab2 = alpha * alpha + beta * beta;
  const double sinth = (alpha * gamma - beta * sqrt(fmax(0.0, ab2 - gamma * gamma))) / ab2;
  const double costh = sqrt(fmax(0.0, 1.0 - sinth * sinth));
  const d3 a3 = mk(-ya2 * sinth, ya2 * costh, za1);
  const d3 b3 = mk(xb2 * costh - yb2 * sinth, xb2 * sinth + yb2 * costh, zb1);
  const d3 c3 = mk(-xb2 * costh - yc2 * sinth, -xb2 * sinth + yc2 * costh, zc1);
  n[0] = com + a3.x * ex + a3.y * ey + a3.z * ez;
  n[1] = com + b3.x * ex + b3.y * ey + b3.z * ez;
  n[2] = com + c3.x * ex + c3.y * ey + c3.z * ez;
}

// SHAKE for an X-H_m cluster (m = 1..3): exact for one bond, otherwise the
// iterative bond-by-bond scheme of Ryckaert, Ciccotti & Berendsen (1977) to a
// relative tolerance of 1e-10 (at most 200 sweeps).  o = reference
// (constrained) positions, n = positions to correct.
__device__ void shake(const d3 *o, d3 *n, int m, float4 p) {
  const double ic = p.x, ih = p.w, b2 = p.z;
  if (m == 1) {
    const d3 r = o[0] - o[1], q = n[0] - n[1];
    const double rr = dot(r, r), rq = dot(r, q), qq = dot(q, q);
    const double lam = (-rq + sqrt(fmax(0.0, rq * rq + rr * (b2 - qq)))) / (rr * (ic + ih));
    n[0] = n[0] + (ic * lam) * r;
    n[1] = n[1] - (ih * lam) * r;
    return;
  }
  for (int it = 0; it < 200; ++it) {
    bool done = true;
    for (int h = 1; h <= m; ++h) {
      const d3 q = n[0] - n[h];
      const double diff = b2 - dot(q, q);
      if (fabs(diff) > 2e-10 * b2) {
        done = false;
        const d3 r = o[0] - o[h];
        const double g = diff / (2.0 * dot(r, q) * (ic + ih));
        n[0] = n[0] + (ic * g) * r;
        n[h] = n[h] - (ih * g) * r;
      }
    }
    if (done) break;
  }
}

__device__ __forceinline__ void apply_constraint(int kind, int m, const d3 *o, d3 *n,
                                                 const SettleConst &sk, const float4 *shake_p,
                                                 int pidx) {
  if (kind == kSettle) settle(o, n, sk);
  else if (kind == kShake) shake(o, n, m - 1, shake_p[pidx]);
}

// gradient of an atom from the fixed-point slot buffer; the slot is cleared
// for the next force evaluation
__device__ __forceinline__ d3 take_grad(long long *f, int stride, int slot) {
  const long long gx = f[slot], gy = f[stride + slot], gz = f[2 * stride + slot];
  f[slot] = 0;
  f[stride + slot] = 0;
  f[2 * stride + slot] = 0;
  return mk((double)gx * kInvForceScale, (double)gy * kInvForceScale,
            (double)gz * kInvForceScale);
}

// new FP64 position -> state, atom-order floats, and the sorted
// cluster-local floats (position + image shift - cluster origin, in FP64)
__device__ __forceinline__ void store_position(int a, d3 x, double4 *coords, float4 *xyzq,
                                               const int *glo2loc, const double4 *slot_off,
                                               float4 *xyzq_s) {
  const double q = coords[a].w;
  coords[a] = make_double4(x.x, x.y, x.z, q);
  xyzq[a] = make_float4((float)x.x, (float)x.y, (float)x.z, (float)q);
  const int s = glo2loc[a];
  const double4 o = slot_off[s];
  xyzq_s[s] = make_float4((float)(x.x + o.x), (float)(x.y + o.y), (float)(x.z + o.z), (float)q);
}

// block-wide sum of two doubles; thread 0 writes partials[2*block + k]
__device__ void block_partials(double a, double b, double *partials) {
  __shared__ double sh[2][kThreads / 32];
  a = warp_sum(a);
  b = warp_sum(b);
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = a;
    sh[1][threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0, s1 = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      s0 += sh[0][w];
      s1 += sh[1][w];
    }
    partials[2 * blockIdx.x] = s0;
    partials[2 * blockIdx.x + 1] = s1;
  }
}

// true in the block that finishes last; partials of all blocks are visible
__device__ bool is_last_block(unsigned *counter) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  return last;
}

// sum of the partials in a fixed order (same result for every run)
__device__ void sum_partials(const double *partials, double &s0, double &s1) {
  double a = 0, b = 0;
  if (threadIdx.x < 32) {
    for (int k = threadIdx.x; k < (int)gridDim.x; k += 32) {
      a += partials[2 * k];
      b += partials[2 * k + 1];
    }
    a = warp_sum(a);
    b = warp_sum(b);
  }
  s0 = a;
  s1 = b;
}

struct Common {
  // several systems: atom -> system, first atom of every system, and every
  // system's noise seed (null for one system)
  const int *sys_of_atom;
  const int *atom_off;
  const unsigned long long *sys_seed;
  // several systems: noise position of every system when this integrator
  // started, and the number of steps each system may take from then on
  // (groups of a system past its limit are left as they are); null = none
  const unsigned long long *sys_rng0;
  const long long *sys_stop;
  int ngroups;
  const int4 *groups;   // atoms (-1 unused)
  const int2 *gmeta;    // (kind, shake parameter index)
  const float4 *shake_p;
  double4 *coords, *vel, *dprev, *delta, *dpred, *ref;
  float4 *xyzq;
  long long *force;
  int stride;
  const int *glo2loc;
  const double4 *slot_off;
  float4 *xyzq_s;
  Scalars *sc;
  double *partials;
  // the neighbour list's error word: once a list build has overflowed or
  // met non-finite coordinates, every step kernel leaves the state as it is
  const unsigned *err;
  SettleConst sk;
  int ndegf;
  double dt;
};

__device__ __forceinline__ int group_atoms(const Common &c, int g, int (&at)[4]) {
  const int4 a = c.groups[g];
  at[0] = a.x;
  at[1] = a.y;
  at[2] = a.z;
  at[3] = a.w;
  return 1 + (a.y >= 0) + (a.z >= 0) + (a.w >= 0);
}

__device__ void finish_temperature(const Common &c, double ke0, double ke1) {
  c.sc->ke[0] = ke0;
  c.sc->ke[1] = ke1;
  const double s = (double)(c.sc->window + 1);
  for (int k = 0; k < 2; ++k) {
    const double t = (k ? ke1 : ke0) / (0.5 * c.ndegf * kBoltz);
    c.sc->avgT[k] += (t - c.sc->avgT[k]) / s;
  }
  c.sc->window += 1;
}

// ------------------------------------------------------------ Langevin step
// Position-Verlet "delta" Langevin of src/CudaLangevinThermostatIntegrator.cu:576-640:
//   delta = alpha*delta_prev - dt^2/m/(1+g/2) * (grad + sqrt(2 g kT m)/dt * xi)
//   x += delta; constrain; delta = x - x_old;
//   v = sqrt(1+g/2)/(2 dt) * (delta + delta_prev)
// Four lanes per constraint group (a water, an X-H cluster, a run of free
// atoms): each lane loads, draws the noise for and moves one atom, the
// lanes exchange the group's old and new positions by shuffles and each
// applies the group's constraint to the whole group (the same arithmetic,
// in the same order, as one thread per group), then keeps and stores its own
// atom.  Four times the threads of one per group: the step is bound by the
// latency of its dependent loads and arithmetic, not by throughput.
__device__ __forceinline__ d3 pick(const d3 (&v)[4], int k) {
  return k == 0 ? v[0] : (k == 1 ? v[1] : (k == 2 ? v[2] : v[3]));
}

__global__ void __launch_bounds__(kThreads) langevin_kernel(Common c, double gamma, double kbt,
                                                            unsigned long long seed) {
  // the error word is the same for every block; it is looked at before the
  // first store, after the loads are under way
  const unsigned err = *c.err;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int g = t >> 2, k = t & 3;
  const int base = (threadIdx.x & 31) & ~3;
  const double dt = c.dt, dt2 = dt * dt;
  const double hg = 0.5 * gamma, denom = 1.0 / (1.0 + hg), alpha = (1.0 - hg) * denom;
  const double vfac = 0.5 * sqrt(1.0 + hg) / dt, idt = 1.0 / dt;
  double ke0 = 0.0, ke1 = 0.0;
  const unsigned long long pos = c.sc->rngpos;
  const bool gvalid = g < c.ngroups;
  int at[4] = {0, 0, 0, 0};
  int m = 0;
  int2 meta = make_int2(0, 0);
  if (gvalid) {
    m = group_atoms(c, g, at);
    meta = c.gmeta[g];
  }
  const bool mine = gvalid && k < m;
  const int a = k == 0 ? at[0] : (k == 1 ? at[1] : (k == 2 ? at[2] : at[3]));
  bool run = gvalid;
  if (run && c.sys_stop && c.sc->step >= c.sys_stop[c.sys_of_atom[at[0]]])
    run = false;  // a system past its step limit: its gradient slots are consumed all the same
  double4 x = make_double4(0.0, 0.0, 0.0, 0.0), vm = x, dpv = x, so = x;
  int slot = 0;
  if (mine) {
    x = c.coords[a];
    vm = c.vel[a];
    dpv = c.dprev[a];
    slot = c.glo2loc[a];
  }
  long long gi0 = 0, gi1 = 0, gi2 = 0;
  if (mine) {
    gi0 = c.force[slot];
    gi1 = c.force[c.stride + slot];
    gi2 = c.force[2 * c.stride + slot];
    so = c.slot_off[slot];
  }
  if (err) return;
  const d3 o = xyz(x), dp = xyz(dpv);
  const double im = vm.w;
  d3 n = o;
  if (mine) {  // cleared for the next force evaluation
    c.force[slot] = 0;
    c.force[c.stride + slot] = 0;
    c.force[2 * c.stride + slot] = 0;
    if (run) {
      const d3 gr = mk((double)gi0 * kInvForceScale, (double)gi1 * kInvForceScale,
                       (double)gi2 * kInvForceScale);
      curandStatePhilox4_32_10_t st;
      unsigned long long p = pos;
      if (c.sys_seed) {  // a system's own stream, the same alone or among others
        const int sy = c.sys_of_atom[a];
        curand_init(seed ^ c.sys_seed[sy], (unsigned long long)(a - c.atom_off[sy]), 0ull, &st);
        if (c.sys_rng0) p += c.sys_rng0[sy];
      } else {
        curand_init(seed, (unsigned long long)a, 0ull, &st);
      }
      skipahead(p, &st);
      const float4 rn = curand_normal4(&st);
      const double rdf = sqrt(2.0 * gamma * kbt / im) / dt;
      const double fact = dt2 * im * denom;
      const d3 f = gr + rdf * mk(rn.x, rn.y, rn.z);
      n = o + (alpha * dp - fact * f);
    }
  }
  // the group's old and new positions in every lane of the group
  d3 og[4], ng[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    og[q] = mk(__shfl_sync(0xffffffffu, o.x, base + q), __shfl_sync(0xffffffffu, o.y, base + q),
               __shfl_sync(0xffffffffu, o.z, base + q));
    ng[q] = mk(__shfl_sync(0xffffffffu, n.x, base + q), __shfl_sync(0xffffffffu, n.y, base + q),
               __shfl_sync(0xffffffffu, n.z, base + q));
  }
  if (run) apply_constraint(meta.x, m, og, ng, c.sk, c.shake_p, meta.y);
  if (mine && run) {
    const d3 nk = pick(ng, k);
    const d3 d = nk - o;
    const d3 v = vfac * (d + dp);
    const double mass = 1.0 / im;
    const d3 u1 = idt * dp, u2 = idt * d;
    const double kon = 0.5 * mass * dot(v, v);
    ke0 = (0.5 * mass * dot(u1, u1) + kon + 0.5 * mass * dot(u2, u2)) / 3.0;
    ke1 = kon;
    c.vel[a] = make_double4(v.x, v.y, v.z, im);
    c.dprev[a] = make_double4(d.x, d.y, d.z, 0.0);
    c.coords[a] = make_double4(nk.x, nk.y, nk.z, x.w);
    c.xyzq[a] = make_float4((float)nk.x, (float)nk.y, (float)nk.z, (float)x.w);
    c.xyzq_s[slot] = make_float4((float)(nk.x + so.x), (float)(nk.y + so.y),
                                 (float)(nk.z + so.z), (float)x.w);
  }
  block_partials(ke0, ke1, c.partials);
  if (is_last_block(&c.sc->counter)) {
    double s0, s1;
    sum_partials(c.partials, s0, s1);
    if (threadIdx.x == 0) {
      finish_temperature(c, s0, s1);
      c.sc->rngpos += 4;  // curand_normal4 consumes four values per step
      c.sc->step += 1;
      c.sc->counter = 0;
    }
  }
}

// -------------------------------------------------------- Nose-Hoover step
// src/CudaNoseHooverIntegrator.cu:647-1004, split at the grid-wide
// kinetic-energy reductions:
//   K0 half step + constraint + KE(v_old) + piston update
//   K1..K3 predictor-corrector (K1, K2 also KE + piston)
//   K4 constraint + on-step velocity + KE + piston + average temperature
__device__ void piston_update(Scalars *sc, double ke_sel, double ke_ref, double dt) {
  sc->piston_f = 2.0 * dt * (ke_sel - ke_ref) / sc->piston_mass;
  if (sc->piston_f_prev == 0.0) sc->piston_f_prev = sc->piston_f;
  sc->piston_v = sc->piston_v_prev + 0.5 * (sc->piston_f + sc->piston_f_prev);
}

__global__ void __launch_bounds__(kThreads) nh_half_kernel(Common c, double ke_ref, int use_old) {
  if (*c.err) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const double dt = c.dt, dt2 = dt * dt, idt = 1.0 / dt;
  double ke0 = 0, ke1 = 0;
  if (g < c.ngroups) {
    int at[4];
    const int m = group_atoms(c, g, at);
    const int2 meta = c.gmeta[g];
    // every load of the group first (each level of the chain atom -> slot ->
    // gradient for all atoms at once), then the arithmetic, then the stores:
    // at a million atoms the kernel is bound by memory latency
    double4 x[4], vm[4], dp[4];
    int slot[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k < m) {
        const int a = at[k];
        x[k] = c.coords[a];
        vm[k] = c.vel[a];
        dp[k] = c.dprev[a];
        slot[k] = c.glo2loc[a];
      }
    }
    long long gi[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k < m) {
        gi[k][0] = c.force[slot[k]];
        gi[k][1] = c.force[c.stride + slot[k]];
        gi[k][2] = c.force[2 * c.stride + slot[k]];
      }
    }
    d3 o[4], n[4], n0[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k < m) {  // the slots are cleared for the next force evaluation
        c.force[slot[k]] = 0;
        c.force[c.stride + slot[k]] = 0;
        c.force[2 * c.stride + slot[k]] = 0;
        const d3 gr = mk((double)gi[k][0] * kInvForceScale, (double)gi[k][1] * kInvForceScale,
                         (double)gi[k][2] * kInvForceScale);
        o[k] = xyz(x[k]);
        n[k] = o[k] + (xyz(dp[k]) - (dt2 * vm[k].w) * gr);
        n0[k] = n[k];
      }
    }
    apply_constraint(meta.x, m, o, n, c.sk, c.shake_p, meta.y);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k < m) {
        const int a = at[k];
        const d3 d = n[k] - o[k];
        c.ref[a] = x[k];
        c.delta[a] = make_double4(d.x, d.y, d.z, 0.0);
        c.dpred[a] = make_double4(d.x, d.y, d.z, 0.0);
        c.coords[a] = make_double4(n[k].x, n[k].y, n[k].z, x[k].w);
        const double mass = 1.0 / vm[k].w;
        // the on-step velocity of the first predictor-corrector pass carries
        // the constraint's displacement over dt, as the reference's constraint
        // pass adds it to the velocities (src/CudaHolonomicConstraint.cu:94-106,
        // src/CudaNoseHooverIntegrator.cu:905-930)
        const d3 v = xyz(vm[k]) + idt * (n[k] - n0[k]);
        const d3 u1 = idt * xyz(dp[k]), u2 = idt * d;
        const double kon = 0.5 * mass * dot(v, v);
        ke0 += (0.5 * mass * dot(u1, u1) + kon + 0.5 * mass * dot(u2, u2)) / 3.0;
        ke1 += kon;
      }
    }
  }
  block_partials(ke0, ke1, c.partials);
  if (is_last_block(&c.sc->counter)) {
    double s0, s1;
    sum_partials(c.partials, s0, s1);
    if (threadIdx.x == 0) {
      c.sc->piston_v_prev = c.sc->piston_v;
      c.sc->piston_f_prev = c.sc->piston_f;
      piston_update(c.sc, use_old ? s1 : s0, ke_ref, dt);
      c.sc->counter = 0;
    }
  }
}

// predictor-corrector pass over atoms; with KE also the next piston update
template <bool KE>
__global__ void __launch_bounds__(kThreads) nh_pc_kernel(Common c, int natom, double ke_ref,
                                                         int use_old) {
  if (*c.err) return;
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const double dt = c.dt, idt = 1.0 / dt, fact = 0.5 / dt;
  const double xi = c.sc->piston_v;
  double ke0 = 0, ke1 = 0;
  if (a < natom) {
    const d3 dprev = xyz(c.dprev[a]), dpred = xyz(c.dpred[a]), d = xyz(c.delta[a]);
    const d3 v = fact * (dprev + dpred);
    const d3 np = d - (dt * dt * xi) * v;
    c.dpred[a] = make_double4(np.x, np.y, np.z, 0.0);
    c.vel[a] = make_double4(v.x, v.y, v.z, c.vel[a].w);
    const d3 r = xyz(c.ref[a]);
    c.coords[a] = make_double4(r.x + np.x, r.y + np.y, r.z + np.z, c.coords[a].w);
    if (KE) {
      const double mass = 1.0 / c.vel[a].w;
      const d3 u1 = idt * dprev, u2 = idt * d;
      const double kon = 0.5 * mass * dot(v, v);
      ke0 = (0.5 * mass * dot(u1, u1) + kon + 0.5 * mass * dot(u2, u2)) / 3.0;
      ke1 = kon;
    }
  }
  if (KE) {
    block_partials(ke0, ke1, c.partials);
    if (is_last_block(&c.sc->counter)) {
      double s0, s1;
      sum_partials(c.partials, s0, s1);
      if (threadIdx.x == 0) {
        piston_update(c.sc, use_old ? s1 : s0, ke_ref, dt);
        c.sc->counter = 0;
      }
    }
  }
}

__global__ void __launch_bounds__(kThreads) nh_final_kernel(Common c, double ke_ref, int use_old) {
  if (*c.err) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const double dt = c.dt, idt = 1.0 / dt, fact = 0.5 / dt;
  double ke0 = 0, ke1 = 0;
  if (g < c.ngroups) {
    int at[4];
    const int m = group_atoms(c, g, at);
    const int2 meta = c.gmeta[g];
    // loads first (as nh_half_kernel), then the constraint, then the stores
    d3 o[4], n[4], dp[4];
    double q[4], im[4];
    int slot[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k < m) {
        const int a = at[k];
        o[k] = xyz(c.ref[a]);
        const double4 x = c.coords[a];
        n[k] = xyz(x);
        q[k] = x.w;
        dp[k] = xyz(c.dprev[a]);
        im[k] = c.vel[a].w;
        slot[k] = c.glo2loc[a];
      }
    }
    double4 so[4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k < m) so[k] = c.slot_off[slot[k]];
    apply_constraint(meta.x, m, o, n, c.sk, c.shake_p, meta.y);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k < m) {
        const int a = at[k];
        const d3 d = n[k] - o[k];
        const d3 v = fact * (d + dp[k]);
        const double mass = 1.0 / im[k];
        const d3 u1 = idt * dp[k], u2 = idt * d;
        const double kon = 0.5 * mass * dot(v, v);
        ke0 += (0.5 * mass * dot(u1, u1) + kon + 0.5 * mass * dot(u2, u2)) / 3.0;
        ke1 += kon;
        c.vel[a] = make_double4(v.x, v.y, v.z, im[k]);
        c.dprev[a] = make_double4(d.x, d.y, d.z, 0.0);
        c.coords[a] = make_double4(n[k].x, n[k].y, n[k].z, q[k]);
        c.xyzq[a] = make_float4((float)n[k].x, (float)n[k].y, (float)n[k].z, (float)q[k]);
        c.xyzq_s[slot[k]] = make_float4((float)(n[k].x + so[k].x), (float)(n[k].y + so[k].y),
                                        (float)(n[k].z + so[k].z), (float)q[k]);
      }
    }
  }
  block_partials(ke0, ke1, c.partials);
  if (is_last_block(&c.sc->counter)) {
    double s0, s1;
    sum_partials(c.partials, s0, s1);
    if (threadIdx.x == 0) {
      piston_update(c.sc, use_old ? s1 : s0, ke_ref, dt);
      finish_temperature(c, s0, s1);
      c.sc->step += 1;
      c.sc->counter = 0;
    }
  }
}

// ---------------------------------------------------------------- leapfrog
// v -= dt grad/m; x += dt v (src/CudaLeapFrogIntegrator.cu:22-41).  The
// reference advances only the single-precision copy; here the FP64 state is
// advanced and the single-precision copies are refreshed from it.
__global__ void leapfrog_kernel(Common c, int natom) {
  if (*c.err) return;
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  double ke1 = 0;
  if (a < natom) {
    const d3 gr = take_grad(c.force, c.stride, c.glo2loc[a]);
    double4 v = c.vel[a];
    const d3 nv = xyz(v) - (c.dt * v.w) * gr;
    c.vel[a] = make_double4(nv.x, nv.y, nv.z, v.w);
    const d3 x = xyz(c.coords[a]) + c.dt * nv;
    store_position(a, x, c.coords, c.xyzq, c.glo2loc, c.slot_off, c.xyzq_s);
    ke1 = 0.5 * dot(nv, nv) / v.w;
  }
  block_partials(ke1, ke1, c.partials);
  if (is_last_block(&c.sc->counter)) {
    double s0, s1;
    sum_partials(c.partials, s0, s1);
    if (threadIdx.x == 0) {
      finish_temperature(c, s0, s1);
      c.sc->step += 1;
      c.sc->counter = 0;
    }
  }
}

// ----------------------------------------------------- initialisation / COM
// delta and delta_prev from velocities and the first forces
// (src/CudaLangevinThermostatIntegrator.cu:138-165)
__global__ void init_delta_kernel(Common c, int natom, double gamma) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natom) return;
  const double dt = c.dt, hg = 0.5 * gamma;
  const double a0 = dt * sqrt(1.0 + hg), a1 = dt * (1.0 - hg) / sqrt(1.0 + hg);
  const d3 gr = take_grad(c.force, c.stride, c.glo2loc[a]);
  const double4 v = c.vel[a];
  const double fact = 0.5 * dt * dt * v.w;
  const d3 d = a0 * xyz(v) - fact * gr;
  const d3 dp = a1 * xyz(v) + fact * gr;
  c.delta[a] = make_double4(d.x, d.y, d.z, 0.0);
  c.dprev[a] = make_double4(dp.x, dp.y, dp.z, 0.0);
}

// mode 0: constrain the current positions against themselves (projection
// onto the constraint surface); mode 1: back step x - delta_prev, constrain
// against x, then delta_prev = x - x_constrained.  As the reference's
// handleHolonomicConstraints (src/CudaHolonomicConstraint.cu:94-106), every
// constraint pass also adds its displacement over dt to the velocities; in
// mode 0 that correction reaches the initial position-Verlet delta.
__global__ void init_constrain_kernel(Common c, int mode) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= c.ngroups) return;
  int at[4];
  const int m = group_atoms(c, g, at);
  const int2 meta = c.gmeta[g];
  d3 o[4], n[4], n0[4];
  for (int k = 0; k < m; ++k) {
    o[k] = xyz(c.coords[at[k]]);
    n[k] = mode == 0 ? o[k] : o[k] - xyz(c.dprev[at[k]]);
    n0[k] = n[k];
  }
  apply_constraint(meta.x, m, o, n, c.sk, c.shake_p, meta.y);
  const double idt = 1.0 / c.dt;
  for (int k = 0; k < m; ++k) {
    const int a = at[k];
    const double4 v = c.vel[a];
    const d3 dv = idt * (n[k] - n0[k]);
    c.vel[a] = make_double4(v.x + dv.x, v.y + dv.y, v.z + dv.z, v.w);
    if (mode == 0) {
      store_position(a, n[k], c.coords, c.xyzq, c.glo2loc, c.slot_off, c.xyzq_s);
    } else {
      const d3 d = o[k] - n[k];
      c.dprev[a] = make_double4(d.x, d.y, d.z, 0.0);
    }
  }
}

// centre-of-mass motion removal from delta_prev, every `freq` steps
// (src/CudaLangevinThermostatIntegrator.cu:832-875), gated on the device
// step counter so the same graph serves every segment
__global__ void com_sum_kernel(Common c, int natom, int freq) {
  if (*c.err || c.sc->step % freq != 0) return;
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  __shared__ double sh[4][kThreads / 32];
  double v[4] = {0, 0, 0, 0};
  if (a < natom) {
    const double mass = 1.0 / c.vel[a].w;
    const double4 d = c.dprev[a];
    v[0] = d.x * mass;
    v[1] = d.y * mass;
    v[2] = d.z * mass;
    v[3] = mass;
  }
  for (int k = 0; k < 4; ++k) {
    const double s = warp_sum(v[k]);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = s;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double s = 0;
    for (int w = 0; w < kThreads / 32; ++w) s += sh[threadIdx.x][w];
    c.partials[4 * blockIdx.x + threadIdx.x] = s;
  }
  if (is_last_block(&c.sc->counter)) {
    if (threadIdx.x < 4) {
      double s = 0;
      for (int b = 0; b < (int)gridDim.x; ++b) s += c.partials[4 * b + threadIdx.x];
      c.sc->com[threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) c.sc->counter = 0;
  }
}

__global__ void com_apply_kernel(Common c, int natom, int freq) {
  if (*c.err || c.sc->step % freq != 0) return;
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natom) return;
  const double im = 1.0 / c.sc->com[3];
  double4 d = c.dprev[a];
  d.x -= c.sc->com[0] * im;
  d.y -= c.sc->com[1] * im;
  d.z -= c.sc->com[2] * im;
  c.dprev[a] = d;
}

// --------------------------------------------------------- Langevin piston
// src/CudaLangevinPistonIntegrator.cu:1705-2060 in three kinds of launch:
//   lp_half   half step, constraint, constraint forces and virial, the
//             pressure tensor and its static part; last block: the first
//             pass's piston move (one normal per piston degree of freedom)
//             and thermostat update from its kinetic energy
//   lp_pc     (per pass) atoms follow piston and thermostat; last block:
//             the pressure difference with the new half-step kinetic term,
//             then the next pass's piston move and thermostat update
//   lp_final  constraints on the new and the scaled reference positions,
//             on-step velocities, kinetic energy, pressure averages, the box
constexpr double kAtmosp = 1.4584007e-05;           // atm in AKMA pressure units
constexpr double kPatmos = 1.0 / kAtmosp;
constexpr double kSurfaceTensionFactor = 98.6923;   // dyne/cm to atm A

}  // namespace

struct PistonScalars {
  double box[3], box_pred[3];
  double vir[9];                 // internal virial of the step with the constraint part
  double pref[9], dp[9], dp_static[9];
  double p[9], pavg[9];
  double pscalar, pavg_scalar;
  double lp_delta[3], lp_delta_pred[3], lp_delta_prev[3];
  double lp_onpos[3], lp_halfpos[3], lp_onvel[3], lp_dpress[3];
  double cf_on[3], cf_half[3];
  double box_old[3];             // the box before the last step (for the list's shifts)
  double vfac, lp_vfac;          // patm / V and V pbfact atmosp of the step's box
  unsigned long long rngpos;     // normals drawn per piston degree of freedom
  unsigned counter, pad;
};

namespace {

struct PistonArgs {
  PistonScalars *ps;
  curandStatePhilox4_32_10_t *rng;
  double *partials;
  const long long *vir_fixed;    // the force manager's virial slots
  NbSetup *setup;                // the force manager's direct-space set-up
  NbSysDims *lsys;               // the list's dims
  double4 *dbox;                 // the force manager's device box
  double inv_mass[3], prfwd[3];
  double palpha, pbfact;
  double st;                     // surface tension x dyne/cm factor
  double ke_ref;
  int crystal, dof, use_nh, use_old, const_st, hol;
};

template <int N>
__device__ void block_partials_n(const double (&v)[N], double *partials) {
  __shared__ double sh[N][kThreads / 32];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const double s = warp_sum(v[k]);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = s;
  }
  __syncthreads();
  if (threadIdx.x < N) {
    double s = 0;
    for (int w = 0; w < kThreads / 32; ++w) s += sh[threadIdx.x][w];
    partials[N * blockIdx.x + threadIdx.x] = s;
  }
}

// totals of the N partials of every block, in block order, into tot[]
template <int N>
__device__ void sum_partials_n(const double *partials, double *tot) {
  if (threadIdx.x < N) {
    double s = 0;
    for (int b = 0; b < (int)gridDim.x; ++b) s += partials[N * b + threadIdx.x];
    tot[threadIdx.x] = s;
  }
  __syncthreads();
}

// piston move of one predictor-corrector pass (one thread)
// (UpdateLangevinPistonKernel, src/CudaLangevinPistonIntegrator.cu:1297-1452)
__device__ void lp_move(const PistonArgs &a, double dt) {
  PistonScalars *ps = a.ps;
  double *b = ps->box_pred;
  const double *dP = ps->dp;
  const Crystal cr = (Crystal)a.crystal;
  if (cr == Crystal::Cubic) {
    ps->lp_dpress[0] = (dP[0] + dP[4] + dP[8]) / b[0];
  } else if (cr == Crystal::Tetragonal) {
    ps->lp_dpress[0] = (dP[0] + dP[4]) / b[0];
    ps->lp_dpress[1] = dP[8] / b[2];
  } else {
    ps->lp_dpress[0] = dP[0] / b[0];
    ps->lp_dpress[1] = dP[4] / b[1];
    ps->lp_dpress[2] = dP[8] / b[2];
  }
  for (int i = 0; i < a.dof; ++i) {
    curandStatePhilox4_32_10_t st = a.rng[i];
    ps->lp_delta_prev[i] = ps->lp_delta_pred[i];
    ps->lp_delta_pred[i] = a.palpha * ps->lp_delta_pred[i] +
                           a.inv_mass[i] * ps->lp_dpress[i] * ps->lp_vfac +
                           a.pbfact * a.prfwd[i] * curand_normal_double(&st);
    ps->lp_onvel[i] = 0.5 * (ps->lp_delta_pred[i] + ps->lp_delta_prev[i]) / dt;
    a.rng[i] = st;
  }
  ps->rngpos += 1;
  if (cr == Crystal::Cubic) {
    ps->lp_onpos[0] = (b[0] + b[1] + b[2]) / 3.0;
  } else if (cr == Crystal::Tetragonal) {
    ps->lp_onpos[0] = (b[0] + b[1]) / 2.0;
    ps->lp_onpos[1] = b[2];
  } else {
    ps->lp_onpos[0] = b[0];
    ps->lp_onpos[1] = b[1];
    ps->lp_onpos[2] = b[2];
  }
  for (int i = 0; i < a.dof; ++i) {
    ps->lp_onpos[i] += ps->lp_delta_pred[i];
    ps->lp_halfpos[i] = ps->lp_onpos[i] - 0.5 * ps->lp_delta_pred[i];
  }
  // scaling factors of the edges (on-step: piston velocity over the edge;
  // half-step: displacement over the half-step edge), then the new edges
  double *on = ps->cf_on, *hf = ps->cf_half;
  const double *dl = ps->lp_delta_pred, *hp = ps->lp_halfpos, *op = ps->lp_onpos,
               *ov = ps->lp_onvel;
  if (cr == Crystal::Cubic) {
    on[0] = on[1] = on[2] = dt * ov[0] / b[0];
    hf[0] = hf[1] = hf[2] = dl[0] / hp[0];
    b[0] = b[1] = b[2] = op[0];
  } else if (cr == Crystal::Tetragonal) {
    on[0] = on[1] = dt * ov[0] / b[0];
    on[2] = dt * ov[1] / b[2];
    hf[0] = hf[1] = dl[0] / hp[0];
    hf[2] = dl[1] / hp[1];
    b[0] = b[1] = op[0];
    b[2] = op[1];
  } else {
    for (int d = 0; d < 3; ++d) {
      on[d] = dt * ov[d] / b[d];
      hf[d] = dl[d] / hp[d];
      b[d] = op[d];
    }
  }
}

// start of a predictor-corrector pass (one thread): the piston moves from
// the step's box and displacement with the current pressure difference, the
// thermostat from the kinetic energy (ke0 three-term, ke1 on-step)
__device__ void lp_pass_start(const Common &c, const PistonArgs &a, double ke0, double ke1,
                              double dt) {
  PistonScalars *ps = a.ps;
  for (int d = 0; d < 3; ++d) {
    ps->box_pred[d] = ps->box[d];
    ps->lp_delta_pred[d] = ps->lp_delta[d];
  }
  lp_move(a, dt);
  piston_update(c.sc, a.use_old ? ke1 : ke0, a.ke_ref, dt);
}

__global__ void __launch_bounds__(kThreads) lp_half_kernel(Common c, PistonArgs a) {
  if (*c.err) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const double dt = c.dt, dt2 = dt * dt, idt = 1.0 / dt;
  // [0..8] constraint virial, [9..17] sum d d m/dt^2 of the new half step,
  // [18..26] the same of the previous half step, [27..28] the kinetic
  // energy of the first predictor-corrector pass
  double v[29];
#pragma unroll
  for (int k = 0; k < 29; ++k) v[k] = 0.0;
  if (g < c.ngroups) {
    int at[4];
    const int m = group_atoms(c, g, at);
    const int2 meta = c.gmeta[g];
    double4 x[4], vm[4], dp[4];
    int slot[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k < m) {
        const int i = at[k];
        x[k] = c.coords[i];
        vm[k] = c.vel[i];
        dp[k] = c.dprev[i];
        slot[k] = c.glo2loc[i];
      }
    }
    d3 o[4], n[4], n0[4], du[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k < m) {
        const d3 gr = mk((double)c.force[slot[k]] * kInvForceScale,
                         (double)c.force[c.stride + slot[k]] * kInvForceScale,
                         (double)c.force[2 * c.stride + slot[k]] * kInvForceScale);
        o[k] = xyz(x[k]);
        du[k] = xyz(dp[k]) - (dt2 * vm[k].w) * gr;
        n[k] = o[k] + du[k];
        n0[k] = n[k];
      }
    }
    if (a.hol) apply_constraint(meta.x, m, o, n, c.sk, c.shake_p, meta.y);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k < m) {
        const int i = at[k];
        const double f = 1.0 / (dt2 * vm[k].w);
        d3 d = du[k];
        if (a.hol) {
          // constraint force m (x_constrained - x_free) / dt^2 and its virial
          // (ComputeHolonomicConstraintForces/VirialKernel)
          const d3 fc = mk(f * (n[k].x - o[k].x - du[k].x), f * (n[k].y - o[k].y - du[k].y),
                           f * (n[k].z - o[k].z - du[k].z));
          const double r[3] = {o[k].x, o[k].y, o[k].z}, q[3] = {fc.x, fc.y, fc.z};
#pragma unroll
          for (int u = 0; u < 3; ++u)
#pragma unroll
            for (int w = 0; w < 3; ++w) v[3 * u + w] += r[u] * q[w];
          d = n[k] - o[k];
        }
        const double dd[3] = {d.x, d.y, d.z}, pp[3] = {dp[k].x, dp[k].y, dp[k].z};
#pragma unroll
        for (int u = 0; u < 3; ++u)
#pragma unroll
          for (int w = 0; w < 3; ++w) {
            v[9 + 3 * u + w] += f * dd[u] * dd[w];
            v[18 + 3 * u + w] += f * pp[u] * pp[w];
          }
        c.ref[i] = x[k];
        c.delta[i] = make_double4(d.x, d.y, d.z, 0.0);
        c.dpred[i] = make_double4(d.x, d.y, d.z, 0.0);
        const d3 xn = o[k] + d;
        c.coords[i] = make_double4(a.hol ? n[k].x : xn.x, a.hol ? n[k].y : xn.y,
                                   a.hol ? n[k].z : xn.z, x[k].w);
        // a constraint pass adds its displacement over dt to the velocities
        // (src/CudaHolonomicConstraint.cu:94-106): the first pass's on-step
        // kinetic energy sees it
        const d3 vn = xyz(vm[k]) + idt * (n[k] - n0[k]);
        c.vel[i] = make_double4(vn.x, vn.y, vn.z, vm[k].w);
        const d3 u1 = idt * xyz(dp[k]), u2 = idt * d;
        const double kon = 0.5 * dot(vn, vn) / vm[k].w;
        v[27] += (0.5 * dot(u1, u1) / vm[k].w + kon + 0.5 * dot(u2, u2) / vm[k].w) / 3.0;
        v[28] += kon;
      }
    }
  }
  block_partials_n<29>(v, a.partials);
  if (is_last_block(&a.ps->counter)) {
    __shared__ double tot[29];
    sum_partials_n<29>(a.partials, tot);
    if (threadIdx.x == 0) {
      PistonScalars *ps = a.ps;
      const double V = ps->box[0] * ps->box[1] * ps->box[2];
      ps->vfac = kPatmos / V;
      ps->lp_vfac = V * a.pbfact * kAtmosp;
      for (int k = 0; k < 9; ++k) {
        ps->vir[k] = (double)a.vir_fixed[k] * kInvEnergyScale + tot[k];
        const double kin = 0.5 * (tot[9 + k] + tot[18 + k]);
        ps->p[k] = ps->vfac * (kin + ps->vir[k]);
        ps->dp[k] = ps->p[k] - ps->pref[k];
      }
      ps->pscalar = (ps->p[0] + ps->p[4] + ps->p[8]) / 3.0;
      if (a.const_st) {
        ps->pref[0] = ps->pref[8] - a.st / ps->box[2];
        ps->pref[4] = ps->pref[0];
      }
      for (int k = 0; k < 9; ++k) ps->dp_static[k] = ps->dp[k] - 0.25 * ps->vfac * tot[9 + k];
      c.sc->piston_v_prev = c.sc->piston_v;
      c.sc->piston_f_prev = c.sc->piston_f;
      lp_pass_start(c, a, tot[27], tot[28], dt);
      ps->counter = 0;
    }
  }
}

// predictor-corrector pass over atoms: atoms follow piston and thermostat;
// the last block forms the new pressure difference and, when another pass
// follows (`more`), starts it from the kinetic energy of the new velocities
__global__ void __launch_bounds__(kThreads) lp_pc_kernel(Common c, PistonArgs a, int natom,
                                                         int more) {
  if (*c.err) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double dt = c.dt, dt2 = dt * dt, idt = 1.0 / dt, fact = 0.5 / dt;
  const PistonScalars *ps = a.ps;
  const double nh = a.use_nh ? dt2 * c.sc->piston_v : 0.0;
  // [0..8] sum d d m/dt^2 of the predicted half step, [9..10] kinetic energy
  double v[11];
#pragma unroll
  for (int k = 0; k < 11; ++k) v[k] = 0.0;
  if (i < natom) {
    const d3 dprev = xyz(c.dprev[i]), dpred = xyz(c.dpred[i]), d = xyz(c.delta[i]);
    const d3 r = xyz(c.ref[i]);
    const double4 x = c.coords[i];
    const d3 u = fact * (dprev + dpred);
    const d3 np = mk(d.x - (nh + dt * ps->cf_on[0]) * u.x, d.y - (nh + dt * ps->cf_on[1]) * u.y,
                     d.z - (nh + dt * ps->cf_on[2]) * u.z);
    c.dpred[i] = make_double4(np.x, np.y, np.z, 0.0);
    const double im = c.vel[i].w;
    c.vel[i] = make_double4(u.x, u.y, u.z, im);
    const d3 h = 0.5 * (r + xyz(x));
    c.coords[i] = make_double4(r.x + np.x + ps->cf_half[0] * h.x, r.y + np.y + ps->cf_half[1] * h.y,
                               r.z + np.z + ps->cf_half[2] * h.z, x.w);
    const double f = 1.0 / (dt2 * im);
    const double nn[3] = {np.x, np.y, np.z};
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
      for (int q = 0; q < 3; ++q) v[3 * p + q] = f * nn[p] * nn[q];
    if (more) {
      const d3 u1 = idt * dprev, u2 = idt * np;
      const double kon = 0.5 * dot(u, u) / im;
      v[9] = (0.5 * dot(u1, u1) / im + kon + 0.5 * dot(u2, u2) / im) / 3.0;
      v[10] = kon;
    }
  }
  block_partials_n<11>(v, a.partials);
  if (is_last_block(&a.ps->counter)) {
    __shared__ double tot[11];
    sum_partials_n<11>(a.partials, tot);
    if (threadIdx.x == 0) {
      for (int k = 0; k < 9; ++k) a.ps->dp[k] = a.ps->dp_static[k] + 0.25 * a.ps->vfac * tot[k];
      if (more) lp_pass_start(c, a, tot[9], tot[10], dt);
      a.ps->counter = 0;
    }
  }
}

__global__ void __launch_bounds__(kThreads) lp_final_kernel(Common c, PistonArgs a) {
  if (*c.err) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const double dt = c.dt, dt2 = dt * dt, idt = 1.0 / dt, fact = 0.5 / dt;
  // [0] 3-term kinetic energy, [1] on-step, [2..10] sum (d d + dp dp) m/dt^2
  double v[11];
#pragma unroll
  for (int k = 0; k < 11; ++k) v[k] = 0.0;
  if (g < c.ngroups) {
    int at[4];
    const int m = group_atoms(c, g, at);
    const int2 meta = c.gmeta[g];
    d3 o[4], n[4], dp[4], dn[4], rs[4];
    double q[4], im[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k < m) {
        const int i = at[k];
        o[k] = xyz(c.ref[i]);
        const double4 x = c.coords[i];
        n[k] = xyz(x);
        q[k] = x.w;
        dp[k] = xyz(c.dprev[i]);
        dn[k] = xyz(c.dpred[i]);
        im[k] = c.vel[i].w;
      }
    }
    if (a.hol) {
      // the new positions onto the constraints, the reference positions
      // scaled with the box and constrained against the new ones, the
      // displacement between them (src/CudaLangevinPistonIntegrator.cu:1955-1980)
      apply_constraint(meta.x, m, o, n, c.sk, c.shake_p, meta.y);
      const PistonScalars *ps = a.ps;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (k < m) {
          const d3 h = 0.5 * (o[k] + n[k]);
          rs[k] = o[k] + mk(ps->cf_half[0] * h.x, ps->cf_half[1] * h.y, ps->cf_half[2] * h.z);
        }
      }
      apply_constraint(meta.x, m, n, rs, c.sk, c.shake_p, meta.y);
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (k < m) dn[k] = n[k] - rs[k];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k < m) {
        const int i = at[k];
        const d3 d = dn[k];
        const d3 u = fact * (d + dp[k]);
        const d3 u1 = idt * dp[k], u2 = idt * d;
        const double kon = 0.5 * dot(u, u) / im[k];
        v[0] += (0.5 * dot(u1, u1) / im[k] + kon + 0.5 * dot(u2, u2) / im[k]) / 3.0;
        v[1] += kon;
        const double f = 1.0 / (dt2 * im[k]);
        const double dd[3] = {d.x, d.y, d.z}, pp[3] = {dp[k].x, dp[k].y, dp[k].z};
#pragma unroll
        for (int s = 0; s < 3; ++s)
#pragma unroll
          for (int w = 0; w < 3; ++w) v[2 + 3 * s + w] += f * (dd[s] * dd[w] + pp[s] * pp[w]);
        c.delta[i] = make_double4(d.x, d.y, d.z, 0.0);
        c.dprev[i] = make_double4(d.x, d.y, d.z, 0.0);
        c.vel[i] = make_double4(u.x, u.y, u.z, im[k]);
        c.coords[i] = make_double4(n[k].x, n[k].y, n[k].z, q[k]);
        c.xyzq[i] = make_float4((float)n[k].x, (float)n[k].y, (float)n[k].z, (float)q[k]);
      }
    }
  }
  block_partials_n<11>(v, a.partials);
  if (is_last_block(&a.ps->counter)) {
    __shared__ double tot[11];
    sum_partials_n<11>(a.partials, tot);
    if (threadIdx.x == 0) {
      PistonScalars *ps = a.ps;
      piston_update(c.sc, a.use_old ? tot[1] : tot[0], a.ke_ref, dt);
      const double s = (double)(c.sc->window + 1);
      for (int k = 0; k < 9; ++k) {
        ps->p[k] = ps->vfac * (0.5 * tot[2 + k] + ps->vir[k]);
        ps->pavg[k] += (ps->p[k] - ps->pavg[k]) / s;
      }
      ps->pscalar = (ps->p[0] + ps->p[4] + ps->p[8]) / 3.0;
      ps->pavg_scalar += (ps->pscalar - ps->pavg_scalar) / s;
      finish_temperature(c, tot[0], tot[1]);
      for (int d = 0; d < 3; ++d) {
        ps->box_old[d] = ps->box[d];
        ps->box[d] = ps->box_pred[d];
        ps->lp_delta[d] = ps->lp_delta_pred[d];
      }
      // the new box where the next step's kernels read it: the force
      // manager's device box, its direct-space set-up (the conversions of
      // make_nb_setup) and the list's dims
      const double L[3] = {ps->box[0], ps->box[1], ps->box[2]};
      *a.dbox = make_double4(L[0], L[1], L[2], 0.0);
      NbSetup &st = *a.setup;
      st.Lxd = L[0];
      st.Lyd = L[1];
      st.Lzd = L[2];
      st.Lx_lo = (float)(L[0] - (double)(float)L[0]);
      st.Ly_lo = (float)(L[1] - (double)(float)L[1]);
      st.Lz_lo = (float)(L[2] - (double)(float)L[2]);
      st.Lx = (float)L[0];
      st.Ly = (float)L[1];
      st.Lz = (float)L[2];
      NbSysDims &ls = *a.lsys;
      ls.Lx = (float)L[0];
      ls.Ly = (float)L[1];
      ls.Lz = (float)L[2];
      ls.Lxd = L[0];
      ls.Lyd = L[1];
      ls.Lzd = L[2];
      c.sc->step += 1;
      ps->counter = 0;
    }
  }
}

// one Philox state per piston degree of freedom: subsequence = dof index,
// then `pos` draws skipped (InitializeRngKernel)
__global__ void lp_rng_init_kernel(curandStatePhilox4_32_10_t *st, int n,
                                   unsigned long long seed, unsigned long long pos,
                                   PistonScalars *ps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) ps->rngpos = pos;
  if (i >= n) return;
  curand_init(seed, (unsigned long long)i, 0ull, st + i);
  skipahead(pos, st + i);
}

template <typename T>
void upload(DeviceArray<T> &d, const std::vector<T> &v) {
  d.upload(v.empty() ? std::vector<T>(1) : v);
}

}  // namespace

struct IntegratorState {
  DeviceArray<int> atom_off;
  DeviceArray<unsigned long long> sys_seed, sys_rng0;
  DeviceArray<long long> sys_stop;
  DeviceArray<int4> groups;
  DeviceArray<int2> gmeta;
  DeviceArray<float4> shake_p;
  DeviceArray<double4> dprev, delta, dpred, ref;
  DeviceArray<Scalars> sc;
  DeviceArray<double> partials;
  int ngroups = 0, natom = 0;
  Common c{};
  int blocks_groups = 0, blocks_atoms = 0, blocks_lanes = 0;  // lanes: 4 per group
  // the error word after each of the last two segments, copied to pinned
  // host memory behind the segment, and the events that say it has landed
  unsigned *h_err = nullptr;
  cudaEvent_t seg_done[2] = {nullptr, nullptr};
  IntegratorState() {
    APO_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&h_err), 2 * sizeof(unsigned),
                           cudaHostAllocDefault));
    h_err[0] = h_err[1] = 0;
    for (auto &e : seg_done) APO_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  ~IntegratorState() {
    for (auto &e : seg_done)
      if (e) cudaEventDestroy(e);
    if (h_err) cudaFreeHost(h_err);
  }
};

// -------------------------------------------------------------- base class

CudaIntegrator::CudaIntegrator(double ps) : m_Dt(ps / kTimfac) {
  if (!(ps > 0)) throw std::invalid_argument("time step must be positive");
}

CudaIntegrator::~CudaIntegrator() { clearGraphs(); }

void CudaIntegrator::clearGraphs() {
  for (auto &kv : m_Graphs) cudaGraphExecDestroy(kv.second);
  m_Graphs.clear();
}

void CudaIntegrator::setTimeStep(double ps) {
  if (!(ps > 0)) throw std::invalid_argument("time step must be positive");
  m_Dt = ps / kTimfac;
  clearGraphs();
  if (m_S) m_S->c.dt = m_Dt;
}

void CudaIntegrator::setNonbondedListUpdateFrequency(int f) {
  if (f < 1) throw std::invalid_argument("list update frequency must be >= 1");
  m_ListFreq = f;
  clearGraphs();
}

cudaStream_t CudaIntegrator::stream() const { return m_Ctx ? m_Ctx->stream() : nullptr; }

int CudaIntegrator::kernelsPerRebuild() const { return 11; }

void CudaIntegrator::setCharmmContext(std::shared_ptr<CharmmContext> ctx) {
  if (m_Ctx) throw std::invalid_argument("A CharmmContext object was already set for this CudaIntegrator.");
  if (!ctx) throw std::invalid_argument("null CharmmContext");
  m_Ctx = std::move(ctx);
  // centre-of-mass removal sums over all atoms: with several systems it
  // would couple them, so it is not applied (Langevin damps the drift)
  if (m_Ctx->getForceManager()->isMulti()) m_ComFreq = 0;
  buildGroups();
  initialize();
  m_Initialized = true;
}

void CudaIntegrator::buildGroups() {
  auto fm = m_Ctx->getForceManager();
  const Topology &t = fm->topology();
  const int n = t.natom;
  const bool hol = m_Ctx->isUsingHolonomicConstraints();
  std::vector<int> owner(n, -1);
  std::vector<int4> groups;
  std::vector<int2> meta;
  if (hol) {
    for (auto &w : t.waters) {
      owner[w.x] = owner[w.y] = owner[w.z] = (int)groups.size();
      groups.push_back({w.x, w.y, w.z, -1});
      meta.push_back({kSettle, 0});
    }
    for (size_t k = 0; k < t.shake_atoms.size(); ++k) {
      const int4 s = t.shake_atoms[k];
      bool clash = owner[s.x] >= 0 || owner[s.y] >= 0 || (s.z >= 0 && owner[s.z] >= 0) ||
                   (s.w >= 0 && owner[s.w] >= 0);
      if (clash) throw std::invalid_argument("an atom belongs to two constraint groups");
      owner[s.x] = owner[s.y] = (int)groups.size();
      if (s.z >= 0) owner[s.z] = (int)groups.size();
      if (s.w >= 0) owner[s.w] = (int)groups.size();
      groups.push_back(s);
      meta.push_back({kShake, (int)k});
    }
  }
  // free atoms in runs of up to four consecutive atoms of one system
  std::vector<int> sys_end(n, n);
  if (fm->isMulti()) {
    const auto &off = fm->atomOffsets();
    for (size_t k = 0; k + 1 < off.size(); ++k)
      for (int a = off[k]; a < off[k + 1]; ++a) sys_end[a] = off[k + 1];
  }
  for (int i = 0; i < n;) {
    if (owner[i] >= 0) {
      ++i;
      continue;
    }
    int4 g = {i, -1, -1, -1};
    int *slot = &g.y;
    int k = 0;
    int j = i + 1;
    while (k < 3 && j < sys_end[i] && owner[j] < 0) {
      slot[k++] = j;
      ++j;
    }
    groups.push_back(g);
    meta.push_back({kFree, 0});
    i = j;
  }
  m_S = std::make_unique<IntegratorState>();
  IntegratorState &S = *m_S;
  S.natom = n;
  S.ngroups = (int)groups.size();
  S.groups.upload(groups);
  S.gmeta.upload(meta);
  upload(S.shake_p, t.shake_p);
  S.dprev.alloc(n);
  S.delta.alloc(n);
  S.dpred.alloc(n);
  S.ref.alloc(n);
  APO_CUDA(cudaMemset(S.dprev.p, 0, n * sizeof(double4)));
  APO_CUDA(cudaMemset(S.delta.p, 0, n * sizeof(double4)));
  S.sc.alloc(1);
  Scalars z{};
  APO_CUDA(cudaMemcpy(S.sc.p, &z, sizeof(z), cudaMemcpyHostToDevice));
  S.blocks_groups = (S.ngroups + kThreads - 1) / kThreads;
  S.blocks_atoms = (n + kThreads - 1) / kThreads;
  S.blocks_lanes = (4 * S.ngroups + kThreads - 1) / kThreads;
  if (std::max(S.blocks_lanes, S.blocks_atoms) > kMaxBlocks * 64)
    throw std::invalid_argument("system too large for the integrator's reduction buffer");
  S.partials.alloc((size_t)4 * std::max(S.blocks_lanes, S.blocks_atoms) + 8);
  Common &c = S.c;
  c.sys_of_atom = nullptr;
  c.atom_off = nullptr;
  c.sys_seed = nullptr;
  c.sys_rng0 = nullptr;
  c.sys_stop = nullptr;
  if (fm->isMulti()) {
    std::vector<unsigned long long> seeds;
    for (auto &y : fm->systemSpecs()) seeds.push_back((unsigned long long)y.seed);
    S.atom_off.upload(fm->atomOffsets());
    S.sys_seed.upload(seeds);
    c.sys_of_atom = fm->sysOfAtom();
    c.atom_off = S.atom_off.p;
    c.sys_seed = S.sys_seed.p;
  }
  c.ngroups = S.ngroups;
  c.groups = S.groups.p;
  c.gmeta = S.gmeta.p;
  c.shake_p = S.shake_p.p;
  c.coords = m_Ctx->coords();
  c.vel = m_Ctx->velMass();
  c.dprev = S.dprev.p;
  c.delta = S.delta.p;
  c.dpred = S.dpred.p;
  c.ref = S.ref.p;
  c.xyzq = m_Ctx->xyzq();
  c.force = fm->forceFixed();
  c.stride = fm->forceStride();
  c.glo2loc = fm->neighborList().glo2loc;
  c.slot_off = fm->neighborList().slot_off;
  c.xyzq_s = fm->neighborList().xyzq_s;
  c.sc = S.sc.p;
  c.partials = S.partials.p;
  c.err = fm->neighborList().error;
  c.sk = make_settle();
  c.ndegf = m_Ctx->getDegreesOfFreedom();
  c.dt = m_Dt;
}

void CudaIntegrator::forcesForStep(cudaStream_t s) {
  m_Ctx->getForceManager()->calcForce(m_Ctx->xyzq(), false, false, s, /*clear=*/false);
}

void CudaIntegrator::segment(int nsteps, cudaStream_t s) {
  IntegratorState &S = *m_S;
  auto fm = m_Ctx->getForceManager();
  fm->rewindKernelTimers();
  // a force evaluation requested between propagate() calls leaves gradients
  // in the shared buffer; every segment starts from a cleared one (the step
  // kernels clear each slot they consume afterwards)
  APO_CUDA(cudaMemsetAsync(fm->forceFixed(), 0, (size_t)3 * fm->forceStride() * sizeof(long long), s));
  if (m_ComFreq > 0) {
    com_sum_kernel<<<S.blocks_atoms, kThreads, 0, s>>>(S.c, S.natom, m_ComFreq);
    com_apply_kernel<<<S.blocks_atoms, kThreads, 0, s>>>(S.c, S.natom, m_ComFreq);
    APO_LAUNCH_CHECK();
  }
  m_Ctx->resetNeighborList(s);
  for (int k = 0; k < nsteps; ++k) {
    forcesForStep(s);
    stepKernels(s);
  }
}

void CudaIntegrator::subscribe(std::shared_ptr<Subscriber> sub) {
  if (!sub) throw std::invalid_argument("null subscriber");
  sub->attach(this);
  m_Subscribers.push_back(std::move(sub));
}

bool CudaIntegrator::unsubscribe(const std::shared_ptr<Subscriber> &sub) {
  for (size_t k = 0; k < m_Subscribers.size(); ++k)
    if (m_Subscribers[k] == sub) {
      m_Subscribers[k]->attach(nullptr);
      m_Subscribers.erase(m_Subscribers.begin() + k);
      return true;
    }
  return false;
}

void CudaIntegrator::launchSegment(int len, cudaStream_t s) {
  if (m_UseGraphs) {
    auto it = m_Graphs.find(len);
    if (it == m_Graphs.end()) {
      cudaGraph_t graph;
      APO_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      try {
        segment(len, s);
      } catch (...) {
        cudaStreamEndCapture(s, &graph);
        throw;
      }
      APO_CUDA(cudaStreamEndCapture(s, &graph));
      cudaGraphExec_t exec;
      // keep the stream priorities of the captured launches
      APO_CUDA(cudaGraphInstantiate(&exec, graph, cudaGraphInstantiateFlagUseNodePriority));
      APO_CUDA(cudaGraphDestroy(graph));
      it = m_Graphs.emplace(len, exec).first;
    }
    APO_CUDA(cudaGraphLaunch(it->second, s));
  } else {
    segment(len, s);
  }
}

// Segments are launched without waiting.  A neighbour-list build that
// overflows its buffers (or meets non-finite coordinates) sets the list's
// error word, and from then on every step kernel leaves the state alone, so
// the state stays at the start of the failed segment.  The word is copied
// to pinned memory behind every segment and looked at, without waiting,
// two launches later; at the end (and before every subscriber report) it is
// read after a synchronisation.  On an overflow the list is grown at the
// frozen coordinates and the run continues from the device's step counter:
// the segments after it start at the same steps as in an uninterrupted run,
// so the trajectory is the same.  Non-finite coordinates end the call with
// an exception and the state frozen at the failed segment
// (the reference checks its energies at the report frequency,
// src/CudaIntegrator.cu:357-369).
void CudaIntegrator::propagate(int numSteps) {
  if (!m_Ctx)
    throw std::invalid_argument("CudaIntegrator::propagate: no CharmmContext was set for this CudaIntegrator.");
  if (numSteps <= 0) return;
  cudaStream_t s = m_Ctx->stream();
  IntegratorState &S = *m_S;
  auto fm = m_Ctx->getForceManager();
  // the first list build sizes the buffers synchronously: never inside a
  // capture; a list made stale by new coordinates is rebuilt by the first
  // segment, which starts with a rebuild (an overflow there is grown and
  // the segment run again, below)
  m_Ctx->ensureListBuffers();
  const long long step0 = m_Step;
  const long long dev0 = deviceStep();
  long long done = 0;
  int regrowths = 0;
  for (;;) {
    const int gen = fm->pluginGeneration();
    if (gen != m_PluginGen) {  // a plug-in force or a list buffer changed: capture again
      clearGraphs();
      m_PluginGen = gen;
    }
    long long launched = done;
    int k = 0;
    bool seen = false;
    while (launched < numSteps && !seen) {
      int len = (int)std::min<long long>(numSteps - launched, m_ListFreq);
      // stop a segment at the next report of any subscriber
      for (auto &sub : m_Subscribers) {
        const long long f = sub->getReportFrequency();
        const long long next = (launched / f + 1) * f;
        len = (int)std::min<long long>(len, next - launched);
      }
      const int slot = k & 1;
      if (k >= 2 && cudaEventQuery(S.seg_done[slot]) == cudaSuccess && S.h_err[slot]) {
        seen = true;
        break;
      }
      launchSegment(len, s);
      APO_CUDA(cudaMemcpyAsync(&S.h_err[slot], S.c.err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
      APO_CUDA(cudaEventRecord(S.seg_done[slot], s));
      launched += len;
      ++k;
      bool report = false;
      for (auto &sub : m_Subscribers) report |= launched % sub->getReportFrequency() == 0;
      if (report) {
        APO_CUDA(cudaStreamSynchronize(s));
        if (S.h_err[slot]) {
          seen = true;
          break;
        }
        m_Step = step0 + launched;
        beforeReport();
        for (auto &sub : m_Subscribers)
          if (launched % sub->getReportFrequency() == 0) sub->update(*m_Ctx, m_Step, getTimeStep());
      }
    }
    APO_CUDA(cudaStreamSynchronize(s));
    const unsigned e = fm->readDeviceError(s);
    done = deviceStep() - dev0;
    m_Step = step0 + done;
    if (!e) {
      if (done >= numSteps) return;
      throw std::runtime_error("CudaIntegrator::propagate: the device step counter stopped at " +
                               std::to_string(done) + " of " + std::to_string(numSteps) + " steps");
    }
    if (e & kErrNaN)
      throw std::runtime_error("non-finite coordinates during propagation (state kept at step " +
                               std::to_string(m_Step) + ")");
    if (e & kErrCopyTimeout)
      throw std::runtime_error("a tensor copy of the reciprocal-space grid did not complete "
                               "(state kept at step " + std::to_string(m_Step) + ")");
    if (e & kErrColumnOverflow)
      throw std::runtime_error("neighbour list: a cell column outgrew the column sort during "
                               "propagation (state kept at step " + std::to_string(m_Step) + ")");
    if (++regrowths > 8)
      throw std::runtime_error("neighbour list capacity exceeded repeatedly during propagation "
                               "(device error " + std::to_string(e) + ")");
    fm->growNeighborList(m_Ctx->xyzq(), s);
  }
}

double CudaIntegrator::getInstantaneousTemperature() {
  Scalars h;
  APO_CUDA(cudaStreamSynchronize(stream()));
  APO_CUDA(cudaMemcpy(&h, m_S->sc.p, sizeof(h), cudaMemcpyDeviceToHost));
  return h.ke[0] / (0.5 * m_Ctx->getDegreesOfFreedom() * kBoltz);
}

double CudaIntegrator::getAverageTemperature() {
  Scalars h;
  APO_CUDA(cudaStreamSynchronize(stream()));
  APO_CUDA(cudaMemcpy(&h, m_S->sc.p, sizeof(h), cudaMemcpyDeviceToHost));
  return h.avgT[0];
}

void CudaIntegrator::resetAverageTemperature() {
  Scalars h;
  APO_CUDA(cudaStreamSynchronize(stream()));
  APO_CUDA(cudaMemcpy(&h, m_S->sc.p, sizeof(h), cudaMemcpyDeviceToHost));
  h.avgT[0] = h.avgT[1] = 0.0;
  h.window = 0;
  APO_CUDA(cudaMemcpy(m_S->sc.p, &h, sizeof(h), cudaMemcpyHostToDevice));
}

// ---------------------------------------------------------------- Langevin

CudaLangevinThermostatIntegrator::CudaLangevinThermostatIntegrator(double ps)
    : CudaIntegrator(ps) {
  std::random_device rd;
  m_Seed = rd();
  m_KernelsPerStep = 1;
}

void CudaLangevinThermostatIntegrator::setThermostatFriction(double f) {
  if (f < 0) throw std::invalid_argument("friction must be >= 0");
  m_Friction = f;
  clearGraphs();
}

double4 *CudaIntegrator::deltaState() const { return m_S ? m_S->dprev.p : nullptr; }

void CudaIntegrator::setSystemLimits(const std::vector<unsigned long long> &rng0,
                                     const std::vector<long long> &stop) {
  if (!m_S || !m_Ctx) throw std::runtime_error("setSystemLimits: no context set");
  auto fm = m_Ctx->getForceManager();
  if (!fm->isMulti()) throw std::invalid_argument("setSystemLimits: not a multi-system context");
  if ((int)rng0.size() != fm->numSystems() || (int)stop.size() != fm->numSystems())
    throw std::invalid_argument("setSystemLimits: one entry per system expected");
  m_S->sys_rng0.upload(rng0);
  m_S->sys_stop.upload(stop);
  m_S->c.sys_rng0 = m_S->sys_rng0.p;
  m_S->c.sys_stop = m_S->sys_stop.p;
  clearGraphs();  // the graphs hold the launch arguments
}

long long CudaIntegrator::deviceStep() {
  Scalars h;
  APO_CUDA(cudaStreamSynchronize(stream()));
  APO_CUDA(cudaMemcpy(&h, m_S->sc.p, sizeof(h), cudaMemcpyDeviceToHost));
  return h.step;
}

RestartRecord CudaIntegrator::restartRecord() {
  if (!m_S || !m_Ctx) throw std::runtime_error("restart: no CharmmContext was set for this integrator");
  auto *lt = dynamic_cast<CudaLangevinThermostatIntegrator *>(this);
  auto *nh = dynamic_cast<CudaNoseHooverIntegrator *>(this);
  auto *lp = dynamic_cast<CudaLangevinPistonIntegrator *>(this);
  if (!lt && !nh && !lp)
    throw std::runtime_error("Attempted to write a restart file for an unsupported integrator type. "
                             "The supported integrators are CudaNoseHooverIntegrator, "
                             "CudaLangevinPistonIntegrator and CudaLangevinThermostatIntegrator.");
  if (m_Ctx->getForceManager()->isMulti())
    throw std::runtime_error("restart files describe one system: not available for a "
                             "multi-system context");
  cudaStream_t s = stream();
  Scalars h;
  APO_CUDA(cudaStreamSynchronize(s));
  APO_CUDA(cudaMemcpy(&h, m_S->sc.p, sizeof(h), cudaMemcpyDeviceToHost));
  RestartRecord r;
  r.box = m_Ctx->getForceManager()->getBoxDimensions();
  r.natom = m_S->natom;
  r.npriv = m_Step;
  r.nstep = m_Step;
  r.ndegf = m_Ctx->getDegreesOfFreedom();
  r.avetem = h.avgT[0];
  if (lt) {
    r.seed = lt->getThermostatRngSeed();
    r.has_rng = true;
    r.rngpos = h.rngpos;
  } else {
    r.pnhv = h.piston_v;
    r.pnhf = h.piston_f;
  }
  if (lp) {  // src/RestartSubscriber.cu:124-139, 246-250
    r.seed = lp->getLangevinPistonFrictionSeed();
    r.has_rng = true;
    r.rngpos = lp->getRngSequencePos();
    const Crystal c = lp->getCrystalType();
    r.crystal = c == Crystal::Cubic ? "CUBI" : (c == Crystal::Tetragonal ? "TETR" : "ORTH");
    const auto d = lp->getLangevinPistonDeltaPosition();
    for (size_t k = 0; k < d.size() && k < 3; ++k) r.hdot[k] = d[k];
  }
  r.xold = m_Ctx->getCoordinates();
  r.vel = m_Ctx->getVelocities();
  std::vector<double4> d(m_S->natom);
  APO_CUDA(cudaMemcpy(d.data(), m_S->dprev.p, d.size() * sizeof(double4), cudaMemcpyDeviceToHost));
  r.delta.resize((size_t)3 * m_S->natom);
  for (int i = 0; i < m_S->natom; ++i) {
    r.delta[3 * (size_t)i] = d[i].x;
    r.delta[3 * (size_t)i + 1] = d[i].y;
    r.delta[3 * (size_t)i + 2] = d[i].z;
  }
  return r;
}

void CudaIntegrator::initializeFromRestartFile(const std::string &path) {
  if (path.empty()) throw std::invalid_argument("initializeFromRestartFile: empty file name");
  if (!m_S || !m_Ctx)
    throw std::runtime_error("CharmmContext must be set before initializing from a restart file");
  auto *lt = dynamic_cast<CudaLangevinThermostatIntegrator *>(this);
  auto *nh = dynamic_cast<CudaNoseHooverIntegrator *>(this);
  auto *lp = dynamic_cast<CudaLangevinPistonIntegrator *>(this);
  if (!lt && !nh && !lp)
    throw std::runtime_error("initializeFromRestartFile: only the Langevin thermostat, "
                             "Nose-Hoover and Langevin piston integrators read restart files");
  auto fm = m_Ctx->getForceManager();
  if (fm->isMulti())
    throw std::runtime_error("restart files describe one system: not available for a "
                             "multi-system context");
  const RestartRecord r = readRestartFile(path);
  if (r.natom != m_Ctx->getNumAtoms())
    throw std::invalid_argument("NATOM mismatch in restart file \"" + path + "\"");
  if (r.ndegf != m_Ctx->getDegreesOfFreedom())
    throw std::invalid_argument("NDEGF mismatch in restart file \"" + path + "\"");
  // The file's box becomes the context's, as in the reference
  // (src/CudaLangevinThermostatIntegrator.cu:394): the force manager is set
  // up again for it (spline order and FFT grid unchanged) and this
  // integrator's state is built again over the manager's new buffers.  A
  // file written with 16 significant digits (the reference's form) need not
  // give back the last bit of a box that is already the same.
  const auto box = fm->getBoxDimensions();
  bool other_box = false;
  for (int k = 0; k < 3; ++k) other_box |= std::fabs(r.box[k] - box[k]) > 1e-12 * std::fabs(box[k]);
  if (other_box) {
    fm->setBoxDimensions({r.box[0], r.box[1], r.box[2]});
    fm->initialize();
    fm->setStateCoordinates(m_Ctx->coords());
    clearGraphs();
    buildGroups();
    initialize();
  }
  m_Ctx->setCoordinates(r.xold);
  m_Ctx->setVelocities(r.vel);
  std::vector<double4> d(r.natom);
  for (int i = 0; i < r.natom; ++i)
    d[i] = make_double4(r.delta[3 * (size_t)i], r.delta[3 * (size_t)i + 1],
                        r.delta[3 * (size_t)i + 2], 0.0);
  APO_CUDA(cudaMemcpy(m_S->dprev.p, d.data(), d.size() * sizeof(double4), cudaMemcpyHostToDevice));
  Scalars h;
  APO_CUDA(cudaMemcpy(&h, m_S->sc.p, sizeof(h), cudaMemcpyDeviceToHost));
  h.step = r.npriv;
  if (lt) {
    lt->setThermostatRngSeed(r.seed);
    // a file without the APO tag carries no RNG position (as the reference reads it)
    h.rngpos = (r.apo && r.has_rng) ? r.rngpos : 0ull;
  } else {
    h.piston_v = r.pnhv;
    h.piston_f = r.pnhf;
  }
  APO_CUDA(cudaMemcpy(m_S->sc.p, &h, sizeof(h), cudaMemcpyHostToDevice));
  m_Step = r.npriv;
  clearGraphs();  // the captured launches hold the seed
  if (lp) lp->applyRestartRecord(r);
}

unsigned long long CudaLangevinThermostatIntegrator::getRngSequencePos() {
  Scalars h;
  APO_CUDA(cudaStreamSynchronize(stream()));
  APO_CUDA(cudaMemcpy(&h, m_S->sc.p, sizeof(h), cudaMemcpyDeviceToHost));
  return h.rngpos;
}

void CudaLangevinThermostatIntegrator::initialize() {
  IntegratorState &S = *m_S;
  cudaStream_t s = m_Ctx->stream();
  const double gamma = m_Dt * kTimfac * m_Friction;
  if (m_Ctx->isUsingHolonomicConstraints())
    init_constrain_kernel<<<S.blocks_groups, kThreads, 0, s>>>(S.c, 0);
  m_Ctx->getForceManager()->calcForceChecked(m_Ctx->xyzq(), false, false, s);
  init_delta_kernel<<<S.blocks_atoms, kThreads, 0, s>>>(S.c, S.natom, gamma);
  if (m_Ctx->isUsingHolonomicConstraints())
    init_constrain_kernel<<<S.blocks_groups, kThreads, 0, s>>>(S.c, 1);
  APO_LAUNCH_CHECK();
  APO_CUDA(cudaStreamSynchronize(s));
}

void CudaLangevinThermostatIntegrator::stepKernels(cudaStream_t s) {
  IntegratorState &S = *m_S;
  const double gamma = m_Dt * kTimfac * m_Friction;
  const double kbt = kBoltz * m_RefT;
  langevin_kernel<<<S.blocks_lanes, kThreads, 0, s>>>(S.c, gamma, kbt, m_Seed);
  APO_LAUNCH_CHECK();
}

// ------------------------------------------------------------- Nose-Hoover

CudaNoseHooverIntegrator::CudaNoseHooverIntegrator(double ps) : CudaIntegrator(ps) {
  m_KernelsPerStep = 5;
}

void CudaNoseHooverIntegrator::setNoseHooverPistonMass(double m) {
  m_PistonMass = m;
  if (m_S) {  // after initialisation the mass lives on the device
    APO_CUDA(cudaStreamSynchronize(stream()));
    APO_CUDA(cudaMemcpy(reinterpret_cast<char *>(m_S->sc.p) + offsetof(Scalars, piston_mass), &m,
                        sizeof(double), cudaMemcpyHostToDevice));
  }
}

void CudaNoseHooverIntegrator::initialize() {
  if (m_Ctx->getForceManager()->isMulti())
    throw std::invalid_argument("Nose-Hoover couples all atoms through one piston: it is not "
                                "available for a multi-system context");
  IntegratorState &S = *m_S;
  cudaStream_t s = m_Ctx->stream();
  if (m_PistonMass == -9999.9999) {
    // 0.2 x total mass (src/CudaNoseHooverIntegrator.cu:1009-1021)
    double tm = 0;
    for (double mm : m_Ctx->getForceManager()->topology().mass) tm += mm;
    m_PistonMass = 0.2 * tm;
  }
  Scalars h{};
  h.piston_mass = m_PistonMass;
  APO_CUDA(cudaMemcpy(S.sc.p, &h, sizeof(h), cudaMemcpyHostToDevice));
  if (m_Ctx->isUsingHolonomicConstraints())
    init_constrain_kernel<<<S.blocks_groups, kThreads, 0, s>>>(S.c, 0);
  m_Ctx->getForceManager()->calcForceChecked(m_Ctx->xyzq(), false, false, s);
  init_delta_kernel<<<S.blocks_atoms, kThreads, 0, s>>>(S.c, S.natom, 0.0);
  if (m_Ctx->isUsingHolonomicConstraints())
    init_constrain_kernel<<<S.blocks_groups, kThreads, 0, s>>>(S.c, 1);
  APO_LAUNCH_CHECK();
  APO_CUDA(cudaStreamSynchronize(s));
}

void CudaNoseHooverIntegrator::stepKernels(cudaStream_t s) {
  IntegratorState &S = *m_S;
  const double ke_ref = 0.5 * m_Ctx->getDegreesOfFreedom() * kBoltz * m_RefT;
  const int old = m_OldT ? 1 : 0;
  nh_half_kernel<<<S.blocks_groups, kThreads, 0, s>>>(S.c, ke_ref, old);
  nh_pc_kernel<true><<<S.blocks_atoms, kThreads, 0, s>>>(S.c, S.natom, ke_ref, old);
  nh_pc_kernel<true><<<S.blocks_atoms, kThreads, 0, s>>>(S.c, S.natom, ke_ref, old);
  nh_pc_kernel<false><<<S.blocks_atoms, kThreads, 0, s>>>(S.c, S.natom, ke_ref, old);
  nh_final_kernel<<<S.blocks_groups, kThreads, 0, s>>>(S.c, ke_ref, old);
  APO_LAUNCH_CHECK();
}

// --------------------------------------------------------- Langevin piston

struct PistonState {
  DeviceArray<PistonScalars> ps;
  DeviceArray<curandStatePhilox4_32_10_t> rng;
  DeviceArray<double> partials;
};

CudaLangevinPistonIntegrator::CudaLangevinPistonIntegrator(double ps) : CudaIntegrator(ps) {
  std::random_device rd;
  m_Seed = rd();
  m_KernelsPerStep = 3 + m_MaxPC;
}

CudaLangevinPistonIntegrator::~CudaLangevinPistonIntegrator() = default;

void CudaLangevinPistonIntegrator::setCrystalType(Crystal c) {
  switch (c) {
    case Crystal::Cubic: m_Dof = 1; break;
    case Crystal::Tetragonal: m_Dof = 2; break;
    case Crystal::Orthorhombic: m_Dof = 3; break;
    default:
      throw std::invalid_argument("CudaLangevinPiston::setCrystalType: crystalType must be either "
                                  "CRYSTAL::CUBIC, CRYSTAL::TETRAGONAL, or CRYSTAL::ORTHORHOMBIC");
  }
  m_Crystal = c;
  // default piston mass 0.02 x total mass and no friction, as the reference
  // sets them with the crystal type (src/CudaLangevinPistonIntegrator.cu:183-213)
  double tm = -9999.9999;
  if (m_Ctx) {
    tm = 0.0;
    for (double mm : m_Ctx->getForceManager()->topology().mass) tm += mm;
    tm *= 0.02;
  }
  m_PMass.assign(m_Dof, tm);
  m_PGamma = 0.0;
  m_RngDirty = true;
  clearGraphs();  // the captured steps hold the crystal type and the piston constants
}

void CudaLangevinPistonIntegrator::setPressure(const std::vector<double> &p) {
  if (p.size() != 9)
    throw std::invalid_argument("CudaLangevinPistonIntegrator::setPressure: reference pressure "
                                "must be of length 9 (XX, XY, XZ, YX, YY, YZ, ZX, ZY, ZZ)");
  m_Pref = p;
  if (m_P) {
    APO_CUDA(cudaStreamSynchronize(stream()));
    APO_CUDA(cudaMemcpy(reinterpret_cast<char *>(m_P->ps.p) + offsetof(PistonScalars, pref),
                        m_Pref.data(), 9 * sizeof(double), cudaMemcpyHostToDevice));
  }
}

void CudaLangevinPistonIntegrator::setLangevinPistonMass(const std::vector<double> &m) {
  if (m_Dof == -1)
    throw std::runtime_error("CudaLangevinPistonIntegrator::setLangevinPistonMass: CrystalType "
                             "must be set before Langevin piston mass");
  if ((int)m.size() != m_Dof)
    throw std::invalid_argument("CudaLangevinPistonIntegrator::setLangevinPistonMass: length of "
                                "input vector must be equal to the degrees of freedom of the "
                                "Langevin piston (" + std::to_string(m_Dof) + ")");
  m_PMass = m;
  clearGraphs();
}

void CudaLangevinPistonIntegrator::setNoseHooverPistonMass(double m) {
  m_NHMass = m;
  if (m_P) {
    APO_CUDA(cudaStreamSynchronize(stream()));
    APO_CUDA(cudaMemcpy(reinterpret_cast<char *>(m_S->sc.p) + offsetof(Scalars, piston_mass), &m,
                        sizeof(double), cudaMemcpyHostToDevice));
  }
}

void CudaLangevinPistonIntegrator::setLangevinPistonFrictionSeed(uint64_t seed) {
  // the states are drawn again from the new seed at the current position
  // (the reference's initializeRng with m_RngSequencePos)
  m_RngPos = getRngSequencePos();
  m_Seed = seed;
  m_RngDirty = true;
}

void CudaLangevinPistonIntegrator::setRngSequencePos(unsigned long long pos) {
  m_RngPos = pos;
  m_RngDirty = true;
}

unsigned long long CudaLangevinPistonIntegrator::getRngSequencePos() {
  if (!m_P || m_RngDirty) return m_RngPos;
  PistonScalars h;
  APO_CUDA(cudaStreamSynchronize(stream()));
  APO_CUDA(cudaMemcpy(&h, m_P->ps.p, sizeof(h), cudaMemcpyDeviceToHost));
  return h.rngpos;
}

void CudaLangevinPistonIntegrator::setMaxPredictorCorrectorIterations(int n) {
  if (n < 1)
    throw std::invalid_argument("setMaxPredictorCorrectorIterations: at least one pass is needed");
  m_MaxPC = n;
  m_KernelsPerStep = 3 + m_MaxPC;
  clearGraphs();
}

void CudaLangevinPistonIntegrator::resetAverages() {
  if (!m_P) return;
  resetAverageTemperature();
  PistonScalars h;
  APO_CUDA(cudaMemcpy(&h, m_P->ps.p, sizeof(h), cudaMemcpyDeviceToHost));
  for (double &x : h.pavg) x = 0.0;
  h.pavg_scalar = 0.0;
  APO_CUDA(cudaMemcpy(m_P->ps.p, &h, sizeof(h), cudaMemcpyHostToDevice));
}

namespace {
PistonScalars read_piston(const std::unique_ptr<PistonState> &P, cudaStream_t s) {
  if (!P) throw std::runtime_error("CudaLangevinPistonIntegrator: no CharmmContext was set");
  PistonScalars h;
  APO_CUDA(cudaStreamSynchronize(s));
  APO_CUDA(cudaMemcpy(&h, P->ps.p, sizeof(h), cudaMemcpyDeviceToHost));
  return h;
}
}  // namespace

std::vector<double> CudaLangevinPistonIntegrator::getInstantaneousPressureTensor() {
  const PistonScalars h = read_piston(m_P, stream());
  return std::vector<double>(h.p, h.p + 9);
}
double CudaLangevinPistonIntegrator::getInstantaneousPressureScalar() {
  return read_piston(m_P, stream()).pscalar;
}
std::vector<double> CudaLangevinPistonIntegrator::getAveragePressureTensor() {
  const PistonScalars h = read_piston(m_P, stream());
  return std::vector<double>(h.pavg, h.pavg + 9);
}
double CudaLangevinPistonIntegrator::getAveragePressureScalar() {
  return read_piston(m_P, stream()).pavg_scalar;
}
std::vector<double> CudaLangevinPistonIntegrator::getLangevinPistonOnStepPosition() {
  const PistonScalars h = read_piston(m_P, stream());
  return std::vector<double>(h.lp_onpos, h.lp_onpos + std::max(m_Dof, 0));
}
std::vector<double> CudaLangevinPistonIntegrator::getLangevinPistonDeltaPosition() {
  const PistonScalars h = read_piston(m_P, stream());
  return std::vector<double>(h.lp_delta, h.lp_delta + std::max(m_Dof, 0));
}

std::vector<double> CudaLangevinPistonIntegrator::getLangevinPistonHalfStepPosition() {
  const PistonScalars h = read_piston(m_P, stream());
  return std::vector<double>(h.lp_halfpos, h.lp_halfpos + std::max(m_Dof, 0));
}
std::vector<double> CudaLangevinPistonIntegrator::getLangevinPistonOnStepVelocity() {
  const PistonScalars h = read_piston(m_P, stream());
  return std::vector<double>(h.lp_onvel, h.lp_onvel + std::max(m_Dof, 0));
}
std::vector<double> CudaLangevinPistonIntegrator::getLangevinPistonDeltaPressure() {
  const PistonScalars h = read_piston(m_P, stream());
  return std::vector<double>(h.lp_dpress, h.lp_dpress + std::max(m_Dof, 0));
}
double CudaLangevinPistonIntegrator::getInstantaneousSurfaceTension() {
  // 0.5 Lz (Pzz - (Pxx + Pyy) / 2) / factor
  // (src/CudaLangevinPistonIntegrator.cu:533-541)
  const PistonScalars h = read_piston(m_P, stream());
  return 0.5 * h.box[2] * (h.p[8] - 0.5 * (h.p[0] + h.p[4])) / kSurfaceTensionFactor;
}
std::vector<double> CudaLangevinPistonIntegrator::getNoseHooverPistonState() {
  if (!m_S) throw std::runtime_error("CudaLangevinPistonIntegrator: no CharmmContext was set");
  Scalars h;
  APO_CUDA(cudaStreamSynchronize(stream()));
  APO_CUDA(cudaMemcpy(&h, m_S->sc.p, sizeof(h), cudaMemcpyDeviceToHost));
  return {h.piston_v, h.piston_v_prev, h.piston_f, h.piston_f_prev};
}
void CudaLangevinPistonIntegrator::setNoseHooverPistonState(double v, double v_prev, double f,
                                                            double f_prev) {
  if (!m_S) throw std::runtime_error("CudaLangevinPistonIntegrator: no CharmmContext was set");
  Scalars h;
  APO_CUDA(cudaStreamSynchronize(stream()));
  APO_CUDA(cudaMemcpy(&h, m_S->sc.p, sizeof(h), cudaMemcpyDeviceToHost));
  h.piston_v = v;
  h.piston_v_prev = v_prev;
  h.piston_f = f;
  h.piston_f_prev = f_prev;
  APO_CUDA(cudaMemcpy(m_S->sc.p, &h, sizeof(h), cudaMemcpyHostToDevice));
}

void CudaLangevinPistonIntegrator::initialize() {
  auto fm = m_Ctx->getForceManager();
  if (fm->isMulti())
    throw std::invalid_argument("the Langevin piston scales one box: it is not available for a "
                                "multi-system context");
  if (m_Dof == -1)
    throw std::runtime_error("CudaLangevinPistonIntegrator::initialize: CrystalType must be set "
                             "before initialization (try setting the crystal type before setting "
                             "the Charmm Context)");
  double tm = 0.0;
  for (double mm : fm->topology().mass) tm += mm;
  if (m_NHMass == -9999.9999) m_NHMass = 0.2 * tm;
  if (m_PMass.empty() || m_PMass[0] == -9999.9999) m_PMass.assign(m_Dof, 0.02 * tm);
  IntegratorState &S = *m_S;
  cudaStream_t s = m_Ctx->stream();
  m_P = std::make_unique<PistonState>();
  PistonState &P = *m_P;
  P.ps.alloc(1);
  P.rng.alloc(3);
  P.partials.alloc((size_t)32 * std::max(S.blocks_groups, S.blocks_atoms) + 32);
  PistonScalars h{};
  const auto &box = fm->getBoxDimensions();
  for (int d = 0; d < 3; ++d) h.box[d] = h.box_pred[d] = box[d];
  for (int k = 0; k < 9; ++k) h.pref[k] = m_Pref[k];
  APO_CUDA(cudaMemcpy(P.ps.p, &h, sizeof(h), cudaMemcpyHostToDevice));
  Scalars sc{};
  sc.piston_mass = m_NHMass;
  APO_CUDA(cudaMemcpy(S.sc.p, &sc, sizeof(sc), cudaMemcpyHostToDevice));
  lp_rng_init_kernel<<<1, 32, 0, s>>>(P.rng.p, m_Dof, m_Seed, m_RngPos, P.ps.p);
  m_RngDirty = false;
  fm->useDeviceBox();
  clearGraphs();
  // as Nose-Hoover: constraints, first forces, the position-Verlet deltas
  // (src/CudaLangevinPistonIntegrator.cu:626-704)
  if (m_Ctx->isUsingHolonomicConstraints())
    init_constrain_kernel<<<S.blocks_groups, kThreads, 0, s>>>(S.c, 0);
  fm->calcForceChecked(m_Ctx->xyzq(), false, false, s);
  init_delta_kernel<<<S.blocks_atoms, kThreads, 0, s>>>(S.c, S.natom, 0.0);
  if (m_Ctx->isUsingHolonomicConstraints())
    init_constrain_kernel<<<S.blocks_groups, kThreads, 0, s>>>(S.c, 1);
  APO_LAUNCH_CHECK();
  APO_CUDA(cudaStreamSynchronize(s));
}

void CudaLangevinPistonIntegrator::applyRestartRecord(const RestartRecord &r) {
  const Crystal c = r.crystal == "CUBI" ? Crystal::Cubic
                    : r.crystal == "TETR" ? Crystal::Tetragonal
                    : r.crystal == "ORTH" ? Crystal::Orthorhombic
                                          : Crystal::None;
  if (c == Crystal::None)
    throw std::runtime_error("restart file: crystal type \"" + r.crystal +
                             "\" is not one the Langevin piston moves");
  // another crystal type resets the piston mass and friction to their
  // defaults, as the reference's reader does (it always calls setCrystalType)
  if (c != m_Crystal) setCrystalType(c);
  auto fm = m_Ctx->getForceManager();
  APO_CUDA(cudaStreamSynchronize(stream()));
  fm->updateBoxDimensions(r.box);
  PistonScalars h;
  APO_CUDA(cudaMemcpy(&h, m_P->ps.p, sizeof(h), cudaMemcpyDeviceToHost));
  for (int d = 0; d < 3; ++d) {
    h.box[d] = h.box_pred[d] = r.box[d];
    h.lp_delta[d] = d < m_Dof ? r.hdot[d] : 0.0;
  }
  APO_CUDA(cudaMemcpy(m_P->ps.p, &h, sizeof(h), cudaMemcpyHostToDevice));
  setLangevinPistonFrictionSeed(r.seed);
  // a file without the APO tag carries no RNG position (as the reference reads it)
  setRngSequencePos((r.apo && r.has_rng) ? r.rngpos : 0ull);
}

// the step after the forces: half step, the predictor-corrector passes, the
// final pass and the list's shifts moved with the new box, with the piston
// constants of the current settings (a setter drops the captured segments);
// the box itself is read and written on the device only
void CudaLangevinPistonIntegrator::stepKernels(cudaStream_t s) {
  IntegratorState &S = *m_S;
  PistonState &P = *m_P;
  auto fm = m_Ctx->getForceManager();
  PistonArgs a{};
  a.ps = P.ps.p;
  a.rng = P.rng.p;
  a.partials = P.partials.p;
  a.vir_fixed = fm->deviceVirial();
  a.setup = fm->deviceSetup();
  a.lsys = fm->deviceListDims();
  a.dbox = fm->deviceBox();
  // piston friction terms (setLangevinPistonFriction,
  // src/CudaLangevinPistonIntegrator.cu:262-283)
  const double kbt = kBoltz * m_RefT;
  const double pgam = kTimfac * m_Dt * m_PGamma;
  a.palpha = (1.0 - 0.5 * pgam) / (1.0 + 0.5 * pgam);
  a.pbfact = m_Dt * m_Dt / (1.0 + 0.5 * pgam);
  for (int i = 0; i < m_Dof; ++i) {
    a.inv_mass[i] = m_PMass[i] == 0.0 ? 0.0 : 1.0 / m_PMass[i];
    a.prfwd[i] = std::sqrt(2.0 * a.inv_mass[i] * pgam * kbt) / m_Dt;
  }
  a.st = m_SurfaceTension * kSurfaceTensionFactor;
  a.ke_ref = 0.5 * (double)m_Ctx->getDegreesOfFreedom() * kBoltz * m_RefT;
  a.crystal = (int)m_Crystal;
  a.dof = m_Dof;
  a.use_nh = m_UseNH ? 1 : 0;
  a.use_old = m_OldT ? 1 : 0;
  a.const_st = m_ConstST ? 1 : 0;
  a.hol = m_Ctx->isUsingHolonomicConstraints() ? 1 : 0;
  lp_half_kernel<<<S.blocks_groups, kThreads, 0, s>>>(S.c, a);
  for (int k = 0; k < m_MaxPC; ++k)
    lp_pc_kernel<<<S.blocks_atoms, kThreads, 0, s>>>(S.c, a, S.natom, k + 1 < m_MaxPC ? 1 : 0);
  lp_final_kernel<<<S.blocks_groups, kThreads, 0, s>>>(S.c, a);
  APO_LAUNCH_CHECK();
  const char *ps = reinterpret_cast<const char *>(P.ps.p);
  fm->neighborList().rescale_box_device(
      reinterpret_cast<const double *>(ps + offsetof(PistonScalars, box_old)),
      reinterpret_cast<const double *>(ps + offsetof(PistonScalars, box)), S.c.err, s);
}

void CudaLangevinPistonIntegrator::forcesForStep(cudaStream_t s) {
  // forces and virial; the sorted coordinates refreshed from the FP64 state
  // the step kernels wrote, the gradient slots cleared
  m_Ctx->getForceManager()->calcForce(m_Ctx->xyzq(), false, true, s, /*clear=*/true);
}

void CudaLangevinPistonIntegrator::adoptBox() {
  if (!m_P) return;
  PistonScalars h;
  APO_CUDA(cudaStreamSynchronize(stream()));
  APO_CUDA(cudaMemcpy(&h, m_P->ps.p, sizeof(h), cudaMemcpyDeviceToHost));
  m_Ctx->getForceManager()->adoptDeviceBox({h.box[0], h.box[1], h.box[2]});
}

void CudaLangevinPistonIntegrator::beforeReport() { adoptBox(); }

// Captured 20-step segments as for the other integrators (a list build,
// then the steps; the list follows the box in between, the box never
// leaves the device); the host copies of the box are refreshed before
// every subscriber report and at the end.
void CudaLangevinPistonIntegrator::propagate(int numSteps) {
  if (!m_Ctx)
    throw std::invalid_argument("CudaIntegrator::propagate: no CharmmContext was set for this CudaIntegrator.");
  if (numSteps <= 0) return;
  if (m_RngDirty) {
    lp_rng_init_kernel<<<1, 32, 0, stream()>>>(m_P->rng.p, m_Dof, m_Seed, m_RngPos, m_P->ps.p);
    APO_LAUNCH_CHECK();
    m_RngDirty = false;
  }
  try {
    CudaIntegrator::propagate(numSteps);
  } catch (...) {
    adoptBox();
    throw;
  }
  adoptBox();
}

// ---------------------------------------------------------------- leapfrog

CudaLeapFrogIntegrator::CudaLeapFrogIntegrator(double ps) : CudaIntegrator(ps) {
  m_KernelsPerStep = 1;
}

void CudaLeapFrogIntegrator::initialize() {}

void CudaLeapFrogIntegrator::stepKernels(cudaStream_t s) {
  IntegratorState &S = *m_S;
  leapfrog_kernel<<<S.blocks_atoms, kThreads, 0, s>>>(S.c, S.natom);
  APO_LAUNCH_CHECK();
}

}  // namespace apo
