// Smooth PME reciprocal space: charge spread, 3D real FFT, influence
// function, inverse FFT and force gather, all hand-written.
//
// Replaces CudaPMERecip (src/CudaPMERecip.cu) in its P1 "BOX" mode:
// spread_charge (:1935, body include/cuda_pme_spread.h), cuFFT R2C/C2R
// (:2547-2645), scalar_sum_ortho_kernel (:674-929), gather_force
// (:2381, body include/cuda_pme_gather.h), calc_self_energy (:2267).
//
// Pipeline (5 launches):
//   spread      int32 fixed-point atomics into the real grid (deterministic)
//   plane_fwd   one CTA per z-plane: R2C along x (two rows packed into one
//               complex FFT), C2C along y; the plane lives in shared memory
//   pencil      one CTA per (y-row, 16 x-columns): FFT along z, multiply by
//               the influence function (energy/virial reduced on the way),
//               inverse FFT along z
//   plane_inv   inverse of plane_fwd, writes the real potential grid
//   gather      gradient from the potential, 8 threads per atom
// The FFTs are in-place mixed-radix (2..8) shared-memory transforms.  A
// decimation-in-frequency pass leaves its output in digit-reversed order and
// a decimation-in-time pass takes digit-reversed input, so pairing them
// (z: DIF forward / DIT inverse, y: DIF forward stored as-is / DIT inverse,
// x: DIT forward from a scattered load / DIF inverse with a scattered store)
// needs no reordering pass at all.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <vector>

namespace apo {

// x / d for 0 <= x < 2^31 as a multiply-high and a shift (division by an
// invariant integer, Granlund & Montgomery 1994); mul == 0 means d == 1
struct FastDiv {
  unsigned mul, shift;
};
FastDiv make_fastdiv(unsigned d);
__host__ __device__ inline unsigned fdiv(unsigned x, FastDiv f) {
#ifdef __CUDA_ARCH__
  return f.mul ? (__umulhi(x, f.mul) >> f.shift) : x;
#else
  return f.mul ? (unsigned)(((unsigned long long)x * f.mul >> 32) >> f.shift) : x;
#endif
}

struct FftAxis {
  int n;
  int nrad;
  int radix[8];
  // per stage s: n / radix[s], and the sub-block length over the radix of
  // the decimation-in-frequency (n / radix[0..s]) and the decimation-in-time
  // (radix[s+1..]) passes
  FastDiv per_line[8], dif_mr[8], dit_mr[8];
  FastDiv by_n;      // x / n
  FastDiv by_nxc;    // x / (n/2 + 1)
  FastDiv by_nxcp;   // x / the even pitch of n/2 + 1
  FastDiv by_ngrp;   // x / ((n/2 + 1)/2 + 1): the real-to-complex split groups
};
// fills the fast divisors of an axis whose n, nrad and radix are set
void fill_axis_divisors(FftAxis &a);

struct PmeDims {
  // nxc = nx/2 + 1 complex values per half-spectrum row, stored with an
  // even pitch nxcp (rows of a multiple of 16 bytes, as a tensor-memory
  // copy needs)
  int nx, ny, nz, nxc, nxcp, order;
  float Lx, Ly, Lz;       // box
  double rLx, rLy, rLz;   // 1 / box, for the FP64 grid anchoring
  float kappa;
  FftAxis ax, ay, az;
};

// One system of a multi-system PME: its grid dimensions and its slices of
// the concatenated buffers.
struct PmeSysArgs {
  PmeDims d;
  int *qgrid;
  float2 *cgrid;
  float *phi;
  const float2 *tw;          // twiddles: x (nx), y (ny), z (nz)
  const float *prefac;       // B-spline moduli 1/|b|^2: x, y, z
  const double *prefac_d;
  long long *energy;         // this system's energy slots
  long long *virial;         // this system's virial slots
  int plane0, pencil0;       // first plane / pencil block of this system
};

class Pme {
 public:
  Pme() = default;
  ~Pme();
  Pme(const Pme &) = delete;
  Pme &operator=(const Pme &) = delete;

  void setup(int nx, int ny, int nz, int order, double kappa, double Lx, double Ly,
             double Lz);
  // sorted coordinates in, fixed-point gradients added to `force` (sorted
  // slot order, SoA with `stride`); ewks energy added to energy[kEEwks]
  // virial (non-null): also add the reciprocal virial (3x3, 2^32 fixed point)
  // origin (non-null): xyzq_s holds coordinates relative to a per-32-slot
  // origin (NeighborList::cl_origin)
  void compute(const float4 *xyzq_s, const int *counts, long long *force, int stride,
               long long *energy, bool calc_energy, bool fp64_influence, cudaStream_t s,
               long long *virial = nullptr, const float4 *origin = nullptr);
  // the individual stages (exposed for tests and profiling)
  void spread(const float4 *xyzq_s, const int *counts, cudaStream_t s,
              const float4 *origin = nullptr);
  void forward(cudaStream_t s);
  void convolve(long long *energy, bool calc_energy, bool fp64_influence, cudaStream_t s,
                long long *virial = nullptr);
  void backward(cudaStream_t s);
  void gather(const float4 *xyzq_s, const int *counts, long long *force, int stride,
              cudaStream_t s, const float4 *origin = nullptr);

  const PmeDims &dims() const { return m_d; }
  // the z pencils move their slabs with tiled tensor copies (on by default
  // where the driver offers the encoder); a copy that does not complete sets
  // kErrCopyTimeout in `err`
  void set_tensor_copies(bool on) { m_tma_on = on; }
  // the kernels read the box from device memory (x, y, z edges; null: the
  // box of set-up / set_box), for a box that changes every step
  void set_device_box(const double4 *p) { m_dbox = p; }
  // a new box on the same grid (the influence function is formed from the
  // box at every evaluation)
  void set_box(double Lx, double Ly, double Lz) {
    m_d.Lx = (float)Lx;
    m_d.Ly = (float)Ly;
    m_d.Lz = (float)Lz;
    m_d.rLx = 1.0 / Lx;
    m_d.rLy = 1.0 / Ly;
    m_d.rLz = 1.0 / Lz;
  }
  bool tensor_copies() const { return m_tma_on && m_tma; }
  void set_error_word(unsigned *err) { m_err = err; }
  int *qgrid = nullptr;     // nz*ny*nx int32 fixed point (zeroed by plane_fwd)
  float2 *cgrid = nullptr;  // nz * ny * nxc complex (y rows in digit-reversed order)
  float *phi = nullptr;     // nz*ny*nx real potential
  int max_slots = 0;

  static FftAxis plan_axis(int n);

 private:
  void release();
  PmeDims m_d{};
  CUtensorMap m_tmap{};     // the padded complex grid as floats [nz][ny][2 nxcp]
  bool m_tma = false, m_tma_on = true;
  unsigned *m_err = nullptr;
  const double4 *m_dbox = nullptr;
  float2 *m_tw = nullptr;   // twiddles: x (nx), y (ny), z (nz) consecutive
  float *m_prefac = nullptr;  // B-spline moduli 1/|b|^2: x, y, z consecutive
  double *m_prefac_d = nullptr;
};

// Reciprocal space of many independent systems (one spline order) with one
// launch per stage: blocks map to (system, plane) or (system, pencil)
// through tables, and spread/gather blocks (one 32-slot cluster each) take
// the cluster's system from the neighbour list.
struct PmeSystemSpec {
  int nx, ny, nz;
  double kappa, Lx, Ly, Lz;
};

class PmeMulti {
 public:
  PmeMulti() = default;
  ~PmeMulti();
  PmeMulti(const PmeMulti &) = delete;
  PmeMulti &operator=(const PmeMulti &) = delete;
  // energy (+ virial) slots of system s start at energy + s * energy_stride
  void setup(const std::vector<PmeSystemSpec> &systems, int order, long long *energy,
             int energy_stride, int max_slots);
  void compute(const float4 *xyzq_s, const float4 *origin, const int *cl_sys, const int *counts,
               long long *force, int stride, bool calc_energy, bool calc_virial,
               bool fp64_influence, cudaStream_t s);
  int num_systems() const { return (int)m_host.size(); }

 private:
  void release();
  std::vector<PmeSysArgs> m_host;
  PmeSysArgs *m_args = nullptr;
  int *m_plane_sys = nullptr, *m_pencil_sys = nullptr;
  int m_planes = 0, m_pencils = 0, m_order = 4, m_max_slots = 0;
  size_t m_plane_smem = 0;
  int *m_q = nullptr;
  float2 *m_c = nullptr;
  float *m_phi = nullptr;
  float2 *m_tw = nullptr;
  float *m_pf = nullptr;
  double *m_pfd = nullptr;
};

}  // namespace apo

namespace apo {

// Size of the file-scope device scratch area used by pme_reciprocal_static.
constexpr size_t kPmeStaticScratchBytes = size_t(8) << 20;  // 8 MiB

// Bytes of that area a grid needs (tables, charge grid, complex grid,
// potential grid, each 256-byte aligned).
size_t pme_static_scratch_bytes(int nx, int ny, int nz);

// Reciprocal-space gradient and energy of `n` charges (xyzq, device, any
// order) with the kernels of Pme, but with every buffer of its own carved
// from one file-scope __device__ array of kPmeStaticScratchBytes instead of
// device allocations.  Gradients (2^40 fixed point) are added to the
// caller's int64 SoA `grad` (x at [0, n), y at [stride, ...), z at
// [2 stride, ...)); the energy (ewks) is written to energy[0] (device) when
// `energy` is not null.  Calls on one device share the area and must not
// overlap in time.
void pme_reciprocal_static(const float4 *xyzq, int n, double Lx, double Ly, double Lz, int nx,
                           int ny, int nz, int order, double kappa, long long *grad, int stride,
                           double *energy, bool fp64_influence, cudaStream_t s);

}  // namespace apo
