// ForceManager / CharmmContext; see engine.h.
#include "engine.h"

#include <climits>
#include <type_traits>

#include <algorithm>
#include <cmath>
#include <random>
#include <sstream>

#include "device_util.cuh"

namespace apo {
namespace {

__global__ void fixed_to_global_kernel(int n, const long long *__restrict__ f, int stride,
                                       const int *__restrict__ glo2loc, double *__restrict__ out) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  int s = glo2loc[g];
  out[3 * g + 0] = (double)f[s] * kInvForceScale;
  out[3 * g + 1] = (double)f[stride + s] * kInvForceScale;
  out[3 * g + 2] = (double)f[2 * stride + s] * kInvForceScale;
}

// slot-order fixed-point gradient -> atom-order planes `ostride` apart
template <typename T>
__global__ void fixed_to_planes_kernel(int n, const long long *__restrict__ f, int stride,
                                       const int *__restrict__ glo2loc, T *__restrict__ out,
                                       int ostride) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  int s = glo2loc[g];
  if constexpr (std::is_integral<T>::value) {
    out[g] = f[s];
    out[ostride + g] = f[stride + s];
    out[2 * ostride + g] = f[2 * stride + s];
  } else {
    out[g] = (T)f[s] * (T)kInvForceScale;
    out[ostride + g] = (T)f[stride + s] * (T)kInvForceScale;
    out[2 * ostride + g] = (T)f[2 * stride + s] * (T)kInvForceScale;
  }
}

__global__ void xyzq_to_state_kernel(int n, const float4 *__restrict__ xq,
                                     double4 *__restrict__ c) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const float4 p = xq[g];
  c[g] = make_double4(p.x, p.y, p.z, p.w);
}

// one bonded component moved back into the box: its centroid, and a shift
// of one box length per axis where the centroid left [-L/2, L/2]
// (src/CharmmContext.cu:276-372).  Components of more than
// kSmallComponent atoms come first and take a warp each (centroid by a warp
// reduction); the rest take one thread each.
constexpr int kSmallComponent = 8;

__device__ __forceinline__ void component_box(const int2 g, const int *sys_of_atom,
                                              const double4 *boxes, double &Lx, double &Ly,
                                              double &Lz) {
  if (sys_of_atom) {  // several systems: this component's own box
    const double4 b = boxes[sys_of_atom[g.x]];
    Lx = b.x;
    Ly = b.y;
    Lz = b.z;
  }
}

__device__ __forceinline__ double image_shift(double gc, double L) {
  return gc < -0.5 * L ? L : (gc > 0.5 * L ? -L : 0.0);
}

__global__ void image_centering_kernel(double4 *__restrict__ c, float4 *__restrict__ xq,
                                       const int2 *__restrict__ groups, int ng, int nbig,
                                       int big_blocks, double Lx0, double Ly0, double Lz0,
                                       const int *__restrict__ sys_of_atom,
                                       const double4 *__restrict__ boxes) {
  double Lx = Lx0, Ly = Ly0, Lz = Lz0;
  if ((int)blockIdx.x < big_blocks) {  // a warp per large component
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= nbig) return;
    const int2 g = groups[i];
    component_box(g, sys_of_atom, boxes, Lx, Ly, Lz);
    double gx = 0, gy = 0, gz = 0;
    for (int j = g.x + lane; j <= g.y; j += 32) {
      gx += c[j].x;
      gy += c[j].y;
      gz += c[j].z;
    }
    gx = warp_sum(gx);
    gy = warp_sum(gy);
    gz = warp_sum(gz);
    const double inv = 1.0 / (double)(g.y - g.x + 1);
    const double sx = image_shift(gx * inv, Lx), sy = image_shift(gy * inv, Ly),
                 sz = image_shift(gz * inv, Lz);
    if (sx != 0.0 || sy != 0.0 || sz != 0.0) {
      for (int j = g.x + lane; j <= g.y; j += 32) {
        c[j].x += sx;
        c[j].y += sy;
        c[j].z += sz;
        xq[j].x += (float)sx;
        xq[j].y += (float)sy;
        xq[j].z += (float)sz;
      }
    }
    return;
  }
  const int i = nbig + ((int)blockIdx.x - big_blocks) * blockDim.x + threadIdx.x;
  if (i >= ng) return;  // a thread per small component
  const int2 g = groups[i];
  component_box(g, sys_of_atom, boxes, Lx, Ly, Lz);
  double4 a[kSmallComponent];
  const int m = g.y - g.x + 1;
  double gx = 0, gy = 0, gz = 0;
#pragma unroll
  for (int k = 0; k < kSmallComponent; ++k) {
    if (k < m) {
      a[k] = c[g.x + k];
      gx += a[k].x;
      gy += a[k].y;
      gz += a[k].z;
    }
  }
  const double inv = 1.0 / (double)m;
  const double sx = image_shift(gx * inv, Lx), sy = image_shift(gy * inv, Ly),
               sz = image_shift(gz * inv, Lz);
  if (sx != 0.0 || sy != 0.0 || sz != 0.0) {
#pragma unroll
    for (int k = 0; k < kSmallComponent; ++k) {
      if (k < m) {
        const int j = g.x + k;
        c[j] = make_double4(a[k].x + sx, a[k].y + sy, a[k].z + sz, a[k].w);
        float4 f = xq[j];
        f.x += (float)sx;
        f.y += (float)sy;
        f.z += (float)sz;
        xq[j] = f;
      }
    }
  }
}

__global__ void coords_to_xyzq_kernel(const double4 *__restrict__ c, float4 *__restrict__ xq,
                                      int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const double4 v = c[i];
    xq[i] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)v.w);
  }
}

}  // namespace

void launch_image_centering(double4 *coords, float4 *xyzq, const int2 *groups, int ngroups,
                            int nbig, double Lx, double Ly, double Lz, cudaStream_t s,
                            const int *sys_of_atom, const double4 *boxes) {
  if (ngroups <= 0) return;
  const int big_blocks = (nbig + 3) / 4;  // 4 warps a block
  const int small_blocks = (ngroups - nbig + 127) / 128;
  image_centering_kernel<<<big_blocks + small_blocks, 128, 0, s>>>(
      coords, xyzq, groups, ngroups, nbig, big_blocks, Lx, Ly, Lz, sys_of_atom, boxes);
  APO_LAUNCH_CHECK();
}

int order_components(std::vector<int2> &groups, int small) {
  std::stable_partition(groups.begin(), groups.end(),
                        [small](const int2 &g) { return g.y - g.x + 1 > small; });
  int nbig = 0;
  for (const int2 &g : groups) nbig += g.y - g.x + 1 > small ? 1 : 0;
  return nbig;
}

void launch_coords_to_xyzq(const double4 *coords, float4 *xyzq, int n, cudaStream_t s) {
  coords_to_xyzq_kernel<<<(n + 255) / 256, 256, 0, s>>>(coords, xyzq, n);
  APO_LAUNCH_CHECK();
}

// ------------------------------------------------------------- ForceManager

ForceManager::ForceManager(std::shared_ptr<CharmmPSF> psf, std::shared_ptr<CharmmParameters> prm)
    : m_Psf(std::move(psf)), m_Prm(std::move(prm)) {
  if (!m_Psf || !m_Prm) throw std::invalid_argument("ForceManager: null PSF or parameters");
}

ForceManager::ForceManager(const std::vector<SystemSpec> &systems, int order, int tilesPerWork,
                           bool precise)
    : m_Multi(true), m_Specs(systems) {
  if (systems.empty()) throw std::invalid_argument("ForceManager: no systems");
  m_Order = order;
  m_TilesPerWork = tilesPerWork;
  m_Precise = precise;
  initializeMulti();
}

ForceManager::~ForceManager() {
  for (cudaStream_t s : {m_SNb, m_SPme, m_SBond})
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t e : {m_EvFork, m_EvNb, m_EvPme, m_EvBond})
    if (e) cudaEventDestroy(e);
  for (auto &p : m_Timers) {
    cudaEventDestroy(p.first);
    cudaEventDestroy(p.second);
  }
}

void ForceManager::setBoxDimensions(const std::array<double, 3> &box) {
  for (double b : box)
    if (b < 0)
      throw std::invalid_argument("Box dimensions: " + std::to_string(box[0]) + " x " +
                                  std::to_string(box[1]) + " x " + std::to_string(box[2]) +
                                  " are NOT valid");
  m_Box = box;
  m_Initialized = false;
}

void ForceManager::updateBoxDimensions(const std::array<double, 3> &box) {
  if (!m_Initialized) throw std::runtime_error("ForceManager is not initialized");
  if (m_Multi)
    throw std::invalid_argument("updateBoxDimensions: a multi-system force manager keeps its boxes");
  for (double b : box)
    if (!(b > 0.0) || !std::isfinite(b))
      throw std::invalid_argument("Box dimensions: " + std::to_string(box[0]) + " x " +
                                  std::to_string(box[1]) + " x " + std::to_string(box[2]) +
                                  " are NOT valid");
  for (double b : box)
    if (m_Cutoff > b / 2.0)
      throw std::runtime_error("the box shrank below twice the cutoff (" + std::to_string(b) +
                               " A edge, cutoff " + std::to_string(m_Cutoff) + " A)");
  m_Box = box;
  m_HostSetup = make_nb_setup(m_Box[0], m_Box[1], m_Box[2], m_Kappa, m_Ctofnb, m_Ctonnb);
  APO_CUDA(cudaMemcpy(m_Setup.p, &m_HostSetup, sizeof(NbSetup), cudaMemcpyHostToDevice));
  m_Nbl.set_box(0, m_Box[0], m_Box[1], m_Box[2]);
  m_ListDirty = true;
  m_Pme.set_box(m_Box[0], m_Box[1], m_Box[2]);
  if (m_DevBox.p) {
    const double4 b = make_double4(m_Box[0], m_Box[1], m_Box[2], 0.0);
    APO_CUDA(cudaMemcpy(m_DevBox.p, &b, sizeof(b), cudaMemcpyHostToDevice));
  }
  ++m_PluginGen;  // captured graphs hold the old box
}

void ForceManager::useDeviceBox() {
  if (!m_Initialized) throw std::runtime_error("ForceManager is not initialized");
  if (m_Multi) throw std::invalid_argument("useDeviceBox: one system only");
  if (!m_DevBox.p) m_DevBox.alloc(1);
  const double4 b = make_double4(m_Box[0], m_Box[1], m_Box[2], 0.0);
  APO_CUDA(cudaMemcpy(m_DevBox.p, &b, sizeof(b), cudaMemcpyHostToDevice));
  m_Pme.set_device_box(m_DevBox.p);
  ++m_PluginGen;  // captured graphs hold the launches without it
}

void ForceManager::adoptDeviceBox(const std::array<double, 3> &box) {
  m_Box = box;
  m_HostSetup = make_nb_setup(m_Box[0], m_Box[1], m_Box[2], m_Kappa, m_Ctofnb, m_Ctonnb);
  m_Nbl.set_box_host(0, m_Box[0], m_Box[1], m_Box[2]);
  m_Pme.set_box(m_Box[0], m_Box[1], m_Box[2]);
}

void ForceManager::setFFTGrid(int nx, int ny, int nz) {
  m_Nfft[0] = nx;
  m_Nfft[1] = ny;
  m_Nfft[2] = nz;
  m_Initialized = false;
}

void ForceManager::setDirectKernel(int v) {
  if (v != kNbTileBatches && v != kNbGroupedQueues && v != kNbOctetLists)
    throw std::invalid_argument("direct-space kernel form must be 0 (tile batches), 1 "
                                "(grouped queues) or 2 (octet lists)");
  m_NbVariant = v;
}

void ForceManager::setVdwType(int type) {
  if (type != VDW_VFSW)
    throw std::invalid_argument("only the VDW_VFSW (force switch) Lennard-Jones model is "
                                "implemented on this engine");
  m_VdwType = type;
}

void ForceManager::setPeriodicBoundaryCondition(PBC pbc) {
  if (pbc != PBC::P1)
    throw std::invalid_argument("only P1 periodic boundary conditions are implemented");
}

std::array<int, 3> ForceManager::computeFFTGridSize() const {
  // 2 * floor(L/2) (src/ForceManager.cu:923-944)
  std::array<int, 3> n;
  for (int d = 0; d < 3; ++d) n[d] = std::max(2, 2 * ((int)m_Box[d] / 2));
  return n;
}

void ForceManager::initialize() {
  if (m_Multi) {
    initializeMulti();
    return;
  }
  if (m_Box[0] == -9999.9999 || m_Box[1] == -9999.9999 || m_Box[2] == -9999.9999)
    throw std::invalid_argument("Error: Box dimension was not set");
  if (m_Cutoff <= 0.0 || m_Cutoff > m_Box[0] / 2.0)
    throw std::invalid_argument("Error: Cutoff value (" + std::to_string(m_Cutoff) +
                                ") not valid (boxx: " + std::to_string(m_Box[0]) + ")");
  if (m_Ctofnb > m_Cutoff)
    throw std::invalid_argument("ctofnb must not exceed the list cutoff (cutnb)");
  if (m_Nfft[0] <= 0 || m_Nfft[1] <= 0 || m_Nfft[2] <= 0) {
    auto n = computeFFTGridSize();
    setFFTGrid(n[0], n[1], n[2]);
  }
  m_Top = build_topology(*m_Psf, *m_Prm);
  const int n = m_Top.natom;

  m_VdwTypeD.upload(m_Top.vdwtype);
  m_Vdw.upload(m_Top.vdw);
  m_Vdw14.upload(m_Top.vdw14);
  m_BondIJ.upload(m_Top.bond_ij);
  m_BondP.upload(m_Top.bond_p);
  m_UbIJ.upload(m_Top.ub_ij);
  m_UbP.upload(m_Top.ub_p);
  m_AngleIJK.upload(m_Top.angle_ijk);
  m_AngleP.upload(m_Top.angle_p);
  m_DiheIJKL.upload(m_Top.dihe_ijkl);
  m_DiheTerms.upload(m_Top.dihe_terms);
  m_DiheCoef.upload(m_Top.dihe_coef);
  m_ImpIJKL.upload(m_Top.imp_ijkl);
  m_ImpP.upload(m_Top.imp_p);
  m_In14.upload(m_Top.in14);
  m_Ex14.upload(m_Top.ex14);

  // the reference's direct-space set-up uses roff = ctofnb, ron = ctonnb
  // (src/ForceManager.cu:513-514)
  m_HostSetup = make_nb_setup(m_Box[0], m_Box[1], m_Box[2], m_Kappa, m_Ctofnb, m_Ctonnb);
  m_Setup.upload(std::vector<NbSetup>{m_HostSetup});

  m_Nbl.setup(n, m_Box[0], m_Box[1], m_Box[2], (float)m_Cutoff,
              m_Top.excl_ptr, m_Top.excl_idx, m_VdwTypeD.p, m_TilesPerWork);
  m_Pme.setup(m_Nfft[0], m_Nfft[1], m_Nfft[2], m_Order, m_Kappa, m_Box[0], m_Box[1], m_Box[2]);
  m_Pme.max_slots = m_Nbl.dims().slot_cap;
  m_Pme.set_error_word(m_Nbl.error);
  m_Pme.set_tensor_copies(m_PmeTensorCopies);
  m_Stride = m_Nbl.dims().slot_cap;
  m_Force.alloc((size_t)3 * m_Stride);
  APO_CUDA(cudaMemset(m_Force.p, 0, (size_t)3 * m_Stride * sizeof(long long)));
  // energy terms, then the 3x3 virial (row major), all 2^32 fixed point
  m_Energy.alloc(kNumEnergyTerms + 9);
  APO_CUDA(cudaMemset(m_Energy.p, 0, (kNumEnergyTerms + 9) * sizeof(long long)));

  double q2 = 0.0;
  for (double q : m_Top.charge) q2 += q * q;
  m_SelfEnergy = -m_Kappa * kCcelec / std::sqrt(M_PI) * q2;

  createStreams();
  m_ListBuilt = false;
  m_Initialized = true;
  for (auto &p : m_Plugins) p.second->initialize(m_Top.natom, m_Box);
}

void ForceManager::createStreams() {
  if (!m_SNb) {
    // the reciprocal-space chain (five dependent, latency-bound kernels) and
    // the bonded kernel get the higher priority: their blocks go first
    // whenever direct-space blocks retire
    int lo = 0, hi = 0;
    APO_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    APO_CUDA(cudaStreamCreateWithPriority(&m_SNb, cudaStreamNonBlocking, lo));
    APO_CUDA(cudaStreamCreateWithPriority(&m_SPme, cudaStreamNonBlocking, hi));
    APO_CUDA(cudaStreamCreateWithPriority(&m_SBond, cudaStreamNonBlocking, hi));
    for (cudaEvent_t *e : {&m_EvFork, &m_EvNb, &m_EvPme, &m_EvBond})
      APO_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  }
}

namespace {

template <typename T>
void append(std::vector<T> &dst, const std::vector<T> &src) {
  dst.insert(dst.end(), src.begin(), src.end());
}
int2 shift2(int2 v, int o) { return make_int2(v.x + o, v.y + o); }
int4 shift4(int4 v, int o, int n) {  // first n components are atoms (-1 stays -1)
  int *c = &v.x;
  for (int k = 0; k < n; ++k)
    if (c[k] >= 0) c[k] += o;
  return v;
}

}  // namespace

void ForceManager::initializeMulti() {
  m_SysTop.clear();
  m_AtomOff.assign(1, 0);
  m_SelfEnergies.clear();
  Topology T;
  std::vector<NbSetup> setups;
  std::vector<NbListSystem> lists;
  std::vector<PmeSystemSpec> pmes;
  std::vector<double4> boxes;
  for (size_t k = 0; k < m_Specs.size(); ++k) {
    SystemSpec &y = m_Specs[k];
    if (!y.psf || !y.prm) throw std::invalid_argument("ForceManager: null PSF or parameters");
    for (double b : y.box)
      if (!(b > 0.0)) throw std::invalid_argument("ForceManager: system box must be positive");
    if (y.cutnb <= 0.0 || y.cutnb > y.box[0] / 2.0 || y.cutnb > y.box[1] / 2.0 ||
        y.cutnb > y.box[2] / 2.0)
      throw std::invalid_argument("ForceManager: list cutoff exceeds half the box");
    if (y.ctofnb > y.cutnb) throw std::invalid_argument("ctofnb must not exceed the list cutoff (cutnb)");
    for (int d = 0; d < 3; ++d)
      if (y.nfft[d] <= 0) y.nfft[d] = std::max(2, 2 * ((int)y.box[d] / 2));
    Topology t = y.topology ? *y.topology : build_topology(*y.psf, *y.prm);
    if (t.natom != y.psf->getNumAtoms())
      throw std::invalid_argument("ForceManager: a system's topology does not match its PSF");
    if ((int)t.types.size() > kMaxMultiTypes)
      throw std::invalid_argument("ForceManager: a system of a multi-system manager has more than " +
                                  std::to_string(kMaxMultiTypes) + " Lennard-Jones types");
    const int off = T.natom;
    NbSetup su = make_nb_setup(y.box[0], y.box[1], y.box[2], y.kappa, y.ctofnb, y.ctonnb);
    su.vdw_off = (int)T.vdw.size();
    su.vdw14_off = (int)T.vdw14.size();
    su.ntype = (int)t.types.size();
    setups.push_back(su);
    lists.push_back(NbListSystem{t.natom, y.box[0], y.box[1], y.box[2], (float)y.cutnb});
    pmes.push_back(PmeSystemSpec{y.nfft[0], y.nfft[1], y.nfft[2], y.kappa, y.box[0], y.box[1],
                                 y.box[2]});
    boxes.push_back(make_double4(y.box[0], y.box[1], y.box[2], 0.0));
    double q2 = 0.0;
    for (double q : t.charge) q2 += q * q;
    m_SelfEnergies.push_back(-y.kappa * kCcelec / std::sqrt(M_PI) * q2);
    // concatenate, atom indices shifted by the system's offset
    append(T.charge, t.charge);
    append(T.mass, t.mass);
    append(T.vdwtype, t.vdwtype);
    append(T.vdw, t.vdw);
    append(T.vdw14, t.vdw14);
    if (T.excl_ptr.empty()) T.excl_ptr.push_back(0);
    const int ebase = (int)T.excl_idx.size();
    for (int a = 1; a <= t.natom; ++a) T.excl_ptr.push_back(ebase + t.excl_ptr[a]);
    for (int e : t.excl_idx) T.excl_idx.push_back(e + off);
    for (auto v : t.in14) T.in14.push_back(shift2(v, off));
    for (auto v : t.ex14) T.ex14.push_back(shift2(v, off));
    for (auto v : t.bond_ij) T.bond_ij.push_back(shift2(v, off));
    append(T.bond_p, t.bond_p);
    for (auto v : t.ub_ij) T.ub_ij.push_back(shift2(v, off));
    append(T.ub_p, t.ub_p);
    for (auto v : t.angle_ijk) T.angle_ijk.push_back(shift4(v, off, 3));
    append(T.angle_p, t.angle_p);
    const int cbase = (int)T.dihe_coef.size();
    for (auto v : t.dihe_ijkl) T.dihe_ijkl.push_back(shift4(v, off, 4));
    for (auto v : t.dihe_terms) T.dihe_terms.push_back(make_int2(v.x + cbase, v.y));
    append(T.dihe_coef, t.dihe_coef);
    for (auto v : t.imp_ijkl) T.imp_ijkl.push_back(shift4(v, off, 4));
    append(T.imp_p, t.imp_p);
    for (auto v : t.waters) T.waters.push_back(shift4(v, off, 3));
    for (auto v : t.shake_atoms) T.shake_atoms.push_back(shift4(v, off, 4));
    append(T.shake_p, t.shake_p);
    for (auto v : t.groups) T.groups.push_back(shift2(v, off));
    T.natom += t.natom;
    m_AtomOff.push_back(T.natom);
    m_SysTop.push_back(std::move(t));
  }
  if (T.excl_ptr.empty()) T.excl_ptr.push_back(0);
  T.types = m_SysTop[0].types;  // per-system tables are addressed through the set-ups
  m_Top = std::move(T);
  m_Box = m_Specs[0].box;
  m_Kappa = m_Specs[0].kappa;
  m_Cutoff = m_Specs[0].cutnb;
  m_Ctonnb = m_Specs[0].ctonnb;
  m_Ctofnb = m_Specs[0].ctofnb;
  for (int d = 0; d < 3; ++d) m_Nfft[d] = m_Specs[0].nfft[d];
  m_HostSetup = setups[0];

  m_VdwTypeD.upload(m_Top.vdwtype);
  m_Vdw.upload(m_Top.vdw);
  m_Vdw14.upload(m_Top.vdw14);
  m_BondIJ.upload(m_Top.bond_ij);
  m_BondP.upload(m_Top.bond_p);
  m_UbIJ.upload(m_Top.ub_ij);
  m_UbP.upload(m_Top.ub_p);
  m_AngleIJK.upload(m_Top.angle_ijk);
  m_AngleP.upload(m_Top.angle_p);
  m_DiheIJKL.upload(m_Top.dihe_ijkl);
  m_DiheTerms.upload(m_Top.dihe_terms);
  m_DiheCoef.upload(m_Top.dihe_coef);
  m_ImpIJKL.upload(m_Top.imp_ijkl);
  m_ImpP.upload(m_Top.imp_p);
  m_In14.upload(m_Top.in14);
  m_Ex14.upload(m_Top.ex14);
  m_Setup.upload(setups);
  m_Boxes.upload(boxes);

  m_Nbl.setup(lists, m_Top.excl_ptr, m_Top.excl_idx, m_VdwTypeD.p, m_TilesPerWork);
  m_Stride = m_Nbl.dims().slot_cap;
  m_Force.alloc((size_t)3 * m_Stride);
  APO_CUDA(cudaMemset(m_Force.p, 0, (size_t)3 * m_Stride * sizeof(long long)));
  m_EStride = kNumEnergyTerms + 9;
  m_Energy.alloc((size_t)m_EStride * m_Specs.size());
  APO_CUDA(cudaMemset(m_Energy.p, 0, m_Energy.n * sizeof(long long)));
  m_PmeMulti.setup(pmes, m_Order, m_Energy.p, m_EStride, m_Stride);
  createStreams();
  m_ListBuilt = false;
  m_Initialized = true;
}

void ForceManager::resetNeighborList(const float4 *d_xyzq, cudaStream_t s) {
  if (!m_Initialized) throw std::runtime_error("ForceManager is not initialized");
  if (!m_ListBuilt) {
    // first build: size the tile buffers from the real demand (synchronous)
    m_Nbl.ensure_capacity(d_xyzq, s);
    m_ListBuilt = true;
  } else {
    m_Nbl.build(d_xyzq, s);
  }
  m_ListDirty = false;
}

void ForceManager::setListCapacity(int tiles) {
  if (!m_Initialized) throw std::runtime_error("ForceManager is not initialized");
  if (tiles < 1) throw std::invalid_argument("ForceManager::setListCapacity: capacity must be positive");
  const int ncl = m_Nbl.dims().slot_cap / kTile;
  m_Nbl.set_capacity(tiles, tiles / std::max(1, m_Nbl.dims().tiles_per_work) + ncl + 16);
  // no tile or work item is published until the next build fills the new
  // buffers
  APO_CUDA(cudaMemset(m_Nbl.counts + 1, 0, 4 * sizeof(int)));
  m_ListDirty = true;
  ++m_PluginGen;  // the captured graphs hold the old buffers
}

void ForceManager::setPmeTensorCopies(bool on) {
  m_PmeTensorCopies = on;
  m_Pme.set_tensor_copies(on);
  ++m_PluginGen;  // captured graphs hold the other kernel form
}

void ForceManager::calcForceChecked(const float4 *d_xyzq, bool calcEnergy, bool calcVirial,
                                    cudaStream_t s) {
  calcForce(d_xyzq, calcEnergy, calcVirial, s, true);
  APO_CUDA(cudaStreamSynchronize(s));
  const unsigned e = readDeviceError(s);
  if (e & kErrCopyTimeout)
    throw std::runtime_error("a tensor copy of the reciprocal-space grid did not complete");
  if (e & (kErrTileOverflow | kErrWorkOverflow)) {
    growNeighborList(d_xyzq, s);
    calcForce(d_xyzq, calcEnergy, calcVirial, s, true);
    APO_CUDA(cudaStreamSynchronize(s));
  }
}

bool ForceManager::growNeighborList(const float4 *d_xyzq, cudaStream_t s) {
  APO_CUDA(cudaStreamSynchronize(s));
  const int t0 = m_Nbl.dims().tile_cap, w0 = m_Nbl.dims().work_cap;
  m_Nbl.clear_error(s);
  m_Nbl.ensure_capacity(d_xyzq, s);
  m_Nbl.clear_error(s);
  APO_CUDA(cudaStreamSynchronize(s));
  const bool moved = m_Nbl.dims().tile_cap != t0 || m_Nbl.dims().work_cap != w0;
  if (moved) ++m_PluginGen;
  return moved;
}

void ForceManager::calcForce(const float4 *d_xyzq, bool calcEnergy, bool calcVirial,
                             cudaStream_t s, bool clear) {
  if (!m_Initialized) throw std::runtime_error("ForceManager is not initialized");
  if (!m_ListBuilt || m_ListDirty) resetNeighborList(d_xyzq, s);
  else if (clear) m_Nbl.refresh(s);
  if (clear) APO_CUDA(cudaMemsetAsync(m_Force.p, 0, (size_t)3 * m_Stride * sizeof(long long), s));
  if (calcVirial) calcEnergy = true;
  long long *virial = calcVirial ? m_Energy.p + kNumEnergyTerms : nullptr;
  if (m_Multi)
    APO_CUDA(cudaMemsetAsync(m_Energy.p, 0, m_Energy.n * sizeof(long long), s));
  else
    APO_CUDA(cudaMemsetAsync(m_Energy.p, 0,
                             (kNumEnergyTerms + (calcVirial ? 9 : 0)) * sizeof(long long), s));
  m_VirialValid = calcVirial;
  m_EvalMask = m_ComponentMask;
  APO_CUDA(cudaEventRecord(m_EvFork, s));
  if (m_ComponentMask & 2) {
    APO_CUDA(cudaStreamWaitEvent(m_SNb, m_EvFork, 0));
    NbArgs a;
    a.xyzq_s = m_Nbl.xyzq_s;
    a.origin = m_Nbl.cl_origin;
    a.perm = m_Nbl.perm;
    a.type_s = m_Nbl.type_s;
    a.tiles = m_Nbl.tiles;
    a.masks = m_Nbl.masks;
    a.work = m_Nbl.work;
    a.counts = m_Nbl.counts;
    a.vdw = m_Vdw.p;
    a.ntype = (int)m_Top.types.size();
    a.force = m_Force.p;
    a.stride = m_Stride;
    a.energy = m_Energy.p;
    a.setups = m_Setup.p;
    a.virial = virial;
    a.variant = m_NbVariant;
    a.sched = m_Nbl.counts + 6;  // counts[6..7]: zero between launches
    a.items_per_warp = m_ItemsPerWarp;
    a.work_cap = m_Nbl.dims().work_cap;
    cudaEvent_t t1 = nullptr;
    bool timer_capture = false;
    if (m_Timing) {
      if (m_TimerCursor >= (int)m_Timers.size()) {
        cudaEvent_t e0, e1;
        APO_CUDA(cudaEventCreate(&e0));
        APO_CUDA(cudaEventCreate(&e1));
        m_Timers.emplace_back(e0, e1);
      }
      // while the stream is captured, external records stay real event nodes
      cudaStreamCaptureStatus cs;
      APO_CUDA(cudaStreamIsCapturing(m_SNb, &cs));
      timer_capture = cs == cudaStreamCaptureStatusActive;
      if (timer_capture)
        APO_CUDA(cudaEventRecordWithFlags(m_Timers[m_TimerCursor].first, m_SNb,
                                          cudaEventRecordExternal));
      else
        APO_CUDA(cudaEventRecord(m_Timers[m_TimerCursor].first, m_SNb));
      t1 = m_Timers[m_TimerCursor].second;
      ++m_TimerCursor;
    }
    if (m_Multi) {
      a.energy_stride = m_EStride;
      launch_nonbonded_multi(a, calcEnergy, m_Precise, m_SNb, calcVirial);
    } else {
      launch_nonbonded(a, calcEnergy, m_Precise, m_SNb, calcVirial);
    }
    if (t1) {
      if (timer_capture) APO_CUDA(cudaEventRecordWithFlags(t1, m_SNb, cudaEventRecordExternal));
      else APO_CUDA(cudaEventRecord(t1, m_SNb));
    }
    APO_CUDA(cudaEventRecord(m_EvNb, m_SNb));
    APO_CUDA(cudaStreamWaitEvent(s, m_EvNb, 0));
  }
  if (m_ComponentMask & 4) {
    APO_CUDA(cudaStreamWaitEvent(m_SPme, m_EvFork, 0));
    if (m_Multi)
      m_PmeMulti.compute(m_Nbl.xyzq_s, m_Nbl.cl_origin, m_Nbl.cl_sys, m_Nbl.counts, m_Force.p,
                         m_Stride, calcEnergy, calcVirial, m_Precise, m_SPme);
    else
      m_Pme.compute(m_Nbl.xyzq_s, m_Nbl.counts, m_Force.p, m_Stride, m_Energy.p, calcEnergy,
                    m_Precise, m_SPme, virial, m_Nbl.cl_origin);
    APO_CUDA(cudaEventRecord(m_EvPme, m_SPme));
    APO_CUDA(cudaStreamWaitEvent(s, m_EvPme, 0));
  }
  // bonded terms proper; the 1-4 pairs and exclusion corrections go with
  // them or, under kComponent14WithDirect, with the direct space
  const bool bonded_proper = m_ComponentMask & 1;
  const bool pairs14 = (m_ComponentMask & kComponent14WithDirect) ? (m_ComponentMask & 2)
                                                                   : (m_ComponentMask & 1);
  if (bonded_proper || pairs14) {
    APO_CUDA(cudaStreamWaitEvent(m_SBond, m_EvFork, 0));
    BondedArgs b;
    if (!m_StateCoords) throw std::runtime_error("ForceManager: no state coordinates attached");
    b.coords = m_StateCoords;
    b.glo2loc = m_Nbl.glo2loc;
    b.force = m_Force.p;
    b.stride = m_Stride;
    b.energy = m_Energy.p;
    b.nbond = (int)m_BondIJ.n; b.bond_ij = m_BondIJ.p; b.bond_p = m_BondP.p;
    b.nub = (int)m_UbIJ.n; b.ub_ij = m_UbIJ.p; b.ub_p = m_UbP.p;
    b.nangle = (int)m_AngleIJK.n; b.angle_ijk = m_AngleIJK.p; b.angle_p = m_AngleP.p;
    b.ndihe = (int)m_DiheIJKL.n; b.dihe_ijkl = m_DiheIJKL.p; b.dihe_terms = m_DiheTerms.p;
    b.dihe_coef = m_DiheCoef.p;
    b.nimp = (int)m_ImpIJKL.n; b.imp_ijkl = m_ImpIJKL.p; b.imp_p = m_ImpP.p;
    b.nin14 = (int)m_In14.n; b.in14 = m_In14.p;
    b.nex14 = (int)m_Ex14.n; b.ex14 = m_Ex14.p;
    if (!bonded_proper) b.nbond = b.nub = b.nangle = b.ndihe = b.nimp = 0;
    if (!pairs14) b.nin14 = b.nex14 = 0;
    b.vdwtype = m_VdwTypeD.p;
    b.vdw14 = m_Vdw14.p;
    b.ntype = (int)m_Top.types.size();
    b.nb = m_HostSetup;
    b.virial = virial;
    if (m_Multi) {
      b.sys_of_atom = m_Nbl.sys_of_atom;
      b.setups = m_Setup.p;
      b.energy_stride = m_EStride;
      launch_bonded_multi(b, calcEnergy, m_SBond, calcVirial);
    } else {
      launch_bonded(b, calcEnergy, m_SBond, calcVirial);
    }
    APO_CUDA(cudaEventRecord(m_EvBond, m_SBond));
    APO_CUDA(cudaStreamWaitEvent(s, m_EvBond, 0));
  }
  if (!m_Plugins.empty()) {
    if (!m_StateCoords) throw std::runtime_error("ForceManager: no state coordinates attached");
    if (calcEnergy)
      APO_CUDA(cudaMemsetAsync(m_PluginEnergy.p, 0, kMaxPlugins * sizeof(long long), s));
    for (size_t k = 0; k < m_Plugins.size(); ++k) {
      ForcePluginArgs pa;
      pa.natom = m_Top.natom;
      pa.coords = m_StateCoords;
      pa.xyzq = d_xyzq;
      pa.glo2loc = m_Nbl.glo2loc;
      pa.force = m_Force.p;
      pa.stride = m_Stride;
      pa.energy = m_PluginEnergy.p + k;
      for (int d = 0; d < 3; ++d) pa.box[d] = m_Box[d];
      m_Plugins[k].second->calcForce(pa, calcEnergy, calcVirial, s);
    }
  }
}

void ForceManager::subscribe(std::shared_ptr<ForcePlugin> force, const std::string &tag) {
  if (!force) throw std::invalid_argument("ForceManager::subscribe: null force");
  if (m_Multi)
    throw std::invalid_argument("ForceManager::subscribe: plug-in forces need a single-system "
                                "force manager");
  if (tag.empty()) throw std::invalid_argument("ForceManager::subscribe: empty tag");
  for (int k = 0; k < kNumEnergyTerms; ++k)
    if (tag == kEnergyNames[k])
      throw std::invalid_argument("ForceManager::subscribe: tag '" + tag + "' names a built-in term");
  for (auto &p : m_Plugins)
    if (p.first == tag)
      throw std::invalid_argument("ForceManager::subscribe: tag '" + tag + "' is already in use");
  if ((int)m_Plugins.size() >= kMaxPlugins)
    throw std::invalid_argument("ForceManager::subscribe: at most 16 plug-in forces");
  if (!m_PluginEnergy.p) {
    m_PluginEnergy.alloc(kMaxPlugins);
    APO_CUDA(cudaMemset(m_PluginEnergy.p, 0, kMaxPlugins * sizeof(long long)));
  }
  if (m_Initialized) force->initialize(m_Top.natom, m_Box);
  m_Plugins.emplace_back(tag, std::move(force));
  ++m_PluginGen;
}

bool ForceManager::unsubscribe(const std::string &tag) {
  for (size_t k = 0; k < m_Plugins.size(); ++k)
    if (m_Plugins[k].first == tag) {
      m_Plugins.erase(m_Plugins.begin() + k);
      ++m_PluginGen;
      return true;
    }
  return false;
}

bool ForceManager::unsubscribe(const ForcePlugin *force) {
  for (size_t k = 0; k < m_Plugins.size(); ++k)
    if (m_Plugins[k].second.get() == force) {
      m_Plugins.erase(m_Plugins.begin() + k);
      ++m_PluginGen;
      return true;
    }
  return false;
}

std::map<std::string, double> ForceManager::getEnergyComponents(cudaStream_t s) {
  if (m_Multi) {  // the sum over all systems
    std::map<std::string, double> t;
    for (int k = 0; k < (int)m_Specs.size(); ++k)
      for (auto &kv : getEnergyComponents(k, s)) t[kv.first] += kv.second;
    return t;
  }
  long long e[kNumEnergyTerms];
  APO_CUDA(cudaMemcpyAsync(e, m_Energy.p, sizeof(e), cudaMemcpyDeviceToHost, s));
  APO_CUDA(cudaStreamSynchronize(s));
  std::map<std::string, double> m;
  for (int k = 0; k < kNumEnergyTerms; ++k) m[kEnergyNames[k]] = (double)e[k] * kInvEnergyScale;
  m["ewse"] = (m_EvalMask & 4) ? m_SelfEnergy : 0.0;
  if (!m_Plugins.empty()) {
    long long pe[kMaxPlugins];
    APO_CUDA(cudaMemcpyAsync(pe, m_PluginEnergy.p, sizeof(pe), cudaMemcpyDeviceToHost, s));
    APO_CUDA(cudaStreamSynchronize(s));
    for (size_t k = 0; k < m_Plugins.size(); ++k)
      m[m_Plugins[k].first] = (double)pe[k] * kInvEnergyScale;
  }
  return m;
}

std::map<std::string, double> ForceManager::getEnergyComponents(int sys, cudaStream_t s) {
  if (!m_Multi) {
    if (sys != 0) throw std::invalid_argument("getEnergyComponents: system index out of range");
    return getEnergyComponents(s);
  }
  if (sys < 0 || sys >= (int)m_Specs.size())
    throw std::invalid_argument("getEnergyComponents: system index out of range");
  long long e[kNumEnergyTerms];
  APO_CUDA(cudaMemcpyAsync(e, m_Energy.p + (size_t)sys * m_EStride, sizeof(e),
                           cudaMemcpyDeviceToHost, s));
  APO_CUDA(cudaStreamSynchronize(s));
  std::map<std::string, double> m;
  for (int k = 0; k < kNumEnergyTerms; ++k) m[kEnergyNames[k]] = (double)e[k] * kInvEnergyScale;
  m["ewse"] = (m_EvalMask & 4) ? m_SelfEnergies[sys] : 0.0;
  return m;
}

std::vector<double> ForceManager::getVirial(int sys, cudaStream_t s) {
  if (!m_Multi) {
    if (sys != 0) throw std::invalid_argument("getVirial: system index out of range");
    return getVirial(s);
  }
  if (sys < 0 || sys >= (int)m_Specs.size())
    throw std::invalid_argument("getVirial: system index out of range");
  if (!m_VirialValid)
    throw std::runtime_error("getVirial: the last force evaluation did not compute the virial");
  long long v[9];
  APO_CUDA(cudaMemcpyAsync(v, m_Energy.p + (size_t)sys * m_EStride + kNumEnergyTerms, sizeof(v),
                           cudaMemcpyDeviceToHost, s));
  APO_CUDA(cudaStreamSynchronize(s));
  std::vector<double> out(9);
  for (int k = 0; k < 9; ++k) out[k] = (double)v[k] * kInvEnergyScale;
  return out;
}

std::vector<double> ForceManager::getVirial(cudaStream_t s) {
  if (!m_Initialized) throw std::runtime_error("ForceManager is not initialized");
  if (m_Multi) {  // the sum over all systems
    std::vector<double> t(9, 0.0);
    for (int k = 0; k < (int)m_Specs.size(); ++k) {
      auto v = getVirial(k, s);
      for (int j = 0; j < 9; ++j) t[j] += v[j];
    }
    return t;
  }
  if (!m_VirialValid)
    throw std::runtime_error("getVirial: the last force evaluation did not compute the virial");
  long long v[9];
  APO_CUDA(cudaMemcpyAsync(v, m_Energy.p + kNumEnergyTerms, sizeof(v), cudaMemcpyDeviceToHost, s));
  APO_CUDA(cudaStreamSynchronize(s));
  std::vector<double> out(9);
  for (int k = 0; k < 9; ++k) out[k] = (double)v[k] * kInvEnergyScale;
  return out;
}

double ForceManager::getPotentialEnergy(cudaStream_t s) {
  double t = 0.0;
  for (auto &kv : getEnergyComponents(s)) t += kv.second;
  return t;
}

void ForceManager::getForces(std::vector<double> &out, cudaStream_t s) {
  const int n = m_Top.natom;
  if (m_Scratch.n < (size_t)3 * n) m_Scratch.alloc((size_t)3 * n);
  fixed_to_global_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, m_Force.p, m_Stride, m_Nbl.glo2loc,
                                                          m_Scratch.p);
  APO_LAUNCH_CHECK();
  out.resize((size_t)3 * n);
  APO_CUDA(cudaMemcpyAsync(out.data(), m_Scratch.p, (size_t)3 * n * sizeof(double),
                           cudaMemcpyDeviceToHost, s));
  APO_CUDA(cudaStreamSynchronize(s));
}

void ForceManager::getForcesDevice(double *d_out, int stride, cudaStream_t s) {
  const int n = m_Top.natom;
  if (!m_Initialized) throw std::runtime_error("ForceManager is not initialized");
  if (!d_out || stride < n) throw std::invalid_argument("getForcesDevice: buffer or stride too small");
  fixed_to_planes_kernel<double><<<(n + 255) / 256, 256, 0, s>>>(n, m_Force.p, m_Stride,
                                                                 m_Nbl.glo2loc, d_out, stride);
  APO_LAUNCH_CHECK();
}

void ForceManager::getForceFixedDevice(long long *d_out, int stride, cudaStream_t s) {
  const int n = m_Top.natom;
  if (!m_Initialized) throw std::runtime_error("ForceManager is not initialized");
  if (!d_out || stride < n)
    throw std::invalid_argument("getForceFixedDevice: buffer or stride too small");
  fixed_to_planes_kernel<long long><<<(n + 255) / 256, 256, 0, s>>>(n, m_Force.p, m_Stride,
                                                                    m_Nbl.glo2loc, d_out, stride);
  APO_LAUNCH_CHECK();
}

void ForceManager::calcForceXyzq(const float4 *d_xyzq, bool reset, bool calcEnergy,
                                 bool calcVirial, int components, cudaStream_t s) {
  if (m_Multi) throw std::invalid_argument("calcForceXyzq: needs a single-system force manager");
  if (!d_xyzq) throw std::invalid_argument("calcForceXyzq: xyzq is NULL");
  if (components < 0 || components > 15)
    throw std::invalid_argument("calcForceXyzq: components must be a mask of 1, 2, 4 and 8");
  if (!m_Initialized) initialize();
  const int n = m_Top.natom;
  if (m_XyzqState.n != (size_t)n) m_XyzqState.alloc(n);
  xyzq_to_state_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, d_xyzq, m_XyzqState.p);
  APO_LAUNCH_CHECK();
  // the state of an attached context comes back afterwards; the sorted
  // coordinates it refreshes next are then its own again, and a list built
  // here from other coordinates is rebuilt before its next use
  const double4 *attached = m_StateCoords;
  const int mask = m_ComponentMask;
  setStateCoordinates(m_XyzqState.p);
  m_ComponentMask = components;
  try {
    if (reset || !m_ListBuilt || m_ListDirty) resetNeighborList(d_xyzq, s);
    calcForceChecked(d_xyzq, calcEnergy, calcVirial, s);
  } catch (...) {
    m_ComponentMask = mask;
    setStateCoordinates(attached);
    throw;
  }
  m_ComponentMask = mask;
  setStateCoordinates(attached);
  if (reset && attached) m_ListDirty = true;
}

unsigned ForceManager::readDeviceError(cudaStream_t s) { return m_Nbl.read_error(s); }

void ForceManager::setKernelTiming(bool on) {
  m_Timing = on;
  m_TimerCursor = 0;
}

double ForceManager::kernelTimeMs(int &launches) {
  double t = 0.0;
  launches = 0;
  for (int k = 0; k < m_TimerCursor && k < (int)m_Timers.size(); ++k) {
    float ms = 0.f;
    APO_CUDA(cudaEventSynchronize(m_Timers[k].second));
    APO_CUDA(cudaEventElapsedTime(&ms, m_Timers[k].first, m_Timers[k].second));
    t += ms;
    ++launches;
  }
  return t;
}

// ------------------------------------------------------------ CharmmContext

CharmmContext::CharmmContext(std::shared_ptr<ForceManager> fm) : m_Fm(std::move(fm)) {
  if (!m_Fm) throw std::invalid_argument("CharmmContext: null ForceManager");
  if (!m_Fm->isInitialized()) m_Fm->initialize();
  m_N = m_Fm->getNumAtoms();
  APO_CUDA(cudaStreamCreateWithFlags(&m_Stream, cudaStreamNonBlocking));
  m_Coords.alloc(m_N);
  m_VelMass.alloc(m_N);
  m_Xyzq.alloc(m_N);
  const Topology &t = m_Fm->topology();
  std::vector<double4> vm(m_N);
  std::vector<double4> c(m_N);
  for (int i = 0; i < m_N; ++i) {
    vm[i] = make_double4(0.0, 0.0, 0.0, 1.0 / t.mass[i]);
    c[i] = make_double4(0.0, 0.0, 0.0, t.charge[i]);
  }
  m_VelMass.upload(vm);
  m_Coords.upload(c);
  launch_coords_to_xyzq(m_Coords.p, m_Xyzq.p, m_N, m_Stream);
  {  // large components first (a warp each), then the small ones (a thread each)
    std::vector<int2> groups = t.groups;
    m_NumBigGroups = order_components(groups, kSmallComponent);
    m_Groups.upload(groups);
  }
  m_Fm->setStateCoordinates(m_Coords.p);
  std::random_device rd;
  m_Seed = rd();
  useHolonomicConstraints(true);
}

CharmmContext::~CharmmContext() {
  if (m_Stream) cudaStreamDestroy(m_Stream);
}

void CharmmContext::useHolonomicConstraints(bool flag) {
  m_Holonomic = flag;
  if (m_Fm->isMulti()) {  // every system loses its own centre of mass
    m_Ndegf = 0;
    m_SysNdegf.clear();
    for (const Topology &t : m_Fm->systemTopologies()) {
      m_SysNdegf.push_back(t.degrees_of_freedom(flag));
      m_Ndegf += m_SysNdegf.back();
    }
  } else {
    m_Ndegf = m_Fm->topology().degrees_of_freedom(flag);
    m_SysNdegf.assign(1, m_Ndegf);
  }
}

namespace {

// first atom with a non-finite coordinate (atomicMin over the array)
__global__ void check_finite_kernel(const double *__restrict__ xyz, int n, int *__restrict__ bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (!isfinite(xyz[3 * i]) || !isfinite(xyz[3 * i + 1]) || !isfinite(xyz[3 * i + 2]))
    atomicMin(bad, i);
}

// interleaved x,y,z -> the .x/.y/.z of double4 (w kept); skipped entirely
// when the check above found a bad atom, so the state stays unchanged
__global__ void pack_xyz_kernel(const double *__restrict__ xyz, int n, double4 *__restrict__ out,
                                const int *__restrict__ bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || (bad && *bad != INT_MAX)) return;
  double4 v = out[i];
  v.x = xyz[3 * i];
  v.y = xyz[3 * i + 1];
  v.z = xyz[3 * i + 2];
  out[i] = v;
}

__global__ void unpack_xyz_kernel(const double4 *__restrict__ in, int n, double *__restrict__ xyz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 v = in[i];
  xyz[3 * i] = v.x;
  xyz[3 * i + 1] = v.y;
  xyz[3 * i + 2] = v.z;
}

}  // namespace

void CharmmContext::setCoordinates(const std::vector<double> &xyz) {
  if ((int)xyz.size() != 3 * m_N) {
    std::ostringstream m;
    m << "setCoordinates: expected " << 3 * m_N << " values, got " << xyz.size();
    throw std::invalid_argument(m.str());
  }
  setCoordinatesXyz(xyz.data());
}

void CharmmContext::setCoordinatesXyz(const double *xyz, int first, int count, bool rebuild) {
  if (count < 0) count = m_N - first;
  if (first < 0 || count < 0 || first + count > m_N)
    throw std::invalid_argument("setCoordinates: atom range out of bounds");
  if (m_Stage.n != (size_t)3 * m_N) m_Stage.alloc((size_t)3 * m_N);
  if (m_BadAtom.n != 1) m_BadAtom.alloc(1);
  const int ok = INT_MAX;
  APO_CUDA(cudaMemcpyAsync(m_BadAtom.p, &ok, sizeof(int), cudaMemcpyHostToDevice, m_Stream));
  APO_CUDA(cudaMemcpyAsync(m_Stage.p + 3 * (size_t)first, xyz, (size_t)3 * count * sizeof(double),
                           cudaMemcpyHostToDevice, m_Stream));
  const int b = (count + 255) / 256;
  if (count > 0) {
    check_finite_kernel<<<b, 256, 0, m_Stream>>>(m_Stage.p + 3 * (size_t)first, count,
                                                 m_BadAtom.p);
    APO_LAUNCH_CHECK();
    pack_xyz_kernel<<<b, 256, 0, m_Stream>>>(m_Stage.p + 3 * (size_t)first, count,
                                             m_Coords.p + first, m_BadAtom.p);
    APO_LAUNCH_CHECK();
  }
  int bad = INT_MAX;
  APO_CUDA(cudaMemcpyAsync(&bad, m_BadAtom.p, sizeof(int), cudaMemcpyDeviceToHost, m_Stream));
  APO_CUDA(cudaStreamSynchronize(m_Stream));
  if (bad != INT_MAX)
    throw std::invalid_argument("setCoordinates: non-finite coordinate for atom " +
                                std::to_string(first + bad));
  launch_coords_to_xyzq(m_Coords.p, m_Xyzq.p, m_N, m_Stream);
  m_HasCoords = true;
  if (rebuild) {
    resetNeighborList(m_Stream);
  } else {
    m_ListStale = true;
  }
  APO_CUDA(cudaStreamSynchronize(m_Stream));
}

void CharmmContext::saveStateDevice(double4 *dst, int first, int count) {
  if (first < 0 || count < 0 || first + count > m_N)
    throw std::invalid_argument("saveStateDevice: atom range out of bounds");
  if (!count) return;
  APO_CUDA(cudaMemcpyAsync(dst, m_Coords.p + first, count * sizeof(double4),
                           cudaMemcpyDeviceToDevice, m_Stream));
  APO_CUDA(cudaMemcpyAsync(dst + count, m_VelMass.p + first, count * sizeof(double4),
                           cudaMemcpyDeviceToDevice, m_Stream));
}

void CharmmContext::loadStateDevice(const double4 *src, int first, int count) {
  if (first < 0 || count < 0 || first + count > m_N)
    throw std::invalid_argument("loadStateDevice: atom range out of bounds");
  if (!count) return;
  APO_CUDA(cudaMemcpyAsync(m_Coords.p + first, src, count * sizeof(double4),
                           cudaMemcpyDeviceToDevice, m_Stream));
  APO_CUDA(cudaMemcpyAsync(m_VelMass.p + first, src + count, count * sizeof(double4),
                           cudaMemcpyDeviceToDevice, m_Stream));
  launch_coords_to_xyzq(m_Coords.p + first, m_Xyzq.p + first, count, m_Stream);
  m_HasCoords = true;
  m_ListStale = true;
}

std::vector<double> CharmmContext::getCoordinates() {
  std::vector<double> out((size_t)3 * m_N);
  getCoordinatesXyz(out.data());
  return out;
}

void CharmmContext::getCoordinatesXyz(double *xyz, int first, int count) {
  if (count < 0) count = m_N - first;
  if (first < 0 || count < 0 || first + count > m_N)
    throw std::invalid_argument("getCoordinates: atom range out of bounds");
  if (m_Stage.n != (size_t)3 * m_N) m_Stage.alloc((size_t)3 * m_N);
  if (count > 0) {
    unpack_xyz_kernel<<<(count + 255) / 256, 256, 0, m_Stream>>>(m_Coords.p + first, count,
                                                                 m_Stage.p + 3 * (size_t)first);
    APO_LAUNCH_CHECK();
  }
  APO_CUDA(cudaMemcpyAsync(xyz, m_Stage.p + 3 * (size_t)first, (size_t)3 * count * sizeof(double),
                           cudaMemcpyDeviceToHost, m_Stream));
  APO_CUDA(cudaStreamSynchronize(m_Stream));
}

void CharmmContext::setVelocities(const std::vector<double> &v) {
  if ((int)v.size() != 3 * m_N) throw std::invalid_argument("setVelocities: wrong length");
  setVelocitiesXyz(v.data());
}

void CharmmContext::setVelocitiesXyz(const double *v, int first, int count) {
  if (count < 0) count = m_N - first;
  if (first < 0 || count < 0 || first + count > m_N)
    throw std::invalid_argument("setVelocities: atom range out of bounds");
  if (m_Stage.n != (size_t)3 * m_N) m_Stage.alloc((size_t)3 * m_N);
  APO_CUDA(cudaMemcpyAsync(m_Stage.p + 3 * (size_t)first, v, (size_t)3 * count * sizeof(double),
                           cudaMemcpyHostToDevice, m_Stream));
  if (count > 0) {
    pack_xyz_kernel<<<(count + 255) / 256, 256, 0, m_Stream>>>(m_Stage.p + 3 * (size_t)first,
                                                               count, m_VelMass.p + first, nullptr);
    APO_LAUNCH_CHECK();
  }
  APO_CUDA(cudaStreamSynchronize(m_Stream));
}

std::vector<double> CharmmContext::getVelocities() {
  std::vector<double> out((size_t)3 * m_N);
  getVelocitiesXyz(out.data());
  return out;
}

void CharmmContext::getVelocitiesXyz(double *v, int first, int count) {
  if (count < 0) count = m_N - first;
  if (first < 0 || count < 0 || first + count > m_N)
    throw std::invalid_argument("getVelocities: atom range out of bounds");
  if (m_Stage.n != (size_t)3 * m_N) m_Stage.alloc((size_t)3 * m_N);
  if (count > 0) {
    unpack_xyz_kernel<<<(count + 255) / 256, 256, 0, m_Stream>>>(m_VelMass.p + first, count,
                                                                 m_Stage.p + 3 * (size_t)first);
    APO_LAUNCH_CHECK();
  }
  APO_CUDA(cudaMemcpyAsync(v, m_Stage.p + 3 * (size_t)first, (size_t)3 * count * sizeof(double),
                           cudaMemcpyDeviceToHost, m_Stream));
  APO_CUDA(cudaStreamSynchronize(m_Stream));
}

// Maxwell-Boltzmann velocities with std::mt19937 and one
// std::normal_distribution per atom, as src/CharmmContext.cu:478-525
void CharmmContext::assignVelocitiesAtTemperature(double temperature) {
  if (!m_HasCoords)
    throw std::invalid_argument("assignVelocitiesAtTemperature: coordinates not set");
  APO_CUDA(cudaStreamSynchronize(m_Stream));
  std::vector<double4> vm = m_VelMass.download();
  const double boltz = kBoltz * (float)temperature;
  // one generator per system, seeded with the system's own seed, so that a
  // system gets the same velocities alone and among others
  const std::vector<int> &off = m_Fm->isMulti() ? m_Fm->atomOffsets() : std::vector<int>{0, m_N};
  for (size_t k = 0; k + 1 < off.size(); ++k) {
    const uint64_t seed = m_Fm->isMulti() ? m_Fm->systemSpecs()[k].seed : m_Seed;
    std::mt19937 gen{(std::mt19937::result_type)seed};
    for (int i = off[k]; i < off[k + 1]; ++i) {
      double sd = std::sqrt(boltz * vm[i].w);
      std::normal_distribution<> d(0, sd);
      vm[i].x = d(gen);
      vm[i].y = d(gen);
      vm[i].z = d(gen);
    }
  }
  APO_CUDA(cudaMemcpy(m_VelMass.p, vm.data(), m_N * sizeof(double4), cudaMemcpyHostToDevice));
}

namespace {
// kinetic energy of every system (2^32 fixed point, order-free)
__global__ void system_ke_kernel(const double4 *__restrict__ vm, int n,
                                 const int *__restrict__ sys_of_atom, long long *__restrict__ ke) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 v = vm[i];
  const double e = 0.5 * (v.x * v.x + v.y * v.y + v.z * v.z) / v.w;
  add_fixed(ke + (sys_of_atom ? sys_of_atom[i] : 0), __double2ll_rn(e * kEnergyScale));
}
}  // namespace

std::vector<double> CharmmContext::systemTemperatures() {
  const int ns = m_Fm->numSystems();
  if (m_SysKe.n != (size_t)ns) m_SysKe.alloc(ns);
  APO_CUDA(cudaMemsetAsync(m_SysKe.p, 0, ns * sizeof(long long), m_Stream));
  if (m_N > 0) {
    system_ke_kernel<<<(m_N + 255) / 256, 256, 0, m_Stream>>>(
        m_VelMass.p, m_N, m_Fm->isMulti() ? m_Fm->sysOfAtom() : nullptr, m_SysKe.p);
    APO_LAUNCH_CHECK();
  }
  std::vector<long long> ke(ns);
  APO_CUDA(cudaMemcpyAsync(ke.data(), m_SysKe.p, ns * sizeof(long long), cudaMemcpyDeviceToHost,
                           m_Stream));
  APO_CUDA(cudaStreamSynchronize(m_Stream));
  std::vector<double> t(ns);
  for (int k = 0; k < ns; ++k)
    t[k] = (double)ke[k] * kInvEnergyScale / (0.5 * m_SysNdegf[k] * kBoltz);
  return t;
}

double CharmmContext::getKineticEnergy() {
  APO_CUDA(cudaStreamSynchronize(m_Stream));
  std::vector<double4> vm = m_VelMass.download();
  double ke = 0.0;
  for (auto &v : vm) ke += 0.5 * (v.x * v.x + v.y * v.y + v.z * v.z) / v.w;
  return ke;
}

double CharmmContext::computeTemperature() {
  return getKineticEnergy() / (0.5 * m_Ndegf * kBoltz);
}

void CharmmContext::imageCentering(cudaStream_t s) {
  auto b = m_Fm->getBoxDimensions();
  if (m_Fm->isMulti())
    launch_image_centering(m_Coords.p, m_Xyzq.p, m_Groups.p, (int)m_Groups.n, m_NumBigGroups,
                           b[0], b[1], b[2], s, m_Fm->sysOfAtom(), m_Fm->systemBoxes());
  else if (m_Fm->hasDeviceBox())  // the box may have changed on the device
    launch_image_centering(m_Coords.p, m_Xyzq.p, m_Groups.p, (int)m_Groups.n, m_NumBigGroups,
                           b[0], b[1], b[2], s, m_Fm->neighborList().sys_of_atom,
                           m_Fm->deviceBox());
  else
    launch_image_centering(m_Coords.p, m_Xyzq.p, m_Groups.p, (int)m_Groups.n, m_NumBigGroups,
                           b[0], b[1], b[2], s);
}

void CharmmContext::resetNeighborList(cudaStream_t s) {
  imageCentering(s);
  m_Fm->resetNeighborList(m_Xyzq.p, s);
  m_ListStale = false;
}

void CharmmContext::ensureNeighborList() {
  if (!m_HasCoords) throw std::runtime_error("coordinates not set");
  if (m_ListStale || !m_Fm->isListBuilt()) {
    resetNeighborList(m_Stream);
    APO_CUDA(cudaStreamSynchronize(m_Stream));
  }
}

void CharmmContext::ensureListBuffers() {
  if (!m_HasCoords) throw std::runtime_error("coordinates not set");
  if (!m_Fm->isListBuilt()) {
    resetNeighborList(m_Stream);
    APO_CUDA(cudaStreamSynchronize(m_Stream));
  }
}

void CharmmContext::calculateForces(bool reset, bool calcEnergy, bool calcVirial) {
  if (!m_HasCoords) throw std::runtime_error("calculateForces: coordinates not set");
  if (reset || m_ListStale) resetNeighborList(m_Stream);
  m_Fm->calcForceChecked(m_Xyzq.p, calcEnergy, calcVirial, m_Stream);
}

double CharmmContext::calculatePotentialEnergy(bool reset, bool /*print*/) {
  calculateForces(reset, true, true);
  return m_Fm->getPotentialEnergy(m_Stream);
}

}  // namespace apo
