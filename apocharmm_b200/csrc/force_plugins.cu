// Force plug-ins; see force_plugins.h.
#include "force_plugins.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>

#include "common.h"
#include "device_util.cuh"

namespace apo {

namespace {

constexpr int kThreads = 256;

__global__ void harmonic_restraint_kernel(const int *__restrict__ count,
                                          const int *__restrict__ atoms,
                                          const double4 *__restrict__ target,
                                          const double4 *__restrict__ coords,
                                          const int *__restrict__ glo2loc,
                                          long long *__restrict__ force, int stride,
                                          long long *__restrict__ energy, double Lx,
                                          double Ly, double Lz, int calc_energy) {
  const int n = *count;
  double e = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int a = atoms[k];
    const double4 t = target[k];
    const double4 x = coords[a];
    double dx = x.x - t.x, dy = x.y - t.y, dz = x.z - t.z;
    dx -= Lx * rint(dx / Lx);  // nearest image
    dy -= Ly * rint(dy / Ly);
    dz -= Lz * rint(dz / Lz);
    const double c = 2.0 * t.w;  // t.w = k m
    const int s = glo2loc[a];
    add_fixed(force + s, to_fixed_force_d(c * dx));
    add_fixed(force + stride + s, to_fixed_force_d(c * dy));
    add_fixed(force + 2 * stride + s, to_fixed_force_d(c * dz));
    e += t.w * (dx * dx + dy * dy + dz * dz);
  }
  if (calc_energy) {
    e = warp_sum(e);
    if ((threadIdx.x & 31) == 0 && e != 0.0) add_energy(energy, e);
  }
}

// atom-order fixed-point gradient of an external force into the slot-order
// buffer; thread 0 adds the FP64 energies as one fixed-point value
__global__ void add_external_kernel(int n, const long long *__restrict__ f, int fstride,
                                    const int *__restrict__ glo2loc,
                                    long long *__restrict__ force, int stride,
                                    const double *__restrict__ e, int ne,
                                    long long *__restrict__ energy) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < n) {
    const int s = glo2loc[g];
    force[s] += f[g];
    force[stride + s] += f[fstride + g];
    force[2 * stride + s] += f[2 * fstride + g];
  }
  if (g == 0 && e) {
    double t = 0.0;
    for (int k = 0; k < ne; ++k) t += e[k];
    add_energy(energy, t);
  }
}

}  // namespace

ExternalForce::ExternalForce(const ExternalForceOps &ops) : m_Ops(ops) {
  if (!ops.calc_force || !ops.get_force)
    throw std::invalid_argument("external force: calc_force and get_force are required");
  if (!ops.stream) throw std::invalid_argument("external force: a stream is required");
  APO_CUDA(cudaEventCreateWithFlags(&m_Fork, cudaEventDisableTiming));
  APO_CUDA(cudaEventCreateWithFlags(&m_Join, cudaEventDisableTiming));
}

ExternalForce::~ExternalForce() {
  if (m_Fork) cudaEventDestroy(m_Fork);
  if (m_Join) cudaEventDestroy(m_Join);
}

void ExternalForce::initialize(int natom, const std::array<double, 3> &box) {
  if (m_Ops.initialize) m_Ops.initialize(m_Ops.object, natom, box.data());
}

void ExternalForce::calcForce(const ForcePluginArgs &a, bool calcEnergy, bool calcVirial,
                              cudaStream_t s) {
  // the manager's gradient slots are only written on s before and after
  // this call, so the additions below need no atomics (glo2loc is one to one)
  APO_CUDA(cudaEventRecord(m_Fork, s));
  APO_CUDA(cudaStreamWaitEvent(m_Ops.stream, m_Fork, 0));
  if (m_Ops.clear) m_Ops.clear(m_Ops.object);
  m_Ops.calc_force(m_Ops.object, reinterpret_cast<const float *>(a.xyzq), calcEnergy ? 1 : 0,
                   calcVirial ? 1 : 0);
  int fstride = 0;
  const long long *f = m_Ops.get_force(m_Ops.object, &fstride);
  int ne = 0;
  const double *e = (calcEnergy && m_Ops.get_energies) ? m_Ops.get_energies(m_Ops.object, &ne)
                                                        : nullptr;
  APO_CUDA(cudaEventRecord(m_Join, m_Ops.stream));
  APO_CUDA(cudaStreamWaitEvent(s, m_Join, 0));
  if (!f || fstride < a.natom)
    throw std::runtime_error("external force: no force buffer, or its stride is below the atom count");
  if (e && ne < 0) throw std::runtime_error("external force: negative energy count");
  add_external_kernel<<<(a.natom + kThreads - 1) / kThreads, kThreads, 0, s>>>(
      a.natom, f, fstride, a.glo2loc, a.force, a.stride, e, ne, a.energy);
  APO_LAUNCH_CHECK();
}

HarmonicRestraintForce::HarmonicRestraintForce(int natom) : m_N(natom) {
  if (natom <= 0) throw std::invalid_argument("HarmonicRestraintForce: number of atoms must be > 0");
  m_Selected.assign(natom, 0);
  m_K.assign(natom, 0.0);
  m_Ref.assign((size_t)4 * natom, 0.0);
  for (int i = 0; i < natom; ++i) m_Ref[4 * (size_t)i + 3] = 1.0;
}

HarmonicRestraintForce::~HarmonicRestraintForce() {
  if (m_Count) cudaFree(m_Count);
  if (m_Atoms) cudaFree(m_Atoms);
  if (m_Target) cudaFree(m_Target);
}

void HarmonicRestraintForce::setSelection(const std::vector<int> &atoms) {
  std::vector<char> sel(m_N, 0);
  for (int a : atoms) {
    if (a < 0 || a >= m_N)
      throw std::invalid_argument("HarmonicRestraintForce: selected atom " + std::to_string(a) +
                                  " out of range");
    sel[a] = 1;
  }
  m_Selected.swap(sel);
  for (int i = 0; i < m_N; ++i)
    if (!m_Selected[i]) m_K[i] = 0.0;
  upload();
}

void HarmonicRestraintForce::setForceConstant(double k) {
  if (!std::isfinite(k)) throw std::invalid_argument("HarmonicRestraintForce: non-finite force constant");
  for (int i = 0; i < m_N; ++i) m_K[i] = m_Selected[i] ? k : 0.0;
  upload();
}

void HarmonicRestraintForce::setForceConstants(const std::vector<double> &k) {
  if ((int)k.size() != m_N)
    throw std::invalid_argument("HarmonicRestraintForce::setForceConstants: one value per atom "
                                "expected (NATOM = " + std::to_string(m_N) + ", got " +
                                std::to_string(k.size()) + ")");
  for (double v : k)
    if (!std::isfinite(v)) throw std::invalid_argument("HarmonicRestraintForce: non-finite force constant");
  for (int i = 0; i < m_N; ++i) m_K[i] = m_Selected[i] ? k[i] : 0.0;
  upload();
}

void HarmonicRestraintForce::setReferenceCoordinates(const std::vector<double> &xyz) {
  if ((int)xyz.size() != 3 * m_N)
    throw std::invalid_argument("HarmonicRestraintForce::setReferenceCoordinates: 3 x NATOM values "
                                "expected (NATOM = " + std::to_string(m_N) + ", got " +
                                std::to_string(xyz.size()) + ")");
  for (int i = 0; i < m_N; ++i)
    for (int d = 0; d < 3; ++d) m_Ref[4 * (size_t)i + d] = xyz[3 * (size_t)i + d];
  upload();
}

void HarmonicRestraintForce::setMasses(const std::vector<double> &m) {
  if ((int)m.size() != m_N)
    throw std::invalid_argument("HarmonicRestraintForce::setMasses: one value per atom expected "
                                "(NATOM = " + std::to_string(m_N) + ", got " +
                                std::to_string(m.size()) + ")");
  for (int i = 0; i < m_N; ++i) m_Ref[4 * (size_t)i + 3] = m[i];
  upload();
}

void HarmonicRestraintForce::setBoxDimensions(const std::array<double, 3> &box) {
  if (box == m_Box) return;
  if (m_Box[0] != 0.0 && m_Box[1] != 0.0 && m_Box[2] != 0.0) {
    for (int i = 0; i < m_N; ++i)
      for (int d = 0; d < 3; ++d) m_Ref[4 * (size_t)i + d] *= box[d] / m_Box[d];
  }
  m_Box = box;
  upload();
}

void HarmonicRestraintForce::initialize(int natom, const std::array<double, 3> &box) {
  if (natom != m_N)
    throw std::runtime_error("HarmonicRestraintForce: Attempted to initialize with different atom "
                             "count");
  if (!m_Atoms) {
    APO_CUDA(cudaMalloc(&m_Count, sizeof(int)));
    APO_CUDA(cudaMalloc(&m_Atoms, (size_t)m_N * sizeof(int)));
    APO_CUDA(cudaMalloc(&m_Target, (size_t)m_N * sizeof(double4)));
  }
  setBoxDimensions(box);
  upload();
}

void HarmonicRestraintForce::upload() {
  if (!m_Atoms) return;  // not on the device yet: initialize() uploads
  std::vector<int> atoms;
  std::vector<double4> target;
  for (int i = 0; i < m_N; ++i) {
    const double km = m_K[i] * m_Ref[4 * (size_t)i + 3];
    if (m_Selected[i] && km != 0.0) {
      atoms.push_back(i);
      target.push_back(make_double4(m_Ref[4 * (size_t)i], m_Ref[4 * (size_t)i + 1],
                                    m_Ref[4 * (size_t)i + 2], km));
    }
  }
  const int n = (int)atoms.size();
  // synchronous copies: a setter runs between force calls, never during one
  if (n) {
    APO_CUDA(cudaMemcpy(m_Atoms, atoms.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice));
    APO_CUDA(cudaMemcpy(m_Target, target.data(), (size_t)n * sizeof(double4),
                        cudaMemcpyHostToDevice));
  }
  APO_CUDA(cudaMemcpy(m_Count, &n, sizeof(int), cudaMemcpyHostToDevice));
}

void HarmonicRestraintForce::calcForce(const ForcePluginArgs &a, bool calcEnergy, bool,
                                       cudaStream_t s) {
  if (!m_Atoms) throw std::runtime_error("HarmonicRestraintForce: not initialized");
  if (a.natom != m_N) throw std::runtime_error("HarmonicRestraintForce: atom count mismatch");
  // a fixed grid (the count may change between captures of the same graph)
  const int blocks = std::min((m_N + kThreads - 1) / kThreads, 148 * 8);
  harmonic_restraint_kernel<<<blocks, kThreads, 0, s>>>(m_Count, m_Atoms, m_Target, a.coords,
                                                        a.glo2loc, a.force, a.stride, a.energy,
                                                        a.box[0], a.box[1], a.box[2],
                                                        calcEnergy ? 1 : 0);
  APO_LAUNCH_CHECK();
}

}  // namespace apo
