// Batch of independent systems; see batch.h.
#include "batch.h"

#include <algorithm>
#include <chrono>
#include <stdexcept>

namespace apo {

Batch::Batch(int order, int tilesPerWork, bool precise)
    : m_Order(order), m_Tpw(tilesPerWork), m_Precise(precise) {
  if (order != 4 && order != 6 && order != 8)
    throw std::invalid_argument("Batch: spline order must be 4, 6 or 8");
  if (tilesPerWork < 1) throw std::invalid_argument("Batch: tiles per work item must be >= 1");
}

int Batch::addSystem(const SystemSpec &spec) {
  if (m_Ctx) throw std::runtime_error("Batch: systems must be added before initialize()");
  if (!spec.psf || !spec.prm) throw std::invalid_argument("Batch: null PSF or parameters");
  m_Specs.push_back(spec);
  return (int)m_Specs.size() - 1;
}

void Batch::initialize() {
  if (m_Specs.empty()) throw std::invalid_argument("Batch: no systems");
  m_Fm = std::make_shared<ForceManager>(m_Specs, m_Order, m_Tpw, m_Precise);
  m_Ctx = std::make_shared<CharmmContext>(m_Fm);
  m_Integ.reset();
}

void Batch::requireInit() const {
  if (!m_Ctx) throw std::runtime_error("Batch: not initialized");
}
void Batch::requireSys(int sys) const {
  requireInit();
  if (sys < 0 || sys >= (int)m_Specs.size())
    throw std::invalid_argument("Batch: system index out of range");
}

int Batch::numAtoms(int sys) const {
  requireInit();
  const auto &off = m_Fm->atomOffsets();
  if (sys < 0) return off.back();
  requireSys(sys);
  return off[sys + 1] - off[sys];
}

int Batch::atomOffset(int sys) const {
  requireSys(sys);
  return m_Fm->atomOffsets()[sys];
}

// sys < 0: every system at once (the concatenated arrays)
void Batch::setCoordinates(int sys, const double *xyz) {
  if (sys < 0) return requireInit(), m_Ctx->setCoordinatesXyz(xyz);
  requireSys(sys);
  // the list is rebuilt before the next evaluation, after every system is loaded
  m_Ctx->setCoordinatesXyz(xyz, atomOffset(sys), numAtoms(sys), /*rebuild=*/false);
}
void Batch::getCoordinates(int sys, double *xyz) {
  if (sys < 0) return requireInit(), m_Ctx->getCoordinatesXyz(xyz);
  requireSys(sys);
  m_Ctx->getCoordinatesXyz(xyz, atomOffset(sys), numAtoms(sys));
}
void Batch::setVelocities(int sys, const double *v) {
  if (sys < 0) return requireInit(), m_Ctx->setVelocitiesXyz(v);
  requireSys(sys);
  m_Ctx->setVelocitiesXyz(v, atomOffset(sys), numAtoms(sys));
}
void Batch::getVelocities(int sys, double *v) {
  if (sys < 0) return requireInit(), m_Ctx->getVelocitiesXyz(v);
  requireSys(sys);
  m_Ctx->getVelocitiesXyz(v, atomOffset(sys), numAtoms(sys));
}

void Batch::saveState(int sys, double4 *dst) {
  requireSys(sys);
  const int o = atomOffset(sys), n = numAtoms(sys);
  cudaStream_t s = m_Ctx->stream();
  m_Ctx->saveStateDevice(dst, o, n);
  if (m_Integ && m_Integ->deltaState())
    APO_CUDA(cudaMemcpyAsync(dst + 2 * (size_t)n, m_Integ->deltaState() + o, n * sizeof(double4),
                             cudaMemcpyDeviceToDevice, s));
  else
    APO_CUDA(cudaMemsetAsync(dst + 2 * (size_t)n, 0, n * sizeof(double4), s));
  APO_CUDA(cudaStreamSynchronize(s));
}

void Batch::loadState(int sys, const double4 *src) {
  requireSys(sys);
  const int o = atomOffset(sys), n = numAtoms(sys);
  cudaStream_t s = m_Ctx->stream();
  m_Ctx->loadStateDevice(src, o, n);
  if (m_Integ && m_Integ->deltaState())
    APO_CUDA(cudaMemcpyAsync(m_Integ->deltaState() + o, src + 2 * (size_t)n, n * sizeof(double4),
                             cudaMemcpyDeviceToDevice, s));
  APO_CUDA(cudaStreamSynchronize(s));
}

void Batch::assignVelocities(double temperature) {
  requireInit();
  m_Ctx->assignVelocitiesAtTemperature(temperature);
}

void Batch::setLangevin(double dtPs, double frictionPerPs, double temperature, uint64_t seed) {
  if (!(dtPs > 0.0)) throw std::invalid_argument("Batch: time step must be positive");
  m_Dt = dtPs;
  m_Friction = frictionPerPs;
  m_Temp = temperature;
  m_Seed = seed;
  m_Integ.reset();
}

void Batch::createIntegrator() {
  requireInit();
  m_Ctx->ensureNeighborList();
  m_Integ = std::make_shared<CudaLangevinThermostatIntegrator>(m_Dt);
  m_Integ->setThermostatFriction(m_Friction);
  m_Integ->setReferenceTemperature(m_Temp);
  m_Integ->setThermostatRngSeed(m_Seed);
  m_Integ->setCharmmContext(m_Ctx);
  m_Fm->setDirectKernel(m_Form);
}

void Batch::propagate(int steps) {
  requireInit();
  if (!m_Integ) createIntegrator();
  m_Integ->propagate(steps);
}

void Batch::calculateForces(bool energy, bool virial) {
  requireInit();
  m_Ctx->calculateForces(false, energy, virial);
  m_Fm->getForces(m_Forces, m_Ctx->stream());
}

std::map<std::string, double> Batch::energyComponents(int sys) {
  requireSys(sys);
  return m_Fm->getEnergyComponents(sys, m_Ctx->stream());
}

void Batch::getForces(int sys, double *xyz) {
  requireInit();
  if (m_Forces.size() != (size_t)3 * numAtoms(-1))
    throw std::runtime_error("Batch: no forces evaluated yet");
  if (sys >= 0) requireSys(sys);
  const int o = sys < 0 ? 0 : atomOffset(sys), n = numAtoms(sys);
  std::copy(m_Forces.begin() + 3 * (size_t)o, m_Forces.begin() + 3 * (size_t)(o + n), xyz);
}

std::vector<double> Batch::temperatures() {
  requireInit();
  return m_Ctx->systemTemperatures();
}

int Batch::autotune(int steps, const std::vector<int> &candidates) {
  requireInit();
  if (candidates.empty()) return m_Tpw;
  steps = std::max(1, steps);
  // the sweep moves the atoms: keep the state and put it back afterwards
  const int n = numAtoms(-1);
  std::vector<double> x((size_t)3 * n), v((size_t)3 * n);
  m_Ctx->getCoordinatesXyz(x.data());
  m_Ctx->getVelocitiesXyz(v.data());
  cudaStream_t s = m_Ctx->stream();
  cudaEvent_t e0, e1;
  APO_CUDA(cudaEventCreate(&e0));
  APO_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int best_t = m_Tpw, best_f = m_Form;
  for (int form : {kNbTileBatches, kNbGroupedQueues, kNbOctetLists})
    for (int t : candidates) {
      if (t < 1) continue;
      m_Form = form;
      m_Fm->setDirectKernel(form);
      m_Fm->neighborList().set_tiles_per_work(t);
      m_Integ.reset();            // graphs hold the old launch arguments
      propagate(steps);           // warm-up: graph capture, first replay
      APO_CUDA(cudaEventRecord(e0, s));
      propagate(steps);
      APO_CUDA(cudaEventRecord(e1, s));
      APO_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      APO_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best) {
        best = ms;
        best_t = t;
        best_f = form;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  m_Fm->setDirectKernel(best_f);
  m_Fm->neighborList().set_tiles_per_work(best_t);
  m_Tpw = best_t;
  m_Form = best_f;
  m_Integ.reset();
  m_Ctx->setCoordinatesXyz(x.data());
  m_Ctx->setVelocitiesXyz(v.data());
  return best_t;
}

}  // namespace apo
