// Integrators and trajectory subscribers: the reference's
// include/CudaIntegrator.h:63-187 (setCharmmContext, propagate,
// setTimeStep, setNonbondedListUpdateFrequency, subscribe / unsubscribe,
// getCurrentPropagatedStep, initializeFromRestartFile),
// include/CudaLangevinThermostatIntegrator.h:24-34,
// include/CudaNoseHooverIntegrator.h, include/CudaLeapFrogIntegrator.h,
// include/CudaLangevinPistonIntegrator.h:18-60 (constant pressure),
// include/Subscriber.h, include/DcdSubscriber.h, include/RestartSubscriber.h,
// header-only over the C ABI.  An integrator keeps its context and its
// subscribers alive.
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "apocharmm/CharmmContext.h"
#include "apocharmm/Check.h"
#include "apocharmm_c/CudaIntegrator.h"
#include "apocharmm_c/CudaLangevinPistonIntegrator.h"
#include "apocharmm_c/CudaLangevinThermostatIntegrator.h"
#include "apocharmm_c/CudaNoseHooverIntegrator.h"
#include "apocharmm_c/DcdSubscriber.h"
#include "apocharmm_c/RestartSubscriber.h"
#include "apocharmm_c/Subscriber.h"

class Subscriber {
 public:
  virtual ~Subscriber() = default;
  int getReportFrequency() const {
    int f = 0;
    apocharmm_detail::check(apo_subscriber_get_report_frequency(&f, m_Base));
    return f;
  }
  void setReportFrequency(const int frequency) {
    apocharmm_detail::check(apo_subscriber_set_report_frequency(m_Base, frequency));
  }
  apo_subscriber *base() { return m_Base; }

 protected:
  apo_subscriber *m_Base = nullptr;  // borrowed view of the concrete handle
};

class DcdSubscriber : public Subscriber {
 public:
  explicit DcdSubscriber(const std::string &fileName) {
    apocharmm_detail::check(apo_dcd_subscriber_create(&m_H, fileName.c_str()));
    apocharmm_detail::check(apo_dcd_subscriber_as_subscriber(&m_Base, m_H));
  }
  DcdSubscriber(const std::string &fileName, const int reportFreq) {
    apocharmm_detail::check(
        apo_dcd_subscriber_create_with_report_frequency(&m_H, fileName.c_str(), reportFreq));
    apocharmm_detail::check(apo_dcd_subscriber_as_subscriber(&m_Base, m_H));
  }
  ~DcdSubscriber() override { apo_dcd_subscriber_destroy(m_H); }
  DcdSubscriber(const DcdSubscriber &) = delete;
  DcdSubscriber &operator=(const DcdSubscriber &) = delete;

 private:
  apo_dcd_subscriber *m_H = nullptr;
};

class RestartSubscriber : public Subscriber {
 public:
  explicit RestartSubscriber(const std::string &fileName) {
    apocharmm_detail::check(apo_restart_subscriber_create(&m_H, fileName.c_str()));
    apocharmm_detail::check(apo_restart_subscriber_as_subscriber(&m_Base, m_H));
  }
  RestartSubscriber(const std::string &fileName, const int reportFreq) {
    apocharmm_detail::check(
        apo_restart_subscriber_create_with_report_frequency(&m_H, fileName.c_str(), reportFreq));
    apocharmm_detail::check(apo_restart_subscriber_as_subscriber(&m_Base, m_H));
  }
  ~RestartSubscriber() override { apo_restart_subscriber_destroy(m_H); }
  RestartSubscriber(const RestartSubscriber &) = delete;
  RestartSubscriber &operator=(const RestartSubscriber &) = delete;

 private:
  apo_restart_subscriber *m_H = nullptr;
};

class CudaIntegrator {
 public:
  virtual ~CudaIntegrator() = default;
  CudaIntegrator(const CudaIntegrator &) = delete;
  CudaIntegrator &operator=(const CudaIntegrator &) = delete;

  double getTimeStep(void) const { return m_Dt; }
  void setTimeStep(const double dt) {
    apocharmm_detail::check(apo_cuda_integrator_set_time_step(m_Base, dt));
    m_Dt = dt;
  }
  void setCharmmContext(std::shared_ptr<CharmmContext> ctx) {
    if (!ctx) throw std::invalid_argument("setCharmmContext: null context");
    apocharmm_detail::check(apo_cuda_integrator_set_charmm_context(m_Base, ctx->handle()));
    m_Ctx = std::move(ctx);
  }
  std::shared_ptr<CharmmContext> getCharmmContext(void) { return m_Ctx; }
  void setNonbondedListUpdateFrequency(const int nfreq) {
    apocharmm_detail::check(apo_cuda_integrator_set_nonbonded_list_update_frequency(m_Base, nfreq));
  }
  void propagate(const int numSteps) {
    apocharmm_detail::check(apo_cuda_integrator_propagate(m_Base, numSteps));
  }
  void subscribe(std::shared_ptr<Subscriber> sub) {
    if (!sub) throw std::invalid_argument("subscribe: null subscriber");
    apocharmm_detail::check(apo_cuda_integrator_subscribe(m_Base, sub->base()));
    m_Subs.push_back(std::move(sub));
  }
  void subscribe(const std::vector<std::shared_ptr<Subscriber>> &sublist) {
    for (auto &s : sublist) subscribe(s);
  }
  void unsubscribe(std::shared_ptr<Subscriber> sub) {
    if (!sub) return;
    int removed = 0;
    apocharmm_detail::check(apo_cuda_integrator_unsubscribe(&removed, m_Base, sub->base()));
    for (size_t k = 0; k < m_Subs.size(); ++k)
      if (m_Subs[k] == sub) {
        m_Subs.erase(m_Subs.begin() + k);
        break;
      }
  }
  std::vector<std::shared_ptr<Subscriber>> &getSubscribers(void) { return m_Subs; }
  long long getCurrentPropagatedStep(void) const {
    long long step = 0;
    apocharmm_detail::check(apo_cuda_integrator_get_current_step(&step, m_Base));
    return step;
  }
  double getInstantaneousTemperature(void) const {
    double t = 0.0;
    apocharmm_detail::check(apo_cuda_integrator_get_instantaneous_temperature(&t, m_Base));
    return t;
  }
  double getAverageTemperature(void) const {
    double t = 0.0;
    apocharmm_detail::check(apo_cuda_integrator_get_average_temperature(&t, m_Base));
    return t;
  }
  void initializeFromRestartFile(const std::string &rstFileName) {
    apocharmm_detail::check(
        apo_cuda_integrator_initialize_from_restart_file(m_Base, rstFileName.c_str()));
  }
  // step through captured CUDA graphs (default on) or plain launches
  void setUseGraphs(const bool flag) {
    apocharmm_detail::check(apo_cuda_integrator_set_use_graphs(m_Base, flag ? 1 : 0));
  }
  int getKernelsPerStep(void) const {
    int k = 0;
    apocharmm_detail::check(apo_cuda_integrator_get_kernels_per_step(&k, m_Base));
    return k;
  }
  apo_cuda_integrator *base() { return m_Base; }

 protected:
  explicit CudaIntegrator(double dt) : m_Dt(dt) {}
  apo_cuda_integrator *m_Base = nullptr;  // borrowed view of the concrete handle
  double m_Dt;
  std::shared_ptr<CharmmContext> m_Ctx;
  std::vector<std::shared_ptr<Subscriber>> m_Subs;
};

class CudaLangevinThermostatIntegrator : public CudaIntegrator {
 public:
  explicit CudaLangevinThermostatIntegrator(const double timeStep) : CudaIntegrator(timeStep) {
    apocharmm_detail::check(apo_cuda_langevin_thermostat_integrator_create(&m_H, timeStep));
    apocharmm_detail::check(apo_cuda_langevin_thermostat_integrator_as_cuda_integrator(&m_Base, m_H));
  }
  ~CudaLangevinThermostatIntegrator() override {
    apo_cuda_langevin_thermostat_integrator_destroy(m_H);
  }
  void setReferenceTemperature(const double referenceTemperature) {
    apocharmm_detail::check(
        apo_cuda_langevin_thermostat_integrator_set_reference_temperature(m_H, referenceTemperature));
    m_RefT = referenceTemperature;
  }
  void setThermostatFriction(const double thermostatFriction) {
    apocharmm_detail::check(
        apo_cuda_langevin_thermostat_integrator_set_thermostat_friction(m_H, thermostatFriction));
    m_Friction = thermostatFriction;
  }
  void setThermostatRngSeed(const std::uint64_t seed) {
    apocharmm_detail::check(apo_cuda_langevin_thermostat_integrator_set_thermostat_rng_seed(m_H, seed));
    m_Seed = seed;
  }
  double getReferenceTemperature(void) const { return m_RefT; }
  double getThermostatFriction(void) const { return m_Friction; }
  std::uint64_t getThermostatRngSeed(void) const { return m_Seed; }
  unsigned long long getRngSequencePos(void) const {
    unsigned long long p = 0;
    apocharmm_detail::check(apo_cuda_langevin_thermostat_integrator_get_rng_sequence_pos(&p, m_H));
    return p;
  }

 private:
  apo_cuda_langevin_thermostat_integrator *m_H = nullptr;
  double m_RefT = 300.0, m_Friction = 0.0;
  std::uint64_t m_Seed = 0;
};

class CudaNoseHooverIntegrator : public CudaIntegrator {
 public:
  explicit CudaNoseHooverIntegrator(const double timeStep) : CudaIntegrator(timeStep) {
    apocharmm_detail::check(apo_cuda_nose_hoover_integrator_create(&m_H, timeStep));
    apocharmm_detail::check(apo_cuda_nose_hoover_integrator_as_cuda_integrator(&m_Base, m_H));
  }
  ~CudaNoseHooverIntegrator() override { apo_cuda_nose_hoover_integrator_destroy(m_H); }
  void setReferenceTemperature(const double referenceTemperature) {
    apocharmm_detail::check(
        apo_cuda_nose_hoover_integrator_set_reference_temperature(m_H, referenceTemperature));
  }
  double getReferenceTemperature(void) const {
    double t = 0.0;
    apocharmm_detail::check(apo_cuda_nose_hoover_integrator_get_reference_temperature(&t, m_H));
    return t;
  }
  void setNoseHooverPistonMass(const double mass) {
    apocharmm_detail::check(apo_cuda_nose_hoover_integrator_set_nose_hoover_piston_mass(m_H, mass));
  }
  void useOldTemperature(const bool flag) {
    apocharmm_detail::check(apo_cuda_nose_hoover_integrator_use_old_temperature(m_H, flag));
  }
  void resetAverageTemperature(void) {
    apocharmm_detail::check(apo_cuda_nose_hoover_integrator_reset_average_temperature(m_H));
  }

 private:
  apo_cuda_nose_hoover_integrator *m_H = nullptr;
};

class CudaLeapFrogIntegrator : public CudaIntegrator {
 public:
  explicit CudaLeapFrogIntegrator(const double timeStep) : CudaIntegrator(timeStep) {
    apocharmm_detail::check(apo_cuda_leap_frog_integrator_create(&m_H, timeStep));
    apocharmm_detail::check(apo_cuda_leap_frog_integrator_as_cuda_integrator(&m_Base, m_H));
  }
  ~CudaLeapFrogIntegrator() override { apo_cuda_leap_frog_integrator_destroy(m_H); }

 private:
  apo_cuda_leap_frog_integrator *m_H = nullptr;
};

// the reference's enum CRYSTAL (include/PBC.h:15)
enum class CRYSTAL { NONE = 0, CUBIC = 1, ORTHORHOMBIC = 2, TETRAGONAL = 3 };

class CudaLangevinPistonIntegrator : public CudaIntegrator {
 public:
  explicit CudaLangevinPistonIntegrator(const double timeStep) : CudaIntegrator(timeStep) {
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_create(&m_H, timeStep));
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_as_cuda_integrator(&m_Base, m_H));
  }
  ~CudaLangevinPistonIntegrator() override { apo_cuda_langevin_piston_integrator_destroy(m_H); }
  void setCrystalType(const CRYSTAL crystalType) {
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_set_crystal_type(m_H, (int)crystalType));
  }
  void setPressure(const std::vector<double> &referencePressure) {
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_set_pressure(
        m_H, referencePressure.data(), referencePressure.size()));
  }
  void setLangevinPistonMass(const std::vector<double> &mass) {
    apocharmm_detail::check(
        apo_cuda_langevin_piston_integrator_set_langevin_piston_mass(m_H, mass.data(), mass.size()));
  }
  std::vector<double> getLangevinPistonMass(void) const {
    std::vector<double> m(3);
    size_t n = 0;
    apocharmm_detail::check(
        apo_cuda_langevin_piston_integrator_get_langevin_piston_mass(m.data(), m.size(), &n, m_H));
    m.resize(n);
    return m;
  }
  void setLangevinPistonFriction(const double pgamma) {
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_set_langevin_piston_friction(m_H, pgamma));
  }
  void setLangevinPistonFrictionSeed(const std::uint64_t seed) {
    apocharmm_detail::check(
        apo_cuda_langevin_piston_integrator_set_langevin_piston_friction_seed(m_H, seed));
  }
  void setRngSequencePos(const unsigned long long pos) {
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_set_rng_sequence_pos(m_H, pos));
  }
  unsigned long long getRngSequencePos(void) const {
    unsigned long long p = 0;
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_get_rng_sequence_pos(&p, m_H));
    return p;
  }
  void setReferenceTemperature(const double referenceTemperature) {
    apocharmm_detail::check(
        apo_cuda_langevin_piston_integrator_set_reference_temperature(m_H, referenceTemperature));
  }
  void useNoseHooverThermostat(const bool flag) {
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_use_nose_hoover_thermostat(m_H, flag));
  }
  void setNoseHooverPistonMass(const double mass) {
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_set_nose_hoover_piston_mass(m_H, mass));
  }
  void useOldTemperature(const bool flag) {
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_use_old_temperature(m_H, flag));
  }
  void setMaxPredictorCorrectorIterations(const int n) {
    apocharmm_detail::check(
        apo_cuda_langevin_piston_integrator_set_max_predictor_corrector_iterations(m_H, n));
  }
  void setConstantSurfaceTension(const bool flag, const double surfaceTension = 0.0) {
    apocharmm_detail::check(
        apo_cuda_langevin_piston_integrator_set_constant_surface_tension(m_H, flag, surfaceTension));
  }
  void resetAverages(void) {
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_reset_averages(m_H));
  }
  std::vector<double> getInstantaneousPressureTensor(void) {
    std::vector<double> p(9);
    apocharmm_detail::check(
        apo_cuda_langevin_piston_integrator_get_instantaneous_pressure_tensor(p.data(), p.size(), m_H));
    return p;
  }
  std::vector<double> getAveragePressureTensor(void) {
    std::vector<double> p(9);
    apocharmm_detail::check(
        apo_cuda_langevin_piston_integrator_get_average_pressure_tensor(p.data(), p.size(), m_H));
    return p;
  }
  double getInstantaneousPressureScalar(void) {
    double p = 0.0;
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_get_instantaneous_pressure_scalar(&p, m_H));
    return p;
  }
  double getAveragePressureScalar(void) {
    double p = 0.0;
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_get_average_pressure_scalar(&p, m_H));
    return p;
  }
  std::vector<double> getLangevinPistonOnStepPosition(void) {
    return vec(apo_cuda_langevin_piston_integrator_get_langevin_piston_on_step_position);
  }
  std::vector<double> getLangevinPistonHalfStepPosition(void) {
    return vec(apo_cuda_langevin_piston_integrator_get_langevin_piston_half_step_position);
  }
  std::vector<double> getLangevinPistonOnStepVelocity(void) {
    return vec(apo_cuda_langevin_piston_integrator_get_langevin_piston_on_step_velocity);
  }
  std::vector<double> getLangevinPistonDeltaPosition(void) {
    return vec(apo_cuda_langevin_piston_integrator_get_langevin_piston_delta_position);
  }
  std::vector<double> getLangevinPistonDeltaPressure(void) {
    return vec(apo_cuda_langevin_piston_integrator_get_langevin_piston_delta_pressure);
  }
  double getInstantaneousSurfaceTension(void) {
    double t = 0.0;
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_get_instantaneous_surface_tension(&t, m_H));
    return t;
  }
  CRYSTAL getCrystalType(void) const {
    int c = 0;
    apocharmm_detail::check(apo_cuda_langevin_piston_integrator_get_crystal_type(&c, m_H));
    return (CRYSTAL)c;
  }
  // velocity, velocity one step back, force, force one step back
  std::vector<double> getNoseHooverPistonState(void) {
    std::vector<double> v(4);
    apocharmm_detail::check(
        apo_cuda_langevin_piston_integrator_get_nose_hoover_piston_state(v.data(), v.size(), m_H));
    return v;
  }
  void setNoseHooverPistonVelocity(const double v) {
    auto s = getNoseHooverPistonState();
    setState(v, s[1], s[2], s[3]);
  }
  void setNoseHooverPistonVelocityPrevious(const double v) {
    auto s = getNoseHooverPistonState();
    setState(s[0], v, s[2], s[3]);
  }
  void setNoseHooverPistonForce(const double f) {
    auto s = getNoseHooverPistonState();
    setState(s[0], s[1], f, s[3]);
  }
  void setNoseHooverPistonForcePrevious(const double f) {
    auto s = getNoseHooverPistonState();
    setState(s[0], s[1], s[2], f);
  }

 private:
  using VecFn = apo_status (*)(double *, const size_t, size_t *, apo_cuda_langevin_piston_integrator *);
  std::vector<double> vec(VecFn fn) {
    std::vector<double> x(3);
    size_t n = 0;
    apocharmm_detail::check(fn(x.data(), x.size(), &n, m_H));
    x.resize(n);
    return x;
  }
  void setState(double v, double vp, double f, double fp) {
    apocharmm_detail::check(
        apo_cuda_langevin_piston_integrator_set_nose_hoover_piston_state(m_H, v, vp, f, fp));
  }
  apo_cuda_langevin_piston_integrator *m_H = nullptr;
};
