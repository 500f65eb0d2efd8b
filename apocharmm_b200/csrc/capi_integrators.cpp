// C ABI: integrators and subscribers (same conventions as capi.cpp).
#include "apocharmm_c/CudaIntegrator.h"
#include "apocharmm_c/CudaLangevinPistonIntegrator.h"
#include "apocharmm_c/CudaLangevinThermostatIntegrator.h"
#include "apocharmm_c/CudaNoseHooverIntegrator.h"
#include "apocharmm_c/DcdSubscriber.h"
#include "apocharmm_c/RestartFile.h"
#include "apocharmm_c/RestartSubscriber.h"
#include "apocharmm_c/Subscriber.h"
#include <algorithm>
#include <cstdio>

#include "capi_internal.h"
#include "integrators.h"
#include "subscribers.h"

using namespace apocapi;

struct apo_subscriber { std::shared_ptr<apo::Subscriber> object; };
struct apo_dcd_subscriber {
  apo_subscriber base;
  std::shared_ptr<apo::DcdSubscriber> object;
};
struct apo_restart_subscriber {
  apo_subscriber base;
  std::shared_ptr<apo::RestartSubscriber> object;
};
struct apo_cuda_integrator { std::shared_ptr<apo::CudaIntegrator> object; };
struct apo_cuda_nose_hoover_integrator {
  apo_cuda_integrator base;
  std::shared_ptr<apo::CudaNoseHooverIntegrator> object;
};
struct apo_cuda_langevin_thermostat_integrator {
  apo_cuda_integrator base;
  std::shared_ptr<apo::CudaLangevinThermostatIntegrator> object;
};
struct apo_cuda_leap_frog_integrator {
  apo_cuda_integrator base;
  std::shared_ptr<apo::CudaLeapFrogIntegrator> object;
};

// ------------------------------------------------------------ base view ----

extern "C" apo_status apo_cuda_integrator_set_time_step(apo_cuda_integrator *it, const double dt) {
  const char *fn = "apo_cuda_integrator_set_time_step";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(it, fn, "CudaIntegrator"));
    if (!(dt > 0) || !std::isfinite(dt)) return invalid(fn, "time step must be positive");
    it->object->setTimeStep(dt);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_integrator_set_charmm_context(apo_cuda_integrator *it,
                                                             apo_charmm_context *ctx) {
  const char *fn = "apo_cuda_integrator_set_charmm_context";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(it, fn, "CudaIntegrator"));
    APO_RETURN_IF(require_handle(ctx, fn, "CharmmContext"));
    it->object->setCharmmContext(ctx->object);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_integrator_subscribe(apo_cuda_integrator *it, apo_subscriber *sub) {
  const char *fn = "apo_cuda_integrator_subscribe";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(it, fn, "CudaIntegrator"));
    APO_RETURN_IF(require_handle(sub, fn, "Subscriber"));
    it->object->subscribe(sub->object);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_integrator_unsubscribe(int *removed, apo_cuda_integrator *it,
                                                      apo_subscriber *sub) {
  const char *fn = "apo_cuda_integrator_unsubscribe";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(removed, fn, "removed"));
    APO_RETURN_IF(require_handle(it, fn, "CudaIntegrator"));
    APO_RETURN_IF(require_handle(sub, fn, "Subscriber"));
    *removed = it->object->unsubscribe(sub->object) ? 1 : 0;
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_integrator_propagate(apo_cuda_integrator *it, const int n) {
  const char *fn = "apo_cuda_integrator_propagate";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(it, fn, "CudaIntegrator"));
    if (n < 0) return invalid(fn, "num_steps must be >= 0");
    it->object->propagate(n);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_integrator_initialize_from_restart_file(apo_cuda_integrator *it,
                                                                       const char *path) {
  const char *fn = "apo_cuda_integrator_initialize_from_restart_file";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(it, fn, "CudaIntegrator"));
    APO_RETURN_IF(require_string(path, fn, "path"));
    it->object->initializeFromRestartFile(path);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_integrator_set_nonbonded_list_update_frequency(apo_cuda_integrator *it,
                                                                              const int f) {
  const char *fn = "apo_cuda_integrator_set_nonbonded_list_update_frequency";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(it, fn, "CudaIntegrator"));
    if (f < 1) return invalid(fn, "frequency must be >= 1");
    it->object->setNonbondedListUpdateFrequency(f);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_integrator_set_use_graphs(apo_cuda_integrator *it, const int g) {
  const char *fn = "apo_cuda_integrator_set_use_graphs";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(it, fn, "CudaIntegrator"));
    it->object->setUseGraphs(g != 0);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_integrator_get_current_step(long long *step,
                                                           const apo_cuda_integrator *it) {
  const char *fn = "apo_cuda_integrator_get_current_step";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(step, fn, "step"));
    APO_RETURN_IF(require_handle(it, fn, "CudaIntegrator"));
    *step = it->object->getCurrentPropagatedStep();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_integrator_get_average_temperature(double *t,
                                                                  const apo_cuda_integrator *it) {
  const char *fn = "apo_cuda_integrator_get_average_temperature";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(t, fn, "temperature"));
    APO_RETURN_IF(require_handle(it, fn, "CudaIntegrator"));
    *t = it->object->getAverageTemperature();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_integrator_get_instantaneous_temperature(double *t,
                                                                        const apo_cuda_integrator *it) {
  const char *fn = "apo_cuda_integrator_get_instantaneous_temperature";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(t, fn, "temperature"));
    APO_RETURN_IF(require_handle(it, fn, "CudaIntegrator"));
    *t = it->object->getInstantaneousTemperature();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_integrator_get_kernels_per_step(int *k, const apo_cuda_integrator *it) {
  const char *fn = "apo_cuda_integrator_get_kernels_per_step";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(k, fn, "kernels"));
    APO_RETURN_IF(require_handle(it, fn, "CudaIntegrator"));
    *k = it->object->kernelsPerStep();
    return APO_STATUS_OK;
  }, fn);
}

// ---------------------------------------------------------- Nose-Hoover ----

extern "C" apo_status apo_cuda_nose_hoover_integrator_create(apo_cuda_nose_hoover_integrator **out,
                                                             const double dt) {
  const char *fn = "apo_cuda_nose_hoover_integrator_create";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    if (!(dt > 0) || !std::isfinite(dt)) return invalid(fn, "time step must be positive");
    auto h = std::make_unique<apo_cuda_nose_hoover_integrator>();
    h->object = std::make_shared<apo::CudaNoseHooverIntegrator>(dt);
    h->base.object = h->object;
    *out = h.release();
    return APO_STATUS_OK;
  }, fn);
}
extern "C" void apo_cuda_nose_hoover_integrator_destroy(apo_cuda_nose_hoover_integrator *it) { delete it; }

#define NH_SET(fname, type, body)                                               \
  extern "C" apo_status fname(apo_cuda_nose_hoover_integrator *it, const type v) { \
    return guard([&]() -> apo_status {                                          \
      APO_RETURN_IF(require_handle(it, #fname, "CudaNoseHooverIntegrator"));    \
      body;                                                                     \
      return APO_STATUS_OK;                                                     \
    }, #fname);                                                                 \
  }
NH_SET(apo_cuda_nose_hoover_integrator_set_reference_temperature, double,
       if (!(v >= 0)) return invalid("set_reference_temperature", "temperature must be >= 0");
       it->object->setReferenceTemperature(v))
NH_SET(apo_cuda_nose_hoover_integrator_set_nose_hoover_piston_mass, double,
       if (!(v > 0)) return invalid("set_nose_hoover_piston_mass", "mass must be positive");
       it->object->setNoseHooverPistonMass(v))
NH_SET(apo_cuda_nose_hoover_integrator_use_old_temperature, bool, it->object->useOldTemperature(v))

extern "C" apo_status apo_cuda_nose_hoover_integrator_reset_average_temperature(
    apo_cuda_nose_hoover_integrator *it) {
  const char *fn = "apo_cuda_nose_hoover_integrator_reset_average_temperature";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(it, fn, "CudaNoseHooverIntegrator"));
    if (it->object->getCharmmContext()) it->object->resetAverageTemperature();
    return APO_STATUS_OK;
  }, fn);
}

#define NH_GET(fname, call)                                                                      \
  extern "C" apo_status fname(double *t, const apo_cuda_nose_hoover_integrator *it) {            \
    return guard([&]() -> apo_status {                                                           \
      APO_RETURN_IF(require_ptr(t, #fname, "temperature"));                                      \
      *t = 0.0;                                                                                  \
      APO_RETURN_IF(require_handle(it, #fname, "CudaNoseHooverIntegrator"));                     \
      *t = call;                                                                                 \
      return APO_STATUS_OK;                                                                      \
    }, #fname);                                                                                  \
  }
NH_GET(apo_cuda_nose_hoover_integrator_get_reference_temperature, it->object->getReferenceTemperature())
NH_GET(apo_cuda_nose_hoover_integrator_get_average_temperature,
       it->object->getCharmmContext() ? it->object->getAverageTemperature() : 0.0)
NH_GET(apo_cuda_nose_hoover_integrator_get_instantaneous_temperature,
       it->object->getCharmmContext() ? it->object->getInstantaneousTemperature() : 0.0)

extern "C" apo_status apo_cuda_nose_hoover_integrator_as_cuda_integrator(
    apo_cuda_integrator **out, apo_cuda_nose_hoover_integrator *it) {
  const char *fn = "apo_cuda_nose_hoover_integrator_as_cuda_integrator";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    APO_RETURN_IF(require_handle(it, fn, "CudaNoseHooverIntegrator"));
    *out = &it->base;
    return APO_STATUS_OK;
  }, fn);
}

// ------------------------------------------------------------- Langevin ----

extern "C" apo_status apo_cuda_langevin_thermostat_integrator_create(
    apo_cuda_langevin_thermostat_integrator **out, const double dt) {
  const char *fn = "apo_cuda_langevin_thermostat_integrator_create";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    if (!(dt > 0) || !std::isfinite(dt)) return invalid(fn, "time step must be positive");
    auto h = std::make_unique<apo_cuda_langevin_thermostat_integrator>();
    h->object = std::make_shared<apo::CudaLangevinThermostatIntegrator>(dt);
    h->base.object = h->object;
    *out = h.release();
    return APO_STATUS_OK;
  }, fn);
}
extern "C" void apo_cuda_langevin_thermostat_integrator_destroy(apo_cuda_langevin_thermostat_integrator *it) {
  delete it;
}

#define LG_SET(fname, type, body)                                                        \
  extern "C" apo_status fname(apo_cuda_langevin_thermostat_integrator *it, const type v) { \
    return guard([&]() -> apo_status {                                                   \
      APO_RETURN_IF(require_handle(it, #fname, "CudaLangevinThermostatIntegrator"));     \
      body;                                                                              \
      return APO_STATUS_OK;                                                              \
    }, #fname);                                                                          \
  }
LG_SET(apo_cuda_langevin_thermostat_integrator_set_thermostat_friction, double,
       if (!(v >= 0)) return invalid("set_thermostat_friction", "friction must be >= 0");
       it->object->setThermostatFriction(v))
LG_SET(apo_cuda_langevin_thermostat_integrator_set_reference_temperature, double,
       if (!(v >= 0)) return invalid("set_reference_temperature", "temperature must be >= 0");
       it->object->setReferenceTemperature(v))
LG_SET(apo_cuda_langevin_thermostat_integrator_set_thermostat_rng_seed, uint64_t,
       it->object->setThermostatRngSeed(v))

extern "C" apo_status apo_cuda_langevin_thermostat_integrator_get_rng_sequence_pos(
    unsigned long long *pos, const apo_cuda_langevin_thermostat_integrator *it) {
  const char *fn = "apo_cuda_langevin_thermostat_integrator_get_rng_sequence_pos";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(pos, fn, "pos"));
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinThermostatIntegrator"));
    *pos = it->object->getCharmmContext() ? it->object->getRngSequencePos() : 0ull;
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_langevin_thermostat_integrator_as_cuda_integrator(
    apo_cuda_integrator **out, apo_cuda_langevin_thermostat_integrator *it) {
  const char *fn = "apo_cuda_langevin_thermostat_integrator_as_cuda_integrator";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinThermostatIntegrator"));
    *out = &it->base;
    return APO_STATUS_OK;
  }, fn);
}

// ------------------------------------------------------------- leapfrog ----

extern "C" apo_status apo_cuda_leap_frog_integrator_create(apo_cuda_leap_frog_integrator **out,
                                                           const double dt) {
  const char *fn = "apo_cuda_leap_frog_integrator_create";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    if (!(dt > 0) || !std::isfinite(dt)) return invalid(fn, "time step must be positive");
    auto h = std::make_unique<apo_cuda_leap_frog_integrator>();
    h->object = std::make_shared<apo::CudaLeapFrogIntegrator>(dt);
    h->base.object = h->object;
    *out = h.release();
    return APO_STATUS_OK;
  }, fn);
}
extern "C" void apo_cuda_leap_frog_integrator_destroy(apo_cuda_leap_frog_integrator *it) { delete it; }
extern "C" apo_status apo_cuda_leap_frog_integrator_as_cuda_integrator(apo_cuda_integrator **out,
                                                                       apo_cuda_leap_frog_integrator *it) {
  const char *fn = "apo_cuda_leap_frog_integrator_as_cuda_integrator";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    APO_RETURN_IF(require_handle(it, fn, "CudaLeapFrogIntegrator"));
    *out = &it->base;
    return APO_STATUS_OK;
  }, fn);
}

// ----------------------------------------------------------- subscribers ----

extern "C" apo_status apo_subscriber_set_report_frequency(apo_subscriber *s, const int f) {
  const char *fn = "apo_subscriber_set_report_frequency";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(s, fn, "Subscriber"));
    if (f <= 0) return invalid(fn, "report frequency must be positive");
    s->object->setReportFrequency(f);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_subscriber_get_report_frequency(int *f, const apo_subscriber *s) {
  const char *fn = "apo_subscriber_get_report_frequency";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(f, fn, "report_frequency"));
    APO_RETURN_IF(require_handle(s, fn, "Subscriber"));
    *f = s->object->getReportFrequency();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_dcd_subscriber_create_with_report_frequency(apo_dcd_subscriber **out,
                                                                      const char *path, const int f) {
  const char *fn = "apo_dcd_subscriber_create_with_report_frequency";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    APO_RETURN_IF(require_string(path, fn, "path"));
    if (f <= 0) return invalid(fn, "report frequency must be positive");
    auto h = std::make_unique<apo_dcd_subscriber>();
    h->object = std::make_shared<apo::DcdSubscriber>(path, f);
    h->base.object = h->object;
    *out = h.release();
    return APO_STATUS_OK;
  }, fn);
}
extern "C" apo_status apo_dcd_subscriber_create(apo_dcd_subscriber **out, const char *path) {
  return apo_dcd_subscriber_create_with_report_frequency(out, path, 1000);
}
extern "C" void apo_dcd_subscriber_destroy(apo_dcd_subscriber *s) { delete s; }
extern "C" apo_status apo_dcd_subscriber_as_subscriber(apo_subscriber **out, apo_dcd_subscriber *s) {
  const char *fn = "apo_dcd_subscriber_as_subscriber";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    APO_RETURN_IF(require_handle(s, fn, "DcdSubscriber"));
    *out = &s->base;
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_restart_subscriber_create_with_report_frequency(apo_restart_subscriber **out,
                                                                          const char *path, const int f) {
  const char *fn = "apo_restart_subscriber_create_with_report_frequency";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    APO_RETURN_IF(require_string(path, fn, "path"));
    if (f <= 0) return invalid(fn, "report frequency must be positive");
    auto h = std::make_unique<apo_restart_subscriber>();
    h->object = std::make_shared<apo::RestartSubscriber>(path, f);
    h->base.object = h->object;
    *out = h.release();
    return APO_STATUS_OK;
  }, fn);
}
extern "C" apo_status apo_restart_subscriber_create(apo_restart_subscriber **out, const char *path) {
  return apo_restart_subscriber_create_with_report_frequency(out, path, 1000);
}
extern "C" void apo_restart_subscriber_destroy(apo_restart_subscriber *s) { delete s; }
extern "C" apo_status apo_restart_subscriber_as_subscriber(apo_subscriber **out, apo_restart_subscriber *s) {
  const char *fn = "apo_restart_subscriber_as_subscriber";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    APO_RETURN_IF(require_handle(s, fn, "RestartSubscriber"));
    *out = &s->base;
    return APO_STATUS_OK;
  }, fn);
}

// ---------------------------------------------------------- restart files ----

extern "C" apo_status apo_restart_file_read_header(const char *path, int *natom, long long *npriv,
                                                   int *ndegf, unsigned long long *seed,
                                                   unsigned long long *rngpos, int *has_rng,
                                                   double *box3, double *pnhv, double *pnhf) {
  const char *fn = "apo_restart_file_read_header";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_string(path, fn, "path"));
    if (!natom || !npriv || !ndegf || !seed || !rngpos || !has_rng || !box3 || !pnhv || !pnhf)
      return invalid(fn, "null output pointer");
    const apo::RestartRecord r = apo::readRestartFile(path);
    *natom = r.natom;
    *npriv = r.npriv;
    *ndegf = r.ndegf;
    *seed = r.seed;
    *rngpos = r.rngpos;
    *has_rng = r.has_rng ? 1 : 0;
    for (int d = 0; d < 3; ++d) box3[d] = r.box[d];
    *pnhv = r.pnhv;
    *pnhf = r.pnhf;
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_restart_file_read_crystal(const char *path, char *crystal5, double *hdot3) {
  const char *fn = "apo_restart_file_read_crystal";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_string(path, fn, "path"));
    if (!crystal5 || !hdot3) return invalid(fn, "null output pointer");
    const apo::RestartRecord r = apo::readRestartFile(path);
    std::snprintf(crystal5, 5, "%s", r.crystal.c_str());
    for (int d = 0; d < 3; ++d) hdot3[d] = r.hdot[d];
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_restart_file_read(const char *path, const int natom, double *xold,
                                            double *vel, double *delta) {
  const char *fn = "apo_restart_file_read";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_string(path, fn, "path"));
    if (!xold || !vel || !delta) return invalid(fn, "null output array");
    const apo::RestartRecord r = apo::readRestartFile(path);
    if (r.natom != natom) return invalid(fn, "natom does not match the file");
    std::copy(r.xold.begin(), r.xold.end(), xold);
    std::copy(r.vel.begin(), r.vel.end(), vel);
    std::copy(r.delta.begin(), r.delta.end(), delta);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_restart_file_write(const char *path, const int natom, const long long npriv,
                                             const int ndegf, const unsigned long long seed,
                                             const unsigned long long rngpos, const int has_rng,
                                             const double *box3, const double pnhv, const double pnhf,
                                             const double *xold, const double *vel,
                                             const double *delta) {
  const char *fn = "apo_restart_file_write";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_string(path, fn, "path"));
    if (natom < 0 || npriv < 0) return invalid(fn, "natom and npriv must be >= 0");
    if (!box3 || (natom > 0 && (!xold || !vel || !delta))) return invalid(fn, "null input array");
    apo::RestartRecord r;
    r.natom = natom;
    r.npriv = r.nstep = npriv;
    r.ndegf = ndegf;
    r.seed = seed;
    r.rngpos = rngpos;
    r.has_rng = has_rng != 0;
    for (int d = 0; d < 3; ++d) r.box[d] = box3[d];
    r.pnhv = pnhv;
    r.pnhf = pnhf;
    const size_t n3 = (size_t)3 * natom;
    r.xold.assign(xold, xold + n3);
    r.vel.assign(vel, vel + n3);
    r.delta.assign(delta, delta + n3);
    apo::writeRestartFile(path, r);
    return APO_STATUS_OK;
  }, fn);
}

// ------------------------------------------------------ Langevin piston ----

struct apo_cuda_langevin_piston_integrator {
  apo_cuda_integrator base;
  std::shared_ptr<apo::CudaLangevinPistonIntegrator> object;
};

extern "C" apo_status apo_cuda_langevin_piston_integrator_create(
    apo_cuda_langevin_piston_integrator **out, const double dt) {
  const char *fn = "apo_cuda_langevin_piston_integrator_create";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    if (!(dt > 0) || !std::isfinite(dt)) return invalid(fn, "time step must be positive");
    auto h = std::make_unique<apo_cuda_langevin_piston_integrator>();
    h->object = std::make_shared<apo::CudaLangevinPistonIntegrator>(dt);
    h->base.object = h->object;
    *out = h.release();
    return APO_STATUS_OK;
  }, fn);
}
extern "C" void apo_cuda_langevin_piston_integrator_destroy(apo_cuda_langevin_piston_integrator *it) {
  delete it;
}

extern "C" apo_status apo_cuda_langevin_piston_integrator_as_cuda_integrator(
    apo_cuda_integrator **out, apo_cuda_langevin_piston_integrator *it) {
  const char *fn = "apo_cuda_langevin_piston_integrator_as_cuda_integrator";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(prepare_out(out, fn));
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinPistonIntegrator"));
    *out = &it->base;
    return APO_STATUS_OK;
  }, fn);
}

#define LP_SET(fname, type, body)                                                   \
  extern "C" apo_status fname(apo_cuda_langevin_piston_integrator *it, const type v) { \
    return guard([&]() -> apo_status {                                              \
      APO_RETURN_IF(require_handle(it, #fname, "CudaLangevinPistonIntegrator"));    \
      body;                                                                         \
      return APO_STATUS_OK;                                                         \
    }, #fname);                                                                     \
  }
LP_SET(apo_cuda_langevin_piston_integrator_set_crystal_type, int,
       if (v < 1 || v > 3) return invalid("set_crystal_type",
                                          "crystal type must be 1 (cubic), 2 (orthorhombic) or 3 (tetragonal)");
       it->object->setCrystalType((apo::Crystal)v))
LP_SET(apo_cuda_langevin_piston_integrator_set_langevin_piston_friction, double,
       if (!(v >= 0) || !std::isfinite(v)) return invalid("set_langevin_piston_friction", "friction must be >= 0");
       it->object->setLangevinPistonFriction(v))
LP_SET(apo_cuda_langevin_piston_integrator_set_langevin_piston_friction_seed, uint64_t,
       it->object->setLangevinPistonFrictionSeed(v))
LP_SET(apo_cuda_langevin_piston_integrator_set_rng_sequence_pos, unsigned long long,
       it->object->setRngSequencePos(v))
LP_SET(apo_cuda_langevin_piston_integrator_set_reference_temperature, double,
       if (!(v >= 0) || !std::isfinite(v)) return invalid("set_reference_temperature", "temperature must be >= 0");
       it->object->setReferenceTemperature(v))
LP_SET(apo_cuda_langevin_piston_integrator_use_nose_hoover_thermostat, bool,
       it->object->useNoseHooverThermostat(v))
LP_SET(apo_cuda_langevin_piston_integrator_set_nose_hoover_piston_mass, double,
       if (!(v > 0) || !std::isfinite(v)) return invalid("set_nose_hoover_piston_mass", "mass must be positive");
       it->object->setNoseHooverPistonMass(v))
LP_SET(apo_cuda_langevin_piston_integrator_use_old_temperature, bool, it->object->useOldTemperature(v))
LP_SET(apo_cuda_langevin_piston_integrator_set_max_predictor_corrector_iterations, int,
       it->object->setMaxPredictorCorrectorIterations(v))

extern "C" apo_status apo_cuda_langevin_piston_integrator_set_constant_surface_tension(
    apo_cuda_langevin_piston_integrator *it, const bool flag, const double tension) {
  const char *fn = "apo_cuda_langevin_piston_integrator_set_constant_surface_tension";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinPistonIntegrator"));
    if (!std::isfinite(tension)) return invalid(fn, "surface tension must be finite");
    it->object->setConstantSurfaceTension(flag);
    it->object->setSurfaceTension(tension);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_langevin_piston_integrator_set_pressure(
    apo_cuda_langevin_piston_integrator *it, const double *p, const size_t len) {
  const char *fn = "apo_cuda_langevin_piston_integrator_set_pressure";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinPistonIntegrator"));
    APO_RETURN_IF(require_ptr(p, fn, "pressure"));
    it->object->setPressure(std::vector<double>(p, p + len));
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_langevin_piston_integrator_set_langevin_piston_mass(
    apo_cuda_langevin_piston_integrator *it, const double *m, const size_t len) {
  const char *fn = "apo_cuda_langevin_piston_integrator_set_langevin_piston_mass";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinPistonIntegrator"));
    APO_RETURN_IF(require_ptr(m, fn, "mass"));
    for (size_t k = 0; k < len; ++k)
      if (!(m[k] >= 0) || !std::isfinite(m[k])) return invalid(fn, "masses must be >= 0");
    it->object->setLangevinPistonMass(std::vector<double>(m, m + len));
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_langevin_piston_integrator_reset_averages(
    apo_cuda_langevin_piston_integrator *it) {
  const char *fn = "apo_cuda_langevin_piston_integrator_reset_averages";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinPistonIntegrator"));
    it->object->resetAverages();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_langevin_piston_integrator_get_rng_sequence_pos(
    unsigned long long *pos, const apo_cuda_langevin_piston_integrator *it) {
  const char *fn = "apo_cuda_langevin_piston_integrator_get_rng_sequence_pos";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(pos, fn, "pos"));
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinPistonIntegrator"));
    *pos = it->object->getRngSequencePos();
    return APO_STATUS_OK;
  }, fn);
}

namespace {
apo_status lp_tensor(double *out, size_t len, apo_cuda_langevin_piston_integrator *it,
                     const char *fn, bool average) {
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_buffer(out, len, 9, fn, "pressure"));
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinPistonIntegrator"));
    if (!it->object->getCharmmContext())
      return set_error(APO_STATUS_NOT_INITIALIZED, std::string(fn) + ": no CharmmContext was set");
    const auto v = average ? it->object->getAveragePressureTensor()
                           : it->object->getInstantaneousPressureTensor();
    std::copy(v.begin(), v.end(), out);
    return APO_STATUS_OK;
  }, fn);
}
apo_status lp_scalar(double *out, apo_cuda_langevin_piston_integrator *it, const char *fn,
                     bool average) {
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(out, fn, "pressure"));
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinPistonIntegrator"));
    if (!it->object->getCharmmContext())
      return set_error(APO_STATUS_NOT_INITIALIZED, std::string(fn) + ": no CharmmContext was set");
    *out = average ? it->object->getAveragePressureScalar()
                   : it->object->getInstantaneousPressureScalar();
    return APO_STATUS_OK;
  }, fn);
}
}  // namespace

extern "C" apo_status apo_cuda_langevin_piston_integrator_get_instantaneous_pressure_tensor(
    double *p, const size_t len, apo_cuda_langevin_piston_integrator *it) {
  return lp_tensor(p, len, it, "apo_cuda_langevin_piston_integrator_get_instantaneous_pressure_tensor",
                   false);
}
extern "C" apo_status apo_cuda_langevin_piston_integrator_get_average_pressure_tensor(
    double *p, const size_t len, apo_cuda_langevin_piston_integrator *it) {
  return lp_tensor(p, len, it, "apo_cuda_langevin_piston_integrator_get_average_pressure_tensor", true);
}
extern "C" apo_status apo_cuda_langevin_piston_integrator_get_instantaneous_pressure_scalar(
    double *p, apo_cuda_langevin_piston_integrator *it) {
  return lp_scalar(p, it, "apo_cuda_langevin_piston_integrator_get_instantaneous_pressure_scalar",
                   false);
}
extern "C" apo_status apo_cuda_langevin_piston_integrator_get_average_pressure_scalar(
    double *p, apo_cuda_langevin_piston_integrator *it) {
  return lp_scalar(p, it, "apo_cuda_langevin_piston_integrator_get_average_pressure_scalar", true);
}

extern "C" apo_status apo_cuda_langevin_piston_integrator_get_langevin_piston_mass(
    double *m, const size_t len, size_t *num, const apo_cuda_langevin_piston_integrator *it) {
  const char *fn = "apo_cuda_langevin_piston_integrator_get_langevin_piston_mass";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(num, fn, "num"));
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinPistonIntegrator"));
    const auto v = it->object->getLangevinPistonMass();
    *num = v.size();
    APO_RETURN_IF(require_buffer(m, len, v.size(), fn, "mass"));
    std::copy(v.begin(), v.end(), m);
    return APO_STATUS_OK;
  }, fn);
}

namespace {
template <typename G>
apo_status lp_vector(double *x, size_t len, size_t *num, apo_cuda_langevin_piston_integrator *it,
                     const char *fn, G get) {
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(num, fn, "num"));
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinPistonIntegrator"));
    if (!it->object->getCharmmContext())
      return set_error(APO_STATUS_NOT_INITIALIZED, std::string(fn) + ": no CharmmContext was set");
    const std::vector<double> v = get(*it->object);
    *num = v.size();
    APO_RETURN_IF(require_buffer(x, len, v.size(), fn, "output"));
    std::copy(v.begin(), v.end(), x);
    return APO_STATUS_OK;
  }, fn);
}
}  // namespace

#define LP_VECTOR(fname, method)                                                              \
  extern "C" apo_status fname(double *x, const size_t len, size_t *num,                      \
                              apo_cuda_langevin_piston_integrator *it) {                     \
    return lp_vector(x, len, num, it, #fname,                                                 \
                     [](apo::CudaLangevinPistonIntegrator &o) { return o.method(); });       \
  }
LP_VECTOR(apo_cuda_langevin_piston_integrator_get_langevin_piston_on_step_position,
          getLangevinPistonOnStepPosition)
LP_VECTOR(apo_cuda_langevin_piston_integrator_get_langevin_piston_half_step_position,
          getLangevinPistonHalfStepPosition)
LP_VECTOR(apo_cuda_langevin_piston_integrator_get_langevin_piston_on_step_velocity,
          getLangevinPistonOnStepVelocity)
LP_VECTOR(apo_cuda_langevin_piston_integrator_get_langevin_piston_delta_position,
          getLangevinPistonDeltaPosition)
LP_VECTOR(apo_cuda_langevin_piston_integrator_get_langevin_piston_delta_pressure,
          getLangevinPistonDeltaPressure)
#undef LP_VECTOR

extern "C" apo_status apo_cuda_langevin_piston_integrator_get_instantaneous_surface_tension(
    double *t, apo_cuda_langevin_piston_integrator *it) {
  const char *fn = "apo_cuda_langevin_piston_integrator_get_instantaneous_surface_tension";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(t, fn, "tension"));
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinPistonIntegrator"));
    if (!it->object->getCharmmContext())
      return set_error(APO_STATUS_NOT_INITIALIZED, std::string(fn) + ": no CharmmContext was set");
    *t = it->object->getInstantaneousSurfaceTension();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_langevin_piston_integrator_get_crystal_type(
    int *c, const apo_cuda_langevin_piston_integrator *it) {
  const char *fn = "apo_cuda_langevin_piston_integrator_get_crystal_type";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(c, fn, "crystal_type"));
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinPistonIntegrator"));
    *c = (int)it->object->getCrystalType();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_langevin_piston_integrator_get_nose_hoover_piston_state(
    double *st, const size_t len, apo_cuda_langevin_piston_integrator *it) {
  const char *fn = "apo_cuda_langevin_piston_integrator_get_nose_hoover_piston_state";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_buffer(st, len, 4, fn, "state"));
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinPistonIntegrator"));
    if (!it->object->getCharmmContext())
      return set_error(APO_STATUS_NOT_INITIALIZED, std::string(fn) + ": no CharmmContext was set");
    const auto v = it->object->getNoseHooverPistonState();
    std::copy(v.begin(), v.end(), st);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_cuda_langevin_piston_integrator_set_nose_hoover_piston_state(
    apo_cuda_langevin_piston_integrator *it, const double v, const double v_prev, const double f,
    const double f_prev) {
  const char *fn = "apo_cuda_langevin_piston_integrator_set_nose_hoover_piston_state";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(it, fn, "CudaLangevinPistonIntegrator"));
    if (!std::isfinite(v) || !std::isfinite(v_prev) || !std::isfinite(f) || !std::isfinite(f_prev))
      return invalid(fn, "values must be finite");
    if (!it->object->getCharmmContext())
      return set_error(APO_STATUS_NOT_INITIALIZED, std::string(fn) + ": no CharmmContext was set");
    it->object->setNoseHooverPistonState(v, v_prev, f, f_prev);
    return APO_STATUS_OK;
  }, fn);
}
