// C ABI of the batch engine (include/apocharmm_c/Batch.h); same conventions
// as the rest of the C ABI: *out = NULL first, apo_status everywhere,
// messages through apo_last_error.
#include "apocharmm_c/Batch.h"

#include <stdexcept>

#include "batch.h"
#include "capi_internal.h"

using namespace apocapi;

struct apo_batch {
  std::shared_ptr<apo::Batch> object;
};

#define APO_RETURN_IF_B(x)               \
  do {                                   \
    apo_status st_ = (x);                \
    if (st_ != APO_STATUS_OK) return st_; \
  } while (0)

namespace {
apo_status require_batch(const apo_batch *b, const char *fn, bool init) {
  if (b == nullptr || !b->object) return invalid(fn, "batch handle is NULL");
  if (init && !b->object->isInitialized())
    return set_error(APO_STATUS_NOT_INITIALIZED, std::string(fn) + ": batch is not initialized");
  return APO_STATUS_OK;
}
apo_status require_len(const apo_batch *b, int sys, size_t len, const char *fn) {
  if (sys >= b->object->numSystems()) return invalid(fn, "system index out of range");
  if (len < 3 * (size_t)b->object->numAtoms(sys)) return invalid(fn, "buffer shorter than 3 N");
  return APO_STATUS_OK;
}
}  // namespace

extern "C" apo_status apo_batch_create(apo_batch **out, const int order, const int tpw,
                                       const int precise) {
  const char *fn = "apo_batch_create";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(prepare_out(out, fn));
    try {
      auto b = std::make_shared<apo::Batch>(order, tpw, precise != 0);
      *out = new apo_batch{b};
    } catch (const std::invalid_argument &e) {
      return set_error(APO_STATUS_INVALID_ARGUMENT, e.what());
    }
    return APO_STATUS_OK;
  }, fn);
}

extern "C" void apo_batch_destroy(apo_batch *b) { delete b; }

extern "C" apo_status apo_batch_add_system(apo_batch *b, const apo_charmm_psf *psf,
                                           const apo_charmm_parameters *prm, const double bx,
                                           const double by, const double bz, const double kappa,
                                           const double cutnb, const double ctonnb,
                                           const double ctofnb, const int nx, const int ny,
                                           const int nz, const unsigned long long seed,
                                           int *index) {
  const char *fn = "apo_batch_add_system";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(require_batch(b, fn, false));
    APO_RETURN_IF_B(require_handle(psf, fn, "CharmmPsf"));
    APO_RETURN_IF_B(require_handle(prm, fn, "CharmmParameters"));
    apo::SystemSpec y;
    y.psf = psf->object;
    y.prm = prm->object;
    y.box = {bx, by, bz};
    y.kappa = kappa;
    y.cutnb = cutnb;
    y.ctonnb = ctonnb;
    y.ctofnb = ctofnb;
    y.nfft = {nx, ny, nz};
    y.seed = seed;
    const int k = b->object->addSystem(y);
    if (index) *index = k;
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_batch_initialize(apo_batch *b) {
  const char *fn = "apo_batch_initialize";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(require_batch(b, fn, false));
    try {
      b->object->initialize();
    } catch (const std::invalid_argument &e) {
      return set_error(APO_STATUS_INVALID_ARGUMENT, std::string(fn) + ": " + e.what());
    }
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_batch_get_num_systems(int *n, const apo_batch *b) {
  const char *fn = "apo_batch_get_num_systems";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(require_ptr(n, fn, "num_systems"));
    APO_RETURN_IF_B(require_batch(b, fn, false));
    *n = b->object->numSystems();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_batch_get_num_atoms(size_t *n, const apo_batch *b, const int sys) {
  const char *fn = "apo_batch_get_num_atoms";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(require_ptr(n, fn, "num_atoms"));
    APO_RETURN_IF_B(require_batch(b, fn, true));
    if (sys >= b->object->numSystems()) return invalid(fn, "system index out of range");
    *n = (size_t)b->object->numAtoms(sys);
    return APO_STATUS_OK;
  }, fn);
}

#define APO_BATCH_XYZ_IN(fname, method)                                                   \
  extern "C" apo_status fname(apo_batch *b, const int sys, const double *xyz,             \
                              const size_t len) {                                         \
    const char *fn = #fname;                                                              \
    return guard([&]() -> apo_status {                                                    \
      APO_RETURN_IF_B(require_batch(b, fn, true));                                        \
      APO_RETURN_IF_B(require_ptr(xyz, fn, "buffer"));                                    \
      APO_RETURN_IF_B(require_len(b, sys, len, fn));                                      \
      b->object->method(sys, xyz);                                                        \
      return APO_STATUS_OK;                                                               \
    }, fn);                                                                               \
  }
APO_BATCH_XYZ_IN(apo_batch_set_coordinates, setCoordinates)
APO_BATCH_XYZ_IN(apo_batch_set_velocities, setVelocities)

#define APO_BATCH_XYZ_OUT(fname, method)                                                  \
  extern "C" apo_status fname(double *xyz, const size_t len, apo_batch *b, const int sys) { \
    const char *fn = #fname;                                                              \
    return guard([&]() -> apo_status {                                                    \
      APO_RETURN_IF_B(require_batch(b, fn, true));                                        \
      APO_RETURN_IF_B(require_ptr(xyz, fn, "buffer"));                                    \
      APO_RETURN_IF_B(require_len(b, sys, len, fn));                                      \
      b->object->method(sys, xyz);                                                        \
      return APO_STATUS_OK;                                                               \
    }, fn);                                                                               \
  }
APO_BATCH_XYZ_OUT(apo_batch_get_coordinates, getCoordinates)
APO_BATCH_XYZ_OUT(apo_batch_get_velocities, getVelocities)
APO_BATCH_XYZ_OUT(apo_batch_get_forces, getForces)

extern "C" apo_status apo_batch_assign_velocities(apo_batch *b, const double t) {
  const char *fn = "apo_batch_assign_velocities";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(require_batch(b, fn, true));
    b->object->assignVelocities(t);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_batch_set_langevin(apo_batch *b, const double dt, const double fr,
                                             const double t, const unsigned long long seed) {
  const char *fn = "apo_batch_set_langevin";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(require_batch(b, fn, false));
    if (!(dt > 0.0)) return invalid(fn, "time step must be positive");
    b->object->setLangevin(dt, fr, t, seed);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_batch_propagate(apo_batch *b, const int steps) {
  const char *fn = "apo_batch_propagate";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(require_batch(b, fn, true));
    if (steps < 0) return invalid(fn, "negative step count");
    b->object->propagate(steps);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_batch_calculate_forces(apo_batch *b, const int e, const int v) {
  const char *fn = "apo_batch_calculate_forces";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(require_batch(b, fn, true));
    b->object->calculateForces(e != 0, v != 0);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_batch_get_energy_components(double *e, const size_t len, apo_batch *b,
                                                      const int sys) {
  const char *fn = "apo_batch_get_energy_components";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(require_batch(b, fn, true));
    APO_RETURN_IF_B(require_buffer(e, len, (size_t)apo::kNumEnergyTerms, fn, "energy buffer"));
    if (sys < 0 || sys >= b->object->numSystems()) return invalid(fn, "system index out of range");
    auto m = b->object->energyComponents(sys);
    for (int k = 0; k < apo::kNumEnergyTerms; ++k) e[k] = m[apo::kEnergyNames[k]];
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_batch_get_temperatures(double *t, const size_t len, apo_batch *b) {
  const char *fn = "apo_batch_get_temperatures";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(require_batch(b, fn, true));
    APO_RETURN_IF_B(require_buffer(t, len, (size_t)b->object->numSystems(), fn, "buffer"));
    auto v = b->object->temperatures();
    std::copy(v.begin(), v.end(), t);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_batch_autotune(int *tpw, apo_batch *b, const int steps,
                                         const int *cand, const int ncand) {
  const char *fn = "apo_batch_autotune";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(require_batch(b, fn, true));
    std::vector<int> c;
    if (cand && ncand > 0) c.assign(cand, cand + ncand);
    else c = {2, 4, 6, 8, 12, 16};
    const int best = b->object->autotune(steps, c);
    if (tpw) *tpw = best;
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_batch_get_stream(void **stream, const apo_batch *b) {
  const char *fn = "apo_batch_get_stream";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(require_ptr(stream, fn, "stream"));
    APO_RETURN_IF_B(require_batch(b, fn, true));
    *stream = (void *)b->object->context()->stream();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_batch_set_component_mask(apo_batch *b, const int mask) {
  const char *fn = "apo_batch_set_component_mask";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(require_batch(b, fn, true));
    if (mask < 0 || mask > 7) return invalid(fn, "mask must be in [0, 7]");
    b->object->forceManager()->setComponentMask(mask);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_batch_get_direct_kernel(int *form, const apo_batch *b) {
  const char *fn = "apo_batch_get_direct_kernel";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_B(require_ptr(form, fn, "form"));
    APO_RETURN_IF_B(require_batch(b, fn, false));
    *form = b->object->directKernel();
    return APO_STATUS_OK;
  }, fn);
}
