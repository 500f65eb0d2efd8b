// C ABI of the request server (include/apocharmm_c/Server.h).
#include "apocharmm_c/Server.h"

#include <stdexcept>

#include "capi_internal.h"
#include "server.h"

using namespace apocapi;

struct apo_server {
  std::unique_ptr<apo::Server> object;
};

#define APO_RETURN_IF_S(x)                \
  do {                                    \
    apo_status st_ = (x);                 \
    if (st_ != APO_STATUS_OK) return st_; \
  } while (0)

namespace {
apo_status require_server(const apo_server *s, const char *fn) {
  if (s == nullptr || !s->object) return invalid(fn, "server handle is NULL");
  return APO_STATUS_OK;
}
// the finished result of `id`, or an error status
apo_status finished(apo_server *s, int id, apo::ServeResult &r, const char *fn) {
  APO_RETURN_IF_S(require_server(s, fn));
  bool done = false;
  try {
    done = s->object->poll(id, &r);
  } catch (const std::invalid_argument &e) {
    return invalid(fn, e.what());
  }
  if (!done) return set_error(APO_STATUS_NOT_INITIALIZED, std::string(fn) + ": request still pending");
  if (r.status == 2) return set_error(APO_STATUS_RUNTIME_ERROR, std::string(fn) + ": " + r.error);
  return APO_STATUS_OK;
}
apo_status copy_out(const std::vector<double> &v, double *out, size_t len, const char *fn,
                    const char *what) {
  if (v.empty()) return invalid(fn, std::string("this request has no ") + what);
  APO_RETURN_IF_S(require_buffer(out, len, v.size(), fn, "buffer"));
  std::copy(v.begin(), v.end(), out);
  return APO_STATUS_OK;
}
}  // namespace

extern "C" apo_status apo_server_create(apo_server **out, const double fraction, const int order,
                                        const int precise, const double dt, const double friction,
                                        const double temperature, const unsigned long long seed) {
  const char *fn = "apo_server_create";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_S(prepare_out(out, fn));
    try {
      auto s = std::make_unique<apo::Server>(fraction, order, precise != 0, dt, friction,
                                             temperature, seed);
      *out = new apo_server{std::move(s)};
    } catch (const std::invalid_argument &e) {
      return set_error(APO_STATUS_INVALID_ARGUMENT, std::string(fn) + ": " + e.what());
    }
    return APO_STATUS_OK;
  }, fn);
}

extern "C" void apo_server_destroy(apo_server *s) { delete s; }

extern "C" apo_status apo_server_submit(int *id, apo_server *s, const int kind,
                                        const apo_charmm_psf *psf,
                                        const apo_charmm_parameters *prm, const double bx,
                                        const double by, const double bz, const double kappa,
                                        const double cutnb, const double ctonnb,
                                        const double ctofnb, const int nx, const int ny,
                                        const int nz, const unsigned long long seed,
                                        const double *xyz, const size_t len,
                                        const long long steps) {
  const char *fn = "apo_server_submit";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_S(require_ptr(id, fn, "id"));
    APO_RETURN_IF_S(require_server(s, fn));
    APO_RETURN_IF_S(require_handle(psf, fn, "CharmmPsf"));
    APO_RETURN_IF_S(require_handle(prm, fn, "CharmmParameters"));
    APO_RETURN_IF_S(require_ptr(xyz, fn, "xyz"));
    apo::ServeRequest r;
    r.kind = kind;
    r.spec.psf = psf->object;
    r.spec.prm = prm->object;
    r.spec.box = {bx, by, bz};
    r.spec.kappa = kappa;
    r.spec.cutnb = cutnb;
    r.spec.ctonnb = ctonnb;
    r.spec.ctofnb = ctofnb;
    r.spec.nfft = {nx, ny, nz};
    r.spec.seed = seed;
    r.xyz.assign(xyz, xyz + len);
    r.steps = steps;
    try {
      *id = s->object->submit(std::move(r));
    } catch (const std::invalid_argument &e) {
      return invalid(fn, e.what());
    }
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_server_poll(int *state, apo_server *s, const int id) {
  const char *fn = "apo_server_poll";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_S(require_ptr(state, fn, "state"));
    APO_RETURN_IF_S(require_server(s, fn));
    apo::ServeResult r;
    try {
      *state = s->object->poll(id, &r) ? r.status : 0;
    } catch (const std::invalid_argument &e) {
      return invalid(fn, e.what());
    }
    if (*state == 2) set_error(APO_STATUS_RUNTIME_ERROR, std::string(fn) + ": " + r.error);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_server_wait(int *state, apo_server *s, const int id,
                                      const double timeout_s) {
  const char *fn = "apo_server_wait";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_S(require_ptr(state, fn, "state"));
    APO_RETURN_IF_S(require_server(s, fn));
    apo::ServeResult r;
    try {
      *state = s->object->wait(id, timeout_s, &r) ? r.status : 0;
    } catch (const std::invalid_argument &e) {
      return invalid(fn, e.what());
    }
    if (*state == 2) set_error(APO_STATUS_RUNTIME_ERROR, std::string(fn) + ": " + r.error);
    return APO_STATUS_OK;
  }, fn);
}

#define APO_SERVER_VEC(fname, field, what)                                               \
  extern "C" apo_status fname(double *out, const size_t len, apo_server *s, const int id) { \
    const char *fn = #fname;                                                             \
    return guard([&]() -> apo_status {                                                   \
      apo::ServeResult r;                                                                \
      APO_RETURN_IF_S(finished(s, id, r, fn));                                           \
      return copy_out(r.field, out, len, fn, what);                                      \
    }, fn);                                                                              \
  }
APO_SERVER_VEC(apo_server_get_coordinates, xyz, "coordinates")
APO_SERVER_VEC(apo_server_get_velocities, vel, "velocities")
APO_SERVER_VEC(apo_server_get_forces, forces, "forces")

extern "C" apo_status apo_server_get_energy_components(double *e, const size_t len, apo_server *s,
                                                       const int id) {
  const char *fn = "apo_server_get_energy_components";
  return guard([&]() -> apo_status {
    apo::ServeResult r;
    APO_RETURN_IF_S(finished(s, id, r, fn));
    if (r.kind != 1) return invalid(fn, "this request has no energies (MD segment)");
    APO_RETURN_IF_S(require_buffer(e, len, (size_t)apo::kNumEnergyTerms, fn, "energy buffer"));
    for (int k = 0; k < apo::kNumEnergyTerms; ++k) e[k] = r.energy[k];
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_server_get_latency(double *seconds, apo_server *s, const int id) {
  const char *fn = "apo_server_get_latency";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_S(require_ptr(seconds, fn, "seconds"));
    apo::ServeResult r;
    APO_RETURN_IF_S(finished(s, id, r, fn));
    *seconds = r.latency_s;
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_server_release(apo_server *s, const int id) {
  const char *fn = "apo_server_release";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_S(require_server(s, fn));
    s->object->release(id);
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_server_get_stats(double *stats, const size_t len, apo_server *s) {
  const char *fn = "apo_server_get_stats";
  return guard([&]() -> apo_status {
    APO_RETURN_IF_S(require_server(s, fn));
    APO_RETURN_IF_S(require_buffer(stats, len, (size_t)6, fn, "stats buffer"));
    const apo::ServerStats st = s->object->stats();
    stats[0] = (double)st.md_steps;
    stats[1] = st.sim_ps;
    stats[2] = (double)st.rebuilds;
    stats[3] = (double)st.segments;
    stats[4] = (double)st.max_active;
    stats[5] = st.busy_s;
    if (len >= 8) {
      stats[6] = st.reform_s;
      stats[7] = (double)st.energy_evals;
    }
    return APO_STATUS_OK;
  }, fn);
}
