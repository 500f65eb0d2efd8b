// Handle definitions and argument checks shared by the C ABI files.
#pragma once

#include <cmath>
#include <memory>
#include <new>
#include <string>

#include "apocharmm_c/CharmmContext.h"
#include "apocharmm_c/CharmmCrd.h"
#include "apocharmm_c/CharmmParameters.h"
#include "apocharmm_c/CharmmPsf.h"
#include "apocharmm_c/Error.h"
#include "apocharmm_c/ForceManager.h"
#include "apocharmm_c/Status.h"
#include "common.h"
#include "engine.h"

struct apo_charmm_psf { std::shared_ptr<apo::CharmmPSF> object; };
struct apo_charmm_crd { std::shared_ptr<apo::CharmmCrd> object; };
struct apo_charmm_parameters { std::shared_ptr<apo::CharmmParameters> object; };
struct apo_force_manager { std::shared_ptr<apo::ForceManager> object; };
struct apo_charmm_context {
  std::shared_ptr<apo::ForceManager> force_manager;  // keeps the manager alive
  std::shared_ptr<apo::CharmmContext> object;
};

namespace apocapi {

void clear_error() noexcept;
apo_status set_error(apo_status s, const std::string &m) noexcept;

inline apo_status invalid(const char *fn, const std::string &m) {
  return set_error(APO_STATUS_INVALID_ARGUMENT, std::string(fn) + ": " + m);
}

template <typename F>
apo_status guard(F &&f, const char *fn) noexcept {
  clear_error();
  try {
    return f();
  } catch (const apo::CudaError &e) {
    return set_error(APO_STATUS_CUDA_ERROR, std::string(fn) + ": " + e.what());
  } catch (const std::exception &e) {
    return set_error(APO_STATUS_RUNTIME_ERROR, e.what());
  } catch (...) {
    return set_error(APO_STATUS_RUNTIME_ERROR, std::string(fn) + ": Unknown C++ exception");
  }
}

template <typename T>
apo_status prepare_out(T **out, const char *fn) {
  if (out == nullptr) return invalid(fn, "out pointer is NULL");
  *out = nullptr;
  return APO_STATUS_OK;
}
inline apo_status require_string(const char *s, const char *fn, const char *arg) {
  if (s != nullptr && s[0] != '\0') return APO_STATUS_OK;
  return invalid(fn, std::string(arg) + " is NULL or empty");
}
template <typename T>
apo_status require_ptr(const T *p, const char *fn, const char *arg) {
  if (p != nullptr) return APO_STATUS_OK;
  return invalid(fn, std::string(arg) + " is NULL");
}
template <typename H>
apo_status require_handle(const H *h, const char *fn, const char *what) {
  if (h == nullptr) return invalid(fn, std::string(what) + " handle is NULL");
  if (!h->object) return set_error(APO_STATUS_NOT_INITIALIZED, std::string(fn) + ": " + what + " is not initialized");
  return APO_STATUS_OK;
}
template <typename T>
apo_status require_buffer(const T *buf, size_t len, size_t need, const char *fn, const char *what) {
  if (buf == nullptr) return invalid(fn, std::string(what) + " is NULL");
  if (len < need)
    return invalid(fn, std::string(what) + " too small (" + std::to_string(len) + " < " +
                           std::to_string(need) + ")");
  return APO_STATUS_OK;
}

}  // namespace apocapi

#define APO_RETURN_IF(expr)                   \
  do {                                        \
    apo_status _st = (expr);                  \
    if (_st != APO_STATUS_OK) return _st;     \
  } while (0)
