// Status and CUDA error checks shared by the C++ classes in this directory.
//
// The classes are header-only: each owns handles of the C ABI
// (include/apocharmm_c/) and turns a failed call into the exception the
// reference throws for it, std::invalid_argument for bad input and
// std::runtime_error otherwise (the reference's cudaCheck aborts; here a
// CUDA error is a std::runtime_error too).
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "apocharmm_c/Error.h"
#include "apocharmm_c/Status.h"

namespace apocharmm_detail {

inline void check(apo_status s) {
  if (s == APO_STATUS_OK) return;
  const char *m = apo_last_error();
  const std::string msg = (m && *m) ? m : "apocharmm: a library call failed";
  if (s == APO_STATUS_INVALID_ARGUMENT) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

inline void cuda_check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace apocharmm_detail
