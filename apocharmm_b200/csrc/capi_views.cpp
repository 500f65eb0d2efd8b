// C ABI: device-side force calls and the ForceView plug-in point (same
// conventions as capi.cpp).
#include <cstdint>
#include <string>
#include <type_traits>

#include "apocharmm_c/ForceView.h"
#include "capi_internal.h"
#include "force_plugins.h"

using namespace apocapi;

namespace {

cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

apo_status require_initialized(const apo_force_manager *fm, const char *fn) {
  if (fm->object->isInitialized()) return APO_STATUS_OK;
  return set_error(APO_STATUS_NOT_INITIALIZED,
                   std::string(fn) + ": the force manager is not initialized");
}

apo_status require_single(const apo_force_manager *fm, const char *fn) {
  if (!fm->object->isMulti()) return APO_STATUS_OK;
  return invalid(fn, "needs a single-system force manager");
}

}  // namespace

extern "C" apo_status apo_force_manager_initialize(apo_force_manager *fm) {
  const char *fn = "apo_force_manager_initialize";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    try {
      fm->object->initialize();
    } catch (const std::invalid_argument &e) {
      return invalid(fn, e.what());
    }
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_force_manager_get_num_atoms(int *n, const apo_force_manager *fm) {
  const char *fn = "apo_force_manager_get_num_atoms";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(n, fn, "num_atoms"));
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    *n = fm->object->getNumAtoms();
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_force_manager_calc_force(apo_force_manager *fm, const float *d_xyzq,
                                                   const int num_atoms, const int reset,
                                                   const int calc_energy, const int calc_virial,
                                                   const int components, void *stream) {
  const char *fn = "apo_force_manager_calc_force";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    APO_RETURN_IF(require_single(fm, fn));
    APO_RETURN_IF(require_ptr(d_xyzq, fn, "xyzq"));
    if (num_atoms != fm->object->getNumAtoms())
      return invalid(fn, "num_atoms (" + std::to_string(num_atoms) + ") differs from the PSF (" +
                             std::to_string(fm->object->getNumAtoms()) + ")");
    if (components < 0 || components > 15)
      return invalid(fn, "components must be a mask of 1, 2, 4 and 8");
    if (reinterpret_cast<uintptr_t>(d_xyzq) % 16 != 0)
      return invalid(fn, "xyzq must be 16-byte aligned (float4 per atom)");
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, d_xyzq) != cudaSuccess ||
        (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)) {
      cudaGetLastError();
      return invalid(fn, "xyzq is not a device pointer");
    }
    const cudaStream_t s = as_stream(stream);
    try {
      fm->object->calcForceXyzq(reinterpret_cast<const float4 *>(d_xyzq), reset != 0,
                                calc_energy != 0, calc_virial != 0, components, s);
    } catch (const std::invalid_argument &e) {
      return invalid(fn, e.what());
    }
    APO_CUDA(cudaStreamSynchronize(s));
    return APO_STATUS_OK;
  }, fn);
}

namespace {

template <typename T>
apo_status device_forces(T *d_xyz, int stride, apo_force_manager *fm, void *stream,
                         const char *fn) {
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(d_xyz, fn, "force buffer"));
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    APO_RETURN_IF(require_single(fm, fn));
    APO_RETURN_IF(require_initialized(fm, fn));
    if (stride < fm->object->getNumAtoms())
      return invalid(fn, "stride (" + std::to_string(stride) + ") is below the atom count");
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, d_xyz) != cudaSuccess ||
        (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)) {
      cudaGetLastError();
      return invalid(fn, "force buffer is not a device pointer");
    }
    if constexpr (std::is_same<T, double>::value)
      fm->object->getForcesDevice(d_xyz, stride, as_stream(stream));
    else
      fm->object->getForceFixedDevice(d_xyz, stride, as_stream(stream));
    return APO_STATUS_OK;
  }, fn);
}

}  // namespace

extern "C" apo_status apo_force_manager_get_forces_device(double *d_xyz, const int stride,
                                                          apo_force_manager *fm, void *stream) {
  return device_forces(d_xyz, stride, fm, stream, "apo_force_manager_get_forces_device");
}

extern "C" apo_status apo_force_manager_get_force_fixed_device(long long *d_xyz, const int stride,
                                                               apo_force_manager *fm,
                                                               void *stream) {
  return device_forces(d_xyz, stride, fm, stream, "apo_force_manager_get_force_fixed_device");
}

extern "C" apo_status apo_force_manager_get_energy_components(double *e, const size_t len,
                                                              apo_force_manager *fm,
                                                              void *stream) {
  const char *fn = "apo_force_manager_get_energy_components";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    APO_RETURN_IF(require_buffer(e, len, (size_t)apo::kNumEnergyTerms, fn, "energy buffer"));
    APO_RETURN_IF(require_initialized(fm, fn));
    auto m = fm->object->getEnergyComponents(as_stream(stream));
    for (int k = 0; k < apo::kNumEnergyTerms; ++k) e[k] = m[apo::kEnergyNames[k]];
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_force_manager_get_energy_component(double *energy, apo_force_manager *fm,
                                                             const char *name, void *stream) {
  const char *fn = "apo_force_manager_get_energy_component";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_ptr(energy, fn, "energy"));
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    APO_RETURN_IF(require_string(name, fn, "name"));
    APO_RETURN_IF(require_initialized(fm, fn));
    auto m = fm->object->getEnergyComponents(as_stream(stream));
    auto it = m.find(name);
    if (it == m.end()) return invalid(fn, std::string("no energy named '") + name + "'");
    *energy = it->second;
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_force_manager_get_virial(double *v, const size_t len,
                                                   apo_force_manager *fm, void *stream) {
  const char *fn = "apo_force_manager_get_virial";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    APO_RETURN_IF(require_buffer(v, len, (size_t)9, fn, "virial buffer"));
    APO_RETURN_IF(require_initialized(fm, fn));
    auto w = fm->object->getVirial(as_stream(stream));
    for (int k = 0; k < 9; ++k) v[k] = w[k];
    return APO_STATUS_OK;
  }, fn);
}

extern "C" apo_status apo_force_manager_subscribe_view(apo_force_manager *fm,
                                                       const apo_force_view *view,
                                                       const char *tag) {
  const char *fn = "apo_force_manager_subscribe_view";
  return guard([&]() -> apo_status {
    APO_RETURN_IF(require_handle(fm, fn, "ForceManager"));
    APO_RETURN_IF(require_ptr(view, fn, "view"));
    APO_RETURN_IF(require_string(tag, fn, "tag"));
    if (!view->calc_force || !view->get_force)
      return invalid(fn, "view needs calc_force and get_force");
    if (!view->stream) return invalid(fn, "view needs a stream (a cudaStream_t other than NULL)");
    apo::ExternalForceOps ops;
    ops.object = view->object;
    ops.initialize = view->initialize;
    ops.clear = view->clear;
    ops.calc_force = view->calc_force;
    ops.get_force = view->get_force;
    ops.get_energies = view->get_energies;
    ops.stream = as_stream(view->stream);
    try {
      fm->object->subscribe(std::make_shared<apo::ExternalForce>(ops), tag);
    } catch (const std::invalid_argument &e) {
      return invalid(fn, e.what());
    }
    return APO_STATUS_OK;
  }, fn);
}
