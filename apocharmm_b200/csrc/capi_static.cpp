// C ABI of the allocation-free reciprocal-space entry point
// (include/apocharmm_c/PmeReciprocalStatic.h).
#include "apocharmm_c/PmeReciprocalStatic.h"

#include <stdexcept>

#include "capi_internal.h"
#include "pme.h"

using namespace apocapi;

extern "C" apo_status apo_pme_reciprocal_static(const void *xyzq, const int num_atoms,
                                                const double box_x, const double box_y,
                                                const double box_z, const int nfft_x,
                                                const int nfft_y, const int nfft_z,
                                                const int spline_order, const double kappa,
                                                long long *gradient, const int stride,
                                                double *energy, const int fp64_influence,
                                                void *stream) {
  return guard([&]() -> apo_status {
    try {
      apo::pme_reciprocal_static(static_cast<const float4 *>(xyzq), num_atoms, box_x, box_y,
                                 box_z, nfft_x, nfft_y, nfft_z, spline_order, kappa, gradient,
                                 stride, energy, fp64_influence != 0, static_cast<cudaStream_t>(stream));
    } catch (const std::invalid_argument &e) {
      return set_error(APO_STATUS_INVALID_ARGUMENT, e.what());
    }
    return APO_STATUS_OK;
  }, "apo_pme_reciprocal_static");
}
