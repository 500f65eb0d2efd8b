/* Langevin thermostat and leapfrog integrators.
 * Additions: the reference capi has no handle for these; each entry point
 * exposes the C++ method cited (src/CudaLangevinThermostatIntegrator.cu:18-110,
 * src/CudaLeapFrogIntegrator.cu). */
#ifndef APOCHARMM_C_CUDA_LANGEVIN_THERMOSTAT_INTEGRATOR_H
#define APOCHARMM_C_CUDA_LANGEVIN_THERMOSTAT_INTEGRATOR_H
#include <stdint.h>
#include "apocharmm_c/CudaIntegrator.h"
#include "apocharmm_c/Export.h"
#include "apocharmm_c/Status.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct apo_cuda_langevin_thermostat_integrator apo_cuda_langevin_thermostat_integrator;
APOCHARMM_C_API apo_status apo_cuda_langevin_thermostat_integrator_create(apo_cuda_langevin_thermostat_integrator **out, const double time_step);
APOCHARMM_C_API void apo_cuda_langevin_thermostat_integrator_destroy(apo_cuda_langevin_thermostat_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_langevin_thermostat_integrator_set_thermostat_friction(apo_cuda_langevin_thermostat_integrator *integrator, const double friction);
APOCHARMM_C_API apo_status apo_cuda_langevin_thermostat_integrator_set_reference_temperature(apo_cuda_langevin_thermostat_integrator *integrator, const double temperature);
APOCHARMM_C_API apo_status apo_cuda_langevin_thermostat_integrator_set_thermostat_rng_seed(apo_cuda_langevin_thermostat_integrator *integrator, const uint64_t seed);
APOCHARMM_C_API apo_status apo_cuda_langevin_thermostat_integrator_get_rng_sequence_pos(unsigned long long *pos, const apo_cuda_langevin_thermostat_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_langevin_thermostat_integrator_as_cuda_integrator(apo_cuda_integrator **out, apo_cuda_langevin_thermostat_integrator *integrator);
typedef struct apo_cuda_leap_frog_integrator apo_cuda_leap_frog_integrator;
APOCHARMM_C_API apo_status apo_cuda_leap_frog_integrator_create(apo_cuda_leap_frog_integrator **out, const double time_step);
APOCHARMM_C_API void apo_cuda_leap_frog_integrator_destroy(apo_cuda_leap_frog_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_leap_frog_integrator_as_cuda_integrator(apo_cuda_integrator **out, apo_cuda_leap_frog_integrator *integrator);
#ifdef __cplusplus
}
#endif
#endif
