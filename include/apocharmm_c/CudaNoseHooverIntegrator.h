/* Nose-Hoover integrator (reference: capi/include/apocharmm_c/CudaNoseHooverIntegrator.h:29-62). */
#ifndef APOCHARMM_C_CUDA_NOSE_HOOVER_INTEGRATOR_H
#define APOCHARMM_C_CUDA_NOSE_HOOVER_INTEGRATOR_H
#ifndef __cplusplus
#include <stdbool.h>
#endif
#include "apocharmm_c/CudaIntegrator.h"
#include "apocharmm_c/Export.h"
#include "apocharmm_c/Status.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct apo_cuda_nose_hoover_integrator apo_cuda_nose_hoover_integrator;
APOCHARMM_C_API apo_status apo_cuda_nose_hoover_integrator_create(apo_cuda_nose_hoover_integrator **out, const double time_step); /* :29 */
APOCHARMM_C_API void apo_cuda_nose_hoover_integrator_destroy(apo_cuda_nose_hoover_integrator *integrator); /* :32 */
APOCHARMM_C_API apo_status apo_cuda_nose_hoover_integrator_set_reference_temperature(apo_cuda_nose_hoover_integrator *integrator, const double temperature); /* :35 */
APOCHARMM_C_API apo_status apo_cuda_nose_hoover_integrator_set_nose_hoover_piston_mass(apo_cuda_nose_hoover_integrator *integrator, const double mass); /* :39 */
APOCHARMM_C_API apo_status apo_cuda_nose_hoover_integrator_use_old_temperature(apo_cuda_nose_hoover_integrator *integrator, const bool flag); /* :43 */
APOCHARMM_C_API apo_status apo_cuda_nose_hoover_integrator_reset_average_temperature(apo_cuda_nose_hoover_integrator *integrator); /* :46 */
APOCHARMM_C_API apo_status apo_cuda_nose_hoover_integrator_get_reference_temperature(double *temperature, const apo_cuda_nose_hoover_integrator *integrator); /* :50 */
APOCHARMM_C_API apo_status apo_cuda_nose_hoover_integrator_get_average_temperature(double *temperature, const apo_cuda_nose_hoover_integrator *integrator); /* :54 */
APOCHARMM_C_API apo_status apo_cuda_nose_hoover_integrator_get_instantaneous_temperature(double *temperature, const apo_cuda_nose_hoover_integrator *integrator); /* :58 */
APOCHARMM_C_API apo_status apo_cuda_nose_hoover_integrator_as_cuda_integrator(apo_cuda_integrator **out, apo_cuda_nose_hoover_integrator *integrator); /* :62 */
#ifdef __cplusplus
}
#endif
#endif
