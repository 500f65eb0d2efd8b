/* Integrator base view (reference: capi/include/apocharmm_c/CudaIntegrator.h:24-36).
 * Handles of concrete integrators hand out a borrowed base view through
 * apo_cuda_*_integrator_as_cuda_integrator, valid while the owner lives. */
#ifndef APOCHARMM_C_CUDA_INTEGRATOR_H
#define APOCHARMM_C_CUDA_INTEGRATOR_H
#include "apocharmm_c/CharmmContext.h"
#include "apocharmm_c/Export.h"
#include "apocharmm_c/Status.h"
#include "apocharmm_c/Subscriber.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct apo_cuda_integrator apo_cuda_integrator;
APOCHARMM_C_API apo_status apo_cuda_integrator_set_time_step(apo_cuda_integrator *integrator, const double time_step); /* :24 */
APOCHARMM_C_API apo_status apo_cuda_integrator_set_charmm_context(apo_cuda_integrator *integrator, apo_charmm_context *context); /* :27 */
APOCHARMM_C_API apo_status apo_cuda_integrator_subscribe(apo_cuda_integrator *integrator, apo_subscriber *subscriber); /* :30 */
/* addition: CudaIntegrator::unsubscribe (include/CudaIntegrator.h:139, C++ only in the
 * reference); *removed = 1 when the subscriber was subscribed */
APOCHARMM_C_API apo_status apo_cuda_integrator_unsubscribe(int *removed, apo_cuda_integrator *integrator, apo_subscriber *subscriber);
APOCHARMM_C_API apo_status apo_cuda_integrator_propagate(apo_cuda_integrator *integrator, const int num_steps); /* :33 */
APOCHARMM_C_API apo_status apo_cuda_integrator_initialize_from_restart_file(apo_cuda_integrator *integrator, const char *path); /* :36 */
/* additions: list-update cadence (CudaIntegrator::setNonbondedListUpdateFrequency,
 * src/CudaIntegrator.cu:231), graph capture on/off, step counter, temperatures */
APOCHARMM_C_API apo_status apo_cuda_integrator_set_nonbonded_list_update_frequency(apo_cuda_integrator *integrator, const int frequency);
APOCHARMM_C_API apo_status apo_cuda_integrator_set_use_graphs(apo_cuda_integrator *integrator, const int use_graphs);
APOCHARMM_C_API apo_status apo_cuda_integrator_get_current_step(long long *step, const apo_cuda_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_integrator_get_average_temperature(double *temperature, const apo_cuda_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_integrator_get_instantaneous_temperature(double *temperature, const apo_cuda_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_integrator_get_kernels_per_step(int *kernels, const apo_cuda_integrator *integrator);
#ifdef __cplusplus
}
#endif
#endif
