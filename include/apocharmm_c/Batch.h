/* Batch of independent systems advanced together (addition: the reference
 * capi has no batch API; each system follows the reference's per-system
 * physics, ForceManager/CharmmContext/CudaLangevinThermostatIntegrator).
 *
 * Every stage of a step is one launch for all systems and a list-update
 * segment is one CUDA graph.  Systems keep their own box, cutoffs, PME grid,
 * LJ tables, velocity seed and noise stream: a system's trajectory is the
 * same alone and in any batch.  Coordinates, velocities and forces of one
 * system are N x 3 doubles of that system's atoms (system < 0: all systems'
 * atoms, concatenated in system order); energies are the 10
 * terms in the order of apo_charmm_context_get_energy_components. */
#ifndef APOCHARMM_C_BATCH_H
#define APOCHARMM_C_BATCH_H
#include <stddef.h>
#include "apocharmm_c/CharmmParameters.h"
#include "apocharmm_c/CharmmPsf.h"
#include "apocharmm_c/Export.h"
#include "apocharmm_c/Status.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct apo_batch apo_batch;
APOCHARMM_C_API apo_status apo_batch_create(apo_batch **out, const int spline_order, const int tiles_per_work, const int precise);
APOCHARMM_C_API void apo_batch_destroy(apo_batch *batch);
/* nfft <= 0: 2 floor(L/2) per axis; *index receives the system's index (may be NULL) */
APOCHARMM_C_API apo_status apo_batch_add_system(apo_batch *batch, const apo_charmm_psf *psf, const apo_charmm_parameters *parameters, const double box_x, const double box_y, const double box_z, const double kappa, const double cutnb, const double ctonnb, const double ctofnb, const int nfft_x, const int nfft_y, const int nfft_z, const unsigned long long seed, int *index);
APOCHARMM_C_API apo_status apo_batch_initialize(apo_batch *batch);
APOCHARMM_C_API apo_status apo_batch_get_num_systems(int *num_systems, const apo_batch *batch);
/* system < 0: all systems */
APOCHARMM_C_API apo_status apo_batch_get_num_atoms(size_t *num_atoms, const apo_batch *batch, const int system);
APOCHARMM_C_API apo_status apo_batch_set_coordinates(apo_batch *batch, const int system, const double *xyz, const size_t len);
APOCHARMM_C_API apo_status apo_batch_get_coordinates(double *xyz, const size_t len, apo_batch *batch, const int system);
APOCHARMM_C_API apo_status apo_batch_set_velocities(apo_batch *batch, const int system, const double *v, const size_t len);
APOCHARMM_C_API apo_status apo_batch_get_velocities(double *v, const size_t len, apo_batch *batch, const int system);
APOCHARMM_C_API apo_status apo_batch_assign_velocities(apo_batch *batch, const double temperature);
APOCHARMM_C_API apo_status apo_batch_set_langevin(apo_batch *batch, const double time_step_ps, const double friction_per_ps, const double temperature, const unsigned long long seed);
APOCHARMM_C_API apo_status apo_batch_propagate(apo_batch *batch, const int steps);
APOCHARMM_C_API apo_status apo_batch_calculate_forces(apo_batch *batch, const int calc_energy, const int calc_virial);
APOCHARMM_C_API apo_status apo_batch_get_forces(double *xyz, const size_t len, apo_batch *batch, const int system);
APOCHARMM_C_API apo_status apo_batch_get_energy_components(double *energies, const size_t len, apo_batch *batch, const int system);
/* instantaneous temperature of every system from its on-step velocities */
APOCHARMM_C_API apo_status apo_batch_get_temperatures(double *temperatures, const size_t len, apo_batch *batch);
/* measured sweep over both direct-space kernel forms and the candidate tiles
 * per work item (NULL: 2 4 6 8 12 16); keeps the fastest pair and returns
 * its tiles per work item; the batch state is restored */
APOCHARMM_C_API apo_status apo_batch_autotune(int *tiles_per_work, apo_batch *batch, const int steps, const int *candidates, const int num_candidates);
/* the direct-space kernel form in use (0 tile batches, 1 grouped queues) */
APOCHARMM_C_API apo_status apo_batch_get_direct_kernel(int *form, const apo_batch *batch);
APOCHARMM_C_API apo_status apo_batch_get_stream(void **stream, const apo_batch *batch);
/* evaluated parts as a bit mask (1 bonded+1-4, 2 direct, 4 reciprocal), as
 * apo_force_manager_set_component_mask */
APOCHARMM_C_API apo_status apo_batch_set_component_mask(apo_batch *batch, const int mask);
#ifdef __cplusplus
}
#endif
#endif
