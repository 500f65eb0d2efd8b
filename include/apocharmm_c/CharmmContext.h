/* Simulation context handle (reference: capi/include/apocharmm_c/CharmmContext.h:30-48).
 *
 * Additions (the reference capi has no getters for these; each exposes the C++
 * CharmmContext/ForceManager call cited):
 *   calculate_forces      CharmmContext::calculateForces (src/CharmmContext.cu:416)
 *   get_forces            ForceManager::getForces (include/ForceManager.h) -- the
 *                         total GRADIENT dU/dx, N x 3 doubles, atom order
 *   get_energy_components ForceManager::getEnergyComponents (src/ForceManager.cu:278),
 *                         10 doubles in the order bond angle ureyb dihe imdihe
 *                         ewks ewse ewex elec vdw
 *   get/set coordinates, get/set velocities (N x 3 doubles)
 *   get_neighbor_pairs    the active (not masked) atom pairs of the tile list
 *                         within `radius`, as (i, j, image code) triples, for
 *                         pair-set parity checks */
#ifndef APOCHARMM_C_CHARMM_CONTEXT_H
#define APOCHARMM_C_CHARMM_CONTEXT_H
#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif
#include "apocharmm_c/CharmmCrd.h"
#include "apocharmm_c/Export.h"
#include "apocharmm_c/ForceManager.h"
#include "apocharmm_c/Status.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct apo_charmm_context apo_charmm_context;
APOCHARMM_C_API apo_status apo_charmm_context_create(apo_charmm_context **out, const apo_force_manager *force_manager); /* :30 */
APOCHARMM_C_API void apo_charmm_context_destroy(apo_charmm_context *context); /* :33 */
APOCHARMM_C_API apo_status apo_charmm_context_set_coordinates(apo_charmm_context *context, const apo_charmm_crd *crd); /* :35 */
APOCHARMM_C_API apo_status apo_charmm_context_set_random_seed_for_velocities(apo_charmm_context *context, const uint64_t seed); /* :38 */
APOCHARMM_C_API apo_status apo_charmm_context_use_holonomic_constraints(apo_charmm_context *context, const bool useHolonomicConstraints); /* :41 */
APOCHARMM_C_API apo_status apo_charmm_context_assign_velocities_at_temperature(apo_charmm_context *context, const double temperature); /* :45 */
APOCHARMM_C_API apo_status apo_charmm_context_compute_temperature(double *temperature, apo_charmm_context *context); /* :48 */
/* additions */
APOCHARMM_C_API apo_status apo_charmm_context_calculate_forces(apo_charmm_context *context, const bool reset_list, const bool calc_energy, const bool calc_virial);
APOCHARMM_C_API apo_status apo_charmm_context_get_forces(double *xyz, const size_t len, apo_charmm_context *context);
APOCHARMM_C_API apo_status apo_charmm_context_get_energy_components(double *energies, const size_t len, apo_charmm_context *context);
/* addition: ForceManager::getVirial (src/ForceManager.cu:393-415) -- the 3x3
 * internal virial (row major, kcal/mol) of the last calculate_forces made
 * with calc_virial (or of calculate_potential_energy); len >= 9 */
APOCHARMM_C_API apo_status apo_charmm_context_get_virial(double *virial, const size_t len, apo_charmm_context *context);
APOCHARMM_C_API apo_status apo_charmm_context_get_potential_energy(double *energy, apo_charmm_context *context);
/* N x 3 doubles; the neighbour list is rebuilt before the next force
 * evaluation, list query or MD segment (an MD segment starts with one) */
APOCHARMM_C_API apo_status apo_charmm_context_set_coordinates_xyz(apo_charmm_context *context, const double *xyz, const size_t len);
APOCHARMM_C_API apo_status apo_charmm_context_get_coordinates(double *xyz, const size_t len, apo_charmm_context *context);
APOCHARMM_C_API apo_status apo_charmm_context_set_velocities(apo_charmm_context *context, const double *v, const size_t len);
APOCHARMM_C_API apo_status apo_charmm_context_get_velocities(double *v, const size_t len, apo_charmm_context *context);
APOCHARMM_C_API apo_status apo_charmm_context_get_num_atoms(size_t *num_atoms, const apo_charmm_context *context);
APOCHARMM_C_API apo_status apo_charmm_context_get_degrees_of_freedom(int *ndegf, const apo_charmm_context *context);
APOCHARMM_C_API apo_status apo_charmm_context_reset_neighbor_list(apo_charmm_context *context);
APOCHARMM_C_API apo_status apo_charmm_context_get_neighbor_pairs(int *pairs, const size_t len, size_t *num_pairs, const double radius, apo_charmm_context *context);
/* addition: every atom pair the tile list holds (the ForceManager's cluster
 * pairs; the reference's list is ientry/tile_indj/tile_excl,
 * src/CudaNeighborListBuild.cu:727,902-912) whose distance, in FP64 from the
 * sorted coordinates and the tile's image shift, is below `radius`, masked
 * or not, as (global i, global j, excluded) triples: excluded = 1 when the
 * tile's exclusion mask drops the pair.  Each unordered pair appears once.
 * With pairs == NULL only *num_pairs is set; len counts ints. */
APOCHARMM_C_API apo_status apo_charmm_context_get_list_pairs(int *pairs, const size_t len, size_t *num_pairs, const double radius, apo_charmm_context *context);
/* CUDA-event timing of the direct-space kernel: enable (clears the
 * integrators' captured graphs on their next propagate is NOT done; enable it
 * before creating the integrator), then read the summed milliseconds and the
 * number of launches recorded since the last integration segment began */
APOCHARMM_C_API apo_status apo_charmm_context_set_kernel_timing(apo_charmm_context *context, const int on);
APOCHARMM_C_API apo_status apo_charmm_context_get_kernel_time(double *ms, int *launches, apo_charmm_context *context);
/* sizes of the current neighbour list: sorted slots, tiles, work items */
APOCHARMM_C_API apo_status apo_charmm_context_get_list_counts(int *slots, int *tiles, int *work_items, apo_charmm_context *context);
/* CUDA stream the context's work is issued on (a cudaStream_t), for timing */
APOCHARMM_C_API apo_status apo_charmm_context_get_stream(void **stream, const apo_charmm_context *context);
#ifdef __cplusplus
}
#endif
#endif
