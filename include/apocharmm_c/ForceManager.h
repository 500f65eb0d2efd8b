/* Force manager handle (reference: capi/include/apocharmm_c/ForceManager.h:24-31).
 *
 * Additions (no C entry point in the reference capi; each exposes the C++
 * ForceManager setter cited): the nonbonded/PME settings that the reference
 * only offers in C++ (include/ForceManager.h:200-225), and the precision form
 * (per-pair 64-bit fixed-point force accumulation + FP64 influence function). */
#ifndef APOCHARMM_C_FORCE_MANAGER_H
#define APOCHARMM_C_FORCE_MANAGER_H
#include "apocharmm_c/CharmmParameters.h"
#include "apocharmm_c/CharmmPsf.h"
#include "apocharmm_c/Export.h"
#include "apocharmm_c/Status.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct apo_force_manager apo_force_manager;
APOCHARMM_C_API apo_status apo_force_manager_create(apo_force_manager **out, const apo_charmm_psf *psf, const apo_charmm_parameters *parameters); /* :24 */
APOCHARMM_C_API void apo_force_manager_destroy(apo_force_manager *force_manager); /* :28 */
APOCHARMM_C_API apo_status apo_force_manager_set_box_dimensions(apo_force_manager *force_manager, const double x, const double y, const double z); /* :31 */
/* the box in force (3 edges, A): changes every step under the Langevin piston */
APOCHARMM_C_API apo_status apo_force_manager_get_box_dimensions(double *box, const size_t len, const apo_force_manager *force_manager);
/* additions: ForceManager::setKappa/setCutoff/setCtonnb/setCtofnb/setFFTGrid/setPmeSplineOrder */
APOCHARMM_C_API apo_status apo_force_manager_set_kappa(apo_force_manager *force_manager, const double kappa);
APOCHARMM_C_API apo_status apo_force_manager_set_cutoff(apo_force_manager *force_manager, const double cutnb);
APOCHARMM_C_API apo_status apo_force_manager_set_ctonnb(apo_force_manager *force_manager, const double ctonnb);
APOCHARMM_C_API apo_status apo_force_manager_set_ctofnb(apo_force_manager *force_manager, const double ctofnb);
APOCHARMM_C_API apo_status apo_force_manager_set_fft_grid(apo_force_manager *force_manager, const int nx, const int ny, const int nz);
APOCHARMM_C_API apo_status apo_force_manager_set_spline_order(apo_force_manager *force_manager, const int order);
/* additions: precision form on/off; tiles per nonbonded work item (tuning);
 * evaluated parts as a bit mask (1 bonded+1-4, 2 direct, 4 reciprocal; + 8
 * moves the 1-4 pairs and exclusion corrections to the direct part) */
APOCHARMM_C_API apo_status apo_force_manager_set_precision_mode(apo_force_manager *force_manager, const int precise);
APOCHARMM_C_API apo_status apo_force_manager_set_tiles_per_work(apo_force_manager *force_manager, const int tiles);
/* addition: work items one warp of the direct-space kernel takes before it
 * retires (0 = persistent grid, the default) */
APOCHARMM_C_API apo_status apo_force_manager_set_work_items_per_warp(apo_force_manager *force_manager, const int items);
APOCHARMM_C_API apo_status apo_force_manager_set_component_mask(apo_force_manager *force_manager, const int mask);
APOCHARMM_C_API apo_status apo_force_manager_get_fft_grid(int *nxyz3, const apo_force_manager *force_manager);
/* addition: direct-space kernel form, 0 = one j-list per tile for the whole
 * i-cluster (default), 1 = one queue per 8-atom i-group across tiles */
APOCHARMM_C_API apo_status apo_force_manager_set_direct_kernel(apo_force_manager *force_manager, const int form);
/* addition: tile capacity of the neighbour list (the work-item capacity
 * follows); needs an initialised manager.  The list is rebuilt before its
 * next use; a list that outgrows the capacity is grown (during propagate,
 * the segment whose build overflowed is run again from the unchanged state,
 * so the trajectory is the same).  Capacity of the last build: get_list_capacity. */
APOCHARMM_C_API apo_status apo_force_manager_set_list_capacity(apo_force_manager *force_manager, const int tiles);
APOCHARMM_C_API apo_status apo_force_manager_get_list_capacity(int *tiles, const apo_force_manager *force_manager);
/* addition: 1 (default) moves the reciprocal-space z-pencil slabs between the
 * complex grid and shared memory with tiled tensor copies (TMA), 0 with plain
 * loads and stores; the results are the same. */
APOCHARMM_C_API apo_status apo_force_manager_set_pme_tensor_copies(apo_force_manager *force_manager, const int on);
/* 1 when an initialised manager moves its pencil slabs by tensor copies */
APOCHARMM_C_API apo_status apo_force_manager_get_pme_tensor_copies(int *on, const apo_force_manager *force_manager);
#ifdef __cplusplus
}
#endif
#endif
