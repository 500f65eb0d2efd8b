/* Device-side force calls of the force manager and the ForceView plug-in
 * point, for callers that keep coordinates and forces in device memory
 * (the C++ classes in include/apocharmm/ sit on these).
 *
 * The reference has these in C++ only:
 *   initialize                ForceManager::initialize (include/ForceManager.h:397)
 *   calc_force                ForceManager::calcForce(xyzq, reset, calcEnergy,
 *                             calcVirial) (include/ForceManager.h:424,
 *                             src/ForceManager.cu:821)
 *   get_forces_device         ForceManager::getForces (include/ForceManager.h:313)
 *   get_force_fixed_device    ForceManager::get{Bonded,Reciprocal,Direct}Forcevalues
 *                             (include/ForceManager.h:305-307): the 2^40 fixed point
 *   get_energy_components     ForceManager::getEnergyComponents (:292)
 *   get_virial                ForceManager::getVirial (:351)
 *   subscribe_view            ForceManager::subscribe<ForceType> with its ForceView
 *                             type erasure (include/ForceManager.h:37-105, 429-442)
 *
 * Coordinates: `d_xyzq` is a device array of num_atoms x (x, y, z, charge)
 * floats in atom order.  Forces are GRADIENTS dU/dx (the reference's sign), in
 * x, y and z planes `stride` elements apart (stride >= num_atoms), atom order.
 * `stream` is a cudaStream_t (NULL: the legacy default stream); the device
 * getters are stream-ordered, calc_force returns after its work on `stream`
 * has finished.
 *
 * components: 1 bonded terms, 2 direct space, 4 reciprocal space (with the
 * self energy); the 1-4 pairs and the exclusion corrections go with the
 * bonded terms, or with the direct space when 8 is added (the reference's
 * split between CudaBondedForce and CudaPMEDirectForce).  7 = everything. */
#ifndef APOCHARMM_C_FORCE_VIEW_H
#define APOCHARMM_C_FORCE_VIEW_H
#include <stddef.h>
#include "apocharmm_c/Export.h"
#include "apocharmm_c/ForceManager.h"
#include "apocharmm_c/Status.h"
#ifdef __cplusplus
extern "C" {
#endif
APOCHARMM_C_API apo_status apo_force_manager_initialize(apo_force_manager *force_manager);
APOCHARMM_C_API apo_status apo_force_manager_get_num_atoms(int *num_atoms, const apo_force_manager *force_manager);
APOCHARMM_C_API apo_status apo_force_manager_calc_force(apo_force_manager *force_manager, const float *d_xyzq, const int num_atoms, const int reset, const int calc_energy, const int calc_virial, const int components, void *stream);
APOCHARMM_C_API apo_status apo_force_manager_get_forces_device(double *d_xyz, const int stride, apo_force_manager *force_manager, void *stream);
APOCHARMM_C_API apo_status apo_force_manager_get_force_fixed_device(long long *d_xyz, const int stride, apo_force_manager *force_manager, void *stream);
/* 10 doubles in the order bond angle ureyb dihe imdihe ewks ewse ewex elec vdw */
APOCHARMM_C_API apo_status apo_force_manager_get_energy_components(double *energies, const size_t len, apo_force_manager *force_manager, void *stream);
/* a built-in term name or a plug-in tag */
APOCHARMM_C_API apo_status apo_force_manager_get_energy_component(double *energy, apo_force_manager *force_manager, const char *name, void *stream);
/* row-major 3x3 of the last calc_force with calc_virial; len >= 9 */
APOCHARMM_C_API apo_status apo_force_manager_get_virial(double *virial, const size_t len, apo_force_manager *force_manager, void *stream);

/* The manager's tile list (the reference's CudaNeighborList<32>,
 * include/CudaNeighborList.h:32-170): sizes of the last build (sorted slots,
 * tiles, work items), every list pair within `radius` as (atom i, atom j,
 * excluded) triples (pairs == NULL: count only; len counts ints), and the
 * device arrays atom -> sorted slot and sorted slot -> atom (-1 = padding)
 * (get_glo2loc / get_ind_sorted, include/CudaNeighborList.h:140-142), valid
 * until the next build. */
APOCHARMM_C_API apo_status apo_force_manager_get_list_counts(int *slots, int *tiles, int *work_items, apo_force_manager *force_manager, void *stream);
APOCHARMM_C_API apo_status apo_force_manager_get_list_pairs(int *pairs, const size_t len, size_t *num_pairs, const double radius, apo_force_manager *force_manager, void *stream);
APOCHARMM_C_API apo_status apo_force_manager_get_list_arrays(const int **glo2loc, const int **ind_sorted, apo_force_manager *force_manager);

/* A force term the caller evaluates: at every force evaluation the manager
 * makes `stream` wait for its own work, calls clear (when set) and
 * calc_force with the atom-order device coordinates, makes its own stream
 * wait for `stream`, and adds the gradient get_force returns (device, atom
 * order, fixed point 2^40, planes `*stride` apart) and, when energies are
 * evaluated, the sum of the `*count` device doubles get_energies returns, as
 * the energy named by the tag.  initialize (when set) is called when the view
 * joins an initialised manager and when the manager is initialised.  The
 * functions must only enqueue stream-ordered work on `stream` (no host
 * synchronisation or allocation); `object` and the buffers must outlive the
 * subscription.  The view's virial is not added to the manager's. */
typedef struct apo_force_view {
  void *object;
  void (*initialize)(void *object, int num_atoms, const double *box3);
  void (*clear)(void *object);
  void (*calc_force)(void *object, const float *d_xyzq, int calc_energy, int calc_virial);
  const long long *(*get_force)(void *object, int *stride);
  const double *(*get_energies)(void *object, int *count);
  void *stream;
} apo_force_view;
/* one system per manager; tags are unique and differ from the built-in term
 * names; removed with apo_force_manager_unsubscribe */
APOCHARMM_C_API apo_status apo_force_manager_subscribe_view(apo_force_manager *force_manager, const apo_force_view *view, const char *tag);
#ifdef __cplusplus
}
#endif
#endif
