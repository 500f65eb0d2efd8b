/* Harmonic positional restraint and the force manager's plug-in point.
 *
 * The reference exposes these in C++ only: HarmonicRestraintForce
 * (include/HarmonicRestraintForce.h: constructor, setSelection,
 * setForceConstant(s), setReferenceCoordinates, setMasses) and
 * ForceManager::subscribe / unsubscribe (include/ForceManager.h:420-475).
 * E = sum_i k_i m_i |r_i - r0_i|^2 over the selected atoms (masses 1 unless
 * set), reported as the energy named by the subscription tag.  The selection
 * starts empty; atoms outside it get force constant 0.  The restraint handle
 * may be destroyed while subscribed: the manager keeps it alive. */
#ifndef APOCHARMM_C_HARMONIC_RESTRAINT_FORCE_H
#define APOCHARMM_C_HARMONIC_RESTRAINT_FORCE_H
#include <stddef.h>
#include "apocharmm_c/CharmmContext.h"
#include "apocharmm_c/Export.h"
#include "apocharmm_c/ForceManager.h"
#include "apocharmm_c/Status.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct apo_harmonic_restraint_force apo_harmonic_restraint_force;
APOCHARMM_C_API apo_status apo_harmonic_restraint_force_create(apo_harmonic_restraint_force **out, const int num_atoms);
APOCHARMM_C_API void apo_harmonic_restraint_force_destroy(apo_harmonic_restraint_force *force);
/* atoms: 0-based indices */
APOCHARMM_C_API apo_status apo_harmonic_restraint_force_set_selection(apo_harmonic_restraint_force *force, const int *atoms, const size_t count);
APOCHARMM_C_API apo_status apo_harmonic_restraint_force_set_force_constant(apo_harmonic_restraint_force *force, const double k);
APOCHARMM_C_API apo_status apo_harmonic_restraint_force_set_force_constants(apo_harmonic_restraint_force *force, const double *k, const size_t len);
/* xyz: 3 x num_atoms */
APOCHARMM_C_API apo_status apo_harmonic_restraint_force_set_reference_coordinates(apo_harmonic_restraint_force *force, const double *xyz, const size_t len);
APOCHARMM_C_API apo_status apo_harmonic_restraint_force_set_masses(apo_harmonic_restraint_force *force, const double *masses, const size_t len);
/* one system per manager; tags are unique and differ from the built-in term names */
APOCHARMM_C_API apo_status apo_force_manager_subscribe_harmonic_restraint(apo_force_manager *force_manager, apo_harmonic_restraint_force *force, const char *tag);
/* *removed = 1 when a plug-in of that tag was subscribed */
APOCHARMM_C_API apo_status apo_force_manager_unsubscribe(int *removed, apo_force_manager *force_manager, const char *tag);
/* any named energy of the last evaluation with energies: a built-in term
 * ("bond", ..., "vdw") or a plug-in tag */
APOCHARMM_C_API apo_status apo_charmm_context_get_energy_component(double *energy, apo_charmm_context *context, const char *name);
#ifdef __cplusplus
}
#endif
#endif
