/* Langevin piston (constant pressure) integrator: additive entry points over
 * the reference's C++ class include/CudaLangevinPistonIntegrator.h:18-60
 * (its C ABI has no piston).  Crystal types as enum CRYSTAL of
 * include/PBC.h:15: 1 cubic, 2 orthorhombic, 3 tetragonal.  Pressures in
 * atm, row-major 3x3 (XX XY XZ YX YY YZ ZX ZY ZZ). */
#ifndef APOCHARMM_C_CUDA_LANGEVIN_PISTON_INTEGRATOR_H
#define APOCHARMM_C_CUDA_LANGEVIN_PISTON_INTEGRATOR_H
#ifndef __cplusplus
#include <stdbool.h>
#endif
#include <stddef.h>
#include <stdint.h>
#include "apocharmm_c/CudaIntegrator.h"
#include "apocharmm_c/Export.h"
#include "apocharmm_c/Status.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct apo_cuda_langevin_piston_integrator apo_cuda_langevin_piston_integrator;
#define APO_CRYSTAL_CUBIC 1
#define APO_CRYSTAL_ORTHORHOMBIC 2
#define APO_CRYSTAL_TETRAGONAL 3
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_create(apo_cuda_langevin_piston_integrator **out, const double time_step); /* :20 */
APOCHARMM_C_API void apo_cuda_langevin_piston_integrator_destroy(apo_cuda_langevin_piston_integrator *integrator); /* :21 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_as_cuda_integrator(apo_cuda_integrator **out, apo_cuda_langevin_piston_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_set_crystal_type(apo_cuda_langevin_piston_integrator *integrator, const int crystal_type); /* :39 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_set_pressure(apo_cuda_langevin_piston_integrator *integrator, const double *pressure, const size_t len); /* :37 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_set_langevin_piston_mass(apo_cuda_langevin_piston_integrator *integrator, const double *mass, const size_t len); /* :40 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_set_langevin_piston_friction(apo_cuda_langevin_piston_integrator *integrator, const double friction); /* :43 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_set_langevin_piston_friction_seed(apo_cuda_langevin_piston_integrator *integrator, const uint64_t seed); /* :41 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_set_rng_sequence_pos(apo_cuda_langevin_piston_integrator *integrator, const unsigned long long pos); /* :42 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_set_reference_temperature(apo_cuda_langevin_piston_integrator *integrator, const double temperature); /* :25 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_use_nose_hoover_thermostat(apo_cuda_langevin_piston_integrator *integrator, const bool flag); /* :24 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_set_nose_hoover_piston_mass(apo_cuda_langevin_piston_integrator *integrator, const double mass); /* :26 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_use_old_temperature(apo_cuda_langevin_piston_integrator *integrator, const bool flag); /* :35 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_set_max_predictor_corrector_iterations(apo_cuda_langevin_piston_integrator *integrator, const int iterations); /* :33 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_set_constant_surface_tension(apo_cuda_langevin_piston_integrator *integrator, const bool flag, const double surface_tension); /* :38 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_reset_averages(apo_cuda_langevin_piston_integrator *integrator); /* :45 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_get_rng_sequence_pos(unsigned long long *pos, const apo_cuda_langevin_piston_integrator *integrator);
/* 9 values each; the average is over the steps since the last reset */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_get_instantaneous_pressure_tensor(double *pressure, const size_t len, apo_cuda_langevin_piston_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_get_average_pressure_tensor(double *pressure, const size_t len, apo_cuda_langevin_piston_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_get_instantaneous_pressure_scalar(double *pressure, apo_cuda_langevin_piston_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_get_average_pressure_scalar(double *pressure, apo_cuda_langevin_piston_integrator *integrator);
/* one value per piston degree of freedom (1 cubic, 2 tetragonal, 3 orthorhombic) */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_get_langevin_piston_mass(double *mass, const size_t len, size_t *num, const apo_cuda_langevin_piston_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_get_langevin_piston_on_step_position(double *position, const size_t len, size_t *num, apo_cuda_langevin_piston_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_get_langevin_piston_half_step_position(double *position, const size_t len, size_t *num, apo_cuda_langevin_piston_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_get_langevin_piston_on_step_velocity(double *velocity, const size_t len, size_t *num, apo_cuda_langevin_piston_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_get_langevin_piston_delta_position(double *delta, const size_t len, size_t *num, apo_cuda_langevin_piston_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_get_langevin_piston_delta_pressure(double *pressure, const size_t len, size_t *num, apo_cuda_langevin_piston_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_get_instantaneous_surface_tension(double *tension, apo_cuda_langevin_piston_integrator *integrator); /* :533 */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_get_crystal_type(int *crystal_type, const apo_cuda_langevin_piston_integrator *integrator); /* :58 */
/* the thermostat piston: velocity, velocity one step back, velocity change
 * ("force"), and that one step back (set/getNoseHooverPiston*, :27-31) */
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_get_nose_hoover_piston_state(double *state, const size_t len, apo_cuda_langevin_piston_integrator *integrator);
APOCHARMM_C_API apo_status apo_cuda_langevin_piston_integrator_set_nose_hoover_piston_state(apo_cuda_langevin_piston_integrator *integrator, const double velocity, const double velocity_previous, const double force, const double force_previous);
#ifdef __cplusplus
}
#endif
#endif
