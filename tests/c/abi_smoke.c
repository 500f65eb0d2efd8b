/* A plain C caller of the C ABI (no device work): every handle type the
 * drop-in declares is created, used for a host-side call and destroyed,
 * and a refused call reports its status and message. */
#include <stdio.h>
#include <string.h>

#include "apocharmm_c/CharmmParameters.h"
#include "apocharmm_c/CharmmPsf.h"
#include "apocharmm_c/CudaLangevinPistonIntegrator.h"
#include "apocharmm_c/CudaLangevinThermostatIntegrator.h"
#include "apocharmm_c/CudaNoseHooverIntegrator.h"
#include "apocharmm_c/DcdSubscriber.h"
#include "apocharmm_c/Error.h"
#include "apocharmm_c/ForceManager.h"

#define CHECK(call)                                                   \
  do {                                                                \
    apo_status st_ = (call);                                          \
    if (st_ != APO_STATUS_OK) {                                       \
      fprintf(stderr, "%s -> %d: %s\n", #call, st_, apo_last_error()); \
      return 1;                                                       \
    }                                                                 \
  } while (0)

int main(int argc, char **argv) {
  if (argc != 4) {
    fprintf(stderr, "usage: %s PSF PRM DCD\n", argv[0]);
    return 2;
  }
  apo_charmm_psf *psf = NULL;
  apo_charmm_parameters *prm = NULL;
  apo_force_manager *fm = NULL;
  CHECK(apo_charmm_psf_create(&psf, argv[1]));
  const char *files[1] = {argv[2]};
  CHECK(apo_charmm_parameters_create_from_files(&prm, files, 1));
  CHECK(apo_force_manager_create(&fm, psf, prm));
  CHECK(apo_force_manager_set_box_dimensions(fm, 20.0, 21.0, 22.0));
  double box[3] = {0, 0, 0};
  CHECK(apo_force_manager_get_box_dimensions(box, 3, fm));
  if (box[0] != 20.0 || box[1] != 21.0 || box[2] != 22.0) return 3;

  apo_cuda_langevin_piston_integrator *lp = NULL;
  apo_cuda_integrator *base = NULL;
  CHECK(apo_cuda_langevin_piston_integrator_create(&lp, 0.002));
  CHECK(apo_cuda_langevin_piston_integrator_as_cuda_integrator(&base, lp));
  if (apo_cuda_langevin_piston_integrator_set_crystal_type(lp, 7) != APO_STATUS_INVALID_ARGUMENT)
    return 4;
  if (strlen(apo_last_error()) == 0) return 5;
  CHECK(apo_cuda_langevin_piston_integrator_set_crystal_type(lp, APO_CRYSTAL_TETRAGONAL));
  int crystal = 0;
  CHECK(apo_cuda_langevin_piston_integrator_get_crystal_type(&crystal, lp));
  if (crystal != APO_CRYSTAL_TETRAGONAL) return 6;
  double mass[3];
  size_t n = 0;
  CHECK(apo_cuda_langevin_piston_integrator_get_langevin_piston_mass(mass, 3, &n, lp));
  if (n != 2) return 7;
  CHECK(apo_cuda_integrator_set_time_step(base, 0.001));

  apo_cuda_nose_hoover_integrator *nh = NULL;
  CHECK(apo_cuda_nose_hoover_integrator_create(&nh, 0.002));
  CHECK(apo_cuda_nose_hoover_integrator_set_reference_temperature(nh, 310.0));
  apo_cuda_langevin_thermostat_integrator *lt = NULL;
  CHECK(apo_cuda_langevin_thermostat_integrator_create(&lt, 0.002));
  CHECK(apo_cuda_langevin_thermostat_integrator_set_thermostat_friction(lt, 5.0));
  apo_dcd_subscriber *dcd = NULL;
  CHECK(apo_dcd_subscriber_create_with_report_frequency(&dcd, argv[3], 100));

  apo_dcd_subscriber_destroy(dcd);
  apo_cuda_langevin_thermostat_integrator_destroy(lt);
  apo_cuda_nose_hoover_integrator_destroy(nh);
  apo_cuda_langevin_piston_integrator_destroy(lp);
  apo_force_manager_destroy(fm);
  apo_charmm_parameters_destroy(prm);
  apo_charmm_psf_destroy(psf);
  printf("ok\n");
  return 0;
}
