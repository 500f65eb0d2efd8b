/* Host-side access to restart files, no device needed.  The layout is the
 * reference writer's (src/RestartSubscriber.cu:39-445) and the fields are the
 * ones its readers take back (src/CudaLangevinThermostatIntegrator.cu:264-545,
 * src/CudaNoseHooverIntegrator.cu:337-615); the reference's C API has no such
 * functions: they let a host program inspect or prepare a restart file.
 * Real numbers carry 17 significant digits wherever the 22 columns allow, so
 * a file read back gives the same doubles. */
#ifndef APOCHARMM_C_RESTART_FILE_H
#define APOCHARMM_C_RESTART_FILE_H
#include "apocharmm_c/Export.h"
#include "apocharmm_c/Status.h"
#ifdef __cplusplus
extern "C" {
#endif
/* scalars of the file; box = the three cell edges; has_rng = 1 when the file
 * holds a Langevin RNG sequence position */
APOCHARMM_C_API apo_status apo_restart_file_read_header(const char *path, int *natom, long long *npriv,
                                                        int *ndegf, unsigned long long *seed,
                                                        unsigned long long *rngpos, int *has_rng,
                                                        double *box3, double *pnhv, double *pnhf);
/* the crystal tag of the header ("CUBI", "TETR", "ORTH"; 5 chars with the
 * terminating zero) and the Langevin piston displacement HDOT (3 values),
 * as src/CudaLangevinPistonIntegrator.cu:706-830 reads them */
APOCHARMM_C_API apo_status apo_restart_file_read_crystal(const char *path, char *crystal5, double *hdot3);
/* per-atom sections, natom x 3 each: XOLD (coordinates), VX (velocities),
 * X (position-Verlet delta); natom must match the file */
APOCHARMM_C_API apo_status apo_restart_file_read(const char *path, const int natom, double *xold,
                                                 double *vel, double *delta);
APOCHARMM_C_API apo_status apo_restart_file_write(const char *path, const int natom, const long long npriv,
                                                  const int ndegf, const unsigned long long seed,
                                                  const unsigned long long rngpos, const int has_rng,
                                                  const double *box3, const double pnhv, const double pnhf,
                                                  const double *xold, const double *vel,
                                                  const double *delta);
#ifdef __cplusplus
}
#endif
#endif
