/* Request server with continuous batching (addition: the reference has no
 * serving layer; each request follows the reference's per-system
 * force/step path).
 *
 * A worker thread owns the GPU.  MD-segment requests (a system, its N x 3
 * coordinates, a step count, a seed) are admitted while their estimated
 * device memory fits the given share of the free HBM, advanced together 20
 * steps at a time, and re-batched as requests arrive and finish; a system's
 * coordinates, velocities and integrator state stay on the device between
 * segments and carry over exactly when the batch changes, so its result is
 * the same alone and among others.  Topologies are built on a second host
 * thread as requests arrive.  Energy/force requests join the running batch
 * and are answered by one force call of it.  A request that cannot join
 * (invalid coordinates, no device memory) fails alone with the error; the
 * server goes on.  Results are kept until released.
 * Langevin settings (time step, friction, temperature, noise seed) are the
 * server's; each system's velocities and noise stream come from its seed. */
#ifndef APOCHARMM_C_SERVER_H
#define APOCHARMM_C_SERVER_H
#include <stddef.h>
#include "apocharmm_c/CharmmParameters.h"
#include "apocharmm_c/CharmmPsf.h"
#include "apocharmm_c/Export.h"
#include "apocharmm_c/Status.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct apo_server apo_server;
APOCHARMM_C_API apo_status apo_server_create(apo_server **out, const double hbm_fraction, const int spline_order, const int precise, const double time_step_ps, const double friction_per_ps, const double temperature, const unsigned long long seed);
/* stops the worker (requests still running are abandoned) and frees everything */
APOCHARMM_C_API void apo_server_destroy(apo_server *server);
/* kind 0: MD segment of `steps` steps; kind 1: energies and forces (steps ignored) */
APOCHARMM_C_API apo_status apo_server_submit(int *id, apo_server *server, const int kind, const apo_charmm_psf *psf, const apo_charmm_parameters *parameters, const double box_x, const double box_y, const double box_z, const double kappa, const double cutnb, const double ctonnb, const double ctofnb, const int nfft_x, const int nfft_y, const int nfft_z, const unsigned long long seed, const double *xyz, const size_t len, const long long steps);
/* *state: 0 pending, 1 done, 2 failed (the message is in apo_last_error) */
APOCHARMM_C_API apo_status apo_server_poll(int *state, apo_server *server, const int id);
/* waits up to timeout_s seconds (< 0: without limit) */
APOCHARMM_C_API apo_status apo_server_wait(int *state, apo_server *server, const int id, const double timeout_s);
/* finished MD requests: final coordinates and velocities; energy requests:
 * the input coordinates, forces (gradient) and the 10 energy terms in the
 * order of apo_charmm_context_get_energy_components */
APOCHARMM_C_API apo_status apo_server_get_coordinates(double *xyz, const size_t len, apo_server *server, const int id);
APOCHARMM_C_API apo_status apo_server_get_velocities(double *v, const size_t len, apo_server *server, const int id);
APOCHARMM_C_API apo_status apo_server_get_forces(double *xyz, const size_t len, apo_server *server, const int id);
APOCHARMM_C_API apo_status apo_server_get_energy_components(double *energies, const size_t len, apo_server *server, const int id);
/* seconds from submission to the result */
APOCHARMM_C_API apo_status apo_server_get_latency(double *seconds, apo_server *server, const int id);
APOCHARMM_C_API apo_status apo_server_release(apo_server *server, const int id);
/* stats[0] system-steps advanced, [1] simulated ps over all requests,
 * [2] batch re-formations, [3] segments, [4] most systems in one batch,
 * [5] seconds the worker spent on device work; with len >= 8 also [6] of
 * which re-forming the batch, [7] force calls made for energy requests */
APOCHARMM_C_API apo_status apo_server_get_stats(double *stats, const size_t len, apo_server *server);
#ifdef __cplusplus
}
#endif
#endif
