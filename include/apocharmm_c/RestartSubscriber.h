/* Restart-file writer (reference: capi/include/apocharmm_c/RestartSubscriber.h:23-34).
 * Writes coordinates, velocities, the position-Verlet delta and the RNG
 * position needed to resume a run. */
#ifndef APOCHARMM_C_RESTART_SUBSCRIBER_H
#define APOCHARMM_C_RESTART_SUBSCRIBER_H
#include "apocharmm_c/Export.h"
#include "apocharmm_c/Status.h"
#include "apocharmm_c/Subscriber.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct apo_restart_subscriber apo_restart_subscriber;
APOCHARMM_C_API apo_status apo_restart_subscriber_create(apo_restart_subscriber **out, const char *path); /* :23 */
APOCHARMM_C_API apo_status apo_restart_subscriber_create_with_report_frequency(apo_restart_subscriber **out, const char *path, const int report_frequency); /* :26 */
APOCHARMM_C_API void apo_restart_subscriber_destroy(apo_restart_subscriber *subscriber); /* :29 */
APOCHARMM_C_API apo_status apo_restart_subscriber_as_subscriber(apo_subscriber **out, apo_restart_subscriber *subscriber); /* :34 */
#ifdef __cplusplus
}
#endif
#endif
