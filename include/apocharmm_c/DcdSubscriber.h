/* DCD trajectory writer (reference: capi/include/apocharmm_c/DcdSubscriber.h:23-33).
 * The subscriber view returned by apo_dcd_subscriber_as_subscriber is borrowed:
 * valid while the DCD handle lives. */
#ifndef APOCHARMM_C_DCD_SUBSCRIBER_H
#define APOCHARMM_C_DCD_SUBSCRIBER_H
#include "apocharmm_c/Export.h"
#include "apocharmm_c/Status.h"
#include "apocharmm_c/Subscriber.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct apo_dcd_subscriber apo_dcd_subscriber;
APOCHARMM_C_API apo_status apo_dcd_subscriber_create(apo_dcd_subscriber **out, const char *path); /* :23 */
APOCHARMM_C_API apo_status apo_dcd_subscriber_create_with_report_frequency(apo_dcd_subscriber **out, const char *path, const int report_frequency); /* :26 */
APOCHARMM_C_API void apo_dcd_subscriber_destroy(apo_dcd_subscriber *subscriber); /* :29 */
APOCHARMM_C_API apo_status apo_dcd_subscriber_as_subscriber(apo_subscriber **out, apo_dcd_subscriber *subscriber); /* :33 */
#ifdef __cplusplus
}
#endif
#endif
