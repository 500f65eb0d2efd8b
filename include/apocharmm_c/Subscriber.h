/* Reporting subscriber base view (reference: capi/include/apocharmm_c/Subscriber.h:22-25). */
#ifndef APOCHARMM_C_SUBSCRIBER_H
#define APOCHARMM_C_SUBSCRIBER_H
#include "apocharmm_c/Export.h"
#include "apocharmm_c/Status.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct apo_subscriber apo_subscriber;
APOCHARMM_C_API apo_status apo_subscriber_set_report_frequency(apo_subscriber *subscriber, const int report_frequency); /* :22 */
APOCHARMM_C_API apo_status apo_subscriber_get_report_frequency(int *report_frequency, const apo_subscriber *subscriber); /* :25 */
#ifdef __cplusplus
}
#endif
#endif
