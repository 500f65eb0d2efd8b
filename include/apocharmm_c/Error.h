/* Thread-local text of the last error (reference: capi/include/apocharmm_c/Error.h:19). */
#ifndef APOCHARMM_C_ERROR_H
#define APOCHARMM_C_ERROR_H
#include "apocharmm_c/Export.h"
#ifdef __cplusplus
extern "C" {
#endif
APOCHARMM_C_API const char *apo_last_error(void);
#ifdef __cplusplus
}
#endif
#endif
