/* CHARMM parameter set handle (reference: capi/include/apocharmm_c/CharmmParameters.h:24-31).
 * Reads .prm files and .str streams (the parameters after "read para"). */
#ifndef APOCHARMM_C_CHARMM_PARAMETERS_H
#define APOCHARMM_C_CHARMM_PARAMETERS_H
#include <stddef.h>
#include "apocharmm_c/Export.h"
#include "apocharmm_c/Status.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct apo_charmm_parameters apo_charmm_parameters;
APOCHARMM_C_API apo_status apo_charmm_parameters_create(apo_charmm_parameters **out, const char *path); /* :24 */
APOCHARMM_C_API apo_status apo_charmm_parameters_create_from_files(apo_charmm_parameters **out, const char *const *paths, const size_t num_paths); /* :27 */
APOCHARMM_C_API void apo_charmm_parameters_destroy(apo_charmm_parameters *parameters); /* :31 */
#ifdef __cplusplus
}
#endif
#endif
