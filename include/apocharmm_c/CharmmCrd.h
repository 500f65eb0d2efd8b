/* CHARMM CARD coordinates handle (reference: capi/include/apocharmm_c/CharmmCrd.h:24-32). */
#ifndef APOCHARMM_C_CHARMM_CRD_H
#define APOCHARMM_C_CHARMM_CRD_H
#include <stddef.h>
#include "apocharmm_c/Export.h"
#include "apocharmm_c/Status.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct apo_charmm_crd apo_charmm_crd;
APOCHARMM_C_API apo_status apo_charmm_crd_create(apo_charmm_crd **out, const char *path);  /* :24 */
APOCHARMM_C_API void apo_charmm_crd_destroy(apo_charmm_crd *crd);                             /* :27 */
APOCHARMM_C_API apo_status apo_charmm_crd_get_num_atoms(size_t *num_atoms, const apo_charmm_crd *crd); /* :29 */
/* xyz: 3*N doubles, atom-major */
APOCHARMM_C_API apo_status apo_charmm_crd_get_coordinates(double *xyz, const size_t xyz_len, const apo_charmm_crd *crd); /* :32 */
#ifdef __cplusplus
}
#endif
#endif
