/* Status codes returned by every C entry point.
 * Same values as the reference (capi/include/apocharmm_c/Status.h:17-24). */
#ifndef APOCHARMM_C_STATUS_H
#define APOCHARMM_C_STATUS_H
#ifdef __cplusplus
extern "C" {
#endif
typedef enum apo_status {
  APO_STATUS_OK = 0,
  APO_STATUS_INVALID_ARGUMENT = 1,
  APO_STATUS_RUNTIME_ERROR = 2,
  APO_STATUS_CUDA_ERROR = 3,
  APO_STATUS_NOT_INITIALIZED = 4,
  APO_STATUS_NOT_IMPLEMENTED = 5,
} apo_status;
#ifdef __cplusplus
}
#endif
#endif
