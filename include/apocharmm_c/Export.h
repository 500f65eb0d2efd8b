/* Symbol visibility of the C ABI (reference: capi/include/apocharmm_c/Export.h). */
#ifndef APOCHARMM_C_EXPORT_H
#define APOCHARMM_C_EXPORT_H
#define APOCHARMM_C_API __attribute__((visibility("default")))
#endif
