/* Reciprocal-space PME without device allocation.
 *
 * No counterpart in the reference: its reciprocal force
 * (CudaPMEReciprocalForce, include/CudaPMEReciprocalForce.h:21-238) owns
 * device buffers it allocates at set-up.  This entry point runs the same
 * spread / FFT / influence / inverse FFT / gather kernels as the context's
 * reciprocal part, with all of its own buffers (grids, twiddles, B-spline
 * moduli, energy accumulator) carved from one file-scope __device__ array of
 * 8 MiB.  It calls no cudaMalloc/cudaFree and no allocating library.
 *
 * For callers that cannot allocate device memory: code running under a
 * fixed device-memory budget that it has already handed out (a serving
 * loop that admits work by free HBM must not change the device's
 * allocation state mid-request), and code that must not trigger the
 * device-wide synchronisation a cudaMalloc/cudaFree implies.
 *
 *   xyzq       device, num_atoms float4 (x, y, z, charge), any order
 *   gradient   device, int64 SoA in 2^40 fixed point: x at [0, num_atoms),
 *              y at [stride, ...), z at [2*stride, ...); dU/dx is ADDED
 *   energy     device, one double; receives the reciprocal energy (ewks,
 *              kcal/mol), or NULL
 *   fp64_influence  nonzero: influence-function products in FP64
 *   stream     cudaStream_t to run on (NULL: the legacy default stream)
 *
 * Limits: grid dimensions even, 2..256, factoring into 2, 3, 5 and 7;
 * spline order 4, 6 or 8; all buffers together within 8 MiB (about 5.5e5
 * grid points, e.g. 80^3); larger grids return APO_STATUS_INVALID_ARGUMENT
 * with a message.  The first call on each device looks the array up
 * (cudaGetSymbolAddress) and sets kernel attributes: make it before any
 * stream capture.  Calls on one device share the array: calls that overlap
 * in time (two streams, two host threads) race; calls queued on one
 * stream are ordered and safe. */
#ifndef APOCHARMM_C_PME_RECIPROCAL_STATIC_H
#define APOCHARMM_C_PME_RECIPROCAL_STATIC_H
#include "apocharmm_c/Export.h"
#include "apocharmm_c/Status.h"
#ifdef __cplusplus
extern "C" {
#endif
APOCHARMM_C_API apo_status apo_pme_reciprocal_static(const void *xyzq, const int num_atoms, const double box_x, const double box_y, const double box_z, const int nfft_x, const int nfft_y, const int nfft_z, const int spline_order, const double kappa, long long *gradient, const int stride, double *energy, const int fp64_influence, void *stream);
#ifdef __cplusplus
}
#endif
#endif
