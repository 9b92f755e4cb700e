/*
 * eqg_noalloc.h -- an entry point of libeqg.so that allocates no memory.
 *
 * It has no counterpart in the reference (sintefmath/equelle has no device
 * code on this path).  It exists for callers that cannot call cudaMalloc:
 * plugins loaded into a host application whose own memory pool owns every
 * device allocation, and programs whose device memory is budgeted once, up
 * front, so that no allocation may happen while they run.  Such a caller
 * passes device pointers for the input and the output; the reduction's
 * scratch (one partial sum per block of 256 elements) lives in a fixed
 * array inside the library.
 */
#ifndef EQG_NOALLOC_H
#define EQG_NOALLOC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Largest n accepted: 65536 partial sums of 256 elements each. */
#define EQG_NOALLOC_MAX_ELEMENTS (65536LL * 256LL)

/* *result = sqrt(sum_i x[i]^2), the value eqg_two_norm computes for a
 * collection holding x, written to device memory.
 *
 *   x       device array of n doubles (may be NULL when n == 0)
 *   n       0 <= n <= EQG_NOALLOC_MAX_ELEMENTS, else EQG_ERR_ARG
 *   result  device pointer to one double
 *   stream  cudaStream_t to run on (NULL: the legacy default stream)
 *
 * The call is asynchronous on `stream`; it allocates nothing and calls no
 * allocating library routine.  The scratch array is shared by every call
 * in the process on a device and keeps the last call's partial sums; calls
 * whose kernels overlap on the GPU (on different streams, or from
 * different host threads without ordering) race on it and must be
 * serialized by the caller.  The first call on each device looks up the
 * scratch array's device address (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture.
 * Returns EQG_OK or an EQG_ERR_* code with the message in eqg_last_error(). */
int eqg_two_norm_noalloc(const double* x, int64_t n, double* result, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* EQG_NOALLOC_H */
