/* ctUtil.h - CUDA test utilities exported by libMKF.so. Replaces MKF src/ctUtil.h:16-27. */
#ifndef CT_UTIL_H
#define CT_UTIL_H
#include "mkf_types.h"
#ifdef __cplusplus
extern "C" {
#endif
/* Number of CUDA devices. */
int ctuInfo(void);
/* Allocate the Context buffers whose byte counts are > 0 and whose pointers are NULL
 * (pinned host + device); returns 1 on success. */
int cuBuffAlloc(Context *pC, unsigned int n);
/* Release every Context buffer; returns 1 on success. */
int cuBuffRelease(Context *pC);
#ifdef __cplusplus
}
#endif
#if defined(__cplusplus) && defined(__CUDACC__)
#include <cuda_runtime.h>
/* Log and return the pending CUDA error (or *pE); C++ linkage as in the original. */
extern cudaError_t ctuErr(cudaError_t *pE, const char *s);
#endif
#endif
