/* binMapCUDA.h - scalar field(s) -> packed binary map on the GPU.
 * Replaces MKF src/binMapCUDA.h:15-24. */
#ifndef BIN_MAP_CUDA_H
#define BIN_MAP_CUDA_H
#include "ctUtil.h"
#include "binMapUtil.h"
#ifdef __cplusplus
extern "C" {
#endif
/* Threshold the field(s) named by pF (device pointers) with pM and write the packed binary map.
 *   pK  optional: dtms[0] receives the kernel time in ms.
 *   pW  device destination, or NULL to use a buffer owned by the library (freed by binMapCUDACleanup).
 *   pO  receives the map organisation (unit dimensions are dropped first, as the original does).
 * Several enabled fields are summed element-wise before thresholding. Returns the device map, or
 * NULL on error. Synchronous on the default stream. */
BMPackWord *binMapCUDA(KernInfo *pK, BMPackWord *pW, BMOrg *pO, const BMFieldInfo *pF, const BinMapF64 *pM);
void binMapCUDACleanup(void);
#ifdef __cplusplus
}
#endif
#endif
