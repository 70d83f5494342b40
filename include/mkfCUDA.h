/* mkfCUDA.h - packed binary map -> binary pattern frequency distribution on the GPU.
 * Replaces MKF src/mkfCUDA.h:18-31. */
#ifndef MKF_CUDA_H
#define MKF_CUDA_H
#include "binMapCUDA.h"
#include "mkfUtil.h"
#include "encoding.h"
#ifdef __cplusplus
extern "C" {
#endif
#define MKFCU_PROFILE_FAST (3)
#define MKFCU_PROFILE_FLEX (2)
/* Add the 256-bin pattern counts of the map pW (device) to pBPFD (device, size_t[256], caller zeroes).
 * Returns pBPFD, NULL when pBPFD is NULL (mkfCUDA.cu:12-61). */
size_t *mkfCUDAGetBPFD(KernInfo *pK, size_t *pBPFD, const BMOrg *pO, const BMPackWord *pW, const int profile);
/* As above, but the counts start from zero and are copied to the host array pBPFDH
 * (NULL: a pinned array owned by the library). Returns the host array or NULL (mkfCUDA.cu:72-91). */
size_t *mkfCUDAGetBPFDH(KernInfo *pK, size_t *pBPFDH, const BMOrg *pO, const BMPackWord *pW, const int profile);
/* Old self-contained path: host field -> device -> map -> counts back to pC->pHZ (mkfCUDA.cu:101-167). */
int mkfCUDAGetBPFDautoCtx(Context *pC, const FieldDef def[3], const BinMapF64 *pMC, const int profile);
/* Free library-owned buffers. Unlike the original, lvl > 0 does NOT reset the device: other work
 * may share it. */
void mkfCUDACleanup(int lvl);
#ifdef __cplusplus
}
#endif
#endif
