/* ref_cuda_harness.cu - entry point into the reference MKF CUDA path (binMapCUDA +
 * mkfCUDAGetBPFD), compiled unmodified from its own sources for sm_100a.
 *
 * TEST AND BASELINE INFRASTRUCTURE ONLY. Linked with binMapCUDA.cu, mkfCUDA.cu, ctUtil.cu,
 * gridUtil.cu, binMapUtil.c, encoding.c and geomSVU.c into oracle/_ref/libmkfrefcuda.so by
 * oracle/Makefile. The function here only arranges arguments and calls the reference's public
 * entry points once per threshold, as a caller of the reference library does; the mapping and
 * counting are the reference's.
 *
 * The reference path is only defined for one planar field whose X extent is a multiple of 32
 * (binMapCUDA.cu:167-178 collapsed mapField; bpfdCUDA.cuh:92-118 reads words 0 .. X/32 - 1 of a
 * row when X % 32 == 0). Anything else is rejected here before a launch. The packed map buffer is
 * the caller's (planeWS * Z words), so the reference's lazily sized static buffer
 * (binMapCUDA.cu:142,158-163), which keeps the size of its first use, is never used.
 */
#include <cstdio>
#include <cuda_runtime.h>
#include "mkfCUDA.h"

#define REFCU_EXPORT extern "C" __attribute__((visibility("default")))

/* util.h declares this; nothing linked here calls it. */
extern "C" SMVal deltaT(void) { return 0; }

/* Words of the packed map the reference builds for def (setBMO, binMapUtil.c:60-87, profile 0). */
REFCU_EXPORT size_t refcu_pbm_words(const int def[3]) { return setBMO(NULL, def, 0); }

/* For each of the nT thresholds t[k]: binMapCUDA (relation string rel, e.g. ">") into pbm, then
 * mkfCUDAGetBPFD with the FAST profile into dBPFD + 256 k (device, u64, zeroed by the caller; the
 * reference adds). The threshold passes through setBinMapF64, which takes a float
 * (binMapUtil.c:37), as every reference caller's does. elemBytes is 4 (FP32) or 8 (FP64).
 * msMap / msBPFD (optional) receive the sums of the reference's own per-stage timings
 * (KernInfo.dtms, utilCUDA.hpp:21-60). Returns 1 on success, 0 when the input is outside the
 * reference's defined domain or a reference call returns NULL. */
REFCU_EXPORT int refcu_bpfd(unsigned long long *dBPFD, unsigned int *pbm, const void *dField, int elemBytes,
                            const int def[3], const double *t, int nT, const char *rel, float *msMap,
                            float *msBPFD)
{
   if (!dBPFD || !pbm || !dField || !def || !t || nT <= 0 || !rel) { return 0; }
   if ((elemBytes != 4 && elemBytes != 8) || def[0] < 32 || (def[0] & 31) || def[1] < 2 || def[2] < 2) {
      return 0;
   }
   void *fields[BMCU_FIELD_MAX] = {const_cast<void *>(dField), NULL, NULL, NULL};
   BMFieldInfo fi;
   if (!setupFields(&fi, fields, 1, def, elemBytes, 0)) { return 0; }
   float sMap = 0, sBPFD = 0;
   for (int k = 0; k < nT; ++k) {
      BinMapF64 bm;
      setBinMapF64(&bm, rel, (float)t[k]);
      BMOrg bmo;
      KernInfo ki = {{0, 0}};
      const BMPackWord *w = binMapCUDA(&ki, pbm, &bmo, &fi, &bm);
      if (!w) { return 0; }
      if (!mkfCUDAGetBPFD(&ki, reinterpret_cast<size_t *>(dBPFD + 256 * (size_t)k), &bmo, w, MKFCU_PROFILE_FAST)) {
         return 0;
      }
      sMap += ki.dtms[0];
      sBPFD += ki.dtms[1];
   }
   if (msMap) { *msMap = sMap; }
   if (msBPFD) { *msBPFD = sBPFD; }
   return cudaGetLastError() == cudaSuccess ? 1 : 0;
}
