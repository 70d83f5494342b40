/* mkfUtil.h - Minkowski measures from a binary pattern frequency distribution (BPFD).
 * Replaces MKF src/mkfUtil.h:35-42. */
#ifndef MKF_UTIL_H
#define MKF_UTIL_H
#include "mkf_types.h"
#include "cell8Sym.h"
#ifdef __cplusplus
extern "C" {
#endif
#define MKF_REFML "Kv Mv Sv Vv"
/* Reference measures (Ohser & Mucklich). Their source is not part of MKF as published, so this
 * returns -1 in all four slots, as the original does when built with NO_REF_MEASURES (mkfUtil.c:83-90). */
void mkfRefMeasureBPFD(float m[4], const size_t aBPFD[MKF_BINS], const float s);
/* m[0] = Kv (integral Gaussian curvature density), m[3] = volume fraction, m[1] = m[2] = -1;
 * symCh receives "Kv       Vv" (12 bytes); returns 2 (mkfUtil.c:94-123). */
int mkfSelectMeasuresBPFD(float m[4], char symCh[16], const size_t aBPFD[MKF_BINS], const float s, const int profID);
/* Fraction of cells whose first corner is set (mkfUtil.c:125-135). */
float volFrac(const size_t hBPD[MKF_BINS]);
#ifdef __cplusplus
}
#endif
#endif
