/* binMapUtil.h - host-side helpers for describing fields and packed binary maps.
 * Each declaration replaces the function of the same name in MKF src/binMapUtil.h. */
#ifndef BIN_MAP_UTIL_H
#define BIN_MAP_UTIL_H
#include "mkf_types.h"
#include "encoding.h"
#include "geomSVU.h"
#ifdef __cplusplus
extern "C" {
#endif
/* Fill a relation descriptor from a string of '<' '=' '>' characters; a leading '!' negates.
 * The threshold is taken as float, as the original does (binMapUtil.h:85). */
BinMapF64 *setBinMapF64(BinMapF64 *pBM64, const char relopChars[], const float t);
/* Fill the packed-map organisation for def; returns the buffer size in 32-bit words
 * (binMapUtil.h:89). profID low nibble != 0 selects a two-plane buffer. */
size_t setBMO(BMOrg *pO, const FieldDef def[3], const char profID);
/* Copy the dimensions > 1 to the front of d, pad the rest with 1 (0 if none); returns their count
 * (binMapUtil.h:91). */
int copyNonZeroDef(FieldDef d[], const FieldDef *pD, const int nD);
/* Field pointer table helpers (binMapUtil.h:93-95). */
int copyValidPtrByMask(ConstFieldPtr r[], const int max, const ConstFieldPtr a[], const uint32_t mask);
int countValidPtrByMask(const ConstFieldPtr a[], uint32_t mask);
/* Stride generation (binMapUtil.h:99-101). */
int genStride(FieldStride fs[], const int n, const int start, const FieldDef *pD, FieldStride stride);
int copyOrGenStride(FieldStride fs[], const int n, const int start, const FieldDef *pD, const FieldStride *pS);
/* Field-table set-up helpers (binMapUtil.h:127-131). */
ConstFieldPtr *asFieldTab(const void **pp, const NumEnc id);
const BMFieldInfo *setupFields(BMFieldInfo *pI, void **ppF, const int nF, const int def[3], const int elemBytes, const int profile);
void **autoFieldPtr(ConstFieldPtr ptr[BMCU_FIELD_MAX], const Context *pC);
#ifdef __cplusplus
}
#endif
#endif
