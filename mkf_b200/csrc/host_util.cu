// host_util.cu - host-side helpers of libMKF.so: the original's field-description utilities,
// encoding helpers, vector helpers, Minkowski measures, CUDA test utilities and error reporting.
// Each exported function keeps the argument meaning and results of the function of the same
// name in the original (file:line given beside each).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include "mkf_common.cuh"
#include "binMapUtil.h"
#include "mkfUtil.h"
#include "ctUtil.h"

namespace mkf {

static thread_local char tErr[512] = "";

void setError(const char *fmt, ...)
{
   va_list ap;
   va_start(ap, fmt);
   vsnprintf(tErr, sizeof(tErr), fmt, ap);
   va_end(ap);
}

int cudaFail(cudaError_t e, const char *what)
{
   if (e == cudaSuccess) { return MKF_OK; }
   setError("%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
   return MKF_ERR_CUDA;
}

void logError(const char *fmt, ...)
{
   va_list ap;
   va_start(ap, fmt);
   vfprintf(stderr, fmt, ap);
   va_end(ap);
}

int smCount()
{
   int dev = 0, n = 0;
   cudaGetDevice(&dev);
   if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
      cudaGetLastError();
      n = 148;
   }
   return n;
}

// Symmetry group of each 2x2x2 pattern under the 48 symmetries of the cube, numbered as the
// original numbers them (mkfUtil.c:40-58, generated by c8sGetMap cell8Sym.c:341-363).
extern const uint8_t kGroupOf[256] = {
   0,  1,  1,  2,  1,  2,  3,  5,  1,  3,  2,  5,  2,  5,  5,  8,
   1,  2,  3,  5,  3,  5,  7,  9,  4,  6,  6,  10, 6,  10, 13, 16,
   1,  3,  2,  5,  4,  6,  6,  10, 3,  7,  5,  9,  6,  13, 10, 16,
   2,  5,  5,  8,  6,  10, 13, 16, 6,  13, 10, 16, 11, 15, 15, 19,
   1,  3,  4,  6,  2,  5,  6,  10, 3,  7,  6,  13, 5,  9,  10, 16,
   2,  5,  6,  10, 5,  8,  13, 16, 6,  13, 11, 15, 10, 16, 15, 19,
   3,  7,  6,  13, 6,  13, 11, 15, 7,  12, 13, 14, 13, 14, 15, 18,
   5,  9,  10, 16, 10, 16, 15, 19, 13, 14, 15, 18, 15, 18, 17, 20,
   1,  4,  3,  6,  3,  6,  7,  13, 2,  6,  5,  10, 5,  10, 9,  16,
   3,  6,  7,  13, 7,  13, 12, 14, 6,  11, 13, 15, 13, 15, 14, 18,
   2,  6,  5,  10, 6,  11, 13, 15, 5,  13, 8,  16, 10, 15, 16, 19,
   5,  10, 9,  16, 13, 15, 14, 18, 10, 15, 16, 19, 15, 17, 18, 20,
   2,  6,  6,  11, 5,  10, 13, 15, 5,  13, 10, 15, 8,  16, 16, 19,
   5,  10, 13, 15, 9,  16, 14, 18, 10, 15, 15, 17, 16, 19, 18, 20,
   5,  13, 10, 15, 10, 15, 15, 17, 9,  14, 16, 18, 16, 18, 19, 20,
   8,  16, 16, 19, 16, 19, 18, 20, 16, 18, 19, 20, 19, 20, 20, 21 };

// Per-group weights of the original: Euler gWK (mkfUtil.c:33-38), surface gWS and mean
// curvature gWM (mkfHacks.c:9-20).
extern const int kWK[22] = { 0, 3, 0, 6, 6, -3, 3, 9, 0, -6, -6, 0, 12, 0, -3, -8, -3, -12, -6, 0, 3, 0 };
extern const double kWS[22] = {
   0, 0.944412, 1.05178, 0.921095, 0.496906, 0.949947, 0.865898, 0.793181, 0.926631, 0.638921, 0.764068,
   0.784616, 0.874463, 0.868666, 0.557639, 0.682786, 0.923863, 0.496906, 0.737983, 0.65947, 0.0812817, 0 };
extern const double kWM[22] = {
   0, 0.763019, 0.642656, 0.616236, 0.686801, 0.187756, 0.167269, 0.161335, 0, -0.431447, -0.287632,
   0, 0, -0.143816, -0.592783, -0.540019, -0.475387, -0.686801, -0.616236, -0.727774, -0.331571, 0 };

// V, S, M, chi of one distribution (see mkfMeasuresF64).
void measures(double r[4], const uint64_t h[256])
{
   uint64_t g[22] = {0};
   for (int c = 0; c < 256; c++) { g[kGroupOf[c]] += h[c]; }
   uint64_t v = 0;
   for (int c = 1; c < 256; c += 2) { v += h[c]; }
   double s = (double)g[0] * kWS[0], mc = (double)g[0] * kWM[0];
   for (int i = 1; i < 22; i++) {
      s += (double)g[i] * kWS[i];
      mc += (double)g[i] * kWM[i];
   }
   int64_t k = 0;
   for (int i = 0; i < 22; i++) { k += (int64_t)kWK[i] * (int64_t)g[i]; }
   r[0] = (double)v;
   r[1] = s;
   r[2] = mc;
   r[3] = (double)k / 24.0;
}

}  // namespace mkf

using namespace mkf;

MKF_API const char *mkfLastError(void) { return tErr; }

// ---------------------------------------------------------------- binMapUtil.c

// binMapUtil.c:37-58. Characters are read until one is not a relation; a '!' in first place
// negates the resulting relation.
MKF_API BinMapF64 *setBinMapF64(BinMapF64 *pM, const char relopChars[], const float t)
{
   bool negate = false;
   uint32_t m = BMC_NV;
   for (int i = 0;; i++) {
      const char c = relopChars[i];
      if (c == '<') { m |= BMC_LT; }
      else if (c == '=') { m |= BMC_EQ; }
      else if (c == '>') { m |= BMC_GT; }
      else if (c == '!' && i == 0) { negate = true; }
      else { break; }
   }
   pM->t[0] = t;
   pM->m = negate ? (m ^ BMC_AL) : m;
   return pM;
}

// binMapUtil.c:60-87.
MKF_API size_t setBMO(BMOrg *pO, const FieldDef def[3], const char profID)
{
   const uint32_t rowWS = (uint32_t)((def[0] + 31) >> 5);
   uint32_t rows = (uint32_t)((def[1] < 2) ? def[1] : 2);
   uint32_t planes = (uint32_t)((def[2] < 2) ? def[2] : 2);
   if ((profID & 0x0F) == 0) { rows = (uint32_t)def[1]; planes = (uint32_t)def[2]; }
   const uint32_t planeWS = rowWS * rows;
   if (pO) {
      pO->rowElem = (uint32_t)def[0];
      pO->rowPairs = rows - 1;
      pO->planePairs = planes - 1;
      pO->rowWS = rowWS;
      pO->planeWS = planeWS;
   }
   return (size_t)planeWS * planes;
}

// binMapUtil.c:89-103.
MKF_API int copyNonZeroDef(FieldDef d[], const FieldDef *pD, const int nD)
{
   int n = 0;
   if (pD) {
      for (int i = 0; i < nD; i++) {
         if (pD[i] > 1) { d[n++] = pD[i]; }
      }
   }
   for (int i = n; i < nD; i++) { d[i] = (n > 0) ? 1 : 0; }
   return n;
}

// binMapUtil.c:107-121: the first `max` enabled, non-NULL entries.
MKF_API int copyValidPtrByMask(ConstFieldPtr r[], const int max, const ConstFieldPtr a[], const uint32_t mask)
{
   int n = 0;
   for (int i = 0; i < 32 && n < max; i++) {
      const uint32_t bit = 1u << i;
      if ((mask & bit) && a[i].p) { r[n++] = a[i]; }
      if (mask <= bit) { break; }
   }
   return n;
}

// binMapUtil.c:123-133.
MKF_API int countValidPtrByMask(const ConstFieldPtr a[], uint32_t mask)
{
   int n = 0;
   for (int i = 0; mask; i++, mask >>= 1) {
      if ((mask & 1u) && a[i].p) { n++; }
   }
   return n;
}

// binMapUtil.c:135-144. As in the original, the stride multiplies by pD[start] at every step
// after the first (the dimension index does not advance), so only n <= 2 gives planar strides
// beyond the first.
MKF_API int genStride(FieldStride fs[], const int n, const int start, const FieldDef *pD, FieldStride stride)
{
   if (!pD || stride == 0) { return 0; }
   for (int i = 0; i < start; i++) { stride *= pD[i]; }
   for (int r = 0; r < n; r++) {
      fs[r] = stride;
      stride *= pD[start];
   }
   return n > 0 ? n : 0;
}

// binMapUtil.c:146-155.
MKF_API int copyOrGenStride(FieldStride fs[], const int n, const int start, const FieldDef *pD, const FieldStride *pS)
{
   if (pS) {
      for (int i = 0; i < n; i++) { fs[i] = pS[i + start]; }
      return n > 0 ? n : 0;
   }
   return genStride(fs, n, start, pD, 1);
}

// binMapUtil.c:158-164.
MKF_API ConstFieldPtr *asFieldTab(const void **pp, const NumEnc id)
{
   (void)id;
   return (ConstFieldPtr *)pp;
}

// binMapUtil.c:166-186.
MKF_API const BMFieldInfo *setupFields(BMFieldInfo *pI, void **ppF, const int n, const int def[3], const int b, const int profile)
{
   if (!pI || n <= 0 || n >= 32) { return nullptr; }
   if (b == (int)sizeof(float)) { pI->elemID = ENC_F32; }
   else if (b == (int)sizeof(double)) { pI->elemID = ENC_F64; }
   else { return nullptr; }
   pI->fieldTableMask = (1u << n) - 1u;
   pI->oprID = 0;
   pI->profID = (uint8_t)profile;
   pI->flags = 0;
   pI->pD = def;
   pI->pS = nullptr;
   pI->pFieldDevPtrTable = asFieldTab((const void **)ppF, pI->elemID);
   return pI;
}

// binMapUtil.c:188-205.
MKF_API void **autoFieldPtr(ConstFieldPtr ptr[BMCU_FIELD_MAX], const Context *pC)
{
   if (pC->nField > 1) {
      const size_t step = (size_t)pC->nElem * pC->bytesElem;
      const int n = pC->nField < BMCU_FIELD_MAX ? pC->nField : BMCU_FIELD_MAX;
      for (int i = 0; i < n; i++) { ptr[i].w = (size_t)pC->pDF + i * step; }
      return (void **)ptr;
   }
   return (void **)&pC->pDF;
}

// ---------------------------------------------------------------- encoding.c

// encoding.c:9-25.
MKF_API size_t encSizeN(int *pElemBits, const size_t n, const NumEnc e)
{
   int b = e & ENC_MASK_NUM;
   size_t bytes;
   const int typ = e & ENC_MASK_TYP;
   if (typ == ENC_TYPE_FPB || typ == ENC_TYPE_INT) {
      bytes = (size_t)b * n;
      b <<= 3;
   } else {
      bytes = ((size_t)b * n) >> 3;
   }
   if (pElemBits) { *pElemBits = b; }
   return bytes;
}

// encoding.c:27-40.
MKF_API int encAlignment(const NumEnc e)
{
   const int b = e & ENC_MASK_NUM;
   const int typ = e & ENC_MASK_TYP;
   if (typ == ENC_TYPE_FPB || typ == ENC_TYPE_INT) { return b; }
   return (b + 7) >> 3;
}

// ---------------------------------------------------------------- geomSVU.c (geomSVU.c:5-108)

MKF_API int *setKNI(int r[], const int n, const int k) { for (int i = 0; i < n; i++) { r[i] = k; } return r; }
MKF_API int *copyNI(int r[], const int n, const int v[]) { for (int i = 0; i < n; i++) { r[i] = v[i]; } return r; }
MKF_API int *addKNI(int r[], const int a[], const int n, const int k) { for (int i = 0; i < n; i++) { r[i] = a[i] + k; } return r; }
MKF_API int sumNI(const int v[], int n) { int s = v[0]; for (int i = 1; i < n; i++) { s += v[i]; } return s; }
MKF_API int prodNI(const int v[], int n) { int s = v[0]; for (int i = 1; i < n; i++) { s *= v[i]; } return s; }
MKF_API int mergeMinMaxNI(int rMin[], int rMax[], const int minA[], const int maxA[], const int minB[], const int maxB[], const int n)
{
   int d = 0;
   for (int i = 0; i < n; i++) {
      rMin[i] = minA[i] < minB[i] ? minA[i] : minB[i];
      rMax[i] = maxA[i] > maxB[i] ? maxA[i] : maxB[i];
      d += rMax[i] > rMin[i];
   }
   return d;
}
MKF_API size_t sumNZ(const size_t a[], size_t n) { size_t s = a[0]; for (size_t i = 1; i < n; i++) { s += a[i]; } return s; }
MKF_API float *scaleFNI(float r[], const int n, const int v[], const float s) { for (int i = 0; i < n; i++) { r[i] = v[i] * s; } return r; }
MKF_API float *setKNF(float r[], const int n, const float k) { for (int i = 0; i < n; i++) { r[i] = k; } return r; }
MKF_API float *copyNF(float r[], const int n, const float v[]) { for (int i = 0; i < n; i++) { r[i] = v[i]; } return r; }
MKF_API float *absNF(float r[], const int n, const float v[]) { for (int i = 0; i < n; i++) { r[i] = fabsf(v[i]); } return r; }
MKF_API float *sqrNF(float r[], const int n, const float v[]) { for (int i = 0; i < n; i++) { r[i] = v[i] * v[i]; } return r; }
MKF_API float sumNF(const float v[], int n) { float s = v[0]; for (int i = 1; i < n; i++) { s += v[i]; } return s; }
MKF_API float sqrMag3D(const float dx, const float dy, const float dz) { return dx * dx + dy * dy + dz * dz; }
MKF_API float sep3D(const float a[3], const float b[3])
{
   const float s2 = sqrMag3D(a[0] - b[0], a[1] - b[1], a[2] - b[2]);
   return s2 > 0 ? sqrtf(s2) : 0;
}

// ---------------------------------------------------------------- cell8Sym.c / mkfUtil.c

// cell8Sym.c:341-363.
MKF_API int c8sGetMap(uint8_t map[CELL8_PATTERNS])
{
   memcpy(map, kGroupOf, 256);
   return CELL8_SYMM_GROUPS;
}

// mkfUtil.c:125-135.
MKF_API float volFrac(const size_t h[MKF_BINS])
{
   size_t s0 = 0, s1 = 0;
   for (int c = 0; c < MKF_BINS; c += 2) { s0 += h[c]; s1 += h[c + 1]; }
   return (float)s1 / (float)(s0 + s1);
}

// mkfUtil.c:83-90 as built with NO_REF_MEASURES (the reference-measure source is not published).
MKF_API void mkfRefMeasureBPFD(float m[4], const size_t aBPFD[MKF_BINS], const float s)
{
   (void)aBPFD;
   (void)s;
   m[0] = m[1] = m[2] = m[3] = -1;
}

// mkfUtil.c:94-123 without the reference-measure branch: m[0] = Kv, m[3] = Vv, single precision
// exactly as the original rounds it.
MKF_API int mkfSelectMeasuresBPFD(float m[4], char symCh[16], const size_t aBPFD[MKF_BINS], const float s, const int profID)
{
   (void)profID;
   size_t g[CELL8_SYMM_GROUPS] = {0};
   size_t t = 0, tg = 0;
   for (int c = 0; c < MKF_BINS; c++) { t += aBPFD[c]; g[kGroupOf[c]] += aBPFD[c]; }
   for (int i = 0; i < CELL8_SYMM_GROUPS; i++) { tg += g[i]; }
   int64_t k = 0;
   for (int i = 0; i < CELL8_SYMM_GROUPS; i++) { k += (int64_t)kWK[i] * (int64_t)g[i]; }
   m[0] = (float)((double)k * M_PI / 6);
   m[3] = volFrac(aBPFD);
   m[1] = m[2] = -1;
   if (t == tg && s > 0) {
      const float rkV = (float)(1.0 / (s * s * s * (float)t));
      m[0] *= rkV;
   }
   memcpy(symCh, "Kv       Vv", 12);
   return 2;
}

MKF_API int mkfMeasuresF64(double *r, const uint64_t *pBPFD, int nSets)
{
   if (!r || !pBPFD || nSets < 0) { setError("mkfMeasuresF64: bad argument"); return MKF_ERR_ARG; }
   for (int i = 0; i < nSets; i++) { measures(r + 4 * i, pBPFD + 256 * (size_t)i); }
   return MKF_OK;
}

// ---------------------------------------------------------------- ctUtil.cu

// ctUtil.cu:8-42: number of devices.
MKF_API int ctuInfo(void)
{
   int n = 0;
   if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); n = 0; }
   return n;
}

// ctUtil.cu:56-80.
MKF_API int cuBuffAlloc(Context *pC, unsigned int n)
{
   (void)n;
   int err = 0;
   if (!pC->pHF && pC->bytesF > 0) { err += cudaMallocHost(&pC->pHF, pC->bytesF) != cudaSuccess; }
   if (!pC->pHU && pC->bytesU > 0) { err += cudaMallocHost((void **)&pC->pHU, pC->bytesU) != cudaSuccess; }
   if (!pC->pHZ && pC->bytesZ > 0) { err += cudaMallocHost(&pC->pHZ, pC->bytesZ) != cudaSuccess; }
   if (!pC->pDF && pC->bytesF > 0) { err += cudaMalloc(&pC->pDF, pC->bytesF) != cudaSuccess; }
   if (!pC->pDU && pC->bytesU > 0) { err += cudaMalloc((void **)&pC->pDU, pC->bytesU) != cudaSuccess; }
   if (!pC->pDZ && pC->bytesZ > 0) { err += cudaMalloc(&pC->pDZ, pC->bytesZ) != cudaSuccess; }
   if (err) { cudaGetLastError(); }
   return err == 0;
}

// ctUtil.cu:82-91.
MKF_API int cuBuffRelease(Context *pC)
{
   int err = 0;
   if (pC->pDF) { err += cudaFree(pC->pDF) != cudaSuccess; pC->pDF = nullptr; }
   if (pC->pDU) { err += cudaFree(pC->pDU) != cudaSuccess; pC->pDU = nullptr; }
   if (pC->pDZ) { err += cudaFree(pC->pDZ) != cudaSuccess; pC->pDZ = nullptr; }
   if (pC->pHF) { err += cudaFreeHost(pC->pHF) != cudaSuccess; pC->pHF = nullptr; }
   if (pC->pHU) { err += cudaFreeHost(pC->pHU) != cudaSuccess; pC->pHU = nullptr; }
   if (pC->pHZ) { err += cudaFreeHost(pC->pHZ) != cudaSuccess; pC->pHZ = nullptr; }
   return err == 0;
}

// ctUtil.cu:94-103 (C++ linkage, as in the original).
__attribute__((visibility("default"))) cudaError_t ctuErr(cudaError_t *pE, const char *s)
{
   const cudaError_t e = pE ? *pE : cudaGetLastError();
   if (e != cudaSuccess) { logError("%s - r=%d -> %s\n", s, (int)e, cudaGetErrorName(e)); }
   return e;
}
