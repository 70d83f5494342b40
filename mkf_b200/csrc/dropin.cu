// dropin.cu - the original MKF GPU entry points, re-implemented for sm_100a.
//
//   binMapCUDA            replaces binMapCUDA.cu:144-264 (kernels binMapCUDA.cuh:282-338)
//   binMapCUDACleanup     replaces binMapCUDA.cu:266-270
//   mkfCUDAGetBPFD        replaces mkfCUDA.cu:12-61 (kernels bpfdCUDA.cuh:92-206)
//   mkfCUDAGetBPFDH       replaces mkfCUDA.cu:72-91
//   mkfCUDACleanup        replaces mkfCUDA.cu:93-99 (never resets the device)
//   mkfCUDAGetBPFDautoCtx replaces mkfCUDA.cu:101-167
//
// Behaviour kept from the original: argument meaning, the packed-map layout, unit dimensions
// dropped before the layout is set (copyNonZeroDef), several enabled fields summed element-wise
// in the field's own precision, FP32 fields compared with the threshold rounded to float, the
// counts accumulating into the caller's array, NULL returns on error, synchronous calls.
// Behaviour that differs (each is undefined or wrong in the original):
//   * FP64 fields are compared in FP64 on every path (the original reads them as float when the
//     row length is not a multiple of 32, when strided, or when several fields are summed);
//   * any row length works (the original's strided kernel shuffles across exited lanes);
//   * padding bits past the row end are written as 0;
//   * rows shorter than 32 elements contribute X-1 cells (the original counts 2X-1).
#include <cstdio>
#include <cstring>
#include "mkf_common.cuh"
#include "binMapCUDA.h"
#include "mkfCUDA.h"

namespace mkf {

struct PackArgs
{
   const void *f[BMCU_FIELD_MAX];
   int nF;
   int64_t sx, sy, sz;
   int X, Y, Z;            // region mapped
   uint32_t rowWS, planeWS;
   double t;
   uint32_t m;
   uint32_t *w;
   long long nWords;       // rowWS * Y * Z
};

// One warp per row (y, z) of the map: lane j thresholds element x = 32 w + j (the sum of the
// fields) of word w, U words per step with all their loads issued before the first ballot (U = 8:
// a 256-element row in one step, 1-2 KB in flight per warp), and a ballot assembles each word;
// lanes 0..U-1 store the step's words. Loads are coalesced along x for planar fields; elements
// past the row end are not read (their bits are 0).
template <typename T, int U>
__global__ void __launch_bounds__(256) packMap(const __grid_constant__ PackArgs a)
{
   const int lane = threadIdx.x & 31;
   const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
   const long long nRows = (long long)a.Y * a.Z;
   const T t = (T)a.t;
   const T *f0 = (const T *)a.f[0];
   for (long long row = gw; row < nRows; row += nw) {
      const uint32_t r32 = (uint32_t)row;  // rows fit 32 bits (checked at launch)
      const int z = (int)(r32 / (uint32_t)a.Y);
      const int y = (int)(r32 - (uint32_t)z * (uint32_t)a.Y);
      const long long base = (long long)y * a.sy + (long long)z * a.sz;
      uint32_t *wrow = a.w + (size_t)z * a.planeWS + (size_t)y * a.rowWS;
      for (int w0 = 0; w0 < (int)a.rowWS; w0 += U) {
         T v[U];
         bool in[U];
#pragma unroll
         for (int u = 0; u < U; u++) {
            const int x = 32 * (w0 + u) + lane;
            in[u] = x < a.X;
            v[u] = in[u] ? __ldg(f0 + base + (long long)x * a.sx) : T(0);
         }
         for (int k = 1; k < a.nF; k++) {
#pragma unroll
            for (int u = 0; u < U; u++) {
               const int x = 32 * (w0 + u) + lane;
               if (in[u]) { v[u] += __ldg((const T *)a.f[k] + base + (long long)x * a.sx); }
            }
         }
         uint32_t mine = 0;
#pragma unroll
         for (int u = 0; u < U; u++) {
            const uint32_t word = __ballot_sync(FULL, in[u] ? (a.m >> relIdx(v[u], t)) & 1u : 0u);
            mine = (lane == u) ? word : mine;
         }
         if (lane < U && w0 + lane < (int)a.rowWS) { wrow[w0 + lane] = mine; }
      }
   }
}

// One planar field whose rows are whole words (X a multiple of 32): map word i is elements
// 32 i .. 32 i + 31 of the field, so the map is a flat pass with no row arithmetic. A warp takes
// kPackWords consecutive words per step: lane j loads element j of each (coalesced loads in
// flight), one ballot per word, and lane i stores word i of the step. The grid is the resident
// CTAs only, each warp looping over steps (measured on the 256^3 FP32 ball, events around the
// call: 16 words per step on a resident grid 21.0-21.2 us, 32 words per step on 8 CTAs per SM
// 23.0 us).
static constexpr int kPackWords = 16;
template <typename T, int U = kPackWords>
__global__ void __launch_bounds__(256) packFlat(const __grid_constant__ PackArgs a)
{
   const int lane = threadIdx.x & 31;
   const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
   const T t = (T)a.t;
   const T *__restrict__ f0 = (const T *)a.f[0];
   for (long long w0 = gw * U; w0 < a.nWords; w0 += nw * U) {
      const int n = (int)min((long long)U, a.nWords - w0);
      const T *p = f0 + w0 * 32 + lane;
      T v[U];
#pragma unroll
      for (int u = 0; u < U; u++) { v[u] = u < n ? __ldg(p + 32 * u) : T(0); }
      uint32_t mine = 0;
#pragma unroll
      for (int u = 0; u < U; u++) {
         const uint32_t word = __ballot_sync(FULL, (a.m >> relIdx(v[u], t)) & 1u);
         mine = (lane == u) ? word : mine;
      }
      if (lane < n) { a.w[w0 + lane] = mine; }
   }
}

template <typename T>
static void launchPack(const PackArgs &a, long long grid)
{
   if (a.nF == 1 && a.sx == 1 && a.sy == a.X && a.sz == (int64_t)a.X * a.Y && (int64_t)a.rowWS * 32 == a.X &&
       (int64_t)a.planeWS == (int64_t)a.rowWS * a.Y) {
      long long g = (a.nWords + kPackWords * 8 - 1) / (kPackWords * 8);  // 8 warps of kPackWords words per CTA
      static std::atomic<int> occ{0};
      const long long cap = (long long)smCount() * cachedOccupancy(occ, packFlat<T>, 256, 0);
      if (g > cap) { g = cap; }
      packFlat<T><<<(unsigned)(g < 1 ? 1 : g), 256>>>(a);
      return;
   }
   // words per step: as many as a row has, up to 8
   if (a.rowWS >= 8) { packMap<T, 8><<<(unsigned)grid, 256>>>(a); }
   else if (a.rowWS >= 4) { packMap<T, 4><<<(unsigned)grid, 256>>>(a); }
   else if (a.rowWS >= 2) { packMap<T, 2><<<(unsigned)grid, 256>>>(a); }
   else { packMap<T, 1><<<(unsigned)grid, 256>>>(a); }
}

struct CountArgs
{
   const uint32_t *w;
   int X;                  // elements per row
   int rows, planes;       // row pairs + 1, plane pairs + 1
   uint32_t rowWS, planeWS;
   long long nItems;       // rowWS * (rows-1) * (planes-1)
   unsigned long long *out;
};

// Packed map -> 256 counts. Each thread takes 32 cells of one row pair of one plane pair: the
// four row words and their successors give eight 32-bit corner masks v0..v7 (bit j = corner i of
// cell x = 32w + j). Uniform cells (all corners equal) are counted by popcount; only mixed cells
// form their 8-bit code, counted in a per-warp shared histogram.
template <typename I>
__global__ void __launch_bounds__(256) countMap(const __grid_constant__ CountArgs a)
{
   __shared__ uint32_t sh[8][256];
   __shared__ unsigned long long sEnds[2];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) { (&sh[0][0])[i] = 0; }
   if (threadIdx.x < 2) { sEnds[threadIdx.x] = 0; }
   __syncthreads();
   uint32_t *h = sh[warp];
   unsigned long long n0 = 0, n255 = 0;
   // (I: 32-bit index arithmetic when every item index fits, else 64-bit)
   const I stride = (I)gridDim.x * blockDim.x, rowWS = (I)a.rowWS, rowPairs = (I)(a.rows - 1);
   for (I i = (I)blockIdx.x * blockDim.x + threadIdx.x; i < (I)a.nItems; i += stride) {
      const I rp = i / rowWS;
      const int wi = (int)(i - rp * rowWS);
      const I zq = rp / rowPairs;
      const int y = (int)(rp - zq * rowPairs);
      const int z = (int)zq;
      const int nValid = min(32, a.X - 1 - 32 * wi);
      if (nValid <= 0) { continue; }
      const uint32_t vmask = (nValid >= 32) ? 0xFFFFFFFFu : ((1u << nValid) - 1u);
      const uint32_t *p0 = a.w + (size_t)z * a.planeWS + (size_t)y * a.rowWS + wi;
      const uint32_t *p1 = p0 + a.planeWS;
      const bool nx = (wi + 1) < (int)a.rowWS;
      const uint32_t r0 = p0[0], r1 = p0[a.rowWS], r2 = p1[0], r3 = p1[a.rowWS];
      const uint32_t n0w = nx ? p0[1] : 0u, n1w = nx ? p0[a.rowWS + 1] : 0u;
      const uint32_t n2w = nx ? p1[1] : 0u, n3w = nx ? p1[a.rowWS + 1] : 0u;
      const uint32_t v0 = r0, v1 = __funnelshift_r(r0, n0w, 1);
      const uint32_t v2 = r1, v3 = __funnelshift_r(r1, n1w, 1);
      const uint32_t v4 = r2, v5 = __funnelshift_r(r2, n2w, 1);
      const uint32_t v6 = r3, v7 = __funnelshift_r(r3, n3w, 1);
      const uint32_t all = v0 & v1 & v2 & v3 & v4 & v5 & v6 & v7 & vmask;
      const uint32_t none = ~(v0 | v1 | v2 | v3 | v4 | v5 | v6 | v7) & vmask;
      uint32_t mixed = vmask & ~(all | none);
      n255 += __popc(all);
      n0 += __popc(none);
      while (mixed) {
         const int j = __ffs(mixed) - 1;
         mixed &= mixed - 1;
         const uint32_t c = ((v0 >> j) & 1u) | (((v1 >> j) & 1u) << 1) | (((v2 >> j) & 1u) << 2) |
                            (((v3 >> j) & 1u) << 3) | (((v4 >> j) & 1u) << 4) | (((v5 >> j) & 1u) << 5) |
                            (((v6 >> j) & 1u) << 6) | (((v7 >> j) & 1u) << 7);
         atomicAdd(h + c, 1u);
      }
   }
   n0 = __reduce_add_sync(FULL, (unsigned)n0) ;
   n255 = __reduce_add_sync(FULL, (unsigned)n255);
   if (lane == 0) {
      if (n0) { atomicAdd(&sEnds[0], n0); }
      if (n255) { atomicAdd(&sEnds[1], n255); }
   }
   __syncthreads();
   for (int c = threadIdx.x; c < 256; c += blockDim.x) {
      unsigned long long s = 0;
      for (int k = 0; k < 8; k++) { s += sh[k][c]; }
      if (c == 0) { s += sEnds[0]; }
      if (c == 255) { s += sEnds[1]; }
      if (s) { atomicAdd(a.out + c, s); }
   }
}

static int launchCount(unsigned long long *out, const BMOrg *pO, const uint32_t *w, cudaStream_t s)
{
   CountArgs a;
   a.w = w;
   a.X = (int)pO->rowElem;
   a.rows = (int)pO->rowPairs + 1;
   a.planes = (int)pO->planePairs + 1;
   a.rowWS = pO->rowWS;
   a.planeWS = pO->planeWS;
   a.out = out;
   if (pO->rowPairs == 0 || pO->planePairs == 0 || pO->rowElem < 2 || pO->rowWS == 0) { return MKF_OK; }
   a.nItems = (long long)a.rowWS * pO->rowPairs * pO->planePairs;
   // at least 4 words per thread, at most 4 CTAs per SM: every CTA ends with up to 256 global
   // atomics on the same 256 counters, so fewer, busier CTAs finish sooner
   long long grid = (a.nItems + 1023) / 1024;
   const long long cap = (long long)smCount() * 4;
   if (grid > cap) { grid = cap; }
   if (grid < 1) { grid = 1; }
   if (a.nItems + grid * 256 < (1LL << 31)) { countMap<uint32_t><<<(unsigned)grid, 256, 0, s>>>(a); }
   else { countMap<unsigned long long><<<(unsigned)grid, 256, 0, s>>>(a); }
   return cudaFail(cudaGetLastError(), "countMap launch");
}

// Library-owned buffers of the original's lazy-allocation convention.
static uint32_t *gMap = nullptr;
static size_t gMapWords = 0;
static size_t *gBPFDDev = nullptr;
static size_t *gBPFDHost = nullptr;

struct EventTimer
{
   cudaEvent_t e0 = nullptr, e1 = nullptr;
   EventTimer() { cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventRecord(e0, 0); }
   ~EventTimer() { cudaEventDestroy(e0); cudaEventDestroy(e1); }
   float stop() {
      float ms = 0;
      cudaEventRecord(e1, 0);
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(&ms, e0, e1);
      return ms;
   }
};

}  // namespace mkf

using namespace mkf;

MKF_API BMPackWord *binMapCUDA(KernInfo *pK, BMPackWord *pW, BMOrg *pO, const BMFieldInfo *pF, const BinMapF64 *pM)
{
   if (!pF || !pM) { return nullptr; }
   int nField = 0;
   if (pF->pFieldDevPtrTable) { nField = countValidPtrByMask(pF->pFieldDevPtrTable, pF->fieldTableMask); }
   FieldDef d[3];
   const int nDim = copyNonZeroDef(d, pF->pD, 3);
   if (nDim <= 0 || nField <= 0) { return nullptr; }
   if (pF->elemID != ENC_F32 && pF->elemID != ENC_F64) {
      logError("binMapCUDA() - element encoding 0x%02X not supported\n", pF->elemID);
      return nullptr;
   }
   BMOrg org;
   const size_t words = setBMO(&org, d, (char)pF->profID);
   if (pO) { *pO = org; }
   if (words == 0) { return nullptr; }
   if (!pW) {
      if (gMapWords < words) {
         if (gMap) { cudaFree(gMap); gMap = nullptr; gMapWords = 0; }
         if (cudaMalloc(&gMap, words * sizeof(uint32_t)) != cudaSuccess) {
            cudaGetLastError();
            logError("binMapCUDA() - cudaMalloc(%zu) failed\n", words * sizeof(uint32_t));
            return nullptr;
         }
         gMapWords = words;
      }
      pW = gMap;
   }
   PackArgs a;
   memset(&a, 0, sizeof(a));
   ConstFieldPtr fp[BMCU_FIELD_MAX];
   a.nF = copyValidPtrByMask(fp, BMCU_FIELD_MAX, pF->pFieldDevPtrTable, pF->fieldTableMask);
   for (int i = 0; i < a.nF; i++) { a.f[i] = fp[i].p; }
   // element strides of the dimensions that copyNonZeroDef kept
   if (pF->pS) {
      int k = 0;
      int64_t st[3] = {0, 0, 0};
      for (int i = 0; i < 3 && k < nDim; i++) {
         if (pF->pD[i] > 1) { st[k++] = pF->pS[i]; }
      }
      a.sx = st[0];
      a.sy = st[1];
      a.sz = st[2];
   } else {
      a.sx = 1;
      a.sy = d[0];
      a.sz = (int64_t)d[0] * d[1];
   }
   a.X = d[0];
   a.Y = (int)org.rowPairs + 1;
   a.Z = (int)org.planePairs + 1;
   a.rowWS = org.rowWS;
   a.planeWS = org.planeWS;
   a.t = (pF->elemID == ENC_F32) ? (double)(float)pM->t[0] : pM->t[0];
   a.m = pM->m;
   a.w = pW;
   a.nWords = (long long)org.rowWS * a.Y * a.Z;
   if ((long long)a.Y * a.Z >= (1LL << 32)) {
      logError("binMapCUDA() - %d x %d rows exceed 2^32\n", a.Y, a.Z);
      return nullptr;
   }
   EventTimer tm;
   long long grid = ((long long)a.Y * a.Z + 7) / 8;  // a warp per row
   const long long cap = (long long)smCount() * 8;      // one wave of 8 CTAs (64 warps) per SM
   if (grid > cap) { grid = cap; }
   if (pF->elemID == ENC_F32) { launchPack<float>(a, grid); }
   else { launchPack<double>(a, grid); }
   cudaError_t e = cudaGetLastError();
   const float ms = tm.stop();
   if (e == cudaSuccess) { e = cudaGetLastError(); }
   if (e != cudaSuccess) {
      logError("binMapCUDA() - r=%d -> %s\n", (int)e, cudaGetErrorName(e));
      return nullptr;
   }
   if (pK) { pK->dtms[0] = ms; }
   return pW;
}

MKF_API void binMapCUDACleanup(void)
{
   if (gMap) { cudaFree(gMap); gMap = nullptr; gMapWords = 0; }
}

MKF_API size_t *mkfCUDAGetBPFD(KernInfo *pK, size_t *pBPFD, const BMOrg *pO, const BMPackWord *pW, const int profile)
{
   (void)profile;  // every profile of the original yields the same counts
   if (!pBPFD) { return nullptr; }
   if (!pO || !pW) { return pBPFD; }
   EventTimer tm;
   const int rc = launchCount((unsigned long long *)pBPFD, pO, pW, 0);
   const float ms = tm.stop();
   if (rc != MKF_OK) { logError("mkfCUDAGetBPFD() - %s\n", mkfLastError()); }
   if (pK) { pK->dtms[1] = ms; }
   return pBPFD;
}

MKF_API size_t *mkfCUDAGetBPFDH(KernInfo *pK, size_t *pBPFDH, const BMOrg *pO, const BMPackWord *pW, const int profile)
{
   const size_t bytes = sizeof(size_t) * MKF_BINS;
   if (!pBPFDH) {
      if (!gBPFDHost && cudaMallocHost(&gBPFDHost, bytes) != cudaSuccess) { cudaGetLastError(); gBPFDHost = nullptr; }
      pBPFDH = gBPFDHost;
   }
   if (!gBPFDDev && cudaMalloc(&gBPFDDev, bytes) != cudaSuccess) { cudaGetLastError(); gBPFDDev = nullptr; }
   if (!pBPFDH || !gBPFDDev) { return nullptr; }
   cudaMemset(gBPFDDev, 0, bytes);
   cudaGetLastError();  // clear any error left by earlier calls before checking ours
   if (!mkfCUDAGetBPFD(pK, gBPFDDev, pO, pW, profile)) { return nullptr; }
   const cudaError_t e = cudaMemcpy(pBPFDH, gBPFDDev, bytes, cudaMemcpyDeviceToHost);
   if (e != cudaSuccess) { logError("mkfCUDAGetBPFDH() - r=%d -> %s\n", (int)e, cudaGetErrorName(e)); return nullptr; }
   return pBPFDH;
}

MKF_API void mkfCUDACleanup(int lvl)
{
   (void)lvl;  // the original resets the device when lvl > 0; a shared device is never reset here
   if (gBPFDHost) { cudaFreeHost(gBPFDHost); gBPFDHost = nullptr; }
   if (gBPFDDev) { cudaFree(gBPFDDev); gBPFDDev = nullptr; }
}

MKF_API int mkfCUDAGetBPFDautoCtx(Context *pC, const FieldDef def[3], const BinMapF64 *pM, const int profile)
{
   cudaError_t r;
   if (!pC) { return 0; }
   if (pC->pHF) {
      if (!pC->pDF) {
         r = cudaMalloc(&pC->pDF, pC->bytesF);
         if (r != cudaSuccess) { logError("cudaMalloc() - r=%d\n", (int)r); pC->pDF = nullptr; }
      }
      if (pC->pDF) {
         r = cudaMemcpy(pC->pDF, pC->pHF, pC->bytesF, cudaMemcpyHostToDevice);
         if (r != cudaSuccess) { logError("cudaMemcpy() - r=%d\n", (int)r); }
      }
      if (!pC->pDU) {
         r = cudaMalloc(&pC->pDU, pC->bytesU);
         if (r != cudaSuccess) { logError("cudaMalloc() - r=%d\n", (int)r); pC->pDU = nullptr; }
      }
      if (pC->pDF && pC->pDU) {
         ConstFieldPtr fieldPtr[BMCU_FIELD_MAX];
         BMFieldInfo fi;
         setupFields(&fi, autoFieldPtr(fieldPtr, pC), pC->nField, def, pC->bytesElem, profile);
         if (!binMapCUDA(&pC->ki, pC->pDU, &pC->bmo, &fi, pM)) { return 0; }
         if (pC->pHU) {
            r = cudaMemcpy(pC->pHU, pC->pDU, pC->bytesU, cudaMemcpyDeviceToHost);
            if (r != cudaSuccess) { logError("cudaMemcpy() - r=%d\n", (int)r); }
         }
      }
   } else if (pC->pHU) {
      r = cudaMemcpy(pC->pDU, pC->pHU, pC->bytesU, cudaMemcpyHostToDevice);
      if (r != cudaSuccess) { logError("cudaMemcpy() - r=%d\n", (int)r); }
      if (!pC->pDZ) {
         r = cudaMalloc(&pC->pDZ, pC->bytesZ);
         if (r != cudaSuccess) { logError("cudaMalloc() - r=%d\n", (int)r); pC->pDZ = nullptr; }
      }
   }
   if (pC->pDU && pC->pDZ) {
      cudaMemset(pC->pDZ, 0, pC->bytesZ);
      mkfCUDAGetBPFD(&pC->ki, (size_t *)pC->pDZ, &pC->bmo, pC->pDU, MKFCU_PROFILE_FAST);
      if (pC->pHZ) {
         r = cudaMemcpy(pC->pHZ, pC->pDZ, pC->bytesZ, cudaMemcpyDeviceToHost);
         if (r != cudaSuccess) { logError("cudaMemcpy() - r=%d\n", (int)r); }
      }
   }
   return 1;
}
