// mkf_common.cuh - shared host/device helpers of libMKF.so (sm_100a).
#pragma once
#include <atomic>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include "mkf_types.h"
#include "mkf_b200.h"

#define MKF_API extern "C" __attribute__((visibility("default")))

namespace mkf {

// Thread-local last error text (mkfLastError).
void setError(const char *fmt, ...);
// Record a CUDA error as the last error; returns MKF_ERR_CUDA when e != cudaSuccess.
int cudaFail(cudaError_t e, const char *what);
int smCount();

// Resident CTAs per SM of `kern` for a block size and dynamic shared-memory size, computed on the
// first call for a cache slot and kept there (a relaxed atomic: host threads that race compute the
// same value). maxSmem > 48 KB is first allowed with cudaFuncSetAttribute.
template <typename K>
int cachedOccupancy(std::atomic<int> &slot, K kern, int threads, size_t smem, size_t maxSmem = 0)
{
   int v = slot.load(std::memory_order_relaxed);
   if (v > 0) { return v; }
   if (maxSmem > 48 * 1024) { cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)maxSmem); }
   int n = 0;
   cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem);
   v = n > 0 ? n : 1;
   slot.store(v, std::memory_order_relaxed);
   return v;
}
// Log a message on stderr the way the original library reports CUDA failures (ctuErr).
void logError(const char *fmt, ...);

static constexpr unsigned FULL = 0xFFFFFFFFu;

// Relation index of f to t as the original computes it (binMapCUDA.cuh:141-145):
// 0 below, 1 equal or unordered, 2 above.
template <typename T>
__device__ __forceinline__ unsigned relIdx(T f, T t) { return 1u - (f < t) + (f > t); }

// Bits [0, r) set, r in [0, 32]: the upper word of (0 : 0xFFFFFFFF) << min(r, 32).
__device__ __forceinline__ uint32_t thermo(uint32_t r) { return __funnelshift_lc(0xFFFFFFFFu, 0u, r); }

// Bit-sliced counter of per-bit-position sums of 32-bit words, via a carry-save (Harley-Seal)
// tree: add() takes words one at a time; each bit position k of the words is summed
// independently. Exact up to 16 * (2^HI - 1) + 15 words between flushes.
template <int HI>
struct SliceCounter
{
   uint32_t ones = 0, twos = 0, fours = 0, eights = 0;
   uint32_t hi[HI];
   uint32_t pend2 = 0, pend4 = 0, pend8 = 0;  // carries waiting for their pair
   int n = 0;                                 // words added since last flush (mod 16)

   __device__ __forceinline__ SliceCounter() {
#pragma unroll
      for (int i = 0; i < HI; i++) { hi[i] = 0; }
   }
   // full adder: a + b + c -> (sum, carry)
   __device__ __forceinline__ static void fa(uint32_t &s, uint32_t &c, uint32_t a, uint32_t b, uint32_t d) {
      s = a ^ b ^ d;
      c = (a & b) | (d & (a ^ b));
   }
   __device__ __forceinline__ void addSixteen(uint32_t w) {
      uint32_t carry = w;
#pragma unroll
      for (int i = 0; i < HI; i++) {
         const uint32_t t = hi[i] & carry;
         hi[i] ^= carry;
         carry = t;
      }
   }
   // Add two words at once (the common case).
   __device__ __forceinline__ void add2(uint32_t a, uint32_t b) {
      uint32_t c2, c4, c8, c16;
      fa(ones, c2, ones, a, b);
      if (!(n & 2)) { pend2 = c2; n += 2; return; }
      fa(twos, c4, twos, pend2, c2);
      if (!(n & 4)) { pend4 = c4; n += 2; return; }
      fa(fours, c8, fours, pend4, c4);
      if (!(n & 8)) { pend8 = c8; n += 2; return; }
      fa(eights, c16, eights, pend8, c8);
      addSixteen(c16);
      n = (n + 2) & 15;
   }
   // Sum of bit position k over every word added so far (pending carries included).
   __device__ __forceinline__ uint32_t total(int k) const {
      uint32_t v = ((ones >> k) & 1u) + 2u * ((twos >> k) & 1u) + 4u * ((fours >> k) & 1u) + 8u * ((eights >> k) & 1u);
      if (n & 2) { v += 2u * ((pend2 >> k) & 1u); }
      if (n & 4) { v += 4u * ((pend4 >> k) & 1u); }
      if (n & 8) { v += 8u * ((pend8 >> k) & 1u); }
#pragma unroll
      for (int i = 0; i < HI; i++) { v += (16u << i) * ((hi[i] >> k) & 1u); }
      return v;
   }
   __device__ __forceinline__ void clear() {
      ones = twos = fours = eights = 0;
      pend2 = pend4 = pend8 = 0;
      n = 0;
#pragma unroll
      for (int i = 0; i < HI; i++) { hi[i] = 0; }
   }
};

}  // namespace mkf

namespace mkf {
// One fused counting pass in plain arguments (see launchFusedPlain in fused.cu).
struct FusedPlain
{
   const void *f;
   int enc;
   int64_t sx, sy, sz;
   int X, Y, Z;
   int K;
   double tlo[MKF_MAX_THRESH], thi[MKF_MAX_THRESH];
   int outRow[MKF_MAX_THRESH];
   uint32_t mask[MKF_MAX_THRESH];  // relation mask of each (sorted) threshold
   uint32_t gtm, eqm, ltm, nanRank;
   int thermo, rankHi, complement;
   uint64_t *out;
};
int launchFusedPlain(const FusedPlain &q, cudaStream_t s);
int launchConstBin(uint64_t *out, int row, int bin, unsigned long long cells, cudaStream_t s);
void floatBoundsPlain(double t, double &tlo, double &thi);
}  // namespace mkf
