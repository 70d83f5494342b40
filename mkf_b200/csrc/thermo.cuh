// thermo.cuh - pieces shared by the rank-table counting kernels (thermo.cu, thermo_tma.cu):
// order-preserving keys, the rank table and its set-up, the all-ones carry-save counters, the
// per-CTA histogram and its flush, and the code gathers. See thermo.cu for the method.
#pragma once
#include <type_traits>
#include "fused.cuh"

namespace mkf {

static constexpr int kThWarps = 8;
#ifndef THERMO_TY
#define THERMO_TY 8
#endif
#ifndef THERMO_MINB
#define THERMO_MINB (THERMO_TY == 8 ? 3 : 2)
#endif
#ifndef THERMO_D
#define THERMO_D 64  // default planes of cells per work item
#endif
// Untuned fields get at least this many work items per SM (the slab depth is halved until they
// do): measured on 128^3 to 512^3 fields with 16 thresholds.
static constexpr int kThItemsPerSM = 14;
static constexpr int kThSlots = 3;       // unpredicated mixed-code slots per cell (K > 1)
static constexpr int kThMaxDepth = 255;  // planes per work item the all-ones counters can hold
static constexpr int kLutShift = 18;
static constexpr int kLutSize = 1 << (32 - kLutShift);

// Order-preserving map of IEEE bits to unsigned: negative values reversed below positive ones.
__host__ __device__ __forceinline__ uint32_t sortKey(uint32_t u)
{
   return u ^ ((uint32_t)((int32_t)u >> 31) | 0x80000000u);
}

// The 32-bit word ranked on the fast path: the whole float, or the high word of a double.
template <typename T>
__device__ __forceinline__ uint32_t loadWord(const T *__restrict__ F, long long i);
template <>
__device__ __forceinline__ uint32_t loadWord<float>(const float *__restrict__ F, long long i)
{
   return __ldg(reinterpret_cast<const unsigned *>(F) + i);
}
template <>
__device__ __forceinline__ uint32_t loadWord<double>(const double *__restrict__ F, long long i)
{
   return __ldg(reinterpret_cast<const unsigned *>(F) + 2 * i + 1);
}

// Exact rank of the element F[i] by binary search over the sorted thresholds in the field's
// precision. Kept out of line: it runs only for the rare elements the fast path cannot decide.
template <typename T, bool GE>
__device__ __noinline__ uint32_t exactRank(const T *__restrict__ F, long long i, const double *sTlo, const double *sThi,
                                           int K, uint32_t nanRank)
{
   const T v = __ldg(F + i);
   uint32_t r = 0;
#pragma unroll
   for (int s = 32; s >= 1; s >>= 1) {
      if (v > sTlo[r + s - 1]) { r += s; }
   }
   if (r > (uint32_t)K) { r = K; }
   if (GE) {
      while (r < (uint32_t)K && v >= sThi[r]) { ++r; }
   }
   return (v != v) ? nanRank : r;
}

// Carry-save accumulation of the all-ones words of one plane, one word per row pair, as a fixed
// tree over NROW = 8 or 16 rows: every word enters at its row index (a compile-time constant in
// the unrolled row loop), so no branch depends on a run-time count. The tree's top carries
// (weight NROW) ripple into bit-sliced counters hi[].
template <int NROW>
struct PlaneOnes
{
   static_assert(NROW == 4 || NROW == 8 || NROW == 16, "tree of 4, 8 or 16 rows");
   uint32_t ones = 0, twos = 0, fours = 0, eights = 0;
   // bit-sliced counts of the NROW-weight carries: at most one carry per plane, so an item of up
   // to kThMaxDepth planes needs 8 slices (a 6-slice count wraps at 64 planes of all-ones cells)
   uint32_t hi[8] = {0, 0, 0, 0, 0, 0, 0, 0};
   uint32_t p1 = 0, p2 = 0, p4 = 0, p8 = 0;
   __device__ __forceinline__ static void fa(uint32_t &s, uint32_t &c, uint32_t a, uint32_t b, uint32_t d)
   {
      s = a ^ b ^ d;
      c = (a & b) | (d & (a ^ b));
   }
   __device__ __forceinline__ void ripple(uint32_t c)
   {
#pragma unroll
      for (int i = 0; i < 8; i++) {
         const uint32_t t = hi[i] & c;
         hi[i] ^= c;
         c = t;
      }
   }
   // J is the row index; called from a fully unrolled loop, so every test on J folds away
   __device__ __forceinline__ void add(const int J, uint32_t w)
   {
      if ((J & 1) == 0) { p1 = w; return; }
      uint32_t c2, c4, c8, c16;
      fa(ones, c2, ones, p1, w);
      if ((J & 2) == 0) { p2 = c2; return; }
      fa(twos, c4, twos, p2, c2);
      if (NROW == 4) { ripple(c4); return; }
      if ((J & 4) == 0) { p4 = c4; return; }
      fa(fours, c8, fours, p4, c4);
      if (NROW == 8) { ripple(c8); return; }
      if ((J & 8) == 0) { p8 = c8; return; }
      fa(eights, c16, eights, p8, c8);
      ripple(c16);
   }
   // the interface of the paired tree below (plane parity unused here)
   __device__ __forceinline__ void add(const int J, uint32_t w, bool) { add(J, w); }
   __device__ __forceinline__ void finish() {}
   __device__ __forceinline__ uint32_t total(int k) const
   {
      uint32_t v = ((ones >> k) & 1u) + 2u * ((twos >> k) & 1u) + 4u * ((fours >> k) & 1u) + 8u * ((eights >> k) & 1u);
#pragma unroll
      for (int i = 0; i < 8; i++) { v += ((uint32_t)NROW << i) * ((hi[i] >> k) & 1u); }
      return v;
   }
};

// The 8-row tree with the weight-8 carries of two planes combined before they ripple: the top
// carry of an even plane waits in p8, the odd plane's joins it in the eights slice, and only
// the weight-16 carry ripples into hi[] (16 << i each), once per two planes. finish() folds a
// carry still waiting after the last plane. HI slices hold 2^HI - 1 such carries: 8 slices
// cover 255 planes (255 x 8 rows = 2040 < 16 x 256), 6 cover 127.
template <int HI>
struct PlaneOnesPairedT
{
   uint32_t ones = 0, twos = 0, fours = 0, eights = 0;
   uint32_t hi[HI];
   uint32_t p1 = 0, p2 = 0, p4 = 0, p8 = 0;
   __device__ __forceinline__ PlaneOnesPairedT()
   {
#pragma unroll
      for (int i = 0; i < HI; i++) { hi[i] = 0; }
   }
   __device__ __forceinline__ void ripple(uint32_t c)
   {
#pragma unroll
      for (int i = 0; i < HI; i++) {
         const uint32_t t = hi[i] & c;
         hi[i] ^= c;
         c = t;
      }
   }
   // J is the row index (compile-time in the unrolled row loop); odd: this plane closes a pair
   __device__ __forceinline__ void add(const int J, uint32_t w, bool odd)
   {
      if ((J & 1) == 0) { p1 = w; return; }
      uint32_t c2, c4, c8, c16;
      PlaneOnes<8>::fa(ones, c2, ones, p1, w);
      if ((J & 2) == 0) { p2 = c2; return; }
      PlaneOnes<8>::fa(twos, c4, twos, p2, c2);
      if ((J & 4) == 0) { p4 = c4; return; }
      PlaneOnes<8>::fa(fours, c8, fours, p4, c4);
      if (!odd) { p8 = c8; return; }
      PlaneOnes<8>::fa(eights, c16, eights, p8, c8);
      p8 = 0;
      ripple(c16);
   }
   __device__ __forceinline__ void finish()
   {
      const uint32_t c16 = eights & p8;
      eights ^= p8;
      p8 = 0;
      ripple(c16);
   }
   __device__ __forceinline__ uint32_t total(int k) const
   {
      uint32_t v = ((ones >> k) & 1u) + 2u * ((twos >> k) & 1u) + 4u * ((fours >> k) & 1u) + 8u * ((eights >> k) & 1u);
#pragma unroll
      for (int i = 0; i < HI; i++) { v += (16u << i) * ((hi[i] >> k) & 1u); }
      return v;
   }
};
using PlaneOnesPaired = PlaneOnesPairedT<8>;

// Shared state of a CTA while it counts one field: the rank table, the thresholds, and the
// per-threshold totals. The [K][256] histogram and the warps' staging planes are dynamic.
// Rank-table value of the buckets whose keys take the exact slow path: above every rank, so one
// compare finds them. They are the keys below 0x00800000 and from 0xFF800000 up: the infinities
// and NaNs of FP32 fields, and of FP64 fields (ranked by the high word) the infinities, NaNs and
// magnitudes of 2^1017 and more.
static constexpr uint32_t kSlowBucket = MKF_MAX_THRESH + 1;
static constexpr int kThKeys = MKF_MAX_THRESH + 8;  // keys indexed up to kSlowBucket + 3
struct ThermoShared
{
   alignas(16) uint8_t lut[kLutSize];
   uint32_t key[kThKeys];  // padded: a bucket's candidates may run past the last key (or the sentinel)
   double tlo[64];
   double thi[64];
   uint32_t ones[MKF_MAX_THRESH];
   unsigned long long cells;
};

// Dynamic shared memory: the [K][256] histogram, rows kHistRow words apart (one word of skew, so
// that equal codes of different thresholds fall in different banks), then one scratch word per
// lane.
#ifndef THERMO_HROW
#define THERMO_HROW 257
#endif
static constexpr int kHistRow = THERMO_HROW;
// Copies of the histogram, picked by lane: neighbouring cells (neighbouring lanes) often add to the
// same (threshold, code) word in the same instruction, and each copy takes a share of those
// same-address updates; the copies sit an odd multiple of 16 banks apart for K odd, 16 for K even.
#ifndef THERMO_HCOPIES
#define THERMO_HCOPIES 2
#endif
static constexpr int kHistCopies = THERMO_HCOPIES;
// (plus per-lane scratch words after it, 32 + 2 rows: an empty slot q adds to scratch + q rows)
__host__ __device__ constexpr size_t thermoDynBytes(int K)
{
   return ((size_t)K * kHistRow * kHistCopies + 32 + 2 * kHistRow) * sizeof(uint32_t);
}

// Load one field's thresholds, build its rank table and clear the histogram (whole CTA).
// copyRows: histogram rows per copy (K, or more when rows past K take discarded counts);
// copies: histogram copies.
template <typename P>
__device__ void ctaSetup(const P &a, ThermoShared &S, uint32_t *hist, int copyRows = 0, int copies = kHistCopies)
{
   const int K = a.K;
   const int rows = copyRows > 0 ? copyRows : K;
   for (int i = threadIdx.x; i < rows * kHistRow * copies; i += blockDim.x) { hist[i] = 0; }
   for (int i = threadIdx.x; i < 64; i += blockDim.x) {
      S.tlo[i] = a.tlo[i];
      S.thi[i] = a.thi[i];
   }
   for (int i = threadIdx.x; i < kThKeys; i += blockDim.x) { S.key[i] = (i < K) ? a.tkey[i] : 0xFFFFFFFFu; }
   __syncthreads();
   // bucket b -> number of threshold keys below the bucket's first key (keys sorted: binary
   // search), four buckets per 32-bit store
   uint32_t *lut4 = reinterpret_cast<uint32_t *>(S.lut);
   for (int w = threadIdx.x; w < kLutSize / 4; w += blockDim.x) {
      uint32_t word = 0;
#pragma unroll
      for (int q = 0; q < 4; q++) {
         const uint32_t start = (uint32_t)(4 * w + q) << kLutShift;
         int lo = 0, hi = K;  // first key >= start
         while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (S.key[mid] < start) { lo = mid + 1; } else { hi = mid; }
         }
         const uint32_t b = 4 * w + q;  // keys < 0x00800000 or >= 0xFF800000
         word |= (b < 32 || b >= kLutSize - 32 ? kSlowBucket : (uint32_t)lo) << (8 * q);
      }
      lut4[w] = word;
   }
   if (threadIdx.x < MKF_MAX_THRESH) { S.ones[threadIdx.x] = 0; }
   if (threadIdx.x == 0) { S.cells = 0; }
   __syncthreads();
}

// Add the CTA's counts of one field to its output rows (whole CTA; call after every warp has
// added its cells to S.cells): mixed codes as counted, 255 from the all-ones sums, 0 = the rest.
template <typename P>
__device__ void ctaFlush(const P &a, ThermoShared &S, const uint32_t *hist, int copyRows = 0, int copies = kHistCopies)
{
   __syncthreads();
   const int K = a.K;
   const int rows = copyRows > 0 ? copyRows : K;
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nWarps = blockDim.x >> 5;
   for (int k = warp; k < K; k += nWarps) {
      uint32_t s = 0;
      for (int c = 1 + lane; c < 255; c += 32) {
         for (int q = 0; q < copies; ++q) { s += hist[(q * rows + k) * kHistRow + c]; }
      }
      s = __reduce_add_sync(FULL, s);
      if (lane == 0) {
         const unsigned long long n1 = S.ones[k];
         const unsigned long long n0 = S.cells - n1 - s;
         uint64_t *o = a.out + (size_t)a.outRow[k] * 256;
         const int c0 = a.complement ? 255 : 0;
         if (n0) { atomicAdd((unsigned long long *)(o + c0), n0); }
         if (n1) { atomicAdd((unsigned long long *)(o + (255 - c0)), n1); }
      }
   }
   for (int i = threadIdx.x; i < K * 256; i += blockDim.x) {
      const int c = i & 255;
      uint32_t v = 0;
      for (int q = 0; q < copies; ++q) { v += hist[(q * rows + (i >> 8)) * kHistRow + c]; }
      if (v && c != 0 && c != 255) {
         const int cc = a.complement ? 255 - c : c;
         atomicAdd((unsigned long long *)(a.out + (size_t)a.outRow[i >> 8] * 256 + cc), (unsigned long long)v);
      }
   }
   __syncthreads();
}

// Gather the top bit of each byte of t, with the top bits of the first word's bytes moved 4 down
// beforehand (bits 3, 11, 19, 27 and 7, 15, 23, 31), into an 8-bit code: the multiply's shifted
// partial products never overlap below bit 32.
__device__ __forceinline__ uint32_t gatherCode(uint32_t t) { return (t * 0x00204081u) >> 24; }

// Add 1 to the shared-memory word at byte address `addr` (a predicated atomic costs a branch, so
// slots with nothing to count add to a per-lane scratch word instead).
__device__ __forceinline__ void redShared(uint32_t addr)
{
   asm volatile("red.shared.add.u32 [%0], 1;" ::"r"(addr) : "memory");
}

// The same at byte address addr + OFF (the offset rides in the instruction).
template <int OFF>
__device__ __forceinline__ void redSharedAt(uint32_t addr)
{
   asm volatile("red.shared.add.u32 [%0+%1], 1;" ::"r"(addr), "n"(OFF) : "memory");
}

// Gather eight bits of t into an 8-bit code with one multiply: for bit 0 of every byte of the
// first corner word at bits 0, 8, 16, 24 and of the second at bits 4, 12, 20, 28, the multiplier
// 0x01020408 moves them to bits 24..31 in corner order; for bit 1 (positions one higher)
// 0x00810204 does, for bit 2 0x00408102. No two partial products meet below bit 32, so no carry
// reaches the code.
__device__ __forceinline__ uint32_t gatherBits(uint32_t t, uint32_t mul) { return (t * mul) >> 24; }

// Pattern of a cell for threshold k from its two faces' packed corner ranks R0 (plane z) and R1
// (plane z + 1), C = 0x7F7F7F7F - k * 0x01010101: adding C sets a byte's top bit iff its rank
// exceeds k (ranks <= 32, no carries between bytes); the top bits of R0's bytes are moved 4 down,
// and one multiply gathers all eight (the shifted partial products never overlap below bit 32).
__device__ __forceinline__ uint32_t cellCode(uint32_t R0, uint32_t R1, uint32_t C)
{
   return gatherCode((((R0 + C) >> 4) & 0x08080808u) | ((R1 + C) & 0x80808080u));
}

// The TMA-staged rank-table kernel (thermo_tma.cu): whether it takes this pass (after prepareKeys
// and itemGrid), and its launch (MKF_ERR_UNSUPPORTED when it does not take it).
static constexpr int kTmItemsPerSM = 80;  // four items per resident warp (20 per SM)
bool thermoTmaEligible(const FusedArgs &a, int enc);
// variant: CTA shape, histogram privatisation and queue kind (kTmVariants in thermo_tma.cu,
// kTmNumVariants of them), 0 = default.
int launchThermoTma(const FusedArgs &a, int enc, int variant, cudaStream_t s);

}  // namespace mkf
