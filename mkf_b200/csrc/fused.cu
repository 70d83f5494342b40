// fused.cu - one read of a scalar field -> K binary pattern frequency distributions.
//
// Replaces the original two-pass path binMapCUDA (binMapCUDA.cu:144-264, threshold + pack) followed
// by mkfCUDAGetBPFD (mkfCUDA.cu:12-61, pack -> 256-bin counts), which makes one full pass per
// threshold and materialises the packed map in device memory. Here the packed map never exists:
//
//  * A warp owns a column of 32 x positions (31 cells; neighbouring columns overlap by one element),
//    TY rows and a slab of D planes, and walks the slab plane by plane. Each lane loads its
//    TY+1 elements of a plane (coalesced along x), maps each to a small integer, and reuses the
//    previous plane's results held in registers, so every element is read once per slab.
//  * THERMO mode (every threshold has the same relation <, <=, > or >=): thresholds are sorted, so
//    the K map bits of an element form a "thermometer" bits[k] = (k < r) described by one rank r
//    (0..K) found by binary search. A cell's pattern for threshold k is all-ones when k is below
//    the smallest corner rank, all-zeros at or above the largest, and only for k in between (a
//    few thresholds near the surface) does the 8-bit code need forming; those codes go to a
//    per-CTA shared-memory histogram with shared atomics. The all-ones counts are summed per
//    threshold with bit-sliced carry-save adders (no atomics); all-zeros counts follow from the
//    number of cells.
//  * GEN mode (relations differ, or = / !=): each element gets a K-bit word of map bits and the
//    same scheme runs on bit words (all-ones = AND of the corners, mixed = OR ^ AND).
//
// Pattern bit order is the original's (bpfdCUDA.cuh:45-61): bit i <-> corner
// (x + (i&1), y + ((i>>1)&1), z + ((i>>2)&1)). Every row of X elements yields X-1 cells.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>
#include "fused.cuh"

namespace mkf {

static constexpr int kWarps = 8;

// Number of sorted thresholds t[0..] with f > t (padding entries are +inf).
template <typename T, int LEVELS>
__device__ __forceinline__ uint32_t rankAbove(T f, const T *__restrict__ t)
{
   uint32_t r = 0;
#pragma unroll
   for (int s = 1 << (LEVELS - 1); s >= 1; s >>= 1) {
      if (f > t[r + s - 1]) { r += s; }
   }
   return r;
}

template <typename T>
__device__ __forceinline__ T loadElem(const T *__restrict__ F, long long i) { return __ldg(F + i); }

// Per-element map value: THERMO -> rank (0..K), GEN -> K-bit word of map bits.
template <typename T, int LEVELS, bool THERMO>
__device__ __forceinline__ uint32_t mapElem(T v, const T *sTlo, const T *sThi, const FusedArgs &a)
{
   uint32_t lo = rankAbove<T, LEVELS>(v, sTlo);
   if (THERMO) {
      uint32_t r = lo;
      if (a.rankHi) {
         while (r < (uint32_t)a.K && v >= sThi[r]) { ++r; }
      }
      return (v != v) ? a.nanRank : r;
   } else {
      uint32_t hi = lo;
      while (hi < (uint32_t)a.K && v >= sThi[hi]) { ++hi; }
      const uint32_t tl = thermo(lo), th = thermo(hi);
      const uint32_t kmask = thermo((uint32_t)a.K);
      const uint32_t p = ((tl & a.gtm) | (th & ~tl & a.eqm) | (~th & a.ltm)) & kmask;
      return (v != v) ? a.nanP : p;
   }
}

template <typename T, int LEVELS, int TY, bool THERMO>
__global__ void __launch_bounds__(kWarps * 32, 2) fusedBPFD(const __grid_constant__ FusedArgs a)
{
   constexpr int NT = 1 << LEVELS;
   __shared__ T sTlo[NT];
   __shared__ T sThi[NT];
   __shared__ uint32_t sOnes[MKF_MAX_THRESH];
   __shared__ unsigned long long sCells;
   extern __shared__ uint32_t sHist[];  // [K][256]

   const int K = a.K;
   for (int i = threadIdx.x; i < K * 256; i += blockDim.x) { sHist[i] = 0; }
   for (int i = threadIdx.x; i < NT; i += blockDim.x) {
      sTlo[i] = (T)a.tlo[i];
      sThi[i] = (T)a.thi[i];
   }
   if (threadIdx.x < MKF_MAX_THRESH) { sOnes[threadIdx.x] = 0; }
   if (threadIdx.x == 0) { sCells = 0; }
   __syncthreads();

   const int lane = threadIdx.x & 31;
   const long long gw = (long long)blockIdx.x * kWarps + (threadIdx.x >> 5);
   const long long nw = (long long)gridDim.x * kWarps;
   const T *__restrict__ F = (const T *)a.f;
   unsigned long long cells = 0;
   SliceCounter<7> ones;

   for (long long it = gw; it < a.nItems; it += nw) {
      const int ix = (int)(it % a.nSegX);
      const long long rest = it / a.nSegX;
      const int iy = (int)(rest % a.nTileY);
      const int iz = (int)(rest / a.nTileY);
      const int x0 = 31 * ix, y0 = TY * iy, z0 = a.D * iz;
      const int x = x0 + lane;
      const bool xin = x < a.X;
      const bool cellx = (lane < 31) && (x < a.X - 1);
      const int nRow = min(TY, a.Y - 1 - y0);
      const int nPln = min(a.D, a.Z - 1 - z0);
      cells += (unsigned long long)max(0, min(31, a.X - 1 - x0)) * (unsigned)nRow * (unsigned)nPln;

      // THERMO state per row pair of the previous plane: face ranks (4 bytes) and min | max << 8.
      // GEN state: map words of the previous plane's elements and of their x+1 neighbours,
      // and the AND / OR over each face.
      uint32_t sF[THERMO ? TY : 1], sM[THERMO ? TY : 1];
      uint32_t sP[THERMO ? 1 : TY + 1], sPR[THERMO ? 1 : TY + 1], sA[THERMO ? 1 : TY], sO[THERMO ? 1 : TY];

      const long long xoff = (long long)x * a.sx;
      for (int p = 0; p <= nPln; ++p) {
         const long long zoff = xoff + (long long)(z0 + p) * a.sz;
         T v[TY + 1];
#pragma unroll
         for (int j = 0; j <= TY; ++j) {
            const int y = y0 + j;
            v[j] = (xin && y < a.Y) ? loadElem(F, zoff + (long long)y * a.sy) : (T)0;
         }
         uint32_t e[TY + 1], er[TY + 1];
#pragma unroll
         for (int j = 0; j <= TY; ++j) {
            e[j] = mapElem<T, LEVELS, THERMO>(v[j], sTlo, sThi, a);
            er[j] = __shfl_down_sync(FULL, e[j], 1);
         }
         uint32_t A[TY];
#pragma unroll
         for (int j = 0; j < TY; ++j) {
            const bool valid = cellx && (j < nRow) && (p > 0);
            A[j] = 0;
            if (THERMO) {
               const uint32_t r00 = e[j], r01 = er[j], r10 = e[j + 1], r11 = er[j + 1];
               const uint32_t fc = r00 | (r01 << 8) | (r10 << 16) | (r11 << 24);
               const uint32_t fmn = min(min(r00, r01), min(r10, r11));
               const uint32_t fmx = max(max(r00, r01), max(r10, r11));
               if (p > 0) {
                  const uint32_t rmin = min(sM[j] & 0xFFu, fmn);
                  const uint32_t rmax = max(sM[j] >> 8, fmx);
                  if (valid) {
                     A[j] = thermo(rmin);
                     const uint32_t R0 = sF[j], R1 = fc;
                     uint32_t C = 0x7F7F7F7Fu - rmin * 0x01010101u;
                     uint32_t *h = sHist + rmin * 256;
                     for (uint32_t k = rmin; k < rmax; ++k) {
                        const uint32_t t0 = (R0 + C) & 0x80808080u;
                        const uint32_t t1 = (R1 + C) & 0x80808080u;
                        const uint32_t c = ((t0 * 0x00204081u) >> 28) | (((t1 * 0x00204081u) >> 24) & 0xF0u);
                        atomicAdd(h + c, 1u);
                        C -= 0x01010101u;
                        h += 256;
                     }
                  }
               }
               sF[j] = fc;
               sM[j] = fmn | (fmx << 8);
            } else {
               const uint32_t ca = e[j] & er[j] & e[j + 1] & er[j + 1];
               const uint32_t co = e[j] | er[j] | e[j + 1] | er[j + 1];
               if (p > 0 && valid) {
                  const uint32_t all = sA[j] & ca;
                  uint32_t mixed = (sO[j] | co) ^ all;
                  A[j] = all;
                  const uint32_t q0 = sP[j], q1 = sPR[j], q2 = sP[j + 1], q3 = sPR[j + 1];
                  const uint32_t q4 = e[j], q5 = er[j], q6 = e[j + 1], q7 = er[j + 1];
                  while (mixed) {
                     const int k = __ffs(mixed) - 1;
                     mixed &= mixed - 1;
                     const uint32_t c = ((q0 >> k) & 1u) | (((q1 >> k) & 1u) << 1) | (((q2 >> k) & 1u) << 2) |
                                        (((q3 >> k) & 1u) << 3) | (((q4 >> k) & 1u) << 4) | (((q5 >> k) & 1u) << 5) |
                                        (((q6 >> k) & 1u) << 6) | (((q7 >> k) & 1u) << 7);
                     atomicAdd(sHist + k * 256 + c, 1u);
                  }
               }
               sA[j] = ca;
               sO[j] = co;
            }
         }
         if (!THERMO) {
#pragma unroll
            for (int j = 0; j <= TY; ++j) { sP[j] = e[j]; sPR[j] = er[j]; }
         }
         if (p > 0) {
#pragma unroll
            for (int j = 0; j + 1 < TY; j += 2) { ones.add2(A[j], A[j + 1]); }
            if (TY & 1) { ones.add2(A[TY - 1], 0u); }
         }
      }
      // per-item flush of the all-ones counts
      for (int k = 0; k < K; ++k) {
         const uint32_t s = __reduce_add_sync(FULL, ones.total(k));
         if (lane == 0 && s) { atomicAdd(&sOnes[k], s); }
      }
      ones.clear();
   }
   if (lane == 0 && cells) { atomicAdd(&sCells, cells); }
   __syncthreads();

   // merge: mixed codes (1..254) as counted, 255 from the all-ones sums, 0 = cells - the rest
   const int warp = threadIdx.x >> 5;
   for (int k = warp; k < K; k += kWarps) {
      uint32_t s = 0;
      for (int c = 1 + lane; c < 255; c += 32) { s += sHist[k * 256 + c]; }
      s = __reduce_add_sync(FULL, s);
      if (lane == 0) {
         const unsigned long long n1 = sOnes[k];
         const unsigned long long n0 = sCells - n1 - s;
         uint64_t *o = a.out + (size_t)a.outRow[k] * 256;
         const int c0 = a.complement ? 255 : 0;
         if (n0) { atomicAdd((unsigned long long *)(o + c0), n0); }
         if (n1) { atomicAdd((unsigned long long *)(o + (255 - c0)), n1); }
      }
   }
   for (int i = threadIdx.x; i < K * 256; i += blockDim.x) {
      const int c = i & 255;
      const uint32_t v = sHist[i];
      if (v && c != 0 && c != 255) {
         const int cc = a.complement ? 255 - c : c;
         atomicAdd((unsigned long long *)(a.out + (size_t)a.outRow[i >> 8] * 256 + cc), (unsigned long long)v);
      }
   }
}

// Add `cells` to bin `bin` of output row `row` (a threshold whose map is constant).
__global__ void addConstBin(uint64_t *out, int row, int bin, unsigned long long cells)
{
   out[(size_t)row * 256 + bin] += cells;
}

// ------------------------------------------------------------------ host side

struct Pass
{
   bool thermo;
   int rankHi, complement;
   std::vector<std::pair<double, int>> thr;  // (threshold, original index)
   std::vector<uint32_t> mask;                // per sorted threshold (GEN)
};

static int levelsFor(int K)
{
   int L = 1;
   while ((1 << L) < K + 1) { ++L; }
   return L;
}

template <typename T, int LEVELS, int TY, bool THERMO>
static int launchFused(const FusedArgs &a, cudaStream_t s)
{
   static std::atomic<int> occ{0};
   const size_t smem = (size_t)a.K * 256 * sizeof(uint32_t);
   auto kern = fusedBPFD<T, LEVELS, TY, THERMO>;
   const int blocksPerSM = cachedOccupancy(occ, kern, kWarps * 32, MKF_MAX_THRESH * 256 * 4, MKF_MAX_THRESH * 256 * 4);
   long long grid = ((long long)a.nItems + kWarps - 1) / kWarps;
   const long long cap = (long long)smCount() * blocksPerSM;
   if (grid > cap) { grid = cap; }
   if (grid < 1) { grid = 1; }
   kern<<<(unsigned)grid, kWarps * 32, smem, s>>>(a);
   return cudaFail(cudaGetLastError(), "fusedBPFD launch");
}

template <typename T, int TY, bool THERMO>
static int dispatchLevels(const FusedArgs &a, cudaStream_t s)
{
   switch (levelsFor(a.K)) {
      case 1: return launchFused<T, 1, TY, THERMO>(a, s);
      case 2: return launchFused<T, 2, TY, THERMO>(a, s);
      case 3: return launchFused<T, 3, TY, THERMO>(a, s);
      case 4: return launchFused<T, 4, TY, THERMO>(a, s);
      case 5: return launchFused<T, 5, TY, THERMO>(a, s);
      default: return launchFused<T, 6, TY, THERMO>(a, s);
   }
}

// Threshold pair (tlo, thi) that makes a FP32 comparison give the exact result of comparing the
// element promoted to double with t: f > t <=> f > tlo and f >= t <=> f >= thi.
static void floatBounds(double t, double &tlo, double &thi)
{
   const float fl = (float)t;
   if ((double)fl == t) { tlo = thi = fl; return; }
   float a, b;
   if ((double)fl > t) { b = fl; a = std::nextafter(fl, -INFINITY); }
   else { a = fl; b = std::nextafter(fl, INFINITY); }
   tlo = a;
   thi = b;
}

// Plain-argument launch of one fused pass, for callers that must not touch the heap. The
// thresholds are already sorted and converted (tlo/thi as the kernel compares them).
int launchFusedPlain(const FusedPlain &q, cudaStream_t s)
{
   FusedArgs a;
   memset(&a, 0, sizeof(a));
   a.f = q.f;
   a.sx = q.sx; a.sy = q.sy; a.sz = q.sz;
   a.X = q.X; a.Y = q.Y; a.Z = q.Z;
   a.K = q.K;
   for (int i = 0; i < 64; i++) { a.tlo[i] = INFINITY; a.thi[i] = INFINITY; }
   for (int k = 0; k < q.K; k++) { a.tlo[k] = q.tlo[k]; a.thi[k] = q.thi[k]; a.outRow[k] = q.outRow[k]; }
   a.gtm = q.gtm; a.eqm = q.eqm; a.ltm = q.ltm; a.nanP = q.eqm;
   a.nanRank = q.nanRank; a.rankHi = q.rankHi; a.complement = q.complement;
   a.out = q.out;
   // the kernel choice of fieldBPFD: the word-parallel kernel for one or two thresholds, and for a
   // few of one relation
   int wordMaxK = std::min(kWordMaxK, q.enc == ENC_F32 ? 5 : 6);
   if (q.thermo && q.K == wordMaxK && tmaRowsAligned(a, q.enc)) { wordMaxK--; }
   if (q.K <= 2 || (q.thermo && q.K <= wordMaxK)) { return launchWords(a, q.enc, q.mask, s); }
   constexpr int TY = 16;
   a.D = 64;
   a.nSegX = (q.X - 1 + 30) / 31;
   a.nTileY = (q.Y - 1 + TY - 1) / TY;
   a.nSlabZ = (q.Z - 1 + a.D - 1) / a.D;
   a.nItems = (long long)a.nSegX * a.nTileY * a.nSlabZ;
   const bool f32 = q.enc == ENC_F32;
   if (q.thermo) {
      FusedArgs b = a;
      const int rc = launchThermo(b, q.enc, s);
      if (rc != MKF_ERR_UNSUPPORTED) { return rc; }
      return f32 ? dispatchLevels<float, TY, true>(a, s) : dispatchLevels<double, TY, true>(a, s);
   }
   return f32 ? dispatchLevels<float, TY, false>(a, s) : dispatchLevels<double, TY, false>(a, s);
}

int launchConstBin(uint64_t *out, int row, int bin, unsigned long long cells, cudaStream_t s)
{
   addConstBin<<<1, 1, 0, s>>>(out, row, bin, cells);
   return cudaFail(cudaGetLastError(), "addConstBin launch");
}

void floatBoundsPlain(double t, double &tlo, double &thi) { floatBounds(t, tlo, thi); }

// Split one field of a batch: constant maps go to `consts` (rows offset by rowBase). One or two
// other thresholds fill `w` for the batched word kernel (returns kPlanWords); more thresholds that
// share one thermometer relation and fit the rank table fill `t` for the batched thermometer
// kernel (kPlanThermo), unless the field has kSoloVoxels or more: such a field fills the GPU on
// its own, and the single-field kernels (the word kernel for a few thresholds, the TMA-staged rank
// table on aligned rows) count it faster than the batched rank-table kernel. Those fields, and
// the rest, take the single-field path (kPlanSingle).
static constexpr double kSoloVoxels = (double)(1 << 23);
int planBatchField(const MKFFieldDesc *pF, const MKFThreshSet *pT, int rowBase, FieldTask &t, WordTask &w,
                   std::vector<ConstEntry> &consts, bool &anyVarying, int depth)
{
   memset(&t, 0, sizeof(t));
   memset(&w, 0, sizeof(w));
   if (depth < 0) {
      // by size: shallow work items for small fields, so that a launch over many of them has
      // items enough for every SM (measured best for batches of fields up to ~400^3)
      const double vox = (double)pF->def[0] * (double)pF->def[1] * (double)pF->def[2];
      depth = vox <= (double)(1 << 25) ? 8 : 0;
   }
   const int K = pT->nT;
   int idx[MKF_MAX_THRESH], n = 0, cls0 = -2;
   for (int i = 0; i < K; i++) {
      const double tv = pT->t[i];
      const uint32_t m = (pT->m ? pT->m[i] : pT->mAll) & BMC_AL;
      if (m == 0 || m == BMC_AL || std::isnan(tv)) {
         const bool one = (m == BMC_AL) || (std::isnan(tv) && (m & BMC_EQ));
         consts.push_back({rowBase + i, one ? 255 : 0});
         continue;
      }
      int cls = -1;
      if (m == BMC_GT) { cls = 0; }
      else if (m == (BMC_GT | BMC_EQ)) { cls = 1; }
      else if (m == BMC_LT) { cls = 2; }
      else if (m == (BMC_LT | BMC_EQ)) { cls = 3; }
      if (n == 0) { cls0 = cls; }
      else if (cls != cls0) { cls0 = -1; }
      idx[n++] = i;
   }
   anyVarying = n > 0;
   if (n == 0) { return kPlanSingle; }
   const int X = pF->def[0], Y = pF->def[1], Z = pF->def[2];
   const bool planar = !(pF->stride[0] | pF->stride[1] | pF->stride[2]);
   if (n <= 2) {
      w.f = pF->p;
      w.sx = planar ? 1 : pF->stride[0];
      w.sy = planar ? (int64_t)X : pF->stride[1];
      w.sz = planar ? (int64_t)X * Y : pF->stride[2];
      w.X = X; w.Y = Y; w.Z = Z;
      w.K = n;
      for (int k = 0; k < n; k++) {
         const double tv = pT->t[idx[k]];
         if (pF->enc == ENC_F32) { floatBounds(tv, w.tlo[k], w.thi[k]); }
         else { w.tlo[k] = w.thi[k] = tv; }
         w.m[k] = (pT->m ? pT->m[idx[k]] : pT->mAll) & BMC_AL;
         w.outRow[k] = rowBase + idx[k];
      }
      prepareWordTask(w, pF->enc, depth);
      return kPlanWords;
   }
   if (cls0 < 0 || (double)X * (double)Y * (double)Z >= kSoloVoxels) { return kPlanSingle; }
   std::stable_sort(idx, idx + n, [&](int x, int y) { return pT->t[x] < pT->t[y]; });
   t.f = pF->p;
   t.sx = planar ? 1 : pF->stride[0];
   t.sy = planar ? (int64_t)X : pF->stride[1];
   t.sz = planar ? (int64_t)X * Y : pF->stride[2];
   t.X = X; t.Y = Y; t.Z = Z;
   t.K = n;
   for (int i = 0; i < 64; i++) { t.tlo[i] = INFINITY; t.thi[i] = INFINITY; }
   for (int k = 0; k < n; k++) {
      const double tv = pT->t[idx[k]];
      if (pF->enc == ENC_F32) { floatBounds(tv, t.tlo[k], t.thi[k]); }
      else { t.tlo[k] = t.thi[k] = tv; }
      t.outRow[k] = rowBase + idx[k];
   }
   t.rankHi = (cls0 == 1 || cls0 == 2);
   t.complement = (cls0 >= 2);
   const bool eqBit = (cls0 == 1 || cls0 == 3);
   t.nanRank = (eqBit != (t.complement != 0)) ? (uint32_t)n : 0u;
   return prepareThermoTask(t, pF->enc, depth) ? kPlanThermo : kPlanSingle;
}

int fieldBPFD(uint64_t *out, const MKFFieldDesc *pF, const MKFThreshSet *pT, int flags, cudaStream_t s,
              const int *rowBase /* output row of threshold i, NULL = identity */)
{
   if (!out || !pF || !pT || !pF->p) { setError("mkfFieldBPFD: NULL argument"); return MKF_ERR_ARG; }
   const int K = pT->nT;
   if (K < 1 || K > MKF_MAX_THRESH || !pT->t) { setError("mkfFieldBPFD: nT=%d out of range 1..%d", K, MKF_MAX_THRESH); return MKF_ERR_ARG; }
   if (pF->enc != ENC_F32 && pF->enc != ENC_F64) { setError("mkfFieldBPFD: encoding 0x%02X not supported", pF->enc); return MKF_ERR_UNSUPPORTED; }
   const int X = pF->def[0], Y = pF->def[1], Z = pF->def[2];
   if (X < 1 || Y < 1 || Z < 1) { setError("mkfFieldBPFD: bad dimensions %d %d %d", X, Y, Z); return MKF_ERR_ARG; }
   if (!(flags & MKF_F_ACCUMULATE)) {
      if (!rowBase) {  // rows 0..K-1: one clear
         cudaError_t e = cudaMemsetAsync(out, 0, (size_t)K * 256 * sizeof(uint64_t), s);
         if (e != cudaSuccess) { return cudaFail(e, "cudaMemsetAsync"); }
      }
      for (int i = 0; rowBase && i < K; i++) {
         cudaError_t e = cudaMemsetAsync(out + (size_t)rowBase[i] * 256, 0, 256 * sizeof(uint64_t), s);
         if (e != cudaSuccess) { return cudaFail(e, "cudaMemsetAsync"); }
      }
   }
   const unsigned long long cells = (unsigned long long)(X - 1) * (unsigned long long)(Y - 1) * (unsigned long long)(Z - 1);
   if (cells == 0) { return MKF_OK; }

   // classify thresholds
   std::vector<ConstEntry> consts;
   Pass th[4];  // > >= < <=
   Pass gen;
   gen.thermo = false;
   for (int i = 0; i < K; i++) {
      const double t = pT->t[i];
      const uint32_t m = (pT->m ? pT->m[i] : pT->mAll) & BMC_AL;
      const int row = rowBase ? rowBase[i] : i;
      if (m == 0 || m == BMC_AL || std::isnan(t)) {
         const bool one = (m == BMC_AL) || (std::isnan(t) && (m & BMC_EQ));
         consts.push_back({row, one ? 255 : 0});
         continue;
      }
      int cls = -1;
      if (m == BMC_GT) { cls = 0; }
      else if (m == (BMC_GT | BMC_EQ)) { cls = 1; }
      else if (m == BMC_LT) { cls = 2; }
      else if (m == (BMC_LT | BMC_EQ)) { cls = 3; }
      if (cls >= 0) { th[cls].thr.push_back({t, row}); th[cls].mask.push_back(m); }
      gen.thr.push_back({t, row});
      gen.mask.push_back(m);
   }
   std::vector<Pass> passes;
   int nThermo = 0, thermoCls = -1;
   for (int c = 0; c < 4; c++) { if (!th[c].thr.empty()) { nThermo++; thermoCls = c; } }
   if (!gen.thr.empty()) {
      if (nThermo == 1 && th[thermoCls].thr.size() == gen.thr.size()) {
         Pass p = th[thermoCls];
         p.thermo = true;
         p.rankHi = (thermoCls == 1 || thermoCls == 2);
         p.complement = (thermoCls >= 2);
         passes.push_back(p);
      } else {
         passes.push_back(gen);
      }
   }

   int rc = MKF_OK;
   for (Pass &ps : passes) {
      // sort ascending by threshold, keep masks and rows with their thresholds
      std::vector<int> idx(ps.thr.size());
      for (size_t i = 0; i < idx.size(); i++) { idx[i] = (int)i; }
      std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return ps.thr[x].first < ps.thr[y].first; });
      FusedArgs a;
      memset(&a, 0, sizeof(a));
      a.f = pF->p;
      const bool planar = !(pF->stride[0] | pF->stride[1] | pF->stride[2]);
      a.sx = planar ? 1 : pF->stride[0];
      a.sy = planar ? (int64_t)X : pF->stride[1];
      a.sz = planar ? (int64_t)X * Y : pF->stride[2];
      a.X = X; a.Y = Y; a.Z = Z;
      a.K = (int)idx.size();
      for (int i = 0; i < 64; i++) { a.tlo[i] = INFINITY; a.thi[i] = INFINITY; }
      uint32_t gtm = 0, eqm = 0, ltm = 0;
      for (int k = 0; k < a.K; k++) {
         const double t = ps.thr[idx[k]].first;
         if (pF->enc == ENC_F32) { floatBounds(t, a.tlo[k], a.thi[k]); }
         else { a.tlo[k] = a.thi[k] = t; }
         a.outRow[k] = ps.thr[idx[k]].second;
         const uint32_t m = ps.mask[idx[k]];
         gtm |= ((m >> 2) & 1u) << k;
         eqm |= ((m >> 1) & 1u) << k;
         ltm |= (m & 1u) << k;
      }
      a.gtm = gtm; a.eqm = eqm; a.ltm = ltm; a.nanP = eqm;
      if (ps.thermo) {
         a.rankHi = ps.rankHi;
         a.complement = ps.complement;
         const bool eqBit = (ps.mask[0] & BMC_EQ) != 0;
         a.nanRank = (eqBit != (ps.complement != 0)) ? (uint32_t)a.K : 0u;
      }
      a.out = out;
      // a few thresholds of one relation: one ballot per row and threshold costs less than the
      // rank table up to 5 (FP32) / 6 (FP64) thresholds, and less than the TMA-staged rank table
      // (16-byte aligned rows) up to 4 / 5 (B200, 512^3 Gaussian field)
      int wordMaxK = std::min(kWordMaxK, pF->enc == ENC_F32 ? 5 : 6);
      if (ps.thermo && a.K == wordMaxK && tmaRowsAligned(a, pF->enc)) { wordMaxK--; }
      if (a.K <= 2 || (ps.thermo && a.K <= wordMaxK)) {
         uint32_t masks[MKF_MAX_THRESH];
         for (int k = 0; k < a.K; k++) { masks[k] = ps.mask[idx[k]]; }
         rc = launchWords(a, pF->enc, masks, s);
         if (rc != MKF_OK) { return rc; }
         continue;
      }
      constexpr int TY = 16;
      a.D = 64;
      a.nSegX = (X - 1 + 30) / 31;
      a.nTileY = (Y - 1 + TY - 1) / TY;
      a.nSlabZ = (Z - 1 + a.D - 1) / a.D;
      a.nItems = (long long)a.nSegX * a.nTileY * a.nSlabZ;
      const bool f32 = pF->enc == ENC_F32;
      if (ps.thermo) {
         FusedArgs b = a;
         rc = launchThermo(b, pF->enc, s);
         if (rc == MKF_ERR_UNSUPPORTED) {
            rc = f32 ? dispatchLevels<float, TY, true>(a, s) : dispatchLevels<double, TY, true>(a, s);
         }
      }
      else { rc = f32 ? dispatchLevels<float, TY, false>(a, s) : dispatchLevels<double, TY, false>(a, s); }
      if (rc != MKF_OK) { return rc; }
   }
   for (const ConstEntry &ce : consts) {
      addConstBin<<<1, 1, 0, s>>>(out, ce.row, ce.bin, cells);
      rc = cudaFail(cudaGetLastError(), "addConstBin launch");
      if (rc != MKF_OK) { return rc; }
   }
   return rc;
}

}  // namespace mkf
