// thermo.cu - fused counting kernel for threshold sets that share one relation (< <= > >=).
//
// Sorted thresholds make an element's K map bits a thermometer, bits[k] = (k < rank), so an
// element reduces to one rank 0..K. The rank is found with a table over order-preserving 32-bit
// keys: key(f) orders like f, the table maps key >> 18 (16384 buckets) to the number of
// threshold keys below the bucket, and one compare with the bucket's candidate threshold (up to
// four when thresholds share a bucket) finishes the count. FP32 keys are exact. A FP64 element is
// read as its high word only (same DRAM sectors, half the load bandwidth into the SM); when that
// word ties with the candidate's, the element is re-read whole and ranked exactly by binary
// search. Infinities and NaNs (and FP64 magnitudes of 2^1017 and more) fall in table buckets
// flagged for the same exact path.
//
// A warp owns 32 x positions (31 cells, neighbouring columns overlap by one element), TY row pairs
// (TY + 1 rows) and D planes; it walks the planes, loading the next plane's TY + 1 words per lane
// into registers while the current one is ranked and counted, and keeping per row pair of the
// previous plane the four corner ranks (one byte each) and their max * 65536 + min. Work items at
// the field's +x / +y edge are shifted back inside the field (their cells already owned by the
// neighbouring item are masked), so no load needs a clamp. A cell's pattern for threshold k is
// all-ones for k < min rank, all-zeros for k >= max rank, and is formed from the two faces'
// packed ranks only for k in between: three unpredicated atomic slots cover the cells spanning up
// to 3 thresholds (99 % on a smooth field); wider cells are queued and counted after the row loop.
// Codes go to the per-CTA [K][256] shared histogram. All-ones counts are summed per threshold with
// bit-sliced carry-save adders and all-zeros counts follow from the number of cells, as in
// fused.cu. The kernel is bound by the integer ALU pipe, so arithmetic that can be a multiply-add
// is written as one (it runs on the FMA pipe).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>
#include "thermo.cuh"

namespace mkf {

// One warp counts one work item (31 x positions, TY row pairs, D planes) of the field described
// by `a` into the CTA's histogram and all-ones totals. Returns the item's number of cells.
// INNER: the field has X >= 32, Y > TY, and a positive row stride whose TY multiple fits 32 bits
// in bytes. NSLOT: 3 mixed-code slots, or 1 for one threshold (a cell then has at most one).
// CMAX: rank-table candidates compared per element (1, or 4 when thresholds share buckets).
template <typename T, int TY, bool GE, int NSLOT, bool INNER, int CMAX, typename P>
__device__ __forceinline__ unsigned long long warpItem(const P &a, long long it, ThermoShared &S, uint32_t *sHist)
{
   static_assert(NSLOT == 1 || NSLOT == 3, "one or three slots");
   constexpr int W = sizeof(T) / 4;  // 32-bit words per element; the ranked word is the last one
   const int lane = threadIdx.x & 31;
   const int K = a.K;
   const uint32_t nanRank = a.nanRank;
   const uint32_t histBase = (uint32_t)__cvta_generic_to_shared(sHist);
   const uint32_t hist32 = histBase + (uint32_t)((lane & (kHistCopies - 1)) * K * kHistRow) * 4u;  // this lane's copy
   const uint32_t trash = histBase + (uint32_t)(K * kHistRow * kHistCopies + lane) * 4u;

   const int ix = (int)(it % a.nSegX);
   const long long rest = it / a.nSegX;
   const int iy = (int)(rest % a.nTileY);
   const int iz = (int)(rest / a.nTileY);
   // this item's cells: x in [xs, xe), y in [ys, ye), z in [z0, z0 + nPln)
   const int xs = 31 * ix, ys = TY * iy, z0 = a.D * iz;
   const int xe = min(xs + 31, a.X - 1), ye = min(ys + TY, a.Y - 1);
   const int nPln = min(a.D, a.Z - 1 - z0);
   // loaded tile: x0 + lane, rows y0 .. y0 + TY (INNER: all inside the field)
   const int x0 = INNER ? min(xs, a.X - 32) : xs;
   const int y0 = INNER ? min(ys, a.Y - 1 - TY) : ys;
   const int xl = INNER ? x0 + lane : min(x0 + lane, a.X - 1);  // clamped: lanes past the row end re-read it
   const int lastRow = a.Y - 1 - y0;                              // clamped: rows past it re-read it
   const int jlo = ys - y0, jhi = ye - y0;                        // counted row pairs j in [jlo, jhi)
   const bool laneIn = x0 + lane >= xs && x0 + lane < xe;
   // bit j: row pair j of this lane is counted
   const uint32_t rowsOK = laneIn ? ((1u << jhi) - 1u) & ~((1u << jlo) - 1u) : 0u;
   const long long rowStep = (long long)W * a.sy, planeStep = (long long)W * a.sz;
   const uint32_t rowBytes = (uint32_t)(rowStep * 4);
   const long long e00 = (long long)xl * a.sx + (long long)y0 * a.sy + (long long)z0 * a.sz;
   const unsigned *__restrict__ Pz = reinterpret_cast<const unsigned *>(a.f) + (W - 1) + (long long)W * e00;

   uint32_t wn[TY + 1];  // the next plane's ranked words
   auto loadPlane = [&](const unsigned *Pp) {
#pragma unroll
      for (int j = 0; j <= TY; ++j) {
         if (INNER) {
            wn[j] = __ldg(reinterpret_cast<const unsigned *>(reinterpret_cast<const char *>(Pp) + (uint64_t)(rowBytes * (uint32_t)j)));
         } else {
            wn[j] = __ldg(Pp + (long long)min(j, lastRow) * rowStep);
         }
      }
   };
   loadPlane(Pz);

   uint32_t sF[TY], sM[TY];  // previous plane: face ranks, max * 65536 + min per row pair
   typename std::conditional<TY == 8, PlaneOnesPaired, PlaneOnes<TY>>::type ones;
   for (int p = 0; p <= nPln; ++p) {
      uint32_t r[TY + 1];
#pragma unroll
      for (int j = 0; j <= TY; ++j) { r[j] = wn[j]; }
      if (p < nPln) { loadPlane(Pz + (long long)(p + 1) * planeStep); }
      bool slow = false;  // some element of this lane's column needs the exact rank
#pragma unroll
      for (int j = 0; j <= TY; ++j) {
         const uint32_t wj = r[j];
         const uint32_t key = sortKey(wj);
         const uint32_t r0 = S.lut[key >> kLutShift];
         const uint32_t cand = S.key[r0];
         r[j] = r0 + (GE ? (key >= cand) : (key > cand));
         bool tie = key == cand;
#pragma unroll
         for (int c = 1; c < CMAX; ++c) {
            // further thresholds of the same bucket; keys of later buckets (or the padding) are
            // above every key of this bucket and add nothing
            const uint32_t cc = S.key[r0 + c];
            r[j] += GE ? (key >= cc) : (key > cc);
            tie = tie || key == cc;
         }
         // FP64: a high word equal to a threshold's needs the low word too
         slow = slow || (W == 2 && tie) || r0 >= kSlowBucket;
      }
      if (slow) {
         const T *Fe = reinterpret_cast<const T *>(a.f);
         const long long e0 = e00 + (long long)p * a.sz;
#pragma unroll
         for (int j = 0; j <= TY; ++j) {
            r[j] = exactRank<T, GE>(Fe, e0 + (long long)(INNER ? j : min(j, lastRow)) * a.sy, S.tlo, S.thi, K, nanRank);
         }
      }
      uint32_t rR = __shfl_down_sync(FULL, r[0], 1);
      // faces as multiply-adds (ranks < 256): e = r | rR << 8, face = e(row j) | e(row j + 1) << 16
      uint32_t ePrev = rR * 256u + r[0];
      uint32_t mnPrev = min(r[0], rR), mxPrev = max(r[0], rR);
      if (p == 0) {
#pragma unroll
         for (int j = 0; j < TY; ++j) {
            rR = __shfl_down_sync(FULL, r[j + 1], 1);
            const uint32_t e = rR * 256u + r[j + 1];
            const uint32_t mn = min(r[j + 1], rR), mx = max(r[j + 1], rR);
            sF[j] = e * 65536u + ePrev;
            sM[j] = max(mxPrev, mx) * 65536u + min(mnPrev, mn);
            ePrev = e;
            mnPrev = mn;
            mxPrev = mx;
         }
         continue;
      }
      const bool oddPlane = (p & 1) == 0;  // counted planes 1, 2 | 3, 4 | ...: this one closes a pair
      uint4 wq[TY];  // cells of this plane spanning more than 3 thresholds (about 1 in 100)
      int nwq = 0;
#pragma unroll
      for (int j = 0; j < TY; ++j) {
         rR = __shfl_down_sync(FULL, r[j + 1], 1);
         const uint32_t e = rR * 256u + r[j + 1];
         const uint32_t mn = min(r[j + 1], rR), mx = max(r[j + 1], rR);
         const uint32_t fc = e * 65536u + ePrev;
         const uint32_t fmn = min(mnPrev, mn), fmx = max(mxPrev, mx);
         // previous face: max * 65536 + min, unpacked by multiplies (FMA pipe, not the ALU's)
         const uint32_t pmx = __umulhi(sM[j], 65536u), pmn = sM[j] - pmx * 65536u;
         const uint32_t rmin = min(pmn, fmn);
         uint32_t rmax;  // uncounted cells: rmax = rmin, no mixed codes
         if (W == 2) {   // (measured: a predicate is faster for FP64 fields, a lane mask for FP32)
            const bool counted = (rowsOK & (1u << j)) != 0;
            rmax = counted ? max(pmx, fmx) : rmin;
            ones.add(j, counted ? thermo(rmin) : 0u, oddPlane);
         } else {
            const uint32_t vmask = (rowsOK & (1u << j)) ? 0xFFFFFFFFu : 0u;
            rmax = vmask ? max(pmx, fmx) : rmin;
            ones.add(j, thermo(rmin) & vmask, oddPlane);
         }
         {
            // Mixed codes, k = rmin .. rmax - 1. With d = corner rank - rmin per byte, the code
            // for k = rmin + q marks the corners with d > q; with b0, b1 the masks of corners
            // whose d has bit 0, 1 set, the codes for a spread rmax - rmin up to 3 are b0 | b1,
            // b1, b0 & b1. Wider cells (1 in 100 on a unit-variance field with thresholds 0.27
            // apart) are queued and counted after the row loop.
            const uint32_t R0 = sF[j], R1 = fc;
            uint32_t spread;  // rmax - rmin as a multiply-add (FMA pipe)
            asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(spread) : "r"(rmin), "r"(0xFFFFFFFFu), "r"(rmax));
            const uint32_t rowAddr = hist32 + rmin * (kHistRow * 4);
            // integer multiply-adds (not shifts and logic) where they serve: the kernel is bound by
            // the integer ALU pipe, and these run on the FMA pipe
            const uint32_t D0 = R0 + rmin * 0xFEFEFEFFu;         // R0 - rmin per byte (no borrows)
            const uint32_t D1s = R1 * 16u + rmin * 0xEFEFEFF0u;  // (R1 - rmin per byte) << 4
            const uint32_t b0 = gatherBits((D0 & 0x01010101u) | (D1s & 0x10101010u), 0x01020408u);
            if (NSLOT == 1) {
               redShared(spread != 0 ? rowAddr + (b0 << 2) : trash);
            } else {
               const uint32_t b1 = gatherBits((D0 & 0x02020202u) | (D1s & 0x20202020u), 0x00810204u);
               const bool fast = spread < 4;
               redSharedAt<0>(fast && spread > 0 ? (b0 | b1) * 4u + rowAddr : trash);
               redSharedAt<kHistRow * 4>(fast && spread > 1 ? b1 * 4u + rowAddr : trash);
               redSharedAt<kHistRow * 8>(fast && spread > 2 ? (b0 & b1) * 4u + rowAddr : trash);
               if (!fast) {  // counted after the row loop: one copy of that code, not one per row
                  wq[nwq] = make_uint4(R0, R1, rmin, rmax);
                  ++nwq;
               }
            }
         }
         sF[j] = fc;
         sM[j] = fmx * 65536u + fmn;
         ePrev = e;
         mnPrev = mn;
         mxPrev = mx;
      }
      // wide cells: every code k = rmin .. rmax - 1 from the packed corner ranks, by seven fixed
      // formulas up to a spread of 7 (no loop whose trip count differs between lanes)
      for (int i = 0; i < nwq; ++i) {
         const uint32_t R0 = wq[i].x, R1 = wq[i].y, rmin = wq[i].z, rmax = wq[i].w;
         const uint32_t spread = rmax - rmin, rowAddr = hist32 + rmin * (kHistRow * 4);
         if (spread < 8) {
            // d = corner rank - rmin < 8: with b0, b1, b2 the masks of corners whose d has bit 0,
            // 1, 2 set, the code for k = rmin + q (corners with d > q) is one formula per q
            const uint32_t D0 = R0 + rmin * 0xFEFEFEFFu, D1s = R1 * 16u + rmin * 0xEFEFEFF0u;
            const uint32_t b0 = gatherBits((D0 & 0x01010101u) | (D1s & 0x10101010u), 0x01020408u);
            const uint32_t b1 = gatherBits((D0 & 0x02020202u) | (D1s & 0x20202020u), 0x00810204u);
            const uint32_t b2 = gatherBits((D0 & 0x04040404u) | (D1s & 0x40404040u), 0x00408102u);
            redSharedAt<0>((b0 | b1 | b2) * 4u + rowAddr);  // spread >= 4: codes q = 0..3 all count
            redSharedAt<kHistRow * 4>((b1 | b2) * 4u + rowAddr);
            redSharedAt<kHistRow * 8>((b2 | (b1 & b0)) * 4u + rowAddr);
            redSharedAt<kHistRow * 12>(b2 * 4u + rowAddr);
            redSharedAt<kHistRow * 16>(spread > 4 ? (b2 & (b1 | b0)) * 4u + rowAddr : trash - kHistRow * 16);
            redSharedAt<kHistRow * 20>(spread > 5 ? (b2 & b1) * 4u + rowAddr : trash - kHistRow * 20);
            redSharedAt<kHistRow * 24>(spread > 6 ? (b2 & b1 & b0) * 4u + rowAddr : trash - kHistRow * 24);
         } else {
            uint32_t C = 0x7F7F7F7Fu - rmin * 0x01010101u, addr = rowAddr;
            for (uint32_t k = rmin; k < rmax; ++k) {
               redShared(addr + (cellCode(R0, R1, C) << 2));
               C -= 0x01010101u;
               addr += kHistRow * 4;
            }
         }
      }
   }
   ones.finish();
   for (int k = 0; k < K; ++k) {
      const uint32_t s = __reduce_add_sync(FULL, ones.total(k));
      if (lane == 0 && s) { atomicAdd(&S.ones[k], s); }
   }
   return (unsigned long long)(xe - xs) * (unsigned)(jhi - jlo) * (unsigned)nPln;
}

template <typename T, int TY, bool GE, int NSLOT, bool INNER, int CMAX>
__global__ void __launch_bounds__(kThWarps * 32, THERMO_MINB) thermoBPFD(const __grid_constant__ FusedArgs a)
{
   __shared__ ThermoShared S;
   extern __shared__ uint32_t sHist[];
   ctaSetup(a, S, sHist);
   const long long gw = (long long)blockIdx.x * kThWarps + (threadIdx.x >> 5);
   const long long nw = (long long)gridDim.x * kThWarps;
   unsigned long long cells = 0;
   for (long long it = gw; it < a.nItems; it += nw) { cells += warpItem<T, TY, GE, NSLOT, INNER, CMAX>(a, it, S, sHist); }
   if ((threadIdx.x & 31) == 0 && cells) { atomicAdd(&S.cells, cells); }
   ctaFlush(a, S, sHist);
}

// ---------------------------------------------------------------- many fields, one launch

// A CTA takes chunks of consecutive work items from a global counter; chunks never span fields.
// When the next chunk belongs to another field, the CTA adds its counts of the previous field to
// that field's output rows, then loads the new field's thresholds and rank table. One kernel per
// element type and variant V (FieldTask::variant without its FP64 bit: bit 0 ">=", bit 2 shifted
// edge items, bit 3 up to four rank-table candidates), so the counting loop is the single-field
// kernel's, with its register budget; a batch launches one kernel per variant it holds.
template <typename T, int TY, int V>
__global__ void __launch_bounds__(kThWarps * 32, THERMO_MINB) thermoBatch(const __grid_constant__ BatchArgs b)
{
   __shared__ ThermoShared S;
   __shared__ FieldTask F;
   __shared__ int sChunk;
   extern __shared__ uint32_t sHist[];
   int cur = -1;
   unsigned long long cells = 0;
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   for (;;) {
      if (threadIdx.x == 0) { sChunk = (int)atomicAdd(b.counter, 1u); }
      __syncthreads();
      const int c = sChunk;
      __syncthreads();
      if (c >= b.nChunks) { break; }
      const BatchChunk ch = b.chunks[c];
      if (ch.field != cur) {
         if (cur >= 0) {
            if (lane == 0 && cells) { atomicAdd(&S.cells, cells); }
            cells = 0;
            ctaFlush(F, S, sHist);
         }
         const uint32_t *src = reinterpret_cast<const uint32_t *>(b.tasks + ch.field);
         for (int i = threadIdx.x; i < (int)(sizeof(FieldTask) / 4); i += blockDim.x) {
            reinterpret_cast<uint32_t *>(&F)[i] = src[i];
         }
         __syncthreads();
         ctaSetup(F, S, sHist);
         cur = ch.field;
      }
      for (long long it = ch.begin + warp; it < ch.end; it += kThWarps) {
         cells += warpItem<T, TY, (V & 1) != 0, kThSlots, (V & 4) != 0, (V & 8) ? 4 : 1>(F, it, S, sHist);
      }
   }
   if (cur >= 0) {
      if (lane == 0 && cells) { atomicAdd(&S.cells, cells); }
      ctaFlush(F, S, sHist);
   }
}

// Host: the key each threshold is compared by, for "f > t" (GE false) or "f >= t" (GE true).
// For a FP32 field the key is exact; for a FP64 field it is the high word's key (ties are
// resolved on the device). Minus and plus zero compare equal: "> 0" uses +0's key, ">= 0" -0's.
static uint32_t thresholdKey(double t, int enc, bool ge)
{
   if (t == 0.0) { t = ge ? -0.0 : 0.0; }
   uint32_t u;
   if (enc == ENC_F32) {
      const float f = (float)t;  // tlo/thi are exactly representable floats here
      memcpy(&u, &f, 4);
   } else {
      uint64_t b;
      memcpy(&b, &t, 8);
      u = (uint32_t)(b >> 32);
   }
   return sortKey(u);
}

template <typename T, int TY, bool GE, int NSLOT, bool INNER, int CMAX>
static int launchThermoT(const FusedArgs &a, cudaStream_t s)
{
   static std::atomic<int> occ[MKF_MAX_THRESH + 1];  // resident CTAs for each K's histogram size
   auto kern = thermoBPFD<T, TY, GE, NSLOT, INNER, CMAX>;
   const int blocksPerSM = cachedOccupancy(occ[a.K], kern, kThWarps * 32, thermoDynBytes(a.K), thermoDynBytes(MKF_MAX_THRESH));
   long long grid = (a.nItems + kThWarps - 1) / kThWarps;
   const long long cap = (long long)smCount() * blocksPerSM;
   if (grid > cap) { grid = cap; }
   if (grid < 1) { grid = 1; }
   kern<<<(unsigned)grid, kThWarps * 32, thermoDynBytes(a.K), s>>>(a);
   return cudaFail(cudaGetLastError(), "thermoBPFD launch");
}

// Whether a field's work items can all be shifted inside it (see warpItem's INNER).
template <typename P>
static bool innerTiles(const P &a, int enc)
{
   const int64_t rowBytes = a.sy * (enc == ENC_F32 ? 4 : 8);
   return a.X >= 32 && a.Y > THERMO_TY && rowBytes > 0 && rowBytes * THERMO_TY < ((int64_t)1 << 32);
}

// Fill the key table of a thermometer pass and return the most thresholds sharing one bucket of
// the rank table (1..4), or 0 when more share one (such passes use the binary-search kernel of
// fused.cu).
template <typename P>
static int prepareKeys(P &a, int enc)
{
   const bool ge = a.rankHi != 0;
   for (int k = 0; k < a.K; k++) { a.tkey[k] = thresholdKey(ge ? a.thi[k] : a.tlo[k], enc, ge); }
   int most = 1, run = 1;
   for (int k = 1; k < a.K; k++) {
      run = ((a.tkey[k] >> kLutShift) == (a.tkey[k - 1] >> kLutShift)) ? run + 1 : 1;
      most = std::max(most, run);
   }
   return most <= 4 ? most : 0;
}

// Work-item grid of a field for the thermometer kernels (TY rows, D planes, 31 cells per item).
template <typename P>
static void itemGrid(P &a, int D)
{
   D = D < 1 ? 1 : (D > kThMaxDepth ? kThMaxDepth : D);  // the all-ones counters hold kThMaxDepth planes
   constexpr int TY = THERMO_TY;
   a.D = D;
   a.nSegX = (a.X - 1 + 30) / 31;
   a.nTileY = (a.Y - 1 + TY - 1) / TY;
   a.nSlabZ = (a.Z - 1 + a.D - 1) / a.D;
   a.nItems = (long long)a.nSegX * a.nTileY * a.nSlabZ;
}

bool prepareThermoTask(FieldTask &t, int enc, int depth)
{
   t.lutC = prepareKeys(t, enc);
   if (t.lutC == 0) { return false; }
   t.variant = (enc == ENC_F32 ? 0 : 2) + (t.rankHi ? 1 : 0) + (innerTiles(t, enc) ? 4 : 0) + (t.lutC > 1 ? 8 : 0);
   itemGrid(t, depth > 0 ? depth : THERMO_D);
   return true;
}

std::vector<ThermoGroup> groupThermoChunks(std::vector<BatchChunk> &chunks, const std::vector<FieldTask> &tasks)
{
   std::vector<ThermoGroup> groups;
   std::vector<BatchChunk> sorted;
   sorted.reserve(chunks.size());
   for (int v = 0; v < kThVariants; v++) {
      ThermoGroup g{v, (int)sorted.size(), 0, 0};
      for (const BatchChunk &c : chunks) {
         const FieldTask &t = tasks[c.field];
         if ((t.variant & 13) == v) {
            sorted.push_back(c);
            g.maxK = std::max(g.maxK, t.K);
         }
      }
      g.c1 = (int)sorted.size();
      if (g.c1 > g.c0) { groups.push_back(g); }
   }
   chunks.swap(sorted);
   return groups;
}

template <typename T, int V>
static int launchThermoBatchV(const BatchArgs &b, int maxK, cudaStream_t s)
{
   constexpr int TY = THERMO_TY;
   static std::atomic<int> occ[MKF_MAX_THRESH + 1];
   auto kern = thermoBatch<T, TY, V>;
   const size_t smem = thermoDynBytes(maxK);  // every field of the group has at most maxK thresholds
   const int blocksPerSM = cachedOccupancy(occ[maxK], kern, kThWarps * 32, smem, thermoDynBytes(MKF_MAX_THRESH));
   long long grid = (long long)smCount() * blocksPerSM;
   if (grid > b.nChunks) { grid = b.nChunks; }
   if (grid < 1) { grid = 1; }
   kern<<<(unsigned)grid, kThWarps * 32, smem, s>>>(b);
   return cudaFail(cudaGetLastError(), "thermoBatch launch");
}

template <typename T>
static int launchThermoBatchT(const BatchArgs &b, int variant, int maxK, cudaStream_t s)
{
   switch (variant) {
      case 0: return launchThermoBatchV<T, 0>(b, maxK, s);
      case 1: return launchThermoBatchV<T, 1>(b, maxK, s);
      case 4: return launchThermoBatchV<T, 4>(b, maxK, s);
      case 5: return launchThermoBatchV<T, 5>(b, maxK, s);
      case 8: return launchThermoBatchV<T, 8>(b, maxK, s);
      case 9: return launchThermoBatchV<T, 9>(b, maxK, s);
      case 12: return launchThermoBatchV<T, 12>(b, maxK, s);
      case 13: return launchThermoBatchV<T, 13>(b, maxK, s);
      default: setError("thermoBatch: bad variant %d", variant); return MKF_ERR_ARG;
   }
}

int launchThermoGroups(const FieldTask *dTasks, const BatchChunk *dChunks, const std::vector<ThermoGroup> &groups,
                       unsigned *counters, int enc, cudaStream_t s)
{
   int rc = MKF_OK;
   for (const ThermoGroup &g : groups) {
      if (rc != MKF_OK) { break; }
      if (g.maxK < 1 || g.maxK > MKF_MAX_THRESH) { setError("thermoBatch: bad threshold count %d", g.maxK); return MKF_ERR_ARG; }
      BatchArgs b;
      b.tasks = dTasks;
      b.chunks = dChunks + g.c0;
      b.nChunks = g.c1 - g.c0;
      b.counter = counters + g.variant;
      rc = enc == ENC_F32 ? launchThermoBatchT<float>(b, g.variant, g.maxK, s)
                          : launchThermoBatchT<double>(b, g.variant, g.maxK, s);
   }
   return rc;
}

template <typename T, bool GE>
static int launchThermoG(const FusedArgs &a, bool inner, cudaStream_t s)
{
   constexpr int TY = THERMO_TY;
   // one threshold: a cell has at most one mixed code (and the rank table one candidate)
   if (a.K == 1) { return inner ? launchThermoT<T, TY, GE, 1, true, 1>(a, s) : launchThermoT<T, TY, GE, 1, false, 1>(a, s); }
   if (a.lutC > 1) {
      return inner ? launchThermoT<T, TY, GE, kThSlots, true, 4>(a, s) : launchThermoT<T, TY, GE, kThSlots, false, 4>(a, s);
   }
   return inner ? launchThermoT<T, TY, GE, kThSlots, true, 1>(a, s) : launchThermoT<T, TY, GE, kThSlots, false, 1>(a, s);
}

int launchThermo(FusedArgs &a, int enc, cudaStream_t s)
{
   a.lutC = prepareKeys(a, enc);
   if (a.lutC == 0) { return MKF_ERR_UNSUPPORTED; }
   const long long perPlane = (long long)((a.X - 1 + 30) / 31) * ((a.Y - 1 + THERMO_TY - 1) / THERMO_TY);
#ifndef MKF_NO_TMA
   // the TMA-staged kernel where the field allows it (up to 16 thresholds, 16-byte aligned rows)
   a.D = THERMO_D;
   if (thermoTmaEligible(a, enc)) {
      itemGrid(a, tunedDepth(kFamThermoTma, enc, a.K, a.X, a.Y, a.Z,
                             sizeDepth(THERMO_D, perPlane, a.Z, (long long)smCount() * kTmItemsPerSM)));
      const int rc = launchThermoTma(a, enc, tunedVariant(kFamThermoTma, enc, a.K, a.X, a.Y, a.Z, 0), s);
      if (rc != MKF_ERR_UNSUPPORTED) { return rc; }
   }
#endif
   itemGrid(a, tunedDepth(kFamThermo, enc, a.K, a.X, a.Y, a.Z,
                          sizeDepth(THERMO_D, perPlane, a.Z, (long long)smCount() * kThItemsPerSM)));
   const bool ge = a.rankHi != 0, inner = innerTiles(a, enc);
   if (enc == ENC_F32) { return ge ? launchThermoG<float, true>(a, inner, s) : launchThermoG<float, false>(a, inner, s); }
   return ge ? launchThermoG<double, true>(a, inner, s) : launchThermoG<double, false>(a, inner, s);
}

}  // namespace mkf
