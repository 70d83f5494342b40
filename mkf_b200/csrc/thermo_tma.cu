// thermo_tma.cu - the rank-table counting kernel with plane tiles staged by TMA, for 3..16
// thresholds of one relation (< <= > >=) on fields whose rows start on 16-byte boundaries.
//
// The method is thermo.cu's (sorted thresholds: an element's K map bits are a thermometer, found
// as a rank through a table over order-preserving keys; a cell is all-ones below its smallest
// corner rank, all-zeros from its largest, and mixed codes exist only in between), with the data
// movement and the per-cell arithmetic rebuilt for the B200:
//  * Each warp owns a ring of plane tiles in shared memory (34 or 36 x positions, 9 rows) filled
//    by cp.async.bulk.tensor (TMA) ahead of the plane it counts; an element is one shared-memory
//    load at a fixed offset, with no per-row address arithmetic, and the next plane's copy is in
//    flight while the current one is counted. The tensor map covers this GPU's own field only; no
//    load uses cluster multicast. Every wait on a copy has a poll limit (mkfKernelFaults).
//  * With K <= 16 an element's thermometer T (bits k < rank) and its complement fit one word,
//    V = T | ~T << 16. AND over a cell's eight corners gives C = T(min) | ~T(max) << 16 in three
//    logic operations per cell (x pair, face, cell); popc(C) = 16 - (max - min) is the number of
//    thresholds the cell does not cross and popc of the low half is its smallest rank.
//  * All-ones counts cost no per-cell work: the three code slots add one count each to rows rmin,
//    rmin + 1 and rmin + 2 (real codes or discarded 0s), so the row totals give, by a recurrence at
//    the flush, the number of cells of each smallest rank; the cells all-ones for threshold k are
//    those whose smallest rank exceeds k.
//  * Mixed codes for k = min, min + 1, min + 2 come from two bit-planes of the corner ranks
//    relative to min; each goes to the shared [K][257] histogram with an unpredicated atomic whose
//    address is the code's top byte masked in place plus the row. Where the cell crosses q or
//    fewer thresholds the code of slot q is 0, and those counts land in bins the flush skips (and
//    in discard rows past K). Cells crossing four or more thresholds (about 1 in 100 on a smooth
//    field with 16 thresholds) are queued, per lane with one store and no warp vote; the warp
//    drains the lanes' queues together, 32 cells at a time, taking back their three slot counts
//    and counting every code they have.
// Masked cells (lanes and rows outside the item) enter C as all ones: they cross nothing, land in
// smallest-rank row 16, and are subtracted from the all-ones counts at the flush.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include "thermo.cuh"
#include "tma.cuh"

namespace mkf {

// Kernel variants (the CTA shape, the histogram privatisation and the wide-cell queue mkfTune
// chooses among; 0 is the default): warps per CTA (one CTA per SM), ring stages for FP64 / FP32
// tiles, histogram copies (lane parity picks the copy; one copy halves that shared memory), queue
// kind for the cells crossing four or more thresholds (1: one queue per lane, appended without a
// warp vote and drained by the whole warp; 0: one queue per warp, appended through a ballot).
// Measured on 512^3 Gaussian fields: the per-lane queue is 4-16 % faster for 5-12 thresholds and
// even at 16 (where more cells are wide); 16 warps with 3 stages need the warp queue's smaller
// shared memory.
struct TmaVariant
{
   int warps, stagesF64, stagesF32, copies, laneQueue;
};
static constexpr TmaVariant kTmVariants[kTmNumVariants] = {{20, 2, 3, 2, 1}, {16, 3, 4, 2, 0}, {20, 2, 3, 1, 1},
                                                           {20, 2, 3, 2, 0}};
static constexpr int kTmRows = 9;           // rows of a plane tile: 8 row pairs
// wide-cell queue entries per warp: a plane adds at most 8 x 31, drained once 32 are waiting (plus
// one discard entry)
static constexpr int kTmQueue = 32 + 8 * 31;  // drained after a plane once 32 are waiting
// per-lane queue: entries per lane (a plane adds at most 8; drained after a plane once a lane
// holds more than kTmLaneQ - 8), entry q of a lane at q * 32 + lane. 14 is what the 227 KB of
// shared memory leaves room for next to the FP64 ring (12 measured 1 % slower: more drains)
static constexpr int kTmLaneQ = 14;
static constexpr int kTmMaxK = 16;          // thresholds a 16-bit thermometer holds
static constexpr int kTmMaxDepth = kThMaxDepth;  // planes per work item

// Element type and variant geometry: tile width (x positions, a multiple of 16 bytes that covers
// 32 lanes plus the alignment shift of the tile's first x), stages in the ring, bytes per stage.
template <typename T, int V = 0>
struct TmaGeom
{
   static constexpr int BX = sizeof(T) == 8 ? 34 : 36;
   static constexpr int ALIGN = 16 / (int)sizeof(T);  // x coordinates of a TMA tile: multiples of this
   static constexpr int WARPS = kTmVariants[V].warps;
   static constexpr int STAGES = sizeof(T) == 8 ? kTmVariants[V].stagesF64 : kTmVariants[V].stagesF32;
   static constexpr int COPIES = kTmVariants[V].copies;
   static constexpr int BYTES = BX * kTmRows * (int)sizeof(T);   // bytes one TMA copy writes
   static constexpr int PITCH = (BYTES + 127) / 128 * 128;       // stage stride
   static constexpr bool LANEQ = kTmVariants[V].laneQueue != 0;
   static constexpr int QWORDS = LANEQ ? kTmLaneQ * 32 : kTmQueue + 1;  // queue entries per warp
};

// Set when a wait of this kernel ran out of polls (never in a correct run); read by mkfKernelFaults.
__device__ unsigned gTmaFault;

// Histogram rows per copy: K real rows, then discard rows up to max(K, 16) + 2, where the slots
// of cells that cross fewer than three thresholds (and of masked cells, whose low half is 16 set
// bits) add their code-0 counts; the flush reads rows < K and codes 1..254 only.
__host__ __device__ constexpr int tmaCopyRows(int K) { return (K > 16 ? K : 16) + 3; }

// Exact rank of the element at p by binary search over the sorted thresholds (rare: ties of FP64
// high words, infinities, NaNs, huge magnitudes). Out of line: it runs only when the fast path
// flags an element, and one copy serves every row.
template <typename T, bool GE>
__device__ __noinline__ uint32_t exactRankAt(const T *p, const double *sTlo, const double *sThi, int K, uint32_t nanRank)
{
   const T v = *p;
   uint32_t r = 0;
#pragma unroll
   for (int s = 16; s >= 1; s >>= 1) {
      if (v > sTlo[r + s - 1]) { r += s; }
   }
   if (r > (uint32_t)K) { r = K; }
   if (GE) {
      while (r < (uint32_t)K && v >= sThi[r]) { ++r; }
   }
   return (v != v) ? nanRank : r;
}

// Word offset of a code held in the top byte of c (bits below masked off), added to base: one
// multiply-high with an addend.
__device__ __forceinline__ uint32_t codeAddr(uint32_t c, uint32_t base)
{
   uint32_t a;  // (the FMA pipe: the integer ALU pipe is the busier one)
   asm("mad.hi.u32 %0, %1, 1024, %2;" : "=r"(a) : "r"(c), "r"(base));
   return a;
}

// Count the queued wide cells (spread >= 4) of a warp: lane i takes entries i, i + 32, ...; an
// entry is the cell's two faces of corner ranks (bytes), its smallest rank and spread follow from
// them. The row loop added three codes for each of them from two rank bit-planes, which are wrong
// past a spread of 3; they are taken back here (the same formulas, minus one), then every code
// k = rmin .. rmax - 1 is counted: fixed formulas up to a spread of 7, one threshold at a time
// beyond (thermo.cu counts them the same way).
__device__ __forceinline__ void wideCell(const uint2 e, uint32_t hist32)
{
   {
      const uint32_t R0 = e.x, R1 = e.y;
      uint32_t rmin = 255, rmax = 0;
#pragma unroll
      for (int b = 0; b < 4; b++) {
         const uint32_t u = (R0 >> (8 * b)) & 255u, v = (R1 >> (8 * b)) & 255u;
         rmin = min(rmin, min(u, v));
         rmax = max(rmax, max(u, v));
      }
      const uint32_t spread = rmax - rmin;
      const uint32_t rowAddr = hist32 + rmin * (kHistRow * 4);
      const uint32_t D0 = R0 + rmin * 0xFEFEFEFFu, D1s = R1 * 16u + rmin * 0xEFEFEFF0u;
      {
         const uint32_t U = D0 | D1s;
         const uint32_t G0 = (U & 0x11111111u) * 0x01020408u, G1 = (U & 0x22222222u) * 0x00810204u;
         const uint32_t a0 = codeAddr((G0 | G1) & 0xFF000000u, rowAddr);
         const uint32_t a1 = codeAddr(G1 & 0xFF000000u, rowAddr);
         const uint32_t a2 = codeAddr((G0 & G1) & 0xFF000000u, rowAddr);
         asm volatile("red.shared.add.u32 [%0], -1;" ::"r"(a0) : "memory");
         asm volatile("red.shared.add.u32 [%0+%1], -1;" ::"r"(a1), "n"(kHistRow * 4) : "memory");
         asm volatile("red.shared.add.u32 [%0+%1], -1;" ::"r"(a2), "n"(kHistRow * 8) : "memory");
      }
      if (spread < 8) {
         const uint32_t b0 = gatherBits((D0 & 0x01010101u) | (D1s & 0x10101010u), 0x01020408u);
         const uint32_t b1 = gatherBits((D0 & 0x02020202u) | (D1s & 0x20202020u), 0x00810204u);
         const uint32_t b2 = gatherBits((D0 & 0x04040404u) | (D1s & 0x40404040u), 0x00408102u);
         redSharedAt<0>((b0 | b1 | b2) * 4u + rowAddr);
         redSharedAt<kHistRow * 4>((b1 | b2) * 4u + rowAddr);
         redSharedAt<kHistRow * 8>((b2 | (b1 & b0)) * 4u + rowAddr);
         redSharedAt<kHistRow * 12>(b2 * 4u + rowAddr);
         if (spread > 4) { redSharedAt<kHistRow * 16>((b2 & (b1 | b0)) * 4u + rowAddr); }
         if (spread > 5) { redSharedAt<kHistRow * 20>((b2 & b1) * 4u + rowAddr); }
         if (spread > 6) { redSharedAt<kHistRow * 24>((b2 & b1 & b0) * 4u + rowAddr); }
      } else {
         uint32_t C = 0x7F7F7F7Fu - rmin * 0x01010101u, addr = rowAddr;
         for (uint32_t k = 0; k < spread; ++k) {
            redShared(addr + (cellCode(R0, R1, C) << 2));
            C -= 0x01010101u;
            addr += kHistRow * 4;
         }
      }
      // row totals count every cell once in rows rmin .. rmin + 2: take back the codes counted in
      // rows rmin + 3 .. rmax - 1 from those rows' spare word
      for (uint32_t q = 3; q < spread; ++q) {
         asm volatile("red.shared.add.u32 [%0+%1], -1;" ::"r"(rowAddr + q * (kHistRow * 4)), "n"(256 * 4) : "memory");
      }
   }
}

// Drain a warp's queue of n entries: lane i takes entries i, i + 32, ...
__device__ __noinline__ void drainWide(const uint2 *q, int n, uint32_t hist32)
{
   __syncwarp();
   for (int i = threadIdx.x & 31; i < n; i += 32) { wideCell(q[i], hist32); }
   __syncwarp();
}

// Drain the per-lane queues of a warp (qw: the warp's first entry; entry q of lane l at
// q * 32 + l; n: this lane's entries), 32 entries per round whatever their owners: entry g of the
// warp (in lane order) belongs to the last lane whose exclusive prefix of counts is <= g, found
// by a binary search over the lanes' prefixes. Inline (measured 1 % faster than a call).
__device__ __forceinline__ void drainLanes(const uint2 *qw, int n, uint32_t hist32)
{
   __syncwarp();  // (orders the other lanes' queue stores before these loads)
   const int lane = threadIdx.x & 31;
   int incl = n;
#pragma unroll
   for (int d = 1; d < 32; d <<= 1) {
      const int t = __shfl_up_sync(FULL, incl, d);
      if (lane >= d) { incl += t; }
   }
   const int excl = incl - n, total = __shfl_sync(FULL, incl, 31);
   for (int base = 0; base < total; base += 32) {
      const int g = base + lane;
      int owner = 0;
#pragma unroll
      for (int s = 16; s >= 1; s >>= 1) {
         const int e = __shfl_sync(FULL, excl, owner + s);
         if (e <= g) { owner += s; }
      }
      const int q = g - __shfl_sync(FULL, excl, owner);
      if (g < total) { wideCell(qw[32 * q + owner], hist32); }
   }
   __syncwarp();
}

// Geometry of one work item: 31 x positions of cells, 8 row pairs, up to D planes of cells.
struct TmItem
{
   int xa, xoff;     // tile x (a multiple of ALIGN) and this item's first lane column in it
   int y0, z0, nPln; // tile rows y0 .. y0 + 8, planes z0 .. z0 + nPln
   uint32_t rowsOK;  // bit j: this lane counts row pair j
   unsigned cells;   // cells the item counts (warp total)
};

template <int ALIGN>
__device__ __forceinline__ TmItem itemOf(const FusedArgs &a, long long it, int lane)
{
   TmItem m;
   const int ix = (int)(it % a.nSegX);
   const long long rest = it / a.nSegX;
   const int iy = (int)(rest % a.nTileY);
   const int iz = (int)(rest / a.nTileY);
   const int xs = 31 * ix, ys = 8 * iy;
   const int xe = min(xs + 31, a.X - 1), ye = min(ys + 8, a.Y - 1);
   const int x0 = min(xs, a.X - 32);  // lanes at x0 + lane, all inside the field
   m.xa = x0 & ~(ALIGN - 1);
   m.xoff = x0 - m.xa;
   m.y0 = min(ys, a.Y - 9);
   m.z0 = a.D * iz;
   m.nPln = min(a.D, a.Z - 1 - m.z0);
   const int jlo = ys - m.y0, jhi = ye - m.y0;
   const bool laneIn = x0 + lane >= xs && x0 + lane < xe;
   m.rowsOK = laneIn ? (((1u << jhi) - 1u) & ~((1u << jlo) - 1u)) : 0u;
   m.cells = (unsigned)(xe - xs) * (unsigned)(jhi - jlo) * (unsigned)m.nPln;
   return m;
}

template <typename T, bool GE, int CMAX, int V>
__global__ void __launch_bounds__(kTmVariants[V].warps * 32, 1)
    thermoTmaBPFD(const __grid_constant__ FusedArgs a, const __grid_constant__ CUtensorMap tm)
{
   using G = TmaGeom<T, V>;
   constexpr int kTmWarps = G::WARPS, kHistCopies = G::COPIES;
   constexpr int W = sizeof(T) / 4;   // 32-bit words per element; the ranked word is the last
   constexpr int S = G::STAGES;
   __shared__ ThermoShared Sh;
   __shared__ alignas(8) uint64_t bars[kTmWarps][G::STAGES];
   __shared__ uint32_t rowTot[kTmMaxK + 1];
   extern __shared__ __align__(128) unsigned char dsm[];
   const int K = a.K;
   const int copyRows = tmaCopyRows(K);
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   uint32_t *hist = reinterpret_cast<uint32_t *>(dsm);
   const size_t histBytes = ((size_t)copyRows * kHistRow * kHistCopies * 4 + 127) / 128 * 128;
   // the ring starts on a 128-byte boundary (TMA destination), whatever the dynamic base's alignment
   // (offset from dsm, so that the compiler keeps these pointers in the shared window)
   const uint32_t histEnd = (uint32_t)__cvta_generic_to_shared(dsm) + (uint32_t)histBytes;
   unsigned char *ring = dsm + histBytes + ((128u - (histEnd & 127u)) & 127u);
   uint2 *queue = reinterpret_cast<uint2 *>(ring + (size_t)kTmWarps * S * G::PITCH) + warp * G::QWORDS;

   if (lane == 0) {
      for (int s = 0; s < S; s++) { mbarInit((uint32_t)__cvta_generic_to_shared(&bars[warp][s]), 1); }
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   ctaSetup(a, Sh, hist, copyRows, kHistCopies);  // (its barriers also order the mbarrier set-up)

   const uint32_t ringW = (uint32_t)__cvta_generic_to_shared(ring) + (uint32_t)(warp * S * G::PITCH);
   const uint32_t bar0 = (uint32_t)__cvta_generic_to_shared(&bars[warp][0]);
   const uint32_t histBase = (uint32_t)__cvta_generic_to_shared(hist);
   const uint32_t hist32 = histBase + (uint32_t)((lane & (kHistCopies - 1)) * copyRows * kHistRow) * 4u;
   const uint32_t nanRank = a.nanRank;
   const uint32_t lanesBelow = (1u << lane) - 1u;
   const long long nw = (long long)gridDim.x * kTmWarps;
   const long long first = (long long)blockIdx.x * kTmWarps + warp;

   // producer cursor (every lane tracks it; lane 0 issues): item, plane, tile coordinates
   long long pIt = first;
   int pP = 0, pX = 0, pY = 0, pZ = 0, pN = -1;
   if (pIt < a.nItems) {
      const TmItem m = itemOf<G::ALIGN>(a, pIt, lane);
      pX = m.xa; pY = m.y0; pZ = m.z0; pN = m.nPln;
   }
   uint32_t gp = 0;  // planes issued by this warp
   auto issue = [&]() {
      if (pIt >= a.nItems) { return; }
      if (lane == 0) {
         const uint32_t st = gp % S;
         tmaTile3D(&tm, ringW + st * G::PITCH, bar0 + 8u * st, pX, pY, pZ + pP, G::BYTES);
      }
      ++gp;
      if (++pP > pN) {
         pIt += nw;
         pP = 0;
         if (pIt < a.nItems) {
            const TmItem m = itemOf<G::ALIGN>(a, pIt, lane);
            pX = m.xa; pY = m.y0; pZ = m.z0; pN = m.nPln;
         }
      }
   };
   for (int s = 0; s + 1 < S; s++) { issue(); }

   uint32_t g = 0;  // planes consumed by this warp
   bool fault = false;
   // wait for plane g's tile, rank the lane's column (9 rows), refill the stage of plane g - 1
   auto plane = [&](int xoff, uint32_t (&r)[kTmRows]) -> bool {
      const uint32_t st = g % S;
      // (the warp leaves together: every lane's wait must have seen the copy)
      if (!__all_sync(FULL, mbarWait(bar0 + 8u * st, (g / S) & 1u))) { return false; }
      // this lane's column of the plane tile (the mbarrier wait orders these loads after the copy)
      const T *col = reinterpret_cast<const T *>(ring + (size_t)(warp * S + (int)st) * G::PITCH) + xoff + lane;
      const uint32_t *colW = reinterpret_cast<const uint32_t *>(col) + (W - 1);
      bool slow = false;   // a FP64 high word equal to a threshold's
      uint32_t rOr = 0;    // slow-path buckets rank above 32
#pragma unroll
      for (int j = 0; j < kTmRows; ++j) {
         const uint32_t key = sortKey(colW[j * G::BX * W]);
         const uint32_t r0 = Sh.lut[key >> kLutShift];
         const uint32_t cand = Sh.key[r0];
         uint32_t rr = r0 + (GE ? (key >= cand) : (key > cand));
         bool tie = key == cand;
#pragma unroll
         for (int c = 1; c < CMAX; ++c) {
            const uint32_t cc = Sh.key[r0 + c];
            rr += GE ? (key >= cc) : (key > cc);
            tie = tie | (key == cc);
         }
         if (W == 2) { slow = slow | tie; }
         rOr |= rr;
         r[j] = rr;
      }
      static_assert(kSlowBucket >= 32 && kTmMaxK < 32, "slow buckets rank at 32 or more");
      slow = slow | (rOr >= 32u);
      if (__any_sync(FULL, slow)) {
         if (slow) {
#pragma unroll
            for (int j = 0; j < kTmRows; ++j) { r[j] = exactRankAt<T, GE>(col + j * G::BX, Sh.tlo, Sh.thi, K, nanRank); }
         }
      }
      __syncwarp();
      issue();  // refill the stage of the previous plane (read by every lane by now)
      ++g;
      return true;
   };
   // thermometer of a rank and its complement: T | ~T << 16, T = bits [0, r); the x neighbour's
   // is formed here from its shuffled rank (one shuffle per row, not two: shuffles share the pipe
   // of the tile loads and the histogram atomics; measured 1 % faster)
   auto thermoV = [](uint32_t r) { return thermo(r) * 0xFFFF0001u + 0xFFFF0000u; };

   unsigned long long cells = 0;
   uint32_t masked = 0;  // masked cells counted (in smallest-rank row 16)
   int qn = 0;           // wide cells queued by the warp (warp queue)
   // per-lane queue: shared address of this lane's first entry and of its next one
   const uint32_t qLane0 = (uint32_t)__cvta_generic_to_shared(queue) + (uint32_t)lane * 8u;
   uint32_t qa = qLane0;
   for (long long it = first; it < a.nItems; it += nw) {
      const TmItem m = itemOf<G::ALIGN>(a, it, lane);
      cells += m.cells;
      masked += (8u - (uint32_t)__popc(m.rowsOK)) * (uint32_t)m.nPln;
      uint32_t sF[8], sV[8];  // previous plane: face ranks (bytes), face thermometer AND
      {
         uint32_t r[kTmRows];
         if (!plane(m.xoff, r)) { fault = true; break; }
         uint32_t rR = __shfl_down_sync(FULL, r[0], 1);
         uint32_t Vt = thermoV(r[0]), VR = thermoV(rR);
         uint32_t ePrev = rR * 256u + r[0], Pprev = Vt & VR;
#pragma unroll
         for (int j = 0; j < 8; ++j) {
            rR = __shfl_down_sync(FULL, r[j + 1], 1);
            Vt = thermoV(r[j + 1]);
            VR = thermoV(rR);
            const uint32_t e = rR * 256u + r[j + 1], P = Vt & VR;
            sF[j] = e * 65536u + ePrev;
            sV[j] = P & Pprev;
            ePrev = e;
            Pprev = P;
         }
      }
      for (int p = 1; p <= m.nPln; ++p) {
         uint32_t r[kTmRows];
         if (!plane(m.xoff, r)) { fault = true; break; }
         uint32_t rR = __shfl_down_sync(FULL, r[0], 1);
         uint32_t Vt = thermoV(r[0]), VR = thermoV(rR);
         uint32_t ePrev = rR * 256u + r[0];
         uint32_t Pprev = Vt & VR;
#pragma unroll
         for (int j = 0; j < 8; ++j) {
            rR = __shfl_down_sync(FULL, r[j + 1], 1);
            Vt = thermoV(r[j + 1]);
            VR = thermoV(rR);
            const uint32_t e = rR * 256u + r[j + 1];
            const uint32_t P = Vt & VR;
            const uint32_t fc = e * 65536u + ePrev;  // face ranks: (x,y) (x+1,y) (x,y+1) (x+1,y+1)
            const uint32_t F = P & Pprev;
            const uint32_t nvm = ((m.rowsOK >> j) & 1u) - 1u;  // all ones for a masked cell
            const uint32_t C = (F & sV[j]) | nvm;
            const uint32_t pc = __popc(C), rmin = __popc(C & 0xFFFFu);
            const uint32_t R0 = sF[j], R1 = fc;
            const uint32_t D0 = R0 + rmin * 0xFEFEFEFFu;         // R0 - rmin per byte
            const uint32_t D1s = R1 * 16u + rmin * 0xEFEFEFF0u;  // (R1 - rmin per byte) << 4
            // bits 0 and 1 of each corner's rank - rmin (below 4 unless the cell is wide): byte b
            // of U holds face z's corner in bits 0-1 and face z + 1's in bits 4-5
            const uint32_t U = D0 | D1s;
            const uint32_t G0 = (U & 0x11111111u) * 0x01020408u;
            const uint32_t G1 = (U & 0x22222222u) * 0x00810204u;
            const uint32_t rowAddr = hist32 + rmin * (kHistRow * 4);
            // codes k = rmin + q mark the corners with rank - rmin > q: b0 | b1, b1, b0 & b1 (the
            // top bytes of G0, G1); a code is 0 where the cell crosses q or fewer thresholds, and
            // such counts land in discard bins
            redSharedAt<0>(codeAddr((G0 | G1) & 0xFF000000u, rowAddr));
            redSharedAt<kHistRow * 4>(codeAddr(G1 & 0xFF000000u, rowAddr));
            redSharedAt<kHistRow * 8>(codeAddr((G0 & G1) & 0xFF000000u, rowAddr));
            // cells crossing 4 or more thresholds join the queue
            if (G::LANEQ) {
               // a predicated 64-bit store and a predicated advance, no branch (measured against
               // two 32-bit stores: 2 % faster; against skipping the stores when no lane of the
               // warp has a wide cell: 3-4 % faster, even with 8 thresholds where none has)
               asm volatile(
                   "{\n\t.reg .pred w;\n\t"
                   "setp.lt.u32 w, %1, 13;\n\t"
                   "@w st.shared.v2.u32 [%0], {%2, %3};\n\t"
                   "@w add.u32 %0, %0, 256;\n\t}"
                   : "+r"(qa)
                   : "r"(pc), "r"(R0), "r"(R1)
                   : "memory");
            } else {
               // every lane stores (the others into the discard entry), so the row body has no branch
               const bool wide = pc < 13u;
               const uint32_t wb = __ballot_sync(FULL, wide);
               queue[wide ? qn + __popc(wb & lanesBelow) : kTmQueue] = make_uint2(R0, R1);
               qn += __popc(wb);
            }
            sF[j] = fc;
            sV[j] = F;
            ePrev = e;
            Pprev = P;
         }
         if (G::LANEQ) {
            if (__any_sync(FULL, qa > qLane0 + (kTmLaneQ - 8) * 256u)) {
               drainLanes(queue, (int)((qa - qLane0) >> 8), hist32);
               qa = qLane0;
            }
         } else if (qn >= 32) {
            drainWide(queue, qn, hist32);
            qn = 0;
         }
      }
      if (fault) { break; }
   }
   // the queue holds ranks only (no item coordinates): it is drained when full and once here
   if (G::LANEQ) {
      if (__any_sync(FULL, qa != qLane0)) { drainLanes(queue, (int)((qa - qLane0) >> 8), hist32); }
   } else if (qn > 0) {
      drainWide(queue, qn, hist32);
   }
   if (fault) {
      if (lane == 0) { atomicOr(&gTmaFault, 1u); }
      // let the copies this warp started finish before its shared memory is released
      for (uint32_t q = g; q < gp; ++q) { mbarWait(bar0 + 8u * (q % S), (q / S) & 1u); }
   }
   if (lane == 0 && cells) { atomicAdd(&Sh.cells, cells); }
   masked = __reduce_add_sync(FULL, masked);  // (per lane: its own masked row pairs)
   if (lane == 0 && masked) { atomicAdd(&Sh.ones[MKF_MAX_THRESH - 1], masked); }
   __syncthreads();
   // All-ones counts. Every cell counted once in each of rows rmin, rmin + 1, rmin + 2 (a code, a
   // discarded 0, or for wide cells the drain's corrections), so row r's total over all 257 words
   // is N[r] + N[r-1] + N[r-2], N[r] the cells whose smallest rank is r; the cells all-ones for
   // threshold k are those with rmin > k, less the masked cells (rmin 16).
   for (int r = warp; r <= kTmMaxK; r += kTmWarps) {
      uint32_t t = 0;
      for (int c = lane; c < kHistRow; c += 32) {
#pragma unroll
         for (int q = 0; q < kHistCopies; ++q) { t += hist[(q * copyRows + r) * kHistRow + c]; }
      }
      t = __reduce_add_sync(FULL, t);
      if (lane == 0) { rowTot[r] = t; }
   }
   __syncthreads();
   if (threadIdx.x == 0) {
      uint32_t n1 = 0, n2 = 0, nr[kTmMaxK + 1];
      for (int r = 0; r <= kTmMaxK; r++) {
         nr[r] = rowTot[r] - n1 - n2;
         n2 = n1;
         n1 = nr[r];
      }
      uint32_t above = nr[kTmMaxK] - Sh.ones[MKF_MAX_THRESH - 1];  // rmin > k, from k = 15 down
      for (int k = kTmMaxK - 1; k >= 0; k--) {
         if (k < K) { Sh.ones[k] = above; }
         above += nr[k];
      }
   }
   ctaFlush(a, Sh, hist, copyRows, kHistCopies);
}

// ---------------------------------------------------------------- host

template <typename T, int V>
static size_t tmaDynBytes(int K)
{
   using G = TmaGeom<T, V>;
   const size_t histBytes = ((size_t)tmaCopyRows(K) * kHistRow * G::COPIES * 4 + 127) / 128 * 128;
   return histBytes + 128 + (size_t)G::WARPS * G::STAGES * G::PITCH + (size_t)G::WARPS * G::QWORDS * sizeof(uint2);
}

static PFN_cuTensorMapEncodeTiled_v12000 encodeFn()
{
   static std::once_flag once;
   static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
   std::call_once(once, [] {
      void *p = nullptr;
      cudaDriverEntryPointQueryResult q;
      if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
          q == cudaDriverEntryPointSuccess) {
         fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
      } else {
         cudaGetLastError();
      }
   });
   return fn;
}

bool encodeField3D(CUtensorMap *tm, const void *base, int enc, int X, int Y, int Z, int64_t sy, int64_t sz, int boxX, int boxY,
                   bool promote256)
{
   const cuuint64_t esz = enc == ENC_F32 ? 4 : 8;
   if (!encodeFn() || ((uintptr_t)base % 16) != 0 || (sy * (int64_t)esz) % 16 != 0 || (sz * (int64_t)esz) % 16 != 0) {
      return false;
   }
   const cuuint64_t dims[3] = {(cuuint64_t)X, (cuuint64_t)Y, (cuuint64_t)Z};
   const cuuint64_t strides[2] = {(cuuint64_t)sy * esz, (cuuint64_t)sz * esz};
   const cuuint32_t box[3] = {(cuuint32_t)boxX, (cuuint32_t)boxY, 1};
   const cuuint32_t estr[3] = {1, 1, 1};
   return encodeFn()(tm, enc == ENC_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                     const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, promote256 ? CU_TENSOR_MAP_L2_PROMOTION_L2_256B : CU_TENSOR_MAP_L2_PROMOTION_NONE,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

unsigned thermoTmaFaults(bool clear)
{
   unsigned v = 0;
   if (cudaMemcpyFromSymbol(&v, gTmaFault, sizeof(v)) != cudaSuccess) { cudaGetLastError(); return 0; }
   if (clear && v) {
      const unsigned z = 0;
      cudaMemcpyToSymbol(gTmaFault, &z, sizeof(z));
   }
   return v;
}

template <typename T, bool GE, int CMAX, int V>
static int launchTmaT(const FusedArgs &a, const CUtensorMap &tm, cudaStream_t s)
{
   using G = TmaGeom<T, V>;
   static std::atomic<int> occ[kTmMaxK + 1];
   auto kern = thermoTmaBPFD<T, GE, CMAX, V>;
   const size_t smem = tmaDynBytes<T, V>(a.K);
   const int blocksPerSM = cachedOccupancy(occ[a.K], kern, G::WARPS * 32, smem, tmaDynBytes<T, V>(kTmMaxK));
   long long grid = (a.nItems + G::WARPS - 1) / G::WARPS;
   const long long cap = (long long)smCount() * blocksPerSM;
   if (grid > cap) { grid = cap; }
   if (grid < 1) { grid = 1; }
   kern<<<(unsigned)grid, G::WARPS * 32, smem, s>>>(a, tm);
   return cudaFail(cudaGetLastError(), "thermoTmaBPFD launch");
}

// Thresholds sharing rank-table buckets (four candidates) take the default variant only.
template <typename T, bool GE>
static int launchTmaG(const FusedArgs &a, const CUtensorMap &tm, int variant, cudaStream_t s)
{
   if (a.lutC > 1) { return launchTmaT<T, GE, 4, 0>(a, tm, s); }
   switch (variant) {
      case 1: return launchTmaT<T, GE, 1, 1>(a, tm, s);
      case 2: return launchTmaT<T, GE, 1, 2>(a, tm, s);
      case 3: return launchTmaT<T, GE, 1, 3>(a, tm, s);
      default: return launchTmaT<T, GE, 1, 0>(a, tm, s);
   }
}

bool tmaRowsAligned(const FusedArgs &a, int enc)
{
   const int64_t esz = enc == ENC_F32 ? 4 : 8;
   return a.K > 2 && a.K <= kTmMaxK && a.sx == 1 && a.X >= 32 && a.Y >= 9 && a.Z >= 2 && ((uintptr_t)a.f % 16) == 0 &&
          (a.sy * esz) % 16 == 0 && (a.sz * esz) % 16 == 0 && a.sy >= a.X && a.sz >= a.sy * a.Y && encodeFn() != nullptr;
}

bool thermoTmaEligible(const FusedArgs &a, int enc)
{
   return tmaRowsAligned(a, enc) && a.lutC >= 1 && a.D >= 1 && a.D <= kTmMaxDepth;
}

// a.tkey / a.lutC filled (prepareKeys) and the item grid set for 8-row items (itemGrid).
int launchThermoTma(const FusedArgs &a, int enc, int variant, cudaStream_t s)
{
   if (!thermoTmaEligible(a, enc)) { return MKF_ERR_UNSUPPORTED; }
   const bool f32 = enc == ENC_F32;
   CUtensorMap tm;
   if (!encodeField3D(&tm, a.f, enc, a.X, a.Y, a.Z, a.sy, a.sz, f32 ? TmaGeom<float>::BX : TmaGeom<double>::BX, kTmRows)) {
      return MKF_ERR_UNSUPPORTED;
   }
   const bool ge = a.rankHi != 0;
   if (f32) { return ge ? launchTmaG<float, true>(a, tm, variant, s) : launchTmaG<float, false>(a, tm, variant, s); }
   return ge ? launchTmaG<double, true>(a, tm, variant, s) : launchTmaG<double, false>(a, tm, variant, s);
}

}  // namespace mkf

MKF_API int mkfKernelFaults(int clear)
{
   const unsigned v = mkf::thermoTmaFaults(clear != 0);
   return (int)v;
}
