// words.cu - fused counting kernel for one or two thresholds of any relations, or up to six of one
// relation, word-parallel (optionally with the field's moments per map value from the same read).
//
// With few thresholds the per-element cost must be a handful of instructions, so cells are
// handled 32 at a time as bit words, as the original's packed binary map does
// (bpfdCUDA.cuh:41-118), but without storing the map. A warp item is a tile of 32 x positions
// (31 cells), 32 rows (31 row pairs) and D planes, walked plane by plane:
//  * load: lane = x; the warp issues the 32 rows' coalesced loads at once;
//  * pack: one ballot per row and threshold gives that row's 32-bit map word; lane r keeps row r's;
//  * count: lane = row pair. A cell's eight corners are bits b and b+1 of four words (this lane's
//    row and the next lane's row, previous and current plane), so all-ones and all-zeros cells
//    are popcounts of ANDs and ORs of the words and their one-bit shifts; only mixed cells form
//    their 8-bit code, counted in a per-CTA shared histogram.
#include <cmath>
#include <cstring>
#include <type_traits>
#include "fused.cuh"

namespace mkf {

#ifndef WORDS_MINB_F32
#define WORDS_MINB_F32 4
#endif
// FP32 fields with one or two thresholds whose items lie inside the field and are at least
// kWdPfDepth planes deep load the next plane while counting the current one (two plane buffers in
// registers at 2 CTAs per SM, 128 registers). Measured: 1.55 x faster on a 1024^3 FP32 GRF with
// one threshold (0.70 vs 1.09 ms), 11 % on 512^3, 24 % on 1024 x 1024 x 512 plane waves; with three
// thresholds 10 % faster on a 512^3 GRF but even to 5 % slower on plane waves, and slower for
// shallow items (small fields) and in the batched kernel (7.5 -> 10.8 ms on 512 uneven fields),
// which therefore keep the single buffer at 3-4 CTAs per SM.
static constexpr int kWdPfDepth = 16;

static constexpr int kWdWarps = 8;
#ifndef WORDS_D
#define WORDS_D 32
#endif
static constexpr int kWdD = WORDS_D;  // default planes of cells per work item (WordTask::D)
// Untuned fields get at least this many work items per SM (the slab depth is halved until they
// do): measured on 256^3 to 512^3 fields, fewer items than ~0.6 of the resident warps leave SMs
// idle while deeper items win nothing.
static constexpr int kWdItemsPerSM = 20;

// Relation class of a threshold: every class is one comparison (NaN maps as the EQ bit says).
enum WordCls { kGT = 0, kGE = 1, kLT = 2, kLE = 3, kGEN = 4 };

template <typename T>
__device__ __forceinline__ uint32_t mapBit(T v, int cls, uint32_t m, T tlo, T thi)
{
   switch (cls) {
      case kGT: return v > tlo;
      case kGE: return !(v < thi);
      case kLT: return v < thi;
      case kLE: return !(v > tlo);
      default: {
         const uint32_t d = 1u - (uint32_t)(v < thi) + (uint32_t)(v > tlo);
         return (m >> d) & 1u;
      }
   }
}

// State of one warp item between planes: the previous plane's map words and the cell counts.
template <int KMAX>
struct WordCarry
{
   uint32_t pw[KMAX], pn[KMAX];  // previous plane: this lane's row word and the next row's
   uint32_t n0[KMAX], n1[KMAX];  // all-zeros and all-ones cells counted by this lane
};

// Load one plane's 32 x 32 tile (lane = x). INNER: every row of the tile lies inside the field
// and the row stride in bytes `syb` times 31 fits 32 bits, so each row address is one multiply-add
// on the plane pointer; otherwise rows past the field end repeat its last row (their cells are
// masked out when counted) and addresses are formed in 64 bits.
template <typename T, bool INNER>
__device__ __forceinline__ void loadPlane(T (&v)[32], const T *__restrict__ p, int64_t sy, uint32_t syb, int nRow)
{
#pragma unroll
   for (int r = 0; r < 32; r++) {
      if (INNER) {
         v[r] = __ldg((const T *)((const char *)p + (uint64_t)(syb * (uint32_t)r)));
      } else {
         v[r] = __ldg(p + (int64_t)min(r, nRow - 1) * sy);
      }
   }
}

// Map, pack and count one plane (see the file comment). `first`: no previous plane yet.
// `sRow` is the warp's 32-word transposition buffer per threshold.
template <typename T, int KMAX, int CLS0, int CLS1>
__device__ __forceinline__ void countPlane(const T (&v)[32], WordCarry<KMAX> &c, const uint32_t *m, const T *tlo,
                                           const T *thi, bool xin, int lane, uint32_t vm, bool first,
                                           uint32_t (*sRow)[32], uint32_t *sHist)
{
#pragma unroll
   for (int r = 0; r < 32; r++) {
#pragma unroll
      for (int k = 0; k < KMAX; k++) {
         const int cls = k == 0 ? CLS0 : CLS1;
         // every lane stores the same (warp-uniform) word
         sRow[k][r] = __ballot_sync(FULL, xin && mapBit<T>(v[r], cls, m[k], tlo[k], thi[k]));
      }
   }
   __syncwarp();
   uint32_t cw[KMAX];
#pragma unroll
   for (int k = 0; k < KMAX; k++) { cw[k] = sRow[k][lane]; }
   __syncwarp();
#pragma unroll
   for (int k = 0; k < KMAX; k++) {
      const uint32_t cn = __shfl_down_sync(FULL, cw[k], 1);
      if (!first) {
         const uint32_t a0 = c.pw[k], a1 = c.pn[k], a2 = cw[k], a3 = cn;
         const uint32_t all = a0 & (a0 >> 1) & a1 & (a1 >> 1) & a2 & (a2 >> 1) & a3 & (a3 >> 1) & vm;
         const uint32_t any = a0 | (a0 >> 1) | a1 | (a1 >> 1) | a2 | (a2 >> 1) | a3 | (a3 >> 1);
         c.n1[k] += __popc(all);
         c.n0[k] += __popc(vm & ~any);
         uint32_t mixed = vm & any & ~all;
         if (mixed) {
            // word j's bits b, b+1 go to code bits 2j, 2j+1: pre-shift j's word left by 2j as a
            // 64-bit (hi:lo) pair, so one funnel shift by b brings them into place
            const uint32_t l1 = a1 << 2, h1 = a1 >> 30, l2 = a2 << 4, h2 = a2 >> 28, l3 = a3 << 6, h3 = a3 >> 26;
            uint32_t *hk = sHist + k * 256;
            do {
               const int b = 31 - __clz(mixed);
               mixed ^= 1u << b;
               uint32_t code = (__funnelshift_r(l1, h1, b) & ~3u) | ((a0 >> b) & 3u);
               code = (__funnelshift_r(l2, h2, b) & ~15u) | (code & 15u);
               code = (__funnelshift_r(l3, h3, b) & ~63u) | (code & 63u);
               atomicAdd(hk + (code & 255u), 1u);
            } while (mixed);
         }
      }
      c.pw[k] = cw[k];
      c.pn[k] = cn;
   }
}

// Descriptive moments of the field by map value (the original's categorical CUDAImgMom,
// binMapCUDA.cuh:67-128): per threshold, the sum of f and of f^2 over the elements mapping to 0
// and to 1, in FP64. Every element is added once: an item owns the elements of its cells, and the
// items at the field's +x / +y / +z ends also the field's last column / row / plane.
template <int KMAX>
struct MomAcc
{
   double s[KMAX][2][2];
};

template <typename T, int KMAX>
__device__ __forceinline__ void addMoments(const T (&v)[32], MomAcc<KMAX> &acc, const uint32_t *m, const T *tlo,
                                           const T *thi, bool ownXZ, int y0, int ys, int ye, bool lastY, int Y)
{
#pragma unroll
   for (int r = 0; r < 32; r++) {
      const int y = y0 + r;
      const bool own = ownXZ && y < Y && ((y >= ys && y < ye) || (lastY && y == Y - 1));
      if (own) {
         const double d = (double)v[r];
         const double d2 = d * d;
#pragma unroll
         for (int k = 0; k < KMAX; k++) {
            const uint32_t b = mapBit<T>(v[r], kGEN, m[k], tlo[k], thi[k]);
            acc.s[k][b][0] += d;
            acc.s[k][b][1] += d2;
         }
      }
   }
}

// One warp counts work item `it` (31 x 31 cells, D planes) of field `a` into the CTA's histogram
// and all-zeros / all-ones totals. INNER: the field is at least 32 x 32 in x and y with a positive
// row stride below 2^32 / 31 bytes; edge tiles are then shifted back inside the field (their cells
// already counted by the neighbouring tile are masked out), so no load needs clamping.
// PF: the next plane's loads are issued before the current plane is counted (two plane buffers
// in registers, alternating; INNER fields without moments only).
template <typename T, int KMAX, int CLS0, int CLS1, bool INNER, bool MOM = false, bool PF = false>
__device__ __forceinline__ void wordItem(const WordTask &a, long long it, const T *tlo, const T *thi,
                                         uint32_t (*sRow)[32], uint32_t *sHist, unsigned long long (*sEnds)[2])
{
   const int lane = threadIdx.x & 31;
   const T *__restrict__ F = (const T *)a.f;
   const uint32_t syb = (uint32_t)(a.sy * (int64_t)sizeof(T));
   const int ix = (int)(it % a.nChunkX);
   const long long rest = it / a.nChunkX;
   const int iy = (int)(rest % a.nTileY);
   const int iz = (int)(rest / a.nTileY);
   // this item's cells: x in [xs, xe), y in [ys, ye), z in [z0, z0 + nPln)
   const int xs = 31 * ix, ys = 31 * iy, z0 = a.D * iz;
   const int xe = min(xs + 31, a.X - 1), ye = min(ys + 31, a.Y - 1);
   const int nPln = min(a.D, a.Z - 1 - z0);
   // tile origin: bit b of a word is x0 + b, lane l counts the row pair y0 + l
   const int x0 = INNER ? min(xs, a.X - 32) : xs;
   const int y0 = INNER ? min(ys, a.Y - 32) : ys;
   const int nRow = INNER ? 32 : min(32, a.Y - y0);
   const bool xin = INNER || x0 + lane < a.X;
   const T *base = F + (long long)(INNER ? x0 + lane : min(x0 + lane, a.X - 1)) * a.sx + (long long)y0 * a.sy +
                   (long long)z0 * a.sz;
   const uint32_t vm = (y0 + lane >= ys && y0 + lane < ye)
                          ? ((0xFFFFFFFFu >> (32 - (xe - x0))) & (0xFFFFFFFFu << (xs - x0)))
                          : 0u;
   WordCarry<KMAX> c;
#pragma unroll
   for (int k = 0; k < KMAX; k++) { c.n0[k] = c.n1[k] = 0; c.pw[k] = c.pn[k] = 0; }
   MomAcc<MOM ? KMAX : 1> acc;
   bool ownX = false, lastY = false, lastZ = false;
   if (MOM) {
      for (int k = 0; k < (MOM ? KMAX : 1); k++) { acc.s[k][0][0] = acc.s[k][0][1] = acc.s[k][1][0] = acc.s[k][1][1] = 0.0; }
      const int x = x0 + lane;
      ownX = x < a.X && ((x >= xs && x < xe) || (ix == a.nChunkX - 1 && x == a.X - 1));
      lastY = iy == a.nTileY - 1;
      lastZ = iz == a.nSlabZ - 1;
   }
   if (PF && INNER && !MOM) {
      T va[32], vb[32];
      loadPlane<T, INNER>(va, base, a.sy, syb, nRow);
      for (int p = 0; p <= nPln; p += 2) {
         if (p + 1 <= nPln) { loadPlane<T, INNER>(vb, base + (long long)(p + 1) * a.sz, a.sy, syb, nRow); }
         countPlane<T, KMAX, CLS0, CLS1>(va, c, a.m, tlo, thi, xin, lane, vm, p == 0, sRow, sHist);
         if (p + 1 > nPln) { break; }
         if (p + 2 <= nPln) { loadPlane<T, INNER>(va, base + (long long)(p + 2) * a.sz, a.sy, syb, nRow); }
         countPlane<T, KMAX, CLS0, CLS1>(vb, c, a.m, tlo, thi, xin, lane, vm, false, sRow, sHist);
      }
   } else {
      for (int p = 0; p <= nPln; ++p) {
         T v[32];
         loadPlane<T, INNER>(v, base + (long long)p * a.sz, a.sy, syb, nRow);
         if (MOM) {
            const bool ownZ = p < nPln || (lastZ && z0 + p == a.Z - 1);
            addMoments<T, MOM ? KMAX : 1>(v, acc, a.m, tlo, thi, ownX && ownZ, y0, ys, ye, lastY, a.Y);
         }
         countPlane<T, KMAX, CLS0, CLS1>(v, c, a.m, tlo, thi, xin, lane, vm, p == 0, sRow, sHist);
      }
   }
   if (MOM) {
#pragma unroll
      for (int k = 0; k < (MOM ? KMAX : 1); k++) {
#pragma unroll
         for (int q = 0; q < 4; q++) {
            double x = acc.s[k][q >> 1][q & 1];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) { x += __shfl_xor_sync(FULL, x, o); }
            if (lane == 0 && x != 0.0) { atomicAdd(a.mom + k * 4 + q, x); }
         }
      }
   }
#pragma unroll
   for (int k = 0; k < KMAX; k++) {
      const unsigned long long s0 = __reduce_add_sync(FULL, c.n0[k]);
      const unsigned long long s1 = __reduce_add_sync(FULL, c.n1[k]);
      if (lane == 0) {
         if (s0) { atomicAdd(&sEnds[k][0], s0); }
         if (s1) { atomicAdd(&sEnds[k][1], s1); }
      }
   }
}

// Add a CTA's counts of one field to its output rows (whole CTA, after a barrier): mixed codes as
// counted, 0 / 255 from the all-zeros / all-ones totals; with `complement` the map was counted
// negated, so code c belongs in bin 255 - c. Clears the counts for the next field.
template <int KMAX>
__device__ void flushWords(const WordTask &a, uint32_t *sHist, unsigned long long (*sEnds)[2])
{
   for (int i = threadIdx.x; i < a.K * 256; i += blockDim.x) {
      const int k = i >> 8, c = i & 255;
      unsigned long long v = sHist[i];
      if (c == 0) { v += sEnds[k][0]; }
      if (c == 255) { v += sEnds[k][1]; }
      const int cc = a.complement ? 255 - c : c;
      if (v) { atomicAdd((unsigned long long *)(a.out + (size_t)a.outRow[k] * 256 + cc), v); }
      sHist[i] = 0;
   }
   __syncthreads();
   if (threadIdx.x < KMAX * 2) { (&sEnds[0][0])[threadIdx.x] = 0; }
   __syncthreads();
}

// One launch counts K = KMAX thresholds of classes CLS0 (and CLS1), compile-time constants.
template <typename T, int KMAX, int CLS0, int CLS1, bool INNER, int MINB, bool MOM = false, bool PF = false>
__global__ void __launch_bounds__(kWdWarps * 32, MINB) wordBPFD(const __grid_constant__ WordTask a)
{
   __shared__ uint32_t sHist[KMAX * 256];
   __shared__ unsigned long long sEnds[KMAX][2];  // all-zeros, all-ones cells
   __shared__ uint32_t sRows[kWdWarps][KMAX][32];
   for (int i = threadIdx.x; i < KMAX * 256; i += blockDim.x) { sHist[i] = 0; }
   if (threadIdx.x < KMAX * 2) { (&sEnds[0][0])[threadIdx.x] = 0; }
   __syncthreads();

   T tlo[KMAX], thi[KMAX];
#pragma unroll
   for (int k = 0; k < KMAX; k++) {
      tlo[k] = (T)a.tlo[k];
      thi[k] = (T)a.thi[k];
   }
   const long long gw = (long long)blockIdx.x * kWdWarps + (threadIdx.x >> 5);
   const long long nw = (long long)gridDim.x * kWdWarps;
   uint32_t (*sRow)[32] = sRows[threadIdx.x >> 5];

   for (long long it = gw; it < a.nItems; it += nw) {
      wordItem<T, KMAX, CLS0, CLS1, INNER, MOM, PF>(a, it, tlo, thi, sRow, sHist, sEnds);
   }
   __syncthreads();
   flushWords<KMAX>(a, sHist, sEnds);
}

template <typename T, int KMAX, int CLS0, int CLS1, bool INNER>
static int launchWordsI(const WordTask &a, cudaStream_t s)
{
   constexpr bool PF = INNER && sizeof(T) == 4 && KMAX <= 2;
   if (PF && a.D >= kWdPfDepth) {
      static std::atomic<int> occPf{0};
      auto kern = wordBPFD<T, KMAX, CLS0, CLS1, INNER, 2, false, PF>;
      const int blocksPerSM = cachedOccupancy(occPf, kern, kWdWarps * 32, 0);
      long long grid = (a.nItems + kWdWarps - 1) / kWdWarps;
      const long long cap = (long long)smCount() * blocksPerSM;
      if (grid > cap) { grid = cap; }
      if (grid < 1) { grid = 1; }
      kern<<<(unsigned)grid, kWdWarps * 32, 0, s>>>(a);
      return cudaFail(cudaGetLastError(), "wordBPFD launch");
   }
   static std::atomic<int> occ{0};
   auto kern = wordBPFD<T, KMAX, CLS0, CLS1, INNER, (INNER && sizeof(T) == 4) ? (KMAX <= 2 ? WORDS_MINB_F32 : 3) : 2>;
   const int blocksPerSM = cachedOccupancy(occ, kern, kWdWarps * 32, 0);
   long long grid = (a.nItems + kWdWarps - 1) / kWdWarps;
   const long long cap = (long long)smCount() * blocksPerSM;
   if (grid > cap) { grid = cap; }
   if (grid < 1) { grid = 1; }
   kern<<<(unsigned)grid, kWdWarps * 32, 0, s>>>(a);
   return cudaFail(cudaGetLastError(), "wordBPFD launch");
}

template <typename T, int KMAX, int CLS0, int CLS1>
static int launchWordsT(const WordTask &a, cudaStream_t s)
{
   const int64_t syb = a.sy * (int64_t)sizeof(T);
   const bool inner = a.X >= 32 && a.Y >= 32 && syb > 0 && syb * 31 < (int64_t)1 << 32;
   return inner ? launchWordsI<T, KMAX, CLS0, CLS1, true>(a, s) : launchWordsI<T, KMAX, CLS0, CLS1, false>(a, s);
}

// 3 .. kWordMaxK thresholds of one relation class CLS.
template <typename T, int CLS>
static int dispatchK(const WordTask &a, cudaStream_t s)
{
   switch (a.K) {
      case 3: return launchWordsT<T, 3, CLS, CLS>(a, s);
      case 4: return launchWordsT<T, 4, CLS, CLS>(a, s);
#if WORDS_MAX_K >= 5
      case 5: return launchWordsT<T, 5, CLS, CLS>(a, s);
#endif
#if WORDS_MAX_K >= 6
      case 6: return launchWordsT<T, 6, CLS, CLS>(a, s);
#endif
      default: setError("word kernel: %d thresholds", a.K); return MKF_ERR_UNSUPPORTED;
   }
}

template <typename T>
static int dispatchWords(const WordTask &a, cudaStream_t s)
{
   if (a.K > 2) {  // one relation for all (checked by launchWords)
      switch (a.cls[0]) {
         case kGT: return dispatchK<T, kGT>(a, s);
         case kGE: return dispatchK<T, kGE>(a, s);
         case kLT: return dispatchK<T, kLT>(a, s);
         default: return dispatchK<T, kLE>(a, s);
      }
   }
   if (a.K == 2) {
      if (a.cls[0] == a.cls[1]) {
         switch (a.cls[0]) {
            case kGT: return launchWordsT<T, 2, kGT, kGT>(a, s);
            case kGE: return launchWordsT<T, 2, kGE, kGE>(a, s);
            case kLT: return launchWordsT<T, 2, kLT, kLT>(a, s);
            case kLE: return launchWordsT<T, 2, kLE, kLE>(a, s);
            default: break;
         }
      }
      return launchWordsT<T, 2, kGEN, kGEN>(a, s);
   }
   switch (a.cls[0]) {
      case kGT: return launchWordsT<T, 1, kGT, kGT>(a, s);
      case kGE: return launchWordsT<T, 1, kGE, kGE>(a, s);
      case kLT: return launchWordsT<T, 1, kLT, kLT>(a, s);
      case kLE: return launchWordsT<T, 1, kLE, kLE>(a, s);
      default: return launchWordsT<T, 1, kGEN, kGEN>(a, s);
   }
}

// Count a field for K = 1 or 2 thresholds (sorted or not; tlo/thi/masks per threshold, rows in
// outRow). Returns MKF_ERR_UNSUPPORTED for other K.
int launchWords(const FusedArgs &f, int enc, const uint32_t *masks, cudaStream_t s)
{
   if (f.K < 1 || f.K > kWordMaxK) { return MKF_ERR_UNSUPPORTED; }
   WordTask a;
   memset(&a, 0, sizeof(a));
   a.f = f.f;
   a.sx = f.sx; a.sy = f.sy; a.sz = f.sz;
   a.X = f.X; a.Y = f.Y; a.Z = f.Z;
   a.K = f.K;
   a.out = f.out;
   for (int k = 0; k < f.K; k++) {
      const uint32_t m = masks[k] & BMC_AL;
      a.m[k] = m;
      a.cls[k] = (m == BMC_GT) ? kGT : (m == (BMC_GT | BMC_EQ)) ? kGE : (m == BMC_LT) ? kLT : (m == (BMC_LT | BMC_EQ)) ? kLE : kGEN;
      a.tlo[k] = f.tlo[k];
      a.thi[k] = f.thi[k];
      a.outRow[k] = f.outRow[k];
   }
   if (f.K > 2) {  // more than two thresholds: one relation < <= > >= for all
      for (int k = 0; k < f.K; k++) {
         if (a.cls[k] != a.cls[0] || a.cls[k] == kGEN) { return MKF_ERR_UNSUPPORTED; }
      }
   }
   a.nChunkX = (a.X - 1 + 30) / 31;
   a.nTileY = (a.Y - 1 + 30) / 31;
   a.D = tunedDepth(kFamWords, enc, a.K, a.X, a.Y, a.Z,
                    sizeDepth(kWdD, (long long)a.nChunkX * a.nTileY, a.Z, (long long)smCount() * kWdItemsPerSM));
   a.nSlabZ = (a.Z - 1 + a.D - 1) / a.D;
   a.nItems = (long long)a.nChunkX * a.nTileY * a.nSlabZ;
   if (enc == ENC_F32) { return dispatchWords<float>(a, s); }
   return dispatchWords<double>(a, s);
}

// ---------------------------------------------------------------- counts and moments in one read

template <typename T, int KMAX, bool INNER>
static int launchMomentsI(const WordTask &a, cudaStream_t s)
{
   static std::atomic<int> occ{0};
   auto kern = wordBPFD<T, KMAX, kGEN, kGEN, INNER, 2, true>;
   const int blocksPerSM = cachedOccupancy(occ, kern, kWdWarps * 32, 0);
   long long grid = (a.nItems + kWdWarps - 1) / kWdWarps;
   const long long cap = (long long)smCount() * blocksPerSM;
   if (grid > cap) { grid = cap; }
   if (grid < 1) { grid = 1; }
   kern<<<(unsigned)grid, kWdWarps * 32, 0, s>>>(a);
   return cudaFail(cudaGetLastError(), "wordBPFD (moments) launch");
}

template <typename T>
static int dispatchMoments(const WordTask &a, bool inner, cudaStream_t s)
{
   if (a.K == 1) { return inner ? launchMomentsI<T, 1, true>(a, s) : launchMomentsI<T, 1, false>(a, s); }
   return inner ? launchMomentsI<T, 2, true>(a, s) : launchMomentsI<T, 2, false>(a, s);
}

int launchWordsMoments(const FusedArgs &f, int enc, const uint32_t *masks, double *mom, cudaStream_t s)
{
   if (f.K < 1 || f.K > 2 || f.X < 2 || f.Y < 2 || f.Z < 2) { return MKF_ERR_UNSUPPORTED; }
   WordTask a;
   memset(&a, 0, sizeof(a));
   a.f = f.f;
   a.sx = f.sx; a.sy = f.sy; a.sz = f.sz;
   a.X = f.X; a.Y = f.Y; a.Z = f.Z;
   a.K = f.K;
   a.out = f.out;
   a.mom = mom;
   for (int k = 0; k < f.K; k++) {
      a.m[k] = masks[k] & BMC_AL;
      a.cls[k] = kGEN;
      a.tlo[k] = f.tlo[k];
      a.thi[k] = f.thi[k];
      a.outRow[k] = f.outRow[k];
   }
   a.nChunkX = (a.X - 1 + 30) / 31;
   a.nTileY = (a.Y - 1 + 30) / 31;
   a.D = sizeDepth(kWdD, (long long)a.nChunkX * a.nTileY, a.Z, (long long)smCount() * kWdItemsPerSM);
   a.nSlabZ = (a.Z - 1 + a.D - 1) / a.D;
   a.nItems = (long long)a.nChunkX * a.nTileY * a.nSlabZ;
   const int64_t syb = a.sy * (enc == ENC_F32 ? 4 : 8);
   const bool inner = a.X >= 32 && a.Y >= 32 && syb > 0 && syb * 31 < ((int64_t)1 << 32);
   if (enc == ENC_F32) { return dispatchMoments<float>(a, inner, s); }
   return dispatchMoments<double>(a, inner, s);
}

// ---------------------------------------------------------------- many fields, one launch

// Batched instantiations (WordTask::variant): 0 one threshold ">", 1 one threshold ">=" (a "<" or
// "<=" threshold is counted as the complement of ">=" or ">"), 2 one threshold of another relation,
// 3 two thresholds; + 4 for fields whose edge items can be shifted inside (INNER).

// A CTA takes chunks of consecutive work items from a global counter; chunks never span fields.
// When the next chunk belongs to another field, the CTA adds its counts of the previous field to
// that field's output rows first. One kernel per element type, so that each keeps its register
// budget (FP32 tiles need more warps in flight per byte).
template <typename T, int MINB>
__global__ void __launch_bounds__(kWdWarps * 32, MINB) wordBatch(const __grid_constant__ WordBatchArgs b)
{
   __shared__ uint32_t sHist[2 * 256];
   __shared__ unsigned long long sEnds[2][2];
   __shared__ uint32_t sRows[kWdWarps][2][32];
   __shared__ WordTask F;
   __shared__ int sChunk;
   for (int i = threadIdx.x; i < 2 * 256; i += blockDim.x) { sHist[i] = 0; }
   if (threadIdx.x < 4) { (&sEnds[0][0])[threadIdx.x] = 0; }
   const int warp = threadIdx.x >> 5;
   uint32_t (*sRow)[32] = sRows[warp];
   int cur = -1;
   for (;;) {
      if (threadIdx.x == 0) { sChunk = (int)atomicAdd(b.counter, 1u); }
      __syncthreads();
      const int c = sChunk;
      __syncthreads();
      if (c >= b.nChunks) { break; }
      const BatchChunk ch = b.chunks[c];
      if (ch.field != cur) {
         if (cur >= 0) { flushWords<2>(F, sHist, sEnds); }
         const uint32_t *src = reinterpret_cast<const uint32_t *>(b.tasks + ch.field);
         for (int i = threadIdx.x; i < (int)(sizeof(WordTask) / 4); i += blockDim.x) {
            reinterpret_cast<uint32_t *>(&F)[i] = src[i];
         }
         __syncthreads();
         cur = ch.field;
      }
      T tlo[2], thi[2];
      tlo[0] = (T)F.tlo[0]; thi[0] = (T)F.thi[0];
      tlo[1] = (T)F.tlo[1]; thi[1] = (T)F.thi[1];
      for (long long it = ch.begin + warp; it < ch.end; it += kWdWarps) {
         switch (F.variant) {
            case 0: wordItem<T, 1, kGT, kGT, false>(F, it, tlo, thi, sRow, sHist, sEnds); break;
            case 1: wordItem<T, 1, kGE, kGE, false>(F, it, tlo, thi, sRow, sHist, sEnds); break;
            case 2: wordItem<T, 1, kGEN, kGEN, false>(F, it, tlo, thi, sRow, sHist, sEnds); break;
            case 3: wordItem<T, 2, kGEN, kGEN, false>(F, it, tlo, thi, sRow, sHist, sEnds); break;
            case 4: wordItem<T, 1, kGT, kGT, true>(F, it, tlo, thi, sRow, sHist, sEnds); break;
            case 5: wordItem<T, 1, kGE, kGE, true>(F, it, tlo, thi, sRow, sHist, sEnds); break;
            case 6: wordItem<T, 1, kGEN, kGEN, true>(F, it, tlo, thi, sRow, sHist, sEnds); break;
            default: wordItem<T, 2, kGEN, kGEN, true>(F, it, tlo, thi, sRow, sHist, sEnds); break;
         }
      }
   }
   if (cur >= 0) {
      __syncthreads();
      flushWords<2>(F, sHist, sEnds);
   }
}

// Fill a word task from a field with one or two varying thresholds (sorted rows and bounds in
// `f`, relation masks in `masks`): relation classes, the batched variant and the item grid.
void prepareWordTask(WordTask &a, int enc, int depth)
{
   int kind;
   for (int k = 0; k < a.K; k++) {
      const uint32_t m = a.m[k] & BMC_AL;
      a.cls[k] = (m == BMC_GT) ? kGT : (m == (BMC_GT | BMC_EQ)) ? kGE : (m == BMC_LT) ? kLT : (m == (BMC_LT | BMC_EQ)) ? kLE : kGEN;
   }
   a.complement = 0;
   if (a.K == 2) {
      kind = 3;
   } else {
      switch (a.cls[0]) {
         case kGT: kind = 0; break;
         case kGE: kind = 1; break;
         case kLT: kind = 1; a.complement = 1; break;  // f < t  is  !(f >= t)
         case kLE: kind = 0; a.complement = 1; break;  // f <= t is  !(f > t)
         default: kind = 2; break;
      }
   }
   const int64_t syb = a.sy * (enc == ENC_F32 ? 4 : 8);
   const bool inner = a.X >= 32 && a.Y >= 32 && syb > 0 && syb * 31 < ((int64_t)1 << 32);
   a.variant = kind + (inner ? 4 : 0);
   a.nChunkX = (a.X - 1 + 30) / 31;
   a.nTileY = (a.Y - 1 + 30) / 31;
   a.D = depth > 0 ? depth : kWdD;
   a.nSlabZ = (a.Z - 1 + a.D - 1) / a.D;
   a.nItems = (long long)a.nChunkX * a.nTileY * a.nSlabZ;
}

int launchWordsBatch(const WordBatchArgs &b, int enc, cudaStream_t s)
{
   static std::atomic<int> occ[2];
   const int e = enc == ENC_F32 ? 0 : 1;
   auto kern = e == 0 ? wordBatch<float, 3> : wordBatch<double, 2>;
   const int blocksPerSM = cachedOccupancy(occ[e], kern, kWdWarps * 32, 0);
   long long grid = (long long)smCount() * blocksPerSM;
   if (grid > b.nChunks) { grid = b.nChunks; }
   if (grid < 1) { grid = 1; }
   kern<<<(unsigned)grid, kWdWarps * 32, 0, s>>>(b);
   return cudaFail(cudaGetLastError(), "wordBatch launch");
}

}  // namespace mkf
