// noalloc.cu - pattern counts of a host field without any allocation by the library.
//
// mkfFieldBPFDHost stages the host field through device buffers that the library allocates
// (cudaMalloc) and keeps. Some callers cannot let a library allocate device memory: an in-situ
// analysis linked into a simulation whose device memory is owned by the simulation's own pool
// (cudaMalloc would take memory the pool has reserved, and implicitly synchronises the device in
// the middle of the simulation's overlapped streams), or a process that runs under a fixed
// device-memory budget. mkfFieldBPFDHostNoAlloc serves them: its scratch (the staging area for
// field slabs and the counts) lives in the file-scope device arrays below, which the CUDA runtime
// places in device memory when the module loads, so every GPU that loads this library holds
// them until the process exits.
//
// The arrays' names are host-side stand-ins, not device addresses: the host code resolves them
// with cudaGetSymbolAddress once per device (with that device current) and passes the resolved
// pointers to the copies and the counting kernel.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include "mkf_common.cuh"

#define MKF_NOALLOC_STAGE_BYTES ((size_t)32 << 20)
#define MKF_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char gNoAllocStage[MKF_NOALLOC_STAGE_BYTES];
static __device__ __align__(256) unsigned long long gNoAllocCounts[MKF_MAX_THRESH * 256];

namespace mkf {

struct NoAllocScratch
{
   bool ready = false;
   unsigned char *stage = nullptr;
   unsigned long long *counts = nullptr;
};
static NoAllocScratch gScratch[MKF_NOALLOC_MAX_DEVICES];
static std::mutex gScratchMu;

// Device addresses of the scratch arrays for the current device (resolved on the first call).
static int scratchForCurrentDevice(NoAllocScratch &out)
{
   int dev = 0;
   cudaError_t e = cudaGetDevice(&dev);
   if (e != cudaSuccess) { return cudaFail(e, "cudaGetDevice"); }
   if (dev < 0 || dev >= MKF_NOALLOC_MAX_DEVICES) {
      setError("mkfFieldBPFDHostNoAlloc: device %d out of range (max %d)", dev, MKF_NOALLOC_MAX_DEVICES);
      return MKF_ERR_UNSUPPORTED;
   }
   std::lock_guard<std::mutex> lock(gScratchMu);
   NoAllocScratch &s = gScratch[dev];
   if (!s.ready) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, gNoAllocStage);
      if (e != cudaSuccess) { return cudaFail(e, "cudaGetSymbolAddress(staging)"); }
      s.stage = (unsigned char *)p;
      e = cudaGetSymbolAddress(&p, gNoAllocCounts);
      if (e != cudaSuccess) { return cudaFail(e, "cudaGetSymbolAddress(counts)"); }
      s.counts = (unsigned long long *)p;
      s.ready = true;
   }
   out = s;
   return MKF_OK;
}

}  // namespace mkf

using namespace mkf;

MKF_API int mkfFieldBPFDHostNoAlloc(uint64_t *pBPFDH, const MKFFieldDesc *pF, const MKFThreshSet *pT, void *stream)
{
   if (!pBPFDH || !pF || !pF->p || !pT || !pT->t) { setError("mkfFieldBPFDHostNoAlloc: NULL argument"); return MKF_ERR_ARG; }
   if (pF->stride[0] | pF->stride[1] | pF->stride[2]) { setError("mkfFieldBPFDHostNoAlloc: host fields must be planar"); return MKF_ERR_UNSUPPORTED; }
   if (pF->enc != ENC_F32 && pF->enc != ENC_F64) { setError("mkfFieldBPFDHostNoAlloc: encoding 0x%02X not supported", pF->enc); return MKF_ERR_UNSUPPORTED; }
   const int K = pT->nT;
   if (K < 1 || K > MKF_MAX_THRESH) { setError("mkfFieldBPFDHostNoAlloc: nT=%d out of range 1..%d", K, MKF_MAX_THRESH); return MKF_ERR_ARG; }
   const int X = pF->def[0], Y = pF->def[1], Z = pF->def[2];
   if (X < 1 || Y < 1 || Z < 1) { setError("mkfFieldBPFDHostNoAlloc: bad dimensions %d %d %d", X, Y, Z); return MKF_ERR_ARG; }
   const size_t esz = (pF->enc == ENC_F32) ? 4 : 8;
   const size_t planeBytes = (size_t)X * Y * esz;
   if (Z > 1 && 2 * planeBytes > MKF_NOALLOC_STAGE_BYTES) {
      setError("mkfFieldBPFDHostNoAlloc: a plane of %d x %d elements is %zu bytes; the staging area holds %zu "
               "bytes and must hold two planes (planes of at most %zu bytes)", X, Y, planeBytes,
               (size_t)MKF_NOALLOC_STAGE_BYTES, (size_t)MKF_NOALLOC_STAGE_BYTES / 2);
      return MKF_ERR_NOMEM;
   }
   NoAllocScratch sc;
   int rc = scratchForCurrentDevice(sc);
   if (rc != MKF_OK) { return rc; }
   cudaStream_t s = (cudaStream_t)stream;
   const unsigned long long cells = (unsigned long long)(X - 1) * (unsigned long long)(Y - 1) * (unsigned long long)(Z - 1);
   cudaError_t e = cudaMemsetAsync(sc.counts, 0, (size_t)K * 256 * sizeof(uint64_t), s);
   if (e != cudaSuccess) { return cudaFail(e, "cudaMemsetAsync"); }

   // classify the thresholds as the heap-using path does: constant maps, one thermometer class
   // (every relation the same, one of > >= < <=) or the general per-threshold path
   int constRow[MKF_MAX_THRESH], constBin[MKF_MAX_THRESH], nConst = 0;
   int idx[MKF_MAX_THRESH], n = 0, cls0 = -2;
   for (int i = 0; i < K; i++) {
      const double t = pT->t[i];
      const uint32_t m = (pT->m ? pT->m[i] : pT->mAll) & BMC_AL;
      if (m == 0 || m == BMC_AL || std::isnan(t)) {
         const bool one = (m == BMC_AL) || (std::isnan(t) && (m & BMC_EQ));
         constRow[nConst] = i;
         constBin[nConst++] = one ? 255 : 0;
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
   // stable insertion sort of the thresholds by value
   for (int a = 1; a < n; a++) {
      const int v = idx[a];
      int b = a - 1;
      while (b >= 0 && pT->t[idx[b]] > pT->t[v]) { idx[b + 1] = idx[b]; b--; }
      idx[b + 1] = v;
   }
   FusedPlain q;
   memset(&q, 0, sizeof(q));
   q.enc = pF->enc;
   q.sx = 1;
   q.sy = X;
   q.sz = (int64_t)X * Y;
   q.X = X;
   q.Y = Y;
   q.K = n;
   q.out = (uint64_t *)sc.counts;
   for (int k = 0; k < n; k++) {
      const double t = pT->t[idx[k]];
      if (pF->enc == ENC_F32) { floatBoundsPlain(t, q.tlo[k], q.thi[k]); }
      else { q.tlo[k] = q.thi[k] = t; }
      q.outRow[k] = idx[k];
      const uint32_t m = (pT->m ? pT->m[idx[k]] : pT->mAll) & BMC_AL;
      q.mask[k] = m;
      q.gtm |= ((m >> 2) & 1u) << k;
      q.eqm |= ((m >> 1) & 1u) << k;
      q.ltm |= (m & 1u) << k;
   }
   q.thermo = (n > 0 && cls0 >= 0);
   if (q.thermo) {
      q.rankHi = (cls0 == 1 || cls0 == 2);
      q.complement = (cls0 >= 2);
      const bool eqBit = (cls0 == 1 || cls0 == 3);
      q.nanRank = (eqBit != (q.complement != 0)) ? (uint32_t)n : 0u;
   }

   if (cells > 0) {
      // slabs of S plane pairs (S+1 planes staged; the last plane is the next slab's first); no
      // copies at all when every threshold is a constant map
      size_t S = MKF_NOALLOC_STAGE_BYTES / planeBytes - 1;
      if (S > (size_t)Z - 1) { S = (size_t)Z - 1; }
      const char *src = (const char *)pF->p;
      for (size_t z0 = 0; n > 0 && z0 + 1 < (size_t)Z && rc == MKF_OK; z0 += S) {
         const size_t nPl = std::min(S + 1, (size_t)Z - z0);
         // same stream: this copy starts only after the previous slab's kernel has finished
         e = cudaMemcpyAsync(sc.stage, src + z0 * planeBytes, nPl * planeBytes, cudaMemcpyHostToDevice, s);
         if (e != cudaSuccess) { rc = cudaFail(e, "slab copy"); break; }
         q.f = sc.stage;
         q.Z = (int)nPl;
         rc = launchFusedPlain(q, s);
      }
      for (int c = 0; c < nConst && rc == MKF_OK; c++) {
         rc = launchConstBin((uint64_t *)sc.counts, constRow[c], constBin[c], cells, s);
      }
   }
   if (rc == MKF_OK) {
      e = cudaMemcpyAsync(pBPFDH, sc.counts, (size_t)K * 256 * sizeof(uint64_t), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) { e = cudaStreamSynchronize(s); }
      rc = cudaFail(e, "count copy-back");
   } else {
      cudaStreamSynchronize(s);
   }
   return rc;
}
