// api.cu - entry points of mkf_b200.h built on the fused counting kernel (fused.cu).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>
#include "mkf_common.cuh"

namespace mkf {
int fieldBPFD(uint64_t *out, const MKFFieldDesc *pF, const MKFThreshSet *pT, int flags, cudaStream_t s, const int *rowBase);
void measures(double r[4], const uint64_t h[256]);
extern const uint8_t kGroupOf[256];
extern const int kWK[22];
extern const double kWS[22];
extern const double kWM[22];

// Device copy of the group map and weights for the measure epilogue.
__constant__ uint8_t cGroupOf[256];
__constant__ int cWK[22];
__constant__ double cWS[22];
__constant__ double cWM[22];

// One thread per distribution, same arithmetic and order as measures() on the host, so the
// device and host results are identical.
__global__ void measuresKernel(double *r, const uint64_t *h, int nSets)
{
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= nSets) { return; }
   const uint64_t *p = h + (size_t)i * 256;
   uint64_t g[22];
   for (int q = 0; q < 22; q++) { g[q] = 0; }
   uint64_t v = 0;
   for (int c = 0; c < 256; c++) {
      g[cGroupOf[c]] += p[c];
      if (c & 1) { v += p[c]; }
   }
   // separate multiply and add (no fused multiply-add), as the host computes it
   double s = __dmul_rn((double)g[0], cWS[0]), mc = __dmul_rn((double)g[0], cWM[0]);
   for (int q = 1; q < 22; q++) {
      s = __dadd_rn(s, __dmul_rn((double)g[q], cWS[q]));
      mc = __dadd_rn(mc, __dmul_rn((double)g[q], cWM[q]));
   }
   long long k = 0;
   for (int q = 0; q < 22; q++) { k += (long long)cWK[q] * (long long)g[q]; }
   r[4 * i + 0] = (double)v;
   r[4 * i + 1] = s;
   r[4 * i + 2] = mc;
   r[4 * i + 3] = (double)k / 24.0;
}

static std::once_flag gConstOnce;
static int gConstRc = MKF_OK;

static int uploadConstants()
{
   std::call_once(gConstOnce, [] {
      cudaError_t e = cudaMemcpyToSymbol(cGroupOf, kGroupOf, sizeof(cGroupOf));
      if (e == cudaSuccess) { e = cudaMemcpyToSymbol(cWK, kWK, sizeof(cWK)); }
      if (e == cudaSuccess) { e = cudaMemcpyToSymbol(cWS, kWS, sizeof(cWS)); }
      if (e == cudaSuccess) { e = cudaMemcpyToSymbol(cWM, kWM, sizeof(cWM)); }
      gConstRc = cudaFail(e, "measure constants upload");
   });
   return gConstRc;
}

// Device buffers reused by the host-field path (grown on demand, guarded by a mutex).
struct HostPathBuffers
{
   std::mutex mu;
   void *stage[2] = {nullptr, nullptr};
   size_t stageBytes = 0;
   uint64_t *counts = nullptr;
   cudaStream_t copy = nullptr, comp = nullptr;
   cudaEvent_t loaded[2] = {nullptr, nullptr}, consumed[2] = {nullptr, nullptr};
};
static HostPathBuffers gHost;

}  // namespace mkf

using namespace mkf;

MKF_API int mkfFieldBPFD(uint64_t *pBPFD, const MKFFieldDesc *pF, const MKFThreshSet *pT, int flags, void *stream)
{
   return fieldBPFD(pBPFD, pF, pT, flags, (cudaStream_t)stream, nullptr);
}

MKF_API int mkfBatchBPFD(uint64_t *pBPFD, const MKFFieldDesc *pF, const MKFThreshSet *pT, int nF, int flags, void *stream)
{
   if (!pBPFD || !pF || !pT || nF < 0) { setError("mkfBatchBPFD: bad argument"); return MKF_ERR_ARG; }
   size_t row = 0;
   for (int i = 0; i < nF; i++) {
      const int rc = fieldBPFD(pBPFD + row * 256, pF + i, pT + i, flags, (cudaStream_t)stream, nullptr);
      if (rc != MKF_OK) { return rc; }
      row += (size_t)pT[i].nT;
   }
   return MKF_OK;
}

MKF_API int mkfMeasuresF64Dev(double *r, const uint64_t *pBPFD, int nSets, void *stream)
{
   if (!r || !pBPFD || nSets < 0) { setError("mkfMeasuresF64Dev: bad argument"); return MKF_ERR_ARG; }
   int rc = uploadConstants();
   if (rc != MKF_OK || nSets == 0) { return rc; }
   measuresKernel<<<(nSets + 63) / 64, 64, 0, (cudaStream_t)stream>>>(r, pBPFD, nSets);
   return cudaFail(cudaGetLastError(), "measuresKernel launch");
}

MKF_API int mkfFieldBPFDHost(uint64_t *pBPFDH, const MKFFieldDesc *pF, const MKFThreshSet *pT)
{
   if (!pBPFDH || !pF || !pF->p || !pT) { setError("mkfFieldBPFDHost: NULL argument"); return MKF_ERR_ARG; }
   if (pF->stride[0] | pF->stride[1] | pF->stride[2]) { setError("mkfFieldBPFDHost: host fields must be planar"); return MKF_ERR_UNSUPPORTED; }
   if (pF->enc != ENC_F32 && pF->enc != ENC_F64) { setError("mkfFieldBPFDHost: encoding not supported"); return MKF_ERR_UNSUPPORTED; }
   const int K = pT->nT;
   if (K < 1 || K > MKF_MAX_THRESH) { setError("mkfFieldBPFDHost: nT out of range"); return MKF_ERR_ARG; }
   const int X = pF->def[0], Y = pF->def[1], Z = pF->def[2];
   if (X < 1 || Y < 1 || Z < 1) { setError("mkfFieldBPFDHost: bad dimensions"); return MKF_ERR_ARG; }
   const size_t esz = (pF->enc == ENC_F32) ? 4 : 8;
   const size_t planeBytes = (size_t)X * Y * esz;
   // slabs of S plane pairs: S+1 planes staged, the last plane is also the next slab's first
   size_t S = std::max<size_t>(1, ((size_t)256 << 20) / planeBytes);
   if (S > (size_t)Z - 1 && Z > 1) { S = (size_t)Z - 1; }
   const size_t slabBytes = (S + 1) * planeBytes;

   std::lock_guard<std::mutex> lock(gHost.mu);
   cudaError_t e = cudaSuccess;
   if (!gHost.copy) {
      e = cudaStreamCreateWithFlags(&gHost.copy, cudaStreamNonBlocking);
      if (e == cudaSuccess) { e = cudaStreamCreateWithFlags(&gHost.comp, cudaStreamNonBlocking); }
      for (int i = 0; i < 2 && e == cudaSuccess; i++) {
         e = cudaEventCreateWithFlags(&gHost.loaded[i], cudaEventDisableTiming);
         if (e == cudaSuccess) { e = cudaEventCreateWithFlags(&gHost.consumed[i], cudaEventDisableTiming); }
      }
      if (e == cudaSuccess) { e = cudaMalloc(&gHost.counts, (size_t)MKF_MAX_THRESH * 256 * sizeof(uint64_t)); }
      if (e != cudaSuccess) { return cudaFail(e, "mkfFieldBPFDHost set-up"); }
   }
   if (gHost.stageBytes < slabBytes) {
      for (int i = 0; i < 2; i++) {
         if (gHost.stage[i]) { cudaFree(gHost.stage[i]); gHost.stage[i] = nullptr; }
      }
      gHost.stageBytes = 0;
      for (int i = 0; i < 2 && e == cudaSuccess; i++) { e = cudaMalloc(&gHost.stage[i], slabBytes); }
      if (e != cudaSuccess) { return cudaFail(e, "mkfFieldBPFDHost staging allocation"); }
      gHost.stageBytes = slabBytes;
   }
   e = cudaMemsetAsync(gHost.counts, 0, (size_t)K * 256 * sizeof(uint64_t), gHost.comp);
   if (e != cudaSuccess) { return cudaFail(e, "cudaMemsetAsync"); }
   const char *src = (const char *)pF->p;
   const size_t nSlab = (Z > 1) ? ((size_t)Z - 1 + S - 1) / S : 1;
   for (int i = 0; i < 2; i++) { cudaEventRecord(gHost.consumed[i], gHost.comp); }
   int rc = MKF_OK;
   for (size_t s = 0; s < nSlab && rc == MKF_OK; s++) {
      const int b = (int)(s & 1);
      const size_t z0 = s * S;
      const size_t nPl = std::min(S + 1, (size_t)Z - z0);
      cudaStreamWaitEvent(gHost.copy, gHost.consumed[b], 0);
      e = cudaMemcpyAsync(gHost.stage[b], src + z0 * planeBytes, nPl * planeBytes, cudaMemcpyHostToDevice, gHost.copy);
      if (e != cudaSuccess) { rc = cudaFail(e, "slab copy"); break; }
      cudaEventRecord(gHost.loaded[b], gHost.copy);
      cudaStreamWaitEvent(gHost.comp, gHost.loaded[b], 0);
      MKFFieldDesc sub = *pF;
      sub.p = gHost.stage[b];
      sub.def[2] = (int32_t)nPl;
      rc = fieldBPFD(gHost.counts, &sub, pT, MKF_F_ACCUMULATE, gHost.comp, nullptr);
      cudaEventRecord(gHost.consumed[b], gHost.comp);
   }
   if (rc == MKF_OK) {
      e = cudaMemcpyAsync(pBPFDH, gHost.counts, (size_t)K * 256 * sizeof(uint64_t), cudaMemcpyDeviceToHost, gHost.comp);
      if (e == cudaSuccess) { e = cudaStreamSynchronize(gHost.comp); }
      rc = cudaFail(e, "count copy-back");
   } else {
      cudaStreamSynchronize(gHost.comp);
      cudaStreamSynchronize(gHost.copy);
   }
   return rc;
}
