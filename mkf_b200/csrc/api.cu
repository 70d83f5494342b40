// api.cu - entry points of mkf_b200.h built on the fused counting kernel (fused.cu).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>
#include "fused.cuh"

namespace mkf {
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

// __constant__ memory belongs to each device: upload the tables once per device, on first use
// with that device current.
static std::mutex gConstMu;
static bool gConstDone[64] = {};

static int uploadConstants()
{
   int dev = 0;
   cudaError_t e = cudaGetDevice(&dev);
   if (e != cudaSuccess) { return cudaFail(e, "cudaGetDevice"); }
   if (dev < 0 || dev >= 64) { setError("measure constants: device %d out of range", dev); return MKF_ERR_UNSUPPORTED; }
   std::lock_guard<std::mutex> lk(gConstMu);
   if (gConstDone[dev]) { return MKF_OK; }
   e = cudaMemcpyToSymbol(cGroupOf, kGroupOf, sizeof(cGroupOf));
   if (e == cudaSuccess) { e = cudaMemcpyToSymbol(cWK, kWK, sizeof(cWK)); }
   if (e == cudaSuccess) { e = cudaMemcpyToSymbol(cWS, kWS, sizeof(cWS)); }
   if (e == cudaSuccess) { e = cudaMemcpyToSymbol(cWM, kWM, sizeof(cWM)); }
   if (e != cudaSuccess) { return cudaFail(e, "measure constants upload"); }
   gConstDone[dev] = true;
   return MKF_OK;
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

MKF_API int mkfFieldBPFDMoments(uint64_t *pBPFD, double *pMom, const MKFFieldDesc *pF, const MKFThreshSet *pT,
                                int flags, void *stream)
{
   if (!pBPFD || !pMom || !pF || !pT || !pF->p || !pT->t) { setError("mkfFieldBPFDMoments: NULL argument"); return MKF_ERR_ARG; }
   const int K = pT->nT;
   if (K < 1 || K > 2) { setError("mkfFieldBPFDMoments: nT=%d, moments are counted for 1 or 2 thresholds", K); return MKF_ERR_UNSUPPORTED; }
   if (pF->enc != ENC_F32 && pF->enc != ENC_F64) { setError("mkfFieldBPFDMoments: encoding 0x%02X not supported", pF->enc); return MKF_ERR_UNSUPPORTED; }
   const int X = pF->def[0], Y = pF->def[1], Z = pF->def[2];
   if (X < 2 || Y < 2 || Z < 2) { setError("mkfFieldBPFDMoments: dimensions %d %d %d (each must be >= 2)", X, Y, Z); return MKF_ERR_ARG; }
   cudaStream_t s = (cudaStream_t)stream;
   if (!(flags & MKF_F_ACCUMULATE)) {
      cudaError_t e = cudaMemsetAsync(pBPFD, 0, (size_t)K * 256 * sizeof(uint64_t), s);
      if (e == cudaSuccess) { e = cudaMemsetAsync(pMom, 0, (size_t)K * 4 * sizeof(double), s); }
      if (e != cudaSuccess) { return cudaFail(e, "cudaMemsetAsync"); }
   }
   FusedArgs a;
   memset(&a, 0, sizeof(a));
   a.f = pF->p;
   const bool planar = !(pF->stride[0] | pF->stride[1] | pF->stride[2]);
   a.sx = planar ? 1 : pF->stride[0];
   a.sy = planar ? (int64_t)X : pF->stride[1];
   a.sz = planar ? (int64_t)X * Y : pF->stride[2];
   a.X = X; a.Y = Y; a.Z = Z;
   a.K = K;
   a.out = pBPFD;
   uint32_t masks[2];
   for (int k = 0; k < K; k++) {
      const double t = pT->t[k];
      if (pF->enc == ENC_F32) { floatBoundsPlain(t, a.tlo[k], a.thi[k]); }
      else { a.tlo[k] = a.thi[k] = t; }
      a.outRow[k] = k;
      masks[k] = (pT->m ? pT->m[k] : pT->mAll) & BMC_AL;
   }
   return launchWordsMoments(a, pF->enc, masks, pMom, s);
}

// ---------------------------------------------------------------- batches

struct MKFBatchPlan
{
   uint64_t *out = nullptr;
   size_t rows = 0;
   FieldTask *dTasks[2] = {nullptr, nullptr};  // thermometer-kernel fields, FP32 and FP64
   BatchChunk *dChunks[2] = {nullptr, nullptr};
   int nChunks[2] = {0, 0};
   std::vector<ThermoGroup> groups[2];  // the thermometer chunks of each kernel variant
   WordTask *dWTasks[2] = {nullptr, nullptr};  // word-kernel fields, FP32 and FP64
   BatchChunk *dWChunks[2] = {nullptr, nullptr};
   int nWChunks[2] = {0, 0};
   unsigned *dCounter = nullptr;  // chunk counters: words FP32, FP64, then thermometer FP32, FP64 per variant
   std::vector<ConstEntry> consts;
   std::vector<unsigned long long> constCells;
   struct Fallback
   {
      MKFFieldDesc d;
      std::vector<double> t;
      std::vector<uint32_t> m;
      uint32_t mAll;
      bool perThreshold;
      size_t rowBase;
   };
   std::vector<Fallback> fallbacks;
   cudaGraph_t graph = nullptr;
   cudaGraphExec_t graphExec = nullptr;
};

static constexpr int kChunkItems = 64;
static constexpr int kPlanCounters = 2 + 2 * kThVariants;

static void freePlan(MKFBatchPlan *p)
{
   if (!p) { return; }
   if (p->graphExec) { cudaGraphExecDestroy(p->graphExec); }
   if (p->graph) { cudaGraphDestroy(p->graph); }
   for (int e = 0; e < 2; e++) {
      if (p->dTasks[e]) { cudaFree(p->dTasks[e]); }
      if (p->dChunks[e]) { cudaFree(p->dChunks[e]); }
      if (p->dWTasks[e]) { cudaFree(p->dWTasks[e]); }
      if (p->dWChunks[e]) { cudaFree(p->dWChunks[e]); }
   }
   if (p->dCounter) { cudaFree(p->dCounter); }
   delete p;
}

// A plan whose work items span `depth` planes (0: each kernel's default).
static int createPlan(MKFBatchPlan **pp, uint64_t *pBPFD, const MKFFieldDesc *pF, const MKFThreshSet *pT, int nF, int depth)
{
   *pp = nullptr;
   MKFBatchPlan *p = new MKFBatchPlan();
   p->out = pBPFD;
   std::vector<FieldTask> tasks[2];
   std::vector<BatchChunk> chunks[2];
   std::vector<WordTask> wtasks[2];
   std::vector<BatchChunk> wchunks[2];
   size_t row = 0;
   for (int i = 0; i < nF; i++) {
      const MKFFieldDesc *d = pF + i;
      const MKFThreshSet *ts = pT + i;
      if (!d->p || !ts->t || ts->nT < 1 || ts->nT > MKF_MAX_THRESH || (d->enc != ENC_F32 && d->enc != ENC_F64) ||
          d->def[0] < 1 || d->def[1] < 1 || d->def[2] < 1) {
         setError("mkfBatchPlanCreate: field %d: bad descriptor or thresholds", i);
         freePlan(p);
         return MKF_ERR_ARG;
      }
      const unsigned long long cells = (unsigned long long)(d->def[0] - 1) * (d->def[1] - 1) * (d->def[2] - 1);
      const size_t c0 = p->consts.size();
      FieldTask t;
      WordTask w;
      bool varying = false;
      const int kind = planBatchField(d, ts, (int)row, t, w, p->consts, varying, depth);
      for (size_t c = c0; c < p->consts.size(); c++) { p->constCells.push_back(cells); }
      if (cells > 0 && kind == kPlanWords) {
         const int e = d->enc == ENC_F32 ? 0 : 1;
         const int f = (int)wtasks[e].size();
         for (long long b = 0; b < w.nItems; b += kChunkItems) {
            wchunks[e].push_back({f, 0, b, std::min<long long>(b + kChunkItems, w.nItems)});
         }
         w.out = pBPFD;
         wtasks[e].push_back(w);
      } else if (cells > 0 && kind == kPlanThermo) {
         const int e = d->enc == ENC_F32 ? 0 : 1;
         const int f = (int)tasks[e].size();
         for (long long b = 0; b < t.nItems; b += kChunkItems) {
            chunks[e].push_back({f, 0, b, std::min<long long>(b + kChunkItems, t.nItems)});
         }
         t.out = pBPFD;
         tasks[e].push_back(t);
      } else if (cells > 0 && varying) {
         MKFBatchPlan::Fallback fb;
         fb.d = *d;
         fb.t.assign(ts->t, ts->t + ts->nT);
         fb.perThreshold = ts->m != nullptr;
         if (fb.perThreshold) { fb.m.assign(ts->m, ts->m + ts->nT); }
         fb.mAll = ts->mAll;
         fb.rowBase = row;
         // constant maps of this field are counted by its own pass
         p->consts.resize(c0);
         p->constCells.resize(c0);
         p->fallbacks.push_back(fb);
      }
      row += (size_t)ts->nT;
   }
   p->rows = row;
   cudaError_t e = cudaMalloc(&p->dCounter, kPlanCounters * sizeof(unsigned));
   for (int k = 0; k < 2 && e == cudaSuccess; k++) {
      if (tasks[k].empty()) { continue; }
      p->groups[k] = groupThermoChunks(chunks[k], tasks[k]);
      e = cudaMalloc(&p->dTasks[k], tasks[k].size() * sizeof(FieldTask));
      if (e == cudaSuccess) { e = cudaMalloc(&p->dChunks[k], chunks[k].size() * sizeof(BatchChunk)); }
      if (e == cudaSuccess) { e = cudaMemcpy(p->dTasks[k], tasks[k].data(), tasks[k].size() * sizeof(FieldTask), cudaMemcpyHostToDevice); }
      if (e == cudaSuccess) { e = cudaMemcpy(p->dChunks[k], chunks[k].data(), chunks[k].size() * sizeof(BatchChunk), cudaMemcpyHostToDevice); }
      p->nChunks[k] = (int)chunks[k].size();
   }
   for (int k = 0; k < 2 && e == cudaSuccess; k++) {
      if (wtasks[k].empty()) { continue; }
      e = cudaMalloc(&p->dWTasks[k], wtasks[k].size() * sizeof(WordTask));
      if (e == cudaSuccess) { e = cudaMalloc(&p->dWChunks[k], wchunks[k].size() * sizeof(BatchChunk)); }
      if (e == cudaSuccess) { e = cudaMemcpy(p->dWTasks[k], wtasks[k].data(), wtasks[k].size() * sizeof(WordTask), cudaMemcpyHostToDevice); }
      if (e == cudaSuccess) { e = cudaMemcpy(p->dWChunks[k], wchunks[k].data(), wchunks[k].size() * sizeof(BatchChunk), cudaMemcpyHostToDevice); }
      p->nWChunks[k] = (int)wchunks[k].size();
   }
   if (e != cudaSuccess) {
      freePlan(p);
      return cudaFail(e, "mkfBatchPlanCreate: device work list");
   }
   *pp = p;
   return MKF_OK;
}

// Everything a launch issues, in stream order (no allocation, no synchronisation: capturable).
static int planLaunchOn(MKFBatchPlan *p, cudaStream_t s)
{
   cudaError_t e = cudaMemsetAsync(p->out, 0, p->rows * 256 * sizeof(uint64_t), s);
   if (e != cudaSuccess) { return cudaFail(e, "batch output clear"); }
   int rc = MKF_OK;
   for (size_t i = 0; i < p->consts.size() && rc == MKF_OK; i++) {
      rc = launchConstBin(p->out, p->consts[i].row, p->consts[i].bin, p->constCells[i], s);
   }
   if (rc == MKF_OK && (p->nChunks[0] > 0 || p->nChunks[1] > 0 || p->nWChunks[0] > 0 || p->nWChunks[1] > 0)) {
      e = cudaMemsetAsync(p->dCounter, 0, kPlanCounters * sizeof(unsigned), s);
      if (e != cudaSuccess) { return cudaFail(e, "batch counter clear"); }
   }
   for (int k = 0; k < 2 && rc == MKF_OK; k++) {
      if (p->nWChunks[k] == 0) { continue; }
      WordBatchArgs w;
      w.tasks = p->dWTasks[k];
      w.chunks = p->dWChunks[k];
      w.nChunks = p->nWChunks[k];
      w.counter = p->dCounter + k;
      rc = launchWordsBatch(w, k == 0 ? ENC_F32 : ENC_F64, s);
   }
   for (int k = 0; k < 2 && rc == MKF_OK; k++) {
      if (p->nChunks[k] == 0) { continue; }
      rc = launchThermoGroups(p->dTasks[k], p->dChunks[k], p->groups[k], p->dCounter + 2 + k * kThVariants,
                              k == 0 ? ENC_F32 : ENC_F64, s);
   }
   for (size_t i = 0; i < p->fallbacks.size() && rc == MKF_OK; i++) {
      const MKFBatchPlan::Fallback &fb = p->fallbacks[i];
      MKFThreshSet ts;
      ts.nT = (int32_t)fb.t.size();
      ts.t = fb.t.data();
      ts.m = fb.perThreshold ? fb.m.data() : nullptr;
      ts.mAll = fb.mAll;
      rc = fieldBPFD(p->out + fb.rowBase * 256, &fb.d, &ts, MKF_F_ACCUMULATE, s, nullptr);
   }
   return rc;
}

MKF_API int mkfBatchPlanCreate(MKFBatchPlan **pp, uint64_t *pBPFD, const MKFFieldDesc *pF, const MKFThreshSet *pT, int nF)
{
   if (!pp || !pBPFD || (nF > 0 && (!pF || !pT)) || nF < 0) { setError("mkfBatchPlanCreate: bad argument"); return MKF_ERR_ARG; }
   *pp = nullptr;
   if (!batchTuning() || nF == 0) { return createPlan(pp, pBPFD, pF, pT, nF, 0); }
   // time one launch of the plan for each candidate slab depth and keep the fastest
   static const int kCand[] = {8, 16, 32, 64};
   cudaStream_t s = nullptr;
   cudaEvent_t e0 = nullptr, e1 = nullptr;
   cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
   if (e == cudaSuccess) { e = cudaEventCreate(&e0); }
   if (e == cudaSuccess) { e = cudaEventCreate(&e1); }
   int rc = (e == cudaSuccess) ? MKF_OK : cudaFail(e, "mkfBatchPlanCreate: tuning set-up");
   MKFBatchPlan *best = nullptr;
   float bestMs = 0.0f;
   for (int c = 0; c < 4 && rc == MKF_OK; c++) {
      MKFBatchPlan *cand = nullptr;
      rc = createPlan(&cand, pBPFD, pF, pT, nF, kCand[c]);
      if (rc != MKF_OK) { break; }
      rc = planLaunchOn(cand, s);  // warm-up
      if (rc == MKF_OK && (e = cudaEventRecord(e0, s)) != cudaSuccess) { rc = cudaFail(e, "event"); }
      if (rc == MKF_OK) { rc = planLaunchOn(cand, s); }
      if (rc == MKF_OK && (e = cudaEventRecord(e1, s)) != cudaSuccess) { rc = cudaFail(e, "event"); }
      if (rc == MKF_OK && (e = cudaEventSynchronize(e1)) != cudaSuccess) { rc = cudaFail(e, "event"); }
      float ms = 0.0f;
      if (rc == MKF_OK && (e = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) { rc = cudaFail(e, "event"); }
      if (rc == MKF_OK && (!best || ms < bestMs)) {
         if (best) { freePlan(best); }
         best = cand;
         bestMs = ms;
      } else {
         cudaStreamSynchronize(s);
         freePlan(cand);
      }
   }
   if (s) { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
   if (e0) { cudaEventDestroy(e0); }
   if (e1) { cudaEventDestroy(e1); }
   if (rc != MKF_OK) {
      if (best) { freePlan(best); }
      return rc;
   }
   *pp = best;
   return MKF_OK;
}

MKF_API int mkfBatchPlanLaunch(MKFBatchPlan *p, void *stream)
{
   if (!p) { setError("mkfBatchPlanLaunch: NULL plan"); return MKF_ERR_ARG; }
   return planLaunchOn(p, (cudaStream_t)stream);
}

MKF_API int mkfBatchPlanLaunchGraph(MKFBatchPlan *p, void *stream)
{
   if (!p) { setError("mkfBatchPlanLaunchGraph: NULL plan"); return MKF_ERR_ARG; }
   cudaError_t e;
   if (!p->graphExec) {
      cudaStream_t cap;
      e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
      if (e != cudaSuccess) { return cudaFail(e, "capture stream"); }
      e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
      int rc = (e == cudaSuccess) ? planLaunchOn(p, cap) : cudaFail(e, "cudaStreamBeginCapture");
      cudaGraph_t g = nullptr;
      e = cudaStreamEndCapture(cap, &g);
      cudaStreamDestroy(cap);
      if (rc != MKF_OK) { if (g) { cudaGraphDestroy(g); } return rc; }
      if (e != cudaSuccess) { return cudaFail(e, "cudaStreamEndCapture"); }
      e = cudaGraphInstantiate(&p->graphExec, g, 0);
      if (e != cudaSuccess) { cudaGraphDestroy(g); return cudaFail(e, "cudaGraphInstantiate"); }
      p->graph = g;
   }
   return cudaFail(cudaGraphLaunch(p->graphExec, (cudaStream_t)stream), "cudaGraphLaunch");
}

MKF_API int mkfBatchPlanDestroy(MKFBatchPlan *p)
{
   freePlan(p);
   return MKF_OK;
}

MKF_API int mkfBatchBPFD(uint64_t *pBPFD, const MKFFieldDesc *pF, const MKFThreshSet *pT, int nF, int flags, void *stream)
{
   (void)flags;
   if (!pBPFD || (nF > 0 && (!pF || !pT)) || nF < 0) { setError("mkfBatchBPFD: bad argument"); return MKF_ERR_ARG; }
   MKFBatchPlan *p = nullptr;
   // one launch: no depth tuning (it would count the batch several times), depth by field size
   int rc = createPlan(&p, pBPFD, pF, pT, nF, -1);
   if (rc != MKF_OK) { return rc; }
   rc = planLaunchOn(p, (cudaStream_t)stream);
   const cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
   if (rc == MKF_OK) { rc = cudaFail(e, "batch synchronisation"); }
   freePlan(p);
   return rc;
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
