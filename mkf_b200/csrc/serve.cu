// serve.cu - request loop for in-situ analysis: many clients submit fields (device pointers or
// pinned host buffers) with their thresholds; one worker thread admits them against a device-memory
// budget, copies host fields on a copy stream, and packs everything admitted since the last launch
// into the next persistent batched launch (the word and thermometer batch kernels of words.cu and
// thermo.cu), while the previous launch may still be running on the other of two launch streams.
// Counts stay in device memory until the client releases them, or are copied to a host array the
// request names. The original MKF has no serving form: it counts one field per synchronous call
// (mkfCUDA.cu:12-91).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include "arena.h"
#include "fused.cuh"

using Clock = std::chrono::steady_clock;

namespace mkf {

static constexpr int kServerCounters = 2 + 2 * kThVariants;  // chunk counters per launch slot

enum ReqState { kQueued, kRunning, kDone };

struct Request
{
   uint64_t ticket = 0;
   MKFFieldDesc field;
   std::vector<double> t;
   std::vector<uint32_t> m;
   uint32_t mAll = 0;
   uint32_t flags = 0;
   uint64_t *hostOut = nullptr;
   size_t fieldBytes = 0;      // host fields: bytes staged on the device
   void *staged = nullptr;     // device copy of a host field
   uint64_t *dCounts = nullptr;
   size_t countBytes = 0;
   size_t hostSlot = 0;        // offset of its counts in the launch's pinned result buffer
   Clock::time_point tSubmit, tDone;
   ReqState state = kQueued;
   int rc = MKF_OK;
   std::string err;
};

// Zero the count arrays of a launch: entry i is (pointer, 64-bit words).
struct ClearEntry
{
   uint64_t *p;
   long long n;
};
__global__ void clearCounts(const ClearEntry *e, int nE)
{
   for (int i = blockIdx.x; i < nE; i += gridDim.x) {
      uint64_t *p = e[i].p;
      for (long long j = threadIdx.x; j < e[i].n; j += blockDim.x) { p[j] = 0; }
   }
}

// Device and pinned-host buffers of one launch slot, grown on demand (a slot is only refilled
// after its previous launch completed, so growing never frees memory a kernel still reads).
struct DevBuf
{
   void *d = nullptr;
   void *h = nullptr;
   size_t cap = 0;
   cudaError_t ensure(size_t bytes)
   {
      if (bytes <= cap) { return cudaSuccess; }
      size_t n = std::max(bytes, cap * 2);
      if (d) { cudaFree(d); d = nullptr; }
      if (h) { cudaFreeHost(h); h = nullptr; }
      cap = 0;
      cudaError_t e = cudaMalloc(&d, n);
      if (e == cudaSuccess) { e = cudaMallocHost(&h, n); }
      if (e == cudaSuccess) { cap = n; }
      return e;
   }
   void destroy()
   {
      if (d) { cudaFree(d); }
      if (h) { cudaFreeHost(h); }
      d = h = nullptr;
      cap = 0;
   }
};

struct LaunchSlot
{
   cudaStream_t stream = nullptr;
   cudaEvent_t copied = nullptr, start = nullptr, done = nullptr;
   std::vector<Request *> reqs;
   DevBuf work;      // tasks, chunks, clear list (uploaded each launch)
   DevBuf results;   // counts of requests that want them on the host
   unsigned *counters = nullptr;  // chunk counters: words FP32, FP64, then thermometer FP32, FP64 per variant
   bool busy = false;
};

}  // namespace mkf

using namespace mkf;

struct MKFServer
{
   int device = 0;
   int maxPerLaunch = 256;
   Arena arena;          // sub-allocates `budgetMem`
   void *budgetMem = nullptr;
   cudaStream_t copyStream = nullptr;
   LaunchSlot slots[2];
   std::mutex mu;
   std::condition_variable cvWork, cvDone;
   std::deque<Request *> incoming;
   std::map<uint64_t, Request *> byTicket;
   uint64_t nextTicket = 1;
   bool stop = false;
   std::thread worker;
   // statistics (under mu)
   std::vector<double> latency;
   uint64_t launches = 0, failed = 0, fieldsLaunched = 0;
   double launchDeviceSec = 0.0, planHostSec = 0.0;
   uint32_t maxInLaunch = 0;
   std::string fatal;
};

namespace mkf {

static void finishRequest(MKFServer *s, Request *r, int rc, const char *msg)
{
   r->rc = rc;
   if (msg) { r->err = msg; }
   r->tDone = Clock::now();
   r->state = kDone;
}

// Plan and issue one launch for the requests in `sl` (worker thread). Returns MKF_OK or an error
// that applies to the whole launch.
static int issueLaunch(MKFServer *s, LaunchSlot &sl)
{
   cudaStream_t st = sl.stream;
   cudaError_t e;
   // host fields: copy on the copy stream, the launch stream waits for the copies
   bool anyCopy = false;
   for (Request *r : sl.reqs) {
      if (r->staged) {
         e = cudaMemcpyAsync(r->staged, r->field.p, r->fieldBytes, cudaMemcpyHostToDevice, s->copyStream);
         if (e != cudaSuccess) { return cudaFail(e, "server: field copy"); }
         anyCopy = true;
      }
   }
   if (anyCopy) {
      if ((e = cudaEventRecord(sl.copied, s->copyStream)) != cudaSuccess) { return cudaFail(e, "server: event"); }
      if ((e = cudaStreamWaitEvent(st, sl.copied, 0)) != cudaSuccess) { return cudaFail(e, "server: wait"); }
   }
   if ((e = cudaEventRecord(sl.start, st)) != cudaSuccess) { return cudaFail(e, "server: event"); }
   // plan every request: word tasks, thermometer tasks, constant maps, single-field fallbacks
   std::vector<FieldTask> tasks[2];
   std::vector<BatchChunk> chunks[2];
   std::vector<WordTask> wtasks[2];
   std::vector<BatchChunk> wchunks[2];
   std::vector<ClearEntry> clears;
   struct Const { uint64_t *out; int row, bin; unsigned long long cells; };
   std::vector<Const> consts;
   struct Single { Request *r; MKFFieldDesc d; };
   std::vector<Single> singles;
   constexpr int kChunk = 64;
   for (Request *r : sl.reqs) {
      MKFFieldDesc d = r->field;
      if (r->staged) {
         d.p = r->staged;
         d.stride[0] = d.stride[1] = d.stride[2] = 0;
      }
      MKFThreshSet ts;
      ts.nT = (int32_t)r->t.size();
      ts.mAll = r->mAll;
      ts.t = r->t.data();
      ts.m = r->m.empty() ? nullptr : r->m.data();
      clears.push_back({r->dCounts, (long long)ts.nT * 256});
      const unsigned long long cells =
         (unsigned long long)(d.def[0] - 1) * (unsigned long long)(d.def[1] - 1) * (unsigned long long)(d.def[2] - 1);
      FieldTask t;
      WordTask w;
      std::vector<ConstEntry> ce;
      bool varying = false;
      const int kind = planBatchField(&d, &ts, 0, t, w, ce, varying, -1);  // depth by field size
      if (cells == 0) { continue; }
      if (kind == kPlanSingle && varying) {
         singles.push_back({r, d});  // counts every threshold, constant maps included
         continue;
      }
      for (const ConstEntry &c : ce) { consts.push_back({r->dCounts, c.row, c.bin, cells}); }
      if (kind == kPlanWords) {
         const int k = d.enc == ENC_F32 ? 0 : 1;
         const int f = (int)wtasks[k].size();
         for (long long b = 0; b < w.nItems; b += kChunk) { wchunks[k].push_back({f, 0, b, std::min<long long>(b + kChunk, w.nItems)}); }
         w.out = r->dCounts;
         wtasks[k].push_back(w);
      } else if (kind == kPlanThermo) {
         const int k = d.enc == ENC_F32 ? 0 : 1;
         const int f = (int)tasks[k].size();
         for (long long b = 0; b < t.nItems; b += kChunk) { chunks[k].push_back({f, 0, b, std::min<long long>(b + kChunk, t.nItems)}); }
         t.out = r->dCounts;
         tasks[k].push_back(t);
      }
   }
   std::vector<ThermoGroup> groups[2];  // thermometer chunks sorted into one run per kernel variant
   for (int k = 0; k < 2; k++) {
      if (!chunks[k].empty()) { groups[k] = groupThermoChunks(chunks[k], tasks[k]); }
   }
   // one upload of the whole work list, segments 256-byte aligned:
   // clears | thermometer tasks, chunks (FP32, FP64) | word tasks, chunks (FP32, FP64)
   struct Seg { const void *src; size_t bytes; size_t off; };
   Seg seg[9] = {{clears.data(), clears.size() * sizeof(ClearEntry), 0},
                 {tasks[0].data(), tasks[0].size() * sizeof(FieldTask), 0},
                 {chunks[0].data(), chunks[0].size() * sizeof(BatchChunk), 0},
                 {tasks[1].data(), tasks[1].size() * sizeof(FieldTask), 0},
                 {chunks[1].data(), chunks[1].size() * sizeof(BatchChunk), 0},
                 {wtasks[0].data(), wtasks[0].size() * sizeof(WordTask), 0},
                 {wchunks[0].data(), wchunks[0].size() * sizeof(BatchChunk), 0},
                 {wtasks[1].data(), wtasks[1].size() * sizeof(WordTask), 0},
                 {wchunks[1].data(), wchunks[1].size() * sizeof(BatchChunk), 0}};
   size_t total = 0;
   for (Seg &g : seg) {
      g.off = total;
      total += (g.bytes + 255) & ~(size_t)255;
   }
   if ((e = sl.work.ensure(total)) != cudaSuccess) { return cudaFail(e, "server: work list buffers"); }
   char *h = (char *)sl.work.h, *dv = (char *)sl.work.d;
   for (const Seg &g : seg) {
      if (g.bytes) { memcpy(h + g.off, g.src, g.bytes); }
   }
   if ((e = cudaMemcpyAsync(dv, h, total, cudaMemcpyHostToDevice, st)) != cudaSuccess) { return cudaFail(e, "server: work list upload"); }
   if ((e = cudaMemsetAsync(sl.counters, 0, kServerCounters * sizeof(unsigned), st)) != cudaSuccess) {
      return cudaFail(e, "server: counters");
   }
   if (!clears.empty()) {
      clearCounts<<<(unsigned)std::min<size_t>(clears.size(), 1024), 256, 0, st>>>((const ClearEntry *)(dv + seg[0].off), (int)clears.size());
      if ((e = cudaGetLastError()) != cudaSuccess) { return cudaFail(e, "server: clear launch"); }
   }
   int rc = MKF_OK;
   for (size_t i = 0; i < consts.size() && rc == MKF_OK; i++) {
      rc = launchConstBin(consts[i].out, consts[i].row, consts[i].bin, consts[i].cells, st);
   }
   for (int k = 0; k < 2 && rc == MKF_OK; k++) {
      if (wchunks[k].empty()) { continue; }
      WordBatchArgs w;
      w.tasks = (const WordTask *)(dv + seg[5 + 2 * k].off);
      w.chunks = (const BatchChunk *)(dv + seg[6 + 2 * k].off);
      w.nChunks = (int)wchunks[k].size();
      w.counter = sl.counters + k;
      rc = launchWordsBatch(w, k == 0 ? ENC_F32 : ENC_F64, st);
   }
   for (int k = 0; k < 2 && rc == MKF_OK; k++) {
      if (chunks[k].empty()) { continue; }
      rc = launchThermoGroups((const FieldTask *)(dv + seg[1 + 2 * k].off), (const BatchChunk *)(dv + seg[2 + 2 * k].off),
                              groups[k], sl.counters + 2 + k * kThVariants, k == 0 ? ENC_F32 : ENC_F64, st);
   }
   for (size_t i = 0; i < singles.size() && rc == MKF_OK; i++) {
      Request *r = singles[i].r;
      MKFThreshSet ts;
      ts.nT = (int32_t)r->t.size();
      ts.mAll = r->mAll;
      ts.t = r->t.data();
      ts.m = r->m.empty() ? nullptr : r->m.data();
      rc = fieldBPFD(r->dCounts, &singles[i].d, &ts, MKF_F_ACCUMULATE, st, nullptr);
   }
   if (rc != MKF_OK) { return rc; }
   // counts wanted on the host: one pinned buffer per launch, copied out at completion
   size_t hostBytes = 0;
   for (Request *r : sl.reqs) {
      if (r->hostOut) {
         r->hostSlot = hostBytes;
         hostBytes += r->countBytes;
      }
   }
   if (hostBytes) {
      if ((e = sl.results.ensure(hostBytes)) != cudaSuccess) { return cudaFail(e, "server: result buffers"); }
      for (Request *r : sl.reqs) {
         if (r->hostOut) {
            e = cudaMemcpyAsync((char *)sl.results.h + r->hostSlot, r->dCounts, r->countBytes, cudaMemcpyDeviceToHost, st);
            if (e != cudaSuccess) { return cudaFail(e, "server: result copy"); }
         }
      }
   }
   if ((e = cudaEventRecord(sl.done, st)) != cudaSuccess) { return cudaFail(e, "server: event"); }
   return MKF_OK;
}

// A launch finished: hand out the results, give the memory back (worker thread, under s->mu).
static void completeLaunch(MKFServer *s, LaunchSlot &sl, int rc, const char *msg)
{
   float ms = 0.0f;
   if (rc == MKF_OK && cudaEventElapsedTime(&ms, sl.start, sl.done) == cudaSuccess) { s->launchDeviceSec += 1e-3 * ms; }
   cudaGetLastError();
   for (Request *r : sl.reqs) {
      if (r->staged) {
         s->arena.release(r->staged, r->fieldBytes);
         r->staged = nullptr;
      }
      if (rc == MKF_OK && r->hostOut) {
         memcpy(r->hostOut, (char *)sl.results.h + r->hostSlot, r->countBytes);
      }
      if (r->hostOut || rc != MKF_OK) {
         s->arena.release(r->dCounts, r->countBytes);
         r->dCounts = nullptr;
      }
      finishRequest(s, r, rc, msg);
      if (rc == MKF_OK) {
         s->latency.push_back(std::chrono::duration<double>(r->tDone - r->tSubmit).count());
      } else {
         s->failed++;
      }
   }
   sl.reqs.clear();
   sl.busy = false;
}

static void workerLoop(MKFServer *s)
{
   cudaSetDevice(s->device);
   std::deque<Request *> pending;
   for (;;) {
      bool progress = false;
      {
         std::unique_lock<std::mutex> lk(s->mu);
         while (!s->incoming.empty()) {
            pending.push_back(s->incoming.front());
            s->incoming.pop_front();
         }
         // completions
         bool anyDone = false;
         for (LaunchSlot &sl : s->slots) {
            if (!sl.busy) { continue; }
            const cudaError_t q = cudaEventQuery(sl.done);
            if (q == cudaErrorNotReady) { continue; }
            if (q == cudaSuccess) {
               completeLaunch(s, sl, MKF_OK, nullptr);
            } else {
               const std::string m = std::string("server: launch failed: ") + cudaGetErrorString(q);
               completeLaunch(s, sl, MKF_ERR_CUDA, m.c_str());
            }
            anyDone = progress = true;
         }
         if (anyDone) { s->cvDone.notify_all(); }
         const bool idle = !s->slots[0].busy && !s->slots[1].busy;
         if (s->stop && pending.empty() && idle) { break; }
         // admission into a free slot: requests in arrival order while the budget allows
         LaunchSlot *sl = !s->slots[0].busy ? &s->slots[0] : (!s->slots[1].busy ? &s->slots[1] : nullptr);
         if (sl && !pending.empty()) {
            while (!pending.empty() && (int)sl->reqs.size() < s->maxPerLaunch) {
               Request *r = pending.front();
               const size_t need = Arena::round(r->countBytes) + Arena::round(r->fieldBytes);
               if (need > s->arena.size()) {
                  pending.pop_front();
                  finishRequest(s, r, MKF_ERR_NOMEM, "server: request larger than the device-memory budget");
                  s->failed++;
                  anyDone = true;
                  continue;
               }
               r->dCounts = (uint64_t *)s->arena.alloc(r->countBytes);
               if (r->dCounts && r->fieldBytes) {
                  r->staged = s->arena.alloc(r->fieldBytes);
                  if (!r->staged) {
                     s->arena.release(r->dCounts, r->countBytes);
                     r->dCounts = nullptr;
                  }
               }
               if (!r->dCounts) { break; }  // wait until a launch completes and frees memory
               pending.pop_front();
               r->state = kRunning;
               sl->reqs.push_back(r);
            }
            if (s->stop && sl->reqs.empty() && !s->slots[0].busy && !s->slots[1].busy) {
               // shutting down, nothing in flight and the head still does not fit: the memory is
               // held by counts the client never released, so the rest can never be admitted
               while (!pending.empty()) {
                  finishRequest(s, pending.front(), MKF_ERR_BUSY, "server: shut down before the request fitted the budget");
                  s->failed++;
                  pending.pop_front();
               }
               anyDone = true;
            }
            if (anyDone) { s->cvDone.notify_all(); }
            if (!sl->reqs.empty()) {
               sl->busy = true;
               s->launches++;
               s->fieldsLaunched += sl->reqs.size();
               s->maxInLaunch = std::max<uint32_t>(s->maxInLaunch, (uint32_t)sl->reqs.size());
               lk.unlock();
               const Clock::time_point t0 = Clock::now();
               const int rc = issueLaunch(s, *sl);
               const double dt = std::chrono::duration<double>(Clock::now() - t0).count();
               lk.lock();
               s->planHostSec += dt;
               if (rc != MKF_OK) {
                  // nothing of a failed launch is trusted: wait for what was issued, then fail it
                  cudaStreamSynchronize(sl->stream);
                  completeLaunch(s, *sl, rc, mkfLastError());
                  s->cvDone.notify_all();
               }
               progress = true;
            }
         }
         if (!progress) {
            // nothing to do now: sleep until a submission, or briefly while launches run
            const bool running = s->slots[0].busy || s->slots[1].busy;
            if (running || !pending.empty()) {
               s->cvWork.wait_for(lk, std::chrono::microseconds(20));
            } else {
               s->cvWork.wait_for(lk, std::chrono::milliseconds(5));
            }
         }
      }
   }
}

}  // namespace mkf

MKF_API int mkfServerCreate(MKFServer **ps, const MKFServerConfig *cfg)
{
   if (!ps) { setError("mkfServerCreate: NULL argument"); return MKF_ERR_ARG; }
   *ps = nullptr;
   MKFServer *s = new MKFServer();
   size_t budget = cfg && cfg->hbmBudget ? (size_t)cfg->hbmBudget : ((size_t)64 << 30);
   s->maxPerLaunch = cfg && cfg->maxFieldsPerLaunch > 0 ? cfg->maxFieldsPerLaunch : 256;
   s->device = cfg ? cfg->device : 0;
   cudaError_t e = cudaSetDevice(s->device);
   if (e == cudaSuccess) { e = cudaMalloc(&s->budgetMem, budget); }
   if (e == cudaSuccess) { s->arena.init(s->budgetMem, budget); }
   if (e == cudaSuccess) { e = cudaStreamCreateWithFlags(&s->copyStream, cudaStreamNonBlocking); }
   for (LaunchSlot &sl : s->slots) {
      if (e == cudaSuccess) { e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking); }
      if (e == cudaSuccess) { e = cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming); }
      if (e == cudaSuccess) { e = cudaEventCreate(&sl.start); }
      if (e == cudaSuccess) { e = cudaEventCreate(&sl.done); }
      if (e == cudaSuccess) { e = cudaMalloc(&sl.counters, kServerCounters * sizeof(unsigned)); }
   }
   if (e != cudaSuccess) {
      const int rc = cudaFail(e, "mkfServerCreate");
      mkfServerDestroy(s);
      return e == cudaErrorMemoryAllocation ? MKF_ERR_NOMEM : rc;
   }
   s->worker = std::thread(workerLoop, s);
   *ps = s;
   return MKF_OK;
}

MKF_API int mkfServerSubmit(MKFServer *s, const MKFRequest *req, uint64_t *ticket)
{
   if (!s || !req || !ticket) { setError("mkfServerSubmit: NULL argument"); return MKF_ERR_ARG; }
   const MKFFieldDesc &f = req->field;
   const MKFThreshSet &ts = req->thresh;
   if (!f.p || (f.enc != ENC_F32 && f.enc != ENC_F64) || f.def[0] < 1 || f.def[1] < 1 || f.def[2] < 1 || !ts.t ||
       ts.nT < 1 || ts.nT > MKF_MAX_THRESH) {
      setError("mkfServerSubmit: bad field descriptor or thresholds");
      return MKF_ERR_ARG;
   }
   const bool host = (req->flags & MKF_REQ_HOST_FIELD) != 0;
   if (host && (f.stride[0] | f.stride[1] | f.stride[2])) {
      setError("mkfServerSubmit: host fields must be planar (stride all zero)");
      return MKF_ERR_UNSUPPORTED;
   }
   Request *r = new Request();
   r->field = f;
   r->t.assign(ts.t, ts.t + ts.nT);
   if (ts.m) { r->m.assign(ts.m, ts.m + ts.nT); }
   r->mAll = ts.mAll;
   r->flags = req->flags;
   r->hostOut = req->hostOut;
   r->countBytes = (size_t)ts.nT * 256 * sizeof(uint64_t);
   if (host) {
      r->fieldBytes = (size_t)f.def[0] * (size_t)f.def[1] * (size_t)f.def[2] * (f.enc == ENC_F32 ? 4 : 8);
   }
   r->tSubmit = Clock::now();
   {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->stop) {
         delete r;
         setError("mkfServerSubmit: server is shutting down");
         return MKF_ERR_BUSY;
      }
      r->ticket = s->nextTicket++;
      s->byTicket[r->ticket] = r;
      s->incoming.push_back(r);
   }
   s->cvWork.notify_one();
   *ticket = r->ticket;
   return MKF_OK;
}

MKF_API int mkfServerWait(MKFServer *s, uint64_t ticket, double timeoutSec, const uint64_t **pDevCounts, double *latencySec)
{
   if (!s) { setError("mkfServerWait: NULL server"); return MKF_ERR_ARG; }
   std::unique_lock<std::mutex> lk(s->mu);
   auto it = s->byTicket.find(ticket);
   if (it == s->byTicket.end()) { setError("mkfServerWait: unknown ticket %llu", (unsigned long long)ticket); return MKF_ERR_NOTFOUND; }
   Request *r = it->second;
   const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(std::max(0.0, timeoutSec)));
   while (r->state != kDone) {
      if (s->cvDone.wait_until(lk, until) == std::cv_status::timeout && r->state != kDone) {
         setError("mkfServerWait: ticket %llu not done within %.3f s", (unsigned long long)ticket, timeoutSec);
         return MKF_ERR_TIMEOUT;
      }
   }
   if (pDevCounts) { *pDevCounts = r->dCounts; }
   if (latencySec) { *latencySec = std::chrono::duration<double>(r->tDone - r->tSubmit).count(); }
   if (r->rc != MKF_OK) { setError("%s", r->err.c_str()); }
   return r->rc;
}

MKF_API int mkfServerCopyCounts(MKFServer *s, uint64_t ticket, uint64_t *dst, void *stream)
{
   if (!s || !dst) { setError("mkfServerCopyCounts: NULL argument"); return MKF_ERR_ARG; }
   const uint64_t *src = nullptr;
   size_t bytes = 0;
   {
      std::lock_guard<std::mutex> lk(s->mu);
      auto it = s->byTicket.find(ticket);
      if (it == s->byTicket.end()) { setError("mkfServerCopyCounts: unknown ticket"); return MKF_ERR_NOTFOUND; }
      Request *r = it->second;
      if (r->state != kDone || r->rc != MKF_OK || !r->dCounts) {
         setError("mkfServerCopyCounts: ticket %llu has no device counts", (unsigned long long)ticket);
         return MKF_ERR_ARG;
      }
      src = r->dCounts;
      bytes = r->countBytes;
   }
   cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, (cudaStream_t)stream);
   if (e == cudaSuccess) { e = cudaStreamSynchronize((cudaStream_t)stream); }
   return e == cudaSuccess ? MKF_OK : cudaFail(e, "mkfServerCopyCounts");
}

MKF_API int mkfServerRelease(MKFServer *s, uint64_t ticket)
{
   if (!s) { setError("mkfServerRelease: NULL server"); return MKF_ERR_ARG; }
   std::lock_guard<std::mutex> lk(s->mu);
   auto it = s->byTicket.find(ticket);
   if (it == s->byTicket.end()) { setError("mkfServerRelease: unknown ticket"); return MKF_ERR_NOTFOUND; }
   Request *r = it->second;
   if (r->state != kDone) { setError("mkfServerRelease: ticket %llu still in flight", (unsigned long long)ticket); return MKF_ERR_BUSY; }
   if (r->dCounts) { s->arena.release(r->dCounts, r->countBytes); }
   s->byTicket.erase(it);
   delete r;
   s->cvWork.notify_one();  // freed memory may admit a waiting request
   return MKF_OK;
}

MKF_API int mkfServerStats(MKFServer *s, MKFServerStats *st, int reset)
{
   if (!s || !st) { setError("mkfServerStats: NULL argument"); return MKF_ERR_ARG; }
   std::lock_guard<std::mutex> lk(s->mu);
   memset(st, 0, sizeof(*st));
   std::vector<double> v = s->latency;
   st->completed = v.size();
   st->failed = s->failed;
   st->launches = s->launches;
   st->maxFieldsInLaunch = s->maxInLaunch;
   st->meanFieldsInLaunch = s->launches ? (double)s->fieldsLaunched / (double)s->launches : 0.0;
   st->deviceBytesInUse = s->arena.used();
   st->launchDeviceSec = s->launchDeviceSec;
   st->planHostSec = s->planHostSec;
   if (!v.empty()) {
      std::sort(v.begin(), v.end());
      auto q = [&](double p) { return v[std::min(v.size() - 1, (size_t)(p * (double)(v.size() - 1) + 0.5))]; };
      st->p50 = q(0.50);
      st->p99 = q(0.99);
      double sum = 0;
      for (double x : v) { sum += x; }
      st->mean = sum / (double)v.size();
      st->max = v.back();
   }
   if (reset) {
      s->latency.clear();
      s->failed = s->launches = s->fieldsLaunched = 0;
      s->launchDeviceSec = s->planHostSec = 0.0;
      s->maxInLaunch = 0;
   }
   return MKF_OK;
}

MKF_API int mkfServerDestroy(MKFServer *s)
{
   if (!s) { return MKF_OK; }
   {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stop = true;
   }
   s->cvWork.notify_all();
   if (s->worker.joinable()) { s->worker.join(); }
   for (auto &kv : s->byTicket) { delete kv.second; }
   s->byTicket.clear();
   for (LaunchSlot &sl : s->slots) {
      if (sl.stream) { cudaStreamDestroy(sl.stream); }
      if (sl.copied) { cudaEventDestroy(sl.copied); }
      if (sl.done) { cudaEventDestroy(sl.done); }
      if (sl.start) { cudaEventDestroy(sl.start); }
      if (sl.counters) { cudaFree(sl.counters); }
      sl.work.destroy();
      sl.results.destroy();
   }
   if (s->copyStream) { cudaStreamDestroy(s->copyStream); }
   if (s->budgetMem) { cudaFree(s->budgetMem); }
   delete s;
   return MKF_OK;
}
