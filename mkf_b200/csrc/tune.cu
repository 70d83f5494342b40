// tune.cu - slab depth (planes of cells per work item) chosen by measurement.
//
// The best depth depends on the kernel, the element type, the threshold count and the field's
// extent: deep slabs save halo re-reads on large fields, shallow ones give small fields enough work
// items to fill 148 SMs. mkfTune times the candidate depths on a caller's field and remembers the
// fastest for fields of the same kind (kernel family, element type, threshold count, and the
// power-of-two size class of each extent); later single-field calls on such fields use it. Batch
// plans time whole candidate plans when they are created (mkfSetTuning switches that off).
#include <map>
#include <mutex>
#include <tuple>
#include <vector>
#include "fused.cuh"

namespace mkf {

struct TuneKey
{
   int family, enc, K, xb, yb, zb;
   bool operator<(const TuneKey &o) const
   {
      return std::tie(family, enc, K, xb, yb, zb) < std::tie(o.family, o.enc, o.K, o.xb, o.yb, o.zb);
   }
};

static int log2Class(int n)
{
   int b = 0;
   while ((1 << (b + 1)) <= n && b < 30) { ++b; }
   return b;
}

static std::mutex gTuneMu;
static std::map<TuneKey, int> gTuned;
static bool gBatchTuning = true;
// while mkfTune runs on this thread: the depth every launch uses, and the kinds of launch it made
static thread_local int tForce = 0;
static thread_local std::vector<TuneKey> *tSeen = nullptr;

int tunedDepth(int family, int enc, int K, int X, int Y, int Z, int def)
{
   const TuneKey key{family, enc, K, log2Class(X), log2Class(Y), log2Class(Z)};
   if (tForce > 0) {
      if (tSeen) { tSeen->push_back(key); }
      return tForce;
   }
   std::lock_guard<std::mutex> lk(gTuneMu);
   auto it = gTuned.find(key);
   return it == gTuned.end() ? def : it->second;
}

int sizeDepth(int def, long long itemsPerPlane, int Z, long long minItems)
{
   int D = def;
   while (D > 4 && itemsPerPlane * ((Z - 1 + D - 1) / D) < minItems) { D >>= 1; }
   return D;
}

bool batchTuning()
{
   std::lock_guard<std::mutex> lk(gTuneMu);
   return gBatchTuning;
}

int fieldBPFD(uint64_t *out, const MKFFieldDesc *pF, const MKFThreshSet *pT, int flags, cudaStream_t s, const int *rowBase);

}  // namespace mkf

using namespace mkf;

MKF_API int mkfSetTuning(int batchPlans)
{
   std::lock_guard<std::mutex> lk(gTuneMu);
   const int prev = gBatchTuning ? 1 : 0;
   gBatchTuning = batchPlans != 0;
   return prev;
}

MKF_API int mkfTune(const MKFFieldDesc *pF, const MKFThreshSet *pT, void *stream)
{
   if (!pF || !pT || pT->nT < 1 || pT->nT > MKF_MAX_THRESH) { setError("mkfTune: bad argument"); return MKF_ERR_ARG; }
   cudaStream_t s = (cudaStream_t)stream;
   uint64_t *tmp = nullptr;
   cudaEvent_t e0 = nullptr, e1 = nullptr;
   cudaError_t e = cudaMalloc(&tmp, (size_t)pT->nT * 256 * sizeof(uint64_t));
   if (e == cudaSuccess) { e = cudaEventCreate(&e0); }
   if (e == cudaSuccess) { e = cudaEventCreate(&e1); }
   int rc = (e == cudaSuccess) ? MKF_OK : cudaFail(e, "mkfTune: set-up");
   static const int kCand[] = {4, 8, 16, 32, 64, 128};
   float best = 0.0f;
   int bestD = 0;
   std::vector<TuneKey> seen;
   for (int c = 0; c < 6 && rc == MKF_OK; c++) {
      tForce = kCand[c];
      tSeen = &seen;
      seen.clear();
      rc = fieldBPFD(tmp, pF, pT, 0, s, nullptr);  // warm-up (and records the launch kinds)
      float ms = 0.0f;
      for (int rep = 0; rep < 2 && rc == MKF_OK; rep++) {
         e = cudaEventRecord(e0, s);
         if (e == cudaSuccess) { rc = fieldBPFD(tmp, pF, pT, 0, s, nullptr); }
         if (rc == MKF_OK && e == cudaSuccess) { e = cudaEventRecord(e1, s); }
         if (rc == MKF_OK && e == cudaSuccess) { e = cudaEventSynchronize(e1); }
         float t = 0.0f;
         if (rc == MKF_OK && e == cudaSuccess) { e = cudaEventElapsedTime(&t, e0, e1); }
         if (e != cudaSuccess && rc == MKF_OK) { rc = cudaFail(e, "mkfTune: timing"); }
         ms = (rep == 0) ? t : std::min(ms, t);
      }
      if (rc == MKF_OK && (bestD == 0 || ms < best)) {
         best = ms;
         bestD = kCand[c];
      }
   }
   tForce = 0;
   tSeen = nullptr;
   if (rc == MKF_OK && bestD > 0) {
      std::lock_guard<std::mutex> lk(gTuneMu);
      for (const TuneKey &k : seen) { gTuned[k] = bestD; }
   }
   if (tmp) { cudaFree(tmp); }
   if (e0) { cudaEventDestroy(e0); }
   if (e1) { cudaEventDestroy(e1); }
   return rc;
}

MKF_API int mkfTuneSet(const MKFFieldDesc *pF, const MKFThreshSet *pT, int depth, void *stream)
{
   if (!pF || !pT || pT->nT < 1 || pT->nT > MKF_MAX_THRESH || depth < 0 || depth > 255) {
      setError("mkfTuneSet: bad argument");
      return MKF_ERR_ARG;
   }
   cudaStream_t s = (cudaStream_t)stream;
   uint64_t *tmp = nullptr;
   cudaError_t e = cudaMalloc(&tmp, (size_t)pT->nT * 256 * sizeof(uint64_t));
   if (e != cudaSuccess) { return cudaFail(e, "mkfTuneSet: set-up"); }
   // one counting run learns the kinds of launch this field takes
   std::vector<TuneKey> seen;
   tForce = depth > 0 ? depth : 4;
   tSeen = &seen;
   int rc = fieldBPFD(tmp, pF, pT, 0, s, nullptr);
   tForce = 0;
   tSeen = nullptr;
   if (rc == MKF_OK) { rc = cudaFail(cudaStreamSynchronize(s), "mkfTuneSet: run"); }
   if (rc == MKF_OK) {
      std::lock_guard<std::mutex> lk(gTuneMu);
      for (const TuneKey &k : seen) {
         if (depth > 0) { gTuned[k] = depth; } else { gTuned.erase(k); }
      }
   }
   cudaFree(tmp);
   return rc;
}
