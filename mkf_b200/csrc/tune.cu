// tune.cu - slab depth and kernel variant chosen by measurement.
//
// The best slab depth (planes of cells per work item) depends on the kernel, the element type, the
// threshold count and the field's extent: deep slabs save halo re-reads on large fields, shallow
// ones give small fields enough work items to fill 148 SMs. The TMA-staged rank-table kernel also
// comes in variants of CTA shape (warps per CTA with the depth of their tile rings) and histogram
// privatisation (one or two copies). mkfTune times the candidates on a caller's field and
// remembers the fastest for fields of the same kind (kernel family, element type, threshold count,
// and the power-of-two size class of each extent, which includes the row width); later
// single-field calls on such fields use it. Batch plans time whole candidate plans when they are
// created (mkfSetTuning switches that off).
#include <algorithm>
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

struct TuneVal
{
   int depth, variant;
};

static int log2Class(int n)
{
   int b = 0;
   while ((1 << (b + 1)) <= n && b < 30) { ++b; }
   return b;
}

static constexpr int kVariantsOf[3] = {1, 1, kTmNumVariants};  // variants per family (words, rank table, TMA rank table)

static std::mutex gTuneMu;
static std::map<TuneKey, TuneVal> gTuned;
static bool gBatchTuning = true;
// on this thread while mkfTune / mkfTuneSet / mkfTuneQuery run: the depth and variant every launch
// uses (0 / -1: not forced), and the kinds of launch made
static thread_local int tForce = 0, tForceVariant = -1;
static thread_local std::vector<TuneKey> *tSeen = nullptr;

static TuneKey keyOf(int family, int enc, int K, int X, int Y, int Z)
{
   return TuneKey{family, enc, K, log2Class(X), log2Class(Y), log2Class(Z)};
}

int tunedDepth(int family, int enc, int K, int X, int Y, int Z, int def)
{
   const TuneKey key = keyOf(family, enc, K, X, Y, Z);
   if (tSeen) { tSeen->push_back(key); }
   if (tForce > 0) { return tForce; }
   std::lock_guard<std::mutex> lk(gTuneMu);
   auto it = gTuned.find(key);
   return (it == gTuned.end() || it->second.depth <= 0) ? def : it->second.depth;
}

int tunedVariant(int family, int enc, int K, int X, int Y, int Z, int def)
{
   const int nv = (family >= 0 && family < 3) ? kVariantsOf[family] : 1;
   if (tForceVariant >= 0) { return tForceVariant < nv ? tForceVariant : 0; }
   std::lock_guard<std::mutex> lk(gTuneMu);
   auto it = gTuned.find(keyOf(family, enc, K, X, Y, Z));
   return (it == gTuned.end() || it->second.variant >= nv) ? def : it->second.variant;
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

// One counting run of the field into a scratch buffer with depth / variant forced (0 / -1: not),
// recording the kinds of launch it made; optionally timed (best of `reps`, ms).
static int runOnce(const MKFFieldDesc *pF, const MKFThreshSet *pT, uint64_t *tmp, cudaStream_t s, int depth, int variant,
                   std::vector<TuneKey> *seen, int reps, cudaEvent_t e0, cudaEvent_t e1, float *best)
{
   tForce = depth;
   tForceVariant = variant;
   tSeen = seen;
   if (seen) { seen->clear(); }
   int rc = fieldBPFD(tmp, pF, pT, 0, s, nullptr);  // warm-up (and the launch kinds)
   tSeen = nullptr;
   for (int rep = 0; rep < reps && rc == MKF_OK; rep++) {
      cudaError_t e = cudaEventRecord(e0, s);
      if (e == cudaSuccess) { rc = fieldBPFD(tmp, pF, pT, 0, s, nullptr); }
      if (rc == MKF_OK && e == cudaSuccess) { e = cudaEventRecord(e1, s); }
      if (rc == MKF_OK && e == cudaSuccess) { e = cudaEventSynchronize(e1); }
      float t = 0.0f;
      if (rc == MKF_OK && e == cudaSuccess) { e = cudaEventElapsedTime(&t, e0, e1); }
      if (e != cudaSuccess && rc == MKF_OK) { rc = cudaFail(e, "mkfTune: timing"); }
      if (rc == MKF_OK) { *best = (rep == 0) ? t : std::min(*best, t); }
   }
   if (rc == MKF_OK && reps == 0) { rc = cudaFail(cudaStreamSynchronize(s), "mkfTune: run"); }
   tForce = 0;
   tForceVariant = -1;
   return rc;
}

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
   // the kinds of launch this field takes, and how many variants the richest of them has
   std::vector<TuneKey> seen;
   float ms = 0.0f;
   if (rc == MKF_OK) { rc = runOnce(pF, pT, tmp, s, kCand[0], 0, &seen, 0, e0, e1, &ms); }
   int nVar = 1;
   for (const TuneKey &k : seen) { nVar = std::max(nVar, (k.family >= 0 && k.family < 3) ? kVariantsOf[k.family] : 1); }
   float best = 0.0f;
   int bestD = 0, bestV = 0;
   for (int v = 0; v < nVar && rc == MKF_OK; v++) {
      for (int c = 0; c < 6 && rc == MKF_OK; c++) {
         rc = runOnce(pF, pT, tmp, s, kCand[c], v, nullptr, 2, e0, e1, &ms);
         if (rc == MKF_OK && (bestD == 0 || ms < best)) {
            best = ms;
            bestD = kCand[c];
            bestV = v;
         }
      }
   }
   if (rc == MKF_OK && bestD > 0) {
      std::lock_guard<std::mutex> lk(gTuneMu);
      for (const TuneKey &k : seen) { gTuned[k] = TuneVal{bestD, k.family < 3 && bestV < kVariantsOf[k.family] ? bestV : 0}; }
   }
   if (tmp) { cudaFree(tmp); }
   if (e0) { cudaEventDestroy(e0); }
   if (e1) { cudaEventDestroy(e1); }
   return rc;
}

MKF_API int mkfTuneSet(const MKFFieldDesc *pF, const MKFThreshSet *pT, int depth, int variant, void *stream)
{
   if (!pF || !pT || pT->nT < 1 || pT->nT > MKF_MAX_THRESH || depth < 0 || depth > 255 || variant < 0 || variant > 15) {
      setError("mkfTuneSet: bad argument");
      return MKF_ERR_ARG;
   }
   cudaStream_t s = (cudaStream_t)stream;
   uint64_t *tmp = nullptr;
   cudaError_t e = cudaMalloc(&tmp, (size_t)pT->nT * 256 * sizeof(uint64_t));
   if (e != cudaSuccess) { return cudaFail(e, "mkfTuneSet: set-up"); }
   std::vector<TuneKey> seen;
   float ms = 0.0f;
   int rc = runOnce(pF, pT, tmp, s, depth > 0 ? depth : 4, 0, &seen, 0, nullptr, nullptr, &ms);
   if (rc == MKF_OK) {
      std::lock_guard<std::mutex> lk(gTuneMu);
      for (const TuneKey &k : seen) {
         if (depth > 0) {
            gTuned[k] = TuneVal{depth, k.family < 3 && variant < kVariantsOf[k.family] ? variant : 0};
         } else {
            gTuned.erase(k);
         }
      }
   }
   cudaFree(tmp);
   return rc;
}

MKF_API int mkfTuneQuery(const MKFFieldDesc *pF, const MKFThreshSet *pT, int *depth, int *variant, void *stream)
{
   if (!pF || !pT || !depth || !variant || pT->nT < 1 || pT->nT > MKF_MAX_THRESH) {
      setError("mkfTuneQuery: bad argument");
      return MKF_ERR_ARG;
   }
   cudaStream_t s = (cudaStream_t)stream;
   uint64_t *tmp = nullptr;
   cudaError_t e = cudaMalloc(&tmp, (size_t)pT->nT * 256 * sizeof(uint64_t));
   if (e != cudaSuccess) { return cudaFail(e, "mkfTuneQuery: set-up"); }
   std::vector<TuneKey> seen;
   float ms = 0.0f;
   const int rc = runOnce(pF, pT, tmp, s, 0, -1, &seen, 0, nullptr, nullptr, &ms);
   *depth = 0;
   *variant = 0;
   if (rc == MKF_OK) {
      std::lock_guard<std::mutex> lk(gTuneMu);
      for (const TuneKey &k : seen) {
         auto it = gTuned.find(k);
         if (it != gTuned.end()) {
            *depth = it->second.depth;
            *variant = it->second.variant;
            break;
         }
      }
   }
   cudaFree(tmp);
   return rc;
}
