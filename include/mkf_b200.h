/* mkf_b200.h - entry points that libMKF.so adds beside the original MKF interface.
 *
 * The original library handles one threshold per call and goes through a packed binary map in
 * device memory. These calls fuse threshold -> pattern code -> histogram into one read of the
 * field, take up to MKF_MAX_THRESH thresholds at once, run many fields in one launch, and
 * return status codes instead of NULL. None of them has a counterpart in the original: the
 * closest original calls are named beside each one.
 *
 * Conventions
 *   - Pointers marked "device" must be CUDA device (or managed) memory of the current device.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream). Calls are
 *     asynchronous with respect to the host unless stated otherwise.
 *   - Returns MKF_OK (0) or a negative MKF_ERR_* code; mkfLastError() gives a message.
 *   - Pattern counts are uint64_t[256] per threshold, laid out [threshold][pattern]. The pattern
 *     code of the cell at (x,y,z) has bit i set when corner (x + (i&1), y + ((i>>1)&1),
 *     z + ((i>>2)&1)) maps to 1, as in the original (bpfdCUDA.cuh:45-61).
 *   - Every row of X elements contributes X-1 cells. The original counts 2X-1 cells for rows
 *     with X < 32, its two counting paths differently (bpfdCUDA.cuh:112-116 re-reads the row's
 *     first word, mkfACC.c:137-150 reads the next row's), so there the counts differ from it.
 */
#ifndef MKF_B200_H
#define MKF_B200_H
#include "mkf_types.h"
#ifdef __cplusplus
extern "C" {
#endif

#define MKF_OK               0
#define MKF_ERR_ARG         -1   /* invalid argument */
#define MKF_ERR_CUDA        -2   /* a CUDA call failed */
#define MKF_ERR_NOMEM       -3   /* allocation failed or over budget */
#define MKF_ERR_TIMEOUT     -4   /* a bounded wait ran out */
#define MKF_ERR_UNSUPPORTED -5   /* encoding / size not supported */
#define MKF_ERR_BUSY        -6   /* queue full, try again */
#define MKF_ERR_NOTFOUND    -7   /* unknown request tag */

#define MKF_MAX_THRESH 32

/* flags */
#define MKF_F_ACCUMULATE 0x1 /* add to the output counts instead of overwriting them */

/* One scalar field. stride[] holds element strides for x, y, z; all zero means planar
 * (x fastest, no padding). enc is ENC_F32 or ENC_F64. */
typedef struct
{
   const void *p;
   NumEnc enc;
   uint8_t pad_[3];
   int32_t def[3];
   int64_t stride[3];
} MKFFieldDesc;

/* A set of thresholds. Threshold k maps f to ((m_k >> (1 - (f < t_k) + (f > t_k))) & 1), with the
 * comparison done exactly (a FP32 field is compared as if promoted to double, so thresholds are
 * never rounded). m may be NULL, then every threshold uses mAll. */
typedef struct
{
   int32_t nT;          /* 1 .. MKF_MAX_THRESH */
   uint32_t mAll;
   const double *t;     /* host array, nT values, any order */
   const uint32_t *m;   /* host array or NULL */
} MKFThreshSet;

/* Last error message of the calling thread. */
const char *mkfLastError(void);

/* ---- fused single field (closest original: binMapCUDA + mkfCUDAGetBPFD, binMapCUDA.cu:144,
 *      mkfCUDA.cu:12) ---- */
/* One read of the field pF->p (device) gives nT pattern distributions in pBPFD (device,
 * uint64_t[nT][256]). */
int mkfFieldBPFD(uint64_t *pBPFD, const MKFFieldDesc *pF, const MKFThreshSet *pT, int flags, void *stream);

/* The same for one or two thresholds of any relations, with the field's descriptive moments from
 * the same read (the original declares them as the categorical CUDAImgMom, binMapCUDA.cuh:67-128,
 * without calling it): pMom (device, double[nT][2][2]) receives per threshold and per map value
 * (0, 1) the sum of f and the sum of f^2 over the elements, in FP64 (summation order is not fixed,
 * so results may differ in the last bits between runs). Dimensions must be >= 2 each. */
int mkfFieldBPFDMoments(uint64_t *pBPFD, double *pMom, const MKFFieldDesc *pF, const MKFThreshSet *pT, int flags,
                        void *stream);

/* The same from a HOST field: the field is copied in slabs through device staging buffers on a
 * copy stream overlapped with the counting kernel, and the counts are copied back to pBPFDH
 * (host, uint64_t[nT][256]). Synchronous. pF->p may be pageable or pinned host memory. */
int mkfFieldBPFDHost(uint64_t *pBPFDH, const MKFFieldDesc *pF, const MKFThreshSet *pT);

/* The same as mkfFieldBPFDHost, but the library allocates nothing: no cudaMalloc, no pinned
 * buffers, no streams or events. It has no counterpart in the original MKF.
 *   Who needs it: callers that must not let a library allocate device memory, such as an in-situ
 *   analysis inside a simulation whose device memory belongs to the simulation's own pool, or a
 *   process held to a fixed device-memory budget (cudaMalloc would also synchronise the device
 *   in the middle of the caller's overlapped work).
 *   Scratch: two file-scope device arrays of the library, a 32 MiB staging area for field slabs
 *   and 32 x 256 counts; every GPU that loads the library holds them until the process exits.
 *   Limit: the staging area must hold two planes, so a plane (X * Y elements) may be at most
 *   16 MiB (e.g. 2048 x 1024 FP64, 2048 x 2048 FP32); larger planes return MKF_ERR_NOMEM.
 *   The first call on each device resolves the arrays' device addresses (cudaGetSymbolAddress)
 *   with that device current and keeps them for the life of the process; a cudaDeviceReset
 *   reloads the module and moves the arrays, so do not call it after a cudaDeviceReset in the
 *   same process (this library never resets a device).
 *   All calls on a device share the arrays: calls whose work overlaps on the GPU (different
 *   streams, or different host threads) race and give wrong counts. The counts are cleared at
 *   the start of every call; the staging area keeps the last call's data.
 *   Work runs in order on `stream` (NULL = legacy default stream) and the call waits for it, so
 *   it must not be called on a stream that is being captured into a CUDA graph. Returns after
 *   the counts are in pBPFDH (host, uint64_t[nT][256]). pF->p is a planar host field. Kernel
 *   choice as mkfFieldBPFD's; when every threshold is a constant map no field data is copied. */
int mkfFieldBPFDHostNoAlloc(uint64_t *pBPFDH, const MKFFieldDesc *pF, const MKFThreshSet *pT, void *stream);

/* ---- many fields, one launch (no original counterpart; the original runs one field per call) ---- */
/* Fields i = 0..nF-1 (device pointers, any shapes, FP32/FP64) with threshold sets pT[i]; the counts
 * of field i are rows nT_0 + ... + nT_{i-1} onwards of pBPFD (device, overwritten). One persistent
 * launch walks a work list of (field, item chunk) entries; fields whose thresholds mix relations
 * are counted by their own pass. A plan keeps the work list on the device so the same batch (same
 * buffers, new contents) can be launched again, also inside a CUDA graph. */
typedef struct MKFBatchPlan MKFBatchPlan;
/* Unless mkfSetTuning(0) switched it off, creation times one launch of the batch for each candidate
 * slab depth (planes per work item) and keeps the fastest: the fields must hold readable data, and
 * pBPFD is written. Synchronous. */
int mkfBatchPlanCreate(MKFBatchPlan **pPlan, uint64_t *pBPFD, const MKFFieldDesc *pF, const MKFThreshSet *pT, int nF);
/* Clear the counts and count every field, asynchronously on `stream`; issues no allocation and no
 * synchronisation, so it may be captured into a CUDA graph. */
int mkfBatchPlanLaunch(MKFBatchPlan *plan, void *stream);
/* The same through a CUDA graph the plan captures on first use and replays afterwards. */
int mkfBatchPlanLaunchGraph(MKFBatchPlan *plan, void *stream);
int mkfBatchPlanDestroy(MKFBatchPlan *plan);
/* One-shot: create a plan, launch it on `stream`, wait for it and destroy it (synchronous). */
int mkfBatchBPFD(uint64_t *pBPFD, const MKFFieldDesc *pF, const MKFThreshSet *pT, int nF, int flags, void *stream);

/* ---- serving: a request loop for in-situ analysis (no original counterpart) ----
 * Clients (any host threads) submit fields with their thresholds; a worker thread of the server
 * admits requests in arrival order while a device-memory budget allows, copies host fields to
 * the device on a copy stream, and packs every request admitted since the last launch into the
 * next persistent batched launch, while the previous launch may still run (two launch streams).
 * Counts stay in device memory (budget-accounted) until mkfServerRelease, or are copied to
 * hostOut when the request names one. A device field must stay valid and unchanged until its
 * request is done; a host field must be pinned (cudaMallocHost / cudaHostRegister) and planar. */
typedef struct MKFServer MKFServer;
typedef struct
{
   uint64_t hbmBudget;          /* device bytes for staged host fields + counts (0 = 64 GiB) */
   int32_t maxFieldsPerLaunch;  /* 0 = 256 */
   int32_t device;              /* CUDA device ordinal */
} MKFServerConfig;

#define MKF_REQ_HOST_FIELD 0x1  /* field.p is pinned host memory: the server stages it */

typedef struct
{
   MKFFieldDesc field;
   MKFThreshSet thresh;         /* copied at submission */
   uint32_t flags;              /* MKF_REQ_* */
   uint32_t pad_;
   uint64_t *hostOut;           /* optional host uint64_t[nT][256]; then the device counts are freed */
} MKFRequest;

typedef struct
{
   uint64_t completed, failed, launches;  /* since creation or the last reset */
   uint32_t maxFieldsInLaunch, pad_;
   double meanFieldsInLaunch;
   double p50, p99, mean, max;  /* latency in seconds, submission to completion seen by the server */
   uint64_t deviceBytesInUse;   /* budget in use now (staged fields + held counts) */
   double launchDeviceSec;      /* summed device time of the launches, from the last staged field
                                 * copied to the last count written (launches on the two launch
                                 * streams may overlap, so this can exceed wall time) */
   double planHostSec;          /* host time the worker spent planning and issuing launches */
} MKFServerStats;

int mkfServerCreate(MKFServer **pServer, const MKFServerConfig *cfg);
/* Non-blocking and thread-safe; returns a ticket. */
int mkfServerSubmit(MKFServer *server, const MKFRequest *req, uint64_t *ticket);
/* Wait up to timeoutSec for a ticket: MKF_OK with *pDevCounts = its device counts (NULL when
 * copied to hostOut) and its latency, MKF_ERR_TIMEOUT, or the request's own error (e.g.
 * MKF_ERR_NOMEM for a request larger than the budget). */
int mkfServerWait(MKFServer *server, uint64_t ticket, double timeoutSec, const uint64_t **pDevCounts, double *latencySec);
/* Copy a finished ticket's device counts to dst (host or device), synchronously on `stream`. */
int mkfServerCopyCounts(MKFServer *server, uint64_t ticket, uint64_t *dst, void *stream);
/* Forget a finished ticket and free its device counts. */
int mkfServerRelease(MKFServer *server, uint64_t ticket);
int mkfServerStats(MKFServer *server, MKFServerStats *stats, int reset);
/* Finishes every submitted request, then frees the server (tickets become invalid). Requests that
 * can no longer be admitted because the budget is held by counts never released fail with
 * MKF_ERR_BUSY instead of waiting. */
int mkfServerDestroy(MKFServer *server);

/* ---- tuning (no original counterpart) ----
 * Two launch parameters are chosen per kind of field: the slab depth (planes of cells per work
 * item: halo re-reads against work items per SM) and, for the TMA-staged rank-table kernel, a
 * variant of CTA shape and histogram privatisation (0: 20 warps per CTA, two-stage FP64 tile rings,
 * two histogram copies; 1: 16 warps, three stages, two copies; 2: 20 warps, two stages, one copy).
 * A kind of field is the kernel, the element type, the threshold count and the power-of-two size
 * class of each extent (so the row width class too).
 * mkfTune times the candidate depths (and variants) on this field with these thresholds (the
 * counting runs several times; synchronous) and keeps the fastest for fields of the same kind;
 * later mkfFieldBPFD calls on such fields use it; without tuning each kernel uses its default.
 * mkfSetTuning(0 / 1) switches the tuning of new batch plans off / on (default on); it returns
 * the previous setting. */
int mkfTune(const MKFFieldDesc *pF, const MKFThreshSet *pT, void *stream);
int mkfSetTuning(int batchPlans);
/* Record `depth` (1..255 planes) and `variant` as the choice for fields of this kind, as mkfTune
 * records what it measured best (for instance a choice measured in an earlier process); depth 0
 * forgets the entry. Counts the field once to learn which kernels it takes (synchronous). */
int mkfTuneSet(const MKFFieldDesc *pF, const MKFThreshSet *pT, int depth, int variant, void *stream);
/* The depth and variant recorded for this field's kind (0 and 0 when none is). Counts the field
 * once to learn which kernels it takes (synchronous). */
int mkfTuneQuery(const MKFFieldDesc *pF, const MKFThreshSet *pT, int *depth, int *variant, void *stream);

/* ---- kernel waits (no original counterpart) ----
 * The kernels that wait on their own asynchronous copies give every wait a limit; a wait that
 * runs out (never in a correct run) ends the kernel early, leaves its counts incomplete and sets a
 * device flag instead of hanging the GPU. mkfKernelFaults returns that flag (0 = none; negative =
 * an MKF_ERR_* code) and clears it when `clear` is nonzero. Synchronous. */
int mkfKernelFaults(int clear);

/* ---- measures (closest original: mkfSelectMeasuresBPFD, mkfUtil.c:94) ---- */
/* For each of nSets distributions (host uint64_t[nSets][256]) write, in double:
 *   r[4*i+0] V   = number of cells whose corner 0 is set (volume in cell units)
 *   r[4*i+1] S   = sum over the 22 symmetry groups of gWS[g] * N_g   (surface estimate)
 *   r[4*i+2] M   = sum of gWM[g] * N_g                                (integral mean curvature)
 *   r[4*i+3] chi = sum of gWK[g] * N_g / 24                           (Euler characteristic)
 * N_g = cells whose pattern is in group g; group map and weights are those of mkfUtil.c:33-58 and
 * mkfHacks.c:9-20. */
int mkfMeasuresF64(double *r, const uint64_t *pBPFD, int nSets);
/* The same on the device: pBPFD and r are device pointers. */
int mkfMeasuresF64Dev(double *r, const uint64_t *pBPFD, int nSets, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* MKF_B200_H */
