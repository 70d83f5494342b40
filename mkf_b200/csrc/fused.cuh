// fused.cuh - arguments shared by the fused counting kernels (fused.cu, thermo.cu).
#pragma once
#include <vector>
#include "mkf_common.cuh"

namespace mkf {

struct FusedArgs
{
   const void *f;
   int64_t sx, sy, sz;   // element strides
   int X, Y, Z;
   int K;                // thresholds in this pass (sorted ascending)
   int D;                // planes of cells per slab
   int nSegX, nTileY, nSlabZ;
   long long nItems;     // nSegX * nTileY * nSlabZ warp work items
   uint32_t gtm, eqm, ltm, nanP;  // GEN: per-threshold relation bits, map word of a NaN element
   uint32_t nanRank;     // THERMO: rank of a NaN element
   int rankHi;           // THERMO: rank counts thresholds <= f (else < f)
   int complement;       // THERMO: stored codes are the bitwise complement of the true codes
   uint64_t *out;        // [.][256] distributions
   int outRow[MKF_MAX_THRESH];  // output row of sorted threshold k
   double tlo[64];       // sorted thresholds for the "f > t" test, +inf padded
   double thi[64];       // sorted thresholds for the "f >= t" test, +inf padded
   // thermometer kernel: order-preserving 32-bit keys of the thresholds it compares against
   // (the high word for FP64 fields), sorted, and the most thresholds sharing one bucket of the
   // 2^14-bucket rank table (1..4; 0 = the table cannot rank these thresholds)
   uint32_t tkey[MKF_MAX_THRESH];
   int lutC;
};


// One field of a batch, as the batched thermometer kernel reads it from device memory.
struct FieldTask
{
   const void *f;
   int64_t sx, sy, sz;
   int X, Y, Z, K, D, nSegX, nTileY, nSlabZ;
   long long nItems;
   uint32_t nanRank;
   int rankHi, complement, variant;  // variant: bit 0 ">=", bit 1 FP64, bit 2 shifted edge items, bit 3 lutC > 1
   int lutC, pad_;
   uint64_t *out;
   int outRow[MKF_MAX_THRESH];
   uint32_t tkey[MKF_MAX_THRESH];
   double tlo[64], thi[64];
};

// Most thresholds the word-parallel kernels take in one read (more than two only when they share
// one relation < <= > >=).
#ifndef WORDS_MAX_K
#define WORDS_MAX_K 6
#endif
constexpr int kWordMaxK = WORDS_MAX_K;

// One field for the word-parallel kernels.
struct WordTask
{
   const void *f;
   int64_t sx, sy, sz;    // element strides
   int X, Y, Z;
   int K;                 // 1 .. kWordMaxK
   int cls[kWordMaxK];    // relation class per threshold (words.cu)
   uint32_t m[kWordMaxK]; // relation masks
   double tlo[kWordMaxK], thi[kWordMaxK];  // exact-equivalent thresholds for "f > t" / "f >= t" tests
   int outRow[kWordMaxK];
   int complement;        // the map is counted negated: code c is stored in bin 255 - c
   int variant;           // batched kernel: which instantiation counts this field
   uint64_t *out;
   double *mom;           // moments kernel: [K][2 map values][sum f, sum f^2]
   int D, pad_;           // planes of cells per work item
   int nChunkX, nTileY, nSlabZ;
   long long nItems;
};

// Consecutive work items [begin, end) of one field.
struct BatchChunk
{
   int field, pad_;
   long long begin, end;
};

struct BatchArgs
{
   const FieldTask *tasks;
   const BatchChunk *chunks;
   int nChunks;
   unsigned *counter;  // next chunk to hand out; zero at launch
};

struct WordBatchArgs
{
   const WordTask *tasks;
   const BatchChunk *chunks;
   int nChunks;
   unsigned *counter;  // next chunk to hand out; zero at launch
};

struct ConstEntry { int row, bin; };
// Count one field for any thresholds (fused.cu): constant maps, one pass per relation class.
// rowBase[i] is the output row of threshold i (NULL = identity).
int fieldBPFD(uint64_t *out, const MKFFieldDesc *pF, const MKFThreshSet *pT, int flags, cudaStream_t s, const int *rowBase);

enum { kPlanSingle = 0, kPlanThermo = 1, kPlanWords = 2 };
// depth: planes of cells per work item; 0 = each kernel's default, -1 = chosen by field size.
int planBatchField(const MKFFieldDesc *pF, const MKFThreshSet *pT, int rowBase, FieldTask &t, WordTask &w,
                   std::vector<ConstEntry> &consts, bool &anyVarying, int depth = 0);

// Slab depth (planes of cells per work item) of a single-field launch of kernel family `family`
// (tune.cu): the depth mkfTune measured best for this kind of field, else `def`.
enum { kFamWords = 0, kFamThermo = 1, kFamThermoTma = 2 };
static constexpr int kTmNumVariants = 4;  // variants of the TMA rank-table kernel (thermo_tma.cu)
int tunedDepth(int family, int enc, int K, int X, int Y, int Z, int def);
// Kernel variant (CTA shape, histogram copies) of such a launch: the one mkfTune measured best for
// this kind of field, else `def`. Families without variants use 0.
int tunedVariant(int family, int enc, int K, int X, int Y, int Z, int def);
// The untuned slab depth: def halved (down to 4) until a field of itemsPerPlane work items per
// plane and Z planes has at least minItems items.
int sizeDepth(int def, long long itemsPerPlane, int Z, long long minItems);
// Whether mkfBatchPlanCreate measures the slab depth of each new plan (tune.cu).
bool batchTuning();

// Fill a task's key table and item grid; false if its thresholds share a rank-table bucket.
bool prepareThermoTask(FieldTask &t, int enc, int depth = 0);
// Launch the batched thermometer kernel over tasks of one element type (enc) whose largest
// threshold count is maxK.
// Chunks of one kernel variant of the batched rank-table kernel: [c0, c1) of the sorted chunk list.
struct ThermoGroup
{
   int variant, c0, c1, maxK;
};
static constexpr int kThVariants = 16;  // variant indices 0..15 (FieldTask::variant & 13 is used)
// Sort a batch's chunks by their field's variant (stable within a variant) and return the groups.
std::vector<ThermoGroup> groupThermoChunks(std::vector<BatchChunk> &chunks, const std::vector<FieldTask> &tasks);
// One launch per group; counters[v] (zeroed beforehand) hands out the chunks of variant v.
int launchThermoGroups(const FieldTask *dTasks, const BatchChunk *dChunks, const std::vector<ThermoGroup> &groups,
                       unsigned *counters, int enc, cudaStream_t s);

// Fill a word task's relation classes, batched variant and item grid (words.cu); launch the
// batched word kernel over the chunks of tasks of one element type.
void prepareWordTask(WordTask &a, int enc, int depth = 0);
int launchWordsBatch(const WordBatchArgs &b, int enc, cudaStream_t s);

// Word-parallel kernel for one or two thresholds of any relations, or up to kWordMaxK thresholds of
// one relation (words.cu); `masks` are the relation masks of f's (sorted) thresholds.
// MKF_ERR_UNSUPPORTED otherwise.
int launchWords(const FusedArgs &f, int enc, const uint32_t *masks, cudaStream_t s);

// Counts and descriptive moments of one or two thresholds (any relations) in one read (words.cu):
// mom is device double[K][2][2], per threshold and map value the sum of f and of f^2.
int launchWordsMoments(const FusedArgs &f, int enc, const uint32_t *masks, double *mom, cudaStream_t s);

// Whether a pass's field and threshold count suit the TMA-staged rank-table kernel (thermo_tma.cu):
// 3..16 thresholds, unit x stride, rows and planes on 16-byte boundaries, X >= 32, Y >= 9.
bool tmaRowsAligned(const FusedArgs &a, int enc);

// Launch the thermometer kernel for a pass whose thresholds all share one relation
// (< <= > >=); fills the key table of `a` first.
int launchThermo(FusedArgs &a, int enc, cudaStream_t s);

}  // namespace mkf
