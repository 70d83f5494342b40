// fused.cuh - arguments shared by the fused counting kernels (fused.cu, thermo.cu).
#pragma once
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
   // (the high word for FP64 fields), sorted, and whether a 2^14-bucket table separates them
   uint32_t tkey[MKF_MAX_THRESH];
   int lutOk;
};


// Launch the thermometer kernel for a pass whose thresholds all share one relation
// (< <= > >=); fills the key table of `a` first.
int launchThermo(FusedArgs &a, int enc, cudaStream_t s);

}  // namespace mkf
