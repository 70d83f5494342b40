/* mkf_oracle.c - CPU restatement of the MKF hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the correctness oracle: it is loaded by the tests, by
 * smoke() and by the CPU-baseline leg of bench.py, and never by the product library. It is
 * written for clarity (one cell at a time), not for speed.
 *
 * Path restated here (MKF reference, paths relative to its src/):
 *   threshold      binMapACC.c:32-40, binMapCUDA.cuh:141-145
 *   packed map     binMapACC.c:43-93, binMapUtil.c:60-87 (layout), binMapCUDA.cuh:282-338
 *   pattern counts mkfACC.c:78-188, bpfdCUDA.cuh:41-118
 *   measures       mkfUtil.c:33-135, mkfHacks.c:9-20
 *
 * One deliberate difference: every row of X elements yields X-1 cells for every X >= 1. The two
 * reference counting paths agree with this for X >= 32 and both count 2X-1 cells per row for
 * X < 32, each in a different way (bpfdCUDA.cuh:112-116 re-reads word 0, mkfACC.c:137-150 reads
 * the next word); see orc_bpfd_pbm.
 */
#include <stdint.h>
#include <stddef.h>
#include <string.h>
#include <stdlib.h>
#include <math.h>

#define ORC_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------ threshold */

/* Relation index of f to t: 0 when f < t, 1 when equal (or either is NaN), 2 when f > t.
 * Follows sgnIdxDiff (binMapACC.c:32-35) and CUDAMap::eval (binMapCUDA.cuh:141-145). */
static inline unsigned orc_rel(double f, double t) { return 1u - (f < t) + (f > t); }

/* Map bit: bit `rel` of the 3-bit relation mask (binMapACC.c:37-40). */
static inline unsigned orc_bit(double f, double t, unsigned m) { return (m >> orc_rel(f, t)) & 1u; }

ORC_EXPORT unsigned orc_map_value(double f, double t, unsigned m) { return orc_bit(f, t, m); }

/* Field element (x,y,z) of a FP32 (enc 0xF4) or FP64 (enc 0xF8) field with element strides s[].
 * A FP32 element is promoted to double exactly, so comparing it with a threshold that is itself
 * a float gives the same result as the FP32 comparison of binMapCUDA.cuh:143. */
static inline double orc_elem(const void *f, int enc, const long s[3], long x, long y, long z)
{
   const long i = x * s[0] + y * s[1] + z * s[2];
   if (enc == 0xF4) { return (double)((const float *)f)[i]; }
   return ((const double *)f)[i];
}

static void orc_strides(long s[3], const int def[3], const long *stride)
{
   if (stride && (stride[0] | stride[1] | stride[2])) { s[0] = stride[0]; s[1] = stride[1]; s[2] = stride[2]; }
   else { s[0] = 1; s[1] = def[0]; s[2] = (long)def[0] * def[1]; }
}

/* ------------------------------------------------------------------ packed binary map */

/* Words per row and per plane of the full-size packed map (setBMO, binMapUtil.c:60-87 with
 * profID 0): rows rounded up to whole 32-bit words, planes contiguous. */
ORC_EXPORT void orc_layout(uint32_t *rowWS, uint32_t *planeWS, const int def[3])
{
   *rowWS = (uint32_t)((def[0] + 31) >> 5);
   *planeWS = *rowWS * (uint32_t)def[1];
}

/* Threshold the sum of nF fields (all of encoding enc, common strides) into a packed map: bit
 * (x & 31) of word (x >> 5) + y*rowWS + z*planeWS is the map of element (x,y,z); padding bits past
 * X in the last word of a row are 0. The sum is formed in the field's own precision in field
 * order, f0 + f1 + ..., as CUDAMultiField::sum does (binMapCUDA.cuh:194-199); with one field it
 * is the element itself (binMapACC.c:43-58, binMapCUDA.cuh:282-294). */
ORC_EXPORT void orc_pack(uint32_t *pbm, const void *const *fields, int nF, int enc, const int def[3],
                         const long *stride, double t, unsigned m, uint32_t rowWS, uint32_t planeWS)
{
   long s[3];
   orc_strides(s, def, stride);
   for (long z = 0; z < def[2]; z++)
   {
      for (long y = 0; y < def[1]; y++)
      {
         uint32_t *row = pbm + (size_t)z * planeWS + (size_t)y * rowWS;
         memset(row, 0, sizeof(uint32_t) * rowWS);
         for (long x = 0; x < def[0]; x++)
         {
            double v;
            if (enc == 0xF4)
            {
               float a = (float)orc_elem(fields[0], enc, s, x, y, z);
               for (int i = 1; i < nF; i++) { a += (float)orc_elem(fields[i], enc, s, x, y, z); }
               v = (double)a;
            }
            else
            {
               double a = orc_elem(fields[0], enc, s, x, y, z);
               for (int i = 1; i < nF; i++) { a += orc_elem(fields[i], enc, s, x, y, z); }
               v = a;
            }
            row[x >> 5] |= (uint32_t)orc_bit(v, t, m) << (x & 31);
         }
      }
   }
}

/* ------------------------------------------------------------------ pattern counts */

static inline unsigned orc_pbm_bit(const uint32_t *pbm, uint32_t rowWS, uint32_t planeWS, long x, long y, long z)
{
   return (pbm[(size_t)z * planeWS + (size_t)y * rowWS + (size_t)(x >> 5)] >> (x & 31)) & 1u;
}

/* Add the 8-bit pattern of every interior 2x2x2 cell of an X*Y*Z packed map to h[256].
 * Pattern bit order (bpfdCUDA.cuh:45-61, mkfACC.c:132-145): bit 0 = (x,y,z), 1 = (x+1,y,z),
 * 2 = (x,y+1,z), 3 = (x+1,y+1,z), 4..7 = the same four corners in plane z+1. Cells lie wholly
 * inside the field (no periodic wrap), so there are (X-1)(Y-1)(Z-1) of them; padding bits are
 * never read. */
ORC_EXPORT void orc_bpfd_pbm(uint64_t h[256], const uint32_t *pbm, int X, int Y, int Z, uint32_t rowWS, uint32_t planeWS)
{
   for (long z = 0; z + 1 < Z; z++)
   {
      for (long y = 0; y + 1 < Y; y++)
      {
         for (long x = 0; x + 1 < X; x++)
         {
            unsigned c = 0;
            for (int i = 0; i < 8; i++)
            {
               c |= orc_pbm_bit(pbm, rowWS, planeWS, x + (i & 1), y + ((i >> 1) & 1), z + ((i >> 2) & 1)) << i;
            }
            h[c]++;
         }
      }
   }
}

/* Pattern counts of a field for K thresholds directly (no map kept): h[k*256 + c]. Each threshold
 * is applied with its own relation mask m[k] and compared exactly in double. Accumulates. */
ORC_EXPORT void orc_bpfd_field(uint64_t *h, const void *f, int enc, const int def[3], const long *stride,
                               int K, const double *t, const unsigned *m)
{
   long s[3];
   orc_strides(s, def, stride);
   const long X = def[0], Y = def[1], Z = def[2];
   if (X < 2 || Y < 2 || Z < 2) { return; }
   /* two planes of per-element threshold words: bit k = map of threshold k */
   const size_t plane = (size_t)X * Y;
   uint32_t *b0 = (uint32_t *)malloc(sizeof(uint32_t) * plane);
   uint32_t *b1 = (uint32_t *)malloc(sizeof(uint32_t) * plane);
   if (!b0 || !b1) { free(b0); free(b1); return; }
   for (long z = 0; z < Z; z++)
   {
      uint32_t *cur = (z & 1) ? b1 : b0;
      const uint32_t *prv = (z & 1) ? b0 : b1;
      for (long y = 0; y < Y; y++)
      {
         for (long x = 0; x < X; x++)
         {
            const double v = orc_elem(f, enc, s, x, y, z);
            uint32_t w = 0;
            for (int k = 0; k < K; k++) { w |= (uint32_t)orc_bit(v, t[k], m[k]) << k; }
            cur[y * X + x] = w;
         }
      }
      if (z == 0) { continue; }
      for (long y = 0; y + 1 < Y; y++)
      {
         for (long x = 0; x + 1 < X; x++)
         {
            const uint32_t q[8] = {
               prv[y * X + x], prv[y * X + x + 1], prv[(y + 1) * X + x], prv[(y + 1) * X + x + 1],
               cur[y * X + x], cur[y * X + x + 1], cur[(y + 1) * X + x], cur[(y + 1) * X + x + 1] };
            for (int k = 0; k < K; k++)
            {
               unsigned c = 0;
               for (int i = 0; i < 8; i++) { c |= ((q[i] >> k) & 1u) << i; }
               h[(size_t)k * 256 + c]++;
            }
         }
      }
   }
   free(b0);
   free(b1);
}

/* ------------------------------------------------------------------ measures */

/* Symmetry group (0..21) of each pattern under the 48 symmetries of the cube, numbered as the
 * reference numbers them; the table is the reference's own data (mkfUtil.c:40-58). The tests
 * check it against the reference's generator c8sGetMap (cell8Sym.c:341-363) and against an
 * independent orbit computation. */
static const uint8_t orc_group[256] = {
   0,  1,  1,  2,  1,  2,  3,  5,  1,  3,  2,  5,  2,  5,  5,  8,
   1,  2,  3,  5,  3,  5,  7,  9,  4,  6,  6,  10, 6,  10, 13, 16,
   1,  3,  2,  5,  4,  6,  6,  10, 3,  7,  5,  9,  6,  13, 10, 16,
   2,  5,  5,  8,  6,  10, 13, 16, 6,  13, 10, 16, 11, 15, 15, 19,
   1,  3,  4,  6,  2,  5,  6,  10, 3,  7,  6,  13, 5,  9,  10, 16,
   2,  5,  6,  10, 5,  8,  13, 16, 6,  13, 11, 15, 10, 16, 15, 19,
   3,  7,  6,  13, 6,  13, 11, 15, 7,  12, 13, 14, 13, 14, 15, 18,
   5,  9,  10, 16, 10, 16, 15, 19, 13, 14, 15, 18, 15, 18, 17, 20,
   1,  4,  3,  6,  3,  6,  7,  13, 2,  6,  5,  10, 5,  10, 9,  16,
   3,  6,  7,  13, 7,  13, 12, 14, 6,  11, 13, 15, 13, 15, 14, 18,
   2,  6,  5,  10, 6,  11, 13, 15, 5,  13, 8,  16, 10, 15, 16, 19,
   5,  10, 9,  16, 13, 15, 14, 18, 10, 15, 16, 19, 15, 17, 18, 20,
   2,  6,  6,  11, 5,  10, 13, 15, 5,  13, 10, 15, 8,  16, 16, 19,
   5,  10, 13, 15, 9,  16, 14, 18, 10, 15, 15, 17, 16, 19, 18, 20,
   5,  13, 10, 15, 10, 15, 15, 17, 9,  14, 16, 18, 16, 18, 19, 20,
   8,  16, 16, 19, 16, 19, 18, 20, 16, 18, 19, 20, 19, 20, 20, 21 };

/* Group weights, the reference's own data: Euler (topological) weights gWK (mkfUtil.c:33-38),
 * surface gWS and mean curvature gWM (mkfHacks.c:9-20). */
static const int orc_wK[22] = { 0, 3, 0, 6, 6, -3, 3, 9, 0, -6, -6, 0, 12, 0, -3, -8, -3, -12, -6, 0, 3, 0 };
static const double orc_wS[22] = {
   0, 0.944412, 1.05178, 0.921095, 0.496906, 0.949947, 0.865898, 0.793181, 0.926631, 0.638921, 0.764068,
   0.784616, 0.874463, 0.868666, 0.557639, 0.682786, 0.923863, 0.496906, 0.737983, 0.65947, 0.0812817, 0 };
static const double orc_wM[22] = {
   0, 0.763019, 0.642656, 0.616236, 0.686801, 0.187756, 0.167269, 0.161335, 0, -0.431447, -0.287632,
   0, 0, -0.143816, -0.592783, -0.540019, -0.475387, -0.686801, -0.616236, -0.727774, -0.331571, 0 };

ORC_EXPORT void orc_group_map(uint8_t map[256]) { memcpy(map, orc_group, 256); }

ORC_EXPORT void orc_weights(int wK[22], double wS[22], double wM[22])
{
   memcpy(wK, orc_wK, sizeof(orc_wK));
   memcpy(wS, orc_wS, sizeof(orc_wS));
   memcpy(wM, orc_wM, sizeof(orc_wM));
}

/* Cells per group (addZMapU8, mkfUtil.c:71-78). */
ORC_EXPORT void orc_group_counts(uint64_t g[22], const uint64_t h[256])
{
   memset(g, 0, sizeof(uint64_t) * 22);
   for (int c = 0; c < 256; c++) { g[orc_group[c]] += h[c]; }
}

/* r[0] V = cells with corner 0 set (the numerator of volFrac, mkfUtil.c:125-135);
 * r[1] S = sum gWS[g] N_g and r[2] M = sum gWM[g] N_g in double, group order 0..21
 *          (sumProdZxF64, mkfHacks.c:22-27);
 * r[3] chi = (sum gWK[g] N_g) / 24: symK returns pi/6 times the integer sum (mkfUtil.c:64-69), the
 *          integral of Gaussian curvature, which is 4 pi chi. */
ORC_EXPORT void orc_measures(double r[4], const uint64_t h[256])
{
   uint64_t g[22];
   orc_group_counts(g, h);
   uint64_t v = 0;
   for (int c = 1; c < 256; c += 2) { v += h[c]; }
   double s = (double)g[0] * orc_wS[0], mc = (double)g[0] * orc_wM[0];
   for (int i = 1; i < 22; i++) { s += (double)g[i] * orc_wS[i]; mc += (double)g[i] * orc_wM[i]; }
   int64_t k = 0;
   for (int i = 0; i < 22; i++) { k += (int64_t)orc_wK[i] * (int64_t)g[i]; }
   r[0] = (double)v;
   r[1] = s;
   r[2] = mc;
   r[3] = (double)k / 24.0;
}

/* The reference's single-precision selection (mkfUtil.c:94-123 without the reference-measure
 * branch, i.e. as built with NO_REF_MEASURES): m[0] = Kv, m[3] = volume fraction, m[1] = m[2] = -1. */
ORC_EXPORT int orc_select_measures(float m[4], char sym[12], const uint64_t h[256], float s)
{
   uint64_t g[22];
   orc_group_counts(g, h);
   uint64_t t = 0, tg = 0, s0 = 0, s1 = 0;
   for (int c = 0; c < 256; c++) { t += h[c]; }
   for (int i = 0; i < 22; i++) { tg += g[i]; }
   int64_t k = 0;
   for (int i = 0; i < 22; i++) { k += (int64_t)orc_wK[i] * (int64_t)g[i]; }
   m[0] = (float)((double)k * M_PI / 6);
   for (int c = 0; c < 256; c += 2) { s0 += h[c]; s1 += h[c + 1]; }
   m[3] = (float)s1 / (float)(s0 + s1);
   m[1] = m[2] = -1;
   if ((t == tg) && (s > 0))
   {
      const float rkV = (float)(1.0 / (s * s * s * (float)t));
      m[0] *= rkV;
   }
   memcpy(sym, "Kv       Vv", 12);
   return 2;
}
