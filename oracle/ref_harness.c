/* ref_harness.c - entry points into the reference MKF C path for the tests and the CPU baseline.
 *
 * TEST INFRASTRUCTURE ONLY. Linked with the unmodified reference sources (binMapACC.c, mkfACC.c,
 * binMapUtil.c, encoding.c, geomSVU.c, cell8Sym.c, mkfUtil.c with NO_REF_MEASURES) into
 * oracle/_ref/libmkfref.so by oracle/Makefile. Every function here only arranges arguments and
 * calls reference code; the counting itself is the reference's.
 */
#include <pthread.h>
#include <time.h>
#include "mkfACC.h"
#include "cell8Sym.h"

#define REFH_EXPORT __attribute__((visibility("default")))

/* util.h declares this; the reference sources linked here do not call it. */
SMVal deltaT(void)
{
   static struct timespec t0;
   struct timespec t;
   clock_gettime(CLOCK_MONOTONIC, &t);
   const double d = (double)(t.tv_sec - t0.tv_sec) + 1e-9 * (double)(t.tv_nsec - t0.tv_nsec);
   t0 = t;
   return d;
}

/* Exported by mkfACC.c (ACC_INLINE is empty when OpenACC is off) but declared in no header. */
extern void addPlaneBPFD(size_t rBPFD[256], const BMPackWord *pPlane0, const BMPackWord *pPlane1,
                         const int rowStride, const int def[3]);

/* mkfAccGetBPFDSimple (mkfACC.c:206-239) on an FP64 field. The field must have 32 readable
 * elements of slack after its end when def[0] % 32 != 0 (binMapACC.c:86-90 reads past each row). */
REFH_EXPORT int refh_bpfd_simple(size_t h[256], const double *f, const int def[3], double t, unsigned m)
{
   BinMapF64 bm;
   bm.t[0] = t;
   bm.m = m;
   const size_t nW = setBMO(NULL, def, 0);
   BMPackWord *w = (BMPackWord *)calloc(nW + 1, sizeof(BMPackWord));
   if (!w) { return 0; }
   mkfAccGetBPFDSimple(h, w, f, def, &bm);
   free(w);
   return 1;
}

/* Packed map of an FP64 field exactly as the reference CPU path builds it (mkfACC.c:227-234). */
REFH_EXPORT void refh_pack(BMPackWord *w, const double *f, const int def[3], double t, unsigned m)
{
   BinMapF64 bm;
   bm.t[0] = t;
   bm.m = m;
   const int rowStride = BITS_TO_WRDSH(def[0], 5);
   const size_t nF = (size_t)def[0] * def[1] * def[2];
   if ((rowStride << 5) == def[0]) { binMapAcc(w, f, nF, &bm); }
   else { binMapRowsAcc(w, f, def[0], rowStride, def[1] * def[2], &bm); }
}

/* Pattern counts of a packed map by the reference CPU path (addPlaneBPFD per plane pair). */
REFH_EXPORT void refh_bpfd_pbm(size_t h[256], const BMPackWord *w, const int def[3])
{
   const int rowStride = BITS_TO_WRDSH(def[0], 5);
   const size_t planeStride = (size_t)rowStride * def[1];
   for (int z = 0; z + 1 < def[2]; z++)
   {
      addPlaneBPFD(h, w + z * planeStride, w + (z + 1) * planeStride, rowStride, def);
   }
}

typedef struct
{
   const double *f;
   int def[3];
   int z0, z1; /* plane pairs [z0, z1) */
   BinMapF64 bm;
   size_t h[256];
   int ok;
} RefSlab;

static void *refh_slab(void *arg)
{
   RefSlab *s = (RefSlab *)arg;
   memset(s->h, 0, sizeof(s->h));
   s->ok = 1;
   if (s->z1 <= s->z0) { return NULL; }
   const int rowStride = BITS_TO_WRDSH(s->def[0], 5);
   const size_t planeStride = (size_t)rowStride * s->def[1];
   const int nPlane = s->z1 - s->z0 + 1;
   BMPackWord *w = (BMPackWord *)calloc(planeStride * nPlane + 1, sizeof(BMPackWord));
   if (!w) { s->ok = 0; return NULL; }
   const double *fz = s->f + (size_t)s->z0 * s->def[0] * s->def[1];
   if ((rowStride << 5) == s->def[0])
   {
      binMapAcc(w, fz, (size_t)s->def[0] * s->def[1] * nPlane, &s->bm);
   }
   else
   {
      binMapRowsAcc(w, fz, s->def[0], rowStride, s->def[1] * nPlane, &s->bm);
   }
   for (int z = 0; z + 1 < nPlane; z++)
   {
      addPlaneBPFD(s->h, w + z * planeStride, w + (z + 1) * planeStride, rowStride, s->def);
   }
   free(w);
   return NULL;
}

/* The reference CPU path on nThreads host threads: z is split into slabs of plane pairs, each
 * thread maps its planes (plus one halo plane) with binMapAcc/binMapRowsAcc and counts them with
 * addPlaneBPFD into a private histogram; the histograms are summed. This is how the reference's
 * OpenACC "parallel loop" over planes (mkfACC.c:183) would run on a multicore host, without its
 * shared-histogram race. Overwrites h. Returns 1 on success. */
REFH_EXPORT int refh_bpfd_mt(size_t h[256], const double *f, const int def[3], double t, unsigned m, int nThreads)
{
   if (nThreads < 1) { nThreads = 1; }
   const int pairs = def[2] - 1;
   if (nThreads > pairs) { nThreads = pairs > 0 ? pairs : 1; }
   RefSlab *sl = (RefSlab *)calloc((size_t)nThreads, sizeof(RefSlab));
   pthread_t *th = (pthread_t *)calloc((size_t)nThreads, sizeof(pthread_t));
   if (!sl || !th) { free(sl); free(th); return 0; }
   for (int i = 0; i < nThreads; i++)
   {
      sl[i].f = f;
      memcpy(sl[i].def, def, sizeof(sl[i].def));
      sl[i].z0 = (int)((long)pairs * i / nThreads);
      sl[i].z1 = (int)((long)pairs * (i + 1) / nThreads);
      sl[i].bm.t[0] = t;
      sl[i].bm.m = m;
      pthread_create(th + i, NULL, refh_slab, sl + i);
   }
   int ok = 1;
   memset(h, 0, sizeof(size_t) * 256);
   for (int i = 0; i < nThreads; i++)
   {
      pthread_join(th[i], NULL);
      ok &= sl[i].ok;
      for (int c = 0; c < 256; c++) { h[c] += sl[i].h[c]; }
   }
   free(sl);
   free(th);
   return ok;
}
