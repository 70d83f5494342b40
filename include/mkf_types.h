/* mkf_types.h - data types and constants shared by every entry point of libMKF.so.
 *
 * These structs are part of the binary interface: a caller built against the
 * original MKF headers passes them by pointer, so member order, widths and
 * padding must stay exactly as the original declares them (x86-64 LP64 layout).
 *
 *   BinMapF64       replaces MKF src/binMapUtil.h:28-32
 *   BinMapF32       replaces MKF src/binMapUtil.h:35-40
 *   BMOrg           replaces MKF src/binMapUtil.h:52-57
 *   ConstFieldPtr   replaces MKF src/binMapUtil.h:65
 *   BMFieldInfo     replaces MKF src/binMapUtil.h:69-79
 *   KernInfo        replaces MKF src/binMapUtil.h:107-110
 *   Context         replaces MKF src/binMapUtil.h:113-125
 *   NumEnc, ENC_*   replace  MKF src/encoding.h:15-31
 *   BMC_*           replace  MKF src/binMapUtil.h:43-47
 */
#ifndef MKF_TYPES_H
#define MKF_TYPES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Number encodings: high nibble = kind, low nibble = bytes (or bits for packed). */
#define ENC_MASK_TYP 0xF0
#define ENC_MASK_NUM 0x0F
#define ENC_TYPE_FPB 0xF0
#define ENC_TYPE_INT 0xE0
#define ENC_TYPE_BTS 0x00
#define ENC_F32 (ENC_TYPE_FPB | 4)
#define ENC_F64 (ENC_TYPE_FPB | 8)
#define ENC_U8  (ENC_TYPE_BTS | 8)
#define ENC_U1  (ENC_TYPE_BTS | 1)
#define ENC_FLOAT  ENC_F32
#define ENC_DOUBLE ENC_F64
typedef uint8_t NumEnc;

/* Relation bits: a scalar f is mapped to 1 when the bit for the relation of f
 * to the threshold (less / equal / greater) is set in the mask. */
#define BMC_LT (0x1)
#define BMC_EQ (0x2)
#define BMC_GT (0x4)
#define BMC_NV (0x0)
#define BMC_AL (0x7)

#define BM_NUMT (1)          /* thresholds per BinMapF64 */
#define BM_TLB (0)           /* index in BinMapF64.t of the threshold compared for '<' */
#define BM_TUB (0)           /* index in BinMapF64.t of the threshold compared for '>' */
#define BM_FLAG_T2IVL (1 << 15)
#define BMCU_FIELD_MAX 4     /* fields summed by one binMapCUDA call */
#define MKF_BINS (1 << 8)    /* 2x2x2 cell patterns */
#define CELL8_PATTERNS (1 << 8)
#define CELL8_SYMM_GROUPS (22)

typedef struct
{
   double t[BM_NUMT];
   uint32_t m;
} BinMapF64;

/* Single-precision form of BinMapF64; no entry point of this library takes it, callers of the
 * original declare it (binMapUtil.h:35-40). */
typedef struct
{
   float t[BM_NUMT];
   uint32_t m;
} BinMapF32;

typedef uint32_t BMStride;
typedef uint32_t BMPackWord;

/* Packed binary map organisation: bit j of word w of a row is element x = 32w + j;
 * rows are padded to whole 32-bit words; planes follow each other. */
typedef struct
{
   uint32_t rowElem;
   uint32_t rowPairs, planePairs;
   BMStride rowWS, planeWS;
} BMOrg;

typedef union { const void *p; const float *pF32; const double *pF64; size_t w; } ConstFieldPtr;

typedef long int FieldStride;
typedef int FieldDef;

typedef struct
{
   struct {
      uint32_t fieldTableMask;  /* bit i enables entry i of pFieldDevPtrTable */
      NumEnc elemID;            /* ENC_F32 or ENC_F64 */
      uint8_t oprID, profID, flags;
   };
   const FieldDef *pD;               /* int def[3], X fastest */
   const FieldStride *pS;            /* element strides, NULL = planar */
   ConstFieldPtr *pFieldDevPtrTable; /* device pointers */
} BMFieldInfo;

typedef struct
{
   float dtms[2]; /* [0] binary map stage, [1] pattern-count stage, milliseconds */
} KernInfo;

typedef struct
{
   int nField, nElem;
   struct { NumEnc enc; uint8_t bytesElem, pad[2]; };
   long bytesF;
   long nU, bytesU;
   long nZ, bytesZ;
   void *pDF, *pHF;
   BMPackWord *pDU, *pHU;
   void *pDZ, *pHZ;
   BMOrg bmo;
   KernInfo ki;
} Context;

#ifdef __cplusplus
}
#endif

#endif /* MKF_TYPES_H */
