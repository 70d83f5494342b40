/* util.h - stand-in for the MKF "Common" utility header, which is not part of the published
 * MKF tree (MKF src/encoding.h:8 includes it from ../Common/src). It supplies only the types and
 * macros the reference C path uses, so that path can be compiled unmodified from its own
 * sources for use as a test oracle. Test infrastructure only: nothing in the product links it. */
#ifndef UTIL_H
#define UTIL_H
#include <stdio.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stddef.h>
#include <math.h>

typedef unsigned int uint;
typedef int64_t I64;
typedef uint8_t U8;
typedef uint16_t U16;
typedef uint32_t U32;
typedef float F32;
typedef double F64;
typedef int Bool32;
typedef int B32;
typedef double SMVal;

#ifndef TRUE
#define TRUE 1
#endif
#ifndef FALSE
#define FALSE 0
#endif

/* Logging is silenced: the oracle must not print while tests run. */
#define LOG(...) ((void)0)
#define LOG_CALL(...) ((void)0)
#define WARN(...) ((void)0)
#define WARN_CALL(...) ((void)0)
#define ERROR(...) fprintf(stderr, __VA_ARGS__)
#define ERROR_CALL(...) ((void)0)

#define MIN(a, b) (((a) < (b)) ? (a) : (b))
#define MAX(a, b) (((a) > (b)) ? (a) : (b))
#define SWAP(T, a, b) do { T swap_tmp_ = (a); (a) = (b); (b) = swap_tmp_; } while (0)
/* n low bits set */
#define BIT_MASK(n) ((1U << (n)) - 1)
#define BITS_TO_BYTES(b) (((b) + 7) >> 3)
/* words of 2^s bits needed for b bits (rounded up), as binMapACC.c:86 expects */
#define BITS_TO_WRDSH(b, s) (((b) + (1 << (s)) - 1) >> (s))

static inline int bitCountZ(size_t z) { return __builtin_popcountll((unsigned long long)z); }

#ifdef __cplusplus
extern "C" {
#endif
SMVal deltaT(void);
#ifdef __cplusplus
}
#endif
#endif /* UTIL_H */
