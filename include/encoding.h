/* encoding.h - numeric encoding helpers exported by libMKF.so.
 * Replaces MKF src/encoding.h:35-37 (encSizeN, encAlignment). */
#ifndef ENCODING_H
#define ENCODING_H
#include "mkf_types.h"
#ifdef __cplusplus
extern "C" {
#endif
/* Bytes needed by n elements of encoding e; *pElemBits (optional) receives the element width in bits.
 * Packed-bit encodings (ENC_U1, ENC_U8 as bits) round down to whole bytes as the original does. */
size_t encSizeN(int *pElemBits, const size_t n, const NumEnc e);
/* Required pointer alignment in bytes for encoding e. */
int encAlignment(const NumEnc e);
#ifdef __cplusplus
}
#endif
#endif
