/* cell8Sym.h - symmetry groups of the 2x2x2 cell patterns.
 * Replaces MKF src/cell8Sym.h:33-35 (c8sGetMap). */
#ifndef CELL8SYM_H
#define CELL8SYM_H
#include "mkf_types.h"
#ifdef __cplusplus
extern "C" {
#endif
/* Write, for each of the 256 patterns, the index (0..21) of its group under the 48 symmetries
 * of the cube; returns the number of groups (22). */
int c8sGetMap(uint8_t map[CELL8_PATTERNS]);
#ifdef __cplusplus
}
#endif
#endif
