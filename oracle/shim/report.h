/* report.h - stand-in for the MKF "Common" report header (not in the published tree). Test
 * infrastructure only; see util.h beside it. */
#ifndef REPORT_H
#define REPORT_H
#include "util.h"
#define report(...) ((void)0)
#define reportBytes(...) ((void)0)
#endif
