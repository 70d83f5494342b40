/* abi_probe.c - prints the size and member offsets of the ABI structs as JSON. Compiled once
 * against the reference MKF headers (to make the golden layout) and, in the tests, against
 * include/ of this library; the two outputs must be equal. */
#include <stdio.h>
#include <stddef.h>
#include "binMapUtil.h"

#define S(T) printf("\"%s\": {\"size\": %zu", #T, sizeof(T))
#define F(T, f) printf(", \"%s\": %zu", #f, offsetof(T, f))
#define E() printf("}")

int main(void)
{
   printf("{");
   S(BinMapF64); F(BinMapF64, t); F(BinMapF64, m); E(); printf(", ");
   S(BMOrg); F(BMOrg, rowElem); F(BMOrg, rowPairs); F(BMOrg, planePairs); F(BMOrg, rowWS); F(BMOrg, planeWS); E(); printf(", ");
   S(ConstFieldPtr); E(); printf(", ");
   S(BMFieldInfo); F(BMFieldInfo, fieldTableMask); F(BMFieldInfo, elemID); F(BMFieldInfo, oprID); F(BMFieldInfo, profID);
   F(BMFieldInfo, flags); F(BMFieldInfo, pD); F(BMFieldInfo, pS); F(BMFieldInfo, pFieldDevPtrTable); E(); printf(", ");
   S(KernInfo); F(KernInfo, dtms); E(); printf(", ");
   S(Context); F(Context, nField); F(Context, nElem); F(Context, enc); F(Context, bytesElem); F(Context, bytesF);
   F(Context, nU); F(Context, bytesU); F(Context, nZ); F(Context, bytesZ); F(Context, pDF); F(Context, pHF);
   F(Context, pDU); F(Context, pHU); F(Context, pDZ); F(Context, pHZ); F(Context, bmo); F(Context, ki); E();
   printf("}\n");
   return 0;
}
