/* geomSVU.h - small integer / float vector helpers that the original libMKF.so exports
 * (MKF src/geomSVU.h:17-54). They are kept so a caller linking the library finds every symbol. */
#ifndef GEOM_SVU_H
#define GEOM_SVU_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
int *setKNI(int r[], const int n, const int k);
int *copyNI(int r[], const int n, const int v[]);
int *addKNI(int r[], const int a[], const int n, const int k);
int sumNI(const int v[], int n);
int prodNI(const int v[], int n);
int mergeMinMaxNI(int rMin[], int rMax[], const int minA[], const int maxA[], const int minB[], const int maxB[], const int n);
size_t sumNZ(const size_t v[], size_t n);
float *scaleFNI(float r[], const int n, const int v[], const float s);
float *setKNF(float r[], const int n, const float k);
float *copyNF(float r[], const int n, const float v[]);
float *absNF(float r[], const int n, const float v[]);
float *sqrNF(float r[], const int n, const float v[]);
float sumNF(const float v[], int n);
float sqrMag3D(const float dx, const float dy, const float dz);
float sep3D(const float a[3], const float b[3]);
#ifdef __cplusplus
}
#endif
#endif
