/* Minimal CBLAS declarations so that the reference's src/compute_SPH.cpp compiles; the
 * reference only reaches cblas_dgemm from its unused host path (compute_SPH.cpp:46-54). */
#ifndef ORACLE_REF_CBLAS_SHIM_H
#define ORACLE_REF_CBLAS_SHIM_H
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
#ifdef __cplusplus
extern "C"
#endif
void cblas_dgemm(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int, int, int, double,
                 const double *, int, const double *, int, double, double *, int);
#endif
