/* Prototype-only CBLAS declarations (standard netlib CBLAS interface) for the
 * five routines the reference engine calls.  The implementation is the LP64
 * OpenBLAS shared library linked by oracle/Makefile. */
#ifndef OA_REF_CBLAS_H
#define OA_REF_CBLAS_H
#ifdef __cplusplus
extern "C" {
#endif
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
void cblas_sgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE,
                 int M, int N, int K, float alpha, const float* A, int lda,
                 const float* B, int ldb, float beta, float* C, int ldc);
void cblas_ssyrk(enum CBLAS_ORDER, enum CBLAS_UPLO, enum CBLAS_TRANSPOSE,
                 int N, int K, float alpha, const float* A, int lda,
                 float beta, float* C, int ldc);
float cblas_sdot(int N, const float* X, int incX, const float* Y, int incY);
void cblas_saxpy(int N, float alpha, const float* X, int incX, float* Y, int incY);
float cblas_snrm2(int N, const float* X, int incX);
#ifdef __cplusplus
}
#endif
#endif
