/* Prototype-only LAPACKE declarations (standard LAPACKE C interface) for the
 * routines the reference engine calls.  LP64: lapack_int is int. */
#ifndef OA_REF_LAPACKE_H
#define OA_REF_LAPACKE_H
#ifdef __cplusplus
extern "C" {
#endif
#define lapack_int int
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
lapack_int LAPACKE_sposv(int layout, char uplo, lapack_int n, lapack_int nrhs,
                         float* a, lapack_int lda, float* b, lapack_int ldb);
lapack_int LAPACKE_spotrf(int layout, char uplo, lapack_int n, float* a, lapack_int lda);
lapack_int LAPACKE_spotri(int layout, char uplo, lapack_int n, float* a, lapack_int lda);
lapack_int LAPACKE_sgels(int layout, char trans, lapack_int m, lapack_int n,
                         lapack_int nrhs, float* a, lapack_int lda, float* b, lapack_int ldb);
lapack_int LAPACKE_sgesvd(int layout, char jobu, char jobvt, lapack_int m, lapack_int n,
                          float* a, lapack_int lda, float* s, float* u, lapack_int ldu,
                          float* vt, lapack_int ldvt, float* superb);
#ifdef __cplusplus
}
#endif
#endif
