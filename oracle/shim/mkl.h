/*
 * BLAS/LAPACK declarations standing in for <mkl.h> so that the reference's
 * own sources compile into the CPU oracle (test infrastructure only).
 *
 * The reference calls cblas_dgemm (src/class_approximation.cpp:49,
 * src/class_approximation-loop-regions-at-finest-level-in-prior.cpp:370,384,
 * src/class_approximation-predict.cpp:135,148), cblas_dgemv
 * (...-prior.cpp:372, ...-predict.cpp:162,175), dtrtrs_ and dpotrf_
 * (src/class_approximation.cpp:139, ...-prior.cpp:160,169,230,241,316,345,
 * ...-predict.cpp:129,143,159,172).  These are the standard CBLAS / Fortran
 * LAPACK entry points; the oracle links them from an OpenBLAS build shipped
 * in the image (see oracle/Makefile), in place of MKL.
 */
#pragma once

extern "C" {

enum CBLAS_LAYOUT { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_LAYOUT CBLAS_LAYOUT;
typedef enum CBLAS_TRANSPOSE CBLAS_TRANSPOSE;

void cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE transa, CBLAS_TRANSPOSE transb,
                 int m, int n, int k, double alpha, const double* a, int lda,
                 const double* b, int ldb, double beta, double* c, int ldc);

void cblas_dgemv(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE trans, int m, int n, double alpha,
                 const double* a, int lda, const double* x, int incx, double beta,
                 double* y, int incy);

void dtrtrs_(const char* uplo, const char* trans, const char* diag, const int* n,
             const int* nrhs, const double* a, const int* lda, double* b, const int* ldb,
             int* info);

void dpotrf_(const char* uplo, const int* n, double* a, const int* lda, int* info);

void dsyrk_(const char* uplo, const char* trans, const int* n, const int* k,
            const double* alpha, const double* a, const int* lda, const double* beta,
            double* c, const int* ldc);

void dgels_(const char* trans, const int* m, const int* n, const int* nrhs, double* a,
            const int* lda, double* b, const int* ldb, double* work, const int* lwork,
            int* info);

void openblas_set_num_threads(int num_threads);
}
