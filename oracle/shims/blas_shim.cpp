// Reference-semantics BLAS routines for the oracle build (test
// infrastructure only): the five Fortran symbols the reference declares in
// include/blas.h, column-major, only the 'N' (no transpose) form it uses
// (src/vecmatop.cpp:36,59,84,111; include/vecmath.hpp:101).
#include <complex>
typedef std::complex<double> zc;

extern "C" {
void zgemv_(char* trans, int* m, int* n, zc* alpha, zc* a, int* lda, zc* x, int* incx, zc* beta,
            zc* y, int* incy) {
    (void)trans;
    const int M = *m, N = *n, L = *lda, ix = *incx, iy = *incy;
    const zc al = *alpha, be = *beta;
    for (int i = 0; i < M; ++i) y[i * iy] = (be == zc(0, 0)) ? zc(0, 0) : be * y[i * iy];
    for (int j = 0; j < N; ++j) {
        const zc t = al * x[j * ix];
        const zc* col = a + (long)j * L;
        for (int i = 0; i < M; ++i) y[i * iy] += t * col[i];
    }
}
void zgemm_(char* ta, char* tb, int* m, int* n, int* k, zc* alpha, zc* a, int* lda, zc* b, int* ldb,
            zc* beta, zc* c, int* ldc) {
    (void)ta; (void)tb;
    const int M = *m, N = *n, K = *k;
    for (int j = 0; j < N; ++j) {
        zc* cc = c + (long)j * *ldc;
        for (int i = 0; i < M; ++i) cc[i] = (*beta == zc(0, 0)) ? zc(0, 0) : *beta * cc[i];
        for (int l = 0; l < K; ++l) {
            const zc t = *alpha * b[l + (long)j * *ldb];
            const zc* col = a + (long)l * *lda;
            for (int i = 0; i < M; ++i) cc[i] += t * col[i];
        }
    }
}
void dgemv_(char* trans, int* m, int* n, double* alpha, double* a, int* lda, double* x, int* incx,
            double* beta, double* y, int* incy) {
    (void)trans;
    for (int i = 0; i < *m; ++i) y[i * *incy] = (*beta == 0.0) ? 0.0 : *beta * y[i * *incy];
    for (int j = 0; j < *n; ++j) {
        const double t = *alpha * x[j * *incx];
        for (int i = 0; i < *m; ++i) y[i * *incy] += t * a[i + (long)j * *lda];
    }
}
void dgemm_(char* ta, char* tb, int* m, int* n, int* k, double* alpha, double* a, int* lda,
            double* b, int* ldb, double* beta, double* c, int* ldc) {
    (void)ta; (void)tb;
    for (int j = 0; j < *n; ++j) {
        double* cc = c + (long)j * *ldc;
        for (int i = 0; i < *m; ++i) cc[i] = (*beta == 0.0) ? 0.0 : *beta * cc[i];
        for (int l = 0; l < *k; ++l) {
            const double t = *alpha * b[l + (long)j * *ldb];
            for (int i = 0; i < *m; ++i) cc[i] += t * a[i + (long)l * *lda];
        }
    }
}
void dscal_(int* n, double* alpha, double* x, int* incx) {
    for (int i = 0; i < *n; ++i) x[i * *incx] *= *alpha;
}
}
