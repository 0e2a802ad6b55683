/*
 * lapack_shim.c -- the three BLAS/LAPACK routines the reference's matrix class
 * calls (src/general/matrix.cpp:528-636: xgemm_, xgetrf_, xgetri_), written
 * from their textbook definitions for the reference step harness (test
 * infrastructure only; this image has no system BLAS/LAPACK).  Column-major
 * storage, Fortran calling convention (every argument by pointer), 1-based
 * pivot indices, as the Fortran interfaces define them.
 *
 *   gemm:  C = alpha op(A) op(B) + beta C, op = identity ('N') or transpose ('T'/'C')
 *   getrf: P A = L U by Gaussian elimination with partial (row) pivoting
 *   getri: inv(A) from the getrf factors: inv(U) by back substitution, then
 *          solve X L = inv(U) for X, then undo the row interchanges on columns
 */
#include <math.h>
#include <stddef.h>

#define DEFINE_LAPACK(T, GEMM, GETRF, GETRI)                                                           \
    void GEMM(const char *ta, const char *tb, const int *m, const int *n, const int *k, const T *alpha, \
              const T *A, const int *lda, const T *B, const int *ldb, const T *beta, T *C, const int *ldc) { \
        const int tA = (*ta == 'T' || *ta == 't' || *ta == 'C' || *ta == 'c');                         \
        const int tB = (*tb == 'T' || *tb == 't' || *tb == 'C' || *tb == 'c');                         \
        for (int j = 0; j < *n; ++j)                                                                   \
            for (int i = 0; i < *m; ++i) {                                                             \
                double s = 0.0;                                                                        \
                for (int p = 0; p < *k; ++p) {                                                         \
                    const T a = tA ? A[p + (size_t)i * *lda] : A[i + (size_t)p * *lda];                 \
                    const T b = tB ? B[j + (size_t)p * *ldb] : B[p + (size_t)j * *ldb];                 \
                    s += (double)a * (double)b;                                                        \
                }                                                                                      \
                T *c = &C[i + (size_t)j * *ldc];                                                       \
                *c = (T)((double)*alpha * s + (*beta == (T)0 ? 0.0 : (double)*beta * (double)*c));      \
            }                                                                                          \
    }                                                                                                  \
    void GETRF(const int *m, const int *n, T *A, const int *lda, int *ipiv, int *info) {               \
        const int mn = *m < *n ? *m : *n;                                                              \
        *info = 0;                                                                                     \
        for (int k = 0; k < mn; ++k) {                                                                 \
            int p = k;                                                                                 \
            for (int i = k + 1; i < *m; ++i)                                                           \
                if (fabs((double)A[i + (size_t)k * *lda]) > fabs((double)A[p + (size_t)k * *lda])) p = i; \
            ipiv[k] = p + 1;                                                                           \
            if (A[p + (size_t)k * *lda] == (T)0) {                                                     \
                if (!*info) *info = k + 1;                                                             \
                continue;                                                                              \
            }                                                                                          \
            if (p != k)                                                                                \
                for (int j = 0; j < *n; ++j) {                                                         \
                    const T t = A[k + (size_t)j * *lda];                                               \
                    A[k + (size_t)j * *lda] = A[p + (size_t)j * *lda];                                 \
                    A[p + (size_t)j * *lda] = t;                                                       \
                }                                                                                      \
            const T piv = A[k + (size_t)k * *lda];                                                     \
            for (int i = k + 1; i < *m; ++i) A[i + (size_t)k * *lda] /= piv;                           \
            for (int j = k + 1; j < *n; ++j) {                                                         \
                const T u = A[k + (size_t)j * *lda];                                                   \
                for (int i = k + 1; i < *m; ++i) A[i + (size_t)j * *lda] -= A[i + (size_t)k * *lda] * u; \
            }                                                                                          \
        }                                                                                              \
    }                                                                                                  \
    void GETRI(const int *n, T *A, const int *lda, const int *ipiv, T *work, const int *lwork, int *info) { \
        const int N = *n;                                                                              \
        *info = 0;                                                                                     \
        if (*lwork == -1) { /* workspace query */                                                      \
            work[0] = (T)(N > 0 ? N : 1);                                                              \
            return;                                                                                    \
        }                                                                                              \
        for (int k = 0; k < N; ++k)                                                                    \
            if (A[k + (size_t)k * *lda] == (T)0) {                                                     \
                *info = k + 1;                                                                         \
                return;                                                                                \
            }                                                                                          \
        /* inv(U) in place (upper triangle), column by column */                                      \
        for (int j = 0; j < N; ++j) {                                                                  \
            A[j + (size_t)j * *lda] = (T)1 / A[j + (size_t)j * *lda];                                  \
            const T ajj = -A[j + (size_t)j * *lda];                                                    \
            for (int i = 0; i < j; ++i) {                                                              \
                double s = 0.0;                                                                        \
                for (int p = i; p < j; ++p)                                                            \
                    s += (double)A[i + (size_t)p * *lda] * (double)A[p + (size_t)j * *lda];            \
                work[i] = (T)s;                                                                        \
            }                                                                                          \
            for (int i = 0; i < j; ++i) A[i + (size_t)j * *lda] = work[i] * ajj;                       \
        }                                                                                              \
        /* solve X L = inv(U), L unit lower, for columns right to left */                            \
        for (int j = N - 2; j >= 0; --j) {                                                             \
            for (int i = j + 1; i < N; ++i) {                                                          \
                work[i] = A[i + (size_t)j * *lda];                                                     \
                A[i + (size_t)j * *lda] = (T)0;                                                        \
            }                                                                                          \
            for (int r = 0; r < N; ++r) {                                                              \
                double s = 0.0;                                                                        \
                for (int i = j + 1; i < N; ++i) s += (double)A[r + (size_t)i * *lda] * (double)work[i]; \
                A[r + (size_t)j * *lda] -= (T)s;                                                       \
            }                                                                                          \
        }                                                                                              \
        /* column interchanges in reverse order */                                                   \
        for (int j = N - 2; j >= 0; --j) {                                                             \
            const int p = ipiv[j] - 1;                                                                 \
            if (p != j)                                                                                \
                for (int r = 0; r < N; ++r) {                                                          \
                    const T t = A[r + (size_t)j * *lda];                                               \
                    A[r + (size_t)j * *lda] = A[r + (size_t)p * *lda];                                 \
                    A[r + (size_t)p * *lda] = t;                                                       \
                }                                                                                      \
        }                                                                                              \
    }

DEFINE_LAPACK(double, dgemm_, dgetrf_, dgetri_)
DEFINE_LAPACK(float, sgemm_, sgetrf_, sgetri_)
