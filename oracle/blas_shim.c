/* Forwarding shim: plain Fortran BLAS/LAPACK names -> the LP64 OpenBLAS that
 * ships inside SciPy's wheel (it prefixes every symbol with `scipy_`).
 *
 * TEST INFRASTRUCTURE ONLY.  The reference DMRG sources call dgemm_, zgemm_,
 * dgesvd_, zgesvd_, dsyev_ and zheev_ (src/dgemm.cpp:14, src/zgemm.cpp:27,
 * src/dgesvd.cpp:28, src/zgesvd.cpp:30, src/dsyev.cpp:19, src/zheev.cpp:21);
 * this file gives them those names so the reference builds unmodified.
 * LAPACK routines get the gfortran hidden CHARACTER lengths (all 1).
 */
#include <stddef.h>

typedef struct { double re, im; } zc;

extern void scipy_dgemm_(const char*, const char*, const int*, const int*, const int*,
                         const double*, const double*, const int*, const double*, const int*,
                         const double*, double*, const int*, size_t, size_t);
extern void scipy_zgemm_(const char*, const char*, const int*, const int*, const int*,
                         const zc*, const zc*, const int*, const zc*, const int*,
                         const zc*, zc*, const int*, size_t, size_t);
extern void scipy_dgesvd_(const char*, const char*, const int*, const int*, double*, const int*,
                          double*, double*, const int*, double*, const int*, double*,
                          const int*, int*, size_t, size_t);
extern void scipy_zgesvd_(const char*, const char*, const int*, const int*, zc*, const int*,
                          double*, zc*, const int*, zc*, const int*, zc*, const int*,
                          double*, int*, size_t, size_t);
extern void scipy_dsyev_(const char*, const char*, const int*, double*, const int*, double*,
                         double*, const int*, int*, size_t, size_t);
extern void scipy_zheev_(const char*, const char*, const int*, zc*, const int*, double*,
                         zc*, const int*, double*, int*, size_t, size_t);

void dgemm_(const char* ta, const char* tb, const int* m, const int* n, const int* k,
            const double* al, const double* a, const int* lda, const double* b, const int* ldb,
            const double* be, double* c, const int* ldc)
{ scipy_dgemm_(ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc, 1, 1); }

void zgemm_(const char* ta, const char* tb, const int* m, const int* n, const int* k,
            const zc* al, const zc* a, const int* lda, const zc* b, const int* ldb,
            const zc* be, zc* c, const int* ldc)
{ scipy_zgemm_(ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc, 1, 1); }

void dgesvd_(const char* ju, const char* jv, const int* m, const int* n, double* a, const int* lda,
             double* s, double* u, const int* ldu, double* vt, const int* ldvt, double* work,
             const int* lwork, int* info)
{ scipy_dgesvd_(ju, jv, m, n, a, lda, s, u, ldu, vt, ldvt, work, lwork, info, 1, 1); }

void zgesvd_(const char* ju, const char* jv, const int* m, const int* n, zc* a, const int* lda,
             double* s, zc* u, const int* ldu, zc* vt, const int* ldvt, zc* work,
             const int* lwork, double* rwork, int* info)
{ scipy_zgesvd_(ju, jv, m, n, a, lda, s, u, ldu, vt, ldvt, work, lwork, rwork, info, 1, 1); }

void dsyev_(const char* jz, const char* up, const int* n, double* a, const int* lda, double* w,
            double* work, const int* lwork, int* info)
{ scipy_dsyev_(jz, up, n, a, lda, w, work, lwork, info, 1, 1); }

void zheev_(const char* jz, const char* up, const int* n, zc* a, const int* lda, double* w,
            zc* work, const int* lwork, double* rwork, int* info)
{ scipy_zheev_(jz, up, n, a, lda, w, work, lwork, rwork, info, 1, 1); }
