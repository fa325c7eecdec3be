/*
 * Minimal stand-in for MATLAB's <blas.h> (libmwblas), used ONLY to compile the
 * reference's own C++ sources in place for the CPU oracle build (oracle/Makefile).
 *
 * The reference calls exactly two BLAS routines with MATLAB's Fortran-style
 * pointer signatures:
 *   - dgemm  (Cpp/src/objgrd.cpp:53, :77)   v = alpha * op(A) * op(B) + beta * C
 *   - ddot   (Cpp/src/objgrd.cpp:56, LBFGS.cpp:51/77/78/104, lineSearch.cpp:50/60/75/82,
 *             getDirection.cpp:23/24/49/50)
 * Both are implemented here naively, column-major, as the reference BLAS
 * specification defines them.  Summation order differs from an optimised BLAS,
 * which changes FP64 results at the 1e-15 relative level only.
 *
 * This is test infrastructure: nothing in the product library includes it.
 */
#ifndef LDDMM_ORACLE_REF_BLAS_H
#define LDDMM_ORACLE_REF_BLAS_H

#include <cstddef>

static inline double ddot(const ptrdiff_t *n, const double *x, const ptrdiff_t *incx,
                          const double *y, const ptrdiff_t *incy)
{
	double acc = 0.0;
	ptrdiff_t ix = 0, iy = 0;
	for (ptrdiff_t k = 0; k < *n; ++k, ix += *incx, iy += *incy)
		acc += x[ix] * y[iy];
	return acc;
}

/* C(m x n) = alpha * op(A)(m x k) * op(B)(k x n) + beta * C, column-major. */
static inline void dgemm(const char *transa, const char *transb,
                         const ptrdiff_t *m, const ptrdiff_t *n, const ptrdiff_t *k,
                         const double *alpha, const double *A, const ptrdiff_t *lda,
                         const double *B, const ptrdiff_t *ldb,
                         const double *beta, double *C, const ptrdiff_t *ldc)
{
	const bool ta = (*transa == 'T' || *transa == 't' || *transa == 'C' || *transa == 'c');
	const bool tb = (*transb == 'T' || *transb == 't' || *transb == 'C' || *transb == 'c');
	for (ptrdiff_t j = 0; j < *n; ++j) {
		double *cj = C + j * (*ldc);
		for (ptrdiff_t i = 0; i < *m; ++i)
			cj[i] = (*beta == 0.0) ? 0.0 : (*beta) * cj[i];
		for (ptrdiff_t l = 0; l < *k; ++l) {
			const double b = tb ? B[j + l * (*ldb)] : B[l + j * (*ldb)];
			const double ab = (*alpha) * b;
			if (!ta) {
				const double *al = A + l * (*lda);
				for (ptrdiff_t i = 0; i < *m; ++i)
					cj[i] += al[i] * ab;
			} else {
				for (ptrdiff_t i = 0; i < *m; ++i)
					cj[i] += A[l + i * (*lda)] * ab;
			}
		}
	}
}

#endif
