/*
 * CPU oracle: FP64 restatement of the reference's C++ LDDMM path (dnhsieh/LDDMM,
 * Cpp/src).  TEST INFRASTRUCTURE ONLY -- the checker for the CUDA product path;
 * never linked, loaded or called by the product library.
 *
 * Differences from the reference, all deliberate and value-preserving:
 *  - objgrd is matrix-free: v = K(q)a is summed pair by pair as the reference's own
 *    multiplyKernel does (Cpp/src/multiplyKernel.cpp:22-292) instead of storing the
 *    N x N x T kernel stack and calling dgemm (Cpp/src/objgrd.cpp:52-54, :77-78).
 *    The math is identical (K is symmetric); FP64 rounding differs at ~1e-16.
 *  - Row sums are parallelised over rows with OpenMP.  Each row's sum runs in the
 *    reference's j order, so results do not depend on the thread count.
 *  - x^2 K0(x) and x K1(x) are computed from the integral representation
 *    K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt with the trapezoidal rule
 *    (step 1/8; the integrand is analytic in the strip |Im t| < pi/2, so the rule
 *    converges like exp(-pi^2 / h) ~ 1e-34), instead of the reference's rational
 *    approximations (Cpp/src/polybesselk.cpp:14-96).  Both are accurate to FP64
 *    rounding; the cut-offs (x < DBL_EPSILON, x > 700) follow the reference.
 *
 * Parity is pinned against the compiled reference (oracle/_ref) by the golden
 * fixtures in tests/golden/.
 */
#include "lddmm_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

void orc_set_threads(int n)
{
#ifdef _OPENMP
	if (n > 0) omp_set_num_threads(n);
#else
	(void)n;
#endif
}

/* ------------------------------------------------------------------ Bessel K */

static void bessel_k01(double x, double *k0, double *k1)
{
	const double h = 0.125;
	double s0 = 0.5 * exp(-x), s1 = 0.5 * exp(-x);
	for (int k = 1; k < 100000; ++k) {
		double t = k * h;
		double ch = cosh(t);
		double e = exp(-x * ch);
		s0 += e;
		s1 += e * ch;
		if (e * ch < 1e-20 * s1 && t > 1.0) break;
	}
	*k0 = h * s0;
	*k1 = h * s1;
}

/* polybesselk.cpp:14-51 (p0 = x^2 K0(x)) */
double orc_p0(double x)
{
	if (x < DBL_EPSILON || x > 700.0) return 0.0;
	double k0, k1;
	bessel_k01(x, &k0, &k1);
	return x * x * k0;
}

/* polybesselk.cpp:53-96 (p1 = x K1(x)) */
double orc_p1(double x)
{
	if (x < DBL_EPSILON) return 1.0;
	if (x > 700.0) return 0.0;
	double k0, k1;
	bessel_k01(x, &k0, &k1);
	return x * k1;
}

/* ------------------------------------------------------- deformation kernels */

static inline double dist(const double *a, const double *b, int dim)
{
	double s = 0.0;
	for (int d = 0; d < dim; ++d) {
		double t = a[d] - b[d];
		s += t * t;
	}
	return sqrt(s);
}

/* Kernel value K(d), d = |qi - qj| / width.
 * Gaussian / 3D Matern: computeKernel.cpp:26-41, :160-238; multiplyKernel.cpp:30-49, :186-288.
 * 2D Matern via p0/p1:   computeKernel.cpp:44-154. */
static inline double knl_val(double d, int order, int dim)
{
	if (order == -1) return exp(-d * d);
	if (dim == 3) {
		double e = exp(-d);
		switch (order) {
		case 0: return e;
		case 1: return (1.0 + d) * e;
		case 2: return (3.0 + d * (3.0 + d)) / 3.0 * e;
		case 3: return (15.0 + d * (15.0 + d * (6.0 + d))) / 15.0 * e;
		case 4: return (105.0 + d * (105.0 + d * (45.0 + d * (10.0 + d)))) / 105.0 * e;
		}
		return 0.0;
	}
	double d2 = d * d;
	double p0 = (order == 0) ? 0.0 : orc_p0(d), p1 = orc_p1(d);
	switch (order) {
	case 0: return p1;
	case 1: return 0.5 * (p0 + 2.0 * p1);
	case 2: return (4.0 * p0 + (8.0 + d2) * p1) / 8.0;
	case 3: return ((24.0 + d2) * p0 + 8.0 * (6.0 + d2) * p1) / 48.0;
	case 4: return (12.0 * (16.0 + d2) * p0 + (384.0 + d2 * (72.0 + d2)) * p1) / 384.0;
	}
	return 0.0;
}

/* dK/dqi = c(d) * (qi - qj).  Returns c(d).
 * Gaussian: dqKernel.cpp:56-57; 3D Matern 1..4: :214-215, :239-240, :264-265, :289-291;
 * 2D Matern 1..4: :86-91, :115-122, :146-153, :177-185.  Order 0 is not
 * differentiable at 0 and the reference leaves its gradient at zero. */
static inline double knl_dq(double d, int order, int dim, double w2)
{
	if (order == -1) return -2.0 * exp(-d * d) / w2;
	if (dim == 3) {
		double e = exp(-d);
		switch (order) {
		case 1: return -e / w2;
		case 2: return -(1.0 + d) * e / (3.0 * w2);
		case 3: return -(3.0 + d * (3.0 + d)) * e / (15.0 * w2);
		case 4: return -(15.0 + d * (15.0 + d * (6.0 + d))) * e / (105.0 * w2);
		}
		return 0.0;
	}
	double d2 = d * d;
	switch (order) {
	case 1: return -1.0 / (2.0 * w2) * orc_p1(d);
	case 2: return -1.0 / (8.0 * w2) * (orc_p0(d) + 2.0 * orc_p1(d));
	case 3: return -1.0 / (48.0 * w2) * (4.0 * orc_p0(d) + (8.0 + d2) * orc_p1(d));
	case 4: return -1.0 / (384.0 * w2) * ((24.0 + d2) * orc_p0(d) + 8.0 * (6.0 + d2) * orc_p1(d));
	}
	return 0.0;
}

/* multiplyKernel.cpp:22-292: v_i = sum_j K(qi, qj) a_j */
void orc_multiply_kernel(double *v, const double *q, const double *a, int order, double width,
                         int n, int dim)
{
#pragma omp parallel for schedule(static)
	for (int i = 0; i < n; ++i) {
		double acc[3] = {0.0, 0.0, 0.0};
		const double *qi = q + (size_t)i * dim;
		for (int j = 0; j < n; ++j) {
			const double *qj = q + (size_t)j * dim;
			double k = knl_val(dist(qi, qj, dim) / width, order, dim);
			for (int d = 0; d < dim; ++d) acc[d] += k * a[(size_t)j * dim + d];
		}
		for (int d = 0; d < dim; ++d) v[(size_t)i * dim + d] = acc[d];
	}
}

/* computeKernel.cpp:21-244: dense K (row-major i, j). */
void orc_compute_kernel(double *K, const double *q, int order, double width, int n, int dim)
{
#pragma omp parallel for schedule(static)
	for (int i = 0; i < n; ++i)
		for (int j = 0; j < n; ++j)
			K[(size_t)i * n + j] = knl_val(dist(q + (size_t)i * dim, q + (size_t)j * dim, dim) / width,
			                               order, dim);
}

/* computeKernel.cpp:246-: two point sets, the reference's column-major ni x nj
 * matrix, K[j * ni + i] = K(qi_i, qj_j). */
void orc_compute_kernel2(double *K, const double *qi, int ni, const double *qj, int nj, int order,
                         double width, int dim)
{
#pragma omp parallel for schedule(static)
	for (int j = 0; j < nj; ++j)
		for (int i = 0; i < ni; ++i)
			K[(size_t)j * ni + i] = knl_val(dist(qi + (size_t)i * dim, qj + (size_t)j * dim, dim)
			                                / width, order, dim);
}

/* multiplyKernel.cpp:294-: v_i = sum_j K(qi_i, qj_j) a_j (a given on the j set) */
void orc_multiply_kernel2(double *v, const double *qi, int ni, const double *qj, int nj,
                          const double *a, int order, double width, int dim)
{
#pragma omp parallel for schedule(static)
	for (int i = 0; i < ni; ++i) {
		double acc[3] = {0.0, 0.0, 0.0};
		const double *x = qi + (size_t)i * dim;
		for (int j = 0; j < nj; ++j) {
			double k = knl_val(dist(x, qj + (size_t)j * dim, dim) / width, order, dim);
			for (int d = 0; d < dim; ++d) acc[d] += k * a[(size_t)j * dim + d];
		}
		for (int d = 0; d < dim; ++d) v[(size_t)i * dim + d] = acc[d];
	}
}

/* dqKernel.cpp:307-: l on the i set, r on the j set,
 *   dqi_i = sum_j (l_i.r_j) c(d_ij) (qi_i - qj_j),  dqj_j = sum_i (l_i.r_j) c(d_ij) (qj_j - qi_i).
 * Two independent passes (over i for dqi, over j for dqj). */
void orc_dq_kernel2(double *dqi, double *dqj, const double *qi, int ni, const double *qj, int nj,
                    const double *l, const double *r, int order, double width, int dim)
{
	double w2 = width * width;
	int has_grad = (order == -1) || (order >= 1 && order <= 4);
#pragma omp parallel for schedule(static)
	for (int i = 0; i < ni; ++i) {
		double acc[3] = {0.0, 0.0, 0.0};
		const double *x = qi + (size_t)i * dim, *li = l + (size_t)i * dim;
		if (has_grad) {
			for (int j = 0; j < nj; ++j) {
				const double *y = qj + (size_t)j * dim, *rj = r + (size_t)j * dim;
				double c = knl_dq(dist(x, y, dim) / width, order, dim, w2), lr = 0.0;
				for (int d = 0; d < dim; ++d) lr += li[d] * rj[d];
				for (int d = 0; d < dim; ++d) acc[d] += lr * c * (x[d] - y[d]);
			}
		}
		for (int d = 0; d < dim; ++d) dqi[(size_t)i * dim + d] = acc[d];
	}
#pragma omp parallel for schedule(static)
	for (int j = 0; j < nj; ++j) {
		double acc[3] = {0.0, 0.0, 0.0};
		const double *y = qj + (size_t)j * dim, *rj = r + (size_t)j * dim;
		if (has_grad) {
			for (int i = 0; i < ni; ++i) {
				const double *x = qi + (size_t)i * dim, *li = l + (size_t)i * dim;
				double c = knl_dq(dist(x, y, dim) / width, order, dim, w2), lr = 0.0;
				for (int d = 0; d < dim; ++d) lr += li[d] * rj[d];
				for (int d = 0; d < dim; ++d) acc[d] += lr * c * (y[d] - x[d]);
			}
		}
		for (int d = 0; d < dim; ++d) dqj[(size_t)j * dim + d] = acc[d];
	}
}

/* dqKernel.cpp:31-305: dq_i = sum_j (l_i.r_j + l_j.r_i) c(d_ij) (q_i - q_j) */
void orc_dq_kernel(double *dq, const double *q, const double *l, const double *r, int order,
                   double width, int n, int dim)
{
	double w2 = width * width;
	int has_grad = (order == -1) || (order >= 1 && order <= 4);
#pragma omp parallel for schedule(static)
	for (int i = 0; i < n; ++i) {
		double acc[3] = {0.0, 0.0, 0.0};
		const double *qi = q + (size_t)i * dim, *li = l + (size_t)i * dim, *ri = r + (size_t)i * dim;
		if (has_grad) {
			for (int j = 0; j < n; ++j) {
				const double *qj = q + (size_t)j * dim, *lj = l + (size_t)j * dim,
				             *rj = r + (size_t)j * dim;
				double c = knl_dq(dist(qi, qj, dim) / width, order, dim, w2);
				double lr = 0.0, lr2 = 0.0;
				for (int d = 0; d < dim; ++d) lr += li[d] * rj[d];
				for (int d = 0; d < dim; ++d) lr2 += lj[d] * ri[d];
				lr += lr2;
				for (int d = 0; d < dim; ++d) acc[d] += lr * c * (qi[d] - qj[d]);
			}
		}
		for (int d = 0; d < dim; ++d) dq[(size_t)i * dim + d] = acc[d];
	}
}

/* ------------------------------------------------------------------ varifold */

/* geometricFunction (varifold3D.cpp:41-93 / varifold2D.cpp:34-84):
 * centre kernel value and its gradient factor dk such that dK/dc1 = dk (c1 - c2). */
static inline double cen_knl(const double *c1, const double *c2, int dim, char type, double w,
                             double *dk)
{
	double s = 0.0;
	for (int d = 0; d < dim; ++d) {
		double t = c1[d] - c2[d];
		s += t * t;
	}
	double w2 = w * w;
	if (type == 'G') {
		double k = exp(-s / w2);
		if (dk) *dk = -2.0 * k / w2;
		return k;
	}
	if (type == 'C') {
		double k = 1.0 / (1.0 + s / w2);
		if (dk) *dk = -2.0 * k * k / w2;
		return k;
	}
	if (dk) *dk = 0.0;
	return 0.0;
}

/* grassmanFunction (varifold3D.cpp:95-188 / varifold2D.cpp:86-178): direction kernel
 * value b(ang) and its derivative db/dang, ang = v1 . v2 (unit vectors). */
static inline double dir_knl(double ang, char type, double w, double *db)
{
	double w2 = w * w;
	switch (type) {
	case 'B': if (db) *db = 2.0 * ang; return ang * ang;
	case 'L': if (db) *db = 1.0; return ang;
	case 'O': {
		double k = exp(2.0 * (ang - 1.0) / w2);
		if (db) *db = 2.0 * k / w2;
		return k;
	}
	case 'U': {
		double k = exp(2.0 * (ang * ang - 1.0) / w2);
		if (db) *db = 4.0 * ang * k / w2;
		return k;
	}
	}
	if (db) *db = 0.0;
	return 0.0;
}

/* landmarksToVarifoldKernel (varifold3D.cpp:8-39, varifold2D.cpp:8-32) */
static void elm_geometry(const orc_problem *P, const double *nde, double *cen, double *dir,
                         double *vol)
{
	int dim = P->dim;
	for (int e = 0; e < P->dfm_elm_num; ++e) {
		const int *v = P->dfm_elm_vtx + (size_t)e * dim;
		if (dim == 3) {
			const double *q0 = nde + 3 * v[0], *q1 = nde + 3 * v[1], *q2 = nde + 3 * v[2];
			double a[3], b[3], n[3];
			for (int d = 0; d < 3; ++d) {
				cen[3 * e + d] = (q0[d] + q1[d] + q2[d]) / 3.0;
				a[d] = q1[d] - q0[d];
				b[d] = q2[d] - q0[d];
			}
			n[0] = a[1] * b[2] - a[2] * b[1];
			n[1] = -a[0] * b[2] + a[2] * b[0];
			n[2] = a[0] * b[1] - a[1] * b[0];
			double len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
			for (int d = 0; d < 3; ++d) dir[3 * e + d] = n[d] / len;
			vol[e] = 0.5 * len;
		} else {
			const double *q0 = nde + 2 * v[0], *q1 = nde + 2 * v[1];
			double t[2];
			for (int d = 0; d < 2; ++d) {
				cen[2 * e + d] = 0.5 * (q0[d] + q1[d]);
				t[d] = q1[d] - q0[d];
			}
			double len = sqrt(t[0] * t[0] + t[1] * t[1]);
			dir[2 * e] = t[0] / len;
			dir[2 * e + 1] = t[1] / len;
			vol[e] = len;
		}
	}
}

/* Target self-term (the last double loop of dqVf_Kernel, varifold3D.cpp:334-354). */
double orc_varifold_tt(const orc_problem *P)
{
	int dim = P->dim, Et = P->tgt_elm_num;
	double *row = (double *)calloc((size_t)Et, sizeof(double));
#pragma omp parallel for schedule(static)
	for (int i = 0; i < Et; ++i) {
		const double *ci = P->tgt_cen_pos + (size_t)i * dim, *ni = P->tgt_uni_dir + (size_t)i * dim;
		double s = 0.0;
		for (int j = 0; j < Et; ++j) {
			const double *cj = P->tgt_cen_pos + (size_t)j * dim, *nj = P->tgt_uni_dir + (size_t)j * dim;
			double ang = 0.0;
			for (int d = 0; d < dim; ++d) ang += ni[d] * nj[d];
			s += cen_knl(ci, cj, dim, P->cen_knl_type, P->cen_knl_width, NULL) *
			     dir_knl(ang, P->dir_knl_type, P->dir_knl_width, NULL) * P->tgt_elm_vol[i] *
			     P->tgt_elm_vol[j];
		}
		row[i] = s;
	}
	double tt = 0.0;
	for (int i = 0; i < Et; ++i) tt += row[i];
	free(row);
	return tt;
}

/* varifold (gradient overload): varifold3D.cpp:410-435 / varifold2D.cpp:378-403,
 * with dqVf_Kernel (3D :259-357, 2D :245-335) and dqVfdGatherKernel
 * (3D :359-391, 2D :337-359). */
int orc_varifold(const orc_problem *P, const double *nde, double *val, double *dq)
{
	int dim = P->dim, Ed = P->dfm_elm_num, Et = P->tgt_elm_num, N = P->nde_num;
	double *cen = (double *)malloc(sizeof(double) * dim * (size_t)Ed);
	double *dir = (double *)malloc(sizeof(double) * dim * (size_t)Ed);
	double *vol = (double *)malloc(sizeof(double) * (size_t)Ed);
	double *dc = (double *)calloc((size_t)dim * Ed, sizeof(double));
	double *dd = (double *)calloc((size_t)dim * Ed, sizeof(double));
	double *row = (double *)calloc((size_t)Ed, sizeof(double));
	if (!cen || !dir || !vol || !dc || !dd || !row) return -5;
	elm_geometry(P, nde, cen, dir, vol);
	/* n1Len in grassmanFunction: 2 * area in 3D (varifold3D.cpp:287), length in 2D
	 * (varifold2D.cpp:273); the area/length derivative w.r.t. the unnormalised
	 * direction is 0.5 n in 3D (:296) and n in 2D (:281). */
	double vfac = (dim == 3) ? 0.5 : 1.0;
	char ct = P->cen_knl_type, dt = P->dir_knl_type;
	double cw = P->cen_knl_width, dw = P->dir_knl_width;
#pragma omp parallel for schedule(static)
	for (int i = 0; i < Ed; ++i) {
		const double *ci = cen + (size_t)i * dim, *ni = dir + (size_t)i * dim;
		double ai = vol[i];
		double nlen = (dim == 3) ? 2.0 * ai : ai;
		double s = 0.0, dci[3] = {0, 0, 0}, ddi[3] = {0, 0, 0};
		for (int pass = 0; pass < 2; ++pass) {
			int M = pass == 0 ? Ed : Et;
			const double *C = pass == 0 ? cen : P->tgt_cen_pos;
			const double *D = pass == 0 ? dir : P->tgt_uni_dir;
			const double *A = pass == 0 ? vol : P->tgt_elm_vol;
			double sgn = pass == 0 ? 1.0 : -1.0;
			double vsc = pass == 0 ? 1.0 : 2.0;
			for (int j = 0; j < M; ++j) {
				const double *cj = C + (size_t)j * dim, *nj = D + (size_t)j * dim;
				double aj = A[j];
				double dk, db;
				double k = cen_knl(ci, cj, dim, ct, cw, &dk);
				double ang = 0.0;
				for (int d = 0; d < dim; ++d) ang += ni[d] * nj[d];
				double b = dir_knl(ang, dt, dw, &db);
				s += sgn * vsc * k * b * ai * aj;
				for (int d = 0; d < dim; ++d) {
					double dkv = dk * (ci[d] - cj[d]);
					double dbv = db / nlen * (-ang * ni[d] + nj[d]);
					dci[d] += sgn * 2.0 * dkv * b * ai * aj;
					ddi[d] += sgn * 2.0 * k * (dbv * ai + b * vfac * ni[d]) * aj;
				}
			}
		}
		row[i] = s;
		for (int d = 0; d < dim; ++d) {
			dc[(size_t)i * dim + d] = dci[d];
			dd[(size_t)i * dim + d] = ddi[d];
		}
	}
	double v = 0.0;
	for (int i = 0; i < Ed; ++i) v += row[i];
	v += orc_varifold_tt(P);
	*val = v;

	int R = P->dfm_elm_ifo_num;
	for (int q = 0; q < N; ++q) {
		const int *ifo = P->dfm_elm_ifo + (size_t)q * R;
		double acc[3] = {0, 0, 0};
		int adj = ifo[0];
		for (int k = 0; k < adj; ++k) {
			if (dim == 3) {
				int e = ifo[1 + 3 * k], a = ifo[2 + 3 * k], b = ifo[3 + 3 * k];
				double ab[3], x[3];
				const double *dde = dd + 3 * (size_t)e;
				for (int d = 0; d < 3; ++d) ab[d] = nde[3 * a + d] - nde[3 * b + d];
				x[0] = dde[1] * ab[2] - dde[2] * ab[1];
				x[1] = -dde[0] * ab[2] + dde[2] * ab[0];
				x[2] = dde[0] * ab[1] - dde[1] * ab[0];
				for (int d = 0; d < 3; ++d) acc[d] += dc[3 * (size_t)e + d] / 3.0 + x[d];
			} else {
				int e = ifo[1 + 2 * k], sg = ifo[2 + 2 * k];
				for (int d = 0; d < 2; ++d) acc[d] += 0.5 * dc[2 * (size_t)e + d] + sg * dd[2 * (size_t)e + d];
			}
		}
		for (int d = 0; d < dim; ++d) dq[(size_t)q * dim + d] = acc[d];
	}
	free(cen); free(dir); free(vol); free(dc); free(dd); free(row);
	return 0;
}

/* --------------------------------------------------------------- objective */

/* objgrd.cpp:26-90, matrix-free. */
int orc_objgrd(const orc_problem *P, const double *alp, double *fcn, double *grd)
{
	int dim = P->dim, N = P->nde_num, T = P->time_num - 1;
	size_t DN = (size_t)dim * N;
	double dt = P->time_stp;
	double *stk = (double *)malloc(sizeof(double) * DN * (T + 1));
	double *v = (double *)malloc(sizeof(double) * DN);
	double *p = (double *)malloc(sizeof(double) * DN);
	double *amp = (double *)malloc(sizeof(double) * DN);
	double *pdot = (double *)malloc(sizeof(double) * DN);
	double *dqv = (double *)malloc(sizeof(double) * DN);
	if (!stk || !v || !p || !amp || !pdot || !dqv) return -5;
	memcpy(stk, P->ini_nde, sizeof(double) * DN);
	double f = 0.0;
	for (int t = 0; t < T; ++t) {
		const double *a = alp + (size_t)t * DN;
		orc_multiply_kernel(v, stk + t * DN, a, P->knl_order, P->knl_width, N, dim);
		double e = 0.0;
		for (size_t k = 0; k < DN; ++k) e += a[k] * v[k];
		f += e;
		for (size_t k = 0; k < DN; ++k) stk[(t + 1) * DN + k] = stk[t * DN + k] + dt * v[k];
	}
	double vfd;
	int rc = orc_varifold(P, stk + T * DN, &vfd, dqv);
	if (rc) return rc;
	*fcn = dt * 0.5 * f + P->dis_wgt * vfd;
	for (size_t k = 0; k < DN; ++k) p[k] = -P->dis_wgt * dqv[k];
	for (int t = T - 1; t >= 0; --t) {
		const double *a = alp + (size_t)t * DN;
		double *g = grd + (size_t)t * DN;
		for (size_t k = 0; k < DN; ++k) amp[k] = a[k] - p[k];
		orc_multiply_kernel(g, stk + t * DN, amp, P->knl_order, P->knl_width, N, dim);
		for (size_t k = 0; k < DN; ++k) amp[k] = amp[k] - 0.5 * a[k];
		orc_dq_kernel(pdot, stk + t * DN, amp, a, P->knl_order, P->knl_width, N, dim);
		for (size_t k = 0; k < DN; ++k) p[k] = p[k] - dt * pdot[k];
	}
	for (size_t k = 0; k < DN * T; ++k) grd[k] = dt * grd[k];
	free(stk); free(v); free(p); free(amp); free(pdot); free(dqv);
	return 0;
}

/* ----------------------------------------------------------------- L-BFGS */

static double dot(const double *a, const double *b, size_t n)
{
	double s = 0.0;
	for (size_t k = 0; k < n; ++k) s += a[k] * b[k];
	return s;
}

/* getDirection.cpp:9-66 (Nocedal & Wright, Algorithm 7.4) */
static void get_direction(double *dir, double H0, const double *g, const double *S, const double *Y,
                          int newIdx, int hisNum, int memNum, double *rec, size_t n)
{
	memcpy(dir, g, sizeof(double) * n);
	for (int h = 0; h < hisNum; ++h) {
		int idx = newIdx - h;
		if (idx < 0) idx += memNum;
		const double *s = S + (size_t)idx * n, *y = Y + (size_t)idx * n;
		double a = dot(s, dir, n) / dot(s, y, n);
		for (size_t k = 0; k < n; ++k) dir[k] -= a * y[k];
		rec[idx] = a;
	}
	for (size_t k = 0; k < n; ++k) dir[k] *= H0;
	int oldIdx = (hisNum < memNum) ? 0 : newIdx + 1;
	if (oldIdx == memNum) oldIdx = 0;
	for (int h = 0; h < hisNum; ++h) {
		int idx = oldIdx + h;
		if (idx >= memNum) idx -= memNum;
		const double *s = S + (size_t)idx * n, *y = Y + (size_t)idx * n;
		double b = dot(y, dir, n) / dot(s, y, n);
		for (size_t k = 0; k < n; ++k) dir[k] += (rec[idx] - b) * s[k];
	}
	for (size_t k = 0; k < n; ++k) dir[k] = -dir[k];
}

typedef struct {
	const orc_problem *P;
	double *trace_f, *trace_g2;
	int cap, len;
} evalctx;

static int eval(evalctx *E, const double *x, double *f, double *g, size_t n)
{
	int rc = orc_objgrd(E->P, x, f, g);
	if (E->len < E->cap) {
		if (E->trace_f) E->trace_f[E->len] = *f;
		if (E->trace_g2) E->trace_g2[E->len] = dot(g, g, n);
	}
	E->len++;
	return rc;
}

/* lineSearch.cpp:26-110 (weak Wolfe bracketing, modified from HANSO 2.0) */
static int line_search(evalctx *E, const double *x, const double *g, const double *d, double f,
                       double w1, double w2, double tol, double *xt, double *gt, double *ft,
                       double *stp, int *cnt, size_t n)
{
	double relL = 0.0, relR = DBL_MAX, t = 1.0;
	double slp = dot(g, d, n);
	if (slp > -DBL_MIN) return 1;
	double dlen = sqrt(dot(d, d, n));
	double lb = log2(1e5 * dlen), le = log2(1e5 / dlen);
	int bisMax = (int)((50 > lb) ? 50 : lb);
	int epdMax = (int)((10 > le) ? 10 : le);
	int bis = 0, epd = 0;
	*cnt = 0;
	while (bis <= bisMax && epd <= epdMax) {
		for (size_t k = 0; k < n; ++k) xt[k] = x[k] + t * d[k];
		if (eval(E, xt, ft, gt, n)) return -5;
		++*cnt;
		if (sqrt(dot(gt, gt, n)) < tol) { *stp = t * dlen; return 0; }
		double st = dot(gt, d, n);
		if (*ft >= f + w1 * t * slp) relR = t;
		else if (st <= w2 * slp) relL = t;
		else { *stp = t * dlen; return 0; }
		if (relR == DBL_MAX) { t *= 2; ++epd; }
		else { t = 0.5 * (relL + relR); ++bis; }
	}
	return (relR == DBL_MAX) ? 2 : 3;
}

/* LBFGS.cpp:25-112 */
int orc_lbfgs(const orc_problem *P, int itr_max, double tol, double wolfe1, double wolfe2,
              int mem_num, double *x, double *fcn_out, double *g,
              int *ls_code, int *iters_out, int *evals_out,
              double *trace_f, double *trace_g2, int trace_cap)
{
	size_t n = (size_t)P->dim * P->nde_num * (P->time_num - 1);
	double *S = (double *)calloc(n * mem_num, sizeof(double));
	double *Y = (double *)calloc(n * mem_num, sizeof(double));
	double *d = (double *)malloc(sizeof(double) * n);
	double *xt = (double *)malloc(sizeof(double) * n);
	double *gt = (double *)malloc(sizeof(double) * n);
	double *rec = (double *)calloc(mem_num, sizeof(double));
	if (!S || !Y || !d || !xt || !gt || !rec) return -5;
	evalctx E = {P, trace_f, trace_g2, trace_cap, 0};
	double f, ft;
	if (ls_code) *ls_code = 0;
	int ret = 0, done = 0;
	if (eval(&E, x, &f, g, n)) return -5;
	double glen = sqrt(dot(g, g, n));
	int newIdx = -1;
	for (int itr = 1; itr <= itr_max; ++itr) {
		if (glen < tol) break;
		double H0 = 1.0;
		if (newIdx != -1) {
			const double *s = S + (size_t)newIdx * n, *y = Y + (size_t)newIdx * n;
			H0 = dot(s, y, n) / dot(y, y, n);
		}
		int his = (itr <= mem_num) ? itr - 1 : mem_num;
		get_direction(d, H0, g, S, Y, newIdx, his, mem_num, rec, n);
		double stp;
		int cnt;
		int err = line_search(&E, x, g, d, f, wolfe1, wolfe2, tol, xt, gt, &ft, &stp, &cnt, n);
		if (err != 0) {
			if (ls_code) *ls_code = err;
			ret = 1;
			break;
		}
		newIdx = (newIdx == mem_num - 1) ? 0 : newIdx + 1;
		for (size_t k = 0; k < n; ++k) {
			S[(size_t)newIdx * n + k] = xt[k] - x[k];
			Y[(size_t)newIdx * n + k] = gt[k] - g[k];
		}
		memcpy(x, xt, sizeof(double) * n);
		memcpy(g, gt, sizeof(double) * n);
		f = ft;
		glen = sqrt(dot(g, g, n));
		++done;
	}
	*fcn_out = f;
	if (iters_out) *iters_out = done;
	if (evals_out) *evals_out = E.len;
	free(S); free(Y); free(d); free(xt); free(gt); free(rec);
	return ret;
}

/* ------------------------------------------------------------- adjacency */

/* getElmIfo.m:1-59.  For each vertex, in increasing element order, the element
 * index and (2D) the sign -1 when the vertex is the element's first vertex, +1
 * otherwise, or (3D) the two other vertices in the order that makes
 * dd x (q_a - q_b) the derivative of the element normal. */
int orc_elm_ifo(const int *elm_vtx, int vpe, int elm_num, int nde_num, int *ifo)
{
	if (vpe != 2 && vpe != 3) return -1;
	int *cnt = (int *)calloc((size_t)nde_num, sizeof(int));
	if (!cnt) return -1;
	for (int e = 0; e < elm_num; ++e)
		for (int k = 0; k < vpe; ++k) {
			int v = elm_vtx[(size_t)e * vpe + k];
			if (v < 0 || v >= nde_num) { free(cnt); return -1; }
			cnt[v]++;
		}
	int mx = 0;
	for (int v = 0; v < nde_num; ++v) if (cnt[v] > mx) mx = cnt[v];
	int rows = 1 + mx * vpe;
	if (ifo) {
		memset(ifo, 0, sizeof(int) * (size_t)rows * nde_num);
		/* MATLAB's find() on a vpe x E matrix walks column-major: element by
		 * element, local vertex by local vertex. */
		for (int e = 0; e < elm_num; ++e)
			for (int k = 0; k < vpe; ++k) {
				int v = elm_vtx[(size_t)e * vpe + k];
				int *col = ifo + (size_t)v * rows;
				int a = col[0]++;
				const int *ev = elm_vtx + (size_t)e * vpe;
				if (vpe == 2) {
					col[1 + 2 * a] = e;
					col[2 + 2 * a] = (k == 0) ? -1 : 1;
				} else {
					col[1 + 3 * a] = e;
					if (k == 0) { col[2 + 3 * a] = ev[2]; col[3 + 3 * a] = ev[1]; }
					else if (k == 1) { col[2 + 3 * a] = ev[0]; col[3 + 3 * a] = ev[2]; }
					else { col[2 + 3 * a] = ev[1]; col[3 + 3 * a] = ev[0]; }
				}
			}
	}
	free(cnt);
	return rows;
}

/* computeNodePosition.m:1-20 */
void orc_shoot(const double *ini, const double *alp, int order, double width, double dt,
               int time_num, int n, int dim, double *nde_stk, double *vlc_stk)
{
	size_t DN = (size_t)dim * n;
	memcpy(nde_stk, ini, sizeof(double) * DN);
	for (int t = 0; t < time_num - 1; ++t) {
		double *v = vlc_stk + t * DN;
		orc_multiply_kernel(v, nde_stk + t * DN, alp + t * DN, order, width, n, dim);
		for (size_t k = 0; k < DN; ++k) nde_stk[(t + 1) * DN + k] = nde_stk[t * DN + k] + dt * v[k];
	}
}
