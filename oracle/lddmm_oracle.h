/*
 * CPU oracle: an FP64 restatement of the reference's C++ LDDMM path
 * (dnhsieh/LDDMM, Cpp/src/*).  TEST INFRASTRUCTURE ONLY: the product library
 * never links, loads or calls it; tests, smoke() and bench.py's CPU baseline use
 * it as the checker.
 *
 * Parity pin: the restatement is checked against the reference itself, compiled in
 * place into oracle/_ref/ (see oracle/Makefile), through the committed golden
 * fixtures in tests/golden/ (generator: tests/golden/make_golden.py).
 *
 * Layout follows the reference's C++ back-end: coordinates D-fastest, then node,
 * then time step (Cpp/src/objgrd.cpp:47-50).  Element/vertex tables are 0-based.
 */
#ifndef LDDMM_ORACLE_H
#define LDDMM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
	int dim;               /* 2 or 3 */
	int nde_num;           /* landmarks N */
	int time_num;          /* number of time points; T = time_num - 1 Euler steps */
	double time_stp;       /* dt */
	int knl_order;         /* -1 Gaussian, 0..4 Matern */
	double knl_width;
	const double *ini_nde; /* dim x N */
	double dis_wgt;
	int dfm_elm_num;
	const int *dfm_elm_vtx; /* dim x E_d (a segment has 2 vertices, a triangle 3) */
	int dfm_elm_ifo_num;    /* rows of the adjacency table */
	const int *dfm_elm_ifo; /* dfm_elm_ifo_num x N */
	int tgt_elm_num;
	const double *tgt_cen_pos; /* dim x E_t */
	const double *tgt_uni_dir; /* dim x E_t */
	const double *tgt_elm_vol; /* E_t */
	char cen_knl_type;         /* 'G' Gaussian, 'C' Cauchy */
	double cen_knl_width;
	char dir_knl_type;         /* 'B' Binet, 'L' linear, 'O' oriented Gauss, 'U' unoriented Gauss */
	double dir_knl_width;
} orc_problem;

/* x^2 K0(x) and x K1(x) (Cpp/src/polybesselk.cpp:14-96 semantics, incl. cut-offs). */
double orc_p0(double x);
double orc_p1(double x);

void orc_multiply_kernel(double *v, const double *q, const double *a, int order, double width,
                         int n, int dim);
void orc_dq_kernel(double *dq, const double *q, const double *l, const double *r, int order,
                   double width, int n, int dim);
void orc_compute_kernel(double *K, const double *q, int order, double width, int n, int dim);
void orc_compute_kernel2(double *K, const double *qi, int ni, const double *qj, int nj, int order,
                         double width, int dim);
void orc_multiply_kernel2(double *v, const double *qi, int ni, const double *qj, int nj,
                          const double *a, int order, double width, int dim);
void orc_dq_kernel2(double *dqi, double *dqj, const double *qi, int ni, const double *qj, int nj,
                    const double *l, const double *r, int order, double width, int dim);

int orc_varifold(const orc_problem *P, const double *nde, double *val, double *dq);
/* Varifold value only, used to time the target self-term alone. */
double orc_varifold_tt(const orc_problem *P);

int orc_objgrd(const orc_problem *P, const double *alp, double *fcn, double *grd);

/* L-BFGS with weak-Wolfe line search (Cpp/src/LBFGS.cpp, lineSearch.cpp, getDirection.cpp).
 * Returns 0, or 1 when the line search failed (its code in *ls_code: 1 not descent,
 * 2 unbounded, 3 bracketed but not satisfied).  Records per evaluation f and |g|^2,
 * and per iteration f and |g|. */
int orc_lbfgs(const orc_problem *P, int itr_max, double tol, double wolfe1, double wolfe2,
              int mem_num, double *alp_inout, double *fcn_out, double *grd_out,
              int *ls_code, int *iters_out, int *evals_out,
              double *trace_f, double *trace_g2, int trace_cap);

/* Vertex -> adjacent element table (Cpp/src/getElmIfo.m).  elm_vtx is 0-based,
 * vtx_per_elm x elm_num.  Writes rows x nde_num (column per vertex) into ifo when it
 * is non-NULL; returns the row count (1 + vtx_per_elm * max adjacency) or -1. */
int orc_elm_ifo(const int *elm_vtx, int vtx_per_elm, int elm_num, int nde_num, int *ifo);

/* Trajectory (Cpp/src/computeNodePosition.m): nde_stk dim x N x time_num,
 * vlc_stk dim x N x (time_num-1). */
void orc_shoot(const double *ini, const double *alp, int order, double width, double dt,
               int time_num, int n, int dim, double *nde_stk, double *vlc_stk);

void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
