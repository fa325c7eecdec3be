/*
 * Project-written driver for the reference's C++ FP64 path, compiled in place from
 * the read-only reference tree by oracle/Makefile into oracle/_ref/libref{2,3}d.so.
 *
 * It replaces the MATLAB MEX entry point (Cpp/src/LDDMM.cpp:11-98) with plain
 * extern "C" functions so the reference can be called through ctypes from the
 * golden-fixture generator and from bench.py's reference (CPU) arm.
 *
 * Workspace sizing and carving follow LDDMM.cpp:57-80 exactly, using the reference's
 * own assignFcnStructMemory / assignOptStructMemory (Cpp/src/assignStructMemory.cpp).
 *
 * The reference's objgrd.cpp is compiled with -Dobjgrd=refimpl_objgrd so that the
 * wrapper `objgrd` below sits between LBFGS/lineSearch and the real objective: it
 * forwards every call unchanged and records (f, |g|^2) per evaluation, which gives an
 * evaluation trace for L-BFGS parity tests.
 *
 * Test infrastructure only: never linked into the product library.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <vector>
#include "struct.h"
#include "constants.h"

long long assignFcnStructMemory(fcndata &, double *);
long long assignOptStructMemory(optdata &, double *);
int  LBFGS(double *, double *, double *, optdata &, fcndata &);
void refimpl_objgrd(double *, double *, double *, fcndata &);
void varifoldITF(double *, double *, double *, fcndata &);
void computeKernel(double *, double *, int, double, int, int);
void multiplyKernel(double *, double *, double *, int, double, int, int);
void dqKernel(double *, double *, double *, double *, int, double, int, int);
void computeKernel(double *, double *, double *, int, double, int, int, int);
void multiplyKernel(double *, double *, double *, double *, int, double, int, int, int);
void dqKernel(double *, double *, double *, double *, double *, double *, int, double, int, int,
              int);

static std::vector<double> g_trace_f;
static std::vector<double> g_trace_g2;
static int g_trace_on = 0;

/* Interposer between the reference optimiser and the reference objective. */
void objgrd(double *fcnVal, double *grdStk, double *alpStk, fcndata &fcnObj)
{
	refimpl_objgrd(fcnVal, grdStk, alpStk, fcnObj);
	if (g_trace_on) {
		double g2 = 0.0;
		for (int k = 0; k < fcnObj.varNum; ++k) g2 += grdStk[k] * grdStk[k];
		g_trace_f.push_back(*fcnVal);
		g_trace_g2.push_back(g2);
	}
}

struct RefProblem {
	fcndata fcn;
	double *work;
};

/* Mirrors LDDMM.cpp:16-80 minus the MEX argument unpacking. */
static int setup(RefProblem &P, const double *iniNde, int ndeNum, int timeNum, double timeStp,
                 int knlOrder, double knlWidth,
                 const int *elmVtx, int dfmElmNum, const int *elmIfo, int elmIfoNum,
                 const double *tgtCen, const double *tgtDir, const double *tgtVol, int tgtElmNum,
                 char cenType, double cenWidth, char dirType, double dirWidth, double disWgt)
{
	fcndata &f = P.fcn;
	memset(&f, 0, sizeof(f));
	f.prm.iniNdeMat = const_cast<double *>(iniNde);
	f.prm.ndeNum = ndeNum;
	f.prm.knlOrder = knlOrder;
	f.prm.knlWidth = knlWidth;
	f.prm.timeStp = timeStp;
	f.prm.timeNum = timeNum;
	f.dis.dfmElmVtxMat = const_cast<int *>(elmVtx);
	f.dis.dfmElmIfoMat = const_cast<int *>(elmIfo);
	f.dis.tgtCenPosMat = const_cast<double *>(tgtCen);
	f.dis.tgtUniDirMat = const_cast<double *>(tgtDir);
	f.dis.tgtElmVolVec = const_cast<double *>(tgtVol);
	f.dis.cenKnlType = cenType;
	f.dis.cenKnlWidth = cenWidth;
	f.dis.dirKnlType = dirType;
	f.dis.dirKnlWidth = dirWidth;
	f.dis.disWgt = disWgt;
	f.dis.dfmNdeNum = ndeNum;
	f.dis.dfmElmNum = dfmElmNum;
	f.dis.dfmElmIfoNum = elmIfoNum;
	f.dis.tgtElmNum = tgtElmNum;
	f.varNum = DIMNUM * ndeNum * (timeNum - 1);

	long long cnt = (long long)dfmElmNum * (DIMNUM * 4 + 1)
	              + (long long)ndeNum * DIMNUM * (timeNum + 5)
	              + (long long)ndeNum * ndeNum * (timeNum - 1);
	P.work = (double *)calloc(cnt, sizeof(double));
	if (!P.work) return -5;
	if (assignFcnStructMemory(f, P.work) != cnt) { free(P.work); return -1; }
	return 0;
}

extern "C" {

int ref_dim(void) { return DIMNUM; }

int ref_objgrd(const double *iniNde, int ndeNum, int timeNum, double timeStp,
               int knlOrder, double knlWidth,
               const int *elmVtx, int dfmElmNum, const int *elmIfo, int elmIfoNum,
               const double *tgtCen, const double *tgtDir, const double *tgtVol, int tgtElmNum,
               char cenType, double cenWidth, char dirType, double dirWidth, double disWgt,
               const double *alp, double *fcn, double *grd)
{
	RefProblem P;
	int rc = setup(P, iniNde, ndeNum, timeNum, timeStp, knlOrder, knlWidth, elmVtx, dfmElmNum,
	               elmIfo, elmIfoNum, tgtCen, tgtDir, tgtVol, tgtElmNum,
	               cenType, cenWidth, dirType, dirWidth, disWgt);
	if (rc) return rc;
	std::vector<double> a(alp, alp + P.fcn.varNum);
	refimpl_objgrd(fcn, grd, a.data(), P.fcn);
	free(P.work);
	return 0;
}

/* LDDMM.cpp:82-88: copy the initial momenta, run LBFGS.  Returns LBFGS's code. */
int ref_lbfgs(const double *iniNde, int ndeNum, int timeNum, double timeStp,
              int knlOrder, double knlWidth,
              const int *elmVtx, int dfmElmNum, const int *elmIfo, int elmIfoNum,
              const double *tgtCen, const double *tgtDir, const double *tgtVol, int tgtElmNum,
              char cenType, double cenWidth, char dirType, double dirWidth, double disWgt,
              int itrMax, double tolVal, double wolfe1, double wolfe2, int memNum, int vbsFlg,
              double *alp_inout, double *fcn_out, double *grd_out,
              double *trace_f, double *trace_g2, int trace_cap, int *trace_len)
{
	RefProblem P;
	int rc = setup(P, iniNde, ndeNum, timeNum, timeStp, knlOrder, knlWidth, elmVtx, dfmElmNum,
	               elmIfo, elmIfoNum, tgtCen, tgtDir, tgtVol, tgtElmNum,
	               cenType, cenWidth, dirType, dirWidth, disWgt);
	if (rc) return rc;
	optdata o;
	memset(&o, 0, sizeof(o));
	o.varNum = P.fcn.varNum;
	o.memNum = memNum;
	o.itrMax = itrMax;
	o.tolVal = tolVal;
	o.wolfe1 = wolfe1;
	o.wolfe2 = wolfe2;
	o.vbsFlg = vbsFlg != 0;
	long long ocnt = (long long)o.varNum * (5 + o.memNum * 2) + o.memNum;
	double *owork = (double *)calloc(ocnt, sizeof(double));
	if (!owork) { free(P.work); return -5; }
	if (assignOptStructMemory(o, owork) != ocnt) { free(owork); free(P.work); return -1; }

	g_trace_f.clear();
	g_trace_g2.clear();
	g_trace_on = 1;
	int ret = LBFGS(fcn_out, grd_out, alp_inout, o, P.fcn);
	g_trace_on = 0;
	fflush(stdout);
	int n = (int)g_trace_f.size();
	if (trace_len) *trace_len = n;
	for (int k = 0; k < n && k < trace_cap; ++k) {
		if (trace_f) trace_f[k] = g_trace_f[k];
		if (trace_g2) trace_g2[k] = g_trace_g2[k];
	}
	free(owork);
	free(P.work);
	return ret;
}

/* varifoldITF (Cpp/src/varifoldITF.cpp:7) at the given landmark positions. */
int ref_varifold(const double *nde, int ndeNum,
                 const int *elmVtx, int dfmElmNum, const int *elmIfo, int elmIfoNum,
                 const double *tgtCen, const double *tgtDir, const double *tgtVol, int tgtElmNum,
                 char cenType, double cenWidth, char dirType, double dirWidth,
                 double *val, double *dq)
{
	RefProblem P;
	int rc = setup(P, nde, ndeNum, 2, 1.0, -1, 1.0, elmVtx, dfmElmNum, elmIfo, elmIfoNum,
	               tgtCen, tgtDir, tgtVol, tgtElmNum, cenType, cenWidth, dirType, dirWidth, 1.0);
	if (rc) return rc;
	std::vector<double> q(nde, nde + DIMNUM * ndeNum);
	varifoldITF(val, dq, q.data(), P.fcn);
	free(P.work);
	return 0;
}

void ref_multiply_kernel(double *v, const double *q, const double *a, int order, double width,
                         int n, int dim)
{
	std::vector<double> qq(q, q + (size_t)dim * n), aa(a, a + (size_t)dim * n);
	multiplyKernel(v, qq.data(), aa.data(), order, width, n, dim);
}

void ref_dq_kernel(double *dq, const double *q, const double *l, const double *r, int order,
                   double width, int n, int dim)
{
	std::vector<double> qq(q, q + (size_t)dim * n), ll(l, l + (size_t)dim * n),
	    rr(r, r + (size_t)dim * n);
	dqKernel(dq, qq.data(), ll.data(), rr.data(), order, width, n, dim);
}

void ref_compute_kernel(double *K, const double *q, int order, double width, int n, int dim)
{
	std::vector<double> qq(q, q + (size_t)dim * n);
	computeKernel(K, qq.data(), order, width, n, dim);
}

/* Two-set overloads (computeKernel.cpp:246, multiplyKernel.cpp:294, dqKernel.cpp:307):
 * K[j * ni + i] = K(qi_i, qj_j); v_i = sum_j K(qi_i, qj_j) a_j;
 * dqi_i = sum_j (l_i . r_j) c (qi_i - qj_j), dqj_j = sum_i (l_i . r_j) c (qj_j - qi_i). */
void ref_compute_kernel2(double *K, const double *qi, int ni, const double *qj, int nj, int order,
                         double width, int dim)
{
	std::vector<double> a(qi, qi + (size_t)dim * ni), b(qj, qj + (size_t)dim * nj);
	computeKernel(K, a.data(), b.data(), order, width, ni, nj, dim);
}

void ref_multiply_kernel2(double *v, const double *qi, int ni, const double *qj, int nj,
                          const double *a, int order, double width, int dim)
{
	std::vector<double> x(qi, qi + (size_t)dim * ni), y(qj, qj + (size_t)dim * nj),
	    aa(a, a + (size_t)dim * nj);
	multiplyKernel(v, x.data(), y.data(), aa.data(), order, width, ni, nj, dim);
}

void ref_dq_kernel2(double *dqi, double *dqj, const double *qi, int ni, const double *qj, int nj,
                    const double *l, const double *r, int order, double width, int dim)
{
	std::vector<double> x(qi, qi + (size_t)dim * ni), y(qj, qj + (size_t)dim * nj),
	    ll(l, l + (size_t)dim * ni), rr(r, r + (size_t)dim * nj);
	dqKernel(dqi, dqj, x.data(), y.data(), ll.data(), rr.data(), order, width, ni, nj, dim);
}

} /* extern "C" */
