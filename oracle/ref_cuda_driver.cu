/*
 * Project-written host driver for the reference's plain FP64 GPU path
 * (CUDA/src/*.cu), compiled in place from the read-only reference tree by
 * `make -C oracle refcu` into oracle/_ref/librefcu{2,3}d.so.
 *
 * It stands in for the MATLAB MEX entry point (CUDA/src/LDDMM.cu:13-151) and for the
 * transposes its MATLAB wrapper performs (CUDA/src/LDDMM.m:8-21): inputs arrive in the
 * C++ path's layouts (coordinate fastest; alpha as (t * N + i) * D + d) and are
 * transposed here into the CUDA path's column-major layouts (q[d * N + i],
 * alpha[(t * D + d) * N + i], element tables element-fastest, the vertex -> element
 * table vertex-fastest).  Workspace sizes follow LDDMM.cu:98-102 and are carved by the
 * reference's own assignFcnStructMemory / assignOptStructMemory
 * (CUDA/src/assignStructMemory.cu).
 *
 * The reference's objgrd.cu is compiled with -Dobjgrd=refimpl_objgrd so that the
 * wrapper below counts the evaluations L-BFGS and the line search request.
 *
 * This is the FP64 GPU baseline of the sweeps (cuBLAS dgemm on an N x N kernel
 * matrix per time step, host-synchronising cublasDdot calls): measurement and test
 * infrastructure only, never linked into the product library.
 */
#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include <cublas_v2.h>
#include "struct.h"
#include "constants.h"

long long assignFcnStructMemory(fcndata &, double *);
long long assignOptStructMemory(optdata &, double *);
int LBFGS(double *, double *, double *, optdata &, fcndata &);
void refimpl_objgrd(double *, double *, double *, fcndata &);

static long long g_evals = 0;

/* Sits between the reference optimiser and the reference objective; counts calls. */
void objgrd(double *fcnVal, double *grdStk, double *alpStk, fcndata &fcnObj)
{
	refimpl_objgrd(fcnVal, grdStk, alpStk, fcnObj);
	++g_evals;
}

namespace {

constexpr int kD = DIMNUM;

struct DevProblem {
	fcndata fcn;
	double *work = nullptr;
	double *nde = nullptr, *tgt_cen = nullptr, *tgt_dir = nullptr, *tgt_vol = nullptr;
	int *vtx = nullptr, *ifo = nullptr;
	bool blas = false;
	~DevProblem()
	{
		cudaFree(work);
		cudaFree(nde);
		cudaFree(tgt_cen);
		cudaFree(tgt_dir);
		cudaFree(tgt_vol);
		cudaFree(vtx);
		cudaFree(ifo);
		if (blas) cublasDestroy(fcn.blasHdl);
	}
};

template <class T>
int upload(T **d, const std::vector<T> &h)
{
	if (cudaMalloc((void **)d, sizeof(T) * (h.empty() ? 1 : h.size())) != cudaSuccess) return -1;
	if (h.empty()) return 0;
	return cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice) == cudaSuccess ? 0 : -1;
}

/* Row-major (rows x cols, row fastest-varying second index) -> column-major. */
template <class T>
std::vector<T> to_col_major(const T *a, long long rows, long long cols)
{
	std::vector<T> b((size_t)(rows * cols));
	for (long long r = 0; r < rows; ++r)
		for (long long c = 0; c < cols; ++c) b[(size_t)(c * rows + r)] = a[r * cols + c];
	return b;
}

int setup(DevProblem &P, const double *iniNde, int ndeNum, int timeNum, double timeStp,
          int knlOrder, double knlWidth, const int *elmVtx, int dfmElmNum, const int *elmIfo,
          int elmIfoRows, const double *tgtCen, const double *tgtDir, const double *tgtVol,
          int tgtElmNum, char cenType, double cenWidth, char dirType, double dirWidth,
          double disWgt)
{
	fcndata &F = P.fcn;
	std::memset(&F, 0, sizeof(F));
	F.prm.ndeNum = ndeNum;
	F.prm.knlOrder = knlOrder;
	F.prm.knlWidth = knlWidth;
	F.prm.timeStp = timeStp;
	F.prm.timeNum = timeNum;
	F.dis.disWgt = disWgt;
	F.dis.dfmNdeNum = ndeNum;
	F.dis.dfmElmNum = dfmElmNum;
	F.dis.tgtElmNum = tgtElmNum;
	F.dis.cenKnlType = cenType;
	F.dis.cenKnlWidth = cenWidth;
	F.dis.dirKnlType = dirType;
	F.dis.dirKnlWidth = dirWidth;
	F.varNum = kD * ndeNum * (timeNum - 1);

	const int vpe = kD;  // vertices per element: segments in 2D, triangles in 3D
	if (upload(&P.nde, to_col_major(iniNde, ndeNum, kD))) return -1;
	if (upload(&P.vtx, to_col_major(elmVtx, dfmElmNum, vpe))) return -1;
	if (upload(&P.ifo, to_col_major(elmIfo, ndeNum, elmIfoRows))) return -1;
	if (upload(&P.tgt_cen, to_col_major(tgtCen, tgtElmNum, kD))) return -1;
	if (upload(&P.tgt_dir, to_col_major(tgtDir, tgtElmNum, kD))) return -1;
	if (upload(&P.tgt_vol, std::vector<double>(tgtVol, tgtVol + tgtElmNum))) return -1;
	F.prm.d_iniNdeMat = P.nde;
	F.dis.d_dfmElmVtxMat = P.vtx;
	F.dis.d_dfmElmIfoMat = P.ifo;
	F.dis.d_tgtCenPosMat = P.tgt_cen;
	F.dis.d_tgtUniDirMat = P.tgt_dir;
	F.dis.d_tgtElmVolVec = P.tgt_vol;

	const long long fcnMemCnt = (long long)dfmElmNum + tgtElmNum + SUMBLKDIM
	                          + (long long)dfmElmNum * (kD * 4 + 1)
	                          + (long long)ndeNum * kD * (timeNum + 5)
	                          + (long long)ndeNum * ndeNum;
	if (cudaMalloc((void **)&P.work, sizeof(double) * fcnMemCnt) != cudaSuccess) return -1;
	if (assignFcnStructMemory(F, P.work) != fcnMemCnt) return -2;
	if (cublasCreate(&F.blasHdl) != CUBLAS_STATUS_SUCCESS) return -1;
	P.blas = true;
	return 0;
}

/* C++ alpha layout (t * N + i) * D + d  <->  CUDA layout (t * D + d) * N + i */
std::vector<double> alpha_to_cuda(const double *a, int N, int T)
{
	std::vector<double> b((size_t)kD * N * T);
	for (int t = 0; t < T; ++t)
		for (int i = 0; i < N; ++i)
			for (int d = 0; d < kD; ++d)
				b[((size_t)t * kD + d) * N + i] = a[((size_t)t * N + i) * kD + d];
	return b;
}

void alpha_from_cuda(const std::vector<double> &b, double *a, int N, int T)
{
	for (int t = 0; t < T; ++t)
		for (int i = 0; i < N; ++i)
			for (int d = 0; d < kD; ++d)
				a[((size_t)t * N + i) * kD + d] = b[((size_t)t * kD + d) * N + i];
}

}  // namespace

#define REFCU_ARGS                                                                          \
	const double *iniNde, int ndeNum, int timeNum, double timeStp, int knlOrder,           \
	    double knlWidth, const int *elmVtx, int dfmElmNum, const int *elmIfo,              \
	    int elmIfoRows, const double *tgtCen, const double *tgtDir, const double *tgtVol,  \
	    int tgtElmNum, char cenType, double cenWidth, char dirType, double dirWidth,       \
	    double disWgt
#define REFCU_PASS                                                                          \
	iniNde, ndeNum, timeNum, timeStp, knlOrder, knlWidth, elmVtx, dfmElmNum, elmIfo,       \
	    elmIfoRows, tgtCen, tgtDir, tgtVol, tgtElmNum, cenType, cenWidth, dirType,         \
	    dirWidth, disWgt

extern "C" int refcu_dim(void) { return kD; }

/* One objective + gradient evaluation (CUDA/src/objgrd.cu:13-76); alp / grd in the
 * C++ layout.  Returns 0, or a negative value on a CUDA / workspace failure. */
extern "C" int refcu_objgrd(REFCU_ARGS, const double *alp, double *fcn, double *grd)
{
	DevProblem P;
	int rc = setup(P, REFCU_PASS);
	if (rc) return rc;
	const int T = timeNum - 1;
	double *d_alp = nullptr, *d_grd = nullptr;
	if (upload(&d_alp, alpha_to_cuda(alp, ndeNum, T))) return -1;
	if (cudaMalloc((void **)&d_grd, sizeof(double) * P.fcn.varNum) != cudaSuccess) {
		cudaFree(d_alp);
		return -1;
	}
	refimpl_objgrd(fcn, d_grd, d_alp, P.fcn);
	std::vector<double> g((size_t)P.fcn.varNum);
	const cudaError_t e = cudaMemcpy(g.data(), d_grd, sizeof(double) * g.size(), cudaMemcpyDeviceToHost);
	cudaFree(d_alp);
	cudaFree(d_grd);
	if (e != cudaSuccess) return -1;
	if (grd) alpha_from_cuda(g, grd, ndeNum, T);
	return 0;
}

/* A whole registration: LBFGS (CUDA/src/LBFGS.cu:34-128) from alp_inout, which
 * receives the optimised momenta (C++ layout).  out[0] = milliseconds inside LBFGS
 * (CUDA events), out[1] = milliseconds of the whole call (set-up, host <-> device
 * copies, optimisation), out[2] = objective evaluations, out[3] = final objective.
 * Returns LBFGS's status (0, or 1 when the line search failed), or a negative value on a
 * CUDA / workspace failure. */
extern "C" int refcu_lbfgs(REFCU_ARGS, int itrMax, double tolVal, double wolfe1,
                           double wolfe2, int memNum, int vbsFlg, double *alp_inout,
                           double *out)
{
	const auto w0 = std::chrono::steady_clock::now();
	DevProblem P;
	int rc = setup(P, REFCU_PASS);
	if (rc) return rc;
	const int T = timeNum - 1;
	optdata O;
	std::memset(&O, 0, sizeof(O));
	O.varNum = P.fcn.varNum;
	O.memNum = memNum;
	O.itrMax = itrMax;
	O.tolVal = tolVal;
	O.wolfe1 = wolfe1;
	O.wolfe2 = wolfe2;
	O.vbsFlg = vbsFlg != 0;
	const long long optMemCnt = (long long)O.varNum * (5 + memNum * 2);
	double *d_opt = nullptr, *d_pos = nullptr, *d_grd = nullptr;
	std::vector<double> rec((size_t)memNum);
	O.h_recVec = rec.data();
	if (cudaMalloc((void **)&d_opt, sizeof(double) * optMemCnt) != cudaSuccess) return -1;
	if (assignOptStructMemory(O, d_opt) != optMemCnt) {
		cudaFree(d_opt);
		return -2;
	}
	if (upload(&d_pos, alpha_to_cuda(alp_inout, ndeNum, T)) ||
	    cudaMalloc((void **)&d_grd, sizeof(double) * O.varNum) != cudaSuccess) {
		cudaFree(d_opt);
		cudaFree(d_pos);
		return -1;
	}
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	g_evals = 0;
	double fcn = 0.0;
	cudaEventRecord(e0);
	const int status = LBFGS(&fcn, d_grd, d_pos, O, P.fcn);
	cudaEventRecord(e1);
	cudaEventSynchronize(e1);
	float ms = 0.0f;
	cudaEventElapsedTime(&ms, e0, e1);
	std::vector<double> a((size_t)O.varNum);
	const cudaError_t e = cudaMemcpy(a.data(), d_pos, sizeof(double) * a.size(), cudaMemcpyDeviceToHost);
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(d_opt);
	cudaFree(d_pos);
	cudaFree(d_grd);
	if (e != cudaSuccess) return -1;
	alpha_from_cuda(a, alp_inout, ndeNum, T);
	if (out) {
		out[0] = ms;
		out[1] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
		out[2] = (double)g_evals;
		out[3] = fcn;
	}
	return status;
}
