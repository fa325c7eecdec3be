/*
 * lddmm_b200 -- C ABI of the B200 (sm_100a) LDDMM landmark/surface registration
 * with varifold matching.
 *
 * These entry points replace the routines the reference's C++/MATLAB drivers hand
 * to L-BFGS (dnhsieh/LDDMM, Cpp/src):
 *
 *   lddmm_objgrd      <- void objgrd(double *fcnVal, double *grdStk, double *alpStk,
 *                                    fcndata &)                    Cpp/src/objgrd.cpp:26
 *   lddmm_lbfgs       <- int LBFGS(double *fcnNow, double *grdNow, double *posNow,
 *                                  optdata &, fcndata &)           Cpp/src/LBFGS.cpp:25
 *                        (with lineSearch, Cpp/src/lineSearch.cpp:26, and
 *                         getDirection, Cpp/src/getDirection.cpp:9, on the device)
 *   lddmm_LDDMM       <- MEX LDDMM2D/LDDMM3D(iniNdeMat, iniAlpVec, ..., Verbose)
 *                                                                  Cpp/src/LDDMM.cpp:11-46
 *   lddmm_shoot       <- computeNodePosition.m (trajectory and velocities)
 *                                                                  Cpp/src/computeNodePosition.m:1
 *   lddmm_elm_ifo     <- getElmIfo.m                               Cpp/src/getElmIfo.m:1
 *   lddmm_multiply_kernel <- multiplyKernel (MEX multiplyKernelITF) Cpp/src/multiplyKernel.cpp:22
 *   lddmm_dq_kernel   <- dqKernel                                  Cpp/src/dqKernel.cpp:31
 *   lddmm_compute_kernel, lddmm_multiply_kernel2, lddmm_dq_kernel2
 *                     <- the two-set computeKernel / multiplyKernel / dqKernel
 *                        overloads  Cpp/src/computeKernel.cpp:246, multiplyKernel.cpp:294,
 *                        dqKernel.cpp:307
 *   lddmm_varifold    <- varifoldITF / varifold (gradient overload) Cpp/src/varifoldITF.cpp:7
 *
 * Layout is the reference's C++ one: coordinates fastest, then node, then time
 * step (Cpp/src/objgrd.cpp:47-50); element and adjacency tables are 0-based int32
 * (Cpp/src/LDDMM.m:7-8).  All buffers passed to entry points without the _device
 * suffix are host memory owned by the caller; a context owns all device memory,
 * its CUDA stream and its CUDA graphs.
 *
 * Return codes: 0 success; 1/2/3 line-search failure codes of the reference
 * (not a descent direction / function may be unbounded below / bracketed but the
 * weak Wolfe conditions not satisfied, Cpp/src/lineSearch.cpp:45,101,109); negative
 * values are errors (LDDMM_ERR_*), with a message from lddmm_last_error().
 * No entry point calls exit() or prints unless asked to (verbose).
 *
 * Threading: a context is used by one host thread at a time; distinct contexts are
 * independent.  Process-wide state, all of it guarded or per thread: the error
 * message (per host thread), one stream-ordered device memory pool per device from
 * which contexts take their memory (guarded by a mutex), and the fixed device array of
 * lddmm_multiply_kernel_noalloc with its cached per-device address.
 */
#ifndef LDDMM_B200_H
#define LDDMM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define LDDMM_OK 0
#define LDDMM_LS_NOT_DESCENT 1
#define LDDMM_LS_UNBOUNDED 2
#define LDDMM_LS_BRACKET 3
#define LDDMM_ERR_ARG (-1)
#define LDDMM_ERR_CUDA (-2)
#define LDDMM_ERR_NONFINITE (-3)
#define LDDMM_ERR_TIMEOUT (-4)
#define LDDMM_ERR_NOMEM (-5)
#define LDDMM_ERR_UNSUPPORTED (-6)

typedef struct lddmm_ctx lddmm_ctx;

/* One registration pair: the fields of `parameters` and `discrepancy`
 * (Cpp/src/struct.h:25-56) plus the sizes the MEX reads from its arrays
 * (Cpp/src/LDDMM.cpp:44-52). */
typedef struct lddmm_problem {
	int dim;                  /* DIMNUM: 2 or 3 */
	int nde_num;              /* ndeNum: landmarks N */
	int time_num;             /* timeNum: time points; T = time_num - 1 Euler steps */
	double time_stp;          /* timeStp */
	int knl_order;            /* knlOrder: -1 Gaussian, 0..4 Matern */
	double knl_width;         /* knlWidth */
	const double *ini_nde;    /* iniNdeMat: dim x N */
	double dis_wgt;           /* disWgt */
	int dfm_elm_num;          /* dfmElmNum */
	const int *dfm_elm_vtx;   /* dfmElmVtxMat: dim x E_d, 0-based */
	int dfm_elm_ifo_num;      /* dfmElmIfoNum: rows of dfmElmIfoMat (0: computed) */
	const int *dfm_elm_ifo;   /* dfmElmIfoMat: rows x N, or NULL to compute it */
	int tgt_elm_num;          /* tgtElmNum */
	const double *tgt_cen_pos;/* tgtCenPosMat: dim x E_t */
	const double *tgt_uni_dir;/* tgtUniDirMat: dim x E_t */
	const double *tgt_elm_vol;/* tgtElmVolVec: E_t */
	char cen_knl_type;        /* cenKnlType: 'G' Gaussian, 'C' Cauchy */
	double cen_knl_width;     /* cenKnlWidth */
	char dir_knl_type;        /* dirKnlType: 'B' Binet, 'L' linear, 'O'/'U' Gaussian */
	double dir_knl_width;     /* dirKnlWidth */
} lddmm_problem;

/* Optimiser options: the fields of `optdata` (Cpp/src/struct.h:4-23). */
typedef struct lddmm_opt {
	int itr_max;              /* itrMax (MaxIterations) */
	double tol_val;           /* tolVal (OptimalityTolerance): stop when |g| < tol */
	double wolfe1;            /* Armijo constant */
	double wolfe2;            /* curvature constant */
	int mem_num;              /* memNum (Columns), any size >= 1: the ring holds
	                             min(memNum, itrMax) pairs (identical iterates);
	                             LDDMM_ERR_NOMEM when that ring cannot fit the device */
	int vbs_flg;              /* print the reference's iteration table per pair */
	double rel_obj_tol;       /* additional stop: |f_prev - f| <= rel_obj_tol |f_prev|;
	                             0 disables (the reference has only the |g| test) */
} lddmm_opt;

/* Launch configuration.  Zero fields take defaults / the autotuner's choice. */
typedef struct lddmm_config {
	int cluster_shoot;        /* CTAs per i-tile (thread-block cluster size, 1..8) */
	int cluster_adjoint;
	int cluster_varifold;
	int autotune;             /* 0 (default) or 1: time the candidate launch shapes at
	                             creation (per-step sweeps: 1 or 2 64-row tiles per work
	                             item x cluster split 1/2/4/8; varifold split 1..8;
	                             persistent time loops vs per-step launches) and keep
	                             the fastest, cached per batch shape for the process;
	                             -1: the built-in rule, no timing */
	int use_graph;            /* 1 (default): capture the L-BFGS cycle in a CUDA graph */
	void *stream;             /* cudaStream_t to run on; NULL: the context creates one */
	int device;               /* CUDA device ordinal (default 0) */
	int persistent;           /* time loops as one persistent cooperative launch per
	                             direction: 0 automatic (when one step of the batch does
	                             not fill the GPU; the form chosen by the autotuner),
	                             1 on (split row groups combined through L2), 2 on
	                             (thread-block clusters own whole row groups and combine
	                             them through distributed shared memory), -1 off */
} lddmm_config;

/* Per-pair outcome of lddmm_lbfgs. */
typedef struct lddmm_result {
	double fcn;               /* objective at the returned point */
	double grd_len;           /* |g| there */
	int status;               /* 0, 1, 2, 3 or an LDDMM_ERR_* value */
	int iters;                /* accepted L-BFGS iterations */
	int evals;                /* objective evaluations */
	int pad_;
} lddmm_result;

const char *lddmm_last_error(void);
const char *lddmm_version(void);

/* Context over `num` independent pairs (a batch; num = 1 for one registration).
 * All pairs must share dim, time_num, knl_order, cen_knl_type and dir_knl_type.
 * Replaces the workspace set-up of Cpp/src/LDDMM.cpp:54-80. */
int lddmm_ctx_create(const lddmm_problem *probs, int num, const lddmm_config *cfg,
                     lddmm_ctx **out);
void lddmm_ctx_destroy(lddmm_ctx *ctx);
int lddmm_ctx_num_pairs(const lddmm_ctx *ctx);
/* Variables of pair `pair` (dim * N * (time_num - 1)) and their offset in the
 * concatenated vectors every batched entry point uses. */
long long lddmm_ctx_var_num(const lddmm_ctx *ctx, int pair);
long long lddmm_ctx_var_offset(const lddmm_ctx *ctx, int pair);
long long lddmm_ctx_var_total(const lddmm_ctx *ctx);
/* The cudaStream_t the context runs on. */
void *lddmm_ctx_stream(const lddmm_ctx *ctx);
/* Cluster sizes in use (after autotuning): out[0..2] = shoot, adjoint, varifold. */
int lddmm_ctx_launch_config(const lddmm_ctx *ctx, int *out3);
/* Launch shape in use: out[0..2] cluster sizes (shoot, adjoint, varifold), out[3..4]
 * 64-row tiles per work item of the shooting / adjoint sweeps, out[5] the form of
 * the time loops (0 per-step launches, 1 persistent with L2 combine, 2 persistent
 * cluster form); the persistent plans: out[6] cluster size and out[7] CTAs of the
 * cluster form (0: unavailable), out[8] CTAs of the L2 form, out[9] / out[10] the
 * largest CTA share (j entries of 16 rows) of the cluster / L2 plan.  Writes at most n
 * values; returns the number written. */
int lddmm_ctx_launch_shape(const lddmm_ctx *ctx, int *out, int n);

/* Objective and gradient of every pair at alp (concatenated, host memory);
 * fcn[num], grd like alp.  objgrd.cpp:26 semantics. */
int lddmm_objgrd(lddmm_ctx *ctx, const double *alp, double *fcn, double *grd);
/* Same on device buffers (no host copies, synchronous on the context stream unless
 * `async` is set). */
int lddmm_objgrd_device(lddmm_ctx *ctx, const double *d_alp, double *d_fcn, double *d_grd,
                        int async);

/* objgrd on device buffers (synchronous) that also returns the adjoint costate:
 * d_pst (like alp) receives, for every step t, p_{t+1}, the costate the backward
 * recursion multiplies at step t -- the gradient of step t is dt K(q_t) (alpha_t -
 * p_{t+1}) (objgrd.cpp:67-87), so alpha_t = p_{t+1} at a stationary point.  d_grd may
 * be NULL. */
int lddmm_objgrd_costate(lddmm_ctx *ctx, const double *d_alp, double *d_fcn, double *d_grd,
                         double *d_pst);

/* L-BFGS from alp_inout (host) for every pair; on return alp_inout holds each pair's
 * last accepted point (the reference's posNow) and res[num] the outcome.  Returns 0
 * when every pair ended with status 0, else the first nonzero status. */
int lddmm_lbfgs(lddmm_ctx *ctx, const lddmm_opt *opt, double *alp_inout, lddmm_result *res);
int lddmm_lbfgs_device(lddmm_ctx *ctx, const lddmm_opt *opt, double *d_alp_inout,
                       lddmm_result *res);
/* Per-iteration record of pair `pair` from the last lddmm_lbfgs call: rows of
 * (f, |g|, step length, evaluations in the line search), row 0 the initial point.
 * Returns the number of rows written (at most cap). */
int lddmm_lbfgs_trace(const lddmm_ctx *ctx, int pair, double *rows4, int cap);
/* Gradient at each pair's last accepted point of the last lddmm_lbfgs /
 * lddmm_lbfgs_device call (the reference's grdNow, Cpp/src/LBFGS.cpp:25), in the
 * variable layout, concatenated like alp; host memory of lddmm_ctx_var_total doubles.
 * LDDMM_ERR_ARG before the first L-BFGS call of the context. */
int lddmm_lbfgs_grad(const lddmm_ctx *ctx, double *grd);

/* Trajectory of every pair: nde_stk (dim x N x time_num per pair) and velocities
 * vlc_stk (dim x N x (time_num - 1) per pair), concatenated by pair.  Either output
 * may be NULL. */
int lddmm_shoot(lddmm_ctx *ctx, const double *alp, double *nde_stk, double *vlc_stk);

/* The whole MEX entry point LDDMM2D/LDDMM3D (Cpp/src/LDDMM.cpp:11-98) for one pair:
 * same 22 arguments in the same order, plus the array sizes MATLAB would supply and
 * the output buffer optAlpVec (dim * N * (timeNum - 1)).  dfmElmIfoMat may be NULL.
 * Returns LBFGS's code like the reference (0, or the line-search code). */
int lddmm_LDDMM(int dim, int nde_num, int dfm_elm_num, int dfm_elm_ifo_num, int tgt_elm_num,
                const double *iniNdeMat, const double *iniAlpVec, const int *dfmElmVtxMat,
                const int *dfmElmIfoMat, const double *tgtCenPosMat, const double *tgtElmVolVec,
                const double *tgtUniDirMat, char cenKnlType, double cenKnlWidth,
                char dirKnlType, double dirKnlWidth, double disWgt, int knlOrder,
                double knlWidth, double timeStp, int timeNum, int MaxIterations,
                double OptimalityTolerance, double Wolfe1, double Wolfe2, int Columns,
                int Verbose, double *optAlpVec);

/* getElmIfo (Cpp/src/getElmIfo.m): vertex -> adjacent element table.  elm_vtx is
 * vpe x elm_num (0-based).  With ifo == NULL returns the row count; otherwise fills
 * rows x nde_num and returns the row count.  Negative on bad input. */
int lddmm_elm_ifo(const int *elm_vtx, int vpe, int elm_num, int nde_num, int *ifo);

/* Single kernel sums on the GPU (host buffers; a temporary device workspace):
 * v_i = sum_j K(q_i, q_j) a_j                    (multiplyKernel.cpp:22)
 * dq_i = sum_j (l_i.r_j + l_j.r_i) dK/dq_i       (dqKernel.cpp:31)
 * V, dV/dq of the varifold discrepancy           (varifold3D.cpp:410, varifold2D.cpp:378) */
int lddmm_multiply_kernel(int dim, int n, const double *q, const double *a, int knl_order,
                          double knl_width, double *v);
int lddmm_dq_kernel(int dim, int n, const double *q, const double *l, const double *r,
                    int knl_order, double knl_width, double *dq);
int lddmm_varifold(const lddmm_problem *prob, const double *nde, double *val, double *dq);

/* Two landmark sets (the reference's two-set overloads, reached through the MEX
 * interfaces computeKernelITF / multiplyKernelITF / dqKernelITF with 4 / 5 / 6
 * inputs).  qi: dim x ni, qj: dim x nj, C++ layout; host buffers; any kernel order
 * (-1 Gaussian, 0..4 Matern) in 2D and 3D.
 *
 * Dense kernel matrix, the reference's column-major ni x nj layout
 * knl[j * ni + i] = K(qi_i, qj_j); qj == NULL gives the one-set matrix of qi
 * (nj is then ignored)  <- computeKernel, Cpp/src/computeKernel.cpp:246 and :21.
 * FP32 evaluation stored as FP64 (relative error ~1e-7 of the largest entry). */
int lddmm_compute_kernel(int dim, int ni, const double *qi, int nj, const double *qj,
                         int knl_order, double knl_width, double *knl);
/* v_i = sum_j K(qi_i, qj_j) a_j, a: dim x nj, v: dim x ni
 *                                  <- multiplyKernel, Cpp/src/multiplyKernel.cpp:294 */
int lddmm_multiply_kernel2(int dim, int ni, const double *qi, int nj, const double *qj,
                           const double *a, int knl_order, double knl_width, double *v);
/* l: dim x ni, r: dim x nj;
 * dqi_i = sum_j (l_i.r_j) dK(qi_i, qj_j)/dqi_i, dqj_j = sum_i (l_i.r_j) dK/dqj_j
 *                                  <- dqKernel, Cpp/src/dqKernel.cpp:307 */
int lddmm_dq_kernel2(int dim, int ni, const double *qi, int nj, const double *qj,
                     const double *l, const double *r, int knl_order, double knl_width,
                     double *dqi, double *dqj);

/* Allocation-free v_i = sum_j K(q_i, q_j) a_j.  No counterpart in the reference.
 *
 * For callers that must not have the library call cudaMalloc/cudaFree: a MEX
 * function working on MATLAB gpuArray data (the device memory belongs to MATLAB's
 * allocator, which the library cannot see), a framework whose caching allocator owns
 * the GPU, or a host loop that cannot afford the device-wide synchronisation that
 * cudaFree implies.  d_q, d_a (inputs, dim x n) and d_v (output, dim x n) are device
 * buffers the caller owns; the working set lives in one fixed array of about 2.3 MB
 * compiled into the library, which every GPU that loads the library holds until the
 * process exits.  Nothing is allocated.
 *
 * Limit: 1 <= n <= LDDMM_NOALLOC_MAX_POINTS; larger n returns LDDMM_ERR_ARG.  Every
 * kernel order of lddmm_multiply_kernel is supported (2D and 3D: Gaussian -1, Matern
 * 0..4).  The first call on a device looks up the array's device address (with that
 * device current) and caches it for the life of the process; make that first call
 * before any stream capture, and do not use this entry point after the device or its
 * primary context has been reset (cudaDeviceReset, MATLAB's reset(gpuDevice)): the
 * cached address would then be stale.  Every call shares the array: calls that
 * overlap on the GPU (other streams, other host threads) race and give wrong results;
 * each call clears what must start at zero.  Asynchronous on `stream` (a cudaStream_t,
 * NULL for the default stream). */
#define LDDMM_NOALLOC_MAX_POINTS 32768
int lddmm_multiply_kernel_noalloc(int dim, int n, const double *d_q, const double *d_a,
                                  int knl_order, double knl_width, double *d_v, void *stream);

/* Measurement.  Evaluates the objective `reps` times at the context's current
 * trial point with CUDA events on the context stream around every sweep launch and
 * writes average milliseconds per launch: ms4[0] shooting step, ms4[1] fused adjoint
 * step, ms4[2] varifold sweep, ms4[3] whole evaluation. */
int lddmm_ctx_time_sweeps(lddmm_ctx *ctx, int reps, double *ms4);
/* Counters of the last lddmm_lbfgs call: out[0] L-BFGS cycles launched, out[1]
 * kernels per cycle, out[2] kernel launches in total, out[3] objective evaluations
 * summed over pairs.  Returns the number of values written (at most n). */
int lddmm_ctx_counters(const lddmm_ctx *ctx, long long *out, int n);

/* Device-side timeline of the last L-BFGS cycle (or objective evaluation), from
 * %globaltimer stamps the cooperative kernels write: us6 = entry and exit, in
 * microseconds relative to the forward sweep's entry, of the forward time-loop sweep,
 * the backward time-loop sweep and the fused optimiser update (-1 when not run). */
int lddmm_ctx_timeline(const lddmm_ctx *ctx, double *us6);

/* Health check of the bounded device waits (no counterpart in the reference).  Runs
 * one grid barrier of the kind the persistent sweeps and the L-BFGS cycle use, on two
 * co-resident CTAs.  never_released = 0: the barrier completes and the call returns 0.
 * never_released != 0: nothing can complete it; every CTA gives up after about a
 * second of polling, the kernel ends, and the call returns LDDMM_ERR_TIMEOUT with the
 * device still usable.  *ms (may be NULL) receives the kernel's duration. */
int lddmm_wait_selftest(int device, int never_released, double *ms);

/* FP32 FMA throughput of this GPU (TFLOP/s, FMA = 2 flops) measured by a probe
 * kernel of independent FMA chains over every SM; the roofline denominator of the
 * FP32-bound sweeps.  Returns 0 and writes the figure to *tflops. */
int lddmm_fp32_peak(int device, double *tflops);

/* Throughput of the pipes the all-pairs sweeps use, measured on `device` by probe
 * kernels (best of three launches): out[0] scalar FP32 FMA TFLOP/s (as
 * lddmm_fp32_peak), out[1] packed FP32x2 FMA TFLOP/s, out[2] ex2.approx (MUFU)
 * results per second, in G/s.  The rooflines of the sweeps are read against these. */
int lddmm_pipe_peaks(int device, double *out);

/* Storage order that lddmm_ctx_create gives the elements of a 3D surface (and the
 * target's): cen is n x 3 element centres; perm[k] receives the element stored in
 * slot k.  Returns 1 when the elements are reordered along a Morton curve of their
 * centres (because that makes the varifold sweep's 32-element blocks more compact),
 * 0 when the given order is kept (perm is then the identity).  Host only. */
int lddmm_spatial_order(const double *cen, int n, int *perm);

/* FLOPs per pair interaction the roofline uses (FMA = 2, as executed), for the
 * shooting step, the fused adjoint step and the varifold pair of the given kinds. */
double lddmm_flops_per_pair(int sweep, int dim, int knl_order, char cen_type, char dir_type);

/* ---------------------------------------------------------------------------------
 * Learned warm start.  No counterpart in the reference: the reference's LBFGS starts
 * from the momenta it is given (LDDMM.m passes zeros).  A small per-point network,
 * trained on momenta that the plain method produced, predicts a registration's
 * initial momenta from the source landmarks and the target's varifold; the plain
 * L-BFGS then runs from that start as usual.  Network: per target triangle
 * (centre, unit normal, area * Et / (4 pi)) -> 64 (GELU) -> 64, max-pooled over the
 * triangles to g; per source landmark (q_i, g) -> 256 (GELU) -> 256 (GELU) -> 3T, the
 * momenta of the T steps divided by label_scale.  BF16 operands, FP32 accumulation on
 * the tensor cores (tcgen05), FP32 master weights, Adam.  All buffers are device
 * pointers on the context's stream; calls are synchronous.
 * --------------------------------------------------------------------------------- */
typedef struct lddmm_ws lddmm_ws;

/* Creates a network for one source shape (n_src landmarks, src_nde n_src x 3, C++
 * layout), time_steps T (3T <= 256 outputs per landmark), batches of up to batch_max
 * pairs with up to tri_max target triangles, labels divided by label_scale, initial
 * weights uniform(+-1/sqrt(fan-in)) from `seed`.  stream: cudaStream_t or NULL (own). */
int lddmm_ws_create(int n_src, const double *src_nde, int time_steps, int batch_max,
                    int tri_max, double label_scale, unsigned long long seed, void *stream,
                    lddmm_ws **out);
/* lddmm_ws_create with local target features: every landmark's point input also holds
 * its local_k (0..27) nearest target triangles (squared centre distance in FP32, ties
 * to the lower index, nearest first), 7 values each: the centre offset (c - q) * 10,
 * the unit normal and area * Et / (4 pi).  The point input is then 3 + 64 + 7 local_k
 * values, padded to a multiple of 16; local_k = 0 is lddmm_ws_create.  Every batch
 * then needs at least local_k triangles per pair. */
int lddmm_ws_create_ex(int n_src, const double *src_nde, int time_steps, int batch_max,
                       int tri_max, double label_scale, unsigned long long seed, int local_k,
                       void *stream, lddmm_ws **out);
void lddmm_ws_destroy(lddmm_ws *ws);
const char *lddmm_ws_last_error(void);
/* Number of FP32 parameters: per layer (target 1, target 2, point 1, point 2, point 3)
 * Wt[out][in] then b[out], dimensions padded to multiples of 16 (7 -> 16,
 * 67 + 7 local_k -> its multiple of 16, 3T -> round16(3T)); padded entries are zero. */
long long lddmm_ws_num_params(const lddmm_ws *ws);
/* Copies the flat parameter vector to (set = 0) or from (set != 0) host memory. */
int lddmm_ws_params(lddmm_ws *ws, float *host, int set);
/* Mean squared error of `pairs` pairs and its gradient (host, num_params floats; may be
 * NULL) without updating the weights.  d_tri7: pairs x tri_num x 7 FP32 target
 * features; d_labels: pairs x n_src x 3T FP32 momenta, label[p][i][3t + d] =
 * alpha_p[(t n_src + i) 3 + d]. */
int lddmm_ws_grad(lddmm_ws *ws, const float *d_tri7, int pairs, int tri_num,
                  const float *d_labels, float *grad_host, double *loss);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) of learning rate lr on one batch. */
int lddmm_ws_train_step(lddmm_ws *ws, const float *d_tri7, int pairs, int tri_num,
                        const float *d_labels, double lr, double *loss);
/* A network with local features (local_k > 0): the nearest target triangles of every
 * landmark of a batch, d_nbr = pairs x n_src x local_k int32 indices (device), as the
 * forward pass finds them.  Computed once per training pair, they spare the search in
 * every later step through lddmm_ws_train_step_nbr (same results, bit for bit). */
int lddmm_ws_neighbours(lddmm_ws *ws, const float *d_tri7, int pairs, int tri_num,
                        int *d_nbr);
int lddmm_ws_train_step_nbr(lddmm_ws *ws, const float *d_tri7, int pairs, int tri_num,
                            const float *d_labels, const int *d_nbr, double lr, double *loss);
/* Predicted momenta of `pairs` pairs in the variable layout (pairs x T x n_src x 3,
 * FP64), ready as the initial point of lddmm_lbfgs_device.  The activations stay on
 * the context for lddmm_ws_backward until the weights change. */
int lddmm_ws_predict(lddmm_ws *ws, const float *d_tri7, int pairs, int tri_num,
                     double *d_alpha);
/* Backward pass of the last lddmm_ws_predict's batch for the loss
 *   label_weight * MSE(labels)  +  sum d_dalpha . alpha
 * d_labels as in lddmm_ws_grad (NULL: no MSE term); d_dalpha: the gradient of an outer
 * loss with respect to the predicted momenta, in their variable layout (pairs x T x
 * n_src x 3 FP64, e.g. lddmm_objgrd_device's gradient at the prediction, scaled), or
 * NULL.  lr > 0: one Adam step (the activations are then spent); lr = 0: the gradient
 * only.  grad_host (num_params floats) and loss (the MSE term, 0 without labels) may be
 * NULL.  LDDMM_ERR_ARG without a prediction since the last weight change. */
int lddmm_ws_backward(lddmm_ws *ws, const float *d_labels, double label_weight,
                      const double *d_dalpha, double lr, float *grad_host, double *loss);
/* The network's BF16 tensor-core GEMM on its own: C[m x n] (FP32, leading dimension
 * ldc) = A[m x k] . B[n x k]^T, A and B BF16 row-major with k contiguous; n = 16..256
 * in steps of 16, k a multiple of 16, lda and ldb multiples of 8.  Asynchronous on
 * `stream`. */
int lddmm_ws_gemm_bf16(const void *d_a, long long lda, const void *d_b, long long ldb, int m,
                       int n, int k, float *d_c, long long ldc, void *stream);

#ifdef __cplusplus
}
#endif
#endif
