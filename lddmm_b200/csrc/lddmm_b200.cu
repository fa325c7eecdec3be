// Host runtime of the B200 LDDMM library: batch layout, device memory, kernel
// dispatch, the objective sweep, the device L-BFGS cycle (CUDA graph) and the C ABI.
#include <algorithm>
#include <cmath>
#include <memory>
#include <map>
#include <mutex>
#include <utility>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lddmm_b200.h"
#include "common.cuh"
#include "cross.cuh"
#include "kernels.cuh"
#include "layout.h"
#include "lbfgs.cuh"
#include "ops.cuh"
#include "persist.cuh"
#include "plan.h"
#include "sweep.cuh"

using namespace lddmm;

static_assert(lddmm::kPlanSub == lddmm::kSub, "plan sub-tile");
static_assert(lddmm::kPlanMaxJobParts == lddmm::kMaxJobParts, "plan job parts");

namespace {

thread_local std::string g_err;

void set_err(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}

#define CU(expr)                                                                    \
  do {                                                                              \
    cudaError_t e_ = (expr);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      set_err("%s:%d %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(e_));   \
      return LDDMM_ERR_CUDA;                                                        \
    }                                                                               \
  } while (0)

#define CUE(expr)                 \
  do {                            \
    cudaError_t e_ = (expr);      \
    if (e_ != cudaSuccess) return e_; \
  } while (0)

constexpr int kWarps = 4;  // warps per sweep CTA
// persistent sweeps are chosen automatically up to this many row groups per resident CTA
constexpr int kPersistAutoUnits = 2;
// polls of the wait self-test's barrier before it gives up (about a second)
constexpr unsigned int kSelftestSpin = 1u << 20;

// Device memory of the contexts comes from one stream-ordered pool per device, owned
// by the library: allocation, zeroing and release are ordered on the context's stream,
// and released blocks stay cached for the next context (up to kPoolKeepBytes), so
// creating and destroying a context neither calls cudaMalloc / cudaFree nor waits for
// the device.
constexpr unsigned long long kPoolKeepBytes = 8ull << 30;
constexpr int kMaxDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxDevices] = {};

cudaError_t device_pool(cudaMemPool_t *out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return e;
    unsigned long long keep = kPoolKeepBytes;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) {
      cudaMemPoolDestroy(pool);
      return e;
    }
    g_pool[dev] = pool;
  }
  *out = g_pool[dev];
  return cudaSuccess;
}

// n zero-initialised elements, ordered on stream s (the current device's pool).
template <class T>
cudaError_t dalloc(cudaStream_t s, T **p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  cudaMemPool_t pool = nullptr;
  cudaError_t e = device_pool(&pool);
  if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void **)p, n * sizeof(T), pool, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(*p, 0, n * sizeof(T), s);
  return e;
}

// Scratch buffer released (stream-ordered) when it goes out of scope.
template <class T>
struct DevBuf {
  T *p = nullptr;
  cudaStream_t s = nullptr;
  explicit DevBuf(cudaStream_t st) : s(st) {}
  ~DevBuf() {
    if (p) cudaFreeAsync(p, s);
  }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
};

int pad_to(int n, int k) { return (n + k - 1) / k * k; }

}  // namespace

// ============================================================== the context

struct lddmm_ctx {
  int D = 3, order = -1, T = 0, time_num = 0, P = 0;
  char ct = 'G', dt = 'B';
  bool has_vfd = true;
  float ow2 = 0.0f;
  int device = 0;
  std::vector<PairDesc> hpd;
  int NPtot = 0, EDtot = 0, ETtot = 0, ntile_tot = 0, ngrp_tot = 0, netile_tot = 0,
      nchunk_tot = 0;
  long long nvar = 0;
  int n_pt_items = 0, n_el_items = 0;
  int n_pt_items2 = 0;  // two-tile items of the per-step shooting sweep
  int S_shoot = 1, S_adj = 1, S_vfd = 1;
  int tpw_shoot = 1, tpw_adj = 1;  // 64-row tiles per work item of the per-step sweeps
  // persistent multi-step sweeps (one cooperative launch per direction)
  bool persistent = false;
  int pers_ctas = 0;          // CTAs of the persistent kernels (one share of work each)
  // cluster form of the persistent sweeps (persist.cuh persistent_cluster_kernel):
  // pers_kind 1 runs it, on pers_cl_ctas CTAs in clusters of pers_C; 0 the L2 form
  int pers_kind = 0, pers_C = 0, pers_cl_ctas = 0;
  long long pers_cl_share = 0, pers_l2_share = 0;  // largest CTA share of each plan
  int4 *cl_segs = nullptr;
  int *cl_cta_seg = nullptr, *cl_job_src = nullptr;
  int2 *cl_job = nullptr;
  int n_units = 0;            // (pair, row group) work units
  int n_segs = 0, n_slots = 0;
  int cycle_grid = 0;         // CTAs of the fused L-BFGS cycle kernel (0: per-pass launches)
  int cycle_grid_lm = 0;      // the same for long L-BFGS memories (every co-resident CTA)
  int2 *units = nullptr;
  int4 *segs = nullptr;       // persistent work plan (persist.cuh)
  int *cta_seg = nullptr;
  int2 *unit_parts = nullptr;
  double *seg_part = nullptr;
  unsigned int *unit_cnt = nullptr;
  StepSync *sync = nullptr;

  // device memory
  PairDesc *pd = nullptr;
  int *act = nullptr;
  PairState *st = nullptr;
  float4 *qs = nullptr, *as = nullptr, *us = nullptr, *ls = nullptr;
  double *q64 = nullptr, *p64 = nullptr;
  float4 *dbb = nullptr, *tbb = nullptr;  // 32-element block boxes (varifold culling)
  float4 *ec = nullptr, *en = nullptr, *el = nullptr, *tc = nullptr, *tn = nullptr,
         *tl = nullptr;
  double *e64 = nullptr, *dcdd = nullptr, *tgt64 = nullptr;
  int4 *elm = nullptr;
  int *pt_pair = nullptr, *adj_ptr = nullptr;
  int4 *adj = nullptr;
  double *reg_part = nullptr, *vfd_part = nullptr, *f_dev = nullptr;
  int2 *pt_items = nullptr, *el_items = nullptr;
  int2 *pt_items2 = nullptr;  // (pair, even tile): tiles tile and tile + 1 when present
  int *chunk_pair = nullptr;
  double *X = nullptr, *G = nullptr, *XT = nullptr, *GT = nullptr, *Dv = nullptr;
  double *pst_out = nullptr;  // costate output of the evaluation in progress (or none)
  double *Sh = nullptr, *Yh = nullptr;
  double *SYm = nullptr, *YYm = nullptr, *coef = nullptr;  // compact-form L-BFGS state
  double *RI = nullptr, *LV = nullptr, *SYd = nullptr, *LU = nullptr;  // long memory
  int m_alloc = 0;
  double *part = nullptr;
  double *rec = nullptr;
  int rec_cap = 0;

  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // device-side L-BFGS loop: a graph whose WHILE node repeats the cycle
  cudaGraphExec_t loop_exec = nullptr;
  bool loop_valid = false;
  OptParams loop_opt{};
  int *cyc = nullptr;  // cycles run by the device loop
  long long last_cycles = 0, last_launches = 0, last_evals = 0;
  int last_mem = 0;  // L-BFGS memory (ring slots) of the last lddmm_lbfgs call
  int lbfgs_calls = 0;  // graphs are captured from the second L-BFGS call on
  bool use_graph = true;
  cudaGraphExec_t cycle_exec = nullptr;
  OptParams graph_opt{};
  bool graph_valid = false;

  // dispatch
  cudaError_t (*shoot)(lddmm_ctx &, int t, double *vlc) = nullptr;
  cudaError_t (*adjoint)(lddmm_ctx &, int t, double *g, double *pdot) = nullptr;
  cudaError_t (*shoot_all)(lddmm_ctx &, double *vlc) = nullptr;
  cudaError_t (*adjoint_all)(lddmm_ctx &, double *g) = nullptr;
  int (*pers_blocks)(int which) = nullptr;  // resident CTAs per SM of the persistent kernels
  // co-resident clusters of C CTAs of the cluster-form persistent kernels (min of both)
  int (*pers_clusters)(int C, int grid) = nullptr;
  cudaError_t (*probe_cluster)(lddmm_ctx &) = nullptr;  // a cluster-form launch, no steps
  cudaError_t (*varifold)(lddmm_ctx &) = nullptr;
  int (*vfd_clusters)(int S) = nullptr;  // co-resident clusters of S varifold CTAs
  cudaError_t (*tt)(lddmm_ctx &, int p, double *part, dim3 grid, double cw, double dw) = nullptr;

  ~lddmm_ctx();
};

template <class T>
static void dfree(T *&p, cudaStream_t s) {
  if (p) cudaFreeAsync((void *)p, s);
  p = nullptr;
}

lddmm_ctx::~lddmm_ctx() {
  if (cycle_exec) cudaGraphExecDestroy(cycle_exec);
  if (loop_exec) cudaGraphExecDestroy(loop_exec);
  // stream-ordered releases: blocks return to the pool once the stream's work is done
  dfree(cyc, stream); dfree(pd, stream); dfree(act, stream); dfree(st, stream);
  dfree(qs, stream); dfree(as, stream); dfree(us, stream); dfree(ls, stream);
  dfree(q64, stream); dfree(p64, stream); dfree(ec, stream); dfree(en, stream);
  dfree(el, stream); dfree(tc, stream); dfree(tn, stream); dfree(tl, stream);
  dfree(e64, stream); dfree(dcdd, stream); dfree(tgt64, stream); dfree(elm, stream);
  dfree(pt_pair, stream); dfree(adj_ptr, stream); dfree(adj, stream); dfree(reg_part, stream);
  dfree(vfd_part, stream); dfree(f_dev, stream); dfree(pt_items, stream); dfree(pt_items2, stream);
  dfree(el_items, stream); dfree(chunk_pair, stream); dfree(X, stream); dfree(G, stream);
  dfree(XT, stream); dfree(GT, stream); dfree(Dv, stream);
  dfree(Sh, stream); dfree(Yh, stream); dfree(part, stream);
  dfree(SYm, stream); dfree(YYm, stream); dfree(coef, stream);
  dfree(RI, stream); dfree(LV, stream); dfree(SYd, stream); dfree(LU, stream);
  dfree(rec, stream); dfree(sync, stream); dfree(units, stream); dfree(segs, stream);
  dfree(cta_seg, stream); dfree(unit_parts, stream); dfree(seg_part, stream);
  dfree(unit_cnt, stream);
  dfree(cl_segs, stream); dfree(cl_cta_seg, stream); dfree(cl_job, stream);
  dfree(cl_job_src, stream);
  dfree(dbb, stream); dfree(tbb, stream);
  if (own_stream && stream) cudaStreamDestroy(stream);
}

// ============================================================ kernel launch

// Every kernel of the objective sweep and the L-BFGS cycle goes through launch():
// programmatic stream serialisation (the kernel calls pdl_wait() before touching its
// predecessor's output) and, for the sweeps, the thread-block cluster size.
template <typename... KArgs, typename... Args>
static cudaError_t launch(void (*kern)(KArgs...), unsigned grid, unsigned block, int cluster,
                          cudaStream_t stream, Args &&...args) {
  if (grid == 0) return cudaSuccess;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  int na = 1;
  if (cluster > 0) {
    attr[1].id = cudaLaunchAttributeClusterDimension;
    attr[1].val.clusterDim.x = (unsigned)cluster;
    attr[1].val.clusterDim.y = 1;
    attr[1].val.clusterDim.z = 1;
    na = 2;
  }
  cfg.attrs = attr;
  cfg.numAttrs = na;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

template <class Op>
static cudaError_t launch_sweep(const Op &op, const int2 *items, int n_items, int S,
                                cudaStream_t stream) {
  return launch(sweep_kernel<Op, kWarps>, (unsigned)(n_items * S), kWarps * 32, S, stream, op,
                items, S);
}

template <int D, int ORDER>
static cudaError_t shoot_impl(lddmm_ctx &c, int t, double *vlc) {
  ShootOp<D, ORDER> op;
  op.pd = c.pd;
  op.act = c.act;
  op.qs_t = c.qs + (size_t)t * c.NPtot;
  op.as_t = c.as + (size_t)t * c.NPtot;
  op.q64_t = c.q64 + (size_t)t * c.NPtot * D;
  op.q64_n = c.q64 + (size_t)(t + 1) * c.NPtot * D;
  op.qs_n = c.qs + (size_t)(t + 1) * c.NPtot;
  op.x64 = c.XT;
  op.vlc64 = vlc;
  op.tile_part = c.reg_part + (size_t)t * c.ntile_tot;
  op.t = t;
  // packed FP32x2 form of the same sweep (bitwise the same sums), on one- or two-tile
  // work items (c.tpw_shoot; the default rule and the autotuner pick it).  Two tiles
  // per item serve four rows per lane from each staged column: the Gaussian sweep,
  // held first by the shared-memory reads, gains (163,842 landmarks: 11.13 -> 10.58
  // ms); the Matern kernels, with a square root per pair and fewer CTAs per SM at the
  // larger register count, were faster on single tiles (40,962: 1.02 vs 1.10 ms).
  if (c.tpw_shoot == 2)
    return launch(sweep_packed_kernel<ShootOp<D, ORDER>, kWarps, 2>,
                  (unsigned)(c.n_pt_items2 * c.S_shoot), kWarps * 32, c.S_shoot, c.stream, op,
                  (const int2 *)c.pt_items2, c.S_shoot);
  else
    return launch(sweep_packed_kernel<ShootOp<D, ORDER>, kWarps>,
                  (unsigned)(c.n_pt_items * c.S_shoot), kWarps * 32, c.S_shoot, c.stream, op,
                  (const int2 *)c.pt_items, c.S_shoot);
}

template <int D, int ORDER>
static cudaError_t adjoint_impl(lddmm_ctx &c, int t, double *g, double *pdot) {
  AdjointOp<D, ORDER> op;
  op.pd = c.pd;
  op.act = c.act;
  op.qs_t = c.qs + (size_t)t * c.NPtot;
  op.us_t = c.us + (size_t)(t & 1) * c.NPtot;
  op.ls_t = c.ls + (size_t)(t & 1) * c.NPtot;
  op.as_t = c.as + (size_t)t * c.NPtot;
  op.p64 = c.p64;
  op.x64 = c.XT;
  op.g64 = g;
  op.pst64 = c.pst_out;
  op.us_n = (t > 0) ? c.us + (size_t)((t - 1) & 1) * c.NPtot : nullptr;
  op.ls_n = (t > 0) ? c.ls + (size_t)((t - 1) & 1) * c.NPtot : nullptr;
  op.pdot64 = pdot;
  op.t = t;
  // packed FP32x2 form of the same sweep (bitwise the same sums), one- or two-tile
  // items as in shoot_impl (c.tpw_adj; Gaussian at 163,842 landmarks: 23.3 -> 22.0 ms
  // with two tiles, at 2 CTAs per SM instead of 3)
  if (c.tpw_adj == 2)
    return launch(sweep_packed_kernel<AdjointOp<D, ORDER>, kWarps, 2>,
                  (unsigned)(c.n_pt_items2 * c.S_adj), kWarps * 32, c.S_adj, c.stream, op,
                  (const int2 *)c.pt_items2, c.S_adj);
  else
    return launch(sweep_packed_kernel<AdjointOp<D, ORDER>, kWarps>,
                  (unsigned)(c.n_pt_items * c.S_adj), kWarps * 32, c.S_adj, c.stream, op,
                  (const int2 *)c.pt_items, c.S_adj);
}

// Cooperative launch of a persistent multi-step sweep (all CTAs co-resident; the
// runtime refuses the launch otherwise).
template <class Op>
static cudaError_t launch_persistent(lddmm_ctx &c, const Op &op, int dir, int T = -1) {
  if (T < 0) T = c.T;
  if (c.pers_kind == 1) {
    ClusterSweepPlan cp;
    cp.units = c.units;
    cp.segs = c.cl_segs;
    cp.cta_seg = c.cl_cta_seg;
    cp.job = c.cl_job;
    cp.job_src = c.cl_job_src;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)c.pers_cl_ctas);
    cfg.blockDim = dim3(kPersistWarps * 32);
    cfg.stream = c.stream;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    attr[1].id = cudaLaunchAttributeClusterDimension;
    attr[1].val.clusterDim.x = (unsigned)c.pers_C;
    attr[1].val.clusterDim.y = 1;
    attr[1].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    return cudaLaunchKernelEx(&cfg, persistent_cluster_kernel<Op>, op, cp, T, dir, c.sync);
  }
  SweepPlan plan;
  plan.units = c.units;
  plan.segs = c.segs;
  plan.cta_seg = c.cta_seg;
  plan.unit_parts = c.unit_parts;
  plan.part = c.seg_part;
  plan.cnt = c.unit_cnt;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)c.pers_ctas);
  cfg.blockDim = dim3(kPersistWarps * 32);
  cfg.stream = c.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, persistent_sweep_kernel<Op>, op, plan, T, dir, c.sync);
}

template <int D, int ORDER>
static cudaError_t shoot_all_impl(lddmm_ctx &c, double *vlc) {
  ShootOp<D, ORDER> op;
  op.pd = c.pd;
  op.act = c.act;
  op.x64 = c.XT;
  op.qs0 = c.qs;
  op.as0 = c.as;
  op.q640 = c.q64;
  op.vlc0 = vlc;
  op.reg0 = c.reg_part;
  op.NP = c.NPtot;
  op.ntile = c.ngrp_tot;
  return launch_persistent(c, op, +1);
}

template <int D, int ORDER>
static cudaError_t adjoint_all_impl(lddmm_ctx &c, double *g) {
  AdjointOp<D, ORDER> op;
  op.pd = c.pd;
  op.act = c.act;
  op.p64 = c.p64;
  op.x64 = c.XT;
  op.g64 = g;
  op.pdot64 = nullptr;
  op.pst64 = c.pst_out;
  op.qs0 = c.qs;
  op.as0 = c.as;
  op.us0 = c.us;
  op.ls0 = c.ls;
  op.NP = c.NPtot;
  return launch_persistent(c, op, -1);
}

// Co-resident clusters of C CTAs of both cluster-form persistent kernels.
template <int D, int ORDER>
static int pers_clusters_impl(int C, int grid) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(grid / C * C));
  cfg.blockDim = dim3(kPersistWarps * 32);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int a = 0, b = 0;
  if (cudaOccupancyMaxActiveClusters(&a, persistent_cluster_kernel<ShootOp<D, ORDER>>, &cfg) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveClusters(&b, persistent_cluster_kernel<AdjointOp<D, ORDER>>, &cfg) !=
          cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return std::min(a, b);
}

// One launch of the cluster-form kernel with no steps: whether the runtime accepts a
// cooperative launch of clusters of this size and grid.
template <int D, int ORDER>
static cudaError_t probe_cluster_impl(lddmm_ctx &c) {
  ShootOp<D, ORDER> op;
  op.pd = c.pd;
  op.act = c.act;
  op.x64 = c.XT;
  op.qs0 = c.qs;
  op.as0 = c.as;
  op.q640 = c.q64;
  op.vlc0 = nullptr;
  op.reg0 = c.reg_part;
  op.NP = c.NPtot;
  op.ntile = c.ngrp_tot;
  const int kind = c.pers_kind;
  c.pers_kind = 1;
  const cudaError_t e = launch_persistent(c, op, +1, 0);
  c.pers_kind = kind;
  return e;
}

template <int D, int ORDER>
static int pers_blocks_impl(int which) {
  int n = 0;
  cudaError_t e = (which == 0)
      ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, persistent_sweep_kernel<ShootOp<D, ORDER>>, kPersistWarps * 32, 0)
      : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, persistent_sweep_kernel<AdjointOp<D, ORDER>>, kPersistWarps * 32, 0);
  return e == cudaSuccess ? n : 0;
}

template <int D, char CT, char DT>
static cudaError_t varifold_impl(lddmm_ctx &c) {
  VarifoldOp<D, CT, DT> op;
  op.pd = c.pd;
  op.act = c.act;
  op.ec = c.ec;
  op.en = c.en;
  op.el = c.el;
  op.tc = c.tc;
  op.tn = c.tn;
  op.tl = c.tl;
  op.e64 = c.e64;
  op.dcdd = c.dcdd;
  op.tile_part = c.vfd_part;
  op.ow2 = c.ow2;
  op.dbb = c.dbb;
  op.tbb = c.tbb;
  return launch(sweep_packed_kernel<VarifoldOp<D, CT, DT>, kWarps>,
                (unsigned)(c.n_el_items * c.S_vfd), kWarps * 32, c.S_vfd, c.stream, op,
                (const int2 *)c.el_items, c.S_vfd);
}

template <int D, char CT, char DT>
static cudaError_t tt_impl(lddmm_ctx &c, int p, double *part, dim3 grid, double cw, double dw) {
  const PairDesc &P = c.hpd[p];
  target_self_kernel<D, CT, DT><<<grid, 256, 0, c.stream>>>(c.tgt64 + (size_t)P.tg_off * 8, P.Et,
                                                            cw, dw, part);
  return cudaGetLastError();
}

template <int D, int ORDER>
static void set_def(lddmm_ctx &c) {
  c.shoot = shoot_impl<D, ORDER>;
  c.adjoint = adjoint_impl<D, ORDER>;
  c.shoot_all = shoot_all_impl<D, ORDER>;
  c.adjoint_all = adjoint_all_impl<D, ORDER>;
  c.pers_blocks = pers_blocks_impl<D, ORDER>;
  c.pers_clusters = pers_clusters_impl<D, ORDER>;
  c.probe_cluster = probe_cluster_impl<D, ORDER>;
}

template <int D>
static bool pick_def(int order, lddmm_ctx &c) {
  switch (order) {
    case -1: set_def<D, -1>(c); return true;
    case 0: set_def<D, 0>(c); return true;
    case 1: set_def<D, 1>(c); return true;
    case 2: set_def<D, 2>(c); return true;
    case 3: set_def<D, 3>(c); return true;
    case 4: set_def<D, 4>(c); return true;
  }
  return false;
}

template <int D, char CT, char DT>
static int vfd_clusters_impl(int S) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(S * 148));
  cfg.blockDim = dim3(kWarps * 32);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)S;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  const cudaError_t e =
      cudaOccupancyMaxActiveClusters(&n, sweep_packed_kernel<VarifoldOp<D, CT, DT>, kWarps>, &cfg);
  cudaGetLastError();
  return e == cudaSuccess ? n : 0;
}

template <int D, char CT, char DT>
static void set_vfd(lddmm_ctx &c) {
  c.varifold = varifold_impl<D, CT, DT>;
  c.tt = tt_impl<D, CT, DT>;
  c.vfd_clusters = vfd_clusters_impl<D, CT, DT>;
}

template <int D, char CT>
static bool pick_vfd_dt(char dt, lddmm_ctx &c) {
  switch (dt) {
    case 'B': set_vfd<D, CT, 'B'>(c); return true;
    case 'L': set_vfd<D, CT, 'L'>(c); return true;
    case 'O': set_vfd<D, CT, 'O'>(c); return true;
    case 'U': set_vfd<D, CT, 'U'>(c); return true;
  }
  return false;
}

template <int D>
static bool pick_vfd(char ct, char dt, lddmm_ctx &c) {
  if (ct == 'G') return pick_vfd_dt<D, 'G'>(dt, c);
  if (ct == 'C') return pick_vfd_dt<D, 'C'>(dt, c);
  return false;
}

// Element geometry at the final positions, the varifold sweep, and the gather that
// starts the adjoint (us_n/ls_n: operands of the first backward step, or null).
static cudaError_t launch_geometry(lddmm_ctx &c, const double *q64T) {
  const unsigned nb = (unsigned)((c.EDtot + 127) / 128);
  if (c.D == 3)
    return launch(geometry_kernel<3>, nb, 128, 0, c.stream, c.pd, c.act, c.elm, c.EDtot, q64T,
                  c.ec, c.en, c.el, c.e64, c.dbb);
  return launch(geometry_kernel<2>, nb, 128, 0, c.stream, c.pd, c.act, c.elm, c.EDtot, q64T, c.ec,
                c.en, c.el, c.e64, c.dbb);
}

static cudaError_t launch_gather(lddmm_ctx &c, const double *q64T, float4 *un, float4 *ln,
                                 double *dq_out) {
  const unsigned nb = (unsigned)(((long long)c.NPtot * kGatherLanes + 127) / 128);
  if (c.D == 3)
    return launch(gather_kernel<3>, nb, 128, 0, c.stream, c.pd, c.act, c.pt_pair, c.NPtot,
                  c.adj_ptr, c.adj, c.dcdd, q64T, c.XT, c.p64, un, ln, dq_out, c.T);
  return launch(gather_kernel<2>, nb, 128, 0, c.stream, c.pd, c.act, c.pt_pair, c.NPtot,
                c.adj_ptr, c.adj, c.dcdd, q64T, c.XT, c.p64, un, ln, dq_out, c.T);
}

static cudaError_t launch_objective(lddmm_ctx &c, PairState *st, double *f_out) {
  const int groups = c.persistent ? kGroup : 0;
  return launch(objective_kernel, (unsigned)c.P, 512, 0, c.stream, c.pd, c.act, c.reg_part,
                groups ? c.ngrp_tot : c.ntile_tot, c.vfd_part, c.T, st, f_out, groups);
}

// FP64 alpha (variable layout) -> FP32 point layout used by the sweeps.
__global__ void alpha_to_f32_kernel(const PairDesc *__restrict__ pd, int P, const double *x,
                                    float4 *as, int NPtot, int D, int T) {
  pdl_wait();
  pdl_trigger();
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  // locate the pair (P is small; linear scan)
  int p = 0;
  while (p + 1 < P && v >= pd[p + 1].var_off) ++p;
  const PairDesc &Q = pd[p];
  if (v >= Q.var_off + Q.var_num) return;
  const long long w = v - Q.var_off;
  const long long nd = (long long)Q.N * D;
  const int t = (int)(w / nd);
  const long long rem = w - (long long)t * nd;
  const int i = (int)(rem / D), d = (int)(rem - (long long)i * D);
  if (t >= T) return;
  reinterpret_cast<float *>(as)[((size_t)t * NPtot + Q.pt_off + i) * 4 + d] = (float)x[v];
}

__global__ void set_int_kernel(int *a, int n, int v) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

static cudaError_t launch_set_active(lddmm_ctx &c, int n) {
  return launch(set_int_kernel, (unsigned)((n + 127) / 128), 128, 0, c.stream, c.act, n, 1);
}

// ==================================================================== setup

static int validate(const lddmm_problem &p) {
  if (p.dim != 2 && p.dim != 3) { set_err("dim must be 2 or 3"); return LDDMM_ERR_ARG; }
  if (p.nde_num <= 0 || !p.ini_nde) { set_err("nde_num must be positive"); return LDDMM_ERR_ARG; }
  if (p.time_num < 2) { set_err("time_num must be >= 2"); return LDDMM_ERR_ARG; }
  if (!(p.knl_width > 0)) { set_err("knl_width must be positive"); return LDDMM_ERR_ARG; }
  if (p.knl_order < -1 || p.knl_order > 4) { set_err("knl_order must be -1..4"); return LDDMM_ERR_ARG; }
  if (p.dfm_elm_num < 0 || p.tgt_elm_num < 0) { set_err("negative element count"); return LDDMM_ERR_ARG; }
  if (p.dfm_elm_num > 0 && !p.dfm_elm_vtx) { set_err("dfm_elm_vtx missing"); return LDDMM_ERR_ARG; }
  if (p.tgt_elm_num > 0 && (!p.tgt_cen_pos || !p.tgt_uni_dir || !p.tgt_elm_vol)) {
    set_err("target arrays missing");
    return LDDMM_ERR_ARG;
  }
  if (p.dfm_elm_num > 0 || p.tgt_elm_num > 0) {
    if (p.cen_knl_type != 'G' && p.cen_knl_type != 'C') { set_err("cen_knl_type must be 'G' or 'C'"); return LDDMM_ERR_ARG; }
    if (p.dir_knl_type != 'B' && p.dir_knl_type != 'L' && p.dir_knl_type != 'O' && p.dir_knl_type != 'U') {
      set_err("dir_knl_type must be 'B', 'L', 'O' or 'U'");
      return LDDMM_ERR_ARG;
    }
    if (!(p.cen_knl_width > 0)) { set_err("cen_knl_width must be positive"); return LDDMM_ERR_ARG; }
    if ((p.dir_knl_type == 'O' || p.dir_knl_type == 'U') && !(p.dir_knl_width > 0)) {
      set_err("dir_knl_width must be positive for 'O'/'U'");
      return LDDMM_ERR_ARG;
    }
  }
  for (int e = 0; e < p.dfm_elm_num * p.dim; ++e)
    if (p.dfm_elm_vtx[e] < 0 || p.dfm_elm_vtx[e] >= p.nde_num) {
      set_err("dfm_elm_vtx entry %d out of range", e);
      return LDDMM_ERR_ARG;
    }
  return 0;
}

extern "C" int lddmm_elm_ifo(const int *elm_vtx, int vpe, int elm_num, int nde_num, int *ifo) {
  // getElmIfo.m:1-59 -- per vertex, adjacent elements in increasing element order
  // with (2D) sign -1 for the element's first vertex, +1 otherwise, or (3D) the
  // element's other two vertices (3,2), (1,3), (2,1) for local vertex 1, 2, 3.
  if ((vpe != 2 && vpe != 3) || elm_num < 0 || nde_num <= 0 || (elm_num > 0 && !elm_vtx)) {
    set_err("lddmm_elm_ifo: bad arguments");
    return LDDMM_ERR_ARG;
  }
  std::vector<int> cnt(nde_num, 0);
  for (int e = 0; e < elm_num * vpe; ++e) {
    const int v = elm_vtx[e];
    if (v < 0 || v >= nde_num) {
      set_err("lddmm_elm_ifo: vertex index out of range");
      return LDDMM_ERR_ARG;
    }
    cnt[v]++;
  }
  int mx = 0;
  for (int v = 0; v < nde_num; ++v) mx = std::max(mx, cnt[v]);
  const int rows = 1 + mx * vpe;
  if (!ifo) return rows;
  std::memset(ifo, 0, sizeof(int) * (size_t)rows * nde_num);
  static const int other3[3][2] = {{2, 1}, {0, 2}, {1, 0}};
  for (int e = 0; e < elm_num; ++e)
    for (int k = 0; k < vpe; ++k) {
      const int *ev = elm_vtx + (size_t)e * vpe;
      int *col = ifo + (size_t)ev[k] * rows;
      const int a = col[0]++;
      if (vpe == 2) {
        col[1 + 2 * a] = e;
        col[2 + 2 * a] = (k == 0) ? -1 : 1;
      } else {
        col[1 + 3 * a] = e;
        col[2 + 3 * a] = ev[other3[k][0]];
        col[3 + 3 * a] = ev[other3[k][1]];
      }
    }
  return rows;
}

static int default_cluster(int n_items, int sms = 148) {
  // aim for >= ~8 CTAs per SM, and split in two while there are fewer than 32 tiles
  // per SM: more, shorter CTAs even out the SMs' loads at the end of the sweep
  // (measured with per-step sweeps on 148 SMs: 40,962 landmarks 12 % and 163,842
  // landmarks 3 % faster per evaluation than one CTA per tile; four-way splits were
  // slower)
  int S = 1;
  while (S < 8 && n_items * S < 8 * sms) S *= 2;
  if (S == 1 && n_items < 32 * sms) S = 2;
  return S;
}

// Storage order of a 3D surface's elements for the varifold sweep, whose distance
// culling tests 32-element blocks by their bounding boxes: blocks of nearby elements
// make small boxes.  Returns the elements sorted along a Morton (Z-order) curve of
// their centres (10 bits per axis over the set's bounding cube, stable) when that
// shrinks the summed extent of the 32-element blocks' boxes below 0.8 of the given
// order's; otherwise an empty vector (keep the given order).  Hierarchically
// subdivided meshes are already ordered better than the curve; re-triangulated or
// decimated ones are not.  cen: n x 3 centres.
static std::vector<int> spatial_order(const std::vector<double> &cen, int n) {
  if (n < 64) return {};
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) lo[d] = hi[d] = cen[d];
  for (int e = 0; e < n; ++e)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], cen[(size_t)e * 3 + d]);
      hi[d] = std::max(hi[d], cen[(size_t)e * 3 + d]);
    }
  const double span = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]});
  if (!(span > 0.0) || !std::isfinite(span)) return {};
  std::vector<uint32_t> code(n);
  for (int e = 0; e < n; ++e) {
    uint32_t m[3];
    for (int d = 0; d < 3; ++d) {
      double u = (cen[(size_t)e * 3 + d] - lo[d]) / span * 1023.0;
      if (!(u > 0.0)) u = 0.0;  // also a non-finite centre
      if (u > 1023.0) u = 1023.0;
      m[d] = (uint32_t)u;
    }
    uint32_t c = 0;
    for (int b = 0; b < 10; ++b)
      for (int d = 0; d < 3; ++d) c |= ((m[d] >> b) & 1u) << (3 * b + d);
    code[e] = c;
  }
  std::vector<int> perm(n);
  for (int e = 0; e < n; ++e) perm[e] = e;
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return code[a] < code[b]; });
  auto extent = [&](const std::vector<int> *order) {
    double sum = 0.0;
    for (int b0 = 0; b0 < n; b0 += 32) {
      double l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (int k = b0; k < std::min(b0 + 32, n); ++k) {
        const int e = order ? (*order)[k] : k;
        for (int d = 0; d < 3; ++d) {
          l[d] = std::min(l[d], cen[(size_t)e * 3 + d]);
          h[d] = std::max(h[d], cen[(size_t)e * 3 + d]);
        }
      }
      sum += (h[0] - l[0]) + (h[1] - l[1]) + (h[2] - l[2]);
    }
    return sum;
  };
  if (extent(&perm) < 0.8 * extent(nullptr)) return perm;
  return {};
}

extern "C" int lddmm_spatial_order(const double *cen, int n, int *perm) {
  if (!cen || n < 0 || !perm) {
    set_err("lddmm_spatial_order: bad arguments");
    return LDDMM_ERR_ARG;
  }
  const std::vector<int> p = spatial_order(std::vector<double>(cen, cen + (size_t)n * 3), n);
  for (int e = 0; e < n; ++e) perm[e] = p.empty() ? e : p[e];
  return p.empty() ? 0 : 1;
}

static int device_sms(int dev) {
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      sms <= 0)
    sms = 148;
  return sms;
}

static cudaError_t run_eval(lddmm_ctx &c, double *g_out, double *f_out, double *vlc,
                            bool grad);

static int autotune(lddmm_ctx &c, const lddmm_config &cf);

extern "C" int lddmm_ctx_create(const lddmm_problem *probs, int num, const lddmm_config *cfg,
                                lddmm_ctx **out) {
  if (!out || !probs || num <= 0) {
    set_err("lddmm_ctx_create: bad arguments");
    return LDDMM_ERR_ARG;
  }
  *out = nullptr;
  for (int p = 0; p < num; ++p) {
    const int rc = validate(probs[p]);
    if (rc) return rc;
    const lddmm_problem &a = probs[p], &b = probs[0];
    if (a.dim != b.dim || a.time_num != b.time_num || a.knl_order != b.knl_order ||
        ((a.dfm_elm_num > 0) != (b.dfm_elm_num > 0)) ||
        (a.dfm_elm_num > 0 && (a.cen_knl_type != b.cen_knl_type || a.dir_knl_type != b.dir_knl_type ||
                               a.dir_knl_width != b.dir_knl_width))) {
      set_err("pairs of one batch must share dim, time_num, knl_order and varifold kernel types");
      return LDDMM_ERR_ARG;
    }
  }
  lddmm_config cf = {};
  if (cfg) cf = *cfg;
  std::unique_ptr<lddmm_ctx> cp(new lddmm_ctx());
  lddmm_ctx &c = *cp;
  const lddmm_problem &p0 = probs[0];
  c.D = p0.dim;
  c.order = p0.knl_order;
  c.time_num = p0.time_num;
  c.T = p0.time_num - 1;
  c.P = num;
  c.has_vfd = p0.dfm_elm_num > 0;
  c.ct = c.has_vfd ? p0.cen_knl_type : 'G';
  c.dt = c.has_vfd ? p0.dir_knl_type : 'B';
  c.ow2 = (c.dt == 'O' || c.dt == 'U') ? (float)(2.0 / (p0.dir_knl_width * p0.dir_knl_width)) : 0.0f;
  c.device = cf.device;
  c.use_graph = (cf.use_graph >= 0);
  CU(cudaSetDevice(c.device));

  bool ok = (c.D == 3) ? pick_def<3>(c.order, c) : pick_def<2>(c.order, c);
  if (!ok) {
    set_err("deformation kernel order %d in %dD is not supported by this build", c.order, c.D);
    return LDDMM_ERR_UNSUPPORTED;
  }
  ok = (c.D == 3) ? pick_vfd<3>(c.ct, c.dt, c) : pick_vfd<2>(c.ct, c.dt, c);
  if (!ok) {
    set_err("varifold kernel types not supported");
    return LDDMM_ERR_UNSUPPORTED;
  }

  // ---- layout
  const int D = c.D;
  c.hpd.resize(num);
  long long voff = 0;
  int pt = 0, el = 0, tg = 0, it = 0, et = 0, ch = 0;
  for (int p = 0; p < num; ++p) {
    const lddmm_problem &a = probs[p];
    PairDesc &P = c.hpd[p];
    std::memset(&P, 0, sizeof(P));
    P.N = a.nde_num;
    P.Npad = pad_to(a.nde_num, kTile);
    P.Ed = a.dfm_elm_num;
    P.Edpad = pad_to(a.dfm_elm_num, kTile);
    P.Et = a.tgt_elm_num;
    P.Etpad = pad_to(a.tgt_elm_num, kTile);
    P.pt_off = pt;
    P.el_off = el;
    P.tg_off = tg;
    P.itile_off = it;
    P.grp_off = it * (kTile / kGroup);
    P.etile_off = et;
    P.var_off = voff;
    P.var_num = (long long)D * a.nde_num * c.T;
    P.chunk_off = ch;
    P.nchunk = (int)((P.var_num + kChunk - 1) / kChunk);
    P.dt = a.time_stp;
    P.dis_wgt = a.dis_wgt;
    def_kernel_scales(a.knl_order, a.dim, a.knl_width, &P.kscale, &P.pd_fac);
    if (c.has_vfd) cen_kernel_scales(a.cen_knl_type, a.cen_knl_width, &P.cscale, &P.dc_fac);
    pt += P.Npad;
    el += P.Edpad;
    tg += P.Etpad;
    it += P.Npad / kTile;
    et += P.Edpad / kTile;
    voff += P.var_num;
    ch += P.nchunk;
  }
  c.NPtot = pt;
  c.EDtot = el;
  c.ETtot = tg;
  c.ntile_tot = it;
  c.ngrp_tot = it * (kTile / kGroup);
  c.netile_tot = et;
  c.nvar = voff;
  c.nchunk_tot = ch;

  // work items, largest pairs first (the block scheduler then runs longest first)
  std::vector<int> order(num);
  for (int p = 0; p < num; ++p) order[p] = p;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return c.hpd[a].Npad > c.hpd[b].Npad; });
  std::vector<int2> pti, eli, pti2;
  for (int p : order)
    for (int k = 0; k < c.hpd[p].Npad / kTile; ++k) pti.push_back(make_int2(p, k));
  for (int p : order)
    for (int k = 0; k < c.hpd[p].Npad / kTile; k += 2) pti2.push_back(make_int2(p, k));
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return c.hpd[a].Edpad + c.hpd[a].Etpad > c.hpd[b].Edpad + c.hpd[b].Etpad;
  });
  for (int p : order)
    for (int k = 0; k < c.hpd[p].Edpad / kTile; ++k) eli.push_back(make_int2(p, k));
  c.n_pt_items = (int)pti.size();
  c.n_pt_items2 = (int)pti2.size();
  c.n_el_items = (int)eli.size();
  std::vector<int2> uni;
  for (const int2 &x : pti)
    for (int g = 0; g < kTile / kGroup; ++g)
      uni.push_back(make_int2(x.x, x.y * (kTile / kGroup) + g));
  c.n_units = (int)uni.size();

  // host-side arrays
  std::vector<float4> h_qs(c.NPtot, make_float4(0, 0, 0, 0));
  std::vector<double> h_q64((size_t)c.NPtot * D, 0.0);
  std::vector<int> h_ptpair(c.NPtot, -1);
  std::vector<int4> h_elm(std::max(c.EDtot, 1), make_int4(0, 0, 0, -1));
  std::vector<float4> h_tc(std::max(c.ETtot, 1), make_float4(0, 0, 0, 0)), h_tn(h_tc), h_tl(h_tc);
  std::vector<char> h_treal(std::max(c.ETtot, 1), 0);  // real (not padding) target element
  std::vector<double> h_tgt64((size_t)std::max(c.ETtot, 1) * 8, 0.0);
  std::vector<int> h_adjptr(c.NPtot + 1, 0);
  std::vector<int4> h_adj;
  std::vector<int> h_chunk(c.nchunk_tot);
  for (int p = 0; p < num; ++p) {
    const lddmm_problem &a = probs[p];
    const PairDesc &P = c.hpd[p];
    for (int k = 0; k < P.nchunk; ++k) h_chunk[P.chunk_off + k] = p;
    for (int i = 0; i < P.N; ++i) {
      const int g = P.pt_off + i;
      h_ptpair[g] = p;
      double q[3] = {0, 0, 0};
      for (int d = 0; d < D; ++d) q[d] = a.ini_nde[(size_t)i * D + d];
      for (int d = 0; d < D; ++d) h_q64[(size_t)g * D + d] = q[d];
      h_qs[g] = make_float4((float)(q[0] * P.kscale), (float)(q[1] * P.kscale),
                            (float)(q[2] * P.kscale), 0.0f);
    }
    // element storage order (3D surfaces: a spatial order when it makes the varifold
    // sweep's 32-element blocks more compact; the sums do not depend on the order)
    std::vector<int> dperm, tperm, dslot;
    if (D == 3 && c.has_vfd) {
      std::vector<double> cen((size_t)P.Ed * 3);
      for (int e = 0; e < P.Ed; ++e)
        for (int d = 0; d < 3; ++d) {
          double sum = 0.0;
          for (int k = 0; k < 3; ++k) sum += a.ini_nde[(size_t)a.dfm_elm_vtx[(size_t)e * 3 + k] * 3 + d];
          cen[(size_t)e * 3 + d] = sum / 3.0;
        }
      dperm = spatial_order(cen, P.Ed);
      tperm = spatial_order(std::vector<double>(a.tgt_cen_pos, a.tgt_cen_pos + (size_t)P.Et * 3),
                            P.Et);
    }
    if (!dperm.empty()) {
      dslot.resize(P.Ed);
      for (int s = 0; s < P.Ed; ++s) dslot[dperm[s]] = s;
    }
    for (int s = 0; s < P.Ed; ++s) {
      const int e = dperm.empty() ? s : dperm[s];
      const int *v = a.dfm_elm_vtx + (size_t)e * D;
      h_elm[P.el_off + s] = make_int4(P.pt_off + v[0], P.pt_off + v[1],
                                      D == 3 ? P.pt_off + v[2] : 0, p);
    }
    for (int s = 0; s < P.Et; ++s) {
      const int g = P.tg_off + s;
      const int e = tperm.empty() ? s : tperm[s];
      double cc[3] = {0, 0, 0}, nn[3] = {0, 0, 0};
      for (int d = 0; d < D; ++d) {
        cc[d] = a.tgt_cen_pos[(size_t)e * D + d];
        nn[d] = a.tgt_uni_dir[(size_t)e * D + d];
      }
      const double vol = a.tgt_elm_vol[e];
      float hi[3], lo[3];
      for (int d = 0; d < 3; ++d) {
        const double x = cc[d] * P.cscale;
        hi[d] = (float)x;
        lo[d] = (float)(x - (double)hi[d]);
      }
      h_tc[g] = make_float4(hi[0], hi[1], hi[2], (float)(-vol));
      h_treal[g] = 1;
      h_tl[g] = make_float4(lo[0], lo[1], lo[2], 0.0f);
      h_tn[g] = make_float4((float)nn[0], (float)nn[1], (float)nn[2], 0.0f);
      double *t8 = &h_tgt64[(size_t)g * 8];
      for (int d = 0; d < 3; ++d) {
        t8[d] = cc[d];
        t8[3 + d] = nn[d];
      }
      t8[6] = vol;
    }
    // adjacency (given table, or computed like getElmIfo)
    std::vector<int> ifo;
    int rows = a.dfm_elm_ifo_num;
    const int *tab = a.dfm_elm_ifo;
    if (P.Ed > 0 && (!tab || rows <= 0)) {
      rows = lddmm_elm_ifo(a.dfm_elm_vtx, D, P.Ed, P.N, nullptr);
      if (rows < 0) return rows;
      ifo.resize((size_t)rows * P.N);
      lddmm_elm_ifo(a.dfm_elm_vtx, D, P.Ed, P.N, ifo.data());
      tab = ifo.data();
    }
    for (int i = 0; i < P.N && P.Ed > 0; ++i) {
      const int *col = tab + (size_t)i * rows;
      const int cnt = col[0];
      if (cnt < 0 || 1 + cnt * D > rows) {
        set_err("dfm_elm_ifo column %d inconsistent", i);
        return LDDMM_ERR_ARG;
      }
      for (int k = 0; k < cnt; ++k) {
        const int e = col[1 + D * k];
        if (e < 0 || e >= P.Ed) {
          set_err("dfm_elm_ifo element index out of range");
          return LDDMM_ERR_ARG;
        }
        if (D == 3) {
          const int va = col[2 + 3 * k], vb = col[3 + 3 * k];
          if (va < 0 || va >= P.N || vb < 0 || vb >= P.N) {
            set_err("dfm_elm_ifo vertex index out of range");
            return LDDMM_ERR_ARG;
          }
          h_adj.push_back(make_int4(P.el_off + (dslot.empty() ? e : dslot[e]), P.pt_off + va,
                                    P.pt_off + vb, 0));
        } else {
          h_adj.push_back(make_int4(P.el_off + (dslot.empty() ? e : dslot[e]), col[2 + 2 * k],
                                    0, 0));
        }
      }
      h_adjptr[P.pt_off + i + 1] = (int)h_adj.size();
    }
    // padded vertices carry the running count
    for (int i = P.N; i < P.Npad; ++i) h_adjptr[P.pt_off + i + 1] = (int)h_adj.size();
    if (P.Ed == 0)
      for (int i = 0; i < P.N; ++i) h_adjptr[P.pt_off + i + 1] = (int)h_adj.size();
  }

  // ---- device memory (stream-ordered on the context's stream)
  if (cf.stream) {
    c.stream = (cudaStream_t)cf.stream;
  } else {
    CU(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    c.own_stream = true;
  }
  CU(dalloc(c.stream, &c.pd, num));
  CU(dalloc(c.stream, &c.act, num));
  CU(dalloc(c.stream, &c.st, num));
  CU(dalloc(c.stream, &c.qs, (size_t)(c.T + 1) * c.NPtot));
  CU(dalloc(c.stream, &c.as, (size_t)c.T * c.NPtot));
  CU(dalloc(c.stream, &c.us, (size_t)2 * c.NPtot));
  CU(dalloc(c.stream, &c.ls, (size_t)2 * c.NPtot));
  CU(dalloc(c.stream, &c.q64, (size_t)(c.T + 1) * c.NPtot * D));
  CU(dalloc(c.stream, &c.p64, (size_t)c.NPtot * D));
  CU(dalloc(c.stream, &c.ec, std::max(c.EDtot, 1)));
  CU(dalloc(c.stream, &c.en, std::max(c.EDtot, 1)));
  CU(dalloc(c.stream, &c.el, std::max(c.EDtot, 1)));
  CU(dalloc(c.stream, &c.tc, std::max(c.ETtot, 1)));
  CU(dalloc(c.stream, &c.tn, std::max(c.ETtot, 1)));
  CU(dalloc(c.stream, &c.tl, std::max(c.ETtot, 1)));
  CU(dalloc(c.stream, &c.dbb, (size_t)std::max(c.EDtot / 32, 1) * 2));
  CU(dalloc(c.stream, &c.tbb, (size_t)std::max(c.ETtot / 32, 1) * 2));
  CU(dalloc(c.stream, &c.e64, (size_t)std::max(c.EDtot, 1) * 4));
  CU(dalloc(c.stream, &c.dcdd, (size_t)std::max(c.EDtot, 1) * 2 * D));
  CU(dalloc(c.stream, &c.tgt64, h_tgt64.size()));
  CU(dalloc(c.stream, &c.elm, h_elm.size()));
  CU(dalloc(c.stream, &c.pt_pair, c.NPtot));
  CU(dalloc(c.stream, &c.adj_ptr, c.NPtot + 1));
  CU(dalloc(c.stream, &c.adj, std::max<size_t>(h_adj.size(), 1)));
  CU(dalloc(c.stream, &c.reg_part, (size_t)c.T * c.ngrp_tot));
  CU(dalloc(c.stream, &c.vfd_part, std::max(c.netile_tot, 1)));
  CU(dalloc(c.stream, &c.f_dev, num));
  CU(dalloc(c.stream, &c.pt_items, std::max(c.n_pt_items, 1)));
  CU(dalloc(c.stream, &c.pt_items2, std::max(c.n_pt_items2, 1)));
  CU(dalloc(c.stream, &c.el_items, std::max(c.n_el_items, 1)));
  CU(dalloc(c.stream, &c.chunk_pair, c.nchunk_tot));
  CU(dalloc(c.stream, &c.XT, c.nvar));
  CU(dalloc(c.stream, &c.GT, c.nvar));
  CU(dalloc(c.stream, &c.part, (size_t)c.nchunk_tot * kPartStride));

  CU(cudaMemcpyAsync(c.qs, h_qs.data(), sizeof(float4) * c.NPtot,
                     cudaMemcpyHostToDevice, c.stream));
  CU(cudaMemcpyAsync(c.q64, h_q64.data(), sizeof(double) * h_q64.size(),
                     cudaMemcpyHostToDevice, c.stream));
  CU(cudaMemcpyAsync(c.pt_pair, h_ptpair.data(), sizeof(int) * c.NPtot,
                     cudaMemcpyHostToDevice, c.stream));
  CU(cudaMemcpyAsync(c.elm, h_elm.data(), sizeof(int4) * h_elm.size(),
                     cudaMemcpyHostToDevice, c.stream));
  CU(cudaMemcpyAsync(c.tc, h_tc.data(), sizeof(float4) * h_tc.size(),
                     cudaMemcpyHostToDevice, c.stream));
  CU(cudaMemcpyAsync(c.tn, h_tn.data(), sizeof(float4) * h_tn.size(),
                     cudaMemcpyHostToDevice, c.stream));
  CU(cudaMemcpyAsync(c.tl, h_tl.data(), sizeof(float4) * h_tl.size(),
                     cudaMemcpyHostToDevice, c.stream));
  {
    // bounding boxes of the target blocks' scaled centres (hi + lo), real elements only
    // (a block of padding gets an empty box; an element with a non-finite centre,
    // direction or weight, all of space); constant for the context (the deformed
    // blocks' boxes come with the geometry)
    std::vector<float4> h_tbb((size_t)std::max(c.ETtot / 32, 1) * 2);
    for (int b = 0; b < c.ETtot / 32; ++b) {
      float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (int k = 32 * b; k < 32 * b + 32; ++k) {
        if (!h_treal[k]) continue;
        const float x[3] = {h_tc[k].x + h_tl[k].x, h_tc[k].y + h_tl[k].y, h_tc[k].z + h_tl[k].z};
        const bool fin = std::isfinite(x[0]) && std::isfinite(x[1]) && std::isfinite(x[2]) &&
                         std::isfinite(h_tn[k].x) && std::isfinite(h_tn[k].y) &&
                         std::isfinite(h_tn[k].z) && std::isfinite(h_tc[k].w);
        for (int d = 0; d < 3; ++d) {
          lo[d] = std::min(lo[d], fin ? x[d] : -INFINITY);
          hi[d] = std::max(hi[d], fin ? x[d] : INFINITY);
        }
      }
      h_tbb[2 * b] = make_float4(lo[0], lo[1], lo[2], 0.0f);
      h_tbb[2 * b + 1] = make_float4(hi[0], hi[1], hi[2], 0.0f);
    }
    CU(cudaMemcpyAsync(c.tbb, h_tbb.data(), sizeof(float4) * h_tbb.size(),
                       cudaMemcpyHostToDevice, c.stream));
    CU(cudaStreamSynchronize(c.stream));  // h_tbb goes out of scope
  }
  CU(cudaMemcpyAsync(c.tgt64, h_tgt64.data(), sizeof(double) * h_tgt64.size(),
                     cudaMemcpyHostToDevice, c.stream));
  CU(cudaMemcpyAsync(c.adj_ptr, h_adjptr.data(), sizeof(int) * h_adjptr.size(),
                     cudaMemcpyHostToDevice, c.stream));
  if (!h_adj.empty())
    CU(cudaMemcpyAsync(c.adj, h_adj.data(), sizeof(int4) * h_adj.size(),
                       cudaMemcpyHostToDevice, c.stream));
  if (c.n_pt_items)
    CU(cudaMemcpyAsync(c.pt_items, pti.data(), sizeof(int2) * pti.size(),
                       cudaMemcpyHostToDevice, c.stream));
  if (c.n_pt_items2)
    CU(cudaMemcpyAsync(c.pt_items2, pti2.data(), sizeof(int2) * pti2.size(),
                       cudaMemcpyHostToDevice, c.stream));
  if (c.n_el_items)
    CU(cudaMemcpyAsync(c.el_items, eli.data(), sizeof(int2) * eli.size(),
                       cudaMemcpyHostToDevice, c.stream));
  CU(dalloc(c.stream, &c.units, std::max(c.n_units, 1)));
  CU(cudaMemcpyAsync(c.units, uni.data(), sizeof(int2) * uni.size(),
                     cudaMemcpyHostToDevice, c.stream));
  CU(cudaMemcpyAsync(c.chunk_pair, h_chunk.data(), sizeof(int) * h_chunk.size(),
                     cudaMemcpyHostToDevice, c.stream));


  // ---- target self-term, FP64, once: every pair's blocks launched, one read-back
  if (c.has_vfd) {
    int sms = 0;
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device));
    std::vector<dim3> grid(num);
    std::vector<size_t> off(num + 1, 0);
    for (int p = 0; p < num; ++p) {
      const int Et = c.hpd[p].Et;
      const int nblk = (Et + 255) / 256;
      // j chunks so that a pair alone fills about four CTAs per SM
      const int ny = Et > 0 ? std::max(1, std::min(64, (4 * sms + nblk - 1) / nblk)) : 0;
      grid[p] = dim3((unsigned)nblk, (unsigned)ny);
      off[p + 1] = off[p] + (size_t)nblk * ny;
    }
    double *part = nullptr;
    CU(dalloc(c.stream, &part, std::max<size_t>(off[num], 1)));
    cudaError_t e = cudaSuccess;
    for (int p = 0; p < num && e == cudaSuccess; ++p) {
      if (c.hpd[p].Et == 0) continue;
      const double dw = probs[p].dir_knl_width > 0 ? probs[p].dir_knl_width : 1.0;
      e = c.tt(c, p, part + off[p], grid[p], probs[p].cen_knl_width, dw);
    }
    std::vector<double> hp(std::max<size_t>(off[num], 1));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(hp.data(), part, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost,
                          c.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    cudaFreeAsync(part, c.stream);
    CU(e);
    for (int p = 0; p < num; ++p) {
      double tt = 0.0;
      for (size_t k = off[p]; k < off[p + 1]; ++k) tt += hp[k];
      c.hpd[p].tt = tt;
    }
  }
  CU(cudaMemcpyAsync(c.pd, c.hpd.data(), sizeof(PairDesc) * num, cudaMemcpyHostToDevice, c.stream));

  const int dev_sms = device_sms(c.device);
  c.S_shoot = cf.cluster_shoot > 0 ? cf.cluster_shoot : default_cluster(c.n_pt_items, dev_sms);
  c.S_adj = cf.cluster_adjoint > 0 ? cf.cluster_adjoint : default_cluster(c.n_pt_items, dev_sms);
  c.S_vfd =
      cf.cluster_varifold > 0 ? cf.cluster_varifold : default_cluster(c.n_el_items, dev_sms);
  if (cf.cluster_varifold <= 0 && c.has_vfd && c.vfd_clusters) {
    // the largest split whose clusters all fit in one resident wave (clusters are
    // placed within a GPC, so the count comes from cudaOccupancyMaxActiveClusters; a
    // partial second wave costs more than the extra split gains: measured 125 us at
    // S = 5 vs 134-150 us at 6-8 for 80 element tiles)
    int S = 0;
    for (int s = 8; s >= 1 && !S; --s)
      if (c.n_el_items <= c.vfd_clusters(s)) S = s;
    if (S) c.S_vfd = S;
  }
  // two-tile work items for the Gaussian per-step sweeps, one tile for the Matern ones
  c.tpw_shoot = c.tpw_adj = (c.order == -1) ? 2 : 1;
  for (int *s : {&c.S_shoot, &c.S_adj, &c.S_vfd})
    if (*s < 1 || *s > 8) {
      set_err("cluster sizes must be 1..8");
      return LDDMM_ERR_ARG;
    }
  // persistent multi-step sweeps: used when one step of the batch does not fill the
  // GPU (per-step launches would be latency-bound), sized to the co-resident grid
  {
    int sms = 0;
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device));
    const int b0 = c.pers_blocks(0), b1 = c.pers_blocks(1);
    const int cap = std::min(b0, b1) * sms;
    // automatic: up to a few row groups per resident CTA the persistent sweep wins (a
    // step is a few microseconds and the plan balances any row-group count); bigger
    // batches keep per-step launches, whose 64-row tiles are cheaper per pair
    c.persistent = cap > 0 && (cf.persistent > 0 ||
                               (cf.persistent == 0 && c.n_units <= kPersistAutoUnits * cap));
    CU(dalloc(c.stream, &c.sync, 1));
    CU(cudaMemsetAsync(c.sync, 0, sizeof(StepSync), c.stream));
    if (c.persistent) {
      const HostPlan h = plan_sweeps(uni, c.hpd, cap);
      c.pers_ctas = (int)h.cta_seg.size() - 1;
      c.n_segs = (int)h.segs.size();
      c.n_slots = h.slots;
      CU(dalloc(c.stream, &c.segs, c.n_segs));
      CU(dalloc(c.stream, &c.cta_seg, h.cta_seg.size()));
      CU(dalloc(c.stream, &c.unit_parts, h.unit_parts.size()));
      CU(dalloc(c.stream, &c.seg_part, (size_t)std::max(c.n_slots, 1) * kGroup * kPartNA));
      CU(dalloc(c.stream, &c.unit_cnt, std::max(c.n_units, 1)));
      CU(cudaMemcpyAsync(c.segs, h.segs.data(), sizeof(int4) * h.segs.size(),
                         cudaMemcpyHostToDevice, c.stream));
      CU(cudaMemcpyAsync(c.cta_seg, h.cta_seg.data(), sizeof(int) * h.cta_seg.size(),
                         cudaMemcpyHostToDevice, c.stream));
      CU(cudaMemcpyAsync(c.unit_parts, h.unit_parts.data(), sizeof(int2) * h.unit_parts.size(),
                         cudaMemcpyHostToDevice, c.stream));
      // the cluster form: the cluster size whose plan has the smallest CTA share
      long long l2_share = 0;
      for (int k = 0; k < c.pers_ctas; ++k) {
        long long sh = 0;
        for (int q = h.cta_seg[k]; q < h.cta_seg[k + 1]; ++q) sh += h.segs[q].z - h.segs[q].y;
        l2_share = std::max(l2_share, sh);
      }
      ClusterHostPlan best;
      int bestC = 0, best_ncl = 0;
      for (int C = 1; C <= kMaxJobParts; ++C) {
        const int ncl = std::min(c.pers_clusters(C, cap), cap / C);
        if (ncl < 1) continue;
        ClusterHostPlan ch = plan_cluster_sweeps(uni, c.hpd, C, ncl);
        if (ch.ok && (!bestC || ch.max_share < best.max_share)) {
          best = std::move(ch);
          bestC = C;
          best_ncl = ncl;
        }
      }
      if (bestC) {
        c.pers_C = bestC;
        c.pers_cl_ctas = best_ncl * bestC;
        CU(dalloc(c.stream, &c.cl_segs, std::max<size_t>(best.segs.size(), 1)));
        CU(dalloc(c.stream, &c.cl_cta_seg, best.cta_seg.size()));
        CU(dalloc(c.stream, &c.cl_job, best.job.size()));
        CU(dalloc(c.stream, &c.cl_job_src, best.job_src.size()));
        CU(cudaMemcpyAsync(c.cl_segs, best.segs.data(), sizeof(int4) * best.segs.size(),
                           cudaMemcpyHostToDevice, c.stream));
        CU(cudaMemcpyAsync(c.cl_cta_seg, best.cta_seg.data(), sizeof(int) * best.cta_seg.size(),
                           cudaMemcpyHostToDevice, c.stream));
        CU(cudaMemcpyAsync(c.cl_job, best.job.data(), sizeof(int2) * best.job.size(),
                           cudaMemcpyHostToDevice, c.stream));
        CU(cudaMemcpyAsync(c.cl_job_src, best.job_src.data(), sizeof(int) * best.job_src.size(),
                           cudaMemcpyHostToDevice, c.stream));
        c.pers_cl_share = best.max_share;
        c.pers_l2_share = l2_share;
        // default: the cluster form unless its balance is clearly worse than the L2
        // form's (it saves the L2 round trips of the split row groups every step)
        c.pers_kind = cf.persistent == 2  ? 1
                      : cf.persistent == 1 ? 0
                                           : ((best.max_share * 100 <= l2_share * 115) ? 1 : 0);
        // the runtime must accept a cooperative launch of these clusters
        cudaError_t pe = c.probe_cluster(c);
        if (pe == cudaSuccess) pe = cudaStreamSynchronize(c.stream);
        if (pe != cudaSuccess) {
          cudaGetLastError();  // a refused launch configuration is not sticky
          c.pers_kind = 0;
          c.pers_C = 0;
        }
        CU(cudaMemsetAsync(c.sync, 0, sizeof(StepSync), c.stream));
      }
      if (cf.persistent == 2 && c.pers_C == 0) {
        set_err("the cluster form of the persistent sweeps is not available for this batch "
                "on this device");
        return LDDMM_ERR_UNSUPPORTED;
      }
    }
    int bc = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bc, lbfgs_cycle_kernel, kVecThreads, 0) ==
            cudaSuccess &&
        bc > 0 && cf.persistent >= 0) {
      c.cycle_grid = std::min(bc * sms, c.nchunk_tot);
      c.cycle_grid_lm = bc * sms;
    }
  }
  if (cf.autotune >= 0) {
    const int rc = autotune(c, cf);
    if (rc) return rc;
  }
  *out = cp.release();
  return 0;
}

// Clears the persistent kernels' barrier / error words and the split row groups'
// arrival counts (start of every entry point; after a clean launch they are zero
// already, after a timed-out one they are not).
static cudaError_t reset_sync(lddmm_ctx &c) {
  CUE(cudaMemsetAsync(c.sync, 0, 4 * sizeof(unsigned int), c.stream));
  if (c.unit_cnt)
    CUE(cudaMemsetAsync(c.unit_cnt, 0, sizeof(unsigned int) * c.n_units, c.stream));
  return cudaSuccess;
}

// LDDMM_ERR_TIMEOUT when a persistent sweep's grid barrier gave up (stream must be
// synchronised by the caller).
static int check_sync(lddmm_ctx &c) {
  if (!c.persistent) return 0;
  unsigned int w[2] = {0, 0};
  CU(cudaMemcpyAsync(w, c.sync, sizeof(w), cudaMemcpyDeviceToHost, c.stream));
  CU(cudaStreamSynchronize(c.stream));
  if (w[1]) {
    set_err("a persistent sweep's grid barrier timed out at step %u (the grid was not "
            "co-resident)", w[1] - 1);
    return LDDMM_ERR_TIMEOUT;
  }
  return 0;
}

extern "C" void lddmm_ctx_destroy(lddmm_ctx *ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  delete ctx;
}

extern "C" int lddmm_ctx_num_pairs(const lddmm_ctx *c) { return c ? c->P : 0; }
extern "C" long long lddmm_ctx_var_num(const lddmm_ctx *c, int p) {
  return (c && p >= 0 && p < c->P) ? c->hpd[p].var_num : -1;
}
extern "C" long long lddmm_ctx_var_offset(const lddmm_ctx *c, int p) {
  return (c && p >= 0 && p < c->P) ? c->hpd[p].var_off : -1;
}
extern "C" long long lddmm_ctx_var_total(const lddmm_ctx *c) { return c ? c->nvar : -1; }
extern "C" void *lddmm_ctx_stream(const lddmm_ctx *c) { return c ? (void *)c->stream : nullptr; }
extern "C" int lddmm_ctx_launch_config(const lddmm_ctx *c, int *o) {
  if (!c || !o) return LDDMM_ERR_ARG;
  o[0] = c->S_shoot;
  o[1] = c->S_adj;
  o[2] = c->S_vfd;
  return 0;
}

extern "C" int lddmm_ctx_launch_shape(const lddmm_ctx *c, int *o, int n) {
  if (!c || !o || n < 0) return LDDMM_ERR_ARG;
  const long long v[11] = {c->S_shoot, c->S_adj, c->S_vfd, c->tpw_shoot, c->tpw_adj,
                           c->persistent ? 1 + c->pers_kind : 0, c->pers_C, c->pers_cl_ctas,
                           c->pers_ctas, c->pers_cl_share, c->pers_l2_share};
  const int k = std::min(n, 11);
  for (int i = 0; i < k; ++i) o[i] = (int)v[i];
  return k;
}

// ================================================================ objective

// One objective (and gradient) evaluation of every active pair at XT / as.
static cudaError_t run_eval(lddmm_ctx &c, double *g_out, double *f_out, double *vlc,
                            bool grad) {
  const int D = c.D;
  if (c.persistent) {
    CUE(c.shoot_all(c, vlc));
  } else {
    for (int t = 0; t < c.T; ++t)
      CUE(c.shoot(c, t, vlc ? vlc + (size_t)t * c.NPtot * D : nullptr));
  }
  const double *q64T = c.q64 + (size_t)c.T * c.NPtot * D;
  if (c.has_vfd) {
    CUE(launch_geometry(c, q64T));
    CUE(c.varifold(c));
  }
  if (grad)
    CUE(launch_gather(c, q64T, c.us + (size_t)((c.T - 1) & 1) * c.NPtot,
                      c.ls + (size_t)((c.T - 1) & 1) * c.NPtot, nullptr));
  CUE(launch_objective(c, c.st, f_out));
  if (grad) {
    if (c.persistent)
      CUE(c.adjoint_all(c, g_out));
    else
      for (int t = c.T - 1; t >= 0; --t) CUE(c.adjoint(c, t, g_out, nullptr));
  }
  return cudaSuccess;
}

static cudaError_t load_trial(lddmm_ctx &c, const double *d_alp, bool host) {
  CUE(cudaMemcpyAsync(c.XT, d_alp, sizeof(double) * c.nvar,
                      host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, c.stream));
  const long long n = c.nvar;
  return launch(alpha_to_f32_kernel, (unsigned)((n + 255) / 256), 256, 0, c.stream, c.pd, c.P,
                (const double *)c.XT, c.as, c.NPtot, c.D, c.T);
}

extern "C" int lddmm_objgrd_device(lddmm_ctx *ctx, const double *d_alp, double *d_fcn,
                                   double *d_grd, int async) {
  if (!ctx || !d_alp || !d_fcn) {
    set_err("lddmm_objgrd_device: bad arguments");
    return LDDMM_ERR_ARG;
  }
  lddmm_ctx &c = *ctx;
  CU(cudaSetDevice(c.device));
  CU(reset_sync(c));
  CU(launch_set_active(c, c.P));
  CU(load_trial(c, d_alp, false));
  CU(run_eval(c, d_grd ? d_grd : c.GT, d_fcn, nullptr, true));
  if (!async) {
    CU(cudaStreamSynchronize(c.stream));
    return check_sync(c);
  }
  return 0;
}

extern "C" int lddmm_objgrd_costate(lddmm_ctx *ctx, const double *d_alp, double *d_fcn,
                                    double *d_grd, double *d_pst) {
  if (!ctx || !d_alp || !d_fcn || !d_pst) {
    set_err("lddmm_objgrd_costate: bad arguments");
    return LDDMM_ERR_ARG;
  }
  lddmm_ctx &c = *ctx;
  CU(cudaSetDevice(c.device));
  CU(reset_sync(c));
  CU(launch_set_active(c, c.P));
  CU(load_trial(c, d_alp, false));
  // the adjoint launches of this evaluation take the output pointer by value; every
  // other evaluation (and every captured graph) sees none
  c.pst_out = d_pst;
  const cudaError_t e = run_eval(c, d_grd ? d_grd : c.GT, d_fcn, nullptr, true);
  c.pst_out = nullptr;
  CU(e);
  CU(cudaStreamSynchronize(c.stream));
  return check_sync(c);
}

extern "C" int lddmm_objgrd(lddmm_ctx *ctx, const double *alp, double *fcn, double *grd) {
  if (!ctx || !alp || !fcn) {
    set_err("lddmm_objgrd: bad arguments");
    return LDDMM_ERR_ARG;
  }
  lddmm_ctx &c = *ctx;
  CU(cudaSetDevice(c.device));
  CU(reset_sync(c));
  CU(launch_set_active(c, c.P));
  CU(load_trial(c, alp, true));
  CU(run_eval(c, c.GT, c.f_dev, nullptr, grd != nullptr));
  CU(cudaMemcpyAsync(fcn, c.f_dev, sizeof(double) * c.P, cudaMemcpyDeviceToHost, c.stream));
  if (grd) CU(cudaMemcpyAsync(grd, c.GT, sizeof(double) * c.nvar, cudaMemcpyDeviceToHost, c.stream));
  CU(cudaStreamSynchronize(c.stream));
  return check_sync(c);
}

extern "C" int lddmm_shoot(lddmm_ctx *ctx, const double *alp, double *nde_stk, double *vlc_stk) {
  if (!ctx || !alp) {
    set_err("lddmm_shoot: bad arguments");
    return LDDMM_ERR_ARG;
  }
  lddmm_ctx &c = *ctx;
  const int D = c.D;
  CU(cudaSetDevice(c.device));
  CU(launch_set_active(c, c.P));
  CU(load_trial(c, alp, true));
  double *vlc = nullptr;
  CU(dalloc(c.stream, &vlc, (size_t)c.T * c.NPtot * D));
  cudaError_t e = reset_sync(c);
  if (e == cudaSuccess && c.persistent) e = c.shoot_all(c, vlc);
  for (int t = 0; t < c.T && e == cudaSuccess && !c.persistent; ++t)
    e = c.shoot(c, t, vlc + (size_t)t * c.NPtot * D);
  std::vector<double> hq((size_t)(c.T + 1) * c.NPtot * D), hv((size_t)c.T * c.NPtot * D);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hq.data(), c.q64, sizeof(double) * hq.size(), cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hv.data(), vlc, sizeof(double) * hv.size(), cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  cudaFreeAsync(vlc, c.stream);
  CU(e);
  {
    const int rc = check_sync(c);
    if (rc) return rc;
  }
  // un-pad: per pair, time-major blocks of N x D
  size_t on = 0, ov = 0;
  for (int p = 0; p < c.P; ++p) {
    const PairDesc &P = c.hpd[p];
    for (int t = 0; t <= c.T; ++t)
      for (int i = 0; i < P.N; ++i)
        for (int d = 0; d < D; ++d) {
          const size_t src = ((size_t)t * c.NPtot + P.pt_off + i) * D + d;
          if (nde_stk) nde_stk[on] = hq[src];
          ++on;
          if (t < c.T) {
            if (vlc_stk) vlc_stk[ov] = hv[src];
            ++ov;
          }
        }
  }
  return 0;
}

// ==================================================================== L-BFGS

// Device bytes of the memory-dependent L-BFGS buffers for memory m (s / y ring, Y^T Y,
// coefficients, dot partials, and for m > kMaxMem the long-memory state).
static size_t lbfgs_mem_bytes(const lddmm_ctx &c, long long m) {
  const long long P = c.P, mc = std::max<long long>(m, kMaxMem);
  long long d = 2 * m * c.nvar + P * m * m + P * (1 + 2 * mc) +
                (long long)c.nchunk_tot * std::max<long long>(kPartStride, 4 * m);
  if (m > kMaxMem) d += P * m * m + P * m * 7;
  return (size_t)d * sizeof(double);
}

static cudaError_t ensure_lbfgs_buffers(lddmm_ctx &c, int m, int rec_cap) {
  if (!c.X) {
    CUE(dalloc(c.stream, &c.X, c.nvar));
    CUE(dalloc(c.stream, &c.G, c.nvar));
    CUE(dalloc(c.stream, &c.Dv, c.nvar));
    CUE(dalloc(c.stream, &c.SYm, (size_t)c.P * kMaxMem * kMaxMem));  // m <= kMaxMem only
  }
  if (c.m_alloc < m) {
    dfree(c.Sh, c.stream); dfree(c.Yh, c.stream); dfree(c.YYm, c.stream);
    dfree(c.coef, c.stream); dfree(c.part, c.stream);
    dfree(c.RI, c.stream); dfree(c.LV, c.stream); dfree(c.SYd, c.stream); dfree(c.LU, c.stream);
    const size_t mm = (size_t)m, mc = (size_t)std::max(m, kMaxMem);
    CUE(dalloc(c.stream, &c.Sh, mm * c.nvar));
    CUE(dalloc(c.stream, &c.Yh, mm * c.nvar));
    CUE(dalloc(c.stream, &c.YYm, (size_t)c.P * mm * mm));
    CUE(dalloc(c.stream, &c.coef, (size_t)c.P * (1 + 2 * mc)));
    CUE(dalloc(c.stream, &c.part, (size_t)c.nchunk_tot * std::max<size_t>(kPartStride, 4 * mm)));
    if (m > kMaxMem) {
      CUE(dalloc(c.stream, &c.RI, (size_t)c.P * mm * mm));
      CUE(dalloc(c.stream, &c.LV, (size_t)c.P * mm * 4));
      CUE(dalloc(c.stream, &c.SYd, (size_t)c.P * mm));
      CUE(dalloc(c.stream, &c.LU, (size_t)c.P * mm * 2));
    }
    c.m_alloc = m;
    c.graph_valid = false;
    c.loop_valid = false;
  }
  if (c.rec_cap < rec_cap) {
    dfree(c.rec, c.stream);
    CUE(dalloc(c.stream, &c.rec, (size_t)c.P * rec_cap * 4));
    c.rec_cap = rec_cap;
    c.graph_valid = false;
  }
  return cudaSuccess;
}

// One cycle: objective sweep of the trial points, then the optimiser update.  With a
// conditional handle the cycle also drives the device-side loop (cycle_control).
static cudaError_t launch_cycle(lddmm_ctx &c, const OptParams &o,
                                cudaGraphConditionalHandle h = 0, int max_cycles = 0) {
  CUE(run_eval(c, c.GT, nullptr, nullptr, true));
  VecArgs A;
  A.pd = c.pd;
  A.st = c.st;
  A.chunk_pair = c.chunk_pair;
  A.X = c.X; A.G = c.G; A.XT = c.XT; A.GT = c.GT; A.Dv = c.Dv;
  A.S = c.Sh; A.Y = c.Yh;
  A.part = c.part;
  A.SY = c.SYm; A.YY = c.YYm; A.coef = c.coef;
  A.nvar = c.nvar;
  A.as = c.as;
  A.NPtot = c.NPtot;
  A.D = c.D;
  A.m = o.mem_num;
  A.lm = o.mem_num > kMaxMem ? 1 : 0;
  A.pstride = A.lm ? 4 * o.mem_num : kPartStride;
  A.cstride = A.lm ? 1 + 2 * o.mem_num : kCoefStride;
  A.RI = c.RI; A.LV = c.LV; A.SYd = c.SYd; A.LU = c.LU;
  const unsigned nb = (unsigned)c.nchunk_tot;
  const int pb = (c.P + 127) / 128;
  if (c.cycle_grid > 0) {
    // the whole optimiser update in one cooperative launch (long memories: on every
    // co-resident CTA, their phases have up to chunks x 8 units)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(A.lm ? c.cycle_grid_lm : c.cycle_grid));
    cfg.blockDim = dim3(kVecThreads);
    cfg.stream = c.stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, lbfgs_cycle_kernel, A, o, c.rec, c.act,
                              c.P, c.nchunk_tot, c.sync, h, max_cycles > 0 ? c.cyc : nullptr,
                              max_cycles);
  }
  auto pass = [&](int mode) -> cudaError_t {
    return launch(vec_pass_kernel, nb, kVecThreads, 0, c.stream, A, mode);
  };
  CUE(pass(kPost));
  CUE(launch(decide_kernel, (unsigned)pb, 128, 0, c.stream, (const PairDesc *)c.pd, c.st, c.P,
             (const double *)c.part, A.pstride, o, c.rec));
  if (A.lm) {
    const long long nslot = (long long)c.P * A.m;
    const long long ngrp = (A.m + kLmGroup - 1) / kLmGroup;
    const long long grid[7] = {c.nchunk_tot, c.nchunk_tot * ngrp, (nslot + 255) / 256,
                               (nslot + 7) / 8, (nslot + 7) / 8, (nslot + 255) / 256,
                               (long long)c.nchunk_tot * kLmSub};
    for (int ph = kLmUpdate; ph <= kLmFin; ++ph)
      CUE(launch(lm_phase_kernel, (unsigned)grid[ph], kVecThreads, 0, c.stream, A, ph, c.P,
                 c.nchunk_tot));
  } else {
    CUE(pass(kAccept));
    CUE(launch(solve_kernel, (unsigned)c.P, kVecThreads, 0, c.stream, A));
    CUE(pass(kFin));
  }
  CUE(launch(ls_init_kernel, (unsigned)pb, 128, 0, c.stream, (const PairDesc *)c.pd, c.st, c.P,
             (const double *)c.part, A.pstride, A.lm ? kLmSub : 1, c.act));
  if (max_cycles > 0)
    CUE(launch(cycle_control_kernel, 1, 256, 0, c.stream, h, (const int *)c.act, c.P, c.cyc,
               max_cycles, (const StepSync *)c.sync));
  return cudaSuccess;
}

static long long kernels_per_cycle(const lddmm_ctx &c, int m) {
  // objective: T shooting + [geometry + varifold] + gather + objective + T adjoint
  // (2 launches when the time loops are persistent); optimiser: POST, DECIDE, ACCEPT,
  // SOLVE, FIN, LSINIT, or POST, DECIDE, the 7 long-memory phases, LSINIT (1 launch
  // when fused)
  const long long sweeps = c.persistent ? 2 : 2LL * c.T;
  const long long opt = c.cycle_grid > 0 ? 1 : (m > kMaxMem ? 10 : 6);
  return sweeps + 2 + (c.has_vfd ? 2 : 0) + opt;
}

static bool same_opt(const OptParams &a, const OptParams &b) {
  return std::memcmp(&a, &b, sizeof(OptParams)) == 0;
}

static int build_graph(lddmm_ctx &c, const OptParams &o) {
  if (c.graph_valid && same_opt(c.graph_opt, o)) return 0;
  if (c.cycle_exec) {
    cudaGraphExecDestroy(c.cycle_exec);
    c.cycle_exec = nullptr;
  }
  cudaGraph_t g = nullptr;
  CU(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = launch_cycle(c, o);
  cudaError_t e2 = cudaStreamEndCapture(c.stream, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    CU(e != cudaSuccess ? e : e2);
  }
  e = cudaGraphInstantiate(&c.cycle_exec, g, 0);
  cudaGraphDestroy(g);
  CU(e);
  c.graph_opt = o;
  c.graph_valid = true;
  return 0;
}

// The whole L-BFGS loop as one graph: a WHILE conditional node whose body is one
// cycle; the cycle's last kernel sets the condition (some pair active and fewer than
// max_cycles cycles run).  Returns false (and leaves no partial state) when the
// runtime cannot build it; the caller then drives the cycles from the host.
static bool build_loop_graph(lddmm_ctx &c, const OptParams &o, int max_cycles) {
  if (c.loop_valid && same_opt(c.loop_opt, o)) return true;
  if (c.loop_exec) {
    cudaGraphExecDestroy(c.loop_exec);
    c.loop_exec = nullptr;
  }
  c.loop_valid = false;
  if (!c.cyc && dalloc(c.stream, &c.cyc, 1) != cudaSuccess) return false;
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) return false;
  bool ok = false;
  cudaGraphConditionalHandle h = 0;
  cudaGraphNode_t node;
  cudaGraphNodeParams np = {};
  if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess) {
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    if (cudaGraphAddNode(&node, g, nullptr, 0, &np) == cudaSuccess) {
      cudaGraph_t body = np.conditional.phGraph_out[0];
      if (cudaStreamBeginCaptureToGraph(c.stream, body, nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const cudaError_t e = launch_cycle(c, o, h, max_cycles);
        cudaGraph_t captured = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(c.stream, &captured);
        ok = (e == cudaSuccess && e2 == cudaSuccess);
      }
    }
  }
  if (ok) ok = cudaGraphInstantiate(&c.loop_exec, g, 0) == cudaSuccess;
  cudaGraphDestroy(g);
  cudaGetLastError();  // clear a refused capture or instantiation
  if (!ok) {
    if (c.loop_exec) cudaGraphExecDestroy(c.loop_exec);
    c.loop_exec = nullptr;
    return false;
  }
  c.loop_opt = o;
  c.loop_valid = true;
  return true;
}

static void print_table(const lddmm_ctx &c, int p, const std::vector<double> &rec, int rows) {
  // the reference's verbose table (Cpp/src/LBFGS.cpp:54-61, 107-108)
  if (c.P > 1) printf("pair %d\n", p);
  printf("%5s   %13s  %13s  %13s  %9s\n", "iter", "f", "|grad f|", "step length", "fcn eval");
  char sep[65] = {0};
  std::memset(sep, '-', 62);
  printf("%s\n", sep);
  for (int k = 0; k < rows; ++k) {
    const double *r = &rec[((size_t)p * c.rec_cap + k) * 4];
    if (k == 0)
      printf("%5d:  %13.6e  %13.6e\n", 0, r[0], r[1]);
    else
      printf("%5d:  %13.6e  %13.6e  %13.6e  %9d\n", k, r[0], r[1], r[2], (int)r[3]);
  }
  fflush(stdout);
}

static int lbfgs_run(lddmm_ctx &c, const lddmm_opt *opt, const double *alp, bool host,
                     double *alp_out, lddmm_result *res) {
  if (!opt || opt->mem_num < 1 || opt->itr_max < 0 || !(opt->tol_val >= 0)) {
    set_err("lddmm_lbfgs: bad options (mem_num >= 1, itr_max >= 0, tol_val >= 0)");
    return LDDMM_ERR_ARG;
  }
  OptParams o;
  std::memset(&o, 0, sizeof(o));
  o.itr_max = opt->itr_max;
  // The ring never holds more pairs than there are accepted iterations, and a ring
  // that never wraps behaves the same whatever its size (LBFGS.cpp:96-99: slot newIdx
  // advances once per iteration, getDirection uses min(itr - 1, memNum) pairs), so
  // min(memNum, itrMax) slots give the reference's iterates exactly for any memNum.
  o.mem_num = std::min(opt->mem_num, std::max(opt->itr_max, 1));
  if (o.mem_num > c.m_alloc) {
    size_t fr = 0, tot = 0;
    CU(cudaSetDevice(c.device));
    CU(cudaMemGetInfo(&fr, &tot));
    const size_t need = lbfgs_mem_bytes(c, o.mem_num);
    if (need > fr + lbfgs_mem_bytes(c, c.m_alloc)) {
      set_err("lddmm_lbfgs: an L-BFGS memory of %d pairs needs %.2f GB of device memory, "
              "%.2f GB are free", o.mem_num, need / 1e9, fr / 1e9);
      return LDDMM_ERR_NOMEM;
    }
  }
  o.tol = opt->tol_val;
  o.wolfe1 = opt->wolfe1;
  o.wolfe2 = opt->wolfe2;
  o.rel_obj_tol = opt->rel_obj_tol;
  o.rec_cap = std::min(opt->itr_max + 1, 100001);
  CU(cudaSetDevice(c.device));
  CU(ensure_lbfgs_buffers(c, o.mem_num, o.rec_cap));
  CU(reset_sync(c));
  // initial state: every pair evaluates its starting point
  std::vector<PairState> hs(c.P);
  for (auto &s : hs) {
    std::memset(&s, 0, sizeof(s));
    s.phase = kPhaseInit;
    s.active = 1;
    s.newIdx = -1;
  }
  CU(cudaMemcpyAsync(c.st, hs.data(), sizeof(PairState) * c.P, cudaMemcpyHostToDevice, c.stream));
  CU(launch_set_active(c, c.P));
  CU(load_trial(c, alp, host));
  CU(cudaMemcpyAsync(c.X, c.XT, sizeof(double) * c.nvar, cudaMemcpyDeviceToDevice, c.stream));
  // safety bound on cycles: every iteration takes at most bisMax + epdMax + 2
  // evaluations (>= 62); the per-pair state machine ends well before this.
  const long long max_cycles = (long long)o.itr_max * 200 + 8;
  std::vector<int> hact(c.P);
  long long cycles = 0;
  const int check_every = 8;
  bool timed_out = false;
  // Capturing and instantiating the loop graph costs far more than one registration's
  // launches, so a context's first L-BFGS call drives the cycles from the host with
  // direct launches; later calls run the whole loop as one device-side graph.
  const bool graphs = c.use_graph && c.lbfgs_calls++ > 0;
  if (graphs && max_cycles < (1LL << 30) && build_loop_graph(c, o, (int)max_cycles)) {
    // the whole loop on the device: one launch, one synchronisation
    CU(cudaMemsetAsync(c.cyc, 0, sizeof(int), c.stream));
    CU(cudaGraphLaunch(c.loop_exec, c.stream));
    int ncyc = 0;
    CU(cudaMemcpyAsync(hact.data(), c.act, sizeof(int) * c.P, cudaMemcpyDeviceToHost, c.stream));
    CU(cudaMemcpyAsync(&ncyc, c.cyc, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CU(cudaStreamSynchronize(c.stream));
    {
      const int rc = check_sync(c);
      if (rc) return rc;
    }
    cycles = ncyc;
    for (int a : hact) timed_out |= (a != 0);
  }
  const bool host_loop = !graphs || !c.loop_valid;
  if (host_loop && graphs) {
    const int rc = build_graph(c, o);
    if (rc) return rc;
  }
  while (host_loop) {
    for (int k = 0; k < check_every; ++k) {
      if (graphs)
        CU(cudaGraphLaunch(c.cycle_exec, c.stream));
      else
        CU(launch_cycle(c, o));
    }
    cycles += check_every;
    CU(cudaMemcpyAsync(hact.data(), c.act, sizeof(int) * c.P, cudaMemcpyDeviceToHost, c.stream));
    CU(cudaStreamSynchronize(c.stream));
    {
      const int rc = check_sync(c);
      if (rc) return rc;
    }
    bool any = false;
    for (int a : hact) any |= (a != 0);
    if (!any) break;
    if (cycles >= max_cycles) {
      timed_out = true;
      break;
    }
  }
  c.last_cycles = cycles;
  c.last_launches = cycles * kernels_per_cycle(c, o.mem_num) + 2;
  c.last_mem = o.mem_num;
  CU(cudaMemcpyAsync(hs.data(), c.st, sizeof(PairState) * c.P, cudaMemcpyDeviceToHost, c.stream));
  CU(cudaMemcpyAsync(alp_out, c.X, sizeof(double) * c.nvar,
                     host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, c.stream));
  CU(cudaStreamSynchronize(c.stream));
  int ret = 0;
  c.last_evals = 0;
  for (int p = 0; p < c.P; ++p) c.last_evals += hs[p].evals;
  for (int p = 0; p < c.P; ++p) {
    const PairState &s = hs[p];
    int status = s.status;
    if (timed_out && (s.phase == kPhaseInit || s.phase == kPhaseLS)) status = LDDMM_ERR_TIMEOUT;
    if (res) {
      res[p].fcn = s.f;
      res[p].grd_len = s.glen;
      res[p].status = status;
      res[p].iters = s.iters;
      res[p].evals = s.evals;
      res[p].pad_ = 0;
    }
    if (status != 0 && ret == 0) ret = status;
  }
  if (opt->vbs_flg) {
    std::vector<double> rec((size_t)c.P * c.rec_cap * 4);
    CU(cudaMemcpyAsync(rec.data(), c.rec, sizeof(double) * rec.size(), cudaMemcpyDeviceToHost,
                       c.stream));
    CU(cudaStreamSynchronize(c.stream));
    for (int p = 0; p < c.P; ++p)
      print_table(c, p, rec, std::min(hs[p].iters + 1, c.rec_cap));
  }
  return ret;
}

extern "C" int lddmm_lbfgs(lddmm_ctx *ctx, const lddmm_opt *opt, double *alp_inout,
                           lddmm_result *res) {
  if (!ctx || !alp_inout) {
    set_err("lddmm_lbfgs: bad arguments");
    return LDDMM_ERR_ARG;
  }
  return lbfgs_run(*ctx, opt, alp_inout, true, alp_inout, res);
}

extern "C" int lddmm_lbfgs_device(lddmm_ctx *ctx, const lddmm_opt *opt, double *d_alp_inout,
                                  lddmm_result *res) {
  if (!ctx || !d_alp_inout) {
    set_err("lddmm_lbfgs_device: bad arguments");
    return LDDMM_ERR_ARG;
  }
  return lbfgs_run(*ctx, opt, d_alp_inout, false, d_alp_inout, res);
}

extern "C" int lddmm_lbfgs_trace(const lddmm_ctx *ctx, int pair, double *rows4, int cap) {
  if (!ctx || pair < 0 || pair >= ctx->P || !rows4 || !ctx->rec) return LDDMM_ERR_ARG;
  PairState s;
  if (cudaMemcpyAsync(&s, ctx->st + pair, sizeof(s), cudaMemcpyDeviceToHost, ctx->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    return LDDMM_ERR_CUDA;
  const int n = std::min({s.iters + 1, ctx->rec_cap, cap});
  if (cudaMemcpyAsync(rows4, ctx->rec + (size_t)pair * ctx->rec_cap * 4, sizeof(double) * 4 * n,
                      cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
      cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    return LDDMM_ERR_CUDA;
  return n;
}

extern "C" int lddmm_lbfgs_grad(const lddmm_ctx *ctx, double *grd) {
  if (!ctx || !grd || !ctx->G) {
    set_err("lddmm_lbfgs_grad: bad arguments or no L-BFGS call yet");
    return LDDMM_ERR_ARG;
  }
  if (cudaMemcpyAsync(grd, ctx->G, sizeof(double) * ctx->nvar, cudaMemcpyDeviceToHost,
                      ctx->stream) != cudaSuccess ||
      cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
    set_err("lddmm_lbfgs_grad: %s", cudaGetErrorString(cudaGetLastError()));
    return LDDMM_ERR_CUDA;
  }
  return 0;
}

extern "C" int lddmm_ctx_timeline(const lddmm_ctx *ctx, double *us6) {
  if (!ctx || !us6 || !ctx->sync) return LDDMM_ERR_ARG;
  StepSync h;
  if (cudaMemcpyAsync(&h, ctx->sync, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
    set_err("lddmm_ctx_timeline: %s", cudaGetErrorString(cudaGetLastError()));
    return LDDMM_ERR_CUDA;
  }
  const double t0 = (double)h.stamp[0][0];
  for (int k = 0; k < 3; ++k) {
    us6[2 * k] = h.stamp[k][0] ? ((double)h.stamp[k][0] - t0) * 1e-3 : -1.0;
    us6[2 * k + 1] = h.stamp[k][1] ? ((double)h.stamp[k][1] - t0) * 1e-3 : -1.0;
  }
  return 0;
}

extern "C" int lddmm_ctx_counters(const lddmm_ctx *ctx, long long *out, int n) {
  if (!ctx || !out || n < 0) return LDDMM_ERR_ARG;
  const long long v[4] = {ctx->last_cycles, ctx->last_cycles ? ctx->last_launches / ctx->last_cycles : 0,
                          ctx->last_launches, ctx->last_evals};
  const int k = std::min(n, 4);
  for (int i = 0; i < k; ++i) out[i] = v[i];
  if (k >= 2 && ctx->last_cycles) out[1] = kernels_per_cycle(*ctx, ctx->last_mem);
  return k;
}

extern "C" int lddmm_ctx_time_sweeps(lddmm_ctx *ctx, int reps, double *ms4) {
  if (!ctx || reps <= 0 || !ms4) return LDDMM_ERR_ARG;
  lddmm_ctx &c = *ctx;
  CU(cudaSetDevice(c.device));
  CU(launch_set_active(c, c.P));
  const int nev = 2 * c.T + 1;
  std::vector<cudaEvent_t> ev(2 * nev + 2);
  for (auto &e : ev) CU(cudaEventCreate(&e));
  double acc[4] = {0, 0, 0, 0};
  int cnt[3] = {0, 0, 0};
  const int D = c.D;
  cudaError_t err = cudaSuccess;
  CU(reset_sync(c));
  for (int r = 0; r < reps && err == cudaSuccess; ++r) {
    cudaEventRecord(ev[2 * nev], c.stream);
    if (c.persistent) {
      cudaEventRecord(ev[0], c.stream);
      err = c.shoot_all(c, nullptr);
      cudaEventRecord(ev[1], c.stream);
    } else {
      for (int t = 0; t < c.T; ++t) {
        cudaEventRecord(ev[2 * t], c.stream);
        if (err == cudaSuccess) err = c.shoot(c, t, nullptr);
        cudaEventRecord(ev[2 * t + 1], c.stream);
      }
    }
    const double *q64T = c.q64 + (size_t)c.T * c.NPtot * D;
    if (c.has_vfd) {
      if (err == cudaSuccess) err = launch_geometry(c, q64T);
      cudaEventRecord(ev[4 * c.T], c.stream);
      if (err == cudaSuccess) err = c.varifold(c);
      cudaEventRecord(ev[4 * c.T + 1], c.stream);
    }
    if (err == cudaSuccess)
      err = launch_gather(c, q64T, c.us + (size_t)((c.T - 1) & 1) * c.NPtot,
                          c.ls + (size_t)((c.T - 1) & 1) * c.NPtot, nullptr);
    if (err == cudaSuccess) err = launch_objective(c, nullptr, c.f_dev);
    if (c.persistent) {
      cudaEventRecord(ev[2 * c.T], c.stream);
      if (err == cudaSuccess) err = c.adjoint_all(c, c.GT);
      cudaEventRecord(ev[2 * c.T + 1], c.stream);
    } else {
      for (int t = c.T - 1; t >= 0 && err == cudaSuccess; --t) {
        cudaEventRecord(ev[2 * c.T + 2 * t], c.stream);
        err = c.adjoint(c, t, c.GT, nullptr);
        cudaEventRecord(ev[2 * c.T + 2 * t + 1], c.stream);
      }
    }
    cudaEventRecord(ev[2 * nev + 1], c.stream);
    if (err == cudaSuccess) err = cudaEventSynchronize(ev[2 * nev + 1]);
    if (err != cudaSuccess) break;
    float ms = 0.0f;
    if (c.persistent) {
      // one launch covers all T steps: report the per-step share
      cudaEventElapsedTime(&ms, ev[0], ev[1]);
      acc[0] += ms / c.T;
      cnt[0]++;
      cudaEventElapsedTime(&ms, ev[2 * c.T], ev[2 * c.T + 1]);
      acc[1] += ms / c.T;
      cnt[1]++;
    } else {
      for (int t = 0; t < c.T; ++t) {
        cudaEventElapsedTime(&ms, ev[2 * t], ev[2 * t + 1]);
        acc[0] += ms;
        cnt[0]++;
        cudaEventElapsedTime(&ms, ev[2 * c.T + 2 * t], ev[2 * c.T + 2 * t + 1]);
        acc[1] += ms;
        cnt[1]++;
      }
    }
    if (c.has_vfd) {
      cudaEventElapsedTime(&ms, ev[4 * c.T], ev[4 * c.T + 1]);
      acc[2] += ms;
      cnt[2]++;
    }
    cudaEventElapsedTime(&ms, ev[2 * nev], ev[2 * nev + 1]);
    acc[3] += ms;
  }
  for (auto &e : ev) cudaEventDestroy(e);
  CU(err);
  ms4[0] = cnt[0] ? acc[0] / cnt[0] : 0.0;
  ms4[1] = cnt[1] ? acc[1] / cnt[1] : 0.0;
  ms4[2] = cnt[2] ? acc[2] / cnt[2] : 0.0;
  ms4[3] = acc[3] / reps;
  return 0;
}

// =============================================================== autotuner

// Choices of the autotuner, cached per launch signature for the life of the process
// (a later context of the same shapes starts with them, without timing anything).
struct TuneChoice {
  int S_shoot, S_adj, S_vfd, tpw_shoot, tpw_adj, persistent, pers_kind;
};
static std::mutex g_tune_mu;
static std::map<std::string, TuneChoice> g_tune_cache;

static std::string tune_key(const lddmm_ctx &c, const lddmm_config &cf) {
  std::string k;
  auto add = [&](long long v) { k += std::to_string(v) + ","; };
  add(c.device); add(c.D); add(c.order); add(c.ct); add(c.dt); add(c.T); add(c.has_vfd);
  add(c.persistent); add(cf.cluster_shoot); add(cf.cluster_adjoint); add(cf.cluster_varifold);
  add(cf.persistent);
  for (const PairDesc &d : c.hpd) {
    add(d.Npad); add(d.Edpad); add(d.Etpad);
  }
  return k;
}

// Median milliseconds of `reps` timed runs of f (after one untimed run).
template <class F>
static cudaError_t time_median(lddmm_ctx &c, cudaEvent_t e0, cudaEvent_t e1, int reps, F &&f,
                               float *ms_out) {
  std::vector<float> ms;
  for (int r = 0; r <= reps; ++r) {
    CUE(cudaEventRecord(e0, c.stream));
    CUE(f());
    CUE(cudaEventRecord(e1, c.stream));
    CUE(cudaEventSynchronize(e1));
    float t = 0.0f;
    CUE(cudaEventElapsedTime(&t, e0, e1));
    if (r > 0) ms.push_back(t);
  }
  std::sort(ms.begin(), ms.end());
  *ms_out = ms[ms.size() / 2];
  return cudaSuccess;
}

static int autotune(lddmm_ctx &c, const lddmm_config &cf) {
  // The launch shape of each sweep, chosen by timing the candidates on this batch
  // (zero momenta; the cost does not depend on the values): per-step shooting and
  // adjoint sweeps over one or two 64-row tiles per work item and a cluster split S of
  // 1, 2, 4 or 8 CTAs per item; the varifold sweep over S = 1..8; and, for a batch on
  // the persistent time-loop sweeps, those against T per-step launches of the tuned
  // shape.  Sizes given in the configuration are kept.  Every candidate gives the same
  // sums up to the order in which a cluster's partial sums are added (two-tile items
  // are bitwise one-tile items), so the choice affects time only.
  const std::string key = tune_key(c, cf);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      const TuneChoice &t = it->second;
      c.S_shoot = t.S_shoot; c.S_adj = t.S_adj; c.S_vfd = t.S_vfd;
      c.tpw_shoot = t.tpw_shoot; c.tpw_adj = t.tpw_adj; c.persistent = t.persistent != 0;
      c.pers_kind = t.pers_kind;
      return 0;
    }
  }
  CU(launch_set_active(c, c.P));
  if (c.has_vfd) CU(launch_geometry(c, c.q64));  // element boxes of the initial surface
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  const int reps = 3;
  cudaError_t err = cudaSuccess;
  auto tune_step = [&](int which, int *S, int *tpw, bool fixS) {
    float best = 1e30f;
    int bS = *S, bT = *tpw;
    for (int T2 = 1; T2 <= 2 && err == cudaSuccess; ++T2)
      for (int Sc : {1, 2, 4, 8}) {
        if (fixS && Sc != bS) continue;
        *S = Sc;
        *tpw = T2;
        float ms = 0.0f;
        err = time_median(c, e0, e1, reps, [&]() {
          return which == 0 ? c.shoot(c, 0, nullptr) : c.adjoint(c, 0, c.GT, nullptr);
        }, &ms);
        if (err != cudaSuccess) break;
        if (ms < best) {
          best = ms;
          bS = Sc;
          bT = T2;
        }
      }
    *S = bS;
    *tpw = bT;
  };
  tune_step(0, &c.S_shoot, &c.tpw_shoot, cf.cluster_shoot > 0);
  tune_step(1, &c.S_adj, &c.tpw_adj, cf.cluster_adjoint > 0);
  if (err == cudaSuccess && c.has_vfd && cf.cluster_varifold <= 0) {
    float best = 1e30f;
    int bS = c.S_vfd;
    for (int Sc = 1; Sc <= 8 && err == cudaSuccess; ++Sc) {
      c.S_vfd = Sc;
      float ms = 0.0f;
      err = time_median(c, e0, e1, reps, [&]() { return c.varifold(c); }, &ms);
      if (err == cudaSuccess && ms < best) {
        best = ms;
        bS = Sc;
      }
    }
    c.S_vfd = bS;
  }
  if (err == cudaSuccess && c.persistent) {
    // whole time loops: the persistent forms (L2 combine; cluster combine when the
    // runtime accepted it) against T per-step launches of the tuned shape
    auto time_loops = [&](float *ms) {
      return time_median(c, e0, e1, reps, [&]() {
        cudaError_t e = c.shoot_all(c, nullptr);
        return e == cudaSuccess ? c.adjoint_all(c, c.GT) : e;
      }, ms);
    };
    err = reset_sync(c);
    float mk[2] = {1e30f, 1e30f};
    const int k0 = cf.persistent == 2 ? 1 : 0;
    const int k1 = (cf.persistent == 1 || !c.pers_C) ? 0 : 1;
    for (int kind = k0; kind <= k1 && err == cudaSuccess; ++kind) {
      c.pers_kind = kind;
      err = time_loops(&mk[kind]);
    }
    if (err == cudaSuccess) {
      const int rc = check_sync(c);  // the persistent trials' bounded waits
      if (rc) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return rc;
      }
    }
    c.pers_kind = (mk[1] < mk[0]) ? 1 : 0;
    if (err == cudaSuccess && cf.persistent == 0) {
      float ms = 0.0f;
      err = time_median(c, e0, e1, reps, [&]() {
        cudaError_t e = cudaSuccess;
        for (int t = 0; t < c.T && e == cudaSuccess; ++t) e = c.shoot(c, t, nullptr);
        for (int t = c.T - 1; t >= 0 && e == cudaSuccess; --t) e = c.adjoint(c, t, c.GT, nullptr);
        return e;
      }, &ms);
      if (err == cudaSuccess && ms < std::min(mk[0], mk[1])) c.persistent = false;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CU(err);
  // the trial sweeps wrote the step-1 positions and adjoint state; reset them
  CU(cudaMemsetAsync(c.p64, 0, sizeof(double) * c.NPtot * c.D, c.stream));
  CU(cudaStreamSynchronize(c.stream));
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = TuneChoice{c.S_shoot, c.S_adj, c.S_vfd, c.tpw_shoot, c.tpw_adj,
                                 c.persistent ? 1 : 0, c.pers_kind};
  return 0;
}

// ===================================================== single-call helpers

static lddmm_problem point_problem(int dim, int n, const double *q, int order, double width) {
  lddmm_problem p;
  std::memset(&p, 0, sizeof(p));
  p.dim = dim;
  p.nde_num = n;
  p.time_num = 2;
  p.time_stp = 1.0;
  p.knl_order = order;
  p.knl_width = width;
  p.ini_nde = q;
  p.dis_wgt = 1.0;
  p.cen_knl_type = 'G';
  p.cen_knl_width = 1.0;
  p.dir_knl_type = 'B';
  return p;
}

extern "C" int lddmm_multiply_kernel(int dim, int n, const double *q, const double *a,
                                     int order, double width, double *v) {
  if (!q || !a || !v) {
    set_err("lddmm_multiply_kernel: bad arguments");
    return LDDMM_ERR_ARG;
  }
  lddmm_problem p = point_problem(dim, n, q, order, width);
  lddmm_ctx *ctx = nullptr;
  lddmm_config cfg = {};
  cfg.use_graph = -1;
  int rc = lddmm_ctx_create(&p, 1, &cfg, &ctx);
  if (rc) return rc;
  std::unique_ptr<lddmm_ctx, void (*)(lddmm_ctx *)> guard(ctx, lddmm_ctx_destroy);
  std::vector<double> vs((size_t)2 * n * dim), qs;
  rc = lddmm_shoot(ctx, a, nullptr, vs.data());
  if (rc) return rc;
  std::memcpy(v, vs.data(), sizeof(double) * n * dim);
  return 0;
}

extern "C" int lddmm_dq_kernel(int dim, int n, const double *q, const double *l, const double *r,
                               int order, double width, double *dq) {
  if (!q || !l || !r || !dq) {
    set_err("lddmm_dq_kernel: bad arguments");
    return LDDMM_ERR_ARG;
  }
  lddmm_problem p = point_problem(dim, n, q, order, width);
  lddmm_ctx *ctx = nullptr;
  lddmm_config cfg = {};
  cfg.use_graph = -1;
  int rc = lddmm_ctx_create(&p, 1, &cfg, &ctx);
  if (rc) return rc;
  std::unique_ptr<lddmm_ctx, void (*)(lddmm_ctx *)> guard(ctx, lddmm_ctx_destroy);
  lddmm_ctx &c = *ctx;
  const PairDesc &P = c.hpd[0];
  std::vector<float4> hl(c.NPtot, make_float4(0, 0, 0, 0)), hr(hl);
  for (int i = 0; i < n; ++i) {
    float a[3] = {0, 0, 0}, b[3] = {0, 0, 0};
    for (int d = 0; d < dim; ++d) {
      a[d] = (float)l[(size_t)i * dim + d];
      b[d] = (float)r[(size_t)i * dim + d];
    }
    hl[P.pt_off + i] = make_float4(a[0], a[1], a[2], 0.0f);
    hr[P.pt_off + i] = make_float4(b[0], b[1], b[2], 0.0f);
  }
  double *pd = nullptr;
  CU(dalloc(c.stream, &pd, (size_t)c.NPtot * dim));
  DevBuf<double> pguard(c.stream);
  pguard.p = pd;
  CU(cudaMemsetAsync(c.us, 0, sizeof(float4) * c.NPtot, c.stream));
  CU(cudaMemcpyAsync(c.ls, hl.data(), sizeof(float4) * c.NPtot, cudaMemcpyHostToDevice, c.stream));
  CU(cudaMemcpyAsync(c.as, hr.data(), sizeof(float4) * c.NPtot, cudaMemcpyHostToDevice, c.stream));
  CU(launch_set_active(c, 1));
  CU(c.adjoint(c, 0, nullptr, pd));
  std::vector<double> h((size_t)c.NPtot * dim);
  CU(cudaMemcpyAsync(h.data(), pd, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c.stream));
  CU(cudaStreamSynchronize(c.stream));
  std::memcpy(dq, h.data() + (size_t)P.pt_off * dim, sizeof(double) * n * dim);
  return 0;
}

// ============================================================ two point sets

namespace {

// One call's device work on its own stream, with every buffer from the device's
// stream-ordered pool; the destructor releases them and the stream.
struct OneShot {
  cudaStream_t st = nullptr;
  std::vector<void *> bufs;
  ~OneShot() {
    for (void *p : bufs) cudaFreeAsync(p, st);
    if (st) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
  }
  cudaError_t init() { return cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking); }
  template <class T>
  cudaError_t alloc(T **p, size_t n) {
    const cudaError_t e = dalloc(st, p, std::max<size_t>(n, 1));
    if (e == cudaSuccess) bufs.push_back((void *)*p);
    return e;
  }
  // n points (dim coordinates each, times `scale`) as FP32 float4, zero-padded to npad
  cudaError_t put_points(float4 **d, const double *x, int n, int npad, int dim, double scale) {
    std::vector<float4> h((size_t)npad, make_float4(0, 0, 0, 0));
    for (int i = 0; i < n; ++i) {
      float c[3] = {0, 0, 0};
      for (int k = 0; k < dim; ++k) c[k] = (float)(x[(size_t)i * dim + k] * scale);
      h[i] = make_float4(c[0], c[1], c[2], 0.0f);
    }
    cudaError_t e = alloc(d, (size_t)npad);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(*d, h.data(), sizeof(float4) * npad, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // h goes out of scope
    return e;
  }
  cudaError_t put_items(int2 **d, int ntiles) {
    std::vector<int2> h((size_t)ntiles);
    for (int k = 0; k < ntiles; ++k) h[k] = make_int2(0, k);
    cudaError_t e = alloc(d, (size_t)ntiles);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(*d, h.data(), sizeof(int2) * ntiles, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
  }
};

int check_sets(const char *fn, int dim, int ni, int nj, int order, double width) {
  if (dim != 2 && dim != 3) {
    set_err("%s: dim must be 2 or 3", fn);
    return LDDMM_ERR_ARG;
  }
  if (ni < 1 || nj < 1 || !(width > 0)) {
    set_err("%s: empty point set or non-positive kernel width", fn);
    return LDDMM_ERR_ARG;
  }
  if (order < -1 || order > 4) {
    set_err("%s: kernel order %d not supported (Gaussian -1, Matern 0..4)", fn, order);
    return LDDMM_ERR_UNSUPPORTED;
  }
  return 0;
}

// Calls f.template run<D, ORDER>() for the runtime (dim, order).
template <class F>
cudaError_t with_kernel(int dim, int order, F &f) {
#define LDDMM_ORDERS(D)                                  \
  switch (order) {                                       \
    case -1: return f.template run<D, -1>();             \
    case 0: return f.template run<D, 0>();               \
    case 1: return f.template run<D, 1>();               \
    case 2: return f.template run<D, 2>();               \
    case 3: return f.template run<D, 3>();               \
    case 4: return f.template run<D, 4>();               \
  }
  if (dim == 2) {
    LDDMM_ORDERS(2)
  } else {
    LDDMM_ORDERS(3)
  }
#undef LDDMM_ORDERS
  return cudaErrorInvalidValue;
}

// One cross sum: rows = set a (na points), columns = set b (nb_pad padded points).
struct CrossRun {
  cudaStream_t st;
  int mode;
  const float4 *qa, *xa, *qb, *yb;
  int na, na_pad, nb_pad;
  double fac;
  double *out;
  const int2 *items;
  int sms = 148;  // the current device's SM count (set by the caller)
  template <int D, int ORDER>
  cudaError_t run() {
    const int ntiles = na_pad / kTile;
    if (mode == kCrossMul) {
      CrossOp<D, ORDER, kCrossMul> op;
      op.qa = qa; op.xa = xa; op.qb = qb; op.yb = yb;
      op.na = na; op.nb_pad = nb_pad; op.fac = fac; op.out = out;
      return launch_sweep(op, items, ntiles, default_cluster(ntiles, sms), st);
    }
    CrossOp<D, ORDER, kCrossDq> op;
    op.qa = qa; op.xa = xa; op.qb = qb; op.yb = yb;
    op.na = na; op.nb_pad = nb_pad; op.fac = fac; op.out = out;
    return launch_sweep(op, items, ntiles, default_cluster(ntiles, sms), st);
  }
};

struct MatrixRun {
  cudaStream_t st;
  const float4 *qi, *qj;
  int ni, nj;
  double *K;
  template <int D, int ORDER>
  cudaError_t run() {
    int dev = 0;
    cudaGetDevice(&dev);
    const int sms = device_sms(dev);
    const long long total = (long long)ni * nj;
    const long long want = (total + 255) / 256;
    const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(want, 8LL * sms));
    return launch(kernel_matrix_kernel<D, ORDER>, grid, 256, 0, st, qi, ni, qj, nj, K);
  }
};

}  // namespace

extern "C" int lddmm_compute_kernel(int dim, int ni, const double *qi, int nj, const double *qj,
                                    int order, double width, double *knl) {
  if (!qj) nj = ni;
  int rc = check_sets("lddmm_compute_kernel", dim, ni, nj, order, width);
  if (rc) return rc;
  if (!qi || !knl) {
    set_err("lddmm_compute_kernel: bad arguments");
    return LDDMM_ERR_ARG;
  }
  if (!qj) qj = qi;
  float kscale = 1.0f;
  double pd_fac = 0.0;
  def_kernel_scales(order, dim, width, &kscale, &pd_fac);
  OneShot w;
  CU(w.init());
  float4 *dqi = nullptr, *dqj = nullptr;
  double *dk = nullptr;
  CU(w.put_points(&dqi, qi, ni, ni, dim, kscale));
  CU(w.put_points(&dqj, qj, nj, nj, dim, kscale));
  const size_t total = (size_t)ni * (size_t)nj;
  CU(w.alloc(&dk, total));
  MatrixRun m{w.st, dqi, dqj, ni, nj, dk};
  CU(with_kernel(dim, order, m));
  CU(cudaMemcpyAsync(knl, dk, sizeof(double) * total, cudaMemcpyDeviceToHost, w.st));
  CU(cudaStreamSynchronize(w.st));
  return 0;
}

extern "C" int lddmm_multiply_kernel2(int dim, int ni, const double *qi, int nj,
                                      const double *qj, const double *a, int order,
                                      double width, double *v) {
  int rc = check_sets("lddmm_multiply_kernel2", dim, ni, nj, order, width);
  if (rc) return rc;
  if (!qi || !qj || !a || !v) {
    set_err("lddmm_multiply_kernel2: bad arguments");
    return LDDMM_ERR_ARG;
  }
  float kscale = 1.0f;
  double pd_fac = 0.0;
  def_kernel_scales(order, dim, width, &kscale, &pd_fac);
  const int ni_pad = pad_to(ni, kTile), nj_pad = pad_to(nj, kTile);
  OneShot w;
  CU(w.init());
  float4 *dqi = nullptr, *dqj = nullptr, *da = nullptr;
  int2 *items = nullptr;
  double *dv = nullptr;
  CU(w.put_points(&dqi, qi, ni, ni_pad, dim, kscale));
  CU(w.put_points(&dqj, qj, nj, nj_pad, dim, kscale));
  CU(w.put_points(&da, a, nj, nj_pad, dim, 1.0));
  CU(w.put_items(&items, ni_pad / kTile));
  CU(w.alloc(&dv, (size_t)ni * dim));
  CrossRun r{w.st, kCrossMul, dqi, nullptr, dqj, da, ni, ni_pad, nj_pad, 1.0, dv, items};
  int dev = 0;
  CU(cudaGetDevice(&dev));
  r.sms = device_sms(dev);
  CU(with_kernel(dim, order, r));
  CU(cudaMemcpyAsync(v, dv, sizeof(double) * ni * dim, cudaMemcpyDeviceToHost, w.st));
  CU(cudaStreamSynchronize(w.st));
  return 0;
}

extern "C" int lddmm_dq_kernel2(int dim, int ni, const double *qi, int nj, const double *qj,
                                const double *l, const double *r, int order, double width,
                                double *dqi, double *dqj) {
  int rc = check_sets("lddmm_dq_kernel2", dim, ni, nj, order, width);
  if (rc) return rc;
  if (!qi || !qj || !l || !r || !dqi || !dqj) {
    set_err("lddmm_dq_kernel2: bad arguments");
    return LDDMM_ERR_ARG;
  }
  float kscale = 1.0f;
  double pd_fac = 0.0;
  def_kernel_scales(order, dim, width, &kscale, &pd_fac);
  const int ni_pad = pad_to(ni, kTile), nj_pad = pad_to(nj, kTile);
  OneShot w;
  CU(w.init());
  float4 *dqi_s = nullptr, *dqj_s = nullptr, *dl = nullptr, *dr = nullptr;
  int2 *items_i = nullptr, *items_j = nullptr;
  double *oi = nullptr, *oj = nullptr;
  CU(w.put_points(&dqi_s, qi, ni, ni_pad, dim, kscale));
  CU(w.put_points(&dqj_s, qj, nj, nj_pad, dim, kscale));
  CU(w.put_points(&dl, l, ni, ni_pad, dim, 1.0));
  CU(w.put_points(&dr, r, nj, nj_pad, dim, 1.0));
  CU(w.put_items(&items_i, ni_pad / kTile));
  CU(w.put_items(&items_j, nj_pad / kTile));
  CU(w.alloc(&oi, (size_t)ni * dim));
  CU(w.alloc(&oj, (size_t)nj * dim));
  // i side: rows qi with l, columns qj with r; j side: rows qj with r, columns qi with l
  int dev = 0;
  CU(cudaGetDevice(&dev));
  CrossRun a{w.st, kCrossDq, dqi_s, dl, dqj_s, dr, ni, ni_pad, nj_pad, pd_fac, oi, items_i};
  a.sms = device_sms(dev);
  CU(with_kernel(dim, order, a));
  CrossRun b{w.st, kCrossDq, dqj_s, dr, dqi_s, dl, nj, nj_pad, ni_pad, pd_fac, oj, items_j};
  b.sms = a.sms;
  CU(with_kernel(dim, order, b));
  CU(cudaMemcpyAsync(dqi, oi, sizeof(double) * ni * dim, cudaMemcpyDeviceToHost, w.st));
  CU(cudaMemcpyAsync(dqj, oj, sizeof(double) * nj * dim, cudaMemcpyDeviceToHost, w.st));
  CU(cudaStreamSynchronize(w.st));
  return 0;
}

extern "C" int lddmm_varifold(const lddmm_problem *prob, const double *nde, double *val,
                              double *dq) {
  if (!prob || !nde || !val) {
    set_err("lddmm_varifold: bad arguments");
    return LDDMM_ERR_ARG;
  }
  lddmm_problem p = *prob;
  p.ini_nde = nde;
  p.time_num = 2;
  p.time_stp = 1.0;
  if (p.knl_order < -1 || p.knl_order > 4 || (p.dim == 2 && p.knl_order != -1)) p.knl_order = -1;
  if (!(p.knl_width > 0)) p.knl_width = 1.0;
  p.dis_wgt = 1.0;
  lddmm_ctx *ctx = nullptr;
  lddmm_config cfg = {};
  cfg.use_graph = -1;
  int rc = lddmm_ctx_create(&p, 1, &cfg, &ctx);
  if (rc) return rc;
  std::unique_ptr<lddmm_ctx, void (*)(lddmm_ctx *)> guard(ctx, lddmm_ctx_destroy);
  lddmm_ctx &c = *ctx;
  const int D = c.D;
  // positions at the final time = nde; zero energy partials
  double *q64T = c.q64 + (size_t)c.T * c.NPtot * D;
  CU(cudaMemcpyAsync(q64T, c.q64, sizeof(double) * c.NPtot * D, cudaMemcpyDeviceToDevice, c.stream));
  CU(cudaMemsetAsync(c.reg_part, 0, sizeof(double) * c.T * c.ngrp_tot, c.stream));
  CU(launch_set_active(c, 1));
  double *dqd = nullptr;
  CU(dalloc(c.stream, &dqd, (size_t)c.NPtot * D));
  DevBuf<double> g2(c.stream);
  g2.p = dqd;
  if (c.has_vfd) {
    CU(launch_geometry(c, q64T));
    CU(c.varifold(c));
    CU(launch_gather(c, q64T, nullptr, nullptr, dqd));
  }
  CU(launch_objective(c, nullptr, c.f_dev));
  std::vector<double> h((size_t)c.NPtot * D);
  CU(cudaMemcpyAsync(val, c.f_dev, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  CU(cudaMemcpyAsync(h.data(), dqd, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c.stream));
  CU(cudaStreamSynchronize(c.stream));
  if (dq) std::memcpy(dq, h.data(), sizeof(double) * (size_t)p.nde_num * D);
  return 0;
}

extern "C" int lddmm_LDDMM(int dim, int nde_num, int dfm_elm_num, int dfm_elm_ifo_num,
                           int tgt_elm_num, const double *iniNdeMat, const double *iniAlpVec,
                           const int *dfmElmVtxMat, const int *dfmElmIfoMat,
                           const double *tgtCenPosMat, const double *tgtElmVolVec,
                           const double *tgtUniDirMat, char cenKnlType, double cenKnlWidth,
                           char dirKnlType, double dirKnlWidth, double disWgt, int knlOrder,
                           double knlWidth, double timeStp, int timeNum, int MaxIterations,
                           double OptimalityTolerance, double Wolfe1, double Wolfe2, int Columns,
                           int Verbose, double *optAlpVec) {
  // Cpp/src/LDDMM.cpp:11-98: build the problem, copy the initial momenta, run LBFGS.
  if (!optAlpVec || !iniAlpVec) {
    set_err("lddmm_LDDMM: bad arguments");
    return LDDMM_ERR_ARG;
  }
  lddmm_problem p;
  std::memset(&p, 0, sizeof(p));
  p.dim = dim;
  p.nde_num = nde_num;
  p.time_num = timeNum;
  p.time_stp = timeStp;
  p.knl_order = knlOrder;
  p.knl_width = knlWidth;
  p.ini_nde = iniNdeMat;
  p.dis_wgt = disWgt;
  p.dfm_elm_num = dfm_elm_num;
  p.dfm_elm_vtx = dfmElmVtxMat;
  p.dfm_elm_ifo_num = dfmElmIfoMat ? dfm_elm_ifo_num : 0;
  p.dfm_elm_ifo = dfmElmIfoMat;
  p.tgt_elm_num = tgt_elm_num;
  p.tgt_cen_pos = tgtCenPosMat;
  p.tgt_uni_dir = tgtUniDirMat;
  p.tgt_elm_vol = tgtElmVolVec;
  p.cen_knl_type = cenKnlType;
  p.cen_knl_width = cenKnlWidth;
  p.dir_knl_type = dirKnlType;
  p.dir_knl_width = dirKnlWidth;
  lddmm_ctx *ctx = nullptr;
  int rc = lddmm_ctx_create(&p, 1, nullptr, &ctx);
  if (rc) return rc;
  std::unique_ptr<lddmm_ctx, void (*)(lddmm_ctx *)> guard(ctx, lddmm_ctx_destroy);
  const long long n = (long long)dim * nde_num * (timeNum - 1);
  std::memcpy(optAlpVec, iniAlpVec, sizeof(double) * n);
  lddmm_opt o;
  std::memset(&o, 0, sizeof(o));
  o.itr_max = MaxIterations;
  o.tol_val = OptimalityTolerance;
  o.wolfe1 = Wolfe1;
  o.wolfe2 = Wolfe2;
  o.mem_num = Columns;
  o.vbs_flg = Verbose;
  lddmm_result r;
  return lddmm_lbfgs(ctx, &o, optAlpVec, &r);
}

// ====================================================== allocation-free entry
//
// lddmm_multiply_kernel_noalloc: the shooting sweep for one point set with its working
// set in a file-scope device array instead of cudaMalloc'd memory.  Byte layout of the
// array (offsets 256-aligned): PairDesc | active flag | i-tile items | tile partials |
// scaled positions | FP32 momenta | next positions (scaled FP32, FP64).

constexpr int kNaMax = LDDMM_NOALLOC_MAX_POINTS;
constexpr int kNaTiles = kNaMax / kTile;
constexpr size_t kNaPd = 0;
constexpr size_t kNaAct = 256;
constexpr size_t kNaItems = 512;
constexpr size_t kNaTile = kNaItems + sizeof(int2) * kNaTiles;
constexpr size_t kNaQs = kNaTile + sizeof(double) * kNaTiles;
constexpr size_t kNaAs = kNaQs + sizeof(float4) * kNaMax;
constexpr size_t kNaQsn = kNaAs + sizeof(float4) * kNaMax;
constexpr size_t kNaQ64n = kNaQsn + sizeof(float4) * kNaMax;
constexpr size_t kNaBytes = kNaQ64n + sizeof(double) * 3 * kNaMax;
static_assert(sizeof(PairDesc) <= 256, "PairDesc must fit its slot");
static_assert(kNaTile % 256 == 0 && kNaQs % 256 == 0 && kNaAs % 256 == 0 &&
                  kNaQsn % 256 == 0 && kNaQ64n % 256 == 0,
              "scratch slots must stay 256-byte aligned");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

// Host-side device addresses of g_noalloc_scratch, one per device ordinal (the symbol
// name itself is only a host stand-in and must never be passed to a kernel).
static std::mutex g_noalloc_mu;
static unsigned char *g_noalloc_addr[128];

static int noalloc_scratch(int dev, unsigned char **out) {
  if (dev < 0 || dev >= 128) {
    set_err("lddmm_multiply_kernel_noalloc: device ordinal %d out of range", dev);
    return LDDMM_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_err("lddmm_multiply_kernel_noalloc: cudaGetSymbolAddress failed: %s",
              cudaGetErrorString(e));
      return LDDMM_ERR_CUDA;
    }
    g_noalloc_addr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_noalloc_addr[dev];
  return 0;
}

// Fills the scratch for one call: pair descriptor, active flag, tile items, and the
// FP32 operands with the padding rows cleared (the array keeps the previous call's
// contents).
__global__ void noalloc_prepare_kernel(unsigned char *scratch, PairDesc desc,
                                       const double *__restrict__ q,
                                       const double *__restrict__ a, int n, int npad, int D) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float4 *qs = reinterpret_cast<float4 *>(scratch + kNaQs);
  float4 *as = reinterpret_cast<float4 *>(scratch + kNaAs);
  if (i == 0) {
    *reinterpret_cast<PairDesc *>(scratch + kNaPd) = desc;
    *reinterpret_cast<int *>(scratch + kNaAct) = 1;
  }
  if (i < npad / kTile) reinterpret_cast<int2 *>(scratch + kNaItems)[i] = make_int2(0, i);
  if (i >= npad) return;
  float x[3] = {0, 0, 0}, y[3] = {0, 0, 0};
  if (i < n)
    for (int d = 0; d < D; ++d) {
      x[d] = (float)(q[(size_t)i * D + d] * desc.kscale);
      y[d] = (float)a[(size_t)i * D + d];
    }
  qs[i] = make_float4(x[0], x[1], x[2], 0.0f);
  as[i] = make_float4(y[0], y[1], y[2], 0.0f);
}

template <int D, int ORDER>
static cudaError_t noalloc_sweep(unsigned char *scratch, const double *q, const double *a,
                                 double *v, int ntiles, cudaStream_t stream) {
  ShootOp<D, ORDER> op;
  op.pd = reinterpret_cast<const PairDesc *>(scratch + kNaPd);
  op.act = reinterpret_cast<const int *>(scratch + kNaAct);
  op.qs_t = reinterpret_cast<const float4 *>(scratch + kNaQs);
  op.as_t = reinterpret_cast<const float4 *>(scratch + kNaAs);
  op.q64_t = q;
  op.q64_n = reinterpret_cast<double *>(scratch + kNaQ64n);
  op.qs_n = reinterpret_cast<float4 *>(scratch + kNaQsn);
  op.x64 = a;
  op.vlc64 = v;
  op.tile_part = reinterpret_cast<double *>(scratch + kNaTile);
  op.t = 0;
  // No programmatic stream serialisation here: the sweep reads its work list (written
  // by noalloc_prepare_kernel just before) ahead of its dependency wait, which is only
  // safe for the static lists of a context.  Without the attribute the sweep starts
  // after the preparation kernel has completed.
  const int S = default_cluster(ntiles);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(ntiles * S));
  cfg.blockDim = dim3(kWarps * 32);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)S;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, sweep_kernel<ShootOp<D, ORDER>, kWarps>, op,
                            reinterpret_cast<const int2 *>(scratch + kNaItems), S);
}

extern "C" int lddmm_multiply_kernel_noalloc(int dim, int n, const double *d_q,
                                             const double *d_a, int knl_order,
                                             double knl_width, double *d_v, void *stream) {
  if (dim != 2 && dim != 3) {
    set_err("lddmm_multiply_kernel_noalloc: dim must be 2 or 3");
    return LDDMM_ERR_ARG;
  }
  if (n < 1 || n > kNaMax) {
    set_err("lddmm_multiply_kernel_noalloc: n = %d outside 1..%d (LDDMM_NOALLOC_MAX_POINTS)",
            n, kNaMax);
    return LDDMM_ERR_ARG;
  }
  if (!d_q || !d_a || !d_v || !(knl_width > 0)) {
    set_err("lddmm_multiply_kernel_noalloc: null buffer or non-positive width");
    return LDDMM_ERR_ARG;
  }
  if (knl_order < -1 || knl_order > 4) {
    set_err("lddmm_multiply_kernel_noalloc: kernel order %d in %dD not supported", knl_order,
            dim);
    return LDDMM_ERR_UNSUPPORTED;
  }
  int dev = 0;
  CU(cudaGetDevice(&dev));
  unsigned char *scratch = nullptr;
  const int rc = noalloc_scratch(dev, &scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  PairDesc desc;
  std::memset(&desc, 0, sizeof(desc));
  desc.N = n;
  desc.Npad = pad_to(n, kTile);
  desc.var_num = (long long)dim * n;
  desc.dt = 1.0;
  def_kernel_scales(knl_order, dim, knl_width, &desc.kscale, &desc.pd_fac);
  const int ntiles = desc.Npad / kTile;
  noalloc_prepare_kernel<<<(desc.Npad + 255) / 256, 256, 0, st>>>(scratch, desc, d_q, d_a, n,
                                                                   desc.Npad, dim);
  CU(cudaGetLastError());
  cudaError_t e = cudaErrorInvalidValue;
  if (dim == 2) {
    switch (knl_order) {
      case -1: e = noalloc_sweep<2, -1>(scratch, d_q, d_a, d_v, ntiles, st); break;
      case 0: e = noalloc_sweep<2, 0>(scratch, d_q, d_a, d_v, ntiles, st); break;
      case 1: e = noalloc_sweep<2, 1>(scratch, d_q, d_a, d_v, ntiles, st); break;
      case 2: e = noalloc_sweep<2, 2>(scratch, d_q, d_a, d_v, ntiles, st); break;
      case 3: e = noalloc_sweep<2, 3>(scratch, d_q, d_a, d_v, ntiles, st); break;
      case 4: e = noalloc_sweep<2, 4>(scratch, d_q, d_a, d_v, ntiles, st); break;
    }
  } else {
    switch (knl_order) {
      case -1: e = noalloc_sweep<3, -1>(scratch, d_q, d_a, d_v, ntiles, st); break;
      case 0: e = noalloc_sweep<3, 0>(scratch, d_q, d_a, d_v, ntiles, st); break;
      case 1: e = noalloc_sweep<3, 1>(scratch, d_q, d_a, d_v, ntiles, st); break;
      case 2: e = noalloc_sweep<3, 2>(scratch, d_q, d_a, d_v, ntiles, st); break;
      case 3: e = noalloc_sweep<3, 3>(scratch, d_q, d_a, d_v, ntiles, st); break;
      case 4: e = noalloc_sweep<3, 4>(scratch, d_q, d_a, d_v, ntiles, st); break;
    }
  }
  CU(e);
  return 0;
}

// ============================================================ FP32 probe

// 8 independent FMA chains per thread; the result is stored only under a condition
// the host never meets, so the compiler keeps every FMA.
__global__ void fp32_probe_kernel(float *out, int iters, float seed) {
  float a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed + threadIdx.x * 1e-6f + k;
  const float m = 0.999999f, c = 1e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], m, c);
  }
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  if (s == -12345.0f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

extern "C" int lddmm_fp32_peak(int device, double *tflops) {
  if (!tflops) return LDDMM_ERR_ARG;
  CU(cudaSetDevice(device));
  int sms = 0;
  CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const int threads = 256, blocks = sms * 8, iters = 1 << 15;
  float *out = nullptr;
  CU(cudaMalloc(&out, sizeof(float) * threads * blocks));
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(e0);
    fp32_probe_kernel<<<blocks, threads>>>(out, iters, 1.0f);
    cudaEventRecord(e1);
    CU(cudaEventSynchronize(e1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0) best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  *tflops = 2.0 * 8.0 * iters * (double)threads * blocks / (best * 1e-3) / 1e12;
  return 0;
}

// Packed form of the probe: 4 independent FP32x2 chains (8 FMAs per iteration, as
// above) through the sm_100 paired FMA.
__global__ void fp32x2_probe_kernel(float *out, int iters, float seed) {
  float2 a[4];
#pragma unroll
  for (int k = 0; k < 4; ++k)
    a[k] = make_float2(seed + threadIdx.x * 1e-6f + k, seed + threadIdx.x * 1e-6f + k + 0.5f);
  const float2 m = make_float2(0.999999f, 0.999999f), c = make_float2(1e-7f, 1e-7f);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 4; ++k) a[k] = __ffma2_rn(a[k], m, c);
  }
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < 4; ++k) s += a[k].x + a[k].y;
  if (s == -12345.0f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// MUFU probe: 8 independent chains x <- 2^-x per thread (the ex2.approx the all-pairs
// loops use; the values stay in [0.5, 1]).
__global__ void ex2_probe_kernel(float *out, int iters, float seed) {
  float a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed * 1e-3f + threadIdx.x * 1e-7f + 0.1f * k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = ex2f(-a[k]);
  }
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  if (s == -12345.0f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Per-pipe throughput on `device`: out[0] scalar FP32 FMA TFLOP/s (the probe of
// lddmm_fp32_peak), out[1] packed FP32x2 FMA TFLOP/s, out[2] ex2.approx Gop/s
// (MUFU).  Best of three timed launches after a warm-up launch each.
extern "C" int lddmm_pipe_peaks(int device, double *out) {
  if (!out) return LDDMM_ERR_ARG;
  CU(cudaSetDevice(device));
  int sms = 0;
  CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const int threads = 256, blocks = sms * 8;
  float *buf = nullptr;
  CU(cudaMalloc(&buf, sizeof(float) * threads * blocks));
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  cudaError_t err = cudaSuccess;
  for (int which = 0; which < 3 && err == cudaSuccess; ++which) {
    const int iters = which == 2 ? 1 << 13 : 1 << 15;
    float best = 1e30f;
    for (int rep = 0; rep < 4 && err == cudaSuccess; ++rep) {
      cudaEventRecord(e0);
      if (which == 0) fp32_probe_kernel<<<blocks, threads>>>(buf, iters, 1.0f);
      else if (which == 1) fp32x2_probe_kernel<<<blocks, threads>>>(buf, iters, 1.0f);
      else ex2_probe_kernel<<<blocks, threads>>>(buf, iters, 1.0f);
      cudaEventRecord(e1);
      err = cudaGetLastError();
      if (err == cudaSuccess) err = cudaEventSynchronize(e1);
      float ms = 0.0f;
      if (err == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0) best = std::min(best, ms);
    }
    const double ops = 8.0 * iters * (double)threads * blocks;
    out[which] = which == 2 ? ops / (best * 1e-3) / 1e9 : 2.0 * ops / (best * 1e-3) / 1e12;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  CU(err);
  return 0;
}

// ================================================================ misc

// ============================================================ wait self-test

// One grid barrier on a cooperative grid of two CTAs.  With never_released the target
// is one arrival more than the grid, so nothing can complete it: every CTA must give
// up after `spin` polls, record the wait in the error word and leave.
__global__ void wait_selftest_kernel(StepSync *sy, int never_released, unsigned int spin) {
  const unsigned int target = gridDim.x + (never_released ? 1u : 0u);
  if (grid_barrier(sy, target, 4242u, spin)) grid_depart(sy);
}

extern "C" int lddmm_wait_selftest(int device, int never_released, double *ms) {
  CU(cudaSetDevice(device));
  cudaStream_t st = nullptr;
  CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  StepSync *sy = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = dalloc(st, &sy, 1);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e == cudaSuccess) e = cudaEventRecord(e0, st);
  if (e == cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2);
    cfg.blockDim = dim3(32);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, wait_selftest_kernel, sy, never_released, kSelftestSpin);
  }
  if (e == cudaSuccess) e = cudaEventRecord(e1, st);
  unsigned int w[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(w, sy, sizeof(w), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  float t = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  if (sy) cudaFreeAsync(sy, st);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  CU(e);
  if (ms) *ms = t;
  if (w[1]) {
    set_err("wait self-test: the grid barrier gave up (tag %u), as a barrier that nothing "
            "can complete must", w[1] - 1);
    return LDDMM_ERR_TIMEOUT;
  }
  return 0;
}

extern "C" const char *lddmm_last_error(void) { return g_err.c_str(); }
extern "C" const char *lddmm_version(void) { return "lddmm_b200 0.1 (sm_100a)"; }

extern "C" double lddmm_flops_per_pair(int sweep, int dim, int order, char ct, char dt) {
  // Arithmetic executed per pair interaction, FMA = 2 flops, MUFU ops = 1,
  // compensation overhead (6 flops per accumulator per 32 pairs) not counted.
  const int D = dim;
  const double dist = D + 2.0 * D;  // D subtracts, D FMAs for -r2
  if (sweep == 0) {                 // shooting: K and D FMAs
    const double k = (order == -1) ? 1.0 : (order == 0 ? 2.0 : (order == 1 ? 5.0 : 5.0 + 2.0 * (order - 1)));
    return dist + k + 2.0 * D;
  }
  if (sweep == 1) {                 // fused adjoint: K, W, lr (2D FMA), s, D + D FMAs
    const double k = (order == -1) ? 1.0 : (order == 0 ? 2.0 : (order == 1 ? 5.0 : 7.0 + 4.0 * (order - 1)));
    return dist + k + 2.0 * (2.0 * D) + 1.0 + 2.0 * D + 2.0 * D;
  }
  // varifold: centre kernel, ang (D FMAs), kw, direction terms, S, A, C
  const double cen = (ct == 'G') ? 1.0 : 3.0;
  double dir = (dt == 'B') ? 3.0 : 6.0;
  return dist + cen + 2.0 * D + 1.0 + dir + 2.0 * D + 2.0 * D + (ct == 'C' ? 1.0 : 0.0);
}
