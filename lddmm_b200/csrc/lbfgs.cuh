// Device-resident FP64 L-BFGS with the weak-Wolfe line search, for a batch of
// independent pairs, without host round trips inside an iteration.
//
// Semantics: Cpp/src/LBFGS.cpp:25-112 (outer loop, H0 = s.y / y.y, ring buffer,
// stop at |g| < tol), Cpp/src/getDirection.cpp:9-66 (two-loop recursion),
// Cpp/src/lineSearch.cpp:26-110 (bracketing by doubling / bisection with the
// heuristic limits bisMax = max(50, log2(1e5 |d|)), epdMax = max(10, log2(1e5/|d|))).
//
// Execution: every objective evaluation of the batch is followed by one "cycle" of
// fixed kernels (captured once in a CUDA graph):
//   POST   dots g_t.g_t, g_t.d over the trial gradients
//   DECIDE per-pair state machine: Wolfe tests, accept / expand / bisect / fail
//   ACCEPT s = x_t - x, y = g_t - g into the ring, x = x_t, g = g_t; dots s.y, y.y, s.g
//   B_0..B_{m-1}  first loop of the two-loop recursion (one dot + one axpy per pass)
//   F_0..F_{m-1}  second loop, right-aligned so every pair ends in F_{m-1}
//   FIN    d = -r, x_t = x + t d, FP32 copy of x_t for the sweeps; dots g.d, d.d
//   LSINIT descent test and line-search limits for pairs with a new direction
// Each vector pass covers all pairs' variables in chunks of kChunk; a chunk belongs
// to one pair and writes its partial dots, and the next pass reduces its pair's
// partials in chunk order (deterministic).  Pairs that do not take part in a pass
// leave in the first instructions of each CTA.
#pragma once

#include <cfloat>

#include "common.cuh"
#include "layout.h"
#include "persist.cuh"

namespace lddmm {

constexpr int kChunk = 2048;  // doubles per vector-pass CTA
constexpr int kVecThreads = 256;

enum PassMode : int { kPost = 0, kAccept = 1, kTwoLoopB = 2, kTwoLoopF = 3, kFin = 4 };

struct VecArgs {
  const PairDesc *pd;
  PairState *st;
  const int *chunk_pair;
  double *X, *G, *XT, *GT, *Dv, *Qv, *S, *Y;
  long long nvar;   // stride between ring slots
  float4 *as;       // FP32 trial alpha in point layout [T][NPtot]
  int NPtot;
  int D;
  int m;            // memory
  const double *part_in;
  double *part_out;
};

// Sum of a pair's chunk partials (component j), by warp 0, fixed order.
__device__ __forceinline__ double pair_partial(const double *part, int c0, int nc, int j) {
  double s = 0.0;
  const int lane = threadIdx.x & 31;
  for (int c = lane; c < nc; c += 32) s += part[(size_t)(c0 + c) * 3 + j];
  return warp_sum(s);
}

__device__ __forceinline__ void store_trial_f32(const VecArgs &A, const PairDesc &P,
                                                long long v, double x) {
  const long long nd = (long long)P.N * A.D;
  const int t = (int)(v / nd);
  const long long rem = v - (long long)t * nd;
  const int i = (int)(rem / A.D), d = (int)(rem - (long long)i * A.D);
  float *f = reinterpret_cast<float *>(A.as);
  f[((size_t)t * A.NPtot + P.pt_off + i) * 4 + d] = (float)x;
}

// One vector pass over chunk c.  `k` = two-loop pass index for kTwoLoopB / kTwoLoopF.
// Called by a whole CTA (it synchronises the CTA).
__device__ void vec_pass_chunk(const VecArgs &A, int mode, int k, int c) {
  __shared__ double s_scal[4];
  __shared__ double s_scr[kVecThreads / 32];
  const int p = A.chunk_pair[c];
  const PairDesc &P = A.pd[p];
  PairState &S = A.st[p];
  const int m = A.m;
  const int first = (c == P.chunk_off);

  // ----- participation and scalar set-up (uniform per CTA)
  bool go = false;
  int idx = 0, idx_next = -1;  // history slots
  double coef = 0.0;
  int final_b = 0;
  if (mode == kPost) {
    go = (S.phase == kPhaseInit || S.phase == kPhaseLS) && S.active;
  } else if (mode == kAccept) {
    go = (S.action == kActAccept || S.action == kActAcceptInit);
  } else if (mode == kTwoLoopB) {
    go = S.need_dir && k < S.hisNum;
    if (go) {
      idx = S.newIdx - k;
      if (idx < 0) idx += m;
      double dprev = 0.0, H0 = 0.0, rho = 0.0;
      if (threadIdx.x < 32) {
        dprev = pair_partial(A.part_in, P.chunk_off, P.nchunk, k == 0 ? 2 : 0);
        if (k == 0) {
          const double sy = pair_partial(A.part_in, P.chunk_off, P.nchunk, 0);
          const double yy = pair_partial(A.part_in, P.chunk_off, P.nchunk, 1);
          rho = 1.0 / sy;
          H0 = sy / yy;
        }
      }
      if (threadIdx.x == 0) {
        if (k == 0) {
          s_scal[1] = H0;
          s_scal[2] = rho;
        } else {
          s_scal[1] = S.H0;
          s_scal[2] = S.rho[idx];
        }
        s_scal[0] = s_scal[2] * dprev;  // alpha_idx = rho (s.q)
      }
      __syncthreads();
      coef = s_scal[0];
      if (first && threadIdx.x == 0) {
        if (k == 0) {
          S.H0 = s_scal[1];
          S.rho[idx] = s_scal[2];
        }
        S.alf[idx] = coef;
      }
      final_b = (k + 1 == S.hisNum);
      if (!final_b) {
        idx_next = idx - 1;
        if (idx_next < 0) idx_next += m;
      } else {
        idx_next = (S.hisNum < m) ? 0 : S.newIdx + 1;  // oldest slot
        if (idx_next >= m) idx_next -= m;
      }
    }
  } else if (mode == kTwoLoopF) {
    const int h = k - (m - S.hisNum);
    go = S.need_dir && h >= 0;
    if (go) {
      int old = (S.hisNum < m) ? 0 : S.newIdx + 1;
      if (old >= m) old -= m;
      idx = old + h;
      if (idx >= m) idx -= m;
      double dprev = 0.0;
      if (threadIdx.x < 32) dprev = pair_partial(A.part_in, P.chunk_off, P.nchunk, 0);
      if (threadIdx.x == 0) s_scal[0] = S.alf[idx] - S.rho[idx] * dprev;  // alpha - beta
      __syncthreads();
      coef = s_scal[0];
      if (h + 1 < S.hisNum) {
        idx_next = idx + 1;
        if (idx_next >= m) idx_next -= m;
      }
    }
  } else {  // kFin
    go = S.need_dir || (S.phase == kPhaseLS && S.action == kActNone && S.active);
  }
  if (!go) return;

  // ----- elementwise work + up to three dots
  const long long base = P.var_off;
  const long long n = P.var_num;
  const long long lo = (long long)(c - P.chunk_off) * kChunk;
  const long long hi = min(lo + kChunk, n);
  const long long NV = A.nvar;
  double d0 = 0.0, d1 = 0.0, d2 = 0.0;

  if (mode == kPost) {
    for (long long v = lo + threadIdx.x; v < hi; v += kVecThreads) {
      const double g = A.GT[base + v];
      d0 += g * g;
      d1 += g * A.Dv[base + v];
    }
  } else if (mode == kAccept) {
    if (S.action == kActAcceptInit) {
      for (long long v = lo + threadIdx.x; v < hi; v += kVecThreads) {
        A.X[base + v] = A.XT[base + v];
        A.G[base + v] = A.GT[base + v];
      }
    } else {
      double *Sv = A.S + (size_t)S.newIdx * NV + base;
      double *Yv = A.Y + (size_t)S.newIdx * NV + base;
      for (long long v = lo + threadIdx.x; v < hi; v += kVecThreads) {
        const double xt = A.XT[base + v], gt = A.GT[base + v];
        const double s = xt - A.X[base + v];
        const double y = gt - A.G[base + v];
        Sv[v] = s;
        Yv[v] = y;
        A.X[base + v] = xt;
        A.G[base + v] = gt;
        d0 += s * y;
        d1 += y * y;
        d2 += s * gt;
      }
    }
  } else if (mode == kTwoLoopB) {
    const double *Yv = A.Y + (size_t)idx * NV + base;
    const double *src = (k == 0) ? (A.G + base) : (A.Qv + base);
    const double H0 = s_scal[1];
    const double *Nx = final_b ? (A.Y + (size_t)idx_next * NV + base)
                               : (A.S + (size_t)idx_next * NV + base);
    for (long long v = lo + threadIdx.x; v < hi; v += kVecThreads) {
      double q = src[v] - coef * Yv[v];
      if (final_b) q *= H0;  // r = H0 q
      A.Qv[base + v] = q;
      d0 += Nx[v] * q;
    }
  } else if (mode == kTwoLoopF) {
    const double *Sv = A.S + (size_t)idx * NV + base;
    const double *Ny = (idx_next >= 0) ? (A.Y + (size_t)idx_next * NV + base) : nullptr;
    for (long long v = lo + threadIdx.x; v < hi; v += kVecThreads) {
      const double r = A.Qv[base + v] + coef * Sv[v];
      A.Qv[base + v] = r;
      if (Ny) d0 += Ny[v] * r;
    }
  } else {  // kFin
    if (S.need_dir) {
      const double *src = (S.hisNum == 0) ? (A.G + base) : (A.Qv + base);
      for (long long v = lo + threadIdx.x; v < hi; v += kVecThreads) {
        const double d = -src[v];
        const double g = A.G[base + v];
        A.Dv[base + v] = d;
        const double xt = A.X[base + v] + d;
        A.XT[base + v] = xt;
        store_trial_f32(A, P, v, xt);
        d0 += g * d;
        d1 += d * d;
      }
    } else {
      const double t = S.t;
      for (long long v = lo + threadIdx.x; v < hi; v += kVecThreads) {
        const double xt = A.X[base + v] + t * A.Dv[base + v];
        A.XT[base + v] = xt;
        store_trial_f32(A, P, v, xt);
      }
    }
  }
  d0 = block_sum(d0, s_scr);
  d1 = block_sum(d1, s_scr);
  d2 = block_sum(d2, s_scr);
  if (threadIdx.x == 0) {
    A.part_out[(size_t)c * 3 + 0] = d0;
    A.part_out[(size_t)c * 3 + 1] = d1;
    A.part_out[(size_t)c * 3 + 2] = d2;
  }
  __syncthreads();
}

// One vector pass as its own launch (one CTA per chunk).
__global__ void __launch_bounds__(kVecThreads) vec_pass_kernel(VecArgs A, int mode, int k) {
  pdl_wait();
  pdl_trigger();
  vec_pass_chunk(A, mode, k, blockIdx.x);
}

__device__ __forceinline__ double serial_partial(const double *part, int c0, int nc, int j) {
  double s = 0.0;
  for (int c = 0; c < nc; ++c) s += part[(size_t)(c0 + c) * 3 + j];
  return s;
}

// After POST.  One thread per pair.  Records (f, |g|, step, evals) per iteration.
__device__ void decide_pair(const PairDesc *__restrict__ pd, PairState *st, int p,
                            const double *__restrict__ part, const OptParams &o, double *rec) {
  PairState &S = st[p];
  const PairDesc &D = pd[p];
  S.action = kActNone;
  S.need_dir = 0;
  if (!S.active || (S.phase != kPhaseInit && S.phase != kPhaseLS)) return;
  const double gg = serial_partial(part, D.chunk_off, D.nchunk, 0);
  const double gd = serial_partial(part, D.chunk_off, D.nchunk, 1);
  const double ft = S.f_try;
  const double glt = sqrt(gg);
  const bool finite = isfinite(ft) && isfinite(gg);
  S.evals += 1;
  double *R = rec ? rec + (size_t)p * o.rec_cap * 4 : nullptr;

  if (S.phase == kPhaseInit) {
    if (!finite) {
      S.phase = kPhaseFailed;
      S.status = -3;
      return;
    }
    S.f = ft;
    S.f_prev = ft;
    S.glen = glt;
    S.action = kActAcceptInit;
    S.itr = 1;
    S.newIdx = -1;
    if (R && o.rec_cap > 0) {
      R[0] = ft; R[1] = glt; R[2] = 0.0; R[3] = 0.0;
    }
    if (glt < o.tol || o.itr_max < 1) {
      S.phase = kPhaseDone;
      return;
    }
    S.need_dir = 1;
    S.hisNum = 0;
    return;
  }

  // line-search trial (lineSearch.cpp:57-91)
  S.objCnt += 1;
  bool accept = false;
  if (finite && glt < o.tol) {
    accept = true;
  } else {
    if (!finite || ft >= S.f + o.wolfe1 * S.t * S.slp)
      S.relR = S.t;
    else if (gd <= o.wolfe2 * S.slp)
      S.relL = S.t;
    else
      accept = true;
  }
  if (!accept) {
    if (S.relR == DBL_MAX) {
      S.t *= 2.0;
      S.epdCnt += 1;
    } else {
      S.t = 0.5 * (S.relL + S.relR);
      S.bisCnt += 1;
    }
    if (!(S.bisCnt <= S.bisMax && S.epdCnt <= S.epdMax)) {
      S.phase = kPhaseFailed;
      S.status = (S.relR == DBL_MAX) ? 2 : 3;
    }
    return;
  }
  // accepted (LBFGS.cpp:94-108)
  S.stp = S.t * S.dlen;
  S.newIdx = (S.newIdx == o.mem_num - 1) ? 0 : S.newIdx + 1;
  S.f_prev = S.f;
  S.f = ft;
  S.glen = glt;
  S.iters += 1;
  S.action = kActAccept;
  if (R && S.iters < o.rec_cap) {
    double *r = R + (size_t)S.iters * 4;
    r[0] = ft; r[1] = glt; r[2] = S.stp; r[3] = S.objCnt;
  }
  S.itr += 1;
  const bool small_change =
      o.rel_obj_tol > 0.0 && fabs(S.f_prev - S.f) <= o.rel_obj_tol * fabs(S.f_prev);
  if (S.itr > o.itr_max || glt < o.tol || small_change) {
    S.phase = kPhaseDone;
    return;
  }
  S.need_dir = 1;
  S.hisNum = (S.itr <= o.mem_num) ? S.itr - 1 : o.mem_num;
}

__global__ void decide_kernel(const PairDesc *__restrict__ pd, PairState *st, int P,
                              const double *__restrict__ part, OptParams o, double *rec) {
  pdl_wait();
  pdl_trigger();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < P) decide_pair(pd, st, p, part, o, rec);
}

// After FIN.  Starts the line search of pairs with a new direction
// (lineSearch.cpp:34-55) and sets the evaluation flags for the next sweep.
__device__ void ls_init_pair(const PairDesc *__restrict__ pd, PairState *st, int p,
                             const double *__restrict__ part, int *act) {
  PairState &S = st[p];
  const PairDesc &D = pd[p];
  if (S.need_dir) {
    const double slp = serial_partial(part, D.chunk_off, D.nchunk, 0);
    const double dd = serial_partial(part, D.chunk_off, D.nchunk, 1);
    if (!(slp <= -DBL_MIN)) {  // not a descent direction (also catches NaN)
      S.phase = kPhaseFailed;
      S.status = isfinite(slp) ? 1 : -3;
    } else {
      S.slp = slp;
      S.dlen = sqrt(dd);
      const double lb = log2(1e5 * S.dlen), le = log2(1e5 / S.dlen);
      S.bisMax = (int)((50.0 > lb) ? 50.0 : lb);
      S.epdMax = (int)((10.0 > le) ? 10.0 : le);
      S.bisCnt = S.epdCnt = S.objCnt = 0;
      S.relL = 0.0;
      S.relR = DBL_MAX;
      S.t = 1.0;
      S.phase = kPhaseLS;
    }
  }
  S.active = (S.phase == kPhaseInit || S.phase == kPhaseLS) ? 1 : 0;
  act[p] = S.active;
}

__global__ void ls_init_kernel(const PairDesc *__restrict__ pd, PairState *st, int P,
                               const double *__restrict__ part, int *act) {
  pdl_wait();
  pdl_trigger();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < P) ls_init_pair(pd, st, p, part, act);
}

// The whole optimiser update of one cycle in one cooperative launch: the passes of
// the per-kernel sequence (POST, DECIDE, ACCEPT, B_0..B_{m-1}, F_0..F_{m-1}, FIN,
// LSINIT) run as grid-stride loops over the chunks, separated by grid barriers
// (bounded waits, persist.cuh).  Same arithmetic and reduction order as the per-kernel
// sequence.  part[0] / part[1] alternate exactly as there.
// Loop control of a device-side L-BFGS loop (CUDA graph WHILE node): counts the cycle
// and keeps the loop running while some pair is active and the cycle bound is not
// reached and no persistent sweep's barrier has timed out (error word).  Called by one
// CTA after the pairs' states are final for this cycle.
__device__ void cycle_control(cudaGraphConditionalHandle h, const int *act, int P, int *cyc,
                              int max_cycles, const StepSync *sy) {
  __shared__ int s_any;
  if (threadIdx.x == 0) s_any = 0;
  __syncthreads();
  int any = 0;
  for (int p = threadIdx.x; p < P; p += blockDim.x) any |= act[p];
  if (any) atomicOr(&s_any, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    const int n = ++(*cyc);
    const bool err = *(volatile const unsigned int *)&sy->error != 0u;
    cudaGraphSetConditional(h, (s_any && n < max_cycles && !err) ? 1u : 0u);
  }
}

__global__ void cycle_control_kernel(cudaGraphConditionalHandle h, const int *act, int P,
                                     int *cyc, int max_cycles, const StepSync *sy) {
  pdl_wait();
  cycle_control(h, act, P, cyc, max_cycles, sy);
}

__global__ void __launch_bounds__(kVecThreads)
    lbfgs_cycle_kernel(VecArgs A, OptParams o, double *part0, double *part1, double *rec,
                       int *act, int P, int nchunk, StepSync *sy, cudaGraphConditionalHandle h,
                       int *cyc, int max_cycles) {
  pdl_wait();
  stamp_entry(sy, 2);
  unsigned int phase = 0;
  auto barrier = [&]() -> bool {
    ++phase;
    return grid_barrier(sy, phase * gridDim.x, 1000u + phase);
  };
  int s = 0;  // pass sequence number: writes part[s & 1], reads part[(s + 1) & 1]
  auto pass = [&](int mode, int k) {
    A.part_out = (s & 1) ? part1 : part0;
    A.part_in = (s & 1) ? part0 : part1;
    for (int c = blockIdx.x; c < nchunk; c += gridDim.x) vec_pass_chunk(A, mode, k, c);
    ++s;
  };
  bool ok = true;
  do {  // one pass; a timed-out barrier breaks out to the loop-control exit below
    pass(kPost, 0);
    if (!(ok = barrier())) break;
    if (blockIdx.x == 0)
      for (int p = threadIdx.x; p < P; p += blockDim.x) decide_pair(A.pd, A.st, p, part0, o, rec);
    if (!(ok = barrier())) break;
    pass(kAccept, 0);
    if (!(ok = barrier())) break;
    for (int k = 0; k < o.mem_num && ok; ++k) {
      pass(kTwoLoopB, k);
      ok = barrier();
    }
    for (int k = 0; k < o.mem_num && ok; ++k) {
      pass(kTwoLoopF, k);
      ok = barrier();
    }
    if (!ok) break;
    pass(kFin, 0);
    if (!(ok = barrier())) break;
    if (blockIdx.x == 0) {
      const double *last = ((s - 1) & 1) ? part1 : part0;
      for (int p = threadIdx.x; p < P; p += blockDim.x) ls_init_pair(A.pd, A.st, p, last, act);
    }
  } while (false);
  if (ok) grid_depart(sy);
  if (blockIdx.x == 0 && cyc) {
    // drives the device-side loop; after a timed-out barrier (error word set) the loop
    // must end, whatever the pairs' state
    __syncthreads();
    if (ok) {
      cycle_control(h, act, P, cyc, max_cycles, sy);
    } else if (threadIdx.x == 0) {
      cudaGraphSetConditional(h, 0u);
    }
  }
  stamp_exit(sy, 2);
  pdl_trigger();
}

}  // namespace lddmm
