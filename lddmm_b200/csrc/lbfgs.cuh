// Device-resident FP64 L-BFGS with the weak-Wolfe line search, for a batch of
// independent pairs, without host round trips inside an iteration.
//
// Semantics: Cpp/src/LBFGS.cpp:25-112 (outer loop, H0 = s.y / y.y of the newest pair,
// ring buffer of memNum pairs, stop at |g| < tol), Cpp/src/getDirection.cpp:9-66 (the
// direction d = -H g of the limited-memory BFGS matrix H built from those pairs and
// H0), Cpp/src/lineSearch.cpp:26-110 (bracketing by doubling / bisection with the
// heuristic limits bisMax = max(50, log2(1e5 |d|)), epdMax = max(10, log2(1e5/|d|))).
//
// The direction uses the compact representation of the same matrix (Byrd, Nocedal and
// Schnabel, "Representations of quasi-Newton matrices and their use in limited memory
// methods", Math. Programming 63, 1994): with the pairs in chronological order,
// R = upper triangle of S^T Y, D = its diagonal and gamma = H0,
//   u = R^-1 (S^T g),   w = R^-T ((D + gamma Y^T Y) u - gamma Y^T g),
//   H g = gamma g + S w - gamma Y u.
// In exact arithmetic this is the reference's two-loop recursion; it needs all its dot
// products in one pass over the vectors instead of 2 m dependent ones.  S^T Y and
// Y^T Y are kept per pair (slot-indexed) and updated with the newest pair only.
//
// Execution: every objective evaluation of the batch is followed by one "cycle":
//   POST   dots g_t.g_t, g_t.d over the trial gradients
//   DECIDE per-pair state machine: Wolfe tests, accept / expand / bisect / fail
//   ACCEPT s = x_t - x, y = g_t - g into the ring, x = x_t, g = g_t; for every history
//          slot i the dots s_i.y, y_i.y, s_i.g, y_i.g (with the new y and g)
//   SOLVE  per pair: S^T Y and Y^T Y updated, the small triangular solves -> the
//          coefficients of g, S and Y in d
//   FIN    d = -(gamma g + S w - gamma Y u), x_t = x + t d, FP32 copy of x_t for the
//          sweeps; dots g.d, d.d
//   LSINIT descent test and line-search limits for pairs with a new direction
// Each vector pass covers all pairs' variables in chunks of kChunk; a chunk belongs to
// one pair and writes its partial dots, which the next phase reduces in chunk order
// (deterministic).  Pairs that do not take part in a pass leave in the first
// instructions of each CTA.
#pragma once

#include <cfloat>

#include "common.cuh"
#include "layout.h"
#include "persist.cuh"

namespace lddmm {

constexpr int kChunk = 2048;  // doubles per vector-pass CTA
constexpr int kVecThreads = 256;
constexpr int kPartStride = 4 * kMaxMem;  // dot partials per chunk (ACCEPT: 4 per slot)
constexpr int kDotGroup = 4;              // history slots per accumulation sweep of a chunk
constexpr int kCoefStride = 1 + 2 * kMaxMem;  // per pair: gamma, S coefficients, Y coefficients

enum PassMode : int { kPost = 0, kAccept = 1, kFin = 2 };

struct VecArgs {
  const PairDesc *pd;
  PairState *st;
  const int *chunk_pair;
  double *X, *G, *XT, *GT, *Dv, *S, *Y;
  long long nvar;   // stride between ring slots
  float4 *as;       // FP32 trial alpha in point layout [T][NPtot]
  int NPtot;
  int D;
  int m;            // memory
  double *part;     // dot partials [chunk][pstride]
  double *SY, *YY;  // per pair [m][m], slot-indexed: SY[i][j] = s_i.y_j (i no newer than j)
  double *coef;     // per pair [cstride]
  int pstride;      // doubles per chunk in `part`: kPartStride, or 4 m (long memory)
  int cstride;      // doubles per pair in `coef`: kCoefStride, or 1 + 2 m (long memory)
  int lm;           // long memory (m > kMaxMem): the phases of the lm_* functions below
  double *RI;       // long memory, per pair [m][m]: R^-1, slot-indexed (see lm_rinv_u)
  double *LV;       // long memory, per pair [m][4]: s_i.y, y_i.y, s_i.g, y_i.g (new y, g)
  double *SYd;      // long memory, per pair [m]: s_i.y_i
  double *LU;       // long memory, per pair [2 m]: u, then t = (D + gamma Y^T Y) u - gamma Y^T g
};

__device__ __forceinline__ void store_trial_f32(const VecArgs &A, const PairDesc &P,
                                                long long v, double x) {
  const long long nd = (long long)P.N * A.D;
  const int t = (int)(v / nd);
  const long long rem = v - (long long)t * nd;
  const int i = (int)(rem / A.D), d = (int)(rem - (long long)i * A.D);
  float *f = reinterpret_cast<float *>(A.as);
  f[((size_t)t * A.NPtot + P.pt_off + i) * 4 + d] = (float)x;
}

// Block sums of K values per thread (fixed order), written to out[0..K) by threads < K.
template <int K>
__device__ __forceinline__ void block_sums(double (&v)[K], double *out, int n_out) {
  __shared__ double s_red[kVecThreads / 32][K];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) s_red[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x < n_out) {
    double t = 0.0;
    for (int w = 0; w < kVecThreads / 32; ++w) t += s_red[w][threadIdx.x];
    out[threadIdx.x] = t;
  }
  __syncthreads();
}

// Number of valid ring slots: slots 0..h-1 until the ring is full, then all m.
__device__ __forceinline__ bool slot_valid(int i, int h, int m) { return h >= m || i < h; }

// One vector pass over chunk c.  Called by a whole CTA (it synchronises the CTA).
__device__ void vec_pass_chunk(const VecArgs &A, int mode, int c) {
  __shared__ double s_coef[kCoefStride];
  const int p = A.chunk_pair[c];
  const PairDesc &P = A.pd[p];
  const PairState &S = A.st[p];
  const int m = A.m;
  bool go;
  if (mode == kPost)
    go = (S.phase == kPhaseInit || S.phase == kPhaseLS) && S.active;
  else if (mode == kAccept)
    go = (S.action == kActAccept || S.action == kActAcceptInit);
  else
    go = S.need_dir || (S.phase == kPhaseLS && S.action == kActNone && S.active);
  if (!go) return;

  const long long base = P.var_off;
  const long long n = P.var_num;
  const long long lo = (long long)(c - P.chunk_off) * kChunk;
  const long long hi = min(lo + kChunk, n);
  const long long NV = A.nvar;
  double *out = A.part + (size_t)c * A.pstride;

  if (mode == kPost) {
    double v[2] = {0.0, 0.0};
    for (long long k = lo + threadIdx.x; k < hi; k += kVecThreads) {
      const double g = A.GT[base + k];
      v[0] += g * g;
      v[1] += g * A.Dv[base + k];
    }
    block_sums<2>(v, out, 2);
    return;
  }
  if (mode == kAccept) {
    if (S.action == kActAcceptInit) {
      for (long long k = lo + threadIdx.x; k < hi; k += kVecThreads) {
        A.X[base + k] = A.XT[base + k];
        A.G[base + k] = A.GT[base + k];
      }
      return;
    }
    const int nw = S.newIdx, h = S.hisNum;
    double *Sn = A.S + (size_t)nw * NV + base;
    double *Yn = A.Y + (size_t)nw * NV + base;
    for (long long k = lo + threadIdx.x; k < hi; k += kVecThreads) {
      const double xt = A.XT[base + k], gt = A.GT[base + k];
      Sn[k] = xt - A.X[base + k];
      Yn[k] = gt - A.G[base + k];
      A.X[base + k] = xt;
      A.G[base + k] = gt;
    }
    // the slot dots with the new y and g, kDotGroup slots per sweep of the chunk (a
    // thread re-reads only the elements it wrote above)
    for (int i0 = 0; i0 < m; i0 += kDotGroup) {
      double v[4 * kDotGroup];
#pragma unroll
      for (int q = 0; q < 4 * kDotGroup; ++q) v[q] = 0.0;
      for (long long k = lo + threadIdx.x; k < hi; k += kVecThreads) {
        const double y = Yn[k], g = A.G[base + k];
#pragma unroll
        for (int q = 0; q < kDotGroup; ++q) {
          const int i = i0 + q;
          if (i < m && slot_valid(i, h, m)) {
            const double si = A.S[(size_t)i * NV + base + k], yi = A.Y[(size_t)i * NV + base + k];
            v[4 * q + 0] += si * y;
            v[4 * q + 1] += yi * y;
            v[4 * q + 2] += si * g;
            v[4 * q + 3] += yi * g;
          }
        }
      }
      block_sums<4 * kDotGroup>(v, out + 4 * i0, min(4 * kDotGroup, 4 * (m - i0)));
    }
    return;
  }
  // kFin
  if (S.need_dir) {
    const int h = S.hisNum;
    if (threadIdx.x < 1 + 2 * m) s_coef[threadIdx.x] = A.coef[(size_t)p * A.cstride + threadIdx.x];
    __syncthreads();
    const double gamma = s_coef[0];
    double v[2] = {0.0, 0.0};
    for (long long k = lo + threadIdx.x; k < hi; k += kVecThreads) {
      const double g = A.G[base + k];
      double hg = gamma * g;
      if (h > 0)
        for (int i = 0; i < m; ++i)
          if (slot_valid(i, h, m))
            hg += s_coef[1 + i] * A.S[(size_t)i * NV + base + k] +
                  s_coef[1 + m + i] * A.Y[(size_t)i * NV + base + k];
      const double d = -hg;
      A.Dv[base + k] = d;
      const double xt = A.X[base + k] + d;
      A.XT[base + k] = xt;
      store_trial_f32(A, P, k, xt);
      v[0] += g * d;
      v[1] += d * d;
    }
    block_sums<2>(v, out, 2);
  } else {
    const double t = S.t;
    for (long long k = lo + threadIdx.x; k < hi; k += kVecThreads) {
      const double xt = A.X[base + k] + t * A.Dv[base + k];
      A.XT[base + k] = xt;
      store_trial_f32(A, P, k, xt);
    }
  }
}

// One vector pass as its own launch (one CTA per chunk).
__global__ void __launch_bounds__(kVecThreads) vec_pass_kernel(VecArgs A, int mode) {
  pdl_wait();
  pdl_trigger();
  vec_pass_chunk(A, mode, blockIdx.x);
}

// Sum of entry j of chunks c0 .. c0 + nc - 1, in chunk order (rows of `stride` doubles).
__device__ __forceinline__ double serial_partial(const double *part, int c0, int nc, int j,
                                                 int stride) {
  double s = 0.0;
  for (int c = 0; c < nc; ++c) s += part[(size_t)(c0 + c) * stride + j];
  return s;
}

// Sum of the pairs (j, j + 2, ..., j + 2 (nsub - 1)) of every chunk, chunk by chunk in
// order: the FIN partials, one (g.d, d.d) pair per sub-chunk (nsub = 1: one per chunk).
__device__ __forceinline__ double serial_partial_sub(const double *part, int c0, int nc, int j,
                                                     int stride, int nsub) {
  double s = 0.0;
  for (int c = 0; c < nc; ++c)
    for (int k = 0; k < nsub; ++k) s += part[(size_t)(c0 + c) * stride + j + 2 * k];
  return s;
}

// After ACCEPT, one CTA per pair with a new direction: the pair's slot dots (chunk
// order), the S^T Y / Y^T Y update with the newest pair, the compact-form solves.
__device__ void solve_pair(const VecArgs &A, int p) {
  __shared__ double s_v[4 * kMaxMem];
  PairState &S = A.st[p];
  if (!S.need_dir) return;  // uniform for the CTA
  const PairDesc &P = A.pd[p];
  const int m = A.m, h = S.hisNum, nw = S.newIdx;
  double *coef = A.coef + (size_t)p * A.cstride;
  if (h == 0) {  // first direction: H0 = 1 (LBFGS.cpp:73-74), d = -g
    if (threadIdx.x == 0) {
      coef[0] = 1.0;
      S.H0 = 1.0;
    }
    return;
  }
  for (int j = threadIdx.x; j < 4 * m; j += blockDim.x)
    s_v[j] = slot_valid(j / 4, h, m)
                 ? serial_partial(A.part, P.chunk_off, P.nchunk, j, A.pstride)
                 : 0.0;
  __syncthreads();
  if (threadIdx.x != 0) return;
  double *SY = A.SY + (size_t)p * m * m, *YY = A.YY + (size_t)p * m * m;
  for (int i = 0; i < m; ++i) {
    if (!slot_valid(i, h, m)) continue;
    SY[(size_t)i * m + nw] = s_v[4 * i + 0];
    YY[(size_t)i * m + nw] = s_v[4 * i + 1];
    YY[(size_t)nw * m + i] = s_v[4 * i + 1];
  }
  const double gamma = s_v[4 * nw + 0] / s_v[4 * nw + 1];  // s.y / y.y, newest pair
  S.H0 = gamma;
  // chronological order of the slots, oldest first
  int ord[kMaxMem];
  const int old = (h < m) ? 0 : (nw + 1 == m ? 0 : nw + 1);
  for (int a = 0; a < h; ++a) ord[a] = (old + a) % m;
  double u[kMaxMem], w[kMaxMem];
  // R u = S^T g  (R[a][b] = s_{o_a}.y_{o_b}, a <= b), back substitution
  for (int a = h - 1; a >= 0; --a) {
    double r = s_v[4 * ord[a] + 2];
    for (int b = a + 1; b < h; ++b) r -= SY[(size_t)ord[a] * m + ord[b]] * u[b];
    u[a] = r / SY[(size_t)ord[a] * m + ord[a]];
  }
  // R^T w = (D + gamma Y^T Y) u - gamma Y^T g, forward substitution
  for (int a = 0; a < h; ++a) {
    double t = SY[(size_t)ord[a] * m + ord[a]] * u[a] - gamma * s_v[4 * ord[a] + 3];
    for (int b = 0; b < h; ++b) t += gamma * YY[(size_t)ord[a] * m + ord[b]] * u[b];
    for (int b = 0; b < a; ++b) t -= SY[(size_t)ord[b] * m + ord[a]] * w[b];
    w[a] = t / SY[(size_t)ord[a] * m + ord[a]];
  }
  coef[0] = gamma;
  for (int i = 0; i < m; ++i) {
    coef[1 + i] = 0.0;
    coef[1 + m + i] = 0.0;
  }
  for (int a = 0; a < h; ++a) {
    coef[1 + ord[a]] = w[a];
    coef[1 + m + ord[a]] = -gamma * u[a];
  }
}

__global__ void __launch_bounds__(kVecThreads) solve_kernel(VecArgs A) {
  pdl_wait();
  pdl_trigger();
  solve_pair(A, blockIdx.x);
}

// ------------------------------------------------------------- long memory (m > kMaxMem)
//
// The reference accepts any memNum (Columns; its own examples pass 10,000,
// Cpp/examples/sphere2cube/run_sphere2cube.m:31).  For memories beyond kMaxMem the same
// compact-representation direction is computed with every O(h^2) step spread over the
// grid instead of one thread per pair, and with R^-1 kept explicitly:
//   * appending the newest pair (s, y) to the chronological order adds a last column
//     r = S^T y (with r_new = s.y) to the upper triangular R; the inverse gains the
//     column -R^-1 r / r_new and the diagonal entry 1 / r_new;
//   * dropping the oldest pair (the ring wraps) removes R's first row and column, and
//     the inverse of the trailing block of an upper triangular matrix is the trailing
//     block of its inverse, so nothing is recomputed.
// RI is slot-indexed like Y^T Y; only entries (a, b) with a no newer than b are read,
// so the stale row of a slot that has just become the newest is never used.  Per cycle:
//   lm_accept_update  s, y into the ring, x, g updated            (chunks)
//   lm_accept_dots    s_i.y, y_i.y, s_i.g, y_i.g for every slot    (chunk x 8 slots)
//   lm_reduce         chunk partials -> LV, Y^T Y row / column, s.y (pair x slot, thread)
//   lm_rinv_u         new column of R^-1 and u = R^-1 S^T g        (pair x row, warp)
//   lm_t              t = (D + gamma Y^T Y) u - gamma Y^T g        (pair x row, warp)
//   lm_w              w = R^-T t, the coefficients of d            (pair x column, thread)
//   lm_fin            d, trial point, g.d, d.d                     (chunk x 256 variables)
// Each sum runs in a fixed order, so results are bit-reproducible run to run.

constexpr int kLmGroup = 8;                   // history slots per lm_accept_dots unit
constexpr int kLmSub = kChunk / kVecThreads;  // lm_fin units per chunk

// Chronological position k (oldest first) of a pair's history -> ring slot.
__device__ __forceinline__ int lm_slot(int k, int h, int nw, int m) {
  const int old = (h < m) ? 0 : (nw + 1 == m ? 0 : nw + 1);
  const int s = old + k;
  return s >= m ? s - m : s;
}

// Pairs that compute a new direction from a non-empty history this cycle.
__device__ __forceinline__ bool lm_solving(const PairState &S) {
  return S.need_dir && S.hisNum > 0;
}

__device__ void lm_accept_update(const VecArgs &A, int c) {
  const int p = A.chunk_pair[c];
  const PairDesc &P = A.pd[p];
  const PairState &S = A.st[p];
  if (S.action != kActAccept && S.action != kActAcceptInit) return;
  const long long base = P.var_off;
  const long long lo = (long long)(c - P.chunk_off) * kChunk;
  const long long hi = min(lo + kChunk, P.var_num);
  if (S.action == kActAcceptInit) {
    for (long long k = lo + threadIdx.x; k < hi; k += kVecThreads) {
      A.X[base + k] = A.XT[base + k];
      A.G[base + k] = A.GT[base + k];
    }
    return;
  }
  double *Sn = A.S + (size_t)S.newIdx * A.nvar + base;
  double *Yn = A.Y + (size_t)S.newIdx * A.nvar + base;
  for (long long k = lo + threadIdx.x; k < hi; k += kVecThreads) {
    const double xt = A.XT[base + k], gt = A.GT[base + k];
    Sn[k] = xt - A.X[base + k];
    Yn[k] = gt - A.G[base + k];
    A.X[base + k] = xt;
    A.G[base + k] = gt;
  }
}

// unit = chunk * ngrp + group: the four dots of slots group * 8 .. + 7 over the chunk.
__device__ void lm_accept_dots(const VecArgs &A, int unit) {
  const int ngrp = (A.m + kLmGroup - 1) / kLmGroup;
  const int c = unit / ngrp, i0 = (unit - c * ngrp) * kLmGroup;
  const int p = A.chunk_pair[c];
  const PairDesc &P = A.pd[p];
  const PairState &S = A.st[p];
  const int m = A.m, h = S.hisNum;
  if (S.action != kActAccept || !(h >= m || i0 < h)) return;  // uniform for the CTA
  const long long base = P.var_off;
  const long long lo = (long long)(c - P.chunk_off) * kChunk;
  const long long hi = min(lo + kChunk, P.var_num);
  const double *Yn = A.Y + (size_t)S.newIdx * A.nvar + base;
  double v[4 * kLmGroup];
#pragma unroll
  for (int q = 0; q < 4 * kLmGroup; ++q) v[q] = 0.0;
  for (long long k = lo + threadIdx.x; k < hi; k += kVecThreads) {
    const double y = Yn[k], g = A.G[base + k];
#pragma unroll
    for (int q = 0; q < kLmGroup; ++q) {
      const int i = i0 + q;
      if (i < m && slot_valid(i, h, m)) {
        const double si = A.S[(size_t)i * A.nvar + base + k];
        const double yi = A.Y[(size_t)i * A.nvar + base + k];
        v[4 * q + 0] += si * y;
        v[4 * q + 1] += yi * y;
        v[4 * q + 2] += si * g;
        v[4 * q + 3] += yi * g;
      }
    }
  }
  block_sums<4 * kLmGroup>(v, A.part + (size_t)c * A.pstride + 4 * i0,
                           min(4 * kLmGroup, 4 * (m - i0)));
}

// unit = p * m + i (one thread): slot i's dots reduced over the pair's chunks.
__device__ void lm_reduce(const VecArgs &A, long long unit) {
  const int m = A.m;
  const int p = (int)(unit / m), i = (int)(unit - (long long)p * m);
  const PairState &S = A.st[p];
  if (!lm_solving(S) || !slot_valid(i, S.hisNum, m)) return;
  const PairDesc &P = A.pd[p];
  double v[4];
#pragma unroll
  for (int q = 0; q < 4; ++q)
    v[q] = serial_partial(A.part, P.chunk_off, P.nchunk, 4 * i + q, A.pstride);
  double *lv = A.LV + ((size_t)p * m + i) * 4;
#pragma unroll
  for (int q = 0; q < 4; ++q) lv[q] = v[q];
  const int nw = S.newIdx;
  double *YY = A.YY + (size_t)p * m * m;
  YY[(size_t)i * m + nw] = v[1];
  YY[(size_t)nw * m + i] = v[1];
  if (i == nw) A.SYd[(size_t)p * m + nw] = v[0];
}

// unit = p * m + k (one warp): chronological row k of R^-1 gets its entry in the new
// column, and u_k = (R^-1 S^T g)_k.
__device__ void lm_rinv_u(const VecArgs &A, long long unit) {
  const int m = A.m, lane = threadIdx.x & 31;
  const int p = (int)(unit / m), k = (int)(unit - (long long)p * m);
  const PairState &S = A.st[p];
  const int h = S.hisNum, nw = S.newIdx;
  if (!lm_solving(S) || k >= h) return;  // uniform for the warp
  const double *lv = A.LV + (size_t)p * m * 4;
  double *RI = A.RI + (size_t)p * m * m;
  double *u = A.LU + (size_t)p * 2 * m;
  const double rho = lv[4 * nw + 0];  // s.y of the newest pair
  const double sg_new = lv[4 * nw + 2];
  if (k == h - 1) {
    if (lane == 0) {
      RI[(size_t)nw * m + nw] = 1.0 / rho;
      u[nw] = sg_new / rho;
    }
    return;
  }
  const int a = lm_slot(k, h, nw, m);
  double c = 0.0, e = 0.0;
  for (int l = k + lane; l < h - 1; l += 32) {
    const int b = lm_slot(l, h, nw, m);
    const double rab = RI[(size_t)a * m + b];
    c += rab * lv[4 * b + 0];
    e += rab * lv[4 * b + 2];
  }
  c = warp_sum(c);
  e = warp_sum(e);
  if (lane == 0) {
    const double col = -c / rho;
    RI[(size_t)a * m + nw] = col;
    u[a] = e + col * sg_new;
  }
}

// unit = p * m + k (one warp): t_a = s_a.y_a u_a + gamma sum_b (y_a.y_b) u_b - gamma y_a.g.
__device__ void lm_t(const VecArgs &A, long long unit) {
  const int m = A.m, lane = threadIdx.x & 31;
  const int p = (int)(unit / m), k = (int)(unit - (long long)p * m);
  const PairState &S = A.st[p];
  const int h = S.hisNum, nw = S.newIdx;
  if (!lm_solving(S) || k >= h) return;  // uniform for the warp
  const double *lv = A.LV + (size_t)p * m * 4;
  const double *YY = A.YY + (size_t)p * m * m;
  double *u = A.LU + (size_t)p * 2 * m;
  const double gamma = lv[4 * nw + 0] / lv[4 * nw + 1];
  const int a = lm_slot(k, h, nw, m);
  double s = 0.0;
  for (int l = lane; l < h; l += 32) {
    const int b = lm_slot(l, h, nw, m);
    s += YY[(size_t)a * m + b] * u[b];
  }
  s = warp_sum(s);
  if (lane == 0)
    u[m + a] = A.SYd[(size_t)p * m + a] * u[a] + gamma * s - gamma * lv[4 * a + 3];
}

// unit = p * m + k (one thread): w_b = sum over rows a no newer than b of R^-1[a][b] t_a,
// then the coefficients of S (w) and Y (-gamma u) in d.  Neighbouring threads take
// neighbouring columns, so the row reads coalesce.
__device__ void lm_w(const VecArgs &A, long long unit) {
  const int m = A.m;
  const int p = (int)(unit / m), k = (int)(unit - (long long)p * m);
  PairState &S = A.st[p];
  const int h = S.hisNum, nw = S.newIdx;
  if (!lm_solving(S) || k >= h) return;
  const double *lv = A.LV + (size_t)p * m * 4;
  const double *RI = A.RI + (size_t)p * m * m;
  const double *u = A.LU + (size_t)p * 2 * m;
  const double gamma = lv[4 * nw + 0] / lv[4 * nw + 1];
  const int b = lm_slot(k, h, nw, m);
  double w = 0.0;
  for (int l = 0; l <= k; ++l) {
    const int a = lm_slot(l, h, nw, m);
    w += RI[(size_t)a * m + b] * u[m + a];
  }
  double *coef = A.coef + (size_t)p * A.cstride;
  coef[1 + b] = w;
  coef[1 + m + b] = -gamma * u[b];
  if (k == 0) {
    coef[0] = gamma;
    S.H0 = gamma;
  }
}

// The first direction of a pair (no history): H0 = 1, d = -g (LBFGS.cpp:73-74).
__device__ void lm_first_direction(const VecArgs &A, int p) {
  PairState &S = A.st[p];
  if (S.need_dir && S.hisNum == 0) {
    A.coef[(size_t)p * A.cstride] = 1.0;
    S.H0 = 1.0;
  }
}

// unit = chunk * kLmSub + sub: 256 variables, one per thread; the sub-chunk's g.d and
// d.d go to entries 2 sub, 2 sub + 1 of the chunk's partial row.
__device__ void lm_fin(const VecArgs &A, int unit) {
  const int c = unit / kLmSub, sub = unit - c * kLmSub;
  const int p = A.chunk_pair[c];
  const PairDesc &P = A.pd[p];
  const PairState &S = A.st[p];
  if (!(S.need_dir || (S.phase == kPhaseLS && S.action == kActNone && S.active))) return;
  const long long base = P.var_off;
  const long long k = (long long)(c - P.chunk_off) * kChunk + (long long)sub * kVecThreads +
                      threadIdx.x;
  const bool in = k < P.var_num;
  if (S.need_dir) {
    const int m = A.m, h = S.hisNum;
    const double *coef = A.coef + (size_t)p * A.cstride;
    double v[2] = {0.0, 0.0};
    if (in) {
      const double g = A.G[base + k];
      double hg = coef[0] * g;
      const int nv = (h >= m) ? m : h;  // valid slots 0 .. nv - 1
      for (int i = 0; i < nv; ++i)
        hg += coef[1 + i] * A.S[(size_t)i * A.nvar + base + k] +
              coef[1 + m + i] * A.Y[(size_t)i * A.nvar + base + k];
      const double d = -hg;
      A.Dv[base + k] = d;
      const double xt = A.X[base + k] + d;
      A.XT[base + k] = xt;
      store_trial_f32(A, P, k, xt);
      v[0] = g * d;
      v[1] = d * d;
    }
    block_sums<2>(v, A.part + (size_t)c * A.pstride + 2 * sub, 2);
  } else if (in) {
    const double xt = A.X[base + k] + S.t * A.Dv[base + k];
    A.XT[base + k] = xt;
    store_trial_f32(A, P, k, xt);
  }
}

enum LmPhase : int {
  kLmUpdate = 0, kLmDots = 1, kLmReduce = 2, kLmRinvU = 3, kLmT = 4, kLmW = 5, kLmFin = 6
};

// One long-memory phase over its units, by CTA `blk` of `nblk` (grid-stride).
__device__ void lm_phase(const VecArgs &A, int phase, int P, int nchunk, int blk, int nblk) {
  const int ngrp = (A.m + kLmGroup - 1) / kLmGroup;
  const long long nslot = (long long)P * A.m;
  const int warp = threadIdx.x >> 5;
  constexpr int kW = kVecThreads / 32;
  switch (phase) {
    case kLmUpdate:
      for (int c = blk; c < nchunk; c += nblk) lm_accept_update(A, c);
      break;
    case kLmDots:
      for (int u = blk; u < nchunk * ngrp; u += nblk) lm_accept_dots(A, u);
      break;
    case kLmReduce:
      for (long long u = (long long)blk * kVecThreads + threadIdx.x; u < nslot;
           u += (long long)nblk * kVecThreads)
        lm_reduce(A, u);
      for (int p = blk * kVecThreads + threadIdx.x; p < P; p += nblk * kVecThreads)
        lm_first_direction(A, p);
      break;
    case kLmRinvU:
      for (long long u = (long long)blk * kW + warp; u < nslot; u += (long long)nblk * kW)
        lm_rinv_u(A, u);
      break;
    case kLmT:
      for (long long u = (long long)blk * kW + warp; u < nslot; u += (long long)nblk * kW)
        lm_t(A, u);
      break;
    case kLmW:
      for (long long u = (long long)blk * kVecThreads + threadIdx.x; u < nslot;
           u += (long long)nblk * kVecThreads)
        lm_w(A, u);
      break;
    case kLmFin:
      for (int u = blk; u < nchunk * kLmSub; u += nblk) lm_fin(A, u);
      break;
  }
}

// One long-memory phase as its own launch.
__global__ void __launch_bounds__(kVecThreads)
    lm_phase_kernel(VecArgs A, int phase, int P, int nchunk) {
  pdl_wait();
  pdl_trigger();
  lm_phase(A, phase, P, nchunk, blockIdx.x, gridDim.x);
}

// After POST.  One thread per pair.  Records (f, |g|, step, evals) per iteration.
__device__ void decide_pair(const PairDesc *__restrict__ pd, PairState *st, int p,
                            const double *__restrict__ part, int pstride, const OptParams &o,
                            double *rec) {
  PairState &S = st[p];
  const PairDesc &D = pd[p];
  S.action = kActNone;
  S.need_dir = 0;
  if (!S.active || (S.phase != kPhaseInit && S.phase != kPhaseLS)) return;
  const double gg = serial_partial(part, D.chunk_off, D.nchunk, 0, pstride);
  const double gd = serial_partial(part, D.chunk_off, D.nchunk, 1, pstride);
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
                              const double *__restrict__ part, int pstride, OptParams o,
                              double *rec) {
  pdl_wait();
  pdl_trigger();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < P) decide_pair(pd, st, p, part, pstride, o, rec);
}

// After FIN.  Starts the line search of pairs with a new direction
// (lineSearch.cpp:34-55) and sets the evaluation flags for the next sweep.
__device__ void ls_init_pair(const PairDesc *__restrict__ pd, PairState *st, int p,
                             const double *__restrict__ part, int pstride, int nsub, int *act) {
  PairState &S = st[p];
  const PairDesc &D = pd[p];
  if (S.need_dir) {
    const double slp = serial_partial_sub(part, D.chunk_off, D.nchunk, 0, pstride, nsub);
    const double dd = serial_partial_sub(part, D.chunk_off, D.nchunk, 1, pstride, nsub);
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
                               const double *__restrict__ part, int pstride, int nsub,
                               int *act) {
  pdl_wait();
  pdl_trigger();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < P) ls_init_pair(pd, st, p, part, pstride, nsub, act);
}

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

// The whole optimiser update of one cycle in one cooperative launch: the phases of
// the per-kernel sequence (POST, DECIDE, ACCEPT, SOLVE, FIN, LSINIT) as grid-stride
// loops over the chunks (pairs for SOLVE), separated by grid barriers (bounded waits,
// persist.cuh).  Same arithmetic and reduction order as the per-kernel sequence.
__global__ void __launch_bounds__(kVecThreads)
    lbfgs_cycle_kernel(VecArgs A, OptParams o, double *rec, int *act, int P, int nchunk,
                       StepSync *sy, cudaGraphConditionalHandle h, int *cyc, int max_cycles) {
  pdl_wait();
  stamp_entry(sy, 2);
  unsigned int phase = 0;
  auto barrier = [&]() -> bool {
    ++phase;
    return grid_barrier(sy, phase * gridDim.x, 1000u + phase);
  };
  auto pass = [&](int mode) {
    for (int c = blockIdx.x; c < nchunk; c += gridDim.x) vec_pass_chunk(A, mode, c);
  };
  bool ok = true;
  do {  // one pass; a timed-out barrier breaks out to the loop-control exit below
    pass(kPost);
    if (!(ok = barrier())) break;
    if (blockIdx.x == 0)
      for (int p = threadIdx.x; p < P; p += blockDim.x)
        decide_pair(A.pd, A.st, p, A.part, A.pstride, o, rec);
    if (!(ok = barrier())) break;
    if (A.lm) {
      // long memory: the lm_* phases in place of ACCEPT, SOLVE and FIN
      bool lm_ok = true;
      for (int ph = kLmUpdate; ph <= kLmFin; ++ph) {
        lm_phase(A, ph, P, nchunk, blockIdx.x, gridDim.x);
        if (!(lm_ok = barrier())) break;
      }
      if (!(ok = lm_ok)) break;
      if (blockIdx.x == 0)
        for (int p = threadIdx.x; p < P; p += blockDim.x)
          ls_init_pair(A.pd, A.st, p, A.part, A.pstride, kLmSub, act);
      break;
    }
    pass(kAccept);
    if (!(ok = barrier())) break;
    for (int p = blockIdx.x; p < P; p += gridDim.x) {
      solve_pair(A, p);
      __syncthreads();
    }
    if (!(ok = barrier())) break;
    pass(kFin);
    if (!(ok = barrier())) break;
    if (blockIdx.x == 0)
      for (int p = threadIdx.x; p < P; p += blockDim.x)
        ls_init_pair(A.pd, A.st, p, A.part, A.pstride, 1, act);
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
