// Learned warm start: a small per-point network that predicts a registration's
// initial momenta from the source landmarks and the target's varifold, trained on
// momenta that the plain method produced.  No counterpart in the reference (the
// reference always starts L-BFGS from the momenta it is given, usually zero).
//
// Network (all matrices BF16, FP32 accumulation on the tensor cores, tc_gemm.cuh):
//   target branch, per triangle:  t = (centre, unit normal, area * Et / 4 pi)   (7)
//       h1 = gelu(t T1 + b)   7 -> 64,     h2 = h1 T2 + b   64 -> 64
//       g  = max over the target's triangles of h2                        (64)
//   point branch, per source landmark i:  x_i = (q_i, g)                 (3 + 64)
//       a1 = gelu(x P1 + b)  67 -> 256,  a2 = gelu(a1 P2 + b)  256 -> 256,
//       y  = a2 P3 + b  256 -> 3T    (the momenta of all T steps, divided by a fixed
//                                     label scale)
// Loss: mean squared error against the plain method's momenta / label scale.
//
// Data layout: every dimension is padded to a multiple of 16 (7 -> 16, 67 -> 80,
// 3T -> multiple of 16) with zero weights, and every pair's rows are padded to a
// multiple of 16 (Np = round16(N) landmarks, Etp = round16(Et) triangles) with zero
// inputs, zero labels and zero loss gradients, so each GEMM's M and K are multiples
// of 16.  Each GEMM output that a weight gradient needs is also written transposed
// (BF16, row length = rows of the batch), so every weight gradient
// dW[out][in] = dY^T X is again a K-major GEMM, split over K (the batch rows) with
// FP32 partials added in split order.  Parameters: one flat FP32 vector, per layer
// Wt[out][in] (row-major) then b[out]; BF16 copies of Wt (forward operand) and of W
// (its transpose, operand of the input gradients) are refreshed after every update.
// Every reduction runs in a fixed order, so training is bit-reproducible.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "lddmm_b200.h"
#include "tc_gemm.cuh"

using bf16 = __nv_bfloat16;
using namespace lddmm::tc;

namespace {

thread_local std::string g_ws_err;

void ws_err(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_ws_err = buf;
}

#define WCU(x)                                                                   \
  do {                                                                           \
    cudaError_t e_ = (x);                                                        \
    if (e_ != cudaSuccess) {                                                     \
      ws_err("CUDA error %s at %s:%d", cudaGetErrorString(e_), __FILE__, __LINE__); \
      return LDDMM_ERR_CUDA;                                                     \
    }                                                                            \
  } while (0)

constexpr int kTriIn = 16;   // 7 features, padded
constexpr int kTriH = 64;
constexpr int kPtIn = 80;    // 3 + 64, padded (the configured network, no local features)
constexpr int kMaxLocal = 27;   // nearest triangles per landmark: 3 + 64 + 7 k <= 256
constexpr float kLocalRel = 10.0f;  // scale of a neighbour's centre offset c_j - q_i
constexpr int kPtH = 256;
constexpr int kThreads = 256;

int round16(int n) { return (n + 15) / 16 * 16; }

struct Layer {
  int in, out;          // padded
  int in_real, out_real;
  size_t w_off, b_off;  // offsets in the flat parameter vector
  bf16 *Wt = nullptr;   // [out][in]
  bf16 *W = nullptr;    // [in][out]
};

// ------------------------------------------------------------------ kernels

// tri7 [B][Et][7] FP32 -> xt [B * Etp][16] BF16 and its transpose [16][B * Etp]
__global__ void tri_input_kernel(const float *tri7, int B, int Et, int Etp, bf16 *xt,
                                 bf16 *xtT) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long M = (long long)B * Etp;
  if (r >= M) return;
  const int p = (int)(r / Etp), e = (int)(r - (long long)p * Etp);
#pragma unroll
  for (int c = 0; c < kTriIn; ++c) {
    float v = 0.0f;
    if (e < Et && c < 7) v = tri7[((size_t)p * Et + e) * 7 + c];
    const bf16 h = __float2bfloat16_rn(v);
    xt[r * kTriIn + c] = h;
    xtT[(size_t)c * M + r] = h;
  }
}

// g[p][c] = max over the pair's Et real rows of h2 (lowest row wins ties); arg = row
__global__ void maxpool_kernel(const float *h2, int Et, int Etp, float *g, int *arg) {
  const int p = blockIdx.x, c = threadIdx.x & 63, part = threadIdx.x >> 6;  // 4 parts
  __shared__ float s_v[4][64];
  __shared__ int s_i[4][64];
  float best = -INFINITY;
  int bi = 0;
  for (int e = part; e < Et; e += 4) {
    const float v = h2[((size_t)p * Etp + e) * kTriH + c];
    if (v > best) {
      best = v;
      bi = e;
    }
  }
  s_v[part][c] = best;
  s_i[part][c] = bi;
  __syncthreads();
  if (part == 0) {
    for (int k = 1; k < 4; ++k)
      if (s_v[k][c] > best || (s_v[k][c] == best && s_i[k][c] < bi)) {
        best = s_v[k][c];
        bi = s_i[k][c];
      }
    g[p * kTriH + c] = best;
    arg[p * kTriH + c] = bi;
  }
}

// The k nearest target triangles of every source landmark: for pair p and landmark i,
// the indices of the k closest triangle centres in ascending order of the squared
// distance, computed in FP32 as ((cx - qx)^2 + (cy - qy)^2) + (cz - qz)^2 with every
// operation rounded (no contraction), ties to the lower index.  One warp per (pair,
// landmark): lane l keeps the sorted list of its k best among triangles l, l + 32, ...
// in shared memory, then the warp merges the 32 lists in k rounds of a (distance,
// index) argmin.  Requires k <= Et.
constexpr int kKnnWarps = 4;
__global__ void __launch_bounds__(kKnnWarps * 32)
    knn_kernel(const float *tri7, int B, int Et, const float *xyz, int N, int k, int *nbr) {
  __shared__ float s_d[kKnnWarps][kMaxLocal][32];
  __shared__ int s_i[kKnnWarps][kMaxLocal][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long item = (long long)blockIdx.x * kKnnWarps + warp;
  if (item >= (long long)B * N) return;  // warp-uniform
  const int p = (int)(item / N), i = (int)(item - (long long)p * N);
  const float qx = xyz[i * 3], qy = xyz[i * 3 + 1], qz = xyz[i * 3 + 2];
  const float *tp = tri7 + (size_t)p * Et * 7;
  float(*ld)[32] = s_d[warp];
  int(*li)[32] = s_i[warp];
  int cnt = 0;
  for (int j = lane; j < Et; j += 32) {
    const float dx = __fsub_rn(tp[j * 7], qx), dy = __fsub_rn(tp[j * 7 + 1], qy),
                dz = __fsub_rn(tp[j * 7 + 2], qz);
    const float d =
        __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    if (cnt < k || d < ld[cnt - 1][lane]) {
      // this lane's candidates come in increasing index, so an equal distance stays
      // behind the entries already kept
      int pos = cnt < k ? cnt : k - 1;
      while (pos > 0 && ld[pos - 1][lane] > d) {
        ld[pos][lane] = ld[pos - 1][lane];
        li[pos][lane] = li[pos - 1][lane];
        --pos;
      }
      ld[pos][lane] = d;
      li[pos][lane] = j;
      if (cnt < k) ++cnt;
    }
  }
  int h = 0;  // head of this lane's list
  for (int r = 0; r < k; ++r) {
    float bd = h < cnt ? ld[h][lane] : INFINITY;
    int bi = h < cnt ? li[h][lane] : 0x7fffffff;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float od = __shfl_xor_sync(0xffffffffu, bd, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (od < bd || (od == bd && oi < bi)) {
        bd = od;
        bi = oi;
      }
    }
    if (h < cnt && li[h][lane] == bi) ++h;  // indices are distinct: one lane advances
    if (lane == 0) nbr[item * k + r] = bi;
  }
}

// xp [B * Np][pt_in] = (q_i, g_p, local features, 0) and its transpose: here every
// column but the local features' (k neighbours x 7, written by local_input_kernel)
__global__ void point_input_kernel(const float *xyz, int N, int Np, int B, const float *g,
                                   int k, int pt_in, bf16 *xp, bf16 *xpT) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long M = (long long)B * Np;
  if (r >= M) return;
  const int p = (int)(r / Np), i = (int)(r - (long long)p * Np);
  const int lo = 3 + kTriH, hi = 3 + kTriH + 7 * k;
  for (int c = 0; c < pt_in; ++c) {
    if (c == lo) c = hi;  // the local columns
    if (c >= pt_in) break;
    float v = 0.0f;
    if (i < N) {
      if (c < 3) v = xyz[i * 3 + c];
      else if (c < 3 + kTriH) v = g[p * kTriH + c - 3];
    }
    const bf16 h = __float2bfloat16_rn(v);
    xp[r * pt_in + c] = h;
    xpT[(size_t)c * M + r] = h;
  }
}

// The local columns of xp / xpT: neighbour n of row r (thread n M + r, rows fastest, so
// the transposed writes coalesce) is the triangle's centre offset (c - q_i) * kLocalRel,
// unit normal and area * Et / (4 pi); zeros on padding rows
__global__ void local_input_kernel(const float *xyz, int N, int Np, int B, const float *tri7,
                                   int Et, const int *nbr, int k, int pt_in, bf16 *xp,
                                   bf16 *xpT) {
  const long long M = (long long)B * Np;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= M * k) return;
  const int n = (int)(idx / M);
  const long long r = idx - (long long)n * M;
  const int p = (int)(r / Np), i = (int)(r - (long long)p * Np);
  float v[7] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  if (i < N) {
    const int j = nbr[((size_t)p * N + i) * k + n];
    const float *t = tri7 + ((size_t)p * Et + j) * 7;
#pragma unroll
    for (int f = 0; f < 7; ++f) v[f] = t[f];
#pragma unroll
    for (int f = 0; f < 3; ++f) v[f] = __fmul_rn(__fsub_rn(v[f], xyz[i * 3 + f]), kLocalRel);
  }
  const int c0 = 3 + kTriH + 7 * n;
#pragma unroll
  for (int f = 0; f < 7; ++f) {
    const bf16 h = __float2bfloat16_rn(v[f]);
    xp[r * pt_in + c0 + f] = h;
    xpT[(size_t)(c0 + f) * M + r] = h;
  }
}

// dy = label_weight 2 (y - label / scale) / count (when label is given) + scale *
// dalpha[p][(t N + i) 3 + d] at column c = 3 t + d (when dalpha is given: the gradient
// of an outer loss with respect to the predicted momenta, alpha = scale y) on real rows /
// columns, 0 elsewhere; block partials of the squared error
__global__ void loss_kernel(const float *y, int ldy, const float *label, float inv_scale, int N,
                            int Np, int B, int n_out, int n_out_pad, float inv_count, bf16 *dy,
                            bf16 *dyT, double *part, float label_weight = 1.0f,
                            const double *dalpha = nullptr, float scale = 1.0f, int T = 0) {
  __shared__ double s[kThreads / 32];
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long M = (long long)B * Np;
  double sq = 0.0;
  if (idx < M * n_out_pad) {
    const long long r = idx / n_out_pad;
    const int c = (int)(idx - r * n_out_pad);
    const int p = (int)(r / Np), i = (int)(r - (long long)p * Np);
    float d = 0.0f;
    if (i < N && c < n_out) {
      if (label) {
        const float t = label[((size_t)p * N + i) * n_out + c] * inv_scale;
        const float e = y[r * ldy + c] - t;
        sq = (double)e * e;
        d = 2.0f * e * inv_count * label_weight;
      }
      if (dalpha) {
        const int t = c / 3, dd = c - 3 * (c / 3);
        d += scale * (float)dalpha[(size_t)p * T * N * 3 + ((size_t)t * N + i) * 3 + dd];
      }
    }
    const bf16 h = __float2bfloat16_rn(d);
    dy[r * n_out_pad + c] = h;
    dyT[(size_t)c * M + r] = h;
  }
  for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) t += s[w];
    part[blockIdx.x] = t;
  }
}

// out[c] = sum over the row of xT[c][0..M) (BF16), fixed order; one block per c
__global__ void rowsum_kernel(const bf16 *xT, long long M, float *out) {
  __shared__ float s[kThreads / 32];
  const bf16 *row = xT + (size_t)blockIdx.x * M;
  float acc = 0.0f;
  for (long long k = threadIdx.x; k < M; k += kThreads) acc += __bfloat162float(row[k]);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < kThreads / 32; ++w) t += s[w];
    out[blockIdx.x] = t;
  }
}

// pair sums of the first point layer's pre-activation gradient, then through the g
// columns of P1: dg[p][c] = sum_o (sum_{i of p} da1[p][i][o]) Wt_P1[o][3 + c];
// block per pair, threads over o
__global__ void dg_kernel(const bf16 *da1T, long long M, int Np, const float *wt_p1, int pt_in,
                          float *dg) {
  const int p = blockIdx.x;
  __shared__ float s_o[kPtH];
  for (int o = threadIdx.x; o < kPtH; o += blockDim.x) {
    const bf16 *row = da1T + (size_t)o * M + (size_t)p * Np;
    float a = 0.0f;
    for (int i = 0; i < Np; ++i) a += __bfloat162float(row[i]);
    s_o[o] = a;
  }
  __syncthreads();
  for (int c = threadIdx.x; c < kTriH; c += blockDim.x) {
    float a = 0.0f;
    for (int o = 0; o < kPtH; ++o) a = fmaf(s_o[o], wt_p1[o * pt_in + 3 + c], a);
    dg[p * kTriH + c] = a;
  }
}

// the max-pool's gradient: dh2 is zero except at each (pair, channel)'s argmax row
__global__ void unpool_kernel(const float *dg, const int *arg, int B, int Etp, long long M,
                              bf16 *dh2, bf16 *dh2T) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= B * kTriH) return;
  const int p = k / kTriH, c = k - p * kTriH;
  const long long r = (long long)p * Etp + arg[k];
  const bf16 h = __float2bfloat16_rn(dg[k]);
  dh2[r * kTriH + c] = h;
  dh2T[(size_t)c * M + r] = h;
}

// grad[i] = sum over splits of part[s][i], split order
__global__ void splitk_reduce_kernel(const float *part, int S, int n, float *grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float a = 0.0f;
  for (int s = 0; s < S; ++s) a += part[(size_t)s * n + i];
  grad[i] = a;
}

// Adam (Kingma & Ba), bias-corrected
__global__ void adam_kernel(float *w, const float *g, float *m, float *v, size_t n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// BF16 copies of a layer's Wt[out][in] and of its transpose W[in][out]
__global__ void weights_bf16_kernel(const float *wt, int out, int in, bf16 *Wt, bf16 *W) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= out * in) return;
  const int o = k / in, c = k - o * in;
  const bf16 h = __float2bfloat16_rn(wt[k]);
  Wt[k] = h;
  W[(size_t)c * out + o] = h;
}

// predictions -> momenta in the variable layout of each pair: a[p][(t N + i) 3 + d]
__global__ void predict_out_kernel(const float *y, int ldy, int N, int Np, int B, int T,
                                   double scale, double *alpha) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = (long long)T * N * 3;
  if (k >= per * B) return;
  const int p = (int)(k / per);
  const long long w = k - p * per;
  const int t = (int)(w / ((long long)N * 3));
  const int rem = (int)(w - (long long)t * N * 3);
  const int i = rem / 3, d = rem - i * 3;
  alpha[k] = scale * (double)y[((size_t)p * Np + i) * ldy + t * 3 + d];
}

}  // namespace

// ------------------------------------------------------------------- context

struct lddmm_ws {
  int N = 0, Np = 0, T = 0, n_out = 0, n_out_pad = 0, batch_max = 0, et_max = 0, etp_max = 0;
  float label_scale = 1.0f;
  int local_k = 0, pt_in = kPtIn;  // nearest triangles per landmark; point input width
  int *nbr = nullptr;              // [batch_max][N][local_k] of the last forward
  int fwd_pairs = 0, fwd_tris = 0;  // batch of the activations of the last prediction
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  Layer L[5];  // T1, T2, P1, P2, P3
  size_t n_params = 0;
  float *params = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
  int step = 0;
  float *xyz = nullptr;
  // activations, sized for batch_max pairs
  bf16 *xt = nullptr, *xtT = nullptr, *h1 = nullptr, *h1T = nullptr, *dh2 = nullptr,
       *dh2T = nullptr, *dh1T = nullptr;
  float *pre_h1 = nullptr, *h2 = nullptr, *g = nullptr, *dg = nullptr;
  int *arg = nullptr;
  bf16 *xp = nullptr, *xpT = nullptr, *a1 = nullptr, *a1T = nullptr, *a2 = nullptr,
       *a2T = nullptr, *dy = nullptr, *dyT = nullptr, *da2 = nullptr, *da2T = nullptr,
       *da1 = nullptr, *da1T = nullptr;
  float *pre_a1 = nullptr, *pre_a2 = nullptr, *y = nullptr, *part = nullptr;
  size_t part_cap = 0;
  double *loss_part = nullptr;
  size_t loss_cap = 0;
  unsigned int *err = nullptr;
  std::vector<void *> owned;
  ~lddmm_ws() {
    for (void *p : owned) cudaFree(p);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
  template <class X>
  cudaError_t alloc(X **p, size_t n) {
    *p = nullptr;
    cudaError_t e = cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(X));
    if (e == cudaSuccess) {
      owned.push_back(*p);
      e = cudaMemsetAsync(*p, 0, std::max<size_t>(n, 1) * sizeof(X), stream);
    }
    return e;
  }
};

namespace {

// host-side deterministic generator for the initial weights (splitmix64)
struct Rng {
  unsigned long long s;
  unsigned long long next() {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

cudaError_t refresh_bf16(lddmm_ws &w) {
  for (Layer &l : w.L) {
    const int n = l.out * l.in;
    weights_bf16_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, w.stream>>>(
        w.params + l.w_off, l.out, l.in, l.Wt, l.W);
  }
  return cudaGetLastError();
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime (the
// library does not link the driver library itself); null when unavailable.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    cudaGetLastError();
  });
  return fn;
}

// 2D TMA map of a K-major BF16 matrix (rows x K, row stride ld elements) read in boxes
// of 64 K-elements (128 bytes) x box_rows rows into the 128-byte swizzled layout;
// false when the operand does not meet TMA's rules (16-byte aligned base and row
// stride) or the encoder refuses it.
bool make_kmajor_map(CUtensorMap *m, const void *base, long long K, long long rows,
                     long long ld, int box_rows) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || ((uintptr_t)base & 15u) || (ld * 2) % 16 || K < 8 || rows < 1) return false;
  cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  cuuint32_t box[2] = {(cuuint32_t)kKC, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1u, 1u};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides,
             box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// 2D TMA map of a row-major FP32 output (rows x cols, row stride ld elements) written
// in 32 x 32 blocks through a 128-byte-swizzled staging buffer; false when the output
// does not meet TMA's rules (16-byte aligned base and row stride).
bool make_out_map(CUtensorMap *m, float *base, long long cols, long long rows, long long ld) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || ((uintptr_t)base & 15u) || (ld * 4) % 16 || cols < 4 || rows < 1) return false;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
  cuuint32_t box[2] = {32u, 32u};
  cuuint32_t es[2] = {1u, 1u};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Launches C = A . B^T on `st`.  One K split with K <= kResK (every layer's forward and
// input-gradient products): the warp-specialised TMA kernel, or the cp.async
// weight-resident kernel when TMA maps cannot be made for the operands; otherwise the
// per-tile kernel (split-K weight gradients).  The kernels' shared-memory limits are
// raised once per device.
cudaError_t launch_gemm(GemmArgs a, int splits, cudaStream_t st) {
  static std::atomic<bool> attr_set[64];  // zero-initialised; setting twice is harmless
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < 64 && !attr_set[dev].load()) {
    e = cudaFuncSetAttribute(gemm_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)gemm_smem_bytes(256));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(gemm_bf16_resident_kernel,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)gemm_resident_smem_bytes(256, kResK));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(gemm_bf16_ws_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)std::max(gemm_ws_smem_bytes(256, kResK, true),
                                             gemm_ws_smem_bytes(256, kResK, false)));
    if (e != cudaSuccess) return e;
    attr_set[dev].store(true);
  }
  if (a.k_split <= 0) a.k_split = (a.K + kKC - 1) / kKC * kKC;
  const int ntiles = (a.M + kTileM - 1) / kTileM;
  if (splits == 1 && a.K <= kResK && a.k_split >= a.K && a.N <= 256 && ntiles > 0) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = std::min(ntiles, std::max(sms, 1));
    CUtensorMap ma, mb, mc;
    std::memset(&mc, 0, sizeof(mc));
    if (make_kmajor_map(&ma, a.A, a.K, a.M, a.lda, kTileM) &&
        make_kmajor_map(&mb, a.B, a.K, a.N, a.ldb, a.N)) {
      // a plain FP32 output leaves through TMA stores
      const bool tma_store = a.out && a.epi == kEpiNone && !a.pre_out && !a.out_bf &&
                             !a.out_bt && make_out_map(&mc, a.out, a.n_valid, a.M, a.ldo);
      gemm_bf16_ws_kernel<<<grid, kWsThreads, gemm_ws_smem_bytes(a.N, a.K, tma_store), st>>>(
          a, ma, mb, mc, tma_store ? 1 : 0, gemm_ws_stages(a.N, a.K, tma_store));
    } else
      gemm_bf16_resident_kernel<<<grid, kGemmThreads, gemm_resident_smem_bytes(a.N, a.K), st>>>(a);
  } else {
    gemm_bf16_kernel<<<dim3(ntiles, splits), kGemmThreads, gemm_smem_bytes(a.N), st>>>(a);
  }
  return cudaGetLastError();
}

// C = A . B^T through the tensor-core GEMM (see tc_gemm.cuh)
cudaError_t gemm(lddmm_ws &w, GemmArgs a, int splits) {
  a.error = w.err;
  return launch_gemm(a, splits, w.stream);
}

GemmArgs fwd_args(const bf16 *A, long long lda, const Layer &l, long long M) {
  GemmArgs a = {};
  a.A = A;
  a.lda = lda;
  a.B = l.Wt;
  a.ldb = l.in;
  a.M = (int)M;
  a.N = l.out;
  a.K = l.in;
  a.n_valid = l.out;
  return a;
}

// dW (FP32, Wt layout) and db of a layer: dW = dY^T X, split over the batch rows
cudaError_t weight_grad(lddmm_ws &w, const Layer &l, const bf16 *dYT, const bf16 *XT,
                        long long M) {
  GemmArgs a = {};
  a.A = dYT;
  a.lda = M;
  a.B = XT;
  a.ldb = M;
  a.M = l.out;
  a.N = l.in;
  a.K = (int)M;
  a.n_valid = l.in;
  const int mt = (l.out + kTileM - 1) / kTileM;
  // about 2 CTAs per SM over all splits, each split a multiple of the staging chunk
  int splits = std::max(1, 296 / mt);
  long long ks = ((M + splits - 1) / splits + kKC - 1) / kKC * kKC;
  splits = (int)((M + ks - 1) / ks);
  if ((size_t)splits * l.out * l.in > w.part_cap) return cudaErrorInvalidValue;
  a.k_split = (int)ks;
  a.out = w.part;
  a.ldo = l.in;
  a.split_stride = (long long)l.out * l.in;
  cudaError_t e = gemm(w, a, splits);
  if (e != cudaSuccess) return e;
  const int n = l.out * l.in;
  splitk_reduce_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, w.stream>>>(
      w.part, splits, n, w.grad + l.w_off);
  rowsum_kernel<<<l.out, kThreads, 0, w.stream>>>(dYT, M, w.grad + l.b_off);
  return cudaGetLastError();
}

int check_batch(lddmm_ws &w, int B, int Et) {
  if (B < 1 || B > w.batch_max || Et < 1 || Et > w.et_max) {
    ws_err("batch of %d pairs x %d triangles outside the context's %d x %d", B, Et, w.batch_max,
           w.et_max);
    return LDDMM_ERR_ARG;
  }
  if (Et < w.local_k) {
    ws_err("%d target triangles, fewer than the %d nearest ones each landmark reads", Et,
           w.local_k);
    return LDDMM_ERR_ARG;
  }
  return 0;
}

// forward pass; returns through w.y [B * Np][n_out_pad]
// nbr_in: the batch's nearest triangles from lddmm_ws_neighbours, or nullptr (searched here)
int forward(lddmm_ws &w, const float *tri7, int B, int Et, const int *nbr_in = nullptr) {
  const int Etp = round16(Et);
  const long long Mt = (long long)B * Etp, Mp = (long long)B * w.Np;
  tri_input_kernel<<<(unsigned)((Mt + kThreads - 1) / kThreads), kThreads, 0, w.stream>>>(
      tri7, B, Et, Etp, w.xt, w.xtT);
  GemmArgs a = fwd_args(w.xt, kTriIn, w.L[0], Mt);
  a.epi = kEpiGelu;
  a.bias = w.params + w.L[0].b_off;
  a.pre_out = w.pre_h1;
  a.ld_pre_out = kTriH;
  a.out_bf = w.h1;
  a.ldb_out = kTriH;
  a.out_bt = w.h1T;
  a.ldt_out = Mt;
  WCU(gemm(w, a, 1));
  a = fwd_args(w.h1, kTriH, w.L[1], Mt);
  a.bias = w.params + w.L[1].b_off;
  a.out = w.h2;
  a.ldo = kTriH;
  WCU(gemm(w, a, 1));
  maxpool_kernel<<<B, 256, 0, w.stream>>>(w.h2, Et, Etp, w.g, w.arg);
  const int *nbr = nbr_in ? nbr_in : w.nbr;
  if (w.local_k > 0 && !nbr_in) {
    const long long items = (long long)B * w.N;
    knn_kernel<<<(unsigned)((items + kKnnWarps - 1) / kKnnWarps), kKnnWarps * 32, 0,
                 w.stream>>>(tri7, B, Et, w.xyz, w.N, w.local_k, w.nbr);
  }
  point_input_kernel<<<(unsigned)((Mp + kThreads - 1) / kThreads), kThreads, 0, w.stream>>>(
      w.xyz, w.N, w.Np, B, w.g, w.local_k, w.pt_in, w.xp, w.xpT);
  if (w.local_k > 0) {
    const long long n = Mp * w.local_k;
    local_input_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, w.stream>>>(
        w.xyz, w.N, w.Np, B, tri7, Et, nbr, w.local_k, w.pt_in, w.xp, w.xpT);
  }
  a = fwd_args(w.xp, w.pt_in, w.L[2], Mp);
  a.epi = kEpiGelu;
  a.bias = w.params + w.L[2].b_off;
  a.pre_out = w.pre_a1;
  a.ld_pre_out = kPtH;
  a.out_bf = w.a1;
  a.ldb_out = kPtH;
  a.out_bt = w.a1T;
  a.ldt_out = Mp;
  WCU(gemm(w, a, 1));
  a = fwd_args(w.a1, kPtH, w.L[3], Mp);
  a.epi = kEpiGelu;
  a.bias = w.params + w.L[3].b_off;
  a.pre_out = w.pre_a2;
  a.ld_pre_out = kPtH;
  a.out_bf = w.a2;
  a.ldb_out = kPtH;
  a.out_bt = w.a2T;
  a.ldt_out = Mp;
  WCU(gemm(w, a, 1));
  a = fwd_args(w.a2, kPtH, w.L[4], Mp);
  a.bias = w.params + w.L[4].b_off;
  a.out = w.y;
  a.ldo = w.n_out_pad;
  WCU(gemm(w, a, 1));
  return 0;
}

// output gradient (labels and / or dalpha, loss_kernel) + backward of the activations
// the last forward left: gradient in w.grad, loss (mean squared error, 0 without labels)
// in *loss
int backward(lddmm_ws &w, int B, int Et, const float *labels, float label_weight,
             const double *dalpha, double *loss) {
  const int Etp = round16(Et);
  const long long Mt = (long long)B * Etp, Mp = (long long)B * w.Np;
  const long long nl = Mp * w.n_out_pad;
  const unsigned nb = (unsigned)((nl + kThreads - 1) / kThreads);
  if (nb > w.loss_cap) {
    ws_err("loss partial buffer too small");
    return LDDMM_ERR_ARG;
  }
  const float inv_count = 1.0f / (float)((double)B * w.N * w.n_out);
  loss_kernel<<<nb, kThreads, 0, w.stream>>>(w.y, w.n_out_pad, labels, 1.0f / w.label_scale, w.N,
                                             w.Np, B, w.n_out, w.n_out_pad, inv_count, w.dy,
                                             w.dyT, w.loss_part, label_weight, dalpha,
                                             w.label_scale, w.T);
  // P3: weight gradient, then input gradient through gelu'(pre_a2)
  WCU(weight_grad(w, w.L[4], w.dyT, w.a2T, Mp));
  GemmArgs a = {};
  a.A = w.dy;
  a.lda = w.n_out_pad;
  a.B = w.L[4].W;
  a.ldb = w.L[4].out;
  a.M = (int)Mp;
  a.N = kPtH;
  a.K = w.L[4].out;
  a.n_valid = kPtH;
  a.epi = kEpiDGelu;
  a.pre_in = w.pre_a2;
  a.ld_pre_in = kPtH;
  a.out_bf = w.da2;
  a.ldb_out = kPtH;
  a.out_bt = w.da2T;
  a.ldt_out = Mp;
  WCU(gemm(w, a, 1));
  // P2
  WCU(weight_grad(w, w.L[3], w.da2T, w.a1T, Mp));
  a.A = w.da2;
  a.lda = kPtH;
  a.B = w.L[3].W;
  a.ldb = kPtH;
  a.K = kPtH;
  a.pre_in = w.pre_a1;
  a.out_bf = w.da1;
  a.out_bt = w.da1T;
  WCU(gemm(w, a, 1));
  // P1 (its input gradient is needed only in the g columns, summed over each pair)
  WCU(weight_grad(w, w.L[2], w.da1T, w.xpT, Mp));
  dg_kernel<<<B, 256, 0, w.stream>>>(w.da1T, Mp, w.Np, w.params + w.L[2].w_off, w.pt_in,
                                     w.dg);
  WCU(cudaMemsetAsync(w.dh2, 0, sizeof(bf16) * Mt * kTriH, w.stream));
  WCU(cudaMemsetAsync(w.dh2T, 0, sizeof(bf16) * Mt * kTriH, w.stream));
  unpool_kernel<<<(B * kTriH + kThreads - 1) / kThreads, kThreads, 0, w.stream>>>(
      w.dg, w.arg, B, Etp, Mt, w.dh2, w.dh2T);
  // T2, then T1 through gelu'(pre_h1)
  WCU(weight_grad(w, w.L[1], w.dh2T, w.h1T, Mt));
  a = GemmArgs{};
  a.A = w.dh2;
  a.lda = kTriH;
  a.B = w.L[1].W;
  a.ldb = kTriH;
  a.M = (int)Mt;
  a.N = kTriH;
  a.K = kTriH;
  a.n_valid = kTriH;
  a.epi = kEpiDGelu;
  a.pre_in = w.pre_h1;
  a.ld_pre_in = kTriH;
  a.out_bt = w.dh1T;
  a.ldt_out = Mt;
  WCU(gemm(w, a, 1));
  WCU(weight_grad(w, w.L[0], w.dh1T, w.xtT, Mt));
  std::vector<double> hp(nb);
  WCU(cudaMemcpyAsync(hp.data(), w.loss_part, sizeof(double) * nb, cudaMemcpyDeviceToHost,
                      w.stream));
  WCU(cudaStreamSynchronize(w.stream));
  unsigned int herr = 0;
  WCU(cudaMemcpy(&herr, w.err, sizeof(herr), cudaMemcpyDeviceToHost));
  if (herr) {
    ws_err("a tensor-core GEMM's barrier wait gave up");
    return LDDMM_ERR_TIMEOUT;
  }
  double s = 0.0;
  for (double x : hp) s += x;
  if (loss) *loss = s / ((double)B * w.N * w.n_out);
  return 0;
}

// forward + loss + backward: gradient in w.grad, loss (mean squared error) in *loss
int forward_backward(lddmm_ws &w, const float *tri7, int B, int Et, const float *labels,
                     double *loss, const int *nbr_in = nullptr) {
  int rc = forward(w, tri7, B, Et, nbr_in);
  if (rc) return rc;
  return backward(w, B, Et, labels, 1.0f, nullptr, loss);
}

void adam_step(lddmm_ws &w, double lr) {
  ++w.step;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, (float)w.step), c2 = 1.0f - std::pow(b2, (float)w.step);
  adam_kernel<<<(unsigned)((w.n_params + kThreads - 1) / kThreads), kThreads, 0, w.stream>>>(
      w.params, w.grad, w.m, w.v, w.n_params, (float)lr, b1, b2, 1e-8f, c1, c2);
}

}  // namespace

extern "C" const char *lddmm_ws_last_error(void) { return g_ws_err.c_str(); }

extern "C" int lddmm_ws_create_ex(int n_src, const double *src_nde, int time_steps,
                                  int batch_max, int tri_max, double label_scale,
                                  unsigned long long seed, int local_k, void *stream,
                                  lddmm_ws **out) {
  if (!out || n_src < 1 || !src_nde || time_steps < 1 || 3 * time_steps > 256 || batch_max < 1 ||
      tri_max < 1 || !(label_scale > 0) || local_k < 0 || local_k > kMaxLocal ||
      local_k > tri_max) {
    ws_err("lddmm_ws_create: bad arguments");
    return LDDMM_ERR_ARG;
  }
  *out = nullptr;
  auto *w = new lddmm_ws();
  std::unique_ptr<lddmm_ws> guard(w);
  w->N = n_src;
  w->Np = round16(n_src);
  w->T = time_steps;
  w->n_out = 3 * time_steps;
  w->n_out_pad = round16(w->n_out);
  w->batch_max = batch_max;
  w->et_max = tri_max;
  w->etp_max = round16(tri_max);
  w->label_scale = (float)label_scale;
  w->local_k = local_k;
  w->pt_in = round16(3 + kTriH + 7 * local_k);
  if (stream) {
    w->stream = (cudaStream_t)stream;
  } else {
    WCU(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking));
    w->own_stream = true;
  }
  const int dims[5][4] = {{kTriIn, kTriH, 7, kTriH},
                          {kTriH, kTriH, kTriH, kTriH},
                          {w->pt_in, kPtH, 3 + kTriH + 7 * local_k, kPtH},
                          {kPtH, kPtH, kPtH, kPtH},
                          {kPtH, w->n_out_pad, kPtH, w->n_out}};
  size_t off = 0;
  for (int k = 0; k < 5; ++k) {
    Layer &l = w->L[k];
    l.in = dims[k][0];
    l.out = dims[k][1];
    l.in_real = dims[k][2];
    l.out_real = dims[k][3];
    l.w_off = off;
    off += (size_t)l.out * l.in;
    l.b_off = off;
    off += l.out;
  }
  w->n_params = off;
  // initial weights: uniform +-1/sqrt(fan-in) on the real entries, zero padding
  std::vector<float> h(off, 0.0f);
  Rng rng{seed};
  for (const Layer &l : w->L) {
    const double a = 1.0 / std::sqrt((double)l.in_real);
    for (int o = 0; o < l.out_real; ++o) {
      for (int c = 0; c < l.in_real; ++c)
        h[l.w_off + (size_t)o * l.in + c] = (float)((2.0 * rng.uniform() - 1.0) * a);
      h[l.b_off + o] = (float)((2.0 * rng.uniform() - 1.0) * a);
    }
  }
  lddmm_ws &W = *w;
  WCU(W.alloc(&W.params, off));
  WCU(W.alloc(&W.grad, off));
  WCU(W.alloc(&W.m, off));
  WCU(W.alloc(&W.v, off));
  WCU(cudaMemcpyAsync(W.params, h.data(), sizeof(float) * off, cudaMemcpyHostToDevice, W.stream));
  for (Layer &l : W.L) {
    WCU(W.alloc(&l.Wt, (size_t)l.out * l.in));
    WCU(W.alloc(&l.W, (size_t)l.out * l.in));
  }
  std::vector<float> hx((size_t)n_src * 3);
  for (size_t k = 0; k < hx.size(); ++k) hx[k] = (float)src_nde[k];
  WCU(W.alloc(&W.xyz, hx.size()));
  WCU(cudaMemcpyAsync(W.xyz, hx.data(), sizeof(float) * hx.size(), cudaMemcpyHostToDevice,
                      W.stream));
  const size_t Mt = (size_t)batch_max * W.etp_max, Mp = (size_t)batch_max * W.Np;
  WCU(W.alloc(&W.xt, Mt * kTriIn));
  WCU(W.alloc(&W.xtT, Mt * kTriIn));
  WCU(W.alloc(&W.h1, Mt * kTriH));
  WCU(W.alloc(&W.h1T, Mt * kTriH));
  WCU(W.alloc(&W.pre_h1, Mt * kTriH));
  WCU(W.alloc(&W.h2, Mt * kTriH));
  WCU(W.alloc(&W.dh2, Mt * kTriH));
  WCU(W.alloc(&W.dh2T, Mt * kTriH));
  WCU(W.alloc(&W.dh1T, Mt * kTriH));
  WCU(W.alloc(&W.g, (size_t)batch_max * kTriH));
  WCU(W.alloc(&W.dg, (size_t)batch_max * kTriH));
  WCU(W.alloc(&W.arg, (size_t)batch_max * kTriH));
  WCU(W.alloc(&W.xp, Mp * W.pt_in));
  WCU(W.alloc(&W.xpT, Mp * W.pt_in));
  WCU(W.alloc(&W.nbr, (size_t)batch_max * n_src * std::max(local_k, 1)));
  for (bf16 **p : {&W.a1, &W.a1T, &W.a2, &W.a2T, &W.da2, &W.da2T, &W.da1, &W.da1T})
    WCU(W.alloc(p, Mp * kPtH));
  WCU(W.alloc(&W.pre_a1, Mp * kPtH));
  WCU(W.alloc(&W.pre_a2, Mp * kPtH));
  WCU(W.alloc(&W.y, Mp * W.n_out_pad));
  WCU(W.alloc(&W.dy, Mp * W.n_out_pad));
  WCU(W.alloc(&W.dyT, Mp * W.n_out_pad));
  W.part_cap = (size_t)300 * kPtH * kPtH;
  WCU(W.alloc(&W.part, W.part_cap));
  W.loss_cap = (Mp * W.n_out_pad + kThreads - 1) / kThreads;
  WCU(W.alloc(&W.loss_part, W.loss_cap));
  WCU(W.alloc(&W.err, 1));
  WCU(cudaFuncSetAttribute(gemm_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)gemm_smem_bytes(256)));
  WCU(refresh_bf16(W));
  WCU(cudaStreamSynchronize(W.stream));
  *out = guard.release();
  return 0;
}

extern "C" int lddmm_ws_create(int n_src, const double *src_nde, int time_steps, int batch_max,
                               int tri_max, double label_scale, unsigned long long seed,
                               void *stream, lddmm_ws **out) {
  return lddmm_ws_create_ex(n_src, src_nde, time_steps, batch_max, tri_max, label_scale, seed,
                            0, stream, out);
}

extern "C" void lddmm_ws_destroy(lddmm_ws *w) {
  if (!w) return;
  if (w->stream) cudaStreamSynchronize(w->stream);
  delete w;
}

extern "C" long long lddmm_ws_num_params(const lddmm_ws *w) { return w ? (long long)w->n_params : -1; }

extern "C" int lddmm_ws_params(lddmm_ws *w, float *host, int set) {
  if (!w || !host) {
    ws_err("lddmm_ws_params: bad arguments");
    return LDDMM_ERR_ARG;
  }
  if (set) {
    w->fwd_pairs = 0;
    WCU(cudaMemcpyAsync(w->params, host, sizeof(float) * w->n_params, cudaMemcpyHostToDevice,
                        w->stream));
    WCU(refresh_bf16(*w));
  } else {
    WCU(cudaMemcpyAsync(host, w->params, sizeof(float) * w->n_params, cudaMemcpyDeviceToHost,
                        w->stream));
  }
  WCU(cudaStreamSynchronize(w->stream));
  return 0;
}

extern "C" int lddmm_ws_grad(lddmm_ws *w, const float *d_tri7, int pairs, int tri_num,
                             const float *d_labels, float *grad_host, double *loss) {
  if (!w || !d_tri7 || !d_labels) {
    ws_err("lddmm_ws_grad: bad arguments");
    return LDDMM_ERR_ARG;
  }
  int rc = check_batch(*w, pairs, tri_num);
  if (rc) return rc;
  w->fwd_pairs = 0;
  rc = forward_backward(*w, d_tri7, pairs, tri_num, d_labels, loss);
  if (rc) return rc;
  if (grad_host) {
    WCU(cudaMemcpyAsync(grad_host, w->grad, sizeof(float) * w->n_params, cudaMemcpyDeviceToHost,
                        w->stream));
    WCU(cudaStreamSynchronize(w->stream));
  }
  return 0;
}

extern "C" int lddmm_ws_neighbours(lddmm_ws *w, const float *d_tri7, int pairs, int tri_num,
                                   int *d_nbr) {
  if (!w || !d_tri7 || !d_nbr || w->local_k < 1) {
    ws_err("lddmm_ws_neighbours: bad arguments (or a network without local features)");
    return LDDMM_ERR_ARG;
  }
  int rc = check_batch(*w, pairs, tri_num);
  if (rc) return rc;
  const long long items = (long long)pairs * w->N;
  knn_kernel<<<(unsigned)((items + kKnnWarps - 1) / kKnnWarps), kKnnWarps * 32, 0,
               w->stream>>>(d_tri7, pairs, tri_num, w->xyz, w->N, w->local_k, d_nbr);
  WCU(cudaGetLastError());
  WCU(cudaStreamSynchronize(w->stream));
  return 0;
}

extern "C" int lddmm_ws_train_step_nbr(lddmm_ws *w, const float *d_tri7, int pairs,
                                       int tri_num, const float *d_labels, const int *d_nbr,
                                       double lr, double *loss) {
  if (!w || !d_tri7 || !d_labels || !(lr > 0) || (w->local_k > 0 && !d_nbr)) {
    ws_err("lddmm_ws_train_step_nbr: bad arguments");
    return LDDMM_ERR_ARG;
  }
  int rc = check_batch(*w, pairs, tri_num);
  if (rc) return rc;
  w->fwd_pairs = 0;
  rc = forward_backward(*w, d_tri7, pairs, tri_num, d_labels, loss,
                        w->local_k > 0 ? d_nbr : nullptr);
  if (rc) return rc;
  adam_step(*w, lr);
  WCU(cudaGetLastError());
  WCU(refresh_bf16(*w));
  return 0;
}

extern "C" int lddmm_ws_train_step(lddmm_ws *w, const float *d_tri7, int pairs, int tri_num,
                                   const float *d_labels, double lr, double *loss) {
  if (!w || !d_tri7 || !d_labels || !(lr > 0)) {
    ws_err("lddmm_ws_train_step: bad arguments");
    return LDDMM_ERR_ARG;
  }
  int rc = check_batch(*w, pairs, tri_num);
  if (rc) return rc;
  w->fwd_pairs = 0;
  rc = forward_backward(*w, d_tri7, pairs, tri_num, d_labels, loss);
  if (rc) return rc;
  adam_step(*w, lr);
  WCU(cudaGetLastError());
  WCU(refresh_bf16(*w));
  return 0;
}

extern "C" int lddmm_ws_backward(lddmm_ws *w, const float *d_labels, double label_weight,
                                 const double *d_dalpha, double lr, float *grad_host,
                                 double *loss) {
  if (!w || !(lr >= 0) || (!d_labels && !d_dalpha) || (d_labels && !(label_weight >= 0))) {
    ws_err("lddmm_ws_backward: bad arguments");
    return LDDMM_ERR_ARG;
  }
  if (w->fwd_pairs < 1) {
    ws_err("lddmm_ws_backward: no lddmm_ws_predict since the last weight change");
    return LDDMM_ERR_ARG;
  }
  const int B = w->fwd_pairs, Et = w->fwd_tris;
  int rc = backward(*w, B, Et, d_labels, (float)label_weight, d_dalpha, loss);
  if (rc) return rc;
  if (grad_host) {
    WCU(cudaMemcpyAsync(grad_host, w->grad, sizeof(float) * w->n_params, cudaMemcpyDeviceToHost,
                        w->stream));
    WCU(cudaStreamSynchronize(w->stream));
  }
  if (lr > 0) {
    w->fwd_pairs = 0;
    adam_step(*w, lr);
    WCU(cudaGetLastError());
    WCU(refresh_bf16(*w));
  }
  return 0;
}

extern "C" int lddmm_ws_predict(lddmm_ws *w, const float *d_tri7, int pairs, int tri_num,
                                double *d_alpha) {
  if (!w || !d_tri7 || !d_alpha) {
    ws_err("lddmm_ws_predict: bad arguments");
    return LDDMM_ERR_ARG;
  }
  int rc = check_batch(*w, pairs, tri_num);
  if (rc) return rc;
  w->fwd_pairs = 0;
  rc = forward(*w, d_tri7, pairs, tri_num);
  if (rc) return rc;
  w->fwd_pairs = pairs;
  w->fwd_tris = tri_num;
  const long long n = (long long)pairs * w->T * w->N * 3;
  predict_out_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, w->stream>>>(
      w->y, w->n_out_pad, w->N, w->Np, pairs, w->T, (double)w->label_scale, d_alpha);
  WCU(cudaGetLastError());
  WCU(cudaStreamSynchronize(w->stream));
  unsigned int herr = 0;
  WCU(cudaMemcpy(&herr, w->err, sizeof(herr), cudaMemcpyDeviceToHost));
  if (herr) {
    ws_err("a tensor-core GEMM's barrier wait gave up");
    return LDDMM_ERR_TIMEOUT;
  }
  return 0;
}

extern "C" int lddmm_ws_gemm_bf16(const void *d_a, long long lda, const void *d_b, long long ldb,
                                  int m, int n, int k, float *d_c, long long ldc, void *stream) {
  if (!d_a || !d_b || !d_c || m < 1 || n < 16 || n > 256 || n % 16 || k < 16 || k % 16 ||
      lda % 8 || ldb % 8) {
    ws_err("lddmm_ws_gemm_bf16: n must be 16..256 in steps of 16, k a multiple of 16, "
           "leading dimensions multiples of 8");
    return LDDMM_ERR_ARG;
  }
  GemmArgs a = {};
  a.A = (const bf16 *)d_a;
  a.lda = lda;
  a.B = (const bf16 *)d_b;
  a.ldb = ldb;
  a.M = m;
  a.N = n;
  a.K = k;
  a.n_valid = n;
  a.k_split = (k + kKC - 1) / kKC * kKC;
  a.out = d_c;
  a.ldo = ldc;
  WCU(launch_gemm(a, 1, (cudaStream_t)stream));
  return 0;
}
