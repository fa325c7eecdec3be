// The three all-pairs sweeps of one objective evaluation and the small kernels
// around them.  Semantics follow Cpp/src/objgrd.cpp:26-90:
//   forward   v_t = K(q_t) a_t,  E += a_t . v_t,  q_{t+1} = q_t + dt v_t     (:45-59)
//   varifold  V(q_T), dV/dq_T; E = dt/2 E + w V; p = -w dV/dq                (:61-67)
//   backward  g_t = dt K(q_t)(a_t - p),
//             p  <- p - dt dqKernel(q_t, a_t/2 - p, a_t)                      (:69-87)
// The backward sweep fuses the kernel-matrix product and the dq sum of one step
// into a single pass over the pairs (they share q_t and the exponential).
#pragma once

#include "kernels.cuh"
#include "layout.h"
#include "sweep.cuh"

namespace lddmm {

constexpr int kGatherLanes = 8;  // lanes per vertex in gather_kernel

// ------------------------------------------------------------------- forward

template <int D, int ORDER>
struct ShootOp {
  static constexpr int JW = 2;
  static constexpr int NA = D;
  static constexpr bool kTileSum = true;
  static constexpr bool kTwoSets = false;
  struct IData {
    float x, y, z;
  };
  const PairDesc *pd;
  const int *act;
  const float4 *qs_t;  // scaled positions at t          [NPtot]
  const float4 *as_t;  // alpha_t (FP32)                 [NPtot]
  const double *q64_t; // positions at t (FP64)          [NPtot * D]
  double *q64_n;       // positions at t + 1
  float4 *qs_n;        // scaled positions at t + 1
  const double *x64;   // FP64 alpha (trial point), variable layout
  double *vlc64;       // optional velocity output       [NPtot * D]
  double *tile_part;   // energy partial per i-tile of this step
  int t;
  // bases for the persistent multi-step sweep (set_step derives the fields above)
  const float4 *qs0, *as0;
  double *q640, *vlc0, *reg0;
  int NP, ntile;  // ntile: stride of reg0 per step (row groups in the persistent sweep)

  __device__ void set_step(int tt) {
    t = tt;
    qs_t = qs0 + (size_t)tt * NP;
    as_t = as0 + (size_t)tt * NP;
    q64_t = q640 + (size_t)tt * NP * D;
    q64_n = q640 + (size_t)(tt + 1) * NP * D;
    qs_n = const_cast<float4 *>(qs0) + (size_t)(tt + 1) * NP;
    vlc64 = vlc0 ? vlc0 + (size_t)tt * NP * D : nullptr;
    tile_part = reg0 + (size_t)tt * ntile;
  }

  __device__ bool active(int p) const { return act[p] != 0; }
  __device__ int j_count(int p) const { return pd[p].Npad; }
  __device__ int i_count(int p) const { return pd[p].Npad; }  // rows (two-tile items)
  __device__ int set_boundary(int p) const { return pd[p].Npad; }
  __device__ void load_i(int p, int row, IData &I) const {
    const float4 q = __ldcg(&qs_t[pd[p].pt_off + row]);
    I.x = q.x;
    I.y = q.y;
    I.z = q.z;
  }
  __device__ void load_j(int p, int j, float4 (&w)[JW]) const {
    const int g = pd[p].pt_off + j;
    w[0] = __ldcg(&qs_t[g]);
    w[1] = __ldcg(&as_t[g]);
  }
  template <int SET>
  __device__ __forceinline__ void pair(const IData &I, const float4 (&w)[JW],
                                       float (&acc)[NA]) const {
    const float dx = I.x - w[0].x, dy = I.y - w[0].y;
    float nr2 = -dx * dx;
    nr2 = fmaf(-dy, dy, nr2);
    if (D == 3) {
      const float dz = I.z - w[0].z;
      nr2 = fmaf(-dz, dz, nr2);
    }
    const float K = DefKernelOf<D, ORDER>::type::val(nr2);
    acc[0] = fmaf(K, w[1].x, acc[0]);
    acc[1] = fmaf(K, w[1].y, acc[1]);
    if (D == 3) acc[D - 1] = fmaf(K, w[1].z, acc[D - 1]);
  }
  static constexpr bool kCull = false;
  // ---- packed form (sweep_packed_kernel): a lane's two rows in one FP32x2 operation,
  // bitwise the scalar pair() per row (x - y == x + (-y); the scalar nr2, built with
  // fma(-d, d, .), is exactly -(the sum of fma(d, d, .))).  Staged j point, each value
  // twice: (-qx,-qx,-qy,-qy) (-qz,-qz,ax,ax) (ay,ay,az,az); 2D: (-qx,-qx,-qy,-qy)
  // (ax,ax,ay,ay).
  static constexpr bool kPacked = true;
  static constexpr int JWP = (D == 3) ? 3 : 2;
  struct IData2 {
    float2 q[D];  // (row0, row1)
  };
  __device__ void load_i2(int p, int r0, int r1, IData2 &I) const {
    IData a, b;
    load_i(p, r0, a);
    load_i(p, r1, b);
    I.q[0] = make_float2(a.x, b.x);
    I.q[1] = make_float2(a.y, b.y);
    if (D == 3) I.q[D - 1] = make_float2(a.z, b.z);
  }
  __device__ void load_j2(int p, int j, float4 (&w)[JWP]) const {
    float4 v[JW];
    load_j(p, j, v);
    if (D == 3) {
      w[0] = make_float4(-v[0].x, -v[0].x, -v[0].y, -v[0].y);
      w[1] = make_float4(-v[0].z, -v[0].z, v[1].x, v[1].x);
      w[JWP - 1] = make_float4(v[1].y, v[1].y, v[1].z, v[1].z);
    } else {
      w[0] = make_float4(-v[0].x, -v[0].x, -v[0].y, -v[0].y);
      w[1] = make_float4(v[1].x, v[1].x, v[1].y, v[1].y);
    }
  }
  template <int SET>
  __device__ __forceinline__ void pair2(const IData2 &I, const float4 (&w)[JWP],
                                        float2 (&acc)[NA]) const {
    float2 mq[D], aj[D];
    mq[0] = make_float2(w[0].x, w[0].y);
    mq[1] = make_float2(w[0].z, w[0].w);
    if (D == 3) {
      mq[D - 1] = make_float2(w[1].x, w[1].y);
      aj[0] = make_float2(w[1].z, w[1].w);
      aj[1] = make_float2(w[JWP - 1].x, w[JWP - 1].y);
      aj[D - 1] = make_float2(w[JWP - 1].z, w[JWP - 1].w);
    } else {
      aj[0] = make_float2(w[1].x, w[1].y);
      aj[1] = make_float2(w[1].z, w[1].w);
    }
    const float2 dx = __fadd2_rn(I.q[0], mq[0]);
    float2 r2 = __fmul2_rn(dx, dx);
#pragma unroll
    for (int d = 1; d < D; ++d) {
      const float2 dd = __fadd2_rn(I.q[d], mq[d]);
      r2 = __ffma2_rn(dd, dd, r2);
    }
    const float2 K = make_float2(DefKernelOf<D, ORDER>::type::val(-r2.x),
                                 DefKernelOf<D, ORDER>::type::val(-r2.y));
#pragma unroll
    for (int d = 0; d < D; ++d) acc[d] = __ffma2_rn(K, aj[d], acc[d]);
  }
  // finalize operands (loaded before the row sums are complete): q_t and a_t of the row
  struct FData {
    double q[3], a[3];
  };
  __device__ void fin_load(int p, int row, FData &F) const {
    const PairDesc &P = pd[p];
    if (row >= P.N) return;
    const size_t g = (size_t)P.pt_off + row;
    const double *a = x64 + P.var_off + ((size_t)t * P.N + row) * D;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      F.q[d] = __ldcg(&q64_t[g * D + d]);
      F.a[d] = __ldcg(&a[d]);
    }
  }
  __device__ double finalize(int p, int row, const double (&v)[NA], const FData &F) const {
    const PairDesc &P = pd[p];
    if (row >= P.N) return 0.0;
    const size_t g = (size_t)P.pt_off + row;
    double e = 0.0, qn[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < D; ++d) {
      qn[d] = F.q[d] + P.dt * v[d];
      q64_n[g * D + d] = qn[d];
      e += F.a[d] * v[d];
      if (vlc64) vlc64[g * D + d] = v[d];
    }
    const double s = P.kscale;
    qs_n[g] = make_float4((float)(qn[0] * s), (float)(qn[1] * s), (float)(qn[2] * s), 0.0f);
    return e;
  }
  __device__ double finalize(int p, int row, const double (&v)[NA]) const {
    FData F;
    fin_load(p, row, F);
    return finalize(p, row, v, F);
  }
  __device__ void write_tile(int p, int tile, double v) const {
    tile_part[pd[p].itile_off + tile] = v;
  }
  __device__ void write_group(int p, int grp, double v) const {
    tile_part[pd[p].grp_off + grp] = v;
  }
};

// ------------------------------------------------------------------ backward
// j data staged as 12 floats (3D) or 8 floats (2D):
//   3D: (qx qy qz ux) (uy uz lx ly) (lz rx ry rz)     2D: (qx qy ux uy) (lx ly rx ry)
// with u = a - p (kernel-product operand), l = a/2 - p, r = a (dq operands).

template <int D, int ORDER>
struct AdjointOp {
  static constexpr int JW = (D == 3) ? 3 : 2;
  static constexpr int NA = 2 * D;
  static constexpr bool kTileSum = false;
  static constexpr bool kTwoSets = false;
  struct IData {
    float q[D], l[D], r[D];
  };
  const PairDesc *pd;
  const int *act;
  const float4 *qs_t;  // scaled positions at t
  const float4 *us_t;  // u_t = a_t - p
  const float4 *ls_t;  // l_t = a_t / 2 - p
  const float4 *as_t;  // r_t = a_t
  double *p64;         // adjoint state (FP64), updated in place
  const double *x64;   // FP64 alpha, variable layout
  double *g64;         // gradient output, variable layout (nullptr: none)
  float4 *us_n;        // u_{t-1} (written when t > 0)
  float4 *ls_n;        // l_{t-1}
  double *pdot64;      // optional raw dq output [NPtot * D] (standalone dq kernel)
  double *pst64 = nullptr;  // optional costate output p_{t+1}, variable layout
  int t;
  // bases for the persistent multi-step sweep
  const float4 *qs0, *as0;
  float4 *us0, *ls0;
  int NP;

  __device__ void set_step(int tt) {
    t = tt;
    qs_t = qs0 + (size_t)tt * NP;
    as_t = as0 + (size_t)tt * NP;
    us_t = us0 + (size_t)(tt & 1) * NP;
    ls_t = ls0 + (size_t)(tt & 1) * NP;
    us_n = tt > 0 ? us0 + (size_t)((tt - 1) & 1) * NP : nullptr;
    ls_n = tt > 0 ? ls0 + (size_t)((tt - 1) & 1) * NP : nullptr;
  }

  __device__ bool active(int p) const { return act[p] != 0; }
  __device__ int j_count(int p) const { return pd[p].Npad; }
  __device__ int i_count(int p) const { return pd[p].Npad; }  // rows (two-tile items)
  __device__ int set_boundary(int p) const { return pd[p].Npad; }
  __device__ void load_i(int p, int row, IData &I) const {
    const int g = pd[p].pt_off + row;
    const float4 q = __ldcg(&qs_t[g]), l = __ldcg(&ls_t[g]), r = __ldcg(&as_t[g]);
    I.q[0] = q.x; I.q[1] = q.y;
    I.l[0] = l.x; I.l[1] = l.y;
    I.r[0] = r.x; I.r[1] = r.y;
    if (D == 3) {
      I.q[D - 1] = q.z;
      I.l[D - 1] = l.z;
      I.r[D - 1] = r.z;
    }
  }
  __device__ void load_j(int p, int j, float4 (&w)[JW]) const {
    const int g = pd[p].pt_off + j;
    const float4 q = __ldcg(&qs_t[g]), u = __ldcg(&us_t[g]), l = __ldcg(&ls_t[g]),
                 r = __ldcg(&as_t[g]);
    if (D == 3) {
      w[0] = make_float4(q.x, q.y, q.z, u.x);
      w[1] = make_float4(u.y, u.z, l.x, l.y);
      w[JW - 1] = make_float4(l.z, r.x, r.y, r.z);
    } else {
      w[0] = make_float4(q.x, q.y, u.x, u.y);
      w[1] = make_float4(l.x, l.y, r.x, r.y);
    }
  }
  template <int SET>
  __device__ __forceinline__ void pair(const IData &I, const float4 (&w)[JW],
                                       float (&acc)[NA]) const {
    float qj[D], uj[D], lj[D], rj[D];
    if (D == 3) {
      qj[0] = w[0].x; qj[1] = w[0].y; qj[D - 1] = w[0].z;
      uj[0] = w[0].w; uj[1] = w[1].x; uj[D - 1] = w[1].y;
      lj[0] = w[1].z; lj[1] = w[1].w; lj[D - 1] = w[JW - 1].x;
      rj[0] = w[JW - 1].y; rj[1] = w[JW - 1].z; rj[D - 1] = w[JW - 1].w;
    } else {
      qj[0] = w[0].x; qj[1] = w[0].y;
      uj[0] = w[0].z; uj[1] = w[0].w;
      lj[0] = w[1].x; lj[1] = w[1].y;
      rj[0] = w[1].z; rj[1] = w[1].w;
    }
    float dq[D];
    float nr2 = 0.0f;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      dq[d] = I.q[d] - qj[d];
      nr2 = fmaf(-dq[d], dq[d], nr2);
    }
    float K, Wt;
    DefKernelOf<D, ORDER>::type::val_w(nr2, K, Wt);
    float lr = I.l[0] * rj[0];
#pragma unroll
    for (int d = 1; d < D; ++d) lr = fmaf(I.l[d], rj[d], lr);
#pragma unroll
    for (int d = 0; d < D; ++d) lr = fmaf(lj[d], I.r[d], lr);
    const float s = lr * Wt;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      acc[d] = fmaf(K, uj[d], acc[d]);
      acc[D + d] = fmaf(s, dq[d], acc[D + d]);
    }
  }
  static constexpr bool kCull = false;
  // ---- packed form (sweep_packed_kernel): a lane's two rows in one FP32x2 operation,
  // bitwise the scalar pair() per row (same operations in the same order; x - y is
  // computed as x + (-y), and nr2 as -(the sum of fma(d, d, .))).  Staged j point,
  // each value twice: -q, u, l, r (3D: 6 float4, 2D: 4).
  static constexpr bool kPacked = true;
  static constexpr int JWP = (D == 3) ? 6 : 4;
  struct IData2 {
    float2 q[D], l[D], r[D];  // (row0, row1)
  };
  __device__ void load_i2(int p, int r0, int r1, IData2 &I) const {
    IData a, b;
    load_i(p, r0, a);
    load_i(p, r1, b);
#pragma unroll
    for (int d = 0; d < D; ++d) {
      I.q[d] = make_float2(a.q[d], b.q[d]);
      I.l[d] = make_float2(a.l[d], b.l[d]);
      I.r[d] = make_float2(a.r[d], b.r[d]);
    }
  }
  __device__ void load_j2(int p, int j, float4 (&w)[JWP]) const {
    const int g = pd[p].pt_off + j;
    const float4 q = __ldcg(&qs_t[g]), u = __ldcg(&us_t[g]), l = __ldcg(&ls_t[g]),
                 r = __ldcg(&as_t[g]);
    // value k of the 4D-padded list (-q, u, l, r) sits at float pair k of w
    float v[4 * D];
    const float qq[3] = {q.x, q.y, q.z}, uu[3] = {u.x, u.y, u.z}, ll[3] = {l.x, l.y, l.z},
                rr[3] = {r.x, r.y, r.z};
#pragma unroll
    for (int d = 0; d < D; ++d) {
      v[d] = -qq[d];
      v[D + d] = uu[d];
      v[2 * D + d] = ll[d];
      v[3 * D + d] = rr[d];
    }
#pragma unroll
    for (int k = 0; k < JWP; ++k)
      w[k] = make_float4(v[2 * k], v[2 * k], v[2 * k + 1], v[2 * k + 1]);
  }
  template <int SET>
  __device__ __forceinline__ void pair2(const IData2 &I, const float4 (&w)[JWP],
                                        float2 (&acc)[NA]) const {
    float2 v[4 * D];
#pragma unroll
    for (int k = 0; k < JWP; ++k) {
      v[2 * k] = make_float2(w[k].x, w[k].y);
      v[2 * k + 1] = make_float2(w[k].z, w[k].w);
    }
    const float2 *mq = v, *uj = v + D, *lj = v + 2 * D, *rj = v + 3 * D;
    float2 dq[D];
    dq[0] = __fadd2_rn(I.q[0], mq[0]);
    float2 r2 = __fmul2_rn(dq[0], dq[0]);
#pragma unroll
    for (int d = 1; d < D; ++d) {
      dq[d] = __fadd2_rn(I.q[d], mq[d]);
      r2 = __ffma2_rn(dq[d], dq[d], r2);
    }
    float Kx, Wx, Ky, Wy;
    DefKernelOf<D, ORDER>::type::val_w(-r2.x, Kx, Wx);
    DefKernelOf<D, ORDER>::type::val_w(-r2.y, Ky, Wy);
    const float2 K = make_float2(Kx, Ky), Wt = make_float2(Wx, Wy);
    float2 lr = __fmul2_rn(I.l[0], rj[0]);
#pragma unroll
    for (int d = 1; d < D; ++d) lr = __ffma2_rn(I.l[d], rj[d], lr);
#pragma unroll
    for (int d = 0; d < D; ++d) lr = __ffma2_rn(lj[d], I.r[d], lr);
    const float2 sv = __fmul2_rn(lr, Wt);
#pragma unroll
    for (int d = 0; d < D; ++d) {
      acc[d] = __ffma2_rn(K, uj[d], acc[d]);
      acc[D + d] = __ffma2_rn(sv, dq[d], acc[D + d]);
    }
  }
  // finalize operands loaded before the row sums are complete: p of the row and, when
  // the next step's u / l are formed, a_{t-1} of the row
  struct FData {
    double p[3], a[3];
  };
  __device__ void fin_load(int p, int row, FData &F) const {
    const PairDesc &P = pd[p];
    if (row >= P.N) return;
    const size_t g = (size_t)P.pt_off + row;
#pragma unroll
    for (int d = 0; d < D; ++d) F.p[d] = __ldcg(&p64[g * D + d]);
    if (t > 0 && us_n) {
      const double *a = x64 + P.var_off + ((size_t)(t - 1) * P.N + row) * D;
#pragma unroll
      for (int d = 0; d < D; ++d) F.a[d] = __ldcg(&a[d]);
    }
  }
  __device__ double finalize(int p, int row, const double (&v)[NA], const FData &F) const {
    const PairDesc &P = pd[p];
    if (row >= P.N) return 0.0;
    const size_t g = (size_t)P.pt_off + row;
    double pn[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const double pdot = P.pd_fac * v[D + d];
      if (pdot64) pdot64[g * D + d] = pdot;
      if (g64) g64[P.var_off + ((size_t)t * P.N + row) * D + d] = P.dt * v[d];
      if (pst64) pst64[P.var_off + ((size_t)t * P.N + row) * D + d] = F.p[d];
      pn[d] = F.p[d] - P.dt * pdot;
      p64[g * D + d] = pn[d];
    }
    if (t > 0 && us_n) {
      double u[3] = {0.0, 0.0, 0.0}, l[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int d = 0; d < D; ++d) {
        u[d] = F.a[d] - pn[d];
        l[d] = 0.5 * F.a[d] - pn[d];
      }
      us_n[g] = make_float4((float)u[0], (float)u[1], (float)u[2], 0.0f);
      ls_n[g] = make_float4((float)l[0], (float)l[1], (float)l[2], 0.0f);
    }
    return 0.0;
  }
  __device__ double finalize(int p, int row, const double (&v)[NA]) const {
    FData F;
    fin_load(p, row, F);
    return finalize(p, row, v, F);
  }
  __device__ void write_tile(int, int, double) const {}
  __device__ void write_group(int, int, double) const {}
};

// ------------------------------------------------------------------ varifold
// Deformed element i against every deformed (DD) and target (DT) element j:
//   value   V_i   = a_i (S_DD + 2 S_DT),  S = sum k(c) b(ang) w_j
//   centre  dc_i  = 2 a_i dc_fac sum kw(c) b w_j dc_scaled
//   normal  dd_i  = f (sum k w_j b'(ang) n_j + n_i sum k w_j (b - ang b'))
// with signed weights w_j = +a_j (deformed) / -a_j (target), f = 1 in 3D, 2 in 2D.
// These are dqVf_Kernel's sums (Cpp/src/varifold3D.cpp:259-332,
// Cpp/src/varifold2D.cpp:245-310) with grassmanFunction's derivative expanded: for
// the unnormalised normal N (|N| = 2 a_i in 3D, a_i in 2D) its 1/|N| cancels the
// a_i / (2 a_i) and the area derivative 0.5 n (3D) / n (2D).
//
// Centres are carried as double-single pairs (hi + lo, both FP32) so the centre
// difference (hi_i - hi_j) + (lo_i - lo_j) is accurate to an ulp of the difference
// itself: near convergence V and dV/dq are small differences of the DD and DT sums,
// and a plain FP32 rounding of the centres (relative 1e-6 on neighbour distances)
// would dominate their error.
// j data, 3D: (chi.xyz, w) (n.xyz, clo.x) (clo.y, clo.z, -, -)
//         2D: (chi.xy, clo.xy) (n.xy, w, -)
// Accumulators: 0 S_DD, 1 S_DT, 2.. A (D), 2+D.. C (D), [2+2D B for non-Binet].

template <int D, char CT, char DT>
struct VarifoldOp {
  static constexpr bool kBinet = (DT == 'B');
  static constexpr int JW = (D == 3) ? 3 : 2;
  static constexpr int NA = 2 + 2 * D + (kBinet ? 0 : 1);
  static constexpr bool kTileSum = true;
  static constexpr bool kTwoSets = true;
  struct IData {
    float ch[D], cl[D], n[D];
  };
  const PairDesc *pd;
  const int *act;
  const float4 *ec, *en;  // deformed: scaled centre hi + area, normal + centre lo.x
  const float4 *el;       // deformed: centre lo (xyz)
  const float4 *tc, *tn, *tl;  // target: same with weight -area
  const double *e64;      // deformed (n.xyz, area) FP64              [EDtot * 4]
  double *dcdd;           // out: dc (D), dd (D) per deformed element [EDtot * 2D]
  double *tile_part;      // varifold value per element tile
  float ow2;              // 2 / dirKnlWidth^2 (Gaussian direction kernels)
  // Distance culling (Gaussian centre kernel only): bounding boxes (lo, hi) of the
  // scaled centres of every 32-element block, deformed (dbb, per EDtot / 32) and
  // target (tbb, per ETtot / 32).  A 32-column block whose box is farther than
  // kCullR2 (scaled squared distance x^2) from the row tile's box is skipped: there
  // k = 2^-x^2 < 2^-64 and its derivative factor x 2^-x^2 <= 8 2^-64, while every
  // direction factor is at most 1 in magnitude.  Each skipped value term is thus below
  // 2^-64 of its pair weight (the product of the two areas) and each skipped gradient
  // term below 2^-61 of its pair weight times the kernel's derivative scale, far
  // below the FP32 resolution of the varifold value (whose deformed-deformed part
  // holds every element's own term, k = 1) and of its gradient.
  const float4 *dbb, *tbb;
  static constexpr bool kCull = (CT == 'G');
  static constexpr float kCullR2 = 64.0f;
  __device__ void row_box(int p, int tile, float (&bx)[6]) const {
    const int b = pd[p].el_off / 32 + 2 * tile;
    const float4 l0 = dbb[2 * b], h0 = dbb[2 * b + 1], l1 = dbb[2 * b + 2], h1 = dbb[2 * b + 3];
    bx[0] = fminf(l0.x, l1.x); bx[1] = fminf(l0.y, l1.y); bx[2] = fminf(l0.z, l1.z);
    bx[3] = fmaxf(h0.x, h1.x); bx[4] = fmaxf(h0.y, h1.y); bx[5] = fmaxf(h0.z, h1.z);
  }
  // true when every column of the aligned 32-column block sb of pair p's j range
  // (deformed blocks, then target blocks: Edpad is a multiple of 64) is beyond the
  // cut-off from the row box rb; an empty box (padding) gives infinite gaps
  __device__ __forceinline__ bool far(int p, const float *rb, int sb) const {
    const PairDesc &P = pd[p];
    const int db = P.Edpad / 32;
    const float4 *bx = sb < db ? dbb + 2 * (P.el_off / 32 + sb) : tbb + 2 * (P.tg_off / 32 + sb - db);
    const float4 lo = bx[0], hi = bx[1];
    const float gx = fmaxf(0.0f, fmaxf(lo.x - rb[3], rb[0] - hi.x));
    const float gy = fmaxf(0.0f, fmaxf(lo.y - rb[4], rb[1] - hi.y));
    const float gz = fmaxf(0.0f, fmaxf(lo.z - rb[5], rb[2] - hi.z));
    return fmaf(gz, gz, fmaf(gy, gy, gx * gx)) > kCullR2;
  }

  __device__ bool active(int p) const { return act[p] != 0; }
  __device__ int j_count(int p) const { return pd[p].Edpad + pd[p].Etpad; }
  __device__ int set_boundary(int p) const { return pd[p].Edpad; }
  __device__ void load_i(int p, int row, IData &I) const {
    const int g = pd[p].el_off + row;
    const float4 c = ec[g], n = en[g], l = el[g];
    I.ch[0] = c.x; I.ch[1] = c.y;
    I.cl[0] = l.x; I.cl[1] = l.y;
    I.n[0] = n.x; I.n[1] = n.y;
    if (D == 3) {
      I.ch[D - 1] = c.z;
      I.cl[D - 1] = l.z;
      I.n[D - 1] = n.z;
    }
  }
  __device__ void load_j(int p, int j, float4 (&w)[JW]) const {
    const PairDesc &P = pd[p];
    float4 c, n, l;
    if (j < P.Edpad) {
      c = __ldcg(&ec[P.el_off + j]);
      n = __ldcg(&en[P.el_off + j]);
      l = __ldcg(&el[P.el_off + j]);
    } else {
      c = __ldcg(&tc[P.tg_off + j - P.Edpad]);
      n = __ldcg(&tn[P.tg_off + j - P.Edpad]);
      l = __ldcg(&tl[P.tg_off + j - P.Edpad]);
    }
    if (D == 3) {
      w[0] = c;
      w[1] = make_float4(n.x, n.y, n.z, l.x);
      w[JW - 1] = make_float4(l.y, l.z, 0.0f, 0.0f);
    } else {
      w[0] = make_float4(c.x, c.y, l.x, l.y);
      w[1] = make_float4(n.x, n.y, c.w, 0.0f);
    }
  }
  template <int SET>
  __device__ __forceinline__ void pair(const IData &I, const float4 (&w)[JW],
                                       float (&acc)[NA]) const {
    float chj[3], clj[3], nj[3], wt;
    if (D == 3) {
      chj[0] = w[0].x; chj[1] = w[0].y; chj[2] = w[0].z; wt = w[0].w;
      nj[0] = w[1].x; nj[1] = w[1].y; nj[2] = w[1].z;
      clj[0] = w[1].w; clj[1] = w[JW - 1].x; clj[2] = w[JW - 1].y;
    } else {
      chj[0] = w[0].x; chj[1] = w[0].y; clj[0] = w[0].z; clj[1] = w[0].w;
      nj[0] = w[1].x; nj[1] = w[1].y; wt = w[1].z;
      chj[2] = clj[2] = nj[2] = 0.0f;
    }
    float dc[D];
    float nr2 = 0.0f, ang = 0.0f;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      dc[d] = (I.ch[d] - chj[d]) + (I.cl[d] - clj[d]);
      nr2 = fmaf(-dc[d], dc[d], nr2);
      ang = fmaf(I.n[d], nj[d], ang);
    }
    float k, kg;
    CenKernel<CT>::val_w(nr2, k, kg);
    const float kw = k * wt;
    if (kBinet) {
      const float t1 = kw * ang;  // k w b'/2
      const float tb = t1 * ang;  // k w b
      acc[SET] += tb;
      const float cg_ = (CT == 'G') ? tb : tb * k;  // kg w b
#pragma unroll
      for (int d = 0; d < D; ++d) {
        acc[2 + d] = fmaf(t1, nj[d], acc[2 + d]);
        acc[2 + D + d] = fmaf(cg_, dc[d], acc[2 + D + d]);
      }
    } else {
      float b, db;
      DirKernel<DT>::val_d(ang, ow2, b, db);
      const float tb = kw * b;
      const float td = kw * db;
      acc[SET] += tb;
      const float cg_ = (CT == 'G') ? tb : tb * k;
#pragma unroll
      for (int d = 0; d < D; ++d) {
        acc[2 + d] = fmaf(td, nj[d], acc[2 + d]);
        acc[2 + D + d] = fmaf(cg_, dc[d], acc[2 + D + d]);
      }
      acc[NA - 1] = fmaf(-ang, td, acc[NA - 1] + tb);
    }
  }
  // ---- packed form (sweep_packed_kernel): a lane's two rows in one FP32x2 operation.
  // Staged j point: the values -ch, -cl, n, w each stored twice:
  //   3D: (-chx,-chx,-chy,-chy) (-chz,-chz,-clx,-clx) (-cly,-cly,-clz,-clz)
  //       (nx,nx,ny,ny) (nz,nz,w,w)
  //   2D: (-chx,-chx,-chy,-chy) (-clx,-clx,-cly,-cly) (nx,nx,ny,ny) (w,w,-,-)
  static constexpr bool kPacked = true;
  static constexpr int JWP = (D == 3) ? 5 : 4;
  struct IData2 {
    float2 ch[D], cl[D], n[D];  // (row0, row1)
  };
  __device__ void load_i2(int p, int r0, int r1, IData2 &I) const {
    IData a, b;
    load_i(p, r0, a);
    load_i(p, r1, b);
#pragma unroll
    for (int d = 0; d < D; ++d) {
      I.ch[d] = make_float2(a.ch[d], b.ch[d]);
      I.cl[d] = make_float2(a.cl[d], b.cl[d]);
      I.n[d] = make_float2(a.n[d], b.n[d]);
    }
  }
  __device__ void load_j2(int p, int j, float4 (&w)[JWP]) const {
    float4 v[JW];
    load_j(p, j, v);
    if (D == 3) {
      // v: (chx chy chz wt) (nx ny nz clx) (cly clz - -)
      w[0] = make_float4(-v[0].x, -v[0].x, -v[0].y, -v[0].y);
      w[1] = make_float4(-v[0].z, -v[0].z, -v[1].w, -v[1].w);
      w[2] = make_float4(-v[JW - 1].x, -v[JW - 1].x, -v[JW - 1].y, -v[JW - 1].y);
      w[3] = make_float4(v[1].x, v[1].x, v[1].y, v[1].y);
      w[JWP - 1] = make_float4(v[1].z, v[1].z, v[0].w, v[0].w);
    } else {
      // v: (chx chy clx cly) (nx ny wt -)
      w[0] = make_float4(-v[0].x, -v[0].x, -v[0].y, -v[0].y);
      w[1] = make_float4(-v[0].z, -v[0].z, -v[0].w, -v[0].w);
      w[2] = make_float4(v[1].x, v[1].x, v[1].y, v[1].y);
      w[JWP - 1] = make_float4(v[1].z, v[1].z, 0.0f, 0.0f);
    }
  }
  template <int SET>
  __device__ __forceinline__ void pair2(const IData2 &I, const float4 (&w)[JWP],
                                        float2 (&acc)[NA]) const {
    float2 mch[D], mcl[D], nj[D], wt;
    if (D == 3) {
      mch[0] = make_float2(w[0].x, w[0].y); mch[1] = make_float2(w[0].z, w[0].w);
      mch[D - 1] = make_float2(w[1].x, w[1].y);
      mcl[0] = make_float2(w[1].z, w[1].w); mcl[1] = make_float2(w[2].x, w[2].y);
      mcl[D - 1] = make_float2(w[2].z, w[2].w);
      nj[0] = make_float2(w[3].x, w[3].y); nj[1] = make_float2(w[3].z, w[3].w);
      nj[D - 1] = make_float2(w[JWP - 1].x, w[JWP - 1].y);
      wt = make_float2(w[JWP - 1].z, w[JWP - 1].w);
    } else {
      mch[0] = make_float2(w[0].x, w[0].y); mch[1] = make_float2(w[0].z, w[0].w);
      mcl[0] = make_float2(w[1].x, w[1].y); mcl[1] = make_float2(w[1].z, w[1].w);
      nj[0] = make_float2(w[2].x, w[2].y); nj[1] = make_float2(w[2].z, w[2].w);
      wt = make_float2(w[JWP - 1].x, w[JWP - 1].y);
    }
    // the scalar pair() computes nr2 = sum fma(-dc, dc, .) = -r2 exactly
    float2 dc[D], r2 = make_float2(0.0f, 0.0f), ang = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int d = 0; d < D; ++d) {
      dc[d] = __fadd2_rn(__fadd2_rn(I.ch[d], mch[d]), __fadd2_rn(I.cl[d], mcl[d]));
      r2 = __ffma2_rn(dc[d], dc[d], r2);
      ang = __ffma2_rn(I.n[d], nj[d], ang);
    }
    float kx, ky, gx, gy;
    CenKernel<CT>::val_w(-r2.x, kx, gx);
    CenKernel<CT>::val_w(-r2.y, ky, gy);
    const float2 k = make_float2(kx, ky);
    const float2 kw = __fmul2_rn(k, wt);
    if (kBinet) {
      const float2 t1 = __fmul2_rn(kw, ang);  // k w b'/2
      const float2 tb = __fmul2_rn(t1, ang);  // k w b
      acc[SET] = __fadd2_rn(acc[SET], tb);
      const float2 cg_ = (CT == 'G') ? tb : __fmul2_rn(tb, k);  // kg w b
#pragma unroll
      for (int d = 0; d < D; ++d) {
        acc[2 + d] = __ffma2_rn(t1, nj[d], acc[2 + d]);
        acc[2 + D + d] = __ffma2_rn(cg_, dc[d], acc[2 + D + d]);
      }
    } else {
      float bx, dbx, by, dby;
      DirKernel<DT>::val_d(ang.x, ow2, bx, dbx);
      DirKernel<DT>::val_d(ang.y, ow2, by, dby);
      const float2 tb = __fmul2_rn(kw, make_float2(bx, by));
      const float2 td = __fmul2_rn(kw, make_float2(dbx, dby));
      acc[SET] = __fadd2_rn(acc[SET], tb);
      const float2 cg_ = (CT == 'G') ? tb : __fmul2_rn(tb, k);
#pragma unroll
      for (int d = 0; d < D; ++d) {
        acc[2 + d] = __ffma2_rn(td, nj[d], acc[2 + d]);
        acc[2 + D + d] = __ffma2_rn(cg_, dc[d], acc[2 + D + d]);
      }
      acc[NA - 1] = __ffma2_rn(make_float2(-ang.x, -ang.y), td,
                               __fadd2_rn(acc[NA - 1], tb));
    }
  }
  __device__ double finalize(int p, int row, const double (&v)[NA]) const {
    const PairDesc &P = pd[p];
    if (row >= P.Ed) return 0.0;
    const size_t g = (size_t)P.el_off + row;
    const double *e = e64 + g * 4;
    const double ai = e[3];
    const double fac = (D == 3) ? 1.0 : 2.0;
    double A[3], B;
    if (kBinet) {
      // b' = 2 ang, b - ang b' = -ang^2: A = 2 sum t1 n_j, B = -(S_DD + S_DT)
      for (int d = 0; d < D; ++d) A[d] = 2.0 * v[2 + d];
      B = -(v[0] + v[1]);
    } else {
      for (int d = 0; d < D; ++d) A[d] = v[2 + d];
      B = v[NA - 1];
    }
    double *o = dcdd + g * (2 * D);
#pragma unroll
    for (int d = 0; d < D; ++d) {
      o[d] = 2.0 * ai * P.dc_fac * v[2 + D + d];
      o[D + d] = fac * (A[d] + B * e[d]);
    }
    return ai * (v[0] + 2.0 * v[1]);
  }
  __device__ void write_tile(int p, int tile, double v) const {
    tile_part[pd[p].etile_off + tile] = v;
  }
};

// --------------------------------------------------------- per-element kernels

// landmarksToVarifoldKernel (Cpp/src/varifold3D.cpp:8-39, varifold2D.cpp:8-32) for
// one element, in FP64 from the final positions: centre (double-single, scaled), unit
// normal / tangent and area / length; writes the FP32 sweep operands and FP64 copies.
// cf: the scaled centre in FP32, for the block's bounding box.
template <int D>
__device__ __forceinline__ void geometry_element(const PairDesc &P, int4 ev, int g,
                                                 const double *__restrict__ q64, float4 *ec,
                                                 float4 *en, float4 *el, double *e64,
                                                 float (&cf)[3]) {
  double c[3] = {0, 0, 0}, n[3] = {0, 0, 0}, a;
  if (D == 3) {
    const double *q0 = q64 + (size_t)ev.x * 3, *q1 = q64 + (size_t)ev.y * 3,
                 *q2 = q64 + (size_t)ev.z * 3;
    double u[3], w[3];
    for (int d = 0; d < 3; ++d) {
      c[d] = (q0[d] + q1[d] + q2[d]) / 3.0;
      u[d] = q1[d] - q0[d];
      w[d] = q2[d] - q0[d];
    }
    n[0] = u[1] * w[2] - u[2] * w[1];
    n[1] = -u[0] * w[2] + u[2] * w[0];
    n[2] = u[0] * w[1] - u[1] * w[0];
    const double len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    for (int d = 0; d < 3; ++d) n[d] /= len;
    a = 0.5 * len;
  } else {
    const double *q0 = q64 + (size_t)ev.x * 2, *q1 = q64 + (size_t)ev.y * 2;
    for (int d = 0; d < 2; ++d) {
      c[d] = 0.5 * (q0[d] + q1[d]);
      n[d] = q1[d] - q0[d];
    }
    const double len = sqrt(n[0] * n[0] + n[1] * n[1]);
    n[0] /= len;
    n[1] /= len;
    a = len;
  }
  const double s = P.cscale;
  float hi[3], lo[3];
  for (int d = 0; d < 3; ++d) {
    const double x = c[d] * s;
    hi[d] = (float)x;
    lo[d] = (float)(x - (double)hi[d]);
  }
  ec[g] = make_float4(hi[0], hi[1], hi[2], (float)a);
  en[g] = make_float4((float)n[0], (float)n[1], (float)n[2], 0.0f);
  el[g] = make_float4(lo[0], lo[1], lo[2], 0.0f);
  double *e = e64 + (size_t)g * 4;
  e[0] = n[0];
  e[1] = n[1];
  e[2] = n[2];
  e[3] = a;
  // a non-finite centre, normal or weight makes every pair of the element non-finite
  // in the all-pairs sums: flagged by a NaN centre, so that its block is never culled
  const bool fin = isfinite(c[0] * s) && isfinite(c[1] * s) && isfinite(c[2] * s) &&
                   isfinite(n[0]) && isfinite(n[1]) && isfinite(n[2]) && isfinite(a);
#pragma unroll
  for (int d = 0; d < 3; ++d) cf[d] = fin ? hi[d] + lo[d] : NAN;
}

template <int D>
__global__ void geometry_kernel(const PairDesc *__restrict__ pd, const int *__restrict__ act,
                                const int4 *__restrict__ elm, int n_elm,
                                const double *__restrict__ q64, float4 *ec, float4 *en,
                                float4 *el, double *e64, float4 *bbox) {
  pdl_wait();
  pdl_trigger();
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int4 ev = g < n_elm ? elm[g] : make_int4(0, 0, 0, -1);
  const bool live = ev.w >= 0 && act[ev.w];
  float cf[3] = {0.0f, 0.0f, 0.0f};
  if (live) geometry_element<D>(pd[ev.w], ev, g, q64, ec, en, el, e64, cf);
  // bounding box of the scaled centres of the warp's 32 elements (one block of one
  // pair: pairs are padded to multiples of 64), for the varifold sweep's distance test.
  // A block of padding gets an empty box; an element flagged non-finite widens the box
  // to all of space, so that no block holding it is ever skipped.
  if (bbox && (g - threadIdx.x % 32) < n_elm) {
    const bool fin = isfinite(cf[0]) && isfinite(cf[1]) && isfinite(cf[2]);
    float lo[3], hi[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      lo[d] = live ? (fin ? cf[d] : -INFINITY) : INFINITY;
      hi[d] = live ? (fin ? cf[d] : INFINITY) : -INFINITY;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], off));
        hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], off));
      }
    }
    if (threadIdx.x % 32 == 0) {
      bbox[2 * (g / 32)] = make_float4(lo[0], lo[1], lo[2], 0.0f);
      bbox[2 * (g / 32) + 1] = make_float4(hi[0], hi[1], hi[2], 0.0f);
    }
  }
}

// dqVfdGatherKernel (Cpp/src/varifold3D.cpp:359-391, varifold2D.cpp:337-359) fused
// with the start of the adjoint (Cpp/src/objgrd.cpp:67): p = -w dV/dq, and the
// operands u, l of the first backward step.  One thread per (padded) vertex.
template <int D>
__global__ void gather_kernel(const PairDesc *__restrict__ pd, const int *__restrict__ act,
                              const int *__restrict__ pt_pair, int n_pt,
                              const int *__restrict__ adj_ptr, const int4 *__restrict__ adj,
                              const double *__restrict__ dcdd, const double *__restrict__ q64T,
                              const double *__restrict__ x64, double *p64, float4 *us_n,
                              float4 *ls_n, double *dq_out, int T) {
  pdl_wait();
  pdl_trigger();
  // kGatherLanes lanes per vertex, each over every kGatherLanes-th adjacent element, so
  // the element loads of a vertex are in flight together; the lanes' sums are then
  // combined by a fixed shuffle tree (deterministic)
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) / kGatherLanes;
  const int sub = threadIdx.x % kGatherLanes;
  int p = -1;
  if (g < n_pt) p = pt_pair[g];
  const bool live = p >= 0 && act[p];
  double acc[3] = {0.0, 0.0, 0.0};
  if (live) {
    const int k1 = adj_ptr[g + 1];
    for (int k = adj_ptr[g] + sub; k < k1; k += kGatherLanes) {
      const int4 e = adj[k];
      const double *o = dcdd + (size_t)e.x * (2 * D);
      if (D == 3) {
        const double *qa = q64T + (size_t)e.y * 3, *qb = q64T + (size_t)e.z * 3;
        const double ab[3] = {qa[0] - qb[0], qa[1] - qb[1], qa[2] - qb[2]};
        const double *dd = o + 3;
        const double x0 = dd[1] * ab[2] - dd[2] * ab[1];
        const double x1 = -dd[0] * ab[2] + dd[2] * ab[0];
        const double x2 = dd[0] * ab[1] - dd[1] * ab[0];
        acc[0] += o[0] / 3.0 + x0;
        acc[1] += o[1] / 3.0 + x1;
        acc[2] += o[2] / 3.0 + x2;
      } else {
        acc[0] += 0.5 * o[0] + e.y * o[2];
        acc[1] += 0.5 * o[1] + e.y * o[3];
      }
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int off = kGatherLanes / 2; off > 0; off >>= 1)
      acc[d] += __shfl_xor_sync(0xffffffffu, acc[d], off);
  if (!live || sub != 0) return;
  const PairDesc &P = pd[p];
  const int row = g - P.pt_off;
  double pn[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < D; ++d) {
    if (dq_out) dq_out[(size_t)g * D + d] = acc[d];
    pn[d] = -P.dis_wgt * acc[d];
    p64[(size_t)g * D + d] = pn[d];
  }
  if (us_n && T > 0) {
    const double *a = x64 + P.var_off + ((size_t)(T - 1) * P.N + row) * D;
    double u[3] = {0, 0, 0}, l[3] = {0, 0, 0};
    for (int d = 0; d < D; ++d) {
      u[d] = a[d] - pn[d];
      l[d] = 0.5 * a[d] - pn[d];
    }
    us_n[g] = make_float4((float)u[0], (float)u[1], (float)u[2], 0.0f);
    ls_n[g] = make_float4((float)l[0], (float)l[1], (float)l[2], 0.0f);
  }
}

// E = dt/2 sum_t a_t.v_t + w (V_DD,DT + V_TT)   (Cpp/src/objgrd.cpp:65).  One CTA
// per pair, partials summed in fixed order.
// reg_part holds one energy partial per (time step, row block): 64-row i-tiles after
// per-step sweeps (groups = 0), `groups`-row groups after persistent sweeps.
__global__ void objective_kernel(const PairDesc *__restrict__ pd, const int *__restrict__ act,
                                 const double *__restrict__ reg_part, int ntile_tot,
                                 const double *__restrict__ vfd_part, int T, PairState *st,
                                 double *f_out, int groups) {
  __shared__ double scr[32];
  pdl_wait();
  pdl_trigger();
  const int p = blockIdx.x;
  if (!act[p]) return;
  const PairDesc &P = pd[p];
  const int nt = P.Npad / (groups > 0 ? groups : kTile), ne = P.Edpad / kTile;
  const int off = groups ? P.grp_off : P.itile_off;
  double r = 0.0, v = 0.0;
  for (int k = threadIdx.x; k < T * nt; k += blockDim.x) {
    const int t = k / nt, i = k - t * nt;
    r += reg_part[(size_t)t * ntile_tot + off + i];
  }
  for (int k = threadIdx.x; k < ne; k += blockDim.x) v += vfd_part[P.etile_off + k];
  const double R = block_sum(r, scr);
  const double V = block_sum(v, scr);
  if (threadIdx.x == 0) {
    const double f = P.dt * 0.5 * R + P.dis_wgt * (V + P.tt);
    if (st) st[p].f_try = f;
    if (f_out) f_out[p] = f;
  }
}

// Target self-term in FP64, once per context (the constant third double loop of
// dqVf_Kernel, Cpp/src/varifold3D.cpp:334-354).  Grid (i blocks, j chunks): block
// (x, y) sums rows [256 x, 256 x + 256) against columns [Et y / ny, Et (y + 1) / ny)
// and writes one partial, part[y * gridDim.x + x]; the host adds them in index order.
template <int D, char CT, char DT>
__global__ void target_self_kernel(const double *__restrict__ tgt, int Et, double cw, double dw,
                                   double *part) {
  __shared__ double scr[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j0 = (int)((long long)Et * blockIdx.y / gridDim.y);
  const int j1 = (int)((long long)Et * (blockIdx.y + 1) / gridDim.y);
  double s = 0.0;
  if (i < Et) {
    const double *ti = tgt + (size_t)i * 8;
    const double iw2 = 1.0 / (cw * cw), ow2 = 2.0 / (dw * dw);
    for (int j = j0; j < j1; ++j) {
      const double *tj = tgt + (size_t)j * 8;
      double r2 = 0.0, ang = 0.0;
      for (int d = 0; d < D; ++d) {
        const double x = ti[d] - tj[d];
        r2 += x * x;
        ang += ti[3 + d] * tj[3 + d];
      }
      const double k = (CT == 'G') ? exp(-r2 * iw2) : 1.0 / (1.0 + r2 * iw2);
      double b;
      if (DT == 'B') b = ang * ang;
      else if (DT == 'L') b = ang;
      else if (DT == 'O') b = exp((ang - 1.0) * ow2);
      else b = exp((ang * ang - 1.0) * ow2);
      s += k * b * tj[6];
    }
    s *= ti[6];
  }
  const double tot = block_sum(s, scr);
  if (threadIdx.x == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = tot;
}

}  // namespace lddmm
