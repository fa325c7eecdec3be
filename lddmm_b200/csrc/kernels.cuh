// Deformation and varifold kernel functions in scaled coordinates.
//
// The host stores positions pre-multiplied by a per-pair scale s so that the
// exponent needs no multiply inside the pair loop:
//   Gaussian  K = exp(-|dq|^2 / sigma^2)  ->  s = sqrt(log2 e) / sigma,  K = 2^(-r2)
//   Matern    K = P_n(d) exp(-d), d = |dq| / sigma  ->  s = log2 e / sigma,
//             r = |dq_s| = d log2 e,  exp(-d) = 2^(-r),  d = r ln 2
// The gradient weight W satisfies  dK/dq_i = pd_fac * W * dq_scaled,  with pd_fac
// folded in per pair on the host (PairDesc::pd_fac).
//
// Kernel definitions follow Cpp/src/computeKernel.cpp:26-41 (Gaussian),
// :160-238 (3D Matern orders 0..4) and their derivatives Cpp/src/dqKernel.cpp:56-57,
// :200-300.  Matern order 0 is not differentiable at 0; the reference leaves its
// gradient at zero (dqKernel.cpp has no order-0 case), and so does W here.
#pragma once

#include <cmath>

#include "common.cuh"

namespace lddmm {

enum KernelFamily : int {
  kGauss = -1,
  kMatern0 = 0,
  kMatern1 = 1,
  kMatern2 = 2,
  kMatern3 = 3,
  kMatern4 = 4,
};

template <int ORDER>
struct DefKernel;

template <>
struct DefKernel<-1> {
  static __device__ __forceinline__ float val(float nr2) { return ex2f(nr2); }
  static __device__ __forceinline__ void val_w(float nr2, float &K, float &W) {
    K = ex2f(nr2);
    W = K;
  }
};

// Matern kernels take the NEGATED squared scaled distance for symmetry with the
// Gaussian (the pair loops produce -r2 with free negation modifiers).
template <int ORDER>
struct DefKernel {
  static __device__ __forceinline__ float poly_k(float d) {
    if (ORDER == 0) return 1.0f;
    if (ORDER == 1) return 1.0f + d;
    if (ORDER == 2) return fmaf(d, fmaf(d, 1.0f / 3.0f, 1.0f), 1.0f);
    if (ORDER == 3) return fmaf(d, fmaf(d, fmaf(d, 1.0f / 15.0f, 0.4f), 1.0f), 1.0f);
    return fmaf(d, fmaf(d, fmaf(d, fmaf(d, 1.0f / 105.0f, 2.0f / 21.0f), 3.0f / 7.0f), 1.0f), 1.0f);
  }
  static __device__ __forceinline__ float poly_w(float d) {
    if (ORDER <= 1) return 1.0f;
    if (ORDER == 2) return 1.0f + d;
    if (ORDER == 3) return fmaf(d, d + 3.0f, 3.0f);
    return fmaf(d, fmaf(d, d + 6.0f, 15.0f), 15.0f);
  }
  static __device__ __forceinline__ float val(float nr2) {
    const float r = sqrtf_approx(-nr2);
    const float e = ex2f(-r);
    if (ORDER == 0) return e;
    return e * poly_k(r * kLn2);
  }
  static __device__ __forceinline__ void val_w(float nr2, float &K, float &W) {
    const float r = sqrtf_approx(-nr2);
    const float e = ex2f(-r);
    if (ORDER == 0) {
      K = e;
      W = 0.0f;
      return;
    }
    const float d = r * kLn2;
    K = e * poly_k(d);
    W = (ORDER == 1) ? e : e * poly_w(d);
  }
};

// Host-side scale and gradient factor for a family (see the header comment).
inline void def_kernel_scales(int order, double width, float *kscale, double *pd_fac) {
  const double log2e = 1.4426950408889634;
  const double w2 = width * width;
  if (order == -1) {
    const double s = std::sqrt(log2e) / width;
    *kscale = (float)s;
    *pd_fac = -2.0 / (w2 * s);
    return;
  }
  const double s = log2e / width;
  *kscale = (float)s;
  switch (order) {
    case 1: *pd_fac = -1.0 / (w2 * s); break;
    case 2: *pd_fac = -1.0 / (3.0 * w2 * s); break;
    case 3: *pd_fac = -1.0 / (15.0 * w2 * s); break;
    case 4: *pd_fac = -1.0 / (105.0 * w2 * s); break;
    default: *pd_fac = 0.0; break;
  }
}

// ------------------------------------------------------------ varifold kernels
// Centre kernels (Cpp/src/varifold3D.cpp:41-93), in centres scaled by cscale:
//   'G'  k = exp(-|dc|^2/sigma^2) = 2^(-r2),  cscale = sqrt(log2 e)/sigma,
//        dk/dc_i = -2 k / sigma^2 dc  ->  gradient weight k
//   'C'  k = 1 / (1 + |dc|^2/sigma^2),         cscale = 1/sigma,
//        dk/dc_i = -2 k^2 / sigma^2 dc  ->  gradient weight k^2
// Both share dc_fac = -2 / (sigma^2 cscale) on the host.
template <char CT>
struct CenKernel {
  static __device__ __forceinline__ void val_w(float nr2, float &k, float &kw) {
    if (CT == 'G') {
      k = ex2f(nr2);
      kw = k;
    } else {
      k = rcpf_approx(1.0f - nr2);
      kw = k * k;
    }
  }
};

inline void cen_kernel_scales(char type, double width, float *cscale, double *dc_fac) {
  const double log2e = 1.4426950408889634;
  const double s = (type == 'G') ? std::sqrt(log2e) / width : 1.0 / width;
  *cscale = (float)s;
  *dc_fac = -2.0 / (width * width * s);
}

// Direction kernels (Cpp/src/varifold3D.cpp:95-188): value b(ang) and derivative
// b'(ang), ang = n_i . n_j.  ow2 = 2 / dirKnlWidth^2 for the Gaussian kinds.
template <char DT>
struct DirKernel {
  static __device__ __forceinline__ void val_d(float ang, float ow2, float &b, float &db) {
    if (DT == 'B') {
      b = ang * ang;
      db = 2.0f * ang;
    } else if (DT == 'L') {
      b = ang;
      db = 1.0f;
    } else if (DT == 'O') {
      b = ex2f((ang - 1.0f) * ow2 * kLog2e);
      db = ow2 * b;
    } else {  // 'U'
      b = ex2f((ang * ang - 1.0f) * ow2 * kLog2e);
      db = 2.0f * ang * ow2 * b;
    }
  }
};

}  // namespace lddmm
