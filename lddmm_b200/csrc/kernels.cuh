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
// :160-238 (3D Matern orders 0..4; the 2D Matern family is MaternBessel2D below) and their derivatives Cpp/src/dqKernel.cpp:56-57,
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

// ------------------------------------------------------ 2D Matern (Bessel K)
// In 2D the reference's Matern family is built from p0(x) = x^2 K0(x) and
// p1(x) = x K1(x), x = |dq| / sigma (Cpp/src/computeKernel.cpp:44-155,
// Cpp/src/dqKernel.cpp:68-195, with p0Fcn / p1Fcn of Cpp/src/polybesselk.cpp:14-96 and
// their cut-offs: p0(0) = 0, p1(0) = 1).  The kernels of orders 0..4 are
//   K0 = p1,  K1 = p0/2 + p1,  K2 = (4 p0 + (8 + x^2) p1) / 8,
//   K3 = ((24 + x^2) p0 + 8 (6 + x^2) p1) / 48,
//   K4 = (12 (16 + x^2) p0 + (384 + x^2 (72 + x^2)) p1) / 384,
// and the reference's dq factor of order n is -K_{n-1} / (2 n sigma^2), so the gradient
// weight here is W = K_{n-1} / (2 n) with pd_fac = -1 / (sigma^2 kscale), kscale = 1 / sigma.
//
// p0 and p1 are evaluated in FP32 from the mathematics of K0 and K1, not from the
// reference's rational approximations:
//   x <= 2       ascending series (Abramowitz & Stegun 9.6.13 and 9.6.11, n = 1), 10 terms
//                in y = x^2 / 4:  K0 = -(ln(x/2) + gamma) I0 + sum_k H_k y^k / (k!)^2,
//                x K1 = 1 + x ln(x/2) I1 - y sum_k (psi(k+1) + psi(k+2)) y^k / (k! (k+1)!);
//   2 < x <= 10  trapezoid rule on K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt, step
//                1/4, 14 nodes (the integrand is analytic in a strip, so the rule converges
//                geometrically);
//   x > 10       asymptotic expansion sqrt(pi / 2x) e^-x sum_k a_k(nu) / x^k, 10 terms.
// Relative error against double-precision K0 / K1 stays below 1e-6 over x in [1e-8, 90].
__device__ __forceinline__ float lg2f_approx(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ void bessel_p01(float x, float &p0, float &p1) {
  constexpr float kGamma = 0.5772156649015329f;
  if (x < 1e-18f) {
    p0 = 0.0f;
    p1 = 1.0f;
    return;
  }
  if (x <= 2.0f) {
    // harmonic numbers H_k and psi(k+1) + psi(k+2) = H_k + H_{k+1} - 2 gamma
    constexpr float H[10] = {0.0f, 1.0f, 1.5f, 1.83333333f, 2.08333333f, 2.28333333f, 2.45f,
                             2.59285714f, 2.71785714f, 2.82896825f};
    constexpr float S[10] = {-0.154431330f, 1.34556867f, 2.17890200f, 2.76223534f,
                             3.21223534f, 3.57890200f, 3.88842581f, 4.15628296f,
                             4.39239407f, 4.60350518f};
    const float y = 0.25f * x * x;
    float t = 1.0f;  // y^k / (k!)^2
    float i0 = 1.0f, s0 = 0.0f, i1 = 1.0f, s1 = S[0];
#pragma unroll
    for (int k = 1; k < 10; ++k) {
      t *= y * (1.0f / (float)(k * k));
      const float u = t * (1.0f / (float)(k + 1));  // y^k / (k! (k+1)!)
      i0 += t;
      s0 = fmaf(H[k], t, s0);
      i1 += u;
      s1 = fmaf(S[k], u, s1);
    }
    const float L = (lg2f_approx(x) - 1.0f) * kLn2;  // ln(x / 2)
    p0 = x * x * fmaf(-(L + kGamma), i0, s0);
    p1 = fmaf(2.0f * y * L, i1, fmaf(-y, s1, 1.0f));
    return;
  }
  if (x <= 10.0f) {
    // nodes t_k = k / 4: C[k] = cosh t_k, A[k] = (cosh t_k - 1) log2 e
    constexpr float C[13] = {1.0314131f, 1.12762597f, 1.29468328f, 1.54308063f, 1.88842388f,
                             2.35240962f, 2.96418831f, 3.76219569f, 4.79656753f, 6.13228948f,
                             7.85327987f, 10.067662f, 12.9145571f};
    constexpr float A[13] = {0.0453195234f, 0.184125347f, 0.425138113f, 0.783499739f,
                             1.28172472f, 1.95111465f, 2.83372473f, 3.98500603f,
                             5.47728915f, 7.40432858f, 9.88719289f, 13.081871f, 17.1890724f};
    float s0 = 0.5f, s1 = 0.5f;
#pragma unroll
    for (int k = 0; k < 13; ++k) {
      const float g = ex2f(-x * A[k]);
      s0 += g;
      s1 = fmaf(C[k], g, s1);
    }
    const float he = 0.25f * ex2f(-x * kLog2e);  // h e^-x
    p0 = x * x * he * s0;
    p1 = x * he * s1;
    return;
  }
  // a_k(nu) / a_{k-1}(nu) = (4 nu^2 - (2k - 1)^2) / (8 k)
  const float r = rcpf_approx(x);
  float t0 = 1.0f, t1 = 1.0f, s0 = 1.0f, s1 = 1.0f;
#pragma unroll
  for (int k = 1; k <= 10; ++k) {
    const float m = (float)((2 * k - 1) * (2 * k - 1));
    t0 *= (-m / (8.0f * k)) * r;
    t1 *= ((4.0f - m) / (8.0f * k)) * r;
    s0 += t0;
    s1 += t1;
  }
  const float c = 1.2533141373155003f * sqrtf_approx(x) * ex2f(-x * kLog2e);  // sqrt(pi x / 2) e^-x
  p0 = x * c * s0;
  p1 = c * s1;
}

template <int ORDER>
struct MaternBessel2D {
  // K_n(x) of the family in terms of p0, p1 and x^2
  template <int N>
  static __device__ __forceinline__ float form(float p0, float p1, float x2) {
    if (N == 0) return p1;
    if (N == 1) return fmaf(0.5f, p0, p1);
    if (N == 2) return fmaf(0.5f, p0, fmaf(0.125f * x2, p1, p1));
    if (N == 3) return fmaf(fmaf(x2, 1.0f / 48.0f, 0.5f), p0, fmaf(x2, 1.0f / 6.0f, 1.0f) * p1);
    return fmaf(fmaf(x2, 1.0f / 32.0f, 0.5f), p0,
                fmaf(x2 * (72.0f + x2), 1.0f / 384.0f, 1.0f) * p1);
  }
  static __device__ __forceinline__ float val(float nr2) {
    const float x = sqrtf_approx(-nr2);
    float p0, p1;
    bessel_p01(x, p0, p1);
    return form<ORDER>(p0, p1, -nr2);
  }
  static __device__ __forceinline__ void val_w(float nr2, float &K, float &W) {
    const float x = sqrtf_approx(-nr2);
    float p0, p1;
    bessel_p01(x, p0, p1);
    K = form<ORDER>(p0, p1, -nr2);
    W = (ORDER == 0) ? 0.0f : form<(ORDER > 0 ? ORDER - 1 : 0)>(p0, p1, -nr2) *
                                  (1.0f / (2.0f * (ORDER > 0 ? ORDER : 1)));
  }
};

// Deformation kernel of dimension D and order: the 2D Matern family has its own
// (Bessel K) definition; every other combination uses DefKernel.
template <int D, int ORDER>
struct DefKernelOf {
  using type = DefKernel<ORDER>;
};
template <int ORDER>
struct DefKernelOf<2, ORDER> {
  using type = MaternBessel2D<ORDER>;
};
template <>
struct DefKernelOf<2, -1> {
  using type = DefKernel<-1>;
};

// Host-side scale and gradient factor for a family (see the header comment).
inline void def_kernel_scales(int order, int dim, double width, float *kscale,
                              double *pd_fac) {
  const double log2e = 1.4426950408889634;
  const double w2 = width * width;
  if (order == -1) {
    const double s = std::sqrt(log2e) / width;
    *kscale = (float)s;
    *pd_fac = -2.0 / (w2 * s);
    return;
  }
  if (dim == 2) {  // Bessel forms in x = |dq| / sigma
    const double s = 1.0 / width;
    *kscale = (float)s;
    *pd_fac = order == 0 ? 0.0 : -1.0 / (w2 * s);
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
