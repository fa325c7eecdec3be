// Kernel sums between two landmark sets, and the dense kernel matrix: the reference's
// two-set overloads (Cpp/src/computeKernel.cpp:246, Cpp/src/multiplyKernel.cpp:294,
// Cpp/src/dqKernel.cpp:307, exposed by the MEX interfaces computeKernelITF /
// multiplyKernelITF / dqKernelITF with 4 / 5 / 6 inputs) and the one-set matrix of
// computeKernel.cpp:21.
//
//   multiply   v_i   = sum_j K(qi_i, qj_j) a_j
//   dq, i side dqi_i = sum_j (l_i . r_j) c(|qi_i - qj_j|) (qi_i - qj_j)
//   dq, j side dqj_j = sum_i (l_i . r_j) c(|qi_i - qj_j|) (qj_j - qi_i)
//
// The two dq sides are the same sum with the sets' roles swapped, so both run on
// CrossOp<kCrossDq> (rows = the side being produced, columns = the other set).  Both
// sums use the all-pairs sweep of sweep.cuh (64-row tiles, cluster split of the j
// range, FP32 pair terms with TwoSum accumulation, FP64 combine in fixed order).
// Positions are carried scaled by the deformation kernel's kscale, as in the
// objective's sweeps, and c(d) (q_i - q_j) = pd_fac * W * (qs_i - qs_j) with W the
// kernel's derivative weight (kernels.cuh).
#pragma once

#include "kernels.cuh"
#include "sweep.cuh"

namespace lddmm {

enum CrossMode : int { kCrossMul = 0, kCrossDq = 1 };

template <int D, int ORDER, int MODE>
struct CrossOp {
  static constexpr int JW = 2;
  static constexpr int NA = D;
  static constexpr bool kTileSum = false;
  static constexpr bool kTwoSets = false;
  struct IData {
    float q[D], x[D];
  };
  const float4 *qa;  // row set, scaled positions            [na padded to kTile]
  const float4 *xa;  // row set, left vectors l (kCrossDq)   [na padded]
  const float4 *qb;  // column set, scaled positions         [nb_pad]
  const float4 *yb;  // column set, a (kCrossMul) or r / l (kCrossDq), zero on padding
  int na, nb_pad;
  double fac;        // output factor: 1 (kCrossMul) or pd_fac (kCrossDq)
  double *out;       // [na * D], FP64

  __device__ bool active(int) const { return true; }
  __device__ int j_count(int) const { return nb_pad; }
  __device__ int set_boundary(int) const { return nb_pad; }
  __device__ void load_i(int, int row, IData &I) const {
    const float4 q = __ldg(&qa[row]);
    I.q[0] = q.x;
    I.q[1] = q.y;
    if (D == 3) I.q[D - 1] = q.z;
    if (MODE == kCrossDq) {
      const float4 x = __ldg(&xa[row]);
      I.x[0] = x.x;
      I.x[1] = x.y;
      if (D == 3) I.x[D - 1] = x.z;
    } else {
#pragma unroll
      for (int d = 0; d < D; ++d) I.x[d] = 0.0f;
    }
  }
  __device__ void load_j(int, int j, float4 (&w)[JW]) const {
    w[0] = __ldg(&qb[j]);
    w[1] = __ldg(&yb[j]);
  }
  template <int SET>
  __device__ __forceinline__ void pair(const IData &I, const float4 (&w)[JW],
                                       float (&acc)[NA]) const {
    const float yj[3] = {w[1].x, w[1].y, w[1].z};
    float dq[D];
    dq[0] = I.q[0] - w[0].x;
    dq[1] = I.q[1] - w[0].y;
    if (D == 3) dq[D - 1] = I.q[D - 1] - w[0].z;
    float nr2 = -dq[0] * dq[0];
#pragma unroll
    for (int d = 1; d < D; ++d) nr2 = fmaf(-dq[d], dq[d], nr2);
    if (MODE == kCrossMul) {
      const float K = DefKernelOf<D, ORDER>::type::val(nr2);
#pragma unroll
      for (int d = 0; d < D; ++d) acc[d] = fmaf(K, yj[d], acc[d]);
    } else {
      float K, Wt;
      DefKernelOf<D, ORDER>::type::val_w(nr2, K, Wt);
      float lr = I.x[0] * yj[0];
#pragma unroll
      for (int d = 1; d < D; ++d) lr = fmaf(I.x[d], yj[d], lr);
      const float s = lr * Wt;
#pragma unroll
      for (int d = 0; d < D; ++d) acc[d] = fmaf(s, dq[d], acc[d]);
    }
  }
  __device__ double finalize(int, int row, const double (&v)[NA]) const {
    if (row < na)
#pragma unroll
      for (int d = 0; d < D; ++d) out[(size_t)row * D + d] = fac * v[d];
    return 0.0;
  }
  __device__ void write_tile(int, int, double) const {}
};

// Dense kernel matrix in the reference's column-major ni x nj layout,
// K[j * ni + i] = K(qi_i, qj_j) (computeKernel.cpp:254-262), FP32 evaluation stored
// as FP64.  Grid-stride over the entries, i fastest: consecutive threads write
// consecutive doubles.  HBM-bound (8 bytes written per entry).
template <int D, int ORDER>
__global__ void kernel_matrix_kernel(const float4 *__restrict__ qi, int ni,
                                     const float4 *__restrict__ qj, int nj, double *K) {
  pdl_wait();
  const long long total = (long long)ni * nj;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
    const int j = (int)(e / ni);
    const int i = (int)(e - (long long)j * ni);
    const float4 a = __ldg(&qi[i]), b = __ldg(&qj[j]);
    const float dx = a.x - b.x, dy = a.y - b.y;
    float nr2 = fmaf(-dy, dy, -dx * dx);
    if (D == 3) {
      const float dz = a.z - b.z;
      nr2 = fmaf(-dz, dz, nr2);
    }
    K[e] = (double)DefKernelOf<D, ORDER>::type::val(nr2);
  }
}

}  // namespace lddmm
