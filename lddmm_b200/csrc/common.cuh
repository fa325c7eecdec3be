// Shared device helpers for the LDDMM sm_100a kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace lddmm {

// ---------------------------------------------------------------- constants

constexpr float kLog2e = 1.4426950408889634f;
constexpr float kLn2 = 0.6931471805599453f;

// Padding granule for points and elements: one i-tile (two rows per lane of a warp).
constexpr int kTile = 64;
constexpr int kSub = 32;  // j sub-tile staged per warp

// ------------------------------------------------------- MUFU approximations
// PTX instructions (ISA-documented approximations), used in the all-pairs loops.
// The caller folds log2(e) and the kernel widths into the coordinates beforehand.

__device__ __forceinline__ float ex2f(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ float sqrtf_approx(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ float rcpf_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// ------------------------------------------- programmatic dependent launch
// Kernels of the objective sweep and the L-BFGS cycle are launched with
// programmatic stream serialisation: a kernel may start while its predecessor is
// still running.  Every such kernel executes pdl_wait() before it reads anything a
// predecessor writes and before any early return (so a grid never completes ahead
// of its predecessor), and pdl_trigger() to let its own successor start launching.
// Without the launch attribute both are no-ops.

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ------------------------------------------------- compensated accumulation
// Knuth's TwoSum: hi + lo carries the running sum exactly up to the rounding of
// the final hi + lo.  Tile partials (32 terms, plain FP32) are folded in here, so
// the compensation costs 6 flops per 32 pairs per accumulator.

__device__ __forceinline__ void two_sum_acc(float &hi, float &lo, float x) {
  float s = hi + x;
  float bb = s - hi;
  float err = (hi - (s - bb)) + (x - bb);
  hi = s;
  lo += err;
}

// ----------------------------------------------------------- FP64 reductions

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum of one double per thread; result valid in thread 0.
// `scratch` must hold blockDim.x / 32 doubles.
__device__ __forceinline__ double block_sum(double v, double *scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < nw; ++w) r += scratch[w];
  return r;
}

}  // namespace lddmm
