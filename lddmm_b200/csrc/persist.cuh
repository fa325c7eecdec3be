// Persistent multi-step sweep: all T time steps of the forward (shooting) or the
// backward (adjoint) recursion in one cooperative launch.
//
// The steps are sequential (step t + 1 reads the positions / adjoint state step t
// finalised) and, for one registration of a few thousand landmarks, one step is only
// a few microseconds of arithmetic.  Per-step launches then spend most of their time
// ramping CTAs up and down and in the cross-CTA reduction of split j ranges.  Here:
//
//   * every CTA stays resident for the whole recursion; steps are separated by a
//     grid barrier;
//   * a work unit is a row group of kGroup = 16 rows of one pair, and its CTA covers
//     the whole j range: the 8 warps take equal contiguous shares, and inside a warp
//     lane l handles rows l % 8 and l % 8 + 8 against every 4th point of each staged
//     32-point sub-tile (lane group l / 8), so each staged operand serves two pairs;
//   * reductions stay inside the CTA: a shuffle butterfly over the 4 lane groups, then
//     the 8 warps through shared memory in warp order, all in FP64 after the per-tile
//     TwoSum, so results are bit-reproducible;
//   * the unit's first 8 threads finalise its rows (Euler step / adjoint update).
//
// The grid barrier is a monotonically increasing arrival counter (reset before the
// launch).  Every wait is bounded: after kSpinLimit polls the CTA records the step in
// the error word and leaves the kernel, so a launch that is not fully co-resident ends
// with an error instead of hanging.  The launch uses the cooperative attribute, with
// which the runtime refuses a grid that cannot be co-resident.
#pragma once

#include "common.cuh"
#include "layout.h"
#include "sweep.cuh"

namespace lddmm {

constexpr int kGroup = 16;                // rows per persistent work unit
constexpr int kRowPairs = kGroup / 2;     // lanes sharing a j entry (2 rows each)
constexpr int kLaneGroups = 32 / kRowPairs;  // j interleave inside a warp
constexpr int kPersistWarps = 8;          // warps per persistent CTA

struct StepSync {
  unsigned int arrive;  // grid barrier arrivals, reset to 0 before every launch
  unsigned int error;   // nonzero: a barrier wait timed out (1 + step index)
  // timeline of the cooperative kernels of the last cycle (%globaltimer, ns):
  // [slot][0] entry of CTA 0, [slot][1] latest CTA exit; slots: 0 forward sweep,
  // 1 backward sweep, 2 optimiser update
  unsigned long long stamp[4][2];
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void stamp_entry(StepSync *sy, int slot) {
  if (blockIdx.x == 0 && threadIdx.x == 0) sy->stamp[slot][0] = global_ns();
}

__device__ __forceinline__ void stamp_exit(StepSync *sy, int slot) {
  if (threadIdx.x == 0) atomicMax(&sy->stamp[slot][1], global_ns());
}

constexpr unsigned int kSpinLimit = 1u << 22;  // polls: a few seconds at most

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Returns false when the wait timed out (the caller must leave the kernel).
__device__ __forceinline__ bool grid_barrier(StepSync *sy, unsigned int target,
                                             unsigned int step) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(&sy->arrive, 1u);
    int ok = 1;
    unsigned int n = 0;
    while (ld_acquire(&sy->arrive) < target) {
      if (ld_acquire(&sy->error) != 0u || ++n > kSpinLimit) {
        atomicCAS(&sy->error, 0u, 1u + step);
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Op: the sweep interface of sweep.cuh plus set_step(t) (pointers of time step t) and
// write_group(p, k, v) (row-group partial of a kTileSum op).  units: (pair, row group).
// dir = +1 runs t = 0..T-1, dir = -1 runs t = T-1..0.
// Two CTAs per SM (<= 128 registers): a single registration of a few thousand
// landmarks then has all its row groups resident at once.
template <class Op>
__global__ void __launch_bounds__(kPersistWarps * 32, 2)
    persistent_sweep_kernel(Op op, const int2 *__restrict__ units, int n_units, int T, int dir,
                            StepSync *sy) {
  constexpr int JW = Op::JW;
  constexpr int NA = Op::NA;
  constexpr int NW = kPersistWarps;
  __shared__ float4 s_j[NW][JW][kSub];
  __shared__ double s_red[NW][kGroup][NA];
  __shared__ double s_scr[NW];
  __shared__ PairDesc s_pd;  // descriptor of the unit in hand, kept across steps
  __shared__ int s_unit[3];  // unit index, pair, active flag
  pdl_wait();
  stamp_entry(sy, dir > 0 ? 0 : 1);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lrow = lane % kRowPairs, lg = lane / kRowPairs;
  if (threadIdx.x == 0) s_unit[0] = -1;
  for (int s = 0; s < T; ++s) {
    const int t = dir > 0 ? s : T - 1 - s;
    Op o = op;
    o.set_step(t);
    for (int u = blockIdx.x; u < n_units; u += gridDim.x) {
      __syncthreads();
      if (s_unit[0] != u) {  // uniform; a CTA with one unit loads it once
        __syncthreads();
        if (threadIdx.x == 0) {
          const int2 un = units[u];
          s_unit[0] = u;
          s_unit[1] = un.x | (un.y << 16);
          s_unit[2] = op.active(un.x);
          s_pd = op.pd[un.x];
        }
        __syncthreads();
      }
      if (!s_unit[2]) continue;  // uniform for the CTA
      const int grp = s_unit[1] >> 16;
      o.pd = &s_pd;  // the op reads descriptor 0 from shared memory from here on
      const int p = 0;
      typename Op::IData I0, I1;
      o.load_i(p, grp * kGroup + lrow, I0);
      o.load_i(p, grp * kGroup + kRowPairs + lrow, I1);
      float hi0[NA], lo0[NA], hi1[NA], lo1[NA];
#pragma unroll
      for (int a = 0; a < NA; ++a) hi0[a] = lo0[a] = hi1[a] = lo1[a] = 0.0f;
      const int J = o.j_count(p);
      const int jb = (int)((long long)J * warp / NW), je = (int)((long long)J * (warp + 1) / NW);
      const int split = Op::kTwoSets ? o.set_boundary(p) : J;
      float4 nxt[JW];
      float acc0[NA], acc1[NA];
      if (jb + lane < je) o.load_j(p, jb + lane, nxt);
      for (int j0 = jb; j0 < je; j0 += kSub) {
        __syncwarp();
#pragma unroll
        for (int x = 0; x < JW; ++x) s_j[warp][x][lane] = nxt[x];
        __syncwarp();
        const int cnt = min(kSub, je - j0);
        const int jn = j0 + kSub;
        if (jn + lane < je) o.load_j(p, jn + lane, nxt);
        const bool fresh = ((j0 - jb) & (4 * kSub - 1)) == 0;
        if (fresh) {
#pragma unroll
          for (int a = 0; a < NA; ++a) acc0[a] = acc1[a] = 0.0f;
        }
        const int b = Op::kTwoSets ? min(max(split - j0, 0), cnt) : cnt;
#pragma unroll 4
        for (int jj = lg; jj < b; jj += kLaneGroups) {
          float4 w[JW];
#pragma unroll
          for (int x = 0; x < JW; ++x) w[x] = s_j[warp][x][jj];
          o.template pair<0>(I0, w, acc0);
          o.template pair<0>(I1, w, acc1);
        }
        if (Op::kTwoSets) {
          // first entry >= b that belongs to this lane group
          const int b1 = b + ((lg - b) % kLaneGroups + kLaneGroups) % kLaneGroups;
#pragma unroll 4
          for (int jj = b1; jj < cnt; jj += kLaneGroups) {
            float4 w[JW];
#pragma unroll
            for (int x = 0; x < JW; ++x) w[x] = s_j[warp][x][jj];
            o.template pair<1>(I0, w, acc0);
            o.template pair<1>(I1, w, acc1);
          }
        }
        // fold into the compensated sum every 4 sub-tiles (<= 32 plain FP32 terms per
        // lane) and after the last one
        if (((j0 - jb) & (4 * kSub - 1)) == 3 * kSub || j0 + kSub >= je) {
#pragma unroll
          for (int a = 0; a < NA; ++a) {
            two_sum_acc(hi0[a], lo0[a], acc0[a]);
            two_sum_acc(hi1[a], lo1[a], acc1[a]);
          }
        }
      }
      // lane groups -> lanes 0..7 (fixed butterfly), then warps in order
#pragma unroll
      for (int a = 0; a < NA; ++a) {
        double v0 = (double)hi0[a] + (double)lo0[a];
        double v1 = (double)hi1[a] + (double)lo1[a];
#pragma unroll
        for (int off = kRowPairs; off < 32; off <<= 1) {
          v0 += __shfl_xor_sync(0xffffffffu, v0, off);
          v1 += __shfl_xor_sync(0xffffffffu, v1, off);
        }
        if (lg == 0) {
          s_red[warp][lrow][a] = v0;
          s_red[warp][kRowPairs + lrow][a] = v1;
        }
      }
      __syncthreads();
      double e = 0.0;
      if (threadIdx.x < kGroup) {
        double v[NA];
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          double x = 0.0;
          for (int w = 0; w < NW; ++w) x += s_red[w][threadIdx.x][a];
          v[a] = x;
        }
        e = o.finalize(p, grp * kGroup + threadIdx.x, v);
      }
      if (Op::kTileSum) {
        const double tot = block_sum(e, s_scr);
        if (threadIdx.x == 0) o.write_group(p, grp, tot);
      }
    }
    if (!grid_barrier(sy, (unsigned)(s + 1) * gridDim.x, (unsigned)s)) return;
  }
  stamp_exit(sy, dir > 0 ? 0 : 1);
  pdl_trigger();
}

}  // namespace lddmm
