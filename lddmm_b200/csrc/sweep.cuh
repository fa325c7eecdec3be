// All-pairs sweep skeleton shared by the shooting, adjoint and varifold kernels.
//
// Work decomposition (one launch per sweep, every pair of the batch in it):
//   item    = (pair, i-tile of kTile = 64 rows); the item list is built on the host,
//             largest pairs first.
//   cluster = S CTAs on one item (thread-block cluster along x); the S x W warps of
//             the cluster split the item's j range into contiguous shares that differ
//             by at most one point (ops with distance culling: aligned 32-point
//             blocks dealt to the warps in turn, see sweep_packed_kernel).
//   CTA     = W warps; every warp owns all 64 rows of the tile (2 rows per lane) and
//             walks its share in 32-point sub-tiles, staged warp-privately in shared
//             memory with the next sub-tile prefetched into registers, so warps never
//             wait on each other inside the j loop.
// Each 32-pair sub-tile is summed in plain FP32 and folded into a (hi, lo) TwoSum
// accumulator.  Warps are combined in FP64 through shared memory, the cluster's
// CTAs through distributed shared memory (DSMEM) in fixed rank order, so every
// result is bit-reproducible run to run.  Rank 0 of the cluster finalises the rows
// and reduces one FP64 value per tile (energy / varifold value) in fixed order.
//
// An Op supplies:
//   JW, NA            float4 words per staged j point; accumulators per row
//   IData             per-row registers
//   active(p)         evaluate pair p in this sweep
//   load_i(p, row, I) load row data
//   j_count(p)        padded j extent (multiple of kTile)
//   set_boundary(p)   first j of the second class (kTwoSets only)
//   load_j(p, j, w)   global -> registers, one j point per lane
//   kTwoSets          the j range holds two classes (deformed / target)
//   pair<SET>(I, w, acc)        accumulate one pair interaction
//   finalize(p, row, acc)       consume the full FP64 row sums; returns a value
//                               that is summed over the tile
//   write_tile(p, tile, v)      store the tile sum
//
// sweep_packed_kernel is the same sweep for Ops that also evaluate a lane's two rows
// at once in packed FP32x2 arithmetic (sm_100 FFMA2 / FADD2 / FMUL2: one instruction,
// two independent IEEE operations), given
//   JWP, IData2        float4 words of a staged j point whose values are stored twice,
//                      (v, v), so both halves of a packed operand come from one
//                      shared-memory load; the two rows' registers, (row0, row1)
//   load_i2(p, r0, r1, I), load_j2(p, j, w), pair2<SET>(I, w, acc)  with float2 acc
//   kCull              skip j blocks beyond a cut-off, given
//   row_box(p, tile, b) the tile's bounding box (lo[3], hi[3]) in shared memory
//   far(p, b, block)   the aligned 32-point block lies beyond the cut-off from b
// Each packed operation applies to each row exactly the scalar operation of pair()
// in the same order, so both kernels give bitwise the same sums.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"

namespace lddmm {

namespace cg = cooperative_groups;

// Entries [lo, hi) of one staged 32-point sub-tile against the warp's two rows.  SET
// is the compile-time class of those entries (the varifold's deformed / target
// halves), so the accumulator index is static and the arrays stay in registers.
template <int SET, class Op>
__device__ __forceinline__ void run_sub(const Op &op, const float4 (*sj)[kSub], int lo, int hi,
                                        const typename Op::IData &I0,
                                        const typename Op::IData &I1, float (&a0)[Op::NA],
                                        float (&a1)[Op::NA]) {
#pragma unroll 8
  for (int jj = lo; jj < hi; ++jj) {
    float4 w[Op::JW];
#pragma unroll
    for (int x = 0; x < Op::JW; ++x) w[x] = sj[x][jj];
    op.template pair<SET>(I0, w, a0);
    op.template pair<SET>(I1, w, a1);
  }
}

// Warps -> CTA (shared memory) -> cluster (DSMEM) reduction of a tile's row sums and
// the finalisation by cluster rank 0 (shared by both sweep kernels).
template <class Op, int W>
__device__ __forceinline__ void finish_tile(const Op &op, int p, int tile, int rank, int S,
                                            const float (&hi0)[Op::NA], const float (&lo0)[Op::NA],
                                            const float (&hi1)[Op::NA], const float (&lo1)[Op::NA]) {
  constexpr int NA = Op::NA;
  __shared__ double s_red[W][kTile][NA];
  __shared__ double s_cta[kTile][NA];
  __shared__ double s_scr[W];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < NA; ++a) {
    s_red[warp][lane][a] = (double)hi0[a] + (double)lo0[a];
    s_red[warp][32 + lane][a] = (double)hi1[a] + (double)lo1[a];
  }
  __syncthreads();
  double v[NA];
  if (threadIdx.x < kTile) {
#pragma unroll
    for (int a = 0; a < NA; ++a) {
      double s = 0.0;
      for (int w = 0; w < W; ++w) s += s_red[w][threadIdx.x][a];
      v[a] = s;
      s_cta[threadIdx.x][a] = s;
    }
  }
  if (S > 1) {
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    if (rank == 0 && threadIdx.x < kTile) {
      for (int r = 1; r < S; ++r) {
        const double *rem = cluster.map_shared_rank(&s_cta[0][0], r);
#pragma unroll
        for (int a = 0; a < NA; ++a) v[a] += rem[threadIdx.x * NA + a];
      }
    }
    cluster.sync();
  }
  if (rank != 0) return;
  double e = 0.0;
  if (threadIdx.x < kTile) e = op.finalize(p, tile * kTile + threadIdx.x, v);
  if (Op::kTileSum) {
    const double tot = block_sum(e, s_scr);
    if (threadIdx.x == 0) op.write_tile(p, tile, tot);
  }
}

template <int SET, class Op>
__device__ __forceinline__ void run_sub2(const Op &op, const float4 (*sj)[kSub], int lo, int hi,
                                         const typename Op::IData2 &I, float2 (&a)[Op::NA]) {
#pragma unroll 8
  for (int jj = lo; jj < hi; ++jj) {
    float4 w[Op::JWP];
#pragma unroll
    for (int x = 0; x < Op::JWP; ++x) w[x] = sj[x][jj];
    op.template pair2<SET>(I, w, a);
  }
}

// Two row tiles against one staged sub-tile: each column is read from shared memory
// once for the lane's four rows (the same operations per row as run_sub2).
template <int SET, class Op>
__device__ __forceinline__ void run_sub2x2(const Op &op, const float4 (*sj)[kSub], int lo,
                                           int hi, const typename Op::IData2 &I,
                                           const typename Op::IData2 &Ib, float2 (&a)[Op::NA],
                                           float2 (&b)[Op::NA]) {
#pragma unroll 4
  for (int jj = lo; jj < hi; ++jj) {
    float4 w[Op::JWP];
#pragma unroll
    for (int x = 0; x < Op::JWP; ++x) w[x] = sj[x][jj];
    op.template pair2<SET>(I, w, a);
    op.template pair2<SET>(Ib, w, b);
  }
}

// TPW (tiles per work item) = 2: an item is row tiles `tile` and `tile + 1` of one
// pair (the second only when the pair has it, Op::i_count), so that every staged
// column serves four rows per lane and the shared-memory reads per pair halve.  Each
// row sees the same column shares in the same order as with TPW = 1, so the sums are
// bitwise the same.
template <class Op, int W, int TPW = 1>
__global__ void __launch_bounds__(W * 32)
    sweep_packed_kernel(const Op op, const int2 *__restrict__ items, int S) {
  constexpr int JWP = Op::JWP;
  constexpr int NA = Op::NA;
  __shared__ float4 s_j[W][JWP][kSub];
  const int item = blockIdx.x / S;
  const int rank = blockIdx.x - item * S;
  const int2 it = items[item];  // static work list
  pdl_wait();
  pdl_trigger();
  const int p = it.x, tile = it.y;
  if (!op.active(p)) return;  // identical for every CTA of the cluster
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ float s_rbox[6];  // the row tile's bounding box (ops with distance culling)
  if constexpr (Op::kCull) {
    if (threadIdx.x == 0) op.row_box(p, tile, s_rbox);
    __syncthreads();
  }
  typename Op::IData2 I, Ib;
  op.load_i2(p, tile * kTile + lane, tile * kTile + 32 + lane, I);
  bool two = false;  // uniform over the cluster: a second row tile in this item
  if constexpr (TPW == 2) {
    two = (tile + 1) * kTile < op.i_count(p);
    if (two) op.load_i2(p, (tile + 1) * kTile + lane, (tile + 1) * kTile + 32 + lane, Ib);
  }
  float hi0[NA], lo0[NA], hi1[NA], lo1[NA], hi2[NA], lo2[NA], hi3[NA], lo3[NA];
#pragma unroll
  for (int a = 0; a < NA; ++a)
    hi0[a] = lo0[a] = hi1[a] = lo1[a] = hi2[a] = lo2[a] = hi3[a] = lo3[a] = 0.0f;
  const int J = op.j_count(p);
  const int nw = S * W, gw = rank * W + warp;
  const int split = Op::kTwoSets ? op.set_boundary(p) : J;
  float4 nxt[JWP];
  auto stage = [&]() {  // prefetched registers -> the warp's shared-memory sub-tile
    __syncwarp();
#pragma unroll
    for (int x = 0; x < JWP; ++x) s_j[warp][x][lane] = nxt[x];
    __syncwarp();
  };
  auto consume = [&](int j0, int cnt) {  // staged [j0, j0 + cnt) -> TwoSum accumulators
    float2 a[NA];
#pragma unroll
    for (int k = 0; k < NA; ++k) a[k] = make_float2(0.0f, 0.0f);
    if constexpr (TPW == 2) {
      static_assert(!Op::kTwoSets, "two-tile items serve one-set sweeps");
      if (two) {
        float2 b[NA];
#pragma unroll
        for (int k = 0; k < NA; ++k) b[k] = make_float2(0.0f, 0.0f);
        run_sub2x2<0>(op, s_j[warp], 0, cnt, I, Ib, a, b);
#pragma unroll
        for (int k = 0; k < NA; ++k) {
          two_sum_acc(hi2[k], lo2[k], b[k].x);
          two_sum_acc(hi3[k], lo3[k], b[k].y);
        }
      } else {
        run_sub2<0>(op, s_j[warp], 0, cnt, I, a);
      }
    } else if (Op::kTwoSets) {
      const int b = min(max(split - j0, 0), cnt);  // [0, b) first set, [b, cnt) second
      if (b > 0) run_sub2<0>(op, s_j[warp], 0, b, I, a);
      if (b < cnt) run_sub2<1>(op, s_j[warp], b, cnt, I, a);
    } else {
      run_sub2<0>(op, s_j[warp], 0, cnt, I, a);
    }
#pragma unroll
    for (int k = 0; k < NA; ++k) {
      two_sum_acc(hi0[k], lo0[k], a[k].x);
      two_sum_acc(hi1[k], lo1[k], a[k].y);
    }
  };
  if constexpr (Op::kCull) {
    // Ops with distance culling: warp gw of the cluster takes the aligned 32-column
    // sub-tiles gw, gw + nw, gw + 2 nw, ... (J is a multiple of kTile), so the
    // columns that survive the cut-off, which cluster in index, spread evenly over
    // the warps; a sub-tile beyond the cut-off is neither loaded nor evaluated.  The
    // cut-off test runs for 32 candidates at once (lane l tests candidate base + l nw)
    // and a ballot keeps the survivors, so the box loads cost one round trip per 32
    // candidates instead of one per skipped sub-tile.
    const int nsub = J / kSub;
    int base = gw - 32 * nw;  // first candidate of the current group
    unsigned mask = 0u;       // survivors of the current group not yet taken
    auto next = [&]() {       // warp-uniform: the next surviving sub-tile, or nsub
      while (mask == 0u) {
        base += 32 * nw;
        if (base >= nsub) return nsub;
        const int sb = base + lane * nw;
        mask = __ballot_sync(0xffffffffu, sb < nsub && !op.far(p, s_rbox, sb));
      }
      const int k = __ffs(mask) - 1;
      mask &= mask - 1u;
      return base + k * nw;
    };
    int s = next();
    if (s < nsub) op.load_j2(p, s * kSub + lane, nxt);
    while (s < nsub) {
      stage();
      const int sn = next();
      if (sn < nsub) op.load_j2(p, sn * kSub + lane, nxt);
      consume(s * kSub, kSub);
      s = sn;
    }
  } else {
    // every warp of the cluster takes one contiguous, equal (+-1) share of the j range
    const int jb = (int)((long long)J * gw / nw), je = (int)((long long)J * (gw + 1) / nw);
    if (jb + lane < je) op.load_j2(p, jb + lane, nxt);
    for (int j0 = jb; j0 < je; j0 += kSub) {
      stage();
      const int jn = j0 + kSub;
      if (jn + lane < je) op.load_j2(p, jn + lane, nxt);
      consume(j0, min(kSub, je - j0));
    }
  }
  finish_tile<Op, W>(op, p, tile, rank, S, hi0, lo0, hi1, lo1);
  if constexpr (TPW == 2) {
    if (two) {
      __syncthreads();  // the first tile's reduction is done with the shared arrays
      finish_tile<Op, W>(op, p, tile + 1, rank, S, hi2, lo2, hi3, lo3);
    }
  }
}

template <class Op, int W>
__global__ void __launch_bounds__(W * 32) sweep_kernel(const Op op, const int2 *__restrict__ items,
                                                       int S) {
  constexpr int JW = Op::JW;
  constexpr int NA = Op::NA;
  __shared__ float4 s_j[W][JW][kSub];

  const int item = blockIdx.x / S;
  const int rank = blockIdx.x - item * S;
  const int2 it = items[item];  // static work list
  pdl_wait();
  pdl_trigger();
  const int p = it.x, tile = it.y;
  if (!op.active(p)) return;  // identical for every CTA of the cluster

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  typename Op::IData I0, I1;
  op.load_i(p, tile * kTile + lane, I0);
  op.load_i(p, tile * kTile + 32 + lane, I1);

  float hi0[NA], lo0[NA], hi1[NA], lo1[NA];
#pragma unroll
  for (int a = 0; a < NA; ++a) hi0[a] = lo0[a] = hi1[a] = lo1[a] = 0.0f;

  // every warp of the cluster takes one contiguous, equal (+-1) share of the j range
  const int J = op.j_count(p);
  const int nw = S * W, gw = rank * W + warp;
  const int jb = (int)((long long)J * gw / nw), je = (int)((long long)J * (gw + 1) / nw);
  const int split = Op::kTwoSets ? op.set_boundary(p) : J;
  float4 nxt[JW];
  if (jb + lane < je) op.load_j(p, jb + lane, nxt);
  for (int j0 = jb; j0 < je; j0 += kSub) {
    __syncwarp();
#pragma unroll
    for (int x = 0; x < JW; ++x) s_j[warp][x][lane] = nxt[x];
    __syncwarp();
    const int cnt = min(kSub, je - j0);
    const int jn = j0 + kSub;
    if (jn + lane < je) op.load_j(p, jn + lane, nxt);
    float a0[NA], a1[NA];
#pragma unroll
    for (int a = 0; a < NA; ++a) a0[a] = a1[a] = 0.0f;
    if (Op::kTwoSets) {
      const int b = min(max(split - j0, 0), cnt);  // [0, b) first set, [b, cnt) second
      if (b > 0) run_sub<0>(op, s_j[warp], 0, b, I0, I1, a0, a1);
      if (b < cnt) run_sub<1>(op, s_j[warp], b, cnt, I0, I1, a0, a1);
    } else {
      run_sub<0>(op, s_j[warp], 0, cnt, I0, I1, a0, a1);
    }
#pragma unroll
    for (int a = 0; a < NA; ++a) {
      two_sum_acc(hi0[a], lo0[a], a0[a]);
      two_sum_acc(hi1[a], lo1[a], a1[a]);
    }
  }

  finish_tile<Op, W>(op, p, tile, rank, S, hi0, lo0, hi1, lo1);
}

}  // namespace lddmm
