// Persistent multi-step sweep: all T time steps of the forward (shooting) or the
// backward (adjoint) recursion in one cooperative launch.
//
// The steps are sequential (step t + 1 reads the positions / adjoint state step t
// finalised) and, for one registration of a few thousand landmarks, one step is only
// a few microseconds of arithmetic.  Per-step launches then spend most of their time
// ramping CTAs up and down.  Here:
//
//   * every CTA stays resident for the whole recursion; steps are separated by a
//     grid barrier;
//   * the work of a step is the list of row groups (kGroup = 16 rows of one pair)
//     times their j ranges, laid end to end and cut into one contiguous share per CTA
//     (host-side plan, snapped to 32-entry boundaries): every CTA gets the same number
//     of pair interactions whatever the row-group count, so no SM idles at the barrier
//     while another runs a second row group.  A CTA's share is a list of segments
//     (row group, j range), taken two at a time ("rounds");
//   * in a round the entries of its (one or two) segments, laid end to end, are cut
//     into 8 equal contiguous warp shares (a share that straddles the two segments is
//     processed as two pieces); lane l handles rows l % 8 and l % 8 + 8 against every
//     4th point of each staged 32-point sub-tile (lane group l / 8), so each staged
//     operand serves two pairs;
//   * reductions: a shuffle butterfly over the 4 lane groups, then all 8 warps through
//     shared memory in warp order (a warp without entries of the segment adds zero),
//     in FP64 after the per-tile TwoSum.  A row
//     group cut over several CTAs stores one FP64 partial per part; the CTA that
//     completes the row group's arrival count (whichever it is) adds the parts in part
//     order and finalises, so results are bit-reproducible for a given plan;
//   * each segment of a round has its own 16-thread epilogue group (lanes 0-15 of warp
//     0 or of warp 1): both run at once, with warp-level synchronisation only.
//
// Grid barrier: a monotonically increasing arrival count (fire-and-forget atomic
// add) that the CTAs poll against (step + 1) x grid.  When a launch ends, each CTA
// counts its departure after its last wait; the last one to leave zeroes both counts,
// so the next launch starts from zero without a memset.  Every wait is bounded: after
// kSpinLimit polls the CTA records the step in the error word and leaves the kernel,
// so a launch that is not fully co-resident ends with an error instead of hanging (the
// host then clears the words).  The launch uses the cooperative attribute, with which
// the runtime refuses a grid that cannot be co-resident.
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
  unsigned int arrive;  // grid barrier arrivals since the launch began
  unsigned int error;   // nonzero: a barrier wait timed out (1 + step index)
  unsigned int depart;  // CTAs past their last wait (resets arrive at launch end)
  unsigned int pad_;
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

constexpr unsigned int kSpinLimit = 1u << 23;  // polls: a few seconds at most

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Arrival count with release semantics (orders this thread's writes, and those of
// threads synchronised with it, before the increment) and no return value.
__device__ __forceinline__ void red_add_release_gpu(unsigned int *p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Atomic add at GPU scope with release and acquire semantics; returns the old value.
__device__ __forceinline__ unsigned int atom_add_acq_rel_gpu(unsigned int *p, unsigned int v) {
  unsigned int old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v)
               : "memory");
  return old;
}

__device__ __forceinline__ unsigned int ld_relaxed(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Waits until `target` arrivals (this CTA's included) have been counted.  Returns
// false when the wait timed out (the caller must leave the kernel without departing).
// `tag` identifies the wait in the error word.  The arrival is a release reduction
// (the CTA's writes, ordered before it by __syncthreads, become visible with it); the
// poll is one acquire load per iteration (the error word is read every 64th), so the
// load that sees the count complete also orders the CTA's later reads after the
// arrivals, with no further round trip to L2.
__device__ __forceinline__ bool grid_barrier(StepSync *sy, unsigned int target,
                                             unsigned int tag,
                                             unsigned int spin = kSpinLimit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    red_add_release_gpu(&sy->arrive, 1u);
    unsigned int n = 0;
    while (ld_acquire(&sy->arrive) < target) {
      if ((++n & 63u) == 0u) {
        if (ld_relaxed(&sy->error) != 0u || n > spin) {
          atomicCAS(&sy->error, 0u, 1u + tag);
          ok = 0;
          break;
        }
        if (n > 4096u) __nanosleep(64);
      }
    }
    // the acquire load that read the complete count read the end of the release
    // sequence of every CTA's arrival (each arrival is a read-modify-write), so their
    // writes are visible to this thread, and through the __syncthreads to the CTA
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// After a CTA's last grid_barrier: the last CTA to depart zeroes the counts.  Every
// CTA has stopped polling `arrive` by then.
__device__ __forceinline__ void grid_depart(StepSync *sy) {
  if (threadIdx.x == 0) {
    const unsigned int old = atomicAdd(&sy->depart, 1u);
    if (old == gridDim.x - 1) {
      sy->arrive = 0u;
      sy->depart = 0u;
    }
  }
}

// Work plan of the persistent sweeps (built on the host when the context is created).
struct SweepPlan {
  const int2 *units;      // (pair, row group) per unit
  const int4 *segs;       // (unit, j begin, j end, part) in CTA order
  const int *cta_seg;     // CTA k owns segs[cta_seg[k] .. cta_seg[k + 1])
  const int2 *unit_parts; // (parts, first partial slot) per unit
  double *part;           // FP64 partials [slot][kGroup][kPartNA]
  unsigned int *cnt;      // per-unit arrival count of split row groups (self-resetting)
};

constexpr int kPartNA = 6;  // accumulators per row in a partial slot (>= every Op::NA)

// One round of a persistent CTA: the entries of its (one or two) segments, laid end
// to end, cut into NW equal contiguous warp shares (a share that straddles the two
// segments is processed as two pieces); every warp leaves its FP64 row sums of
// segment g in s_red[g][warp] (zeros where it has no entries of g).  `o` has the step
// set; o.pd is redirected to the round's descriptors in shared memory.
template <class Op>
__device__ __forceinline__ void persist_round(
    Op &o, int nseg, const int4 *s_seg, const int (*s_uinf)[2], const PairDesc *s_pd,
    float4 (*s_j)[Op::JW][kSub], double (*s_red)[kPersistWarps][kGroup][Op::NA]) {
  constexpr int JW = Op::JW;
  constexpr int NA = Op::NA;
  constexpr int NW = kPersistWarps;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lrow = lane % kRowPairs, lg = lane / kRowPairs;
  const int la = s_seg[0].z - s_seg[0].y, lb = nseg > 1 ? s_seg[1].z - s_seg[1].y : 0;
  const int wb = (int)((long long)(la + lb) * warp / NW);
  const int we = (int)((long long)(la + lb) * (warp + 1) / NW);
#pragma unroll 1
  for (int g = 0; g < nseg; ++g) {
    const int off = g ? la : 0, len = g ? lb : la;
    const int lo = max(wb, off), hi = min(we, off + len);
    if (hi <= lo || !s_uinf[g][1]) {
      // no entries of this segment: a zero contribution to its warp-order sum
      if (lane < kGroup) {
#pragma unroll
        for (int a = 0; a < NA; ++a) s_red[g][warp][lane][a] = 0.0;
      }
      continue;
    }
    const int4 sg = s_seg[g];
    const int grp = s_uinf[g][0] >> 16;
    o.pd = &s_pd[g];  // the op reads descriptor 0 from shared memory from here on
    const int p = 0;
    typename Op::IData I0, I1;
    o.load_i(p, grp * kGroup + lrow, I0);
    o.load_i(p, grp * kGroup + kRowPairs + lrow, I1);
    float hi0[NA], lo0[NA], hi1[NA], lo1[NA];
#pragma unroll
    for (int a = 0; a < NA; ++a) hi0[a] = lo0[a] = hi1[a] = lo1[a] = 0.0f;
    const int jb = sg.y + (lo - off);
    const int je = sg.y + (hi - off);
    const int split = Op::kTwoSets ? o.set_boundary(p) : sg.z;
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
      // fold into the compensated sum every 4 sub-tiles (<= 32 plain FP32 terms
      // per lane) and after the last one
      if (((j0 - jb) & (4 * kSub - 1)) == 3 * kSub || j0 + kSub >= je) {
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          two_sum_acc(hi0[a], lo0[a], acc0[a]);
          two_sum_acc(hi1[a], lo1[a], acc1[a]);
        }
      }
    }
    // lane groups -> lanes 0..7 (fixed butterfly)
#pragma unroll
    for (int a = 0; a < NA; ++a) {
      double v0 = (double)hi0[a] + (double)lo0[a];
      double v1 = (double)hi1[a] + (double)lo1[a];
#pragma unroll
      for (int off2 = kRowPairs; off2 < 32; off2 <<= 1) {
        v0 += __shfl_xor_sync(0xffffffffu, v0, off2);
        v1 += __shfl_xor_sync(0xffffffffu, v1, off2);
      }
      if (lg == 0) {
        s_red[g][warp][lrow][a] = v0;
        s_red[g][warp][kRowPairs + lrow][a] = v1;
      }
    }
  }
}

// Loads the descriptors of the round starting at segment k (nseg segments) into the
// round slots.  Called by the whole CTA.
template <class Op>
__device__ __forceinline__ void persist_load_round(const Op &op, const int4 *segs,
                                                   const int2 *units, int k, int nseg,
                                                   int4 *s_seg, int (*s_uinf)[2],
                                                   PairDesc *s_pd) {
  __syncthreads();  // the previous round's epilogue is done with the round slots
  if (threadIdx.x < nseg) {
    const int4 sg = segs[k + threadIdx.x];
    const int2 un = units[sg.x];
    s_seg[threadIdx.x] = sg;
    s_uinf[threadIdx.x][0] = un.x | (un.y << 16);
    s_uinf[threadIdx.x][1] = op.active(un.x);
    s_pd[threadIdx.x] = op.pd[un.x];
  }
  __syncthreads();
}

// Op: the sweep interface of sweep.cuh plus set_step(t) (pointers of time step t) and
// write_group(p, k, v) (row-group partial of a kTileSum op).
// dir = +1 runs t = 0..T-1, dir = -1 runs t = T-1..0.
// Two CTAs per SM (<= 128 registers), 16 warps per SM.
template <class Op>
__global__ void __launch_bounds__(kPersistWarps * 32, 2)
    persistent_sweep_kernel(Op op, SweepPlan plan, int T, int dir, StepSync *sy) {
  constexpr int JW = Op::JW;
  constexpr int NA = Op::NA;
  constexpr int NW = kPersistWarps;
  static_assert(NA <= kPartNA, "partial slot too small");
  __shared__ float4 s_j[NW][JW][kSub];
  __shared__ double s_red[2][NW][kGroup][NA];  // [segment of the round][warp][row]
  __shared__ PairDesc s_pd[2];  // descriptors of the round's units
  __shared__ int s_uinf[2][2];  // per round slot: pair | group << 16, active
  __shared__ int4 s_seg[2];     // the round's segments
  pdl_wait();
  stamp_entry(sy, dir > 0 ? 0 : 1);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int s0 = plan.cta_seg[blockIdx.x], s1 = plan.cta_seg[blockIdx.x + 1];
  const bool one_round = s1 - s0 <= 2;  // descriptors loaded once for the whole launch
  for (int s = 0; s < T; ++s) {
    const int t = dir > 0 ? s : T - 1 - s;
    Op o = op;
    o.set_step(t);
    for (int k = s0; k < s1; k += 2) {
      const int nseg = min(2, s1 - k);
      if (!one_round || s == 0)
        persist_load_round(op, plan.segs, plan.units, k, nseg, s_seg, s_uinf, s_pd);
      persist_round(o, nseg, s_seg, s_uinf, s_pd, s_j, s_red);
      __syncthreads();
      // epilogue: segment e on lanes 0-15 of warp e (both segments at once); the
      // condition is uniform over those 16 lanes
      const int e = warp;
      if (e < nseg && lane < kGroup && s_uinf[e][1]) {
        const int4 se = s_seg[e];
        const int grp_e = s_uinf[e][0] >> 16;
        Op &oe = o;
        oe.pd = &s_pd[e];
        typename Op::FData F;  // finalize operands, in flight during the combine
        oe.fin_load(0, grp_e * kGroup + lane, F);
        double v[NA];
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          // all NW warps in warp order (zeros from warps without entries here); the
          // loads are independent of the running sum
          double x = 0.0;
#pragma unroll
          for (int w = 0; w < NW; ++w) x += s_red[e][w][lane][a];
          v[a] = x;
        }
        const int2 up = plan.unit_parts[se.x];
        bool fin = true;
        if (up.x > 1) {
          // row group cut over several CTAs: publish this part; the CTA completing the
          // count adds all parts in part order
          double *slot = plan.part + ((size_t)(up.y + se.w) * kGroup + lane) * kPartNA;
#pragma unroll
          for (int a = 0; a < NA; ++a) slot[a] = v[a];
          __syncwarp(0xffffu);  // the 16 lanes' part writes before lane 0's release
          int last = 0;
          if (lane == 0) {
            // release: this part is visible with the count; acquire: the last arriver
            // sees every other part
            last = atom_add_acq_rel_gpu(&plan.cnt[se.x], 1u) == (unsigned int)up.x - 1u;
            if (last) plan.cnt[se.x] = 0u;  // next step's arrivals come after the barrier
          }
          fin = __shfl_sync(0xffffu, last, 0) != 0;
          __syncwarp(0xffffu);
          if (fin) {
#pragma unroll
            for (int a = 0; a < NA; ++a) v[a] = 0.0;
            for (int q = 0; q < up.x; ++q) {
              const double *src = plan.part + ((size_t)(up.y + q) * kGroup + lane) * kPartNA;
#pragma unroll
              for (int a = 0; a < NA; ++a) v[a] += __ldcg(src + a);
            }
          }
        }
        if (fin) {
          double en = oe.finalize(0, grp_e * kGroup + lane, v, F);
          if (Op::kTileSum) {
#pragma unroll
            for (int off = kGroup / 2; off > 0; off >>= 1)
              en += __shfl_xor_sync(0xffffu, en, off);
            if (lane == 0) oe.write_group(0, grp_e, en);
          }
        }
      }
    }
    if (!grid_barrier(sy, (unsigned)(s + 1) * gridDim.x, (unsigned)s)) return;
  }
  grid_depart(sy);
  stamp_exit(sy, dir > 0 ? 0 : 1);
  pdl_trigger();
}

// ---------------------------------------------------------------------------------
// Cluster form of the persistent sweep.  The same rounds and pair arithmetic, but a
// row group is never cut across thread-block clusters: the host plan gives each
// cluster of C CTAs a contiguous range of whole row groups (balanced by work), and
// cuts only inside a cluster.  The parts of a row group split between CTAs of one
// cluster meet in distributed shared memory instead of L2:
//   * a CTA keeps the FP64 partial of a split segment in one of two shared slots (its
//     share's first and last segment are the only ones that can be split);
//   * after its rounds every CTA arrives (release, cluster scope) on the mbarrier of
//     every CTA of its cluster;
//   * the CTA holding a split row group's first part (its "job", at most one per CTA)
//     polls its mbarrier's phase (non-blocking test, acquire; bounded), reads the
//     parts from the owners' slots in part order and finalises the row group.
// A step's slots are rewritten only after the grid barrier, which every CTA reaches
// after its reads.  No L2 round trip, fence at GPU scope or arrival count remains
// between the pair arithmetic and the grid barrier.  All mbarrier waits are bounded
// (timeout: the error word, as for the grid barrier); the only unbounded waits are
// the hardware cluster barriers at entry (mbarriers initialised before any remote
// arrival) and exit (no CTA leaves while a peer may still read its slots), which
// every CTA executes exactly once on every path.

constexpr int kMaxJobParts = 8;  // parts of a row group: at most the cluster size

struct ClusterSweepPlan {
  const int2 *units;    // (pair, row group) per unit
  const int4 *segs;     // (unit, j begin, j end, kind) in CTA order; kind 0: a whole row
                        // group (finalised by its CTA), 1 / 2: a part kept in slot 0 / 1
  const int *cta_seg;   // CTA k owns segs[cta_seg[k] .. cta_seg[k + 1])
  const int2 *job;      // per CTA: (unit whose first part it holds, or -1; parts)
  const int *job_src;   // per CTA, kMaxJobParts entries: cluster rank << 1 | slot of part q
};

__device__ __forceinline__ unsigned int cluster_nctas() {
  unsigned int n;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(n));
  return n;
}

__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
               "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned int count) {
  const unsigned int a = (unsigned int)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrival on the mbarrier at the same shared address in cluster CTA `rank`.
__device__ __forceinline__ void mbar_arrive_cluster(unsigned long long *bar, unsigned int rank) {
  const unsigned int a = (unsigned int)__cvta_generic_to_shared(bar);
  unsigned int ra;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(a), "r"(rank));
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(ra)
               : "memory");
}

// Non-blocking test of the completion of the mbarrier phase with the given parity.
__device__ __forceinline__ bool mbar_test_parity(unsigned long long *bar, unsigned int parity) {
  const unsigned int a = (unsigned int)__cvta_generic_to_shared(bar);
  unsigned int ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0u;
}

template <class Op>
__global__ void __launch_bounds__(kPersistWarps * 32, 2)
    persistent_cluster_kernel(Op op, ClusterSweepPlan plan, int T, int dir, StepSync *sy) {
  constexpr int JW = Op::JW;
  constexpr int NA = Op::NA;
  constexpr int NW = kPersistWarps;
  __shared__ float4 s_j[NW][JW][kSub];
  __shared__ double s_red[2][NW][kGroup][NA];
  __shared__ double s_slot[2][kGroup][NA];  // partials of this CTA's split segments
  __shared__ PairDesc s_pd[2];
  __shared__ int s_uinf[2][2];
  __shared__ int4 s_seg[2];
  __shared__ __align__(8) unsigned long long s_bar;
  pdl_wait();
  stamp_entry(sy, dir > 0 ? 0 : 1);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) mbar_init(&s_bar, cluster_nctas());
  cluster_sync_all();  // every mbarrier initialised before the first remote arrival
  const int s0 = plan.cta_seg[blockIdx.x], s1 = plan.cta_seg[blockIdx.x + 1];
  const bool one_round = s1 - s0 <= 2;
  for (int s = 0; s < T; ++s) {
    const int t = dir > 0 ? s : T - 1 - s;
    Op o = op;
    o.set_step(t);
    for (int k = s0; k < s1; k += 2) {
      const int nseg = min(2, s1 - k);
      if (!one_round || s == 0)
        persist_load_round(op, plan.segs, plan.units, k, nseg, s_seg, s_uinf, s_pd);
      persist_round(o, nseg, s_seg, s_uinf, s_pd, s_j, s_red);
      __syncthreads();
      // epilogue: segment e on lanes 0-15 of warp e; a whole row group is finalised
      // here, a part goes to its slot
      const int e = warp;
      if (e < nseg && lane < kGroup && s_uinf[e][1]) {
        const int4 se = s_seg[e];
        const int grp_e = s_uinf[e][0] >> 16;
        Op oe = o;
        oe.pd = &s_pd[e];
        double v[NA];
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          double x = 0.0;
#pragma unroll
          for (int w = 0; w < NW; ++w) x += s_red[e][w][lane][a];
          v[a] = x;
        }
        if (se.w == 0) {
          double en = oe.finalize(0, grp_e * kGroup + lane, v);
          if (Op::kTileSum) {
#pragma unroll
            for (int off = kGroup / 2; off > 0; off >>= 1)
              en += __shfl_xor_sync(0xffffu, en, off);
            if (lane == 0) oe.write_group(0, grp_e, en);
          }
        } else {
#pragma unroll
          for (int a = 0; a < NA; ++a) s_slot[se.w - 1][lane][a] = v[a];
        }
      }
    }
    __syncthreads();  // this CTA's slots are written
    if (threadIdx.x < cluster_nctas()) {
      asm volatile("fence.acq_rel.cluster;" ::: "memory");
      mbar_arrive_cluster(&s_bar, threadIdx.x);
    }
    // the job (if any) is re-read here rather than kept in registers through the rounds
    const int2 job = warp == 0 ? plan.job[blockIdx.x] : make_int2(-1, 0);
    if (job.x >= 0) {
      // the parts of the split row group whose first part this CTA holds
      const int2 un = plan.units[job.x];
      const int job_pair = un.x, job_grp = un.y, row = job_grp * kGroup + lane;
      Op &oj = o;
      oj.pd = op.pd;  // global descriptors (the rounds pointed o.pd at the round slots)
      typename Op::FData F;  // finalize operands, in flight during the wait
      if (lane < kGroup) oj.fin_load(job_pair, row, F);
      unsigned int n = 0;
      bool ok = true;
      while (!mbar_test_parity(&s_bar, (unsigned int)(s & 1))) {
        if ((++n & 63u) == 0u) {
          if (ld_relaxed(&sy->error) != 0u || n > kSpinLimit) {
            atomicCAS(&sy->error, 0u, 3000u + (unsigned int)s);
            ok = false;
            break;
          }
          if (n > 4096u) __nanosleep(64);
        }
      }
      ok = __all_sync(0xffffffffu, ok);
      if (ok && lane < kGroup && oj.active(job_pair)) {
        double v[NA];
#pragma unroll
        for (int a = 0; a < NA; ++a) v[a] = 0.0;
        for (int q = 0; q < job.y; ++q) {
          const int src = plan.job_src[blockIdx.x * kMaxJobParts + q];
          const double *rem =
              cg::this_cluster().map_shared_rank(&s_slot[src & 1][lane][0], src >> 1);
#pragma unroll
          for (int a = 0; a < NA; ++a) v[a] += rem[a];
        }
        double en = oj.finalize(job_pair, row, v, F);
        if (Op::kTileSum) {
#pragma unroll
          for (int off = kGroup / 2; off > 0; off >>= 1)
            en += __shfl_xor_sync(0xffffu, en, off);
          if (lane == 0) oj.write_group(job_pair, job_grp, en);
        }
      }
    }
    if (!grid_barrier(sy, (unsigned)(s + 1) * gridDim.x, (unsigned)s)) break;
  }
  cluster_sync_all();  // no CTA leaves while a peer may still read its slots
  grid_depart(sy);
  stamp_exit(sy, dir > 0 ? 0 : 1);
  pdl_trigger();
}

}  // namespace lddmm
