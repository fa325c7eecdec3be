// BF16 GEMM on the 5th-generation tensor cores (tcgen05.mma, accumulator in TMEM) for
// the warm-start network.  No counterpart in the reference.
//
//   C[M x N] = A[M x K] . B[N x K]^T      A, B: BF16, K-major (K contiguous); C: FP32
//
// One CTA of 4 warps per 128-row tile of C and per K split (blockIdx.y); N <= 256 is
// one tile (one tcgen05.mma of shape 128 x N x 16 per 16 elements of K).  Operands are
// staged K-chunk by K-chunk (kKC elements) into shared memory in the canonical
// K-major layout without swizzle: "core matrices" of 8 rows x 16 bytes, core (g, c)
// (row group g, 8-element K group c) at byte (g * kKC / 8 + c) * 128, so the leading
// byte offset (next K group) is 128 and the stride byte offset (next row group) is
// kKC * 16.  Two stage buffers: while the MMAs of chunk i run, the CTA copies chunk
// i + 1 into the other buffer with cp.async (global -> shared without registers);
// thread 0 issues a chunk's MMAs and commits them to that buffer's mbarrier, and a
// buffer is restaged only after its mbarrier (bounded wait) says the MMAs reading it
// are done.  The epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM
// lanes 32w..32w+31 = rows of the tile), applies bias / GELU / GELU' and writes FP32,
// BF16 and transposed BF16 outputs as asked, four columns per store where the
// outputs are 16-byte (BF16: 8-byte) aligned.
//
// Shared-memory and instruction descriptor bit layouts follow the PTX ISA
// (tcgen05 "Shared memory descriptor", "Instruction descriptor" for kind::f16).
#pragma once

#include <cuda.h>  // CUtensorMap (the map is encoded on the host, see warmstart.cu)
#include <cuda_bf16.h>
#include <cstdint>

namespace lddmm {
namespace tc {

constexpr int kTileM = 128;
constexpr int kKC = 64;                        // K elements staged per chunk
constexpr int kGemmThreads = 128;
constexpr unsigned int kMbarSpin = 1u << 24;   // bounded wait on the MMA barrier

enum Epilogue : int {
  kEpiNone = 0,   // out = acc (+ bias)
  kEpiGelu = 1,   // pre = acc + bias (stored if asked), out = gelu(pre)
  kEpiDGelu = 2,  // out = acc * gelu'(pre_in)
};

struct GemmArgs {
  const __nv_bfloat16 *A;
  long long lda;  // A[m][k] = A[m * lda + k], m < M
  const __nv_bfloat16 *B;
  long long ldb;  // B[n][k] = B[n * ldb + k], n < N
  int M, N, K;    // N: multiple of 16, <= 256 (the MMA shape); K: multiple of 16
  int n_valid;    // columns written (<= N)
  int k_split;    // K elements per blockIdx.y (multiple of kKC)
  int epi;
  const float *bias;        // [n_valid] or null
  const float *pre_in;      // kEpiDGelu: [M][ld_pre_in]
  long long ld_pre_in;
  float *out;               // FP32 [M][ldo] (+ blockIdx.y * split_stride) or null
  long long ldo, split_stride;
  float *pre_out;           // kEpiGelu: FP32 pre-activation [M][ld_pre_out] or null
  long long ld_pre_out;
  __nv_bfloat16 *out_bf;    // BF16 [M][ldb_out] or null
  long long ldb_out;
  __nv_bfloat16 *out_bt;    // BF16 transposed [n][ldt_out] (column m) or null
  long long ldt_out;
  unsigned int *error;      // set to 1 when the MMA barrier wait gave up
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: start address >> 4 (bits 0-13), leading byte offset
// >> 4 (16-29), stride byte offset >> 4 (32-45), version 1 (46-47), base offset 0,
// layout type 0 = no swizzle (61-63).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// The same for a K-major operand in the 128-byte swizzled layout (rows of 64 BF16 =
// 128 bytes at 128-byte strides, 16-byte chunk c of row r stored at chunk c ^ (r & 7),
// 1024-byte aligned atoms of 8 rows): stride byte offset 1024 (next 8 rows), leading
// byte offset unused for this layout (16), layout type 2 (128-byte swizzle) in bits
// 61-63.  A K step of 16 elements inside the 64-element row advances the start address
// by 32 bytes; the unit applies the swizzle to the addresses it forms.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(16u >> 4) << 16) |
         ((uint64_t)(1024u >> 4) << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor, kind::f16: F32 accumulator (bits 4-5 = 1), A and B BF16
// (7-9 = 1, 10-12 = 1), both K-major (15, 16 = 0), N >> 3 (17-22), M >> 4 (24-28).
__host__ __device__ constexpr uint32_t instr_desc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t *mbar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(mbar))
      : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity) {
  const uint32_t a = smem_u32(mbar);
  for (unsigned int n = 0; n < kMbarSpin; ++n) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ float gelu(float x) {
  return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}

__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) +
         x * 0.39894228040143268f * __expf(-0.5f * x * x);
}

// 32 consecutive accumulator columns of this thread's TMEM lane, without waiting for
// the load (tcgen05.wait::ld before the registers are read).
__device__ __forceinline__ void tmem_ld32_async(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
      "[%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
}

// 32 consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
      "[%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Stage rows [r0, r0 + rows) x K elements [k0, k0 + kKC) of a K-major matrix into the
// canonical layout at `dst` with 16-byte cp.async copies (rows beyond `rmax` and K
// beyond `kmax` are zero-filled: source size 0, source address clamped to `src`).
// Callers guarantee 16-byte alignment: ld a multiple of 8 elements, k0 a multiple of 8.
__device__ __forceinline__ void stage_async(unsigned char *dst, const __nv_bfloat16 *src,
                                            long long ld, int r0, int rows, int rmax, int k0,
                                            int kmax) {
  constexpr int kChunks = kKC / 8;  // 16-byte groups per row
  for (int i = threadIdx.x; i < rows * kChunks; i += kGemmThreads) {
    const int r = i / kChunks, c = i - r * kChunks;
    const int gr = r0 + r, gk = k0 + c * 8;
    const bool ok = gr < rmax && gk < kmax;
    const __nv_bfloat16 *g = ok ? src + (long long)gr * ld + gk : src;
    const uint32_t d = smem_u32(dst + ((r >> 3) * kChunks + c) * 128 + (r & 7) * 16);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(g),
                 "r"(ok ? 16 : 0)
                 : "memory");
  }
}

// Epilogue of one 128-row tile: the accumulator (TMEM; the calling warp reads lane
// quadrant `quad`, lanes 32 quad .. 32 quad + 31 = rows m0 + 32 quad ..; a warp may
// only access the quadrant of its warp index mod 4) through bias / GELU / GELU' into
// the outputs of `g`; `out` is the FP32 output of this K split (or null).  Called by
// four warps covering the four quadrants after the tile's MMAs completed and
// tcgen05.fence::after_thread_sync.
__device__ __forceinline__ void gemm_epilogue(const GemmArgs &g, int m0, uint32_t tmem,
                                              float *out, int quad, int cbeg = 0,
                                              int cend = 1 << 30) {
  const int warp = quad, lane = threadIdx.x & 31;
  const int m = m0 + warp * 32 + lane;
  const bool row_ok = m < g.M;
  // four columns per store where every output in use allows it
  const bool vec =
      (!out || (((uintptr_t)out & 15u) == 0 && (g.ldo & 3) == 0)) &&
      (!g.pre_out || (((uintptr_t)g.pre_out & 15u) == 0 && (g.ld_pre_out & 3) == 0)) &&
      (!g.out_bf || (((uintptr_t)g.out_bf & 7u) == 0 && (g.ldb_out & 3) == 0)) &&
      (g.epi != kEpiDGelu ||
       (((uintptr_t)g.pre_in & 15u) == 0 && (g.ld_pre_in & 3) == 0));
  for (int c0 = cbeg; c0 < g.N && c0 < cend; c0 += 32) {
    float v[32];
    tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
    if (!row_ok) continue;
#pragma unroll
    for (int j = 0; j < 32; j += 4) {
      const int n = c0 + j;
      if (n >= g.n_valid) break;
      if (vec && n + 3 < g.n_valid) {
        float x[4] = {v[j], v[j + 1], v[j + 2], v[j + 3]};
        if (g.bias) {  // the bias sits at any offset of the parameter vector
#pragma unroll
          for (int q = 0; q < 4; ++q) x[q] += g.bias[n + q];
        }
        if (g.epi == kEpiGelu) {
          if (g.pre_out)
            *reinterpret_cast<float4 *>(g.pre_out + (size_t)m * g.ld_pre_out + n) =
                make_float4(x[0], x[1], x[2], x[3]);
#pragma unroll
          for (int q = 0; q < 4; ++q) x[q] = gelu(x[q]);
        } else if (g.epi == kEpiDGelu) {
          const float4 pi =
              *reinterpret_cast<const float4 *>(g.pre_in + (size_t)m * g.ld_pre_in + n);
          x[0] *= gelu_grad(pi.x); x[1] *= gelu_grad(pi.y);
          x[2] *= gelu_grad(pi.z); x[3] *= gelu_grad(pi.w);
        }
        if (out)
          *reinterpret_cast<float4 *>(out + (size_t)m * g.ldo + n) =
              make_float4(x[0], x[1], x[2], x[3]);
        if (g.out_bf || g.out_bt) {
          __nv_bfloat16 h[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) h[q] = __float2bfloat16_rn(x[q]);
          if (g.out_bf) {
            uint2 pk;
            pk.x = (uint32_t)__bfloat16_as_ushort(h[0]) |
                   ((uint32_t)__bfloat16_as_ushort(h[1]) << 16);
            pk.y = (uint32_t)__bfloat16_as_ushort(h[2]) |
                   ((uint32_t)__bfloat16_as_ushort(h[3]) << 16);
            *reinterpret_cast<uint2 *>(g.out_bf + (size_t)m * g.ldb_out + n) = pk;
          }
          if (g.out_bt)
#pragma unroll
            for (int q = 0; q < 4; ++q) g.out_bt[(size_t)(n + q) * g.ldt_out + m] = h[q];
        }
        continue;
      }
      for (int q = 0; q < 4 && n + q < g.n_valid; ++q) {
        const int nn = n + q;
        float x = v[j + q];
        if (g.bias) x += g.bias[nn];
        if (g.epi == kEpiGelu) {
          if (g.pre_out) g.pre_out[(size_t)m * g.ld_pre_out + nn] = x;
          x = gelu(x);
        } else if (g.epi == kEpiDGelu) {
          x *= gelu_grad(g.pre_in[(size_t)m * g.ld_pre_in + nn]);
        }
        if (out) out[(size_t)m * g.ldo + nn] = x;
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        if (g.out_bf) g.out_bf[(size_t)m * g.ldb_out + nn] = h;
        if (g.out_bt) g.out_bt[(size_t)nn * g.ldt_out + m] = h;
      }
    }
  }
}

__global__ void __launch_bounds__(kGemmThreads, 1) gemm_bf16_kernel(GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const size_t stage_bytes = (size_t)(kTileM + g.N) * kKC * 2;
  // stage buffer b: A tile (kTileM x kKC bf16) at smem + b * stage_bytes, B tile
  // (N x kKC bf16) right after it
  auto sA = [&](int b) { return smem + (size_t)b * stage_bytes; };
  auto sB = [&](int b) { return smem + (size_t)b * stage_bytes + kTileM * kKC * 2; };
  __shared__ uint64_t s_mbar[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_ok;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kTileM;
  const int kb = blockIdx.y * g.k_split, ke = min(g.K, kb + g.k_split);
  const int nk = ke > kb ? (ke - kb + kKC - 1) / kKC : 0;
  const uint32_t ncols = g.N <= 32 ? 32u : g.N <= 64 ? 64u : g.N <= 128 ? 128u : 256u;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_ok = 1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const uint32_t idesc = instr_desc_bf16(kTileM, g.N);
  // MMA chunk j committed to s_mbar[j & 1]; each commit is waited exactly once, in
  // order per barrier, with parity (j >> 1) & 1
  auto wait_mma = [&](int j) {
    if (!mbar_wait(&s_mbar[j & 1], (uint32_t)((j >> 1) & 1))) {
      s_ok = 0;
      if (g.error) atomicExch(g.error, 1u);
    }
  };
  auto issue = [&](int buf, int k0) {
    stage_async(sA(buf), g.A, g.lda, m0, kTileM, g.M, k0, ke);
    stage_async(sB(buf), g.B, g.ldb, 0, g.N, g.N, k0, ke);
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  if (nk > 0) issue(0, kb);
  int done = -1;   // last MMA chunk waited for
  int issued = 0;  // MMA chunks committed
  for (int i = 0; i < nk; ++i) {
    if (i + 1 < nk) {
      // the other buffer was read by chunk i - 1: wait for its MMAs, then refill it
      if (i >= 1) {
        wait_mma(i - 1);
        done = i - 1;
        __syncthreads();
        if (!s_ok) break;
      }
      issue((i + 1) & 1, kb + (i + 1) * kKC);
      asm volatile("cp.async.wait_group 1;" ::: "memory");  // chunk i has landed
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(sA(i & 1)), b0 = smem_u32(sB(i & 1));
#pragma unroll
      for (int s = 0; s < kKC / 16; ++s) {
        // K step s covers K groups 2s and 2s + 1 (start advances by 2 core matrices)
        const uint64_t da = smem_desc(a0 + s * 256, 128, kKC * 16);
        const uint64_t db = smem_desc(b0 + s * 256, 128, kKC * 16);
        mma_bf16(tmem, da, db, idesc, (i == 0 && s == 0) ? 0u : 1u);
      }
      mma_commit(&s_mbar[i & 1]);
    }
    ++issued;
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  // the remaining commits, oldest first
  for (int j = done + 1; j < issued; ++j) wait_mma(j);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (s_ok && issued > 0)
    gemm_epilogue(g, m0, tmem, g.out ? g.out + (size_t)blockIdx.y * g.split_stride : nullptr,
                  warp);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

// Weight-resident form for the common case of one K split with K <= kResK and
// N <= 256 (every layer of the warm-start network): persistent CTAs, one per SM, loop
// over 128-row tiles (tile = blockIdx.x + i * gridDim.x).  B (the weights, at most
// 128 KB) is staged into shared memory once; A streams through kResStages cp.async
// buffers in a global sequence of (tile, K-chunk) steps, a buffer refilled only after
// the mbarrier of the MMAs that read it completed; the loads of the next tile's first
// chunks are in flight while a tile's epilogue runs.  Every MMA commit is waited
// exactly once, in order (wait_upto), with bounded waits.
constexpr int kResK = 256;
constexpr int kResStages = 3;

__global__ void __launch_bounds__(kGemmThreads, 1) gemm_bf16_resident_kernel(GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int nk = (g.K + kKC - 1) / kKC;                     // K chunks per tile
  const size_t b_chunk = (size_t)g.N * kKC * 2;             // bytes of one B chunk
  unsigned char *sBres = smem;                               // nk B chunks
  unsigned char *sAst = smem + (size_t)nk * b_chunk;         // kResStages A chunks
  __shared__ uint64_t s_mbar[kResStages];
  __shared__ uint32_t s_tmem;
  __shared__ int s_ok;
  const int warp = threadIdx.x >> 5;
  const int ntiles = (g.M + kTileM - 1) / kTileM;
  const int my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int Q = my_tiles * nk;                               // (tile, chunk) steps
  const uint32_t ncols = g.N <= 32 ? 32u : g.N <= 64 ? 64u : g.N <= 128 ? 128u : 256u;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    for (int b = 0; b < kResStages; ++b)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar[b])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_ok = 1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const uint32_t idesc = instr_desc_bf16(kTileM, g.N);
  // B, all K chunks, one cp.async group (it completes before every later group)
  for (int kc = 0; kc < nk; ++kc)
    stage_async(sBres + kc * b_chunk, g.B, g.ldb, 0, g.N, g.N, kc * kKC, g.K);
  asm volatile("cp.async.commit_group;" ::: "memory");
  auto issue_a = [&](int q) {  // step q: tile blockIdx.x + (q / nk) gridDim.x, chunk q % nk
    const int tile = blockIdx.x + (q / nk) * gridDim.x;
    stage_async(sAst + (size_t)(q % kResStages) * kTileM * kKC * 2, g.A, g.lda, tile * kTileM,
                kTileM, g.M, (q % nk) * kKC, g.K);
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  int waited = 0;  // MMA steps 0 .. waited - 1 are complete
  auto wait_upto = [&](int j) {
    for (; waited <= j; ++waited)
      if (!mbar_wait(&s_mbar[waited % kResStages], (uint32_t)((waited / kResStages) & 1))) {
        s_ok = 0;
        if (g.error) atomicExch(g.error, 1u);
      }
  };
  for (int q = 0; q < kResStages - 1 && q < Q; ++q) issue_a(q);
  int issued = 0;
  for (int q = 0; q < Q; ++q) {
    // A chunk q has landed once at most the groups of the chunks after it are pending
    const int pending = min(Q - 1, q + kResStages - 2) - q;
    if (pending >= 1)
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    else
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    const int kc = q % nk;
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(sAst + (size_t)(q % kResStages) * kTileM * kKC * 2);
      const uint32_t b0 = smem_u32(sBres + kc * b_chunk);
#pragma unroll
      for (int s = 0; s < kKC / 16; ++s) {
        const uint64_t da = smem_desc(a0 + s * 256, 128, kKC * 16);
        const uint64_t db = smem_desc(b0 + s * 256, 128, kKC * 16);
        mma_bf16(tmem, da, db, idesc, (kc == 0 && s == 0) ? 0u : 1u);
      }
      mma_commit(&s_mbar[q % kResStages]);
    }
    ++issued;
    // refill the buffer of step q - 1 with step q + kResStages - 1 once its MMAs are done
    if (q + kResStages - 1 < Q) {
      if (q >= 1) wait_upto(q - 1);
      __syncthreads();
      if (!s_ok) break;
      issue_a(q + kResStages - 1);
    }
    if (kc == nk - 1) {
      // the tile's accumulation is complete once its last commit is
      wait_upto(q);
      __syncthreads();
      if (!s_ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      gemm_epilogue(g, (blockIdx.x + (q / nk) * gridDim.x) * kTileM, tmem, g.out, warp);
      // the next tile's first MMA overwrites the accumulator
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  wait_upto(issued - 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

inline size_t gemm_resident_smem_bytes(int N, int K) {
  const int nk = (K + kKC - 1) / kKC;
  return (size_t)nk * N * kKC * 2 + (size_t)kResStages * kTileM * kKC * 2;
}

// Dynamic shared memory of gemm_bf16_kernel for N columns (two stage buffers).
inline size_t gemm_smem_bytes(int N) { return 2 * (size_t)(kTileM + N) * kKC * 2; }

// ---------------------------------------------------------------------------------
// Warp-specialised weight-resident form (one K split, K <= kResK, N <= 256): the
// layers of the warm-start network move ~250 MB per hidden-layer product and do
// little arithmetic per byte, so the kernel is built to keep HBM busy: loads, MMAs and
// the epilogue of different tiles overlap.  One persistent CTA per SM, 10 warps:
//   warp 0   producer: the weights once, then the A chunks of its tiles, by TMA
//            (cp.async.bulk.tensor, no multicast: this GPU's memory only), into
//            kWsStages stage buffers; a buffer is refilled after the MMAs reading it
//            have committed to its "empty" mbarrier;
//   warp 1   MMA issuer (one thread): tcgen05.mma into one of two TMEM accumulators
//            (tile i uses accumulator i & 1), commit to the buffer's "empty" barrier
//            per chunk and to the accumulator's "full" barrier per tile;
//   warps 2-9 epilogue: tile i's accumulator through gemm_epilogue (warp w reads TMEM
//            lane quadrant w & 3, half of the columns) while tile i + 1 accumulates into
//            the other one, then release it on its "empty" barrier.
// Operands are loaded as 128-byte swizzled K-major tiles: one TMA box of 64 K-elements
// (one 128-byte segment of each row) x 128 rows per A stage, one box of 64 x N per
// 64-element chunk of the weights, so every row segment is a single 128-byte request
// (boxes 8 elements wide, in the canonical layout without swizzle, cost one 16-byte
// request per row and held the A stream back).  Out-of-range rows and K elements are
// zero-filled by the TMA unit.
// The epilogue has 8 warps, two per TMEM lane quadrant, each taking half the columns,
// so that enough TMEM loads are in flight (with 4 warps the epilogue waited on them,
// long-scoreboard stalls, and held the kernel at ~43 % of DRAM bandwidth).
// A plain FP32 output (no activation, at most a bias) leaves through TMA stores: each
// epilogue warp writes its 32 rows x 32 columns into a 4 KB staging buffer in the
// 128-byte swizzled layout (16-byte chunk k of row r at chunk k ^ (r & 7):
// conflict-free) and one lane stores the block with cp.async.bulk.tensor, so HBM sees
// whole 128-byte rows instead of one 16-byte piece per row per instruction; the buffer
// is rewritten after the store has read it (bulk wait_group.read).  Every mbarrier
// wait is bounded (error word); before freeing TMEM the producer waits (bounded) for
// its loads in flight, the MMA thread for its last MMAs and the epilogue lanes for
// their stores.
constexpr int kWsMaxStages = 4;
constexpr int kWsEpiWarps = 8;
constexpr int kWsThreads = 32 * (2 + kWsEpiWarps);
constexpr int kWsStageC = 32 * 32 * 4;  // one epilogue staging buffer (bytes)

__device__ __forceinline__ void mbar_init_n(uint64_t *mbar, uint32_t n) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(n));
}

__device__ __forceinline__ void mbar_arrive1(uint64_t *mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)),
               "r"(bytes)
               : "memory");
}

// TMA store of the box at (x = column, y = row) of a 2D tensor map from src (bulk
// group of the calling thread).  x is a multiple of 4 FP32 columns (16 bytes), y >= 0.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, int x, int y,
                                             const void *src) {
  asm volatile(
      "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(map),
      "r"(x), "r"(y), "r"(smem_u32(src))
      : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// TMA load of the box at (x = K element, y = row) of a 2D tensor map into dst.  x is a
// multiple of 8 elements (16 bytes).
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            uint64_t *mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(mbar))
      : "memory");
}

// Dynamic shared memory of gemm_bf16_ws_kernel: the weights and the A stages, and at
// least 120 KB, so that one CTA runs per SM and its two accumulators (up to 512 TMEM
// columns) never compete with another CTA's for the SM's tensor memory.
// A stages of gemm_bf16_ws_kernel that fit next to the weights (and the epilogue
// staging buffers when the output leaves through TMA stores): up to kWsMaxStages,
// at least 2.
inline int gemm_ws_stages(int N, int K, bool tma_store) {
  const int nk = (K + kKC - 1) / kKC;
  const size_t fixed =
      (size_t)nk * kKC * N * 2 + (tma_store ? kWsEpiWarps * kWsStageC : 0) + 2048;
  const size_t cap = 227 * 1024 - 1024;  // the per-CTA limit less the static barriers
  int st = kWsMaxStages;
  while (st > 2 && fixed + (size_t)st * kTileM * kKC * 2 > cap) --st;
  return st;
}

inline size_t gemm_ws_smem_bytes(int N, int K, bool tma_store) {
  const int nk = (K + kKC - 1) / kKC;
  const size_t need = (size_t)nk * kKC * N * 2 +
                      (size_t)gemm_ws_stages(N, K, tma_store) * kTileM * kKC * 2 +
                      (tma_store ? kWsEpiWarps * kWsStageC : 0) + 1024;  // + alignment
  return need > (size_t)120 * 1024 ? need : (size_t)120 * 1024;
}

// Epilogue of one 128-row tile through TMA stores (plain FP32 output, optional bias):
// warp quadrant `quad`, rows m0 + 32 quad + lane, columns [cbeg, cend) in 32-column
// blocks.  `cstage`: the warp's staging buffer (1024-byte aligned); `nst`: stores
// issued so far by this warp.
__device__ __forceinline__ void gemm_epilogue_tma(const GemmArgs &g, const CUtensorMap *tmC,
                                                  int m0, uint32_t tmem, int quad, int cbeg,
                                                  int cend, unsigned char *cstage, int &nst) {
  const int lane = threadIdx.x & 31;
  const int row0 = m0 + quad * 32;
  const uint32_t tq = tmem + ((uint32_t)(quad * 32) << 16);
  cend = min(cend, g.n_valid);
  // two 32-column blocks per TMEM round trip
  for (int c0 = cbeg; c0 < cend; c0 += 64) {
    const bool two = c0 + 32 < cend;
    uint32_t r[2][32];
    tmem_ld32_async(tq + (uint32_t)c0, r[0]);
    if (two) tmem_ld32_async(tq + (uint32_t)(c0 + 32), r[1]);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    if (row0 >= g.M) continue;  // a quadrant wholly below the matrix stores nothing
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (h == 1 && !two) break;
      const int cb = c0 + 32 * h;
      float v[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[h][j]);
      if (g.bias) {
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (cb + j < g.n_valid) v[j] += g.bias[cb + j];
      }
      unsigned char *buf = cstage;
      if (nst >= 1 && lane == 0)  // the previous store has read the buffer
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
      __syncwarp();
#pragma unroll
      for (int k = 0; k < 8; ++k)
        *reinterpret_cast<float4 *>(buf + lane * 128 + ((k ^ (lane & 7)) << 4)) =
            make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) tma_store_2d(tmC, cb, row0, buf);
      ++nst;
    }
  }
}

__global__ void __launch_bounds__(kWsThreads, 1)
    gemm_bf16_ws_kernel(GemmArgs g, const __grid_constant__ CUtensorMap tmA,
                        const __grid_constant__ CUtensorMap tmB,
                        const __grid_constant__ CUtensorMap tmC, int tma_store, int stages) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint64_t s_full[kWsMaxStages], s_empty[kWsMaxStages], s_accf[2], s_acce[2],
      s_bfull, s_mdone;
  __shared__ uint32_t s_tmem;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = (g.K + kKC - 1) / kKC;
  const uint32_t b_chunk = (uint32_t)g.N * 128;  // bytes of one 64-element K chunk of B
  const int kWsStages = stages;  // A stage buffers (<= kWsMaxStages)
  constexpr uint32_t kStageBytes = kTileM * kKC * 2;
  // every tile 1024-byte aligned (the 128-byte swizzle repeats every 8 rows of 128
  // bytes): the weights, the A stages, then the epilogue staging buffers
  unsigned char *sB = smem + ((1024u - (smem_u32(smem) & 1023u)) & 1023u);
  unsigned char *sA = sB + (size_t)nk * b_chunk;
  unsigned char *sC = sA + (size_t)stages * kStageBytes;
  const int ntiles = (g.M + kTileM - 1) / kTileM;
  const int my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint32_t nacc = g.N <= 32 ? 32u : g.N <= 64 ? 64u : g.N <= 128 ? 128u : 256u;
  const uint32_t ncols = 2 * nacc;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    for (int b = 0; b < kWsStages; ++b) {
      mbar_init_n(&s_full[b], 1);
      mbar_init_n(&s_empty[b], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init_n(&s_accf[b], 1);
      mbar_init_n(&s_acce[b], kWsEpiWarps);  // one arrival per epilogue warp
    }
    mbar_init_n(&s_bfull, 1);
    mbar_init_n(&s_mdone, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  auto fail = [&]() {
    if (g.error) atomicExch(g.error, 1u);
  };
  const int Q = my_tiles * nk;  // (tile, K chunk) steps of this CTA
  if (warp == 0) {
    if (lane == 0) {
      mbar_expect_tx(&s_bfull, (uint32_t)nk * b_chunk);
      for (int c = 0; c < nk; ++c) tma_load_2d(sB + (size_t)c * b_chunk, &tmB, c * kKC, 0, &s_bfull);
      int q = 0;
      for (; q < Q; ++q) {
        const int st = q % kWsStages;
        if (!mbar_wait(&s_empty[st], (uint32_t)(((q / kWsStages) & 1) ^ 1))) {
          fail();
          break;
        }
        mbar_expect_tx(&s_full[st], kStageBytes);
        const int row = (blockIdx.x + (q / nk) * gridDim.x) * kTileM;
        const int k0 = (q % nk) * kKC;
        tma_load_2d(sA + (size_t)st * kStageBytes, &tmA, k0, row, &s_full[st]);
      }
      // the loads in flight complete before the CTA leaves (bounded)
      for (int r = (q > kWsStages ? q - kWsStages : 0); r < q; ++r)
        if (!mbar_wait(&s_full[r % kWsStages], (uint32_t)((r / kWsStages) & 1))) fail();
      if (!mbar_wait(&s_bfull, 0u)) fail();
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = instr_desc_bf16(kTileM, g.N);
      bool ok = mbar_wait(&s_bfull, 0u);
      if (!ok) fail();
      for (int i = 0; ok && i < my_tiles; ++i) {
        const int acc = i & 1;
        if (!mbar_wait(&s_acce[acc], (uint32_t)(((i >> 1) & 1) ^ 1))) {
          fail();
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)acc * nacc;
        for (int kc = 0; kc < nk; ++kc) {
          const int q = i * nk + kc, st = q % kWsStages;
          if (!mbar_wait(&s_full[st], (uint32_t)((q / kWsStages) & 1))) {
            fail();
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a0 = smem_u32(sA + (size_t)st * kStageBytes);
          const uint32_t b0 = smem_u32(sB + (size_t)kc * b_chunk);
#pragma unroll
          for (int s = 0; s < kKC / 16; ++s) {
            const uint64_t da = smem_desc_sw128(a0 + s * 32);
            const uint64_t db = smem_desc_sw128(b0 + s * 32);
            mma_bf16(d, da, db, idesc, (kc == 0 && s == 0) ? 0u : 1u);
          }
          mma_commit(&s_empty[st]);
        }
        if (ok) mma_commit(&s_accf[acc]);
      }
      // every MMA issued has completed before TMEM is freed (bounded)
      mma_commit(&s_mdone);
      if (!mbar_wait(&s_mdone, 0u)) fail();
    }
  } else {
    const int quad = warp & 3;  // TMEM lane quadrant this warp may read
    // the two warps of a quadrant take the first and the second half of the columns
    const int half = (warp - 2) >> 2;
    const int ch = (g.N / 2 + 31) / 32 * 32;
    const int cbeg = half * ch, cend = half ? g.N : ch;
    unsigned char *cstage = sC + (size_t)(warp - 2) * kWsStageC;
    int nst = 0;  // TMA stores issued by this warp
    for (int i = 0; i < my_tiles; ++i) {
      const int acc = i & 1;
      if (!mbar_wait(&s_accf[acc], (uint32_t)((i >> 1) & 1))) {
        fail();
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int m0 = (blockIdx.x + i * gridDim.x) * kTileM;
      if (tma_store)
        gemm_epilogue_tma(g, &tmC, m0, tmem + (uint32_t)acc * nacc, quad, cbeg, cend, cstage,
                          nst);
      else
        gemm_epilogue(g, m0, tmem + (uint32_t)acc * nacc, g.out, quad, cbeg, cend);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive1(&s_acce[acc]);
    }
    // the stores have finished before the CTA leaves
    if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    __syncwarp();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

}  // namespace tc
}  // namespace lddmm
