// gemm_tc.cuh — the training GEMM of the chemistry surrogate on the 5th-generation
// tensor cores: C[M][N] (+)= A[M][K] B[N][K]^T with BF16 operands stored K-major
// (row-major, K contiguous), FP32 accumulation in tensor memory.
//
// One CTA of 256 threads owns 128 rows of C (all N <= 256 columns) and a
// slice of K. K moves through shared memory in chunks of 64 (two stages):
// every thread copies its share of the chunk's A and B rows into the
// canonical no-swizzle K-major layout with 16-byte cp.async (rows of A past M
// are zero-filled), one thread issues the chunk's MMAs (tcgen05.mma kind::f16,
// M = 128, N, K = 16 each) and commits them to the stage's mbarrier, which is
// waited on (bounded by the global timer) before the stage is refilled. The
// copies of chunk c + 1 are issued before chunk c's are waited for, so they
// overlap that wait and chunk c's MMAs. The epilogue reads the accumulators
// with tcgen05.ld (warp w: rows 32 (w % 4) .. + 31, half w / 4 of the
// columns, 32 at a time), turns each 32 x 32 block around in shared memory so
// that a warp writes one row's 32 columns per instruction, and either stores
// C (+ bias, with the BF16 SiLU activation) or adds it atomically (split-K
// over blockIdx.y). A wait that runs out sets the
// error word; the CTA then waits (bounded) for the MMAs it issued, frees its
// tensor memory and returns.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "tc_mlp.cuh"

namespace ostc {
namespace mlp {

struct TcGemmArgs {
  const __nv_bfloat16 *a;  // [M][lda], K contiguous; rows 16-byte aligned
  const __nv_bfloat16 *b;  // [N][ldb], K contiguous; rows 16-byte aligned
  float *c;                // [M][ldc]
  int lda, ldb, ldc;
  int M, N, K;             // N % 16 == 0, 16 <= N <= 256, K % 16 == 0
  int k_per_split;         // K of one blockIdx.y (a multiple of TC_BK)
  const float *bias;       // per column, or null (stored results only)
  __nv_bfloat16 *act;      // bf16 silu(C) [M][ldc], or null
  int atomic;              // add into C (C pre-zeroed) instead of storing
  int *err;                // set when a bounded wait ran out
};

constexpr int TC_BK = 64;                               // K of one chunk
constexpr int TC_THREADS = 256;
constexpr unsigned TC_A_BYTES = 128 * TC_BK * 2;        // 16 KB
constexpr unsigned TC_B_BYTES = 256 * TC_BK * 2;        // 32 KB (N <= 256)
constexpr unsigned TC_STAGE = TC_A_BYTES + TC_B_BYTES;  // 48 KB
constexpr unsigned TC_SMEM = 2 * TC_STAGE + 32;         // two stages, two mbarriers, the TMEM slot

__device__ __forceinline__ void cp_async16_zfill(unsigned dst, const void *src, unsigned src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ float silu_tc(float z) { return z / (1.0f + __expf(-z)); }

__global__ void __launch_bounds__(TC_THREADS, 1) gemm_tc_kernel(TcGemmArgs g) {
  extern __shared__ __align__(1024) unsigned char sm[];
  using namespace tc;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned base = smem_u32(sm);
  const unsigned bar[2] = {base + 2 * TC_STAGE, base + 2 * TC_STAGE + 8};
  unsigned *tmem_slot = (unsigned *)(sm + 2 * TC_STAGE + 16);
  const unsigned ncols = g.N <= 32 ? 32u : (g.N <= 64 ? 64u : (g.N <= 128 ? 128u : 256u));
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar[0]));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar[1]));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const unsigned tmem = *tmem_slot;
  const int m0 = blockIdx.x * 128;
  const int kb = blockIdx.y * g.k_per_split;
  const int ke = min(g.K, kb + g.k_per_split);
  const int nchunks = ke > kb ? (ke - kb + TC_BK - 1) / TC_BK : 0;
  const unsigned idesc = idesc_bf16(g.N);
  unsigned phase[2] = {0u, 0u};
  bool pending[2] = {false, false};
  bool late = false;
  // copies of chunk c into stage c & 1 (one cp.async group per chunk)
  auto load = [&](int c) {
    const int s = c & 1;
    const int k0 = kb + c * TC_BK, kc = min(TC_BK, ke - k0);
    const unsigned sa = base + s * TC_STAGE, sb = sa + TC_A_BYTES;
    const int q = kc / 8;  // 16-byte pieces per row
    for (int i = tid; i < 128 * q; i += TC_THREADS) {
      const int r = i / q, kq = i - r * q;
      const bool ok = m0 + r < g.M;
      const __nv_bfloat16 *src = g.a + (long long)(ok ? m0 + r : 0) * g.lda + k0 + kq * 8;
      cp_async16_zfill(sa + core_off(r, kq * 8, TC_BK), src, ok ? 16u : 0u);
    }
    for (int i = tid; i < g.N * q; i += TC_THREADS) {
      const int n = i / q, kq = i - n * q;
      cp_async16(sb + core_off(n, kq * 8, TC_BK), g.b + (long long)n * g.ldb + k0 + kq * 8);
    }
    cp_async_commit();
  };
  if (nchunks > 0) load(0);
  for (int c = 0; c < nchunks; ++c) {
    const int s = c & 1, s1 = s ^ 1;
    // the next chunk's copies go out before this chunk's are waited for; its
    // stage is free once the MMAs of chunk c - 1 that read it have completed
    if (c + 1 < nchunks) {
      if (pending[s1]) {
        if (bar_wait(bar[s1], phase[s1])) {
          phase[s1] ^= 1u;
          pending[s1] = false;
        } else {
          late = true;
        }
        if (__syncthreads_or(late)) break;
      }
      load(c + 1);
      cp_async_wait_prior1();  // chunk c's group has landed
    } else {
      cp_async_wait_all();
    }
    fence_async_smem();  // the copies (generic proxy) before the MMAs' reads (async proxy)
    __syncthreads();
    if (tid == 0) {
      fence_after();
      const int kc = min(TC_BK, ke - (kb + c * TC_BK));
      const unsigned sa = base + s * TC_STAGE, sb = sa + TC_A_BYTES;
      for (int ks = 0; ks < kc / 16; ++ks) {
        // K-adjacent core matrices 128 B apart, 8-row groups TC_BK / 8 * 128 B apart
        const unsigned long long ad = smem_desc(sa + ks * 256, 128, (TC_BK / 8) * 128);
        const unsigned long long bd = smem_desc(sb + ks * 256, 128, (TC_BK / 8) * 128);
        mma_issue(tmem, ad, bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
      }
      mma_commit(bar[s]);
    }
    pending[s] = true;
  }
  cp_async_wait_all();  // no copy outlives the loop (a timed-out CTA leaves it early)
  // the MMAs still in flight (bounded again after a timeout)
  for (int s = 0; s < 2; ++s)
    if (pending[s]) {
      if (bar_wait(bar[s], phase[s]))
        phase[s] ^= 1u;
      else
        late = true;
    }
  late = __syncthreads_or(late);
  fence_after();
  if (late) {
    if (tid == 0) atomicExch(g.err, 1);
  } else if (nchunks > 0) {
    // the stages are free (every MMA has completed): warp w turns its blocks
    // around in a 32 x 33 float tile of its own
    // (warps w and w + 4 read the same 32 accumulator lanes, each half of the columns)
    float *tile = reinterpret_cast<float *>(sm) + warp * 32 * 33;
    const int quarter = warp & 3, half = warp >> 2;
    const int r0 = m0 + quarter * 32;
    const int cb = g.N <= 32 ? (half ? g.N : 0) : half * ((g.N / 2 + 31) / 32 * 32);
    const int ce = g.N <= 32 ? (half ? g.N : g.N) : min(g.N, cb + (g.N / 2 + 31) / 32 * 32);
    for (int c0 = cb; c0 < ce; c0 += 32) {
      const int w = min(32, g.N - c0);  // 16 for a last block of 16 columns
      float v[32];
      if (w == 32)
        tmem_ld32(tmem + ((unsigned)(quarter * 32) << 16) + (unsigned)c0, v);
      else
        tmem_ld16(tmem + ((unsigned)(quarter * 32) << 16) + (unsigned)c0, v);
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (j < w) tile[lane * 33 + j] = v[j];
      __syncwarp();
      if (lane < w) {
        const float bias = (!g.atomic && g.bias) ? g.bias[c0 + lane] : 0.f;
        for (int r = 0; r < 32 && r0 + r < g.M; ++r) {
          const long long o = (long long)(r0 + r) * g.ldc + c0 + lane;
          const float x = tile[r * 33 + lane];
          if (g.atomic) {
            atomicAdd(g.c + o, x);
          } else {
            const float y = x + bias;
            g.c[o] = y;
            if (g.act) g.act[o] = __float2bfloat16_rn(silu_tc(y));
          }
        }
      }
      __syncwarp();
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

// host launcher: grid (ceil(M / 128), splits); shapes and alignment checked here
inline cudaError_t gemm_tc(const TcGemmArgs &a0, int splits, cudaStream_t s) {
  TcGemmArgs a = a0;
  if (a.N % 16 || a.N < 16 || a.N > 256 || a.K % 16 || a.K <= 0 || a.M <= 0 || a.lda % 8 || a.ldb % 8 ||
      (reinterpret_cast<uintptr_t>(a.a) & 15) || (reinterpret_cast<uintptr_t>(a.b) & 15) || !a.err)
    return cudaErrorInvalidValue;
  splits = splits < 1 ? 1 : splits;
  a.k_per_split = ((a.K + splits - 1) / splits + TC_BK - 1) / TC_BK * TC_BK;
  const int z = (a.K + a.k_per_split - 1) / a.k_per_split;
  a.atomic = z > 1 ? 1 : a.atomic;
  static bool attr = false;
  if (!attr) {
    const cudaError_t e = cudaFuncSetAttribute(gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  gemm_tc_kernel<<<dim3((a.M + 127) / 128, z), TC_THREADS, TC_SMEM, s>>>(a);
  return cudaGetLastError();
}

}  // namespace mlp
}  // namespace ostc
