// tc_mlp.cuh — the surrogate network's forward pass on the 5th-generation
// tensor cores (tcgen05): 128-row tiles, operands in shared memory in the
// canonical no-swizzle K-major layout, FP32 accumulators in tensor memory.
//
// One CTA of 512 threads owns one SM (217 KB of shared memory) and walks
// tiles of 128 rows. Per tile:
//   features (FP64 -> standardised BF16, rows 0..127 by threads 0..127)
//   L1  D[128x256]  = X0[128x16]  W1^T      1 MMA  (W1 resident)
//   L2  D           = A1[128x256] W2^T     16 MMAs (W2 streamed from L2)
//   L3  D           = A2          W3^T     16 MMAs (W3 streamed from L2)
//   L4  D4[128x16]  = A3          W4^T     16 MMAs (W4 resident)
// with the bias + SiLU + BF16 epilogues read from tensor memory by all 16
// warps (warp w reads lanes 32 (w % 4).., columns 64 (w / 4)..). One
// thread issues the MMAs and commits them to an mbarrier that every thread
// waits on for at most WAIT_NS of the global timer. When a wait runs out
// anywhere in the CTA, the whole CTA stops walking tiles: it sets the error
// word, commits once more so that the barrier tracks every MMA it issued,
// waits for that (bounded again) and for its own asynchronous copies, and
// frees its tensor memory before it returns.
#pragma once
#include <cuda_bf16.h>

#include "mlp.cuh"

namespace ostc {
namespace tc {

using mlp::KIN;
using mlp::NH;
using mlp::NOUTP;

constexpr int ROWS = 128;
constexpr int THREADS = 512;
// shared memory map (bytes)
constexpr unsigned SM_ACT = 0;                       // 128 x 256 bf16
constexpr unsigned SM_W = SM_ACT + ROWS * NH * 2;    // 256 x 256 bf16 (W2 or W3)
constexpr unsigned SM_W1 = SM_W + NH * NH * 2;       // 256 x 16 bf16
constexpr unsigned SM_W4 = SM_W1 + NH * KIN * 2;     // 16 x 256 bf16
constexpr unsigned SM_X0 = SM_W4 + NOUTP * NH * 2;   // 128 x 16 bf16
constexpr unsigned SM_BIAS = SM_X0 + ROWS * KIN * 2;  // b1, b2, b3 (FP32), b4 (16)
constexpr unsigned SM_IO = SM_BIAS + (3 * NH + NOUTP) * 4;  // tables of the Io (IO_BYTES)
constexpr unsigned IO_BYTES = 2048;
constexpr unsigned SM_BAR = SM_IO + IO_BYTES;  // mbarrier (8 B)
constexpr unsigned SM_TMEM = SM_BAR + 8;             // allocated tensor-memory base (4 B)
constexpr unsigned SM_BYTES = SM_TMEM + 8;
constexpr unsigned TMEM_COLS = 512;
constexpr unsigned long long WAIT_NS = 1000000000ull;  // 1 s of the global timer per mbarrier wait

// byte offset of element (r, k) of an R x K operand in the canonical K-major
// no-swizzle layout: 8 x 16-byte core matrices, K-adjacent cores 128 B apart
// (leading byte offset), 8-row groups K/8 * 128 B apart (stride byte offset)
__device__ __forceinline__ unsigned core_off(int r, int k, int K) {
  return (unsigned)(((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor (tcgen05): start, LBO, SBO in 16-byte
// units, descriptor version 1, no swizzle
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr, unsigned lbo, unsigned sbo) {
  return (unsigned long long)((addr >> 4) & 0x3FFF) | ((unsigned long long)((lbo >> 4) & 0x3FFF) << 16) |
         ((unsigned long long)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor: BF16 x BF16 -> F32, both K-major, M = 128, N
__host__ __device__ constexpr unsigned idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(n >> 3) << 17) | ((unsigned)(128 >> 4) << 24);
}

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mma_issue(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned idesc,
                                          unsigned accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(unsigned bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// bounded wait for the mbarrier phase `parity`; false when WAIT_NS ran out
__device__ __forceinline__ bool bar_wait(unsigned bar, unsigned parity) {
  const unsigned long long t0 = global_ns();
  for (unsigned it = 0;; ++it) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 31) == 31 && global_ns() - t0 > WAIT_NS) return false;
  }
}

// 32 consecutive FP32 columns of this thread's lane (no wait: tmem_wait_ld)
__device__ __forceinline__ void tmem_ld32_async(unsigned taddr, unsigned *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 32 consecutive FP32 columns of this thread's lane
__device__ __forceinline__ void tmem_ld32(unsigned taddr, float *v) {
  unsigned r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(unsigned taddr, float *v) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ unsigned pack_bf16(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *(const unsigned *)&h;
}

__device__ __forceinline__ void cp_async16(unsigned dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prior1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// copy a row-major global N x K bf16 matrix into the canonical layout; each
// CTA starts at its own offset, so the SMs that stream the same weights at
// the same time spread over the L2 slices instead of queueing on one line
__device__ __forceinline__ void load_weights(unsigned char *smem, unsigned off, const __nv_bfloat16 *w, int N, int K) {
  const int chunks = N * K / 8;
  const int rot = (int)((blockIdx.x * 613u) % (unsigned)chunks);
  for (int i = threadIdx.x; i < chunks; i += THREADS) {
    const int c = i + rot < chunks ? i + rot : i + rot - chunks;
    const int n = c / (K / 8), kc = c % (K / 8);
    cp_async16(smem_u32(smem + off + core_off(n, kc * 8, K)), w + (long long)n * K + kc * 8);
  }
}

// The network core. `Io` supplies
//   void setup(unsigned char *tables)          fills IO_BYTES of shared memory
//                                              (all threads, once per CTA)
// and, per tile, with Io::kPacked false
//   bool load(int tile, int row, float *x12)   standardised features of a row
//                                              (threads 0..127); false: no row
// or with Io::kPacked true
//   void stage(int tile, unsigned char *x0)    all threads: the tile's rows,
//                                              already standardised BF16, into
//                                              the operand layout (cp.async)
// and
//   void store(int tile, int row, const float *y10)   standardised outputs
// Returns nothing; errors go to *err (1 = a wait ran out).
template <typename Io>
__device__ void mlp_tiles(const mlp::Net &net, int n_tiles, Io &io, int *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned bar = smem_u32(smem + SM_BAR);
  unsigned *tmem_slot = (unsigned *)(smem + SM_TMEM);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // resident weights and biases
  load_weights(smem, SM_W1, net.w1(), NH, KIN);
  load_weights(smem, SM_W4, net.w4(), NOUTP, NH);
  float *sbias = (float *)(smem + SM_BIAS);
  for (int c = tid; c < NH; c += THREADS) {
    sbias[c] = net.b1()[c];
    sbias[NH + c] = net.b2()[c];
    sbias[2 * NH + c] = net.b3()[c];
  }
  if (tid < NOUTP) sbias[3 * NH + tid] = net.b4()[tid];
  io.setup(smem + SM_IO);
  cp_async_wait_all();
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const unsigned tmem = *tmem_slot;
  const unsigned tmem_d4 = tmem + NH;  // columns 256..271
  unsigned parity = 0;
  bool timed_out = false;  // CTA-uniform: a bounded wait ran out somewhere in the CTA
  const int row = (warp & 3) * 32 + lane;   // the TMEM lane this thread reads
  const int col0 = (warp >> 2) * (NH / 4);  // first of its 64 columns
  const unsigned lane_addr = (unsigned)((warp & 3) * 32) << 16;

  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    if constexpr (Io::kPacked) {
      // the tile's feature rows first, then W2, which streams during layer 1
      io.stage(tile, smem + SM_X0);
      cp_async_commit();
      load_weights(smem, SM_W, net.w2(), NH, NH);
      cp_async_commit();
      cp_async_wait_prior1();
    } else {
    // stream W2 while the features and layer 1 run
    load_weights(smem, SM_W, net.w2(), NH, NH);
    if (tid < ROWS) {
      float x[12];
      const bool has = io.load(tile, tid, x);
      float xs[16];
#pragma unroll
      for (int i = 0; i < 12; ++i) xs[i] = has ? x[i] : 0.f;
#pragma unroll
      for (int i = 12; i < 16; ++i) xs[i] = 0.f;
      *(uint4 *)(smem + SM_X0 + core_off(tid, 0, KIN)) = make_uint4(
          pack_bf16(xs[0], xs[1]), pack_bf16(xs[2], xs[3]), pack_bf16(xs[4], xs[5]), pack_bf16(xs[6], xs[7]));
      *(uint4 *)(smem + SM_X0 + core_off(tid, 8, KIN)) = make_uint4(
          pack_bf16(xs[8], xs[9]), pack_bf16(xs[10], xs[11]), pack_bf16(xs[12], xs[13]), pack_bf16(xs[14], xs[15]));
    }
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    if (tid == 0) {
      mma_issue(tmem, smem_desc(smem_u32(smem + SM_X0), 128, 2 * 128), smem_desc(smem_u32(smem + SM_W1), 128, 2 * 128),
                idesc_bf16(NH), 0);
      // net.withhold_commit (a diagnostic of the timeout path): no completion
      // signal for this product, so the wait below runs out
      if (!net.withhold_commit) mma_commit(bar);
    }
    for (int layer = 0; layer < 3; ++layer) {
      if (__syncthreads_or(!bar_wait(bar, parity))) {
        timed_out = true;
        break;
      }
      parity ^= 1;
      fence_after();
      if (layer == 1) load_weights(smem, SM_W, net.w3(), NH, NH);  // W2 is no longer read
      // epilogue: bias + SiLU -> BF16 activations (the next layer's A operand)
      const float *b = sbias + layer * NH;
      // both 32-column loads in flight before the one wait
      unsigned acc[NH / 4];
      tmem_ld32_async(tmem + lane_addr + col0, acc);
      tmem_ld32_async(tmem + lane_addr + col0 + 32, acc + 32);
      tmem_wait_ld();
#pragma unroll
      for (int q = 0; q < NH / 4; q += 8) {
        const float4 b0 = *(const float4 *)(b + col0 + q), b1 = *(const float4 *)(b + col0 + q + 4);
        const float bb[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
        unsigned w4[4];
#pragma unroll
        for (int e = 0; e < 8; e += 2) {
          const float z0 = __uint_as_float(acc[q + e]) + bb[e], z1 = __uint_as_float(acc[q + e + 1]) + bb[e + 1];
          w4[e / 2] = pack_bf16(__fdividef(z0, 1.0f + __expf(-z0)), __fdividef(z1, 1.0f + __expf(-z1)));
        }
        *(uint4 *)(smem + SM_ACT + core_off(row, col0 + q, NH)) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
      }
      cp_async_wait_all();
      fence_async_smem();
      fence_before();
      __syncthreads();
      fence_after();
      if (tid == 0) {
        const unsigned a0 = smem_u32(smem + SM_ACT);
        const unsigned w0 = smem_u32(smem + (layer < 2 ? SM_W : SM_W4));
        const unsigned d = layer < 2 ? tmem : tmem_d4;
        const unsigned id = idesc_bf16(layer < 2 ? NH : NOUTP);
        for (int s = 0; s < NH / 16; ++s)
          mma_issue(d, smem_desc(a0 + s * 256, 128, NH * 16), smem_desc(w0 + s * 256, 128, NH * 16), id, s > 0);
        mma_commit(bar);
      }
    }
    if (timed_out || __syncthreads_or(!bar_wait(bar, parity))) {
      timed_out = true;
      break;
    }
    parity ^= 1;
    fence_after();
    if (warp < 4) {
      float v[16], y[10];
      tmem_ld16(tmem_d4 + lane_addr, v);
#pragma unroll
      for (int i = 0; i < 10; ++i) y[i] = v[i] + sbias[3 * NH + i];
      io.store(tile, row, y);
    }
    fence_before();
    __syncthreads();
    fence_after();
  }
  if (timed_out) {
    // drain: one more commit tracks every MMA this CTA issued; wait for it
    // (bounded) and for the CTA's own weight copies before the memory goes
    if (tid == 0) {
      mma_commit(bar);
      if (err) atomicExch(err, 1);
    }
    bar_wait(bar, parity);
    cp_async_wait_all();
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

// rows of 16 standardised BF16 features (12 and 4 zeros, 32 bytes, the
// operand's K) in; rows of 10 FP32 outputs out
struct PackedIo {
  static constexpr bool kPacked = true;
  const __nv_bfloat16 *x;
  float *y;
  int n;
  __device__ void setup(unsigned char *) {}
  __device__ void stage(int tile, unsigned char *x0) const {
    for (int c = threadIdx.x; c < 2 * ROWS; c += THREADS) {
      const int row = c >> 1, half = c & 1;
      const long long q = (long long)tile * ROWS + row;
      unsigned char *dst = x0 + core_off(row, half * 8, KIN);
      if (q < n)
        cp_async16(smem_u32(dst), x + q * KIN + half * 8);
      else
        *(uint4 *)dst = make_uint4(0, 0, 0, 0);
    }
  }
  __device__ void store(int tile, int row, const float *o) const {
    const long long q = (long long)tile * ROWS + row;
    if (q >= n) return;
    float2 *d = (float2 *)(y + q * mlp::NOUT);
#pragma unroll
    for (int i = 0; i < mlp::NOUT / 2; ++i) d[i] = make_float2(o[2 * i], o[2 * i + 1]);
  }
};

}  // namespace tc
}  // namespace ostc
