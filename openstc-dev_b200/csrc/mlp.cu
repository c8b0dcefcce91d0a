// mlp.cu — the network of the chemistry surrogate and its training.
//
// The surrogate maps the standardised features of one cell state (log T,
// log p, nine transformed mass fractions, log dt: 12 inputs) to the
// standardised increments of the FP64 point-implicit integrator (nine dY_k
// and dT: 10 outputs) through a 12-256-256-256-10 perceptron with SiLU
// activations. Weights and activations are BF16, products accumulate in
// FP32, and training keeps FP32 master weights with Adam.
//
// Training runs on hand-written kernels only:
//   gemm_tc_kernel       C = A B^T on the tcgen05 tensor cores (gemm_tc.cuh:
//                        BF16 K-major operands, FP32 accumulators in tensor
//                        memory): the forward products X W^T with a fused
//                        bias + SiLU + BF16 epilogue, the input gradients
//                        dZ W (against the transposed weights) and the weight
//                        gradients dZ^T X (against the transposed gradients
//                        and activations, split over the batch with FP32
//                        atomics);
//   transpose / loss / SiLU-backward / column-sum / Adam kernels for the rest.
// gemm_bf16_kernel (mma.sync m16n8k16, generic strides) serves the
// reference forward of ostc_surrogate_forward.
// The fused inference kernel of the hot path (tcgen05, TMEM accumulators)
// lives in surrogate.cuh and reads the BF16 weights kept here.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/ostc.h"
#include "gemm_tc.cuh"
#include "mlp.cuh"
#include "tc_mlp.cuh"

namespace ostc {
namespace mlp {

// ---------------------------------------------------------------------------
// generic BF16 GEMM on mma.sync: C[m][n] (+)= sum_k A(m,k) B(n,k)
// A(m,k) = a[m*a_sm + k*a_sk], B(n,k) = b[n*b_sn + k*b_sk]; C row-major ldc
// ---------------------------------------------------------------------------
constexpr int BM = 128, BN = 128, BK = 32;
constexpr int PAD = 8;  // bf16 elements of row padding in shared memory

struct GemmArgs {
  const __nv_bfloat16 *a;
  long long a_sm, a_sk;
  const __nv_bfloat16 *b;
  long long b_sn, b_sk;
  float *c;
  long long ldc;
  int M, N, K;
  int k_per_split;     // K range of one blockIdx.z
  const float *bias;   // per column, or null
  __nv_bfloat16 *act;  // bf16 silu(C) (row-major ldc), or null
  int atomic;          // accumulate with atomicAdd (split-K; C pre-zeroed)
};

__device__ __forceinline__ void mma_bf16(float *d, const unsigned *a, const unsigned *b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }

__global__ void __launch_bounds__(256) gemm_bf16_kernel(GemmArgs g) {
  __shared__ __align__(16) __nv_bfloat16 As[BM][BK + PAD];
  __shared__ __align__(16) __nv_bfloat16 Bs[BN][BK + PAD];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps, each 64 x 32
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int kb = blockIdx.z * g.k_per_split;
  const int ke = min(g.K, kb + g.k_per_split);
  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  for (int k0 = kb; k0 < ke; k0 += BK) {
    // stage the tiles; consecutive threads walk the operand's unit-stride axis
    for (int e = tid; e < BM * BK; e += 256) {
      int m, k;
      if (g.a_sk == 1) {
        k = e % BK;
        m = e / BK;
      } else {
        m = e % BM;
        k = e / BM;
      }
      const int gm = m0 + m, gk = k0 + k;
      As[m][k] = (gm < g.M && gk < ke) ? g.a[gm * g.a_sm + gk * g.a_sk] : zero;
    }
    for (int e = tid; e < BN * BK; e += 256) {
      int n, k;
      if (g.b_sk == 1) {
        k = e % BK;
        n = e / BK;
      } else {
        n = e % BN;
        k = e / BN;
      }
      const int gn = n0 + n, gk = k0 + k;
      Bs[n][k] = (gn < g.N && gk < ke) ? g.b[gn * g.b_sn + gk * g.b_sk] : zero;
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < BK; ks += 16) {
      const int gr = lane >> 2, tq = lane & 3;
      unsigned af[4][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = wm * 64 + i * 16 + gr;
        af[i][0] = *(const unsigned *)&As[r][ks + 2 * tq];
        af[i][1] = *(const unsigned *)&As[r + 8][ks + 2 * tq];
        af[i][2] = *(const unsigned *)&As[r][ks + 2 * tq + 8];
        af[i][3] = *(const unsigned *)&As[r + 8][ks + 2 * tq + 8];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = wn * 32 + j * 8 + gr;
        bfr[j][0] = *(const unsigned *)&Bs[c][ks + 2 * tq];
        bfr[j][1] = *(const unsigned *)&Bs[c][ks + 2 * tq + 8];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bfr[j]);
    }
    __syncthreads();
  }
  // epilogue: c0,c1 at (row gr, cols 2tq, 2tq+1); c2,c3 at row gr+8
  const int gr = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int m = m0 + wm * 64 + i * 16 + gr + 8 * h;
        if (m >= g.M) continue;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int n = n0 + wn * 32 + j * 8 + 2 * tq + e;
          if (n >= g.N) continue;
          float v = acc[i][j][2 * h + e];
          if (g.atomic) {
            atomicAdd(&g.c[m * g.ldc + n], v);
          } else {
            if (g.bias) v += g.bias[n];
            g.c[m * g.ldc + n] = v;
            if (g.act) g.act[m * g.ldc + n] = __float2bfloat16_rn(silu(v));
          }
        }
      }
}

cudaError_t gemm(const GemmArgs &a0, int splits, cudaStream_t s) {
  GemmArgs a = a0;
  splits = splits < 1 ? 1 : splits;
  a.k_per_split = ((a.K + splits - 1) / splits + BK - 1) / BK * BK;
  const int z = (a.K + a.k_per_split - 1) / a.k_per_split;
  a.atomic = splits > 1 ? 1 : a.atomic;
  dim3 grid((a.N + BN - 1) / BN, (a.M + BM - 1) / BM, z);
  gemm_bf16_kernel<<<grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// elementwise kernels
// ---------------------------------------------------------------------------
// standardised FP32 inputs [n][12] -> BF16 [n][16] (columns 12..15 zero)
__global__ void pack_inputs_kernel(const float *x, int n, __nv_bfloat16 *x0) {
  const long long e = blockIdx.x * 256ll + threadIdx.x;
  if (e >= (long long)n * KIN) return;
  const long long r = e / KIN, c = e % KIN;
  x0[e] = c < NIN ? __float2bfloat16_rn(x[r * NIN + c]) : __float2bfloat16(0.f);
}

// dZ4 = 2 (Z4 - Y) / (n * 10) on the 10 outputs (0 on the padding), and the loss
__global__ void loss_grad_kernel(const float *z4, const float *y, int n, float *dz, __nv_bfloat16 *dzb,
                                 float *loss_sum) {
  const long long e = blockIdx.x * 256ll + threadIdx.x;
  float l = 0.f;
  if (e < (long long)n * NOUTP) {
    const long long r = e / NOUTP, c = e % NOUTP;
    float d = 0.f;
    if (c < NOUT) {
      const float diff = z4[e] - y[r * NOUT + c];
      l = diff * diff;
      d = 2.f * diff / ((float)n * NOUT);
    }
    dz[e] = d;
    dzb[e] = __float2bfloat16_rn(d);
  }
  // block sum of the squared errors
  __shared__ float red[256];
  red[threadIdx.x] = l;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss_sum, red[0]);
}

// dZ = dA * silu'(Z), FP32 and BF16 copies
__global__ void silu_backward_kernel(const float *da, const float *z, long long count, float *dz,
                                     __nv_bfloat16 *dzb) {
  const long long e = blockIdx.x * 256ll + threadIdx.x;
  if (e >= count) return;
  const float zz = z[e];
  const float sg = 1.0f / (1.0f + __expf(-zz));
  const float d = da[e] * sg * (1.0f + zz * (1.0f - sg));
  dz[e] = d;
  dzb[e] = __float2bfloat16_rn(d);
}

// out[c][b] = in[b][c] for b < rows, 0 for rows <= b < ldo (a K-major operand
// with its K padded to a multiple of 16); 32 x 32 tiles through shared memory
__global__ void transpose_bf16_kernel(const __nv_bfloat16 *in, int rows, int cols, int ldi, __nv_bfloat16 *out,
                                      int ldo) {
  __shared__ __nv_bfloat16 t[32][33];
  const int b0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int b = b0 + r, c = c0 + threadIdx.x;
    t[r][threadIdx.x] = (b < rows && c < cols) ? in[(long long)b * ldi + c] : __float2bfloat16_rn(0.f);
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int c = c0 + r, b = b0 + threadIdx.x;
    if (c < cols && b < ldo) out[(long long)c * ldo + b] = t[threadIdx.x][r];
  }
}

// db[c] = sum_r dz[r][c] over n rows (one CTA per column block of 32)
// blockIdx.y takes rows y, y + gridDim.y * 8, ... in 8 streams; the CTA's
// column sums are added into db (pre-zeroed)
__global__ void colsum_kernel(const float *dz, int n, int ncol, float *db) {
  const int c = blockIdx.x * 32 + (threadIdx.x & 31);
  const int rs = threadIdx.x >> 5;  // 8 row streams
  const int step = 8 * gridDim.y;
  float s = 0.f;
  if (c < ncol)
    for (int r = blockIdx.y * 8 + rs; r < n; r += step) s += dz[(long long)r * ncol + c];
  __shared__ float red[8][32];
  red[rs][threadIdx.x & 31] = s;
  __syncthreads();
  if (rs == 0 && c < ncol) {
    float t = 0.f;
    for (int q = 0; q < 8; ++q) t += red[q][threadIdx.x & 31];
    atomicAdd(db + c, t);
  }
}

// Adam on the FP32 master parameters; refreshes the BF16 copy (padding stays 0)
__global__ void adam_kernel(float *w, const float *g, float *m, float *v, __nv_bfloat16 *wb, const unsigned char *mask,
                            long long count, float lr, float b1t, float b2t) {
  const long long e = blockIdx.x * 256ll + threadIdx.x;
  if (e >= count) return;
  if (!mask[e]) return;
  constexpr float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float gg = g[e];
  const float mm = b1 * m[e] + (1 - b1) * gg;
  const float vv = b2 * v[e] + (1 - b2) * gg * gg;
  m[e] = mm;
  v[e] = vv;
  const float mh = mm / (1 - b1t), vh = vv / (1 - b2t);
  const float nw = w[e] - lr * mh / (sqrtf(vh) + eps);
  w[e] = nw;
  if (wb) wb[e] = __float2bfloat16_rn(nw);
}

__global__ void to_bf16_kernel(const float *w, long long count, __nv_bfloat16 *wb) {
  const long long e = blockIdx.x * 256ll + threadIdx.x;
  if (e < count) wb[e] = __float2bfloat16_rn(w[e]);
}

unsigned blocks(long long n) { return (unsigned)((n + 255) / 256); }

// the tensor-core forward on standardised rows (x [n][12] -> y [n][10])
struct RawIo {
  static constexpr bool kPacked = false;
  const float *x;
  float *y;
  int n;
  __device__ void setup(unsigned char *) {}
  __device__ bool load(int tile, int row, float *f) const {
    const long long q = (long long)tile * tc::ROWS + row;
    if (q >= n) return false;
#pragma unroll
    for (int i = 0; i < NIN; ++i) f[i] = x[q * NIN + i];
    return true;
  }
  __device__ void store(int tile, int row, const float *o) const {
    const long long q = (long long)tile * tc::ROWS + row;
    if (q >= n) return;
#pragma unroll
    for (int i = 0; i < NOUT; ++i) y[q * NOUT + i] = o[i];
  }
};

__global__ void __launch_bounds__(tc::THREADS, 1) surrogate_raw_kernel(Net net, const float *x, float *y, int n,
                                                                        int *err) {
  RawIo io{x, y, n};
  tc::mlp_tiles(net, (n + tc::ROWS - 1) / tc::ROWS, io, err);
}

}  // namespace mlp
}  // namespace ostc

using namespace ostc;
using namespace ostc::mlp;

// ---------------------------------------------------------------------------
// the surrogate object
// ---------------------------------------------------------------------------
struct ostc_surrogate {
  Net net;  // device parameters (mlp.cuh); net.wf is the FP32 master below
  int max_batch = 0;
  int step = 0;
  // FP32 masters / gradients / Adam moments over one flat padded buffer
  float *master = nullptr, *grad = nullptr, *mom1 = nullptr, *mom2 = nullptr;
  unsigned char *mask = nullptr;  // 1 where the padded slot is a real parameter
  // activations of a training batch
  __nv_bfloat16 *x0 = nullptr, *a[3] = {nullptr, nullptr, nullptr}, *dzb[4] = {nullptr, nullptr, nullptr, nullptr};
  float *z[4] = {nullptr, nullptr, nullptr, nullptr}, *dz[4] = {nullptr, nullptr, nullptr, nullptr};
  float *da = nullptr, *loss = nullptr;
  // K-major operands of the backward GEMMs: transposed gradients and
  // activations ([256][batch padded to 16]) and transposed weights of layers 2..4
  __nv_bfloat16 *tg = nullptr, *ta = nullptr, *wt = nullptr;
  int *err = nullptr;  // set by a tensor-core kernel whose bounded wait ran out
  Checks *checks = nullptr;  // device copy of the acceptance tests
  int *list = nullptr, *count = nullptr;
  int list_cap = 0;
  // the learned chemistry step's per-state buffers (list_cap states)
  __nv_bfloat16 *cx = nullptr;
  float *cy = nullptr;
  unsigned char *cenv = nullptr;
  std::vector<void *> owned;
};

namespace {

cudaError_t dalloc(ostc_surrogate *s, void **p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaSuccess) {
    s->owned.push_back(*p);
    e = cudaMemset(*p, 0, bytes);
  }
  return e;
}

// logical (unpadded) flat order of the ABI: W1[256][12] b1 W2 b2 W3 b3 W4[10][256] b4[10]
template <typename F>
void for_each_param(F &&f) {
  long long q = 0;
  for (int r = 0; r < NH; ++r)
    for (int c = 0; c < NIN; ++c) f(q++, OFF_W1 + (long long)r * KIN + c);
  for (int r = 0; r < NH; ++r) f(q++, OFF_B1 + r);
  for (int r = 0; r < NH * NH; ++r) f(q++, OFF_W2 + r);
  for (int r = 0; r < NH; ++r) f(q++, OFF_B2 + r);
  for (int r = 0; r < NH * NH; ++r) f(q++, OFF_W3 + r);
  for (int r = 0; r < NH; ++r) f(q++, OFF_B3 + r);
  for (int r = 0; r < NOUT; ++r)
    for (int c = 0; c < NH; ++c) f(q++, OFF_W4 + (long long)r * NH + c);
  for (int r = 0; r < NOUT; ++r) f(q++, OFF_B4 + r);
}

#define SK(expr)                                 \
  do {                                           \
    cudaError_t e_ = (expr);                     \
    if (e_ != cudaSuccess) return OSTC_ERR_CUDA; \
  } while (0)

ostc_status refresh_bf16(ostc_surrogate *s, cudaStream_t st) {
  to_bf16_kernel<<<blocks(NPAR), 256, 0, st>>>(s->master, NPAR, s->net.wb);
  SK(cudaGetLastError());
  return OSTC_OK;
}

// forward of n standardised rows (x0 packed): z[0..3], a[0..2] (tcgen05)
ostc_status forward(ostc_surrogate *s, int n, cudaStream_t st) {
  const Net &w = s->net;
  const __nv_bfloat16 *in[4] = {s->x0, s->a[0], s->a[1], s->a[2]};
  const __nv_bfloat16 *wl[4] = {w.w1(), w.w2(), w.w3(), w.w4()};
  const float *bl[4] = {w.b1(), w.b2(), w.b3(), w.b4()};
  for (int l = 0; l < 4; ++l) {
    TcGemmArgs g{};
    const int k = l == 0 ? KIN : NH, nn = l == 3 ? NOUTP : NH;
    g.a = in[l], g.lda = k, g.b = wl[l], g.ldb = k;
    g.c = s->z[l], g.ldc = nn, g.M = n, g.N = nn, g.K = k, g.bias = bl[l], g.act = l < 3 ? s->a[l] : nullptr;
    g.err = s->err;
    SK(gemm_tc(g, 1, st));
  }
  return OSTC_OK;
}

// the generic mma.sync forward (the reference of the tensor-core paths' tests)
ostc_status forward_reference(ostc_surrogate *s, int n, cudaStream_t st) {
  const Net &w = s->net;
  GemmArgs g{};
  // layer 1: Z1 = X0 W1^T + b1
  g.a = s->x0, g.a_sm = KIN, g.a_sk = 1;
  g.b = w.w1(), g.b_sn = KIN, g.b_sk = 1;
  g.c = s->z[0], g.ldc = NH, g.M = n, g.N = NH, g.K = KIN, g.bias = w.b1(), g.act = s->a[0];
  SK(gemm(g, 1, st));
  for (int l = 1; l < 3; ++l) {
    g.a = s->a[l - 1], g.a_sm = NH, g.a_sk = 1;
    g.b = l == 1 ? w.w2() : w.w3(), g.b_sn = NH, g.b_sk = 1;
    g.c = s->z[l], g.ldc = NH, g.M = n, g.N = NH, g.K = NH, g.bias = l == 1 ? w.b2() : w.b3(), g.act = s->a[l];
    SK(gemm(g, 1, st));
  }
  g.a = s->a[2], g.a_sm = NH, g.a_sk = 1;
  g.b = w.w4(), g.b_sn = NH, g.b_sk = 1;
  g.c = s->z[3], g.ldc = NOUTP, g.M = n, g.N = NOUTP, g.K = NH, g.bias = w.b4(), g.act = nullptr;
  SK(gemm(g, 1, st));
  return OSTC_OK;
}

// gradients of the mean squared error into s->grad (padded layout); loss sum in s->loss
ostc_status backward(ostc_surrogate *s, const float *y, int n, cudaStream_t st) {
  const Net &w = s->net;
  SK(cudaMemsetAsync(s->loss, 0, sizeof(float), st));
  SK(cudaMemsetAsync(s->grad, 0, sizeof(float) * NPAR, st));
  loss_grad_kernel<<<blocks((long long)n * NOUTP), 256, 0, st>>>(s->z[3], y, n, s->dz[3], s->dzb[3], s->loss);
  SK(cudaGetLastError());
  const int np = (n + 15) / 16 * 16;  // the batch as a K, padded with zero columns
  const __nv_bfloat16 *acts[4] = {s->x0, s->a[0], s->a[1], s->a[2]};
  const int kin[4] = {KIN, NH, NH, NH}, nout[4] = {NH, NH, NH, NOUTP};
  const long long offw[4] = {OFF_W1, OFF_W2, OFF_W3, OFF_W4}, offb[4] = {OFF_B1, OFF_B2, OFF_B3, OFF_B4};
  const __nv_bfloat16 *wl[4] = {w.w1(), w.w2(), w.w3(), w.w4()};
  const dim3 tb(32, 8);
  for (int l = 3; l >= 0; --l) {
    // weight gradient dW[n_out][k_in] = sum_b dZ[b][n_out] A[b][k_in]: dZ^T and A^T
    // as K-major operands, split over the batch so that about two CTAs per SM run
    transpose_bf16_kernel<<<dim3((np + 31) / 32, (nout[l] + 31) / 32), tb, 0, st>>>(s->dzb[l], n, nout[l], nout[l],
                                                                                   s->tg, np);
    SK(cudaGetLastError());
    transpose_bf16_kernel<<<dim3((np + 31) / 32, (kin[l] + 31) / 32), tb, 0, st>>>(acts[l], n, kin[l], kin[l], s->ta,
                                                                                  np);
    SK(cudaGetLastError());
    TcGemmArgs g{};
    g.a = s->tg, g.lda = np, g.b = s->ta, g.ldb = np;
    g.c = s->grad + offw[l], g.ldc = kin[l], g.M = nout[l], g.N = kin[l], g.K = np, g.atomic = 1;
    g.err = s->err;
    const int mt = (nout[l] + 127) / 128;
    const int splits = std::max(1, std::min(np / 1024, 296 / mt));
    SK(gemm_tc(g, splits, st));
    colsum_kernel<<<dim3((nout[l] + 31) / 32, std::max(1, std::min(n / 64, 256))), 256, 0, st>>>(
        s->dz[l], n, nout[l], s->grad + offb[l]);
    SK(cudaGetLastError());
    if (l == 0) break;
    // input gradient dA[b][k] = sum_n dZ[b][n] W[n][k], against W^T [k_in][n_out]
    __nv_bfloat16 *wt = s->wt + (long long)(l - 1) * NH * NH;
    transpose_bf16_kernel<<<dim3((nout[l] + 31) / 32, (kin[l] + 31) / 32), tb, 0, st>>>(wl[l], nout[l], kin[l],
                                                                                       kin[l], wt, nout[l]);
    SK(cudaGetLastError());
    TcGemmArgs h{};
    h.a = s->dzb[l], h.lda = nout[l], h.b = wt, h.ldb = nout[l];
    h.c = s->da, h.ldc = NH, h.M = n, h.N = kin[l], h.K = nout[l];
    h.err = s->err;
    SK(gemm_tc(h, 1, st));
    silu_backward_kernel<<<blocks((long long)n * NH), 256, 0, st>>>(s->da, s->z[l - 1], (long long)n * NH,
                                                                     s->dz[l - 1], s->dzb[l - 1]);
    SK(cudaGetLastError());
  }
  return OSTC_OK;
}

ostc_status pack(ostc_surrogate *s, const float *x, int n, cudaStream_t st) {
  pack_inputs_kernel<<<blocks((long long)n * KIN), 256, 0, st>>>(x, n, s->x0);
  SK(cudaGetLastError());
  return OSTC_OK;
}

}  // namespace

extern "C" {

ostc_status ostc_surrogate_create(int max_batch, unsigned long long seed, ostc_surrogate **out) {
  if (!out || max_batch < 1 || max_batch > (1 << 22)) return OSTC_ERR_INVALID_ARG;
  *out = nullptr;
  auto *s = new ostc_surrogate;
  s->max_batch = max_batch;
  const long long B = max_batch;
  bool ok = dalloc(s, (void **)&s->net.wb, sizeof(__nv_bfloat16) * NPAR) == cudaSuccess &&
            dalloc(s, (void **)&s->master, sizeof(float) * NPAR) == cudaSuccess &&
            dalloc(s, (void **)&s->grad, sizeof(float) * NPAR) == cudaSuccess &&
            dalloc(s, (void **)&s->mom1, sizeof(float) * NPAR) == cudaSuccess &&
            dalloc(s, (void **)&s->mom2, sizeof(float) * NPAR) == cudaSuccess &&
            dalloc(s, (void **)&s->mask, NPAR) == cudaSuccess &&
            dalloc(s, (void **)&s->net.scale, sizeof(double) * SCALE_COUNT) == cudaSuccess &&
            dalloc(s, (void **)&s->x0, sizeof(__nv_bfloat16) * B * KIN) == cudaSuccess &&
            dalloc(s, (void **)&s->da, sizeof(float) * B * NH) == cudaSuccess &&
            dalloc(s, (void **)&s->tg, sizeof(__nv_bfloat16) * NH * ((B + 15) / 16 * 16)) == cudaSuccess &&
            dalloc(s, (void **)&s->ta, sizeof(__nv_bfloat16) * NH * ((B + 15) / 16 * 16)) == cudaSuccess &&
            dalloc(s, (void **)&s->wt, sizeof(__nv_bfloat16) * 3 * NH * NH) == cudaSuccess &&
            dalloc(s, (void **)&s->loss, sizeof(float)) == cudaSuccess &&
            dalloc(s, (void **)&s->err, sizeof(int)) == cudaSuccess &&
            dalloc(s, (void **)&s->count, sizeof(int)) == cudaSuccess &&
            dalloc(s, (void **)&s->checks, sizeof(Checks)) == cudaSuccess;
  for (int l = 0; l < 4 && ok; ++l) {
    const long long w = l == 3 ? NOUTP : NH;
    ok = dalloc(s, (void **)&s->z[l], sizeof(float) * B * w) == cudaSuccess &&
         dalloc(s, (void **)&s->dz[l], sizeof(float) * B * w) == cudaSuccess &&
         dalloc(s, (void **)&s->dzb[l], sizeof(__nv_bfloat16) * B * w) == cudaSuccess;
    if (ok && l < 3) ok = dalloc(s, (void **)&s->a[l], sizeof(__nv_bfloat16) * B * NH) == cudaSuccess;
  }
  if (!ok) {
    ostc_surrogate_destroy(s);
    return OSTC_ERR_CUDA;
  }
  s->net.wf = s->master;
  s->net.checks = s->checks;
  // He-uniform initialisation from a seeded 64-bit LCG (biases zero)
  std::vector<float> host(NPAR, 0.f);
  std::vector<unsigned char> mask(NPAR, 0);
  unsigned long long st = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return ((st >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
  };
  for_each_param([&](long long, long long off) {
    mask[off] = 1;
    double fan_in = 0;
    if (off < OFF_B1) fan_in = NIN;
    else if (off >= OFF_W2 && off < OFF_B2) fan_in = NH;
    else if (off >= OFF_W3 && off < OFF_B3) fan_in = NH;
    else if (off >= OFF_W4 && off < OFF_B4) fan_in = NH;
    host[off] = fan_in > 0 ? (float)(uni() * std::sqrt(6.0 / fan_in)) : 0.f;
  });
  double scale[SCALE_COUNT];
  for (int i = 0; i < SCALE_COUNT; ++i) scale[i] = 0.0;
  for (int i = 0; i < NIN; ++i) scale[SC_IN_STD + i] = 1.0, scale[SC_IN_MIN + i] = -1e300, scale[SC_IN_MAX + i] = 1e300;
  for (int i = 0; i < NOUT; ++i) scale[SC_OUT_STD + i] = 1.0;
  Checks ck;
  if (cudaMemcpy(s->checks, &ck, sizeof(Checks), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(s->master, host.data(), sizeof(float) * NPAR, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(s->mask, mask.data(), NPAR, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(s->net.scale, scale, sizeof(scale), cudaMemcpyHostToDevice) != cudaSuccess ||
      refresh_bf16(s, nullptr) != OSTC_OK || cudaDeviceSynchronize() != cudaSuccess) {
    ostc_surrogate_destroy(s);
    return OSTC_ERR_CUDA;
  }
  *out = s;
  return OSTC_OK;
}

ostc_status ostc_surrogate_destroy(ostc_surrogate *s) {
  if (!s) return OSTC_ERR_INVALID_ARG;
  cudaDeviceSynchronize();
  for (void *p : s->owned) cudaFree(p);
  delete s;
  return OSTC_OK;
}

ostc_status ostc_surrogate_set_scaling(ostc_surrogate *s, const double *in_mean, const double *in_std,
                                       const double *out_mean, const double *out_std, const double *in_min,
                                       const double *in_max, const double *out_r0) {
  if (!s || !in_mean || !in_std || !out_mean || !out_std || !in_min || !in_max) return OSTC_ERR_INVALID_ARG;
  double scale[SCALE_COUNT];
  for (int i = 0; i < NIN; ++i) {
    if (!(in_std[i] > 0)) return OSTC_ERR_INVALID_ARG;
    scale[SC_IN_MEAN + i] = in_mean[i];
    scale[SC_IN_STD + i] = in_std[i];
    scale[SC_IN_MIN + i] = in_min[i];
    scale[SC_IN_MAX + i] = in_max[i];
  }
  for (int i = 0; i < NOUT; ++i) {
    if (!(out_std[i] > 0)) return OSTC_ERR_INVALID_ARG;
    scale[SC_OUT_MEAN + i] = out_mean[i];
    scale[SC_OUT_STD + i] = out_std[i];
    scale[SC_OUT_R0 + i] = out_r0 ? out_r0[i] : 0.0;
    if (!(scale[SC_OUT_R0 + i] >= 0)) return OSTC_ERR_INVALID_ARG;
  }
  SK(cudaMemcpy(s->net.scale, scale, sizeof(scale), cudaMemcpyHostToDevice));
  return OSTC_OK;
}

ostc_status ostc_surrogate_set_checks(ostc_surrogate *s, int n_elem, int n_spec, const double *elem_counts,
                                      const double *elem_mass, double tol_elem, double tol_T) {
  if (!s || n_elem < 0 || n_elem > 4 || n_spec < 1 || n_spec > OSTC_MAX_SPEC || (n_elem && (!elem_counts || !elem_mass)))
    return OSTC_ERR_INVALID_ARG;
  if (!(tol_elem >= 0) || !(tol_T >= 0)) return OSTC_ERR_INVALID_ARG;
  Checks ck;
  ck.n_elem = n_elem;
  for (int e = 0; e < n_elem; ++e) {
    ck.m[e] = elem_mass[e];
    for (int l = 0; l < n_spec; ++l) ck.a[e][l] = elem_counts[e * n_spec + l];
  }
  ck.tol_el = tol_elem;
  ck.tol_T = tol_T;
  SK(cudaMemcpy(s->checks, &ck, sizeof(Checks), cudaMemcpyHostToDevice));
  return OSTC_OK;
}

ostc_status ostc_surrogate_inject_timeout(ostc_surrogate *s, int on) {
  if (!s || (on != 0 && on != 1)) return OSTC_ERR_INVALID_ARG;
  s->net.withhold_commit = on;
  return OSTC_OK;
}

ostc_status ostc_surrogate_get_params(const ostc_surrogate *s, float *host_out) {
  if (!s || !host_out) return OSTC_ERR_INVALID_ARG;
  std::vector<float> pad(NPAR);
  SK(cudaMemcpy(pad.data(), s->master, sizeof(float) * NPAR, cudaMemcpyDeviceToHost));
  for_each_param([&](long long q, long long off) { host_out[q] = pad[off]; });
  return OSTC_OK;
}

ostc_status ostc_surrogate_set_params(ostc_surrogate *s, const float *host_in) {
  if (!s || !host_in) return OSTC_ERR_INVALID_ARG;
  std::vector<float> pad(NPAR, 0.f);
  for_each_param([&](long long q, long long off) { pad[off] = host_in[q]; });
  SK(cudaMemcpy(s->master, pad.data(), sizeof(float) * NPAR, cudaMemcpyHostToDevice));
  SK(cudaMemset(s->mom1, 0, sizeof(float) * NPAR));
  SK(cudaMemset(s->mom2, 0, sizeof(float) * NPAR));
  s->step = 0;
  if (refresh_bf16(s, nullptr)) return OSTC_ERR_CUDA;
  SK(cudaDeviceSynchronize());
  return OSTC_OK;
}

ostc_status ostc_surrogate_forward(ostc_surrogate *s, const float *xs, int n, float *ys, void *stream) {
  if (!s || !xs || !ys || n < 0 || n > s->max_batch) return OSTC_ERR_INVALID_ARG;
  if (n == 0) return OSTC_OK;
  cudaStream_t st = (cudaStream_t)stream;
  ostc_status r;
  if ((r = pack(s, xs, n, st)) || (r = forward_reference(s, n, st))) return r;
  // the 10 outputs of the padded layer
  SK(cudaMemcpy2DAsync(ys, sizeof(float) * NOUT, s->z[3], sizeof(float) * NOUTP, sizeof(float) * NOUT, n,
                       cudaMemcpyDeviceToDevice, st));
  return OSTC_OK;
}

ostc_status ostc_surrogate_forward_tc(ostc_surrogate *s, const float *xs, int n, float *ys, void *stream) {
  if (!s || !xs || !ys || n < 0) return OSTC_ERR_INVALID_ARG;
  if (n == 0) return OSTC_OK;
  cudaStream_t st = (cudaStream_t)stream;
  static int configured_dev = -1;
  int dev = 0;
  SK(cudaGetDevice(&dev));
  if (configured_dev != dev) {
    SK(cudaFuncSetAttribute(surrogate_raw_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SM_BYTES));
    configured_dev = dev;
  }
  int sms = 148;
  SK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int tiles = (n + tc::ROWS - 1) / tc::ROWS;
  SK(cudaMemsetAsync(s->err, 0, sizeof(int), st));
  surrogate_raw_kernel<<<tiles < sms ? tiles : sms, tc::THREADS, tc::SM_BYTES, st>>>(s->net, xs, ys, n, s->err);
  SK(cudaGetLastError());
  int e = 0;
  SK(cudaMemcpyAsync(&e, s->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SK(cudaStreamSynchronize(st));
  return e ? OSTC_ERR_TIMEOUT : OSTC_OK;
}

ostc_status ostc_surrogate_gradients(ostc_surrogate *s, const float *xs, const float *ys, int n, float *grad_host,
                                     float *loss_host, void *stream) {
  if (!s || !xs || !ys || !grad_host || n < 1 || n > s->max_batch) return OSTC_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  ostc_status r;
  if ((r = pack(s, xs, n, st)) || (r = forward(s, n, st)) || (r = backward(s, ys, n, st))) return r;
  std::vector<float> pad(NPAR);
  SK(cudaMemcpyAsync(pad.data(), s->grad, sizeof(float) * NPAR, cudaMemcpyDeviceToHost, st));
  float l = 0;
  SK(cudaMemcpyAsync(&l, s->loss, sizeof(float), cudaMemcpyDeviceToHost, st));
  int late = 0;
  SK(cudaMemcpyAsync(&late, s->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SK(cudaStreamSynchronize(st));
  if (late) {
    SK(cudaMemset(s->err, 0, sizeof(int)));
    return OSTC_ERR_TIMEOUT;
  }
  for_each_param([&](long long q, long long off) { grad_host[q] = pad[off]; });
  if (loss_host) *loss_host = l / ((float)n * NOUT);
  return OSTC_OK;
}

ostc_status ostc_surrogate_train_step(ostc_surrogate *s, const float *xs, const float *ys, int n, float lr,
                                      float *loss_dev, void *stream) {
  if (!s || !xs || !ys || n < 1 || n > s->max_batch || !(lr >= 0)) return OSTC_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  ostc_status r;
  if ((r = pack(s, xs, n, st)) || (r = forward(s, n, st)) || (r = backward(s, ys, n, st))) return r;
  ++s->step;
  const float b1t = std::pow(0.9f, (float)s->step), b2t = std::pow(0.999f, (float)s->step);
  adam_kernel<<<blocks(NPAR), 256, 0, st>>>(s->master, s->grad, s->mom1, s->mom2, s->net.wb, s->mask, NPAR, lr, b1t,
                                            b2t);
  SK(cudaGetLastError());
  if (loss_dev) SK(cudaMemcpyAsync(loss_dev, s->loss, sizeof(float), cudaMemcpyDeviceToDevice, st));
  return OSTC_OK;
}

}  // extern "C"

namespace ostc {
const Net *surrogate_net(const ostc_surrogate *s) { return s ? &s->net : nullptr; }

cudaError_t surrogate_scratch(ostc_surrogate *s, int n, ChemScratch *out) {
  if (n > s->list_cap) {
    for (void *q : {(void *)s->list, (void *)s->cx, (void *)s->cy, (void *)s->cenv}) {
      if (!q) continue;
      cudaFree(q);
      for (auto &p : s->owned)
        if (p == q) p = nullptr;
    }
    s->list = nullptr;
    s->cx = nullptr;
    s->cy = nullptr;
    s->cenv = nullptr;
    s->list_cap = 0;
    cudaError_t e = cudaMalloc(&s->list, sizeof(int) * (size_t)n);
    if (e == cudaSuccess) s->owned.push_back(s->list);
    if (e == cudaSuccess) e = cudaMalloc(&s->cx, sizeof(__nv_bfloat16) * mlp::KIN * (size_t)n);
    if (e == cudaSuccess) s->owned.push_back(s->cx);
    if (e == cudaSuccess) e = cudaMalloc(&s->cy, sizeof(float) * mlp::NOUT * (size_t)n);
    if (e == cudaSuccess) s->owned.push_back(s->cy);
    if (e == cudaSuccess) e = cudaMalloc(&s->cenv, (size_t)n);
    if (e == cudaSuccess) s->owned.push_back(s->cenv);
    if (e != cudaSuccess) return e;
    s->list_cap = n;
  }
  out->list = s->list;
  out->count = s->count;
  out->err = s->err;
  out->x = s->cx;
  out->y = s->cy;
  out->env = s->cenv;
  return cudaSuccess;
}
}  // namespace ostc
