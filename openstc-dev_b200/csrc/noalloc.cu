// noalloc.cu — the residual of one block without any device allocation.
//
// Some callers cannot allocate device memory when they need the residual:
// a host solver that reserves its whole device budget at start-up and
// forbids later allocation, or a driver that embeds this path next to other
// codes sharing one memory pool. ostc_compute_residual_noalloc serves them:
// it computes the same RMS change of (rho, |V|, p, T) as the residual
// epilogue of ostc_rk3_steps (src/Residual.cuh:57-111, before the step-1
// normalisation), with its per-CTA partial sums in a fixed-size array in the
// library's own device memory instead of a buffer from cudaMalloc.
//
// The scratch array lives as long as the library is loaded, on every GPU
// that loads it, and is shared by all calls: calls whose kernels overlap on
// the GPU (other streams, other host threads) race on it. Every slot a call
// reads is written earlier in that same call, so no slot has to start at
// zero and stale contents of a previous call are never read.
#include <atomic>

#include <cuda_runtime.h>

#include "../../include/ostc.h"

namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerCta = kThreads * 8;  // each thread sums 8 cells

// 16384 partials x 4 doubles = 512 KiB: room for 16384 * 2048 = 33,554,432 cells
__device__ __align__(256) double g_residual_scratch[OSTC_NOALLOC_MAX_PARTIALS * 4];

// device address of g_residual_scratch per device: looked up again on every
// call made outside a stream capture (so a context that was torn down and
// re-created gets the new address), remembered for calls made during one
std::atomic<double *> g_scratch_addr[64];

struct Planes {
  const double *bv, *vel, *bv_last;
  int mx, my, mz;
  int d2, d1, dt_;
  long long sz, nsz;
};

__global__ void __launch_bounds__(kThreads) residual_partials(Planes p, double *partial) {
  const long long n = (long long)p.mx * p.my * p.mz;
  const long long base = (long long)blockIdx.x * kCellsPerCta;
  double s[4] = {0, 0, 0, 0};
  for (int r = 0; r < kCellsPerCta / kThreads; ++r) {
    const long long q = base + (long long)r * kThreads + threadIdx.x;
    if (q >= n) break;
    const int i = (int)(q % p.mx);
    const int j = (int)((q / p.mx) % p.my);
    const int k = (int)(q / ((long long)p.mx * p.my));
    const long long g = (long long)k * p.d1 + (long long)j * p.d2 + i + p.dt_;
    const double d0 = p.bv[g] - p.bv_last[q];
    const double d1 = p.vel[g] - p.bv_last[p.nsz + q];
    const double d2 = p.bv[4 * p.sz + g] - p.bv_last[2 * p.nsz + q];
    const double d3 = p.bv[5 * p.sz + g] - p.bv_last[3 * p.nsz + q];
    s[0] += d0 * d0;
    s[1] += d1 * d1;
    s[2] += d2 * d2;
    s[3] += d3 * d3;
  }
  __shared__ double red[4][kThreads];
  for (int l = 0; l < 4; ++l) red[l][threadIdx.x] = s[l];
  __syncthreads();
  for (int o = kThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int l = 0; l < 4; ++l) red[l][threadIdx.x] += red[l][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int l = 0; l < 4; ++l) partial[blockIdx.x * 4 + l] = red[l][0];
}

// one CTA: fixed-order sum of the n_part partials, then sqrt(sum / n_cells)
__global__ void __launch_bounds__(kThreads) residual_finish(const double *partial, int n_part, double n_cells,
                                                            double *out) {
  double s[4] = {0, 0, 0, 0};
  for (int p = threadIdx.x; p < n_part; p += kThreads)
    for (int l = 0; l < 4; ++l) s[l] += partial[p * 4 + l];
  __shared__ double red[4][kThreads];
  for (int l = 0; l < 4; ++l) red[l][threadIdx.x] = s[l];
  __syncthreads();
  for (int o = kThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int l = 0; l < 4; ++l) red[l][threadIdx.x] += red[l][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[threadIdx.x] = sqrt(red[threadIdx.x][0] / n_cells);
}

}  // namespace

extern "C" ostc_status ostc_compute_residual_noalloc(const ostc_zone *zone, double *res_out, void *stream) {
  if (!zone || !res_out || !zone->bv || !zone->vel || !zone->bv_last) return OSTC_ERR_INVALID_ARG;
  if (zone->mx < 1 || zone->my < 1 || zone->mz < 1 || zone->ngg < 0) return OSTC_ERR_INVALID_ARG;
  const long long n = (long long)zone->mx * zone->my * zone->mz;
  const long long n_part = (n + kCellsPerCta - 1) / kCellsPerCta;
  if (n_part > OSTC_NOALLOC_MAX_PARTIALS) return OSTC_ERR_INVALID_ARG;  // more than OSTC_NOALLOC_MAX_CELLS cells
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return OSTC_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) return OSTC_ERR_CUDA;
  double *scratch = g_scratch_addr[dev].load();
  if (cap == cudaStreamCaptureStatusNone) {
    // look up the array's device address (host code may not use the symbol
    // itself as a device pointer)
    double *ptr = nullptr;
    if (cudaGetSymbolAddress((void **)&ptr, g_residual_scratch) != cudaSuccess || !ptr) return OSTC_ERR_CUDA;
    g_scratch_addr[dev].store(ptr);
    scratch = ptr;
  } else if (!scratch) {
    return OSTC_ERR_INVALID_ARG;  // no call outside a capture on this device yet
  }
  Planes p;
  p.bv = zone->bv;
  p.vel = zone->vel;
  p.bv_last = zone->bv_last;
  p.mx = zone->mx;
  p.my = zone->my;
  p.mz = zone->mz;
  const int g = zone->ngg;
  p.d2 = zone->mx + 2 * g;
  p.d1 = (zone->my + 2 * g) * p.d2;
  p.dt_ = (p.d1 + p.d2 + 1) * g;
  p.sz = (long long)(zone->mx + 2 * g) * (zone->my + 2 * g) * (zone->mz + 2 * g);
  p.nsz = n;
  residual_partials<<<(unsigned)n_part, kThreads, 0, s>>>(p, scratch);
  residual_finish<<<1, kThreads, 0, s>>>(scratch, (int)n_part, (double)n, res_out);
  return cudaGetLastError() == cudaSuccess ? OSTC_OK : OSTC_ERR_CUDA;
}
