// epilogue.cu — the per-step epilogues of the time loop (RK.cuh:164-180),
// enqueued at the end of every captured step: the step count and physical
// time (physical_time += dt of the last stage), the monitor points
// (Monitor.cu:196-251, record_monitor_data) and the running sums of the
// statistics collector (StatisticsCollector.cu:14-52). All of it stays on the
// device; the host reads it through ostc_get_monitor / ostc_get_statistics.
#include "common.cuh"
#include "kernels.cuh"

namespace ostc {

__global__ void step_clock_kernel(int *step, double *time, const double *dt_dev, double dt_fixed) {
  *step += 1;
  *time += dt_dev ? *dt_dev : dt_fixed;
}

// one thread per monitor point; the points of other blocks are skipped. The
// record of point p at ring position c holds the bv labels, the sv labels
// and the physical time: data[(p * cap + c) * nv + v]
__global__ void monitor_kernel(DevZone z, int blk, const int4 *pts, int n, const int *labels, int nbv, int nsv,
                               double *data, int cap, const int *counter, const double *time) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int4 q = pts[p];
  if (q.x != blk) return;
  const int g = gidx(z, q.y, q.z, q.w);
  const int nv = nbv + nsv + 1;
  double *d = data + ((long long)p * cap + (*counter % cap)) * nv;
  for (int l = 0; l < nbv; ++l) d[l] = z.bv[labels[l] * z.sz + g];
  for (int l = 0; l < nsv; ++l) d[nbv + l] = z.sv[labels[nbv + l] * z.sz + g];
  d[nv - 1] = *time;
}

__global__ void counter_inc_kernel(int *c) { *c += 1; }

// collect_basic_variable_statistics + collect_species_statistics over the
// interior, once the step count has passed `start`: sums of bv, bv^2 (s12),
// bv^3, bv^4 (s34), uv, uw, vw (srs) and Y_k (syk), interior planes; count
// is the number of samples summed (the step count alone cannot tell it once
// the clock was set back or forward by a restart)
__global__ void __launch_bounds__(256) statistics_kernel(DevZone z, const int *step, int start, double *s12,
                                                         double *s34, double *srs, double *syk, int ns, int *count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= z.mx || j >= z.my || *step <= start) return;
  if (i == 0 && j == 0 && k == 0) *count += 1;
  const int g = gidx(z, i, j, k);
  const long long n = nidx(z, i, j, k), N = z.nsz;
#pragma unroll
  for (int l = 0; l < 6; ++l) {
    const double b = z.bv[l * z.sz + g];
    s12[l * N + n] += b;
    s12[(l + 6) * N + n] += b * b;
    s34[l * N + n] += b * b * b;
    s34[(l + 6) * N + n] += b * b * b * b;
  }
  const double u = z.bv[z.sz + g], v = z.bv[2 * z.sz + g], w = z.bv[3 * z.sz + g];
  srs[n] += u * v;
  srs[N + n] += u * w;
  srs[2 * N + n] += v * w;
  for (int l = 0; l < ns; ++l) syk[l * N + n] += z.sv[l * z.sz + g];
}

cudaError_t launch_step_clock(int *step, double *time, const double *dt_dev, double dt_fixed, cudaStream_t s) {
  step_clock_kernel<<<1, 1, 0, s>>>(step, time, dt_dev, dt_fixed);
  return cudaGetLastError();
}

cudaError_t launch_monitor(const DevZone &z, int blk, const MonitorSet &m, cudaStream_t s) {
  if (m.n <= 0) return cudaSuccess;
  monitor_kernel<<<(m.n + 127) / 128, 128, 0, s>>>(z, blk, m.pts, m.n, m.labels, m.nbv, m.nsv, m.data, m.cap,
                                                    m.counter, m.time);
  return cudaGetLastError();
}

cudaError_t launch_monitor_advance(int *counter, cudaStream_t s) {
  counter_inc_kernel<<<1, 1, 0, s>>>(counter);
  return cudaGetLastError();
}

cudaError_t launch_statistics(const DevZone &z, const int *step, int start, const StatSums &st, int ns,
                              cudaStream_t s) {
  const dim3 blk(32, 8), grid((z.mx + 31) / 32, (z.my + 7) / 8, z.mz);
  statistics_kernel<<<grid, blk, 0, s>>>(z, step, start, st.s12, st.s34, st.srs, st.syk, ns, st.count);
  return cudaGetLastError();
}

}  // namespace ostc
