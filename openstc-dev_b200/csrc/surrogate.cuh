// surrogate.cuh — the learned chemistry step (included by kernels.cu, which
// holds the mechanism in __constant__ memory).
//
//   surrogate_chem_kernel<NS>   one launch per batch of states: features in
//       FP64 (log T, log p, log(Y_k + 1e-10), log dt), training-envelope
//       test, the network on the tensor cores (tc_mlp.cuh), its rates
//       un-standardised and times dt to dY_k, dT, then two residual checks
//       in FP64:
//       element mass sum_k a_ek m_e dY_k / W_k and the internal energy
//       e(T + dT, Y + dY) - e(T, Y) at constant density (as a temperature
//       error, divided by cv). A state that fails any test is appended to a
//       fallback list;
//   chem_fallback_kernel<NS>    the FP64 point-implicit integrator on the
//       listed states (their increments are overwritten).
#pragma once
#include "mlp.cuh"
#include "tc_mlp.cuh"

namespace ostc {


// the 12 raw features of a state (the same formula as the training data)
template <int NS>
__device__ __forceinline__ void surrogate_features(double T, double p, const double *Y, double dt, double *f) {
  f[0] = log(T);
  f[1] = log(p);
#pragma unroll
  for (int l = 0; l < NS; ++l) f[2 + l] = log(Y[l] + 1e-10);
  f[2 + NS] = log(dt);
}

template <int NS>
struct ChemIo {
  const double *T, *p, *Y, *dt;
  double *dY, *dT;
  int n;
  const double *scale;
  const mlp::Checks *ck;
  int *list, *count;
  // per-row state kept by the loading thread for the checks
  double T0, Y0[NS > 0 ? NS : 1];
  bool in_env;

  __device__ bool load(int tile, int row, float *x) {
    const long long q = (long long)tile * tc::ROWS + row;
    if (q >= n) return false;
    if constexpr (NS == mlp::NIN - 3) {
      double f[mlp::NIN];
      T0 = T[q];
      double yy[NS];
#pragma unroll
      for (int l = 0; l < NS; ++l) yy[l] = Y0[l] = Y[(long long)l * n + q];
      surrogate_features<NS>(T0, p[q], yy, dt[q], f);
      in_env = true;
#pragma unroll
      for (int i = 0; i < mlp::NIN; ++i) {
        in_env = in_env && f[i] >= scale[mlp::SC_IN_MIN + i] && f[i] <= scale[mlp::SC_IN_MAX + i];
        x[i] = (float)((f[i] - scale[mlp::SC_IN_MEAN + i]) / scale[mlp::SC_IN_STD + i]);
      }
    }
    return true;
  }

  __device__ void store(int tile, int row, const float *y) {
    const long long q = (long long)tile * tc::ROWS + row;
    if (q >= n) return;
    if constexpr (NS == mlp::NIN - 3) {
      // the network predicts rates: increments are dt * (mean + std * y)
      const double h = dt[q];
      double d[NS], dTq;
#pragma unroll
      for (int l = 0; l < NS; ++l) d[l] = h * (scale[mlp::SC_OUT_MEAN + l] + scale[mlp::SC_OUT_STD + l] * (double)y[l]);
      dTq = h * (scale[mlp::SC_OUT_MEAN + NS] + scale[mlp::SC_OUT_STD + NS] * (double)y[NS]);
      bool ok = in_env;
      // element mass balance
      for (int e = 0; e < ck->n_elem; ++e) {
        double s = 0;
#pragma unroll
        for (int l = 0; l < NS; ++l) s += ck->a[e][l] * d[l] / c_p.mw[l];
        ok = ok && fabs(s * ck->m[e]) <= ck->tol_el;
      }
      // internal energy at constant density, as a temperature error
      double h0[NS], h1[NS], cp1[NS], e0s = 0, e1s = 0, mw0 = 0, mw1 = 0, cv1 = 0;
      enthalpy<NS>(T0, h0);
      enthalpy_cp<NS>(T0 + dTq, h1, cp1);
#pragma unroll
      for (int l = 0; l < NS; ++l) {
        const double y1 = Y0[l] + d[l];
        e0s += Y0[l] * h0[l];
        e1s += y1 * h1[l];
        mw0 += Y0[l] / c_p.mw[l];
        mw1 += y1 / c_p.mw[l];
        cv1 += y1 * cp1[l];
      }
      e0s -= R_u * T0 * mw0;
      e1s -= R_u * (T0 + dTq) * mw1;
      cv1 -= R_u * mw1;
      ok = ok && fabs(e1s - e0s) <= ck->tol_T * fabs(cv1) && isfinite(e1s);
#pragma unroll
      for (int l = 0; l < NS; ++l) dY[(long long)l * n + q] = d[l];
      dT[q] = dTq;
      // warp-aggregated append of the rejected rows (one atomic per warp)
      const unsigned rej = __ballot_sync(__activemask(), !ok);
      if (rej) {
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(rej) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(count, __popc(rej));
        base = __shfl_sync(__activemask(), base, leader);
        if (!ok) list[base + __popc(rej & ((1u << lane) - 1))] = (int)q;
      }
    }
  }
};

template <int NS>
__global__ void __launch_bounds__(tc::THREADS, 1) surrogate_chem_kernel(mlp::Net net, ChemIo<NS> io, int *err) {
  ChemIo<NS> mine = io;  // per-thread copy: holds the state of the thread's row
  tc::mlp_tiles(net, (io.n + tc::ROWS - 1) / tc::ROWS, mine, err);
}

template <int NS>
__global__ void __launch_bounds__(128) chem_fallback_kernel(const int *list, const int *count, int n, const double *T,
                                                            const double *p, const double *Y, const double *dt,
                                                            double *dY, double *dT) {
  if constexpr (NS > 0) {
    const int m = *count;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
      const int q = list[e];
      double y[NS], d[NS], dtq;
      int it;
#pragma unroll
      for (int l = 0; l < NS; ++l) y[l] = Y[(long long)l * n + q];
      point_implicit_increment<NS>(T[q], p[q], y, dt[q], d, dtq, it);
#pragma unroll
      for (int l = 0; l < NS; ++l) dY[(long long)l * n + q] = d[l];
      dT[q] = it ? dtq : __longlong_as_double(0x7ff8000000000000ll);
    }
  }
}

}  // namespace ostc
