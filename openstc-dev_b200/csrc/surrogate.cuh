// surrogate.cuh — the learned chemistry step (included by kernels.cu, which
// holds the mechanism in __constant__ memory).
//
//   surrogate_chem_kernel<NS>   one launch per batch of states: features
//       (log T, log p, log(Y_k + 1e-10), log dt, in FP32), training-envelope
//       test, the network on the tensor cores (tc_mlp.cuh), its rates
//       un-standardised and times dt to dY_k, dT (FP64), then two residual
//       checks in FP32 (their tolerances are far above FP32 rounding):
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


// the 12 raw features of a state (the formula of the training data,
// surrogate.py: features), evaluated in FP32 for the network's input;
// round-off negatives of absent species count as zero
template <int NS>
__device__ __forceinline__ void surrogate_features(float T, float p, const float *Y, float dt, float *f) {
  f[0] = __logf(T);
  f[1] = __logf(p);
#pragma unroll
  for (int l = 0; l < NS; ++l) f[2 + l] = __logf(fmaxf(Y[l], 0.f) + 1e-10f);
  f[2 + NS] = __logf(dt);
}

// FP32 tables of the acceptance tests and the feature scaling, staged in
// shared memory once per CTA
template <int NS>
struct ChemTables {
  float in_mean[mlp::NIN], in_istd[mlp::NIN], in_min[mlp::NIN], in_max[mlp::NIN];
  float lo[NS][7], hi[NS][7], t_low[NS], t_mid[NS], Rmw[NS], imw[NS];
  float a[4][NS], m[4];
  float tol_el, tol_T;
  int n_elem;
};

// e = sum Y h(T) - R_u T sum(Y/W) and (optionally) cv, in FP32 (NASA-7 with
// the linear extension below T_low, as thermo.cuh: enthalpy_cp)
template <int NS>
__device__ __forceinline__ float energy_f(const ChemTables<NS> &tb, float t, const float *Y, float *cv) {
  float e = 0.f, c = 0.f, r = 0.f;
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    const bool below = t < tb.t_low[i];
    const float tt = below ? tb.t_low[i] : t;
    const float *k = (below || t < tb.t_mid[i]) ? tb.lo[i] : tb.hi[i];
    const float cpi = k[0] + tt * (k[1] + tt * (k[2] + tt * (k[3] + tt * k[4])));
    float hi = tt * (k[0] + tt * (0.5f * k[1] + tt * (k[2] * (1.f / 3) + tt * (0.25f * k[3] + tt * 0.2f * k[4])))) + k[5];
    if (below) hi += cpi * (t - tt);
    e += Y[i] * hi * tb.Rmw[i];
    c += Y[i] * cpi * tb.Rmw[i];
    r += Y[i] * tb.imw[i];
  }
  if (cv) *cv = c - (float)R_u * r;
  return e - (float)R_u * t * r;
}

template <int NS>
struct ChemIo {
  const double *T, *p, *Y, *dt;
  double *dY, *dT;
  int n;
  const double *scale;
  const mlp::Checks *ck;
  int *list, *count;
  const ChemTables<NS> *tb = nullptr;  // shared memory
  // per-row state kept by the loading thread for the checks
  float T0, Y0[NS > 0 ? NS : 1];
  double h;
  bool in_env;

  __device__ void setup(unsigned char *mem) {
    static_assert(sizeof(ChemTables<NS>) <= tc::IO_BYTES, "tables exceed the Io's shared memory");
    ChemTables<NS> *t = (ChemTables<NS> *)mem;
    if (threadIdx.x == 0) {
      for (int i = 0; i < mlp::NIN; ++i) {
        t->in_mean[i] = (float)scale[mlp::SC_IN_MEAN + i];
        t->in_istd[i] = (float)(1.0 / scale[mlp::SC_IN_STD + i]);
        // the envelope, widened by 1e-4 in log units so that the FP32
        // features of states on its boundary (Y_k = 0, the coldest T) pass
        t->in_min[i] = __double2float_rd(scale[mlp::SC_IN_MIN + i] - 1e-4);
        t->in_max[i] = __double2float_ru(scale[mlp::SC_IN_MAX + i] + 1e-4);
      }
      for (int l = 0; l < NS; ++l) {
        for (int c = 0; c < 7; ++c) {
          t->lo[l][c] = (float)c_p.lo[l][c];
          t->hi[l][c] = (float)c_p.hi[l][c];
        }
        t->t_low[l] = (float)c_p.t_low[l];
        t->t_mid[l] = (float)c_p.t_mid[l];
        t->Rmw[l] = (float)c_p.Rmw[l];
        t->imw[l] = (float)c_p.imw[l];
      }
      t->n_elem = ck->n_elem;
      for (int e = 0; e < 4; ++e) {
        t->m[e] = (float)ck->m[e];
        for (int l = 0; l < NS; ++l) t->a[e][l] = (float)ck->a[e][l];
      }
      t->tol_el = (float)ck->tol_el;
      t->tol_T = (float)ck->tol_T;
    }
    tb = t;
  }

  __device__ bool load(int tile, int row, float *x) {
    const long long q = (long long)tile * tc::ROWS + row;
    if (q >= n) return false;
    if constexpr (NS == mlp::NIN - 3) {
      float f[mlp::NIN];
      T0 = (float)T[q];
      h = dt[q];
#pragma unroll
      for (int l = 0; l < NS; ++l) Y0[l] = (float)Y[(long long)l * n + q];
      surrogate_features<NS>(T0, (float)p[q], Y0, (float)h, f);
      in_env = true;
#pragma unroll
      for (int i = 0; i < mlp::NIN; ++i) {
        in_env = in_env && f[i] >= tb->in_min[i] && f[i] <= tb->in_max[i];
        x[i] = (f[i] - tb->in_mean[i]) * tb->in_istd[i];
      }
    }
    return true;
  }

  __device__ void store(int tile, int row, const float *y) {
    const long long q = (long long)tile * tc::ROWS + row;
    if (q >= n) return;
    if constexpr (NS == mlp::NIN - 3) {
      // the network predicts (transformed) rates; increments are dt * rate
      double d[NS + 1];
#pragma unroll
      for (int l = 0; l <= NS; ++l) {
        const double z = scale[mlp::SC_OUT_MEAN + l] + scale[mlp::SC_OUT_STD + l] * (double)y[l];
        const double r0 = scale[mlp::SC_OUT_R0 + l];
        d[l] = h * (r0 > 0 ? r0 * sinh(z) : z);
      }
      const double dTq = d[NS];
      // a learned increment never drives a mass fraction below zero
#pragma unroll
      for (int l = 0; l < NS; ++l) {
        const double y0 = Y[(long long)l * n + q];
        if (y0 + d[l] < 0) d[l] = y0 > 0 ? -y0 : 0.0;
      }
      // acceptance tests in FP32: element mass balance, internal energy at
      // constant density as a temperature error
      const ChemTables<NS> &t = *tb;
      bool ok = in_env;
      float Y1[NS];
#pragma unroll
      for (int l = 0; l < NS; ++l) Y1[l] = Y0[l] + (float)d[l];
      for (int e = 0; e < t.n_elem; ++e) {
        float sm = 0.f;
#pragma unroll
        for (int l = 0; l < NS; ++l) sm += t.a[e][l] * (float)d[l] * t.imw[l];
        ok = ok && fabsf(sm * t.m[e]) <= t.tol_el;
      }
      float cv1;
      const float e0 = energy_f<NS>(t, T0, Y0, nullptr);
      const float e1 = energy_f<NS>(t, T0 + (float)dTq, Y1, &cv1);
      ok = ok && fabsf(e1 - e0) <= t.tol_T * fabsf(cv1) && isfinite(e1);
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
