// surrogate.cuh — the learned chemistry step (included by kernels.cu, which
// holds the mechanism in __constant__ memory).
//
//   chem_features_kernel<NS>   one thread per state: features (log T,
//       log p, log(Y_k + 1e-10), log dt, in FP32), training-envelope test,
//       standardised BF16 rows of the network's first operand;
//   surrogate_chem_kernel      the network on the tensor cores over those
//       rows (tc_mlp.cuh), FP32 outputs;
//   chem_checks_kernel<NS>     one thread per state: the rates
//       un-standardised and times dt to dY_k, dT (FP64), then two residual
//       checks in FP32 (their tolerances are far above FP32 rounding):
//       element mass sum_k a_ek m_e dY_k / W_k and the internal energy
//       e(T + dT, Y + dY) - e(T, Y) at constant density (as a temperature
//       error, divided by cv). A state outside the envelope or failing a
//       check is appended to a fallback list;
//   chem_fallback_kernel<NS>    the FP64 point-implicit integrator on the
//       listed states (their increments are overwritten).
// The per-state stages run at full occupancy on every SM, so the
// tensor-core kernel between them carries no per-row work but its I/O.
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

// sinh in FP32 for the un-scaling of the network's outputs (whose own
// error is near 1e-3): the Taylor series to z^7 below |z| = 1/4 (truncation
// below 1e-9 relative), else (e^z - e^-z) / 2
__device__ __forceinline__ float sinh_f(float z) {
  const float a = fabsf(z);
  if (a < 0.25f) {
    const float z2 = z * z;
    return z * (1.f + z2 * (1.f / 6) * (1.f + z2 * (1.f / 20) * (1.f + z2 * (1.f / 42))));
  }
  const float e = __expf(a);
  return copysignf(0.5f * (e - 1.f / e), z);
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

// the scaling and acceptance tables of a CTA (thread 0 fills, the caller syncs)
template <int NS>
__device__ void fill_chem_tables(ChemTables<NS> *t, const double *scale, const mlp::Checks *ck) {
  if (threadIdx.x != 0) return;
  for (int i = 0; i < mlp::NIN; ++i) {
    t->in_mean[i] = (float)scale[mlp::SC_IN_MEAN + i];
    t->in_istd[i] = (float)(1.0 / scale[mlp::SC_IN_STD + i]);
    // the envelope, widened by 1e-4 in log units so that the FP32 features
    // of states on its boundary pass
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

// stage 1 of the learned chemistry step, one thread per state: the FP32
// features, the training-envelope test, and the standardised features as a
// BF16 row of the network's first operand (12 features, 4 zeros)
template <int NS>
__global__ void __launch_bounds__(256) chem_features_kernel(int n, const double *T, const double *p, const double *Y,
                                                            const double *dt, const double *scale,
                                                            const mlp::Checks *ck, __nv_bfloat16 *x,
                                                            unsigned char *env) {
  __shared__ ChemTables<NS> tb;
  fill_chem_tables<NS>(&tb, scale, ck);
  __syncthreads();
  for (long long q = blockIdx.x * 256ll + threadIdx.x; q < n; q += 256ll * gridDim.x) {
    float Yf[NS], f[mlp::NIN], xs[16];
#pragma unroll
    for (int l = 0; l < NS; ++l) Yf[l] = (float)Y[(long long)l * n + q];
    surrogate_features<NS>((float)T[q], (float)p[q], Yf, (float)dt[q], f);
    bool in = true;
#pragma unroll
    for (int i = 0; i < mlp::NIN; ++i) {
      in = in && f[i] >= tb.in_min[i] && f[i] <= tb.in_max[i];
      xs[i] = (f[i] - tb.in_mean[i]) * tb.in_istd[i];
    }
#pragma unroll
    for (int i = mlp::NIN; i < 16; ++i) xs[i] = 0.f;
    uint4 *row = (uint4 *)(x + q * mlp::KIN);
    row[0] = make_uint4(tc::pack_bf16(xs[0], xs[1]), tc::pack_bf16(xs[2], xs[3]), tc::pack_bf16(xs[4], xs[5]),
                        tc::pack_bf16(xs[6], xs[7]));
    row[1] = make_uint4(tc::pack_bf16(xs[8], xs[9]), tc::pack_bf16(xs[10], xs[11]), tc::pack_bf16(xs[12], xs[13]),
                        tc::pack_bf16(xs[14], xs[15]));
    env[q] = in ? 1 : 0;
  }
}

// the network on the tensor cores over the staged rows (tc_mlp.cuh)
static __global__ void __launch_bounds__(tc::THREADS, 1) surrogate_chem_kernel(mlp::Net net, const __nv_bfloat16 *x,
                                                                         float *y, int n, int *err) {
  tc::PackedIo io{x, y, n};
  tc::mlp_tiles(net, (n + tc::ROWS - 1) / tc::ROWS, io, err);
}

// stage 3, one thread per state: the network's rates un-standardised and
// times dt to dY_k, dT (FP64 outputs), clipped at zero mass fraction, then
// the element-mass and internal-energy checks in FP32; a state outside the
// envelope or failing a check goes to the fallback list (warp-aggregated)
template <int NS>
__global__ void __launch_bounds__(256, 2) chem_checks_kernel(int n, const double *T, const double *Y, const double *dt,
                                                          const float *y, const unsigned char *env,
                                                          const double *scale, const mlp::Checks *ck, double *dY,
                                                          double *dT, int *list, int *count) {
  __shared__ ChemTables<NS> tb;
  __shared__ double so[3][mlp::NOUT];  // mean, std, r0 of the transformed targets
  fill_chem_tables<NS>(&tb, scale, ck);
  if (threadIdx.x < mlp::NOUT) {
    so[0][threadIdx.x] = scale[mlp::SC_OUT_MEAN + threadIdx.x];
    so[1][threadIdx.x] = scale[mlp::SC_OUT_STD + threadIdx.x];
    so[2][threadIdx.x] = scale[mlp::SC_OUT_R0 + threadIdx.x];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (long long b0 = blockIdx.x * 256ll; b0 < n; b0 += 256ll * gridDim.x) {
    const long long q = b0 + threadIdx.x;
    bool ok = true;
    if (q < n) {
      const double h = dt[q];
      double d[NS + 1];
      const float2 *yr = (const float2 *)(y + q * mlp::NOUT);
#pragma unroll
      for (int i = 0; i < mlp::NOUT / 2; ++i) {
        const float2 v = yr[i];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const int l = 2 * i + c;
          const float z = (float)(so[0][l] + so[1][l] * (double)(c ? v.y : v.x));
          d[l] = h * (so[2][l] > 0 ? so[2][l] * (double)sinh_f(z) : (double)z);
        }
      }
      const double dTq = d[NS];
      float Y0[NS], Y1[NS];
      // a learned increment never drives a mass fraction below zero
#pragma unroll
      for (int l = 0; l < NS; ++l) {
        const double y0 = Y[(long long)l * n + q];
        if (y0 + d[l] < 0) d[l] = y0 > 0 ? -y0 : 0.0;
        Y0[l] = (float)y0;
        Y1[l] = Y0[l] + (float)d[l];
      }
      ok = env[q] != 0;
      for (int e = 0; e < tb.n_elem; ++e) {
        float sm = 0.f;
#pragma unroll
        for (int l = 0; l < NS; ++l) sm += tb.a[e][l] * (float)d[l] * tb.imw[l];
        ok = ok && fabsf(sm * tb.m[e]) <= tb.tol_el;
      }
      const float T0 = (float)T[q];
      float cv1;
      const float e0 = energy_f<NS>(tb, T0, Y0, nullptr);
      const float e1 = energy_f<NS>(tb, T0 + (float)dTq, Y1, &cv1);
      ok = ok && fabsf(e1 - e0) <= tb.tol_T * fabsf(cv1) && isfinite(e1);
#pragma unroll
      for (int l = 0; l < NS; ++l) dY[(long long)l * n + q] = d[l];
      dT[q] = dTq;
    }
    const unsigned rej = __ballot_sync(0xffffffffu, !ok);
    if (rej) {
      const int leader = __ffs(rej) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(count, __popc(rej));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (!ok) list[base + __popc(rej & ((1u << lane) - 1))] = (int)q;
    }
  }
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
