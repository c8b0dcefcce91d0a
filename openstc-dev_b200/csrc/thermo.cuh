// thermo.cuh — NASA-7 thermodynamics and mixture transport on the device.
//
// Divisions by constants (1/3, 1/6, 1/12) and by molecular weights are
// multiplications by reciprocals here and in the flux, chemistry and update
// kernels (at most one rounding apart from the reference's quotients).
// Arithmetic follows src/Thermo.cu:5-79 and src/Transport.cu:6-145 term by
// term; the species count NS is a compile-time constant so that every
// per-species array lives in registers (the reference keeps MAX_SPEC_NUMBER-
// sized arrays in local memory).
#pragma once
#include "common.cuh"

namespace ostc {

// the NASA-7 coefficients c[0..n) of species i at temperature t: the low
// range below t_mid (and below t_low, where the caller extends linearly), the
// high range above. Selected by value from both rows, so that every
// coefficient address is a compile-time constant of the unrolled species loop.
template <int N>
__device__ __forceinline__ void nasa_coeffs(int i, bool low, double *c) {
#pragma unroll
  for (int k = 0; k < N; ++k) c[k] = low ? c_p.lo[i][k] : c_p.hi[i][k];
}

// enthalpy h_k (J/kg) and cp_k (J/kg/K) at temperature t (Thermo.cu:25-45).
// SEL: coefficients selected by value (nasa_coeffs; the register-starved flux
// kernels) or through a row pointer (one constant load per coefficient; the
// per-cell Newton solves, where it measured faster)
template <int NS, bool SEL = true>
__device__ __forceinline__ void enthalpy_cp(double t, double *h, double *cp) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    double tt = t, tt2 = t2, tt3 = t3, tt4 = t4, tt5 = t5;
    const bool below = t < c_p.t_low[i];
    if (below) {
      tt = c_p.t_low[i];
      tt2 = tt * tt; tt3 = tt2 * tt; tt4 = tt3 * tt; tt5 = tt4 * tt;
    }
    const bool low = below || t < c_p.t_mid[i];
    double cs[6];
    if (SEL) nasa_coeffs<6>(i, low, cs);
    const double *c = SEL ? cs : (low ? c_p.lo[i] : c_p.hi[i]);
    double hi = c[0] * tt + 0.5 * c[1] * tt2 + c[2] * tt3 * (1.0 / 3) + 0.25 * c[3] * tt4 + 0.2 * c[4] * tt5 + c[5];
    const double cpi = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
    if (below) hi += cpi * (t - tt);
    h[i] = hi * c_p.Rmw[i];
    cp[i] = cpi * c_p.Rmw[i];
  }
}

// enthalpy of species i (Thermo.cu:5-23) at t with its powers t2..t5
__device__ __forceinline__ double enthalpy_one(int i, double t, double t2, double t3, double t4, double t5) {
  double tt = t, tt2 = t2, tt3 = t3, tt4 = t4, tt5 = t5;
  const bool below = t < c_p.t_low[i];
  if (below) {
    tt = c_p.t_low[i];
    tt2 = tt * tt; tt3 = tt2 * tt; tt4 = tt3 * tt; tt5 = tt4 * tt;
  }
  double c[6];
  nasa_coeffs<6>(i, below || t < c_p.t_mid[i], c);
  double hi = c[0] * tt + 0.5 * c[1] * tt2 + c[2] * tt3 * (1.0 / 3) + 0.25 * c[3] * tt4 + 0.2 * c[4] * tt5 + c[5];
  if (below) {
    const double cpi = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
    hi += cpi * (t - tt);
  }
  return hi * c_p.Rmw[i];
}

// enthalpy only (Thermo.cu:5-23)
template <int NS>
__device__ __forceinline__ void enthalpy(double t, double *h) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
#pragma unroll
  for (int i = 0; i < NS; ++i) h[i] = enthalpy_one(i, t, t2, t3, t4, t5);
}

// cp only (Thermo.cu:47-61)
template <int NS>
__device__ __forceinline__ void cp_only(double t, double *cp) {
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    double tt = t;
    const double *c = c_p.hi[i];
    if (t < c_p.t_low[i]) {
      tt = c_p.t_low[i];
      c = c_p.lo[i];
    } else if (t < c_p.t_mid[i]) {
      c = c_p.lo[i];
    }
    const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
    cp[i] = (c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4) * c_p.Rmw[i];
  }
}

// g_k/(R T) (Thermo.cu:63-79)
template <int NS>
__device__ __forceinline__ void gibbs_div_rt(double t, double *g) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t_inv = 1 / t, log_t = log(t);
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    if (t < c_p.t_low[i]) {
      const double tt = c_p.t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt_inv = 1 / tt, log_tt = log(tt);
      const double *c = c_p.lo[i];
      g[i] = c[0] * (1.0 - log_tt) - 0.5 * c[1] * tt - c[2] * tt2 * (1.0 / 6) - c[3] * tt3 * (1.0 / 12) - c[4] * tt4 * 0.05 +
             c[5] * tt_inv - c[6];
    } else {
      const double *c = t < c_p.t_mid[i] ? c_p.lo[i] : c_p.hi[i];
      g[i] = c[0] * (1.0 - log_t) - 0.5 * c[1] * t - c[2] * t2 * (1.0 / 6) - c[3] * t3 * (1.0 / 12) - c[4] * t4 * 0.05 +
             c[5] * t_inv - c[6];
    }
  }
}

// Sutherland's law (Transport.cu:6-9)
__device__ __forceinline__ double sutherland(double t) {
  return 1.716e-5 * pow(t / 273, 1.5) * (273 + 111) / (t + 111);
}

}  // namespace ostc
