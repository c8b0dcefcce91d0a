// steady.cuh — kernels of the steady (local time stepping) path, included by
// kernels.cu after the RK3 kernels:
//
//   chem_implicit_kernel<NS>  point-implicit chemistry of the explicit steady
//                             step: EPI / DA (ImplicitTreatmentHPP.cuh:11-32,
//                             FiniteRateChem.cu:234-432)
//   update_bv_kernel<NS>      steady update of bv / sv from dq * dt_local / J
//                             (update_bv, FieldOperation.cuh:221-296)
//   dplur_dq0_kernel<NS>      compute_DQ_0 (DPLUR.cuh:14-79) + the dq0 copy
//   dplur_sweep_kernel<NS>    DPLUR_inner_iteration (DPLUR.cuh:161-280)
//   dplur_finish_kernel       convert_dq_back_to_dqDt (DPLUR.cu:5-17)
//   wall_dq_zero_kernel       set_dq_to_0 (DPLUR.cu:19-31)
//
// The chemical Jacobian is never stored as n_spec^2 planes per step: the
// explicit EPI recomputes it from the state it was built from (the state
// does not change between compute_source and the implicit treatment), and
// DPLUR factorises (diag I - dt J) once per step and keeps the LU factors
// and pivots for its sweeps, which re-solve with identical factors.
#pragma once

namespace ostc {

// the state the chemical Jacobian is built from
template <int NS>
__device__ __forceinline__ void cell_state(const DevZone &z, int g, double &rho, double &T, double *Y) {
  rho = z.bv[g];
  T = z.bv[5 * z.sz + g];
#pragma unroll
  for (int l = 0; l < NS; ++l) Y[l] = z.sv[l * z.sz + g];
}

template <int NS>
__global__ void __launch_bounds__(128) chem_implicit_kernel(DevZone z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= z.mx || j >= z.my) return;
  if constexpr (NS > 0) {
    const int g = gidx(z, i, j, k);
    double *dq = z.dq + qidx(z, i, j, k);
    const double dt = z.dt_local[nidx(z, i, j, k)];
    double rho, T, Y[NS];
    cell_state<NS>(z, g, rho, T, Y);
    double q1[OSTC_MAX_REAC], q2[OSTC_MAX_REAC], om[NS], od[NS];
    chemistry_rates<NS>(rho, T, Y, q1, q2, om, od);
    if (c_p.chemSrcMethod == 1) {  // EPI: (I - dt J) x = dq_species
      double A[NS * NS], b[NS];
      chemistry_jacobian<NS>(rho, Y, q1, q2, A);
#pragma unroll 1
      for (int m = 0; m < NS; ++m)
        for (int n = 0; n < NS; ++n) A[m * NS + n] = m == n ? 1.0 - dt * A[m * NS + n] : -dt * A[m * NS + n];
#pragma unroll
      for (int l = 0; l < NS; ++l) b[l] = dq[(5 + l) * z.qsz];
      lu_solve<NS>(A, b);
#pragma unroll
      for (int l = 0; l < NS; ++l) dq[(5 + l) * z.qsz] = b[l];
    } else if (c_p.chemSrcMethod == 2) {  // DA (FiniteRateChem.cu:218-232, 421-432)
#pragma unroll
      for (int l = 0; l < NS; ++l) {
        const double jd = Y[l] > 1e-25 ? -od[l] / (Y[l] * rho) : 0.0;
        dq[(5 + l) * z.qsz] /= 1 - dt * jd;
      }
    }
  }
}

template <int NS>
__global__ void __launch_bounds__(256) update_bv_kernel(DevZone z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= z.mx || j >= z.my) return;
  const int g = gidx(z, i, j, k);
  const double *dq = z.dq + qidx(z, i, j, k);
  const long long S = z.sz, Q = z.qsz;
  const double rho_n = z.bv[g];
  const double u_n = z.bv[S + g], v_n = z.bv[2 * S + g], w_n = z.bv[3 * S + g];
  // compute_total_energy_1_point (FieldOperation.cuh:197-219)
  double E = 0.5 * (u_n * u_n + v_n * v_n + w_n * w_n);
  if constexpr (NS > 0) {
    double h[NS];
    enthalpy<NS>(z.bv[5 * S + g], h);
#pragma unroll
    for (int l = 0; l < NS; ++l) E += h[l] * z.sv[l * S + g];
    E *= rho_n;
    E -= z.bv[4 * S + g];
  } else {
    E *= rho_n;
    E += z.bv[4 * S + g] / (gamma_air - 1);
  }
  const double dtj = z.dt_local[nidx(z, i, j, k)] / z.jac[g];
  const double rho = rho_n + dq[0] * dtj;
  z.bv[g] = rho;
  const double ri = 1.0 / rho;
  const double u = ri * (rho_n * u_n + dq[Q] * dtj);
  const double v = ri * (rho_n * v_n + dq[2 * Q] * dtj);
  const double w = z.mz == 1 ? 0.0 : ri * (rho_n * w_n + dq[3 * Q] * dtj);
  z.bv[S + g] = u;
  z.bv[2 * S + g] = v;
  z.bv[3 * S + g] = w;
  const double Et = E + dq[4 * Q] * dtj;
  const double V2 = u * u + v * v + w * w;
  // scalars after the species (SST k, omega), FieldOperation.cuh:252-257
  for (int l = NS; l < c_p.n_scalar; ++l) z.sv[l * S + g] = ri * (rho_n * z.sv[l * S + g] + dq[(5 + l) * Q] * dtj);
  if constexpr (NS > 0) {
    double Y[NS];
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      Y[l] = ri * (rho_n * z.sv[l * S + g] + dq[(5 + l) * Q] * dtj);
      z.sv[l * S + g] = Y[l];
    }
    // compute_temperature_and_pressure (FieldOperation.cu:3-39)
    double mw = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) mw += Y[l] * c_p.imw[l];
    mw = 1 / mw;
    const double R = R_u / mw;
    const double e = Et / rho - 0.5 * V2;
    double err = 1, t = z.bv[5 * S + g];
    int iter = 0;
    while (err > 1e-3 && iter++ < 1000) {
      double hh[NS], cp[NS];
      enthalpy_cp<NS, false>(t, hh, cp);
      double cpt = 0, hs = 0;
#pragma unroll
      for (int l = 0; l < NS; ++l) {
        cpt += cp[l] * Y[l];
        hs += hh[l] * Y[l];
      }
      const double t1 = t - (hs - R * t - e) / (cpt - R);
      err = fabs(1 - t1 / t);
      t = t1;
    }
    z.bv[5 * S + g] = t;
    z.bv[4 * S + g] = rho * t * R;
  } else {
    const double p = (gamma_air - 1) * (Et - 0.5 * rho * V2);
    z.bv[4 * S + g] = p;
    z.bv[5 * S + g] = p * mw_air * ri / R_u;
  }
  z.vel[g] = sqrt(V2);
}

// ---------------------------------------------------------------------------
// DPLUR
// ---------------------------------------------------------------------------
// NVX: the largest variable count of the build (the species may be followed
// by the two SST scalars); the variables beyond c_p.n_var are not touched
template <int NS>
constexpr int nvx() {
  return 5 + NS + 2;
}

// SST::implicit_treat_for_SST under the explicit steady path (SST.cu:8-22)
static __global__ void __launch_bounds__(256) turb_implicit_kernel(DevZone z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= z.mx || j >= z.my) return;
  const int n = nidx(z, i, j, k);
  double *dq = z.dq + qidx(z, i, j, k);
  const double dt = z.dt_local[n];
  const int it = 5 + c_p.n_spec;  // i_turb_cv
  dq[it * z.qsz] /= 1 - dt * z.tsj[n];
  dq[(it + 1) * z.qsz] /= 1 - dt * z.tsj[z.nsz + n];
}

template <int NS>
__global__ void __launch_bounds__(128) dplur_dq0_kernel(DevZone z, SteadyArgs a) {
  constexpr int NV = nvx<NS>();
  const int nv = c_p.n_var;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= z.mx || j >= z.my) return;
  const int q = qidx(z, i, j, k), n = nidx(z, i, j, k);
  double *dq = z.dq + q;
  const double dt = z.dt_local[n];
  double d[NV];
#pragma unroll
  for (int l = 0; l < NV; ++l) d[l] = l < nv ? dq[l * z.qsz] * dt : 0.0;
  const double diag = 1 + dt * (z.isr[n] + z.isr[z.nsz + n] + z.isr[2 * z.nsz + n]);
#pragma unroll
  for (int l = 0; l < 5; ++l) d[l] /= diag;
  if constexpr (NS > 0) {
    const int method = c_p.n_reac > 0 ? c_p.chemSrcMethod : 0;
    if (method == 1 || method == 2) {
      const int g = gidx(z, i, j, k);
      double rho, T, Y[NS];
      cell_state<NS>(z, g, rho, T, Y);
      double q1[OSTC_MAX_REAC], q2[OSTC_MAX_REAC], om[NS], od[NS];
      chemistry_rates<NS>(rho, T, Y, q1, q2, om, od);
      if (method == 1) {  // EPI_for_dq0 (FiniteRateChem.cu:259-276)
        double A[NS * NS];
        chemistry_jacobian<NS>(rho, Y, q1, q2, A);
#pragma unroll 1
        for (int m = 0; m < NS; ++m)
          for (int c = 0; c < NS; ++c) A[m * NS + c] = m == c ? diag - dt * A[m * NS + c] : -dt * A[m * NS + c];
        // factorise once and keep the factors for the sweeps
        double b[NS];
#pragma unroll
        for (int l = 0; l < NS; ++l) b[l] = d[5 + l];
        int ipiv[NS];
        lu_factor<NS>(A, ipiv);
        lu_apply<NS>(A, ipiv, b);
#pragma unroll
        for (int l = 0; l < NS; ++l) d[5 + l] = b[l];
        for (int e = 0; e < NS * NS; ++e) a.lu[(long long)e * z.nsz + n] = A[e];
#pragma unroll
        for (int l = 0; l < NS; ++l) a.piv[(long long)l * z.nsz + n] = (unsigned char)ipiv[l];
      } else {  // DA
#pragma unroll
        for (int l = 0; l < NS; ++l) {
          const double jd = Y[l] > 1e-25 ? -od[l] / (Y[l] * rho) : 0.0;
          const double den = diag - dt * jd;
          a.da[(long long)l * z.nsz + n] = den;
          d[5 + l] /= den;
        }
      }
    } else {
#pragma unroll
      for (int l = 5; l < 5 + NS; ++l) d[l] /= diag;
    }
  }
  if (c_p.sst) {  // DPLUR.cuh:72-84 with SST::implicit_treat_for_dq0 (SST.cu:249-258), rows i_turb_cv, +1
    if (c_p.turb_implicit == 1) {
      d[5 + NS] /= diag - dt * z.tsj[n];
      d[6 + NS] /= diag - dt * z.tsj[z.nsz + n];
    } else {
      d[5 + NS] /= diag;
      d[6 + NS] /= diag;
    }
  }
#pragma unroll
  for (int l = 0; l < NV; ++l) {
    if (l < nv) {
      dq[l * z.qsz] = d[l];
      a.dq0[q + l * z.qsz] = d[l];
    }
  }
}

// convective Jacobian times dq at point (i,j,k) for direction dir
// (compute_jacobian_times_dq, DPLUR.cuh:81-140)
template <int NS>
__device__ __forceinline__ void jacobian_times_dq(const DevZone &z, const double *dqv, int i, int j, int k, int dir,
                                                  double lambda, double *out) {
  constexpr int NV = nvx<NS>();
  const int nv = c_p.n_var;
  const int g = gidx(z, i, j, k);
  const int q = qidx(z, i, j, k);
  const double kx = met(z, g, 3 * dir), ky = met(z, g, 3 * dir + 1), kz = met(z, g, 3 * dir + 2);
  const long long S = z.sz, Q = z.qsz;
  const double u = z.bv[S + g], v = z.bv[2 * S + g], w = z.bv[3 * S + g];
  const double U = kx * u + ky * v + kz * w;
  const double lmd1 = U + lambda;
  const double vel = z.vel[g];
  const double e = 0.5 * vel * vel;
  double dqp[NV];
#pragma unroll
  for (int l = 0; l < NV; ++l) dqp[l] = l < nv ? dqv[q + l * Q] : 0.0;
  double gamma = gamma_air, b3 = 0, b4 = 0, h = 0;
  if constexpr (NS == 0) {
    h = gamma / (gamma - 1) * z.bv[4 * S + g] / z.bv[g] + e;
  } else {
    const double t = z.bv[5 * S + g];
    double hk[NS];
    enthalpy<NS>(t, hk);
    gamma = z.gam[g];
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      b3 += R_u * t * c_p.imw[l] * dqp[5 + l];
      b4 += hk[l] * dqp[5 + l];
      h += z.sv[l * S + g] * hk[l];
    }
    b3 *= gamma;
    b4 *= gamma - 1;
    h += e;
  }
  const double b1 = kx * dqp[1] + ky * dqp[2] + kz * dqp[3] - U * dqp[0];
  const double b2 = (gamma - 1) * (e * dqp[0] - u * dqp[1] - v * dqp[2] - w * dqp[3] + dqp[4]);
  out[0] = b1 + lmd1 * dqp[0];
  out[1] = u * b1 + kx * b2 + lmd1 * dqp[1] + kx * (b3 - b4);
  out[2] = v * b1 + ky * b2 + lmd1 * dqp[2] + ky * (b3 - b4);
  out[3] = w * b1 + kz * b2 + lmd1 * dqp[3] + kz * (b3 - b4);
  out[4] = h * b1 + U * b2 + lmd1 * dqp[4] + U * (b3 - b4);
#pragma unroll
  for (int l = 0; l < NS; ++l) out[5 + l] = lmd1 * dqp[5 + l] + z.sv[l * S + g] * b1;
#pragma unroll
  for (int l = NS; l < NV - 5; ++l)  // SST k, omega (n_scalar_transported rows, DPLUR.cuh:131-139)
    out[5 + l] = l < c_p.n_scalar ? lmd1 * dqp[5 + l] + z.sv[l * S + g] * b1 : 0.0;
}

template <int NS>
__global__ void __launch_bounds__(128) dplur_sweep_kernel(DevZone z, SteadyArgs a) {
  constexpr int NV = nvx<NS>();
  const int nv = c_p.n_var;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= z.mx || j >= z.my) return;
  double tot[NV], cj[NV];
#pragma unroll
  for (int l = 0; l < NV; ++l) tot[l] = 0;
  const long long N = z.nsz;
  // neighbours in the order of the reference: i-1, j-1, k-1, i+1, j+1, k+1
  if (i > 0) {
    jacobian_times_dq<NS>(z, a.dq_in, i - 1, j, k, 0, z.isr[nidx(z, i - 1, j, k)], cj);
#pragma unroll
    for (int l = 0; l < NV; ++l) tot[l] += 0.5 * cj[l];
  }
  if (j > 0) {
    jacobian_times_dq<NS>(z, a.dq_in, i, j - 1, k, 1, z.isr[N + nidx(z, i, j - 1, k)], cj);
#pragma unroll
    for (int l = 0; l < NV; ++l) tot[l] += 0.5 * cj[l];
  }
  if (k > 0) {
    jacobian_times_dq<NS>(z, a.dq_in, i, j, k - 1, 2, z.isr[2 * N + nidx(z, i, j, k - 1)], cj);
#pragma unroll
    for (int l = 0; l < NV; ++l) tot[l] += 0.5 * cj[l];
  }
  if (i != z.mx - 1) {
    jacobian_times_dq<NS>(z, a.dq_in, i + 1, j, k, 0, -z.isr[nidx(z, i + 1, j, k)], cj);
#pragma unroll
    for (int l = 0; l < NV; ++l) tot[l] -= 0.5 * cj[l];
  }
  if (j != z.my - 1) {
    jacobian_times_dq<NS>(z, a.dq_in, i, j + 1, k, 1, -z.isr[N + nidx(z, i, j + 1, k)], cj);
#pragma unroll
    for (int l = 0; l < NV; ++l) tot[l] -= 0.5 * cj[l];
  }
  if (k != z.mz - 1) {
    jacobian_times_dq<NS>(z, a.dq_in, i, j, k + 1, 2, -z.isr[2 * N + nidx(z, i, j, k + 1)], cj);
#pragma unroll
    for (int l = 0; l < NV; ++l) tot[l] -= 0.5 * cj[l];
  }
  const int q = qidx(z, i, j, k), n = nidx(z, i, j, k);
  const double dt = z.dt_local[n];
  const double diag = 1 + dt * (z.isr[n] + z.isr[N + n] + z.isr[2 * N + n]);
  double out[NV];
#pragma unroll
  for (int l = 0; l < 5; ++l) out[l] = a.dq0[q + l * z.qsz] + dt * tot[l] / diag;
  if constexpr (NS > 0) {
    const int method = c_p.n_reac > 0 ? c_p.chemSrcMethod : 0;
    if (method == 1) {  // EPI_for_dqk (FiniteRateChem.cu:278-306) with the stored factors
      double A[NS * NS], b[NS];
      int ipiv[NS];
      for (int e = 0; e < NS * NS; ++e) A[e] = a.lu[(long long)e * N + n];
#pragma unroll
      for (int l = 0; l < NS; ++l) {
        ipiv[l] = a.piv[(long long)l * N + n];
        b[l] = tot[5 + l] * dt;
      }
      lu_apply<NS>(A, ipiv, b);
#pragma unroll
      for (int l = 0; l < NS; ++l) out[5 + l] = a.dq0[q + (5 + l) * z.qsz] + b[l];
    } else if (method == 2) {
#pragma unroll
      for (int l = 0; l < NS; ++l)
        out[5 + l] = a.dq0[q + (5 + l) * z.qsz] + dt * tot[5 + l] / a.da[(long long)l * N + n];
    } else {
#pragma unroll
      for (int l = 5; l < 5 + NS; ++l) out[l] = a.dq0[q + l * z.qsz] + dt * tot[l] / diag;
    }
  }
  if (c_p.sst) {  // DPLUR.cuh:262-276 with SST::implicit_treat_for_dqk (SST.cu:260-273), rows i_turb_cv, +1
    constexpr int T0 = 5 + NS, T1 = 6 + NS;
    const double d5 = c_p.turb_implicit == 1 ? diag - dt * z.tsj[n] : diag;
    const double d6 = c_p.turb_implicit == 1 ? diag - dt * z.tsj[N + n] : diag;
    out[T0] = a.dq0[q + T0 * z.qsz] + dt * tot[T0] / d5;
    out[T1] = a.dq0[q + T1 * z.qsz] + dt * tot[T1] / d6;
  }
  if (a.final_div) {
#pragma unroll
    for (int l = 0; l < NV; ++l) out[l] /= dt;
  }
#pragma unroll
  for (int l = 0; l < NV; ++l)
    if (l < nv) a.dq_out[q + l * z.qsz] = out[l];
}

// dq <- src / dt_local (src may be dq itself)
template <int NS>
__global__ void __launch_bounds__(256) dplur_finish_kernel(DevZone z, const double *src) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= z.mx || j >= z.my) return;
  const int q = qidx(z, i, j, k);
  const double dt = z.dt_local[nidx(z, i, j, k)];
  for (int l = 0; l < c_p.n_var; ++l) z.dq[q + l * z.qsz] = src[q + l * z.qsz] / dt;
}

// zero dq on a wall face range; points outside dq's allocation are skipped
template <int NS>
static __global__ void wall_dq_zero_kernel(DevZone z, BcFace b, double *dqv) {
  const int i = b.rs[0] + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = b.rs[1] + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = b.rs[2] + blockIdx.z;
  if (i > b.re[0] || j > b.re[1] || k > b.re[2]) return;
  const int qg = z.qt == 0 ? 0 : 1;
  if (i < -qg || j < -qg || k < -qg || i >= z.mx + qg || j >= z.my + qg || k >= z.mz + qg) return;
  const int q = qidx(z, i, j, k);
  for (int l = 0; l < c_p.n_var; ++l) dqv[q + l * z.qsz] = 0;
}

}  // namespace ostc
