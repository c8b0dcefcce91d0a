// chem.cuh — finite-rate chemistry source and mixture transport properties.
//
// Chemistry follows src/FiniteRateChem.cu:7-194 (forward rates with
// duplicate / third-body / Lindemann / Troe forms, backward rates from the
// Gibbs energy, rates of progress, species source). Stoichiometric
// coefficients sit in __constant__ memory; zero coefficients are skipped
// (multiplying by pow(c,0) = 1 or adding 0 is exact) and c^nu uses exact
// small-integer powers. Transport follows
// src/Transport.cu:40-109 (Wilke viscosity, the 1.065/0.065 conductivity
// rule, mixture-averaged rho*D_k).
#pragma once
#include "common.cuh"
#include "thermo.cuh"

namespace ostc {

__device__ __forceinline__ double ipow(double c, int n) {
  switch (n) {
    case 0: return 1.0;
    case 1: return c;
    case 2: return c * c;
    case 3: return c * c * c;
    default: return pow(c, (double)n);
  }
}

// A t^b exp(-Ea/t) as one exponential: A exp(b ln t - Ea / t)
__device__ __forceinline__ double arrhenius(double lnT, double invT, double A, double b, double Ea) {
  return A * exp(b * lnT - Ea * invT);
}

// rate of progress of reaction r: q1 = kf prod c^nu', q2 = kb prod c^nu''
// (forward_reaction_rate, backward_reaction_rate and rate_of_progress of
// FiniteRateChem.cu:65-176 for one reaction); g is the Gibbs energy / RT
template <int NS>
__device__ __forceinline__ void reaction_q(int r, double t, double lnT, double invT, double ln_temp_t,
                                           const double *c, const double *g, double &q1, double &q2) {
  const int type = c_p.reac_type[r];
  double kf = arrhenius(lnT, invT, c_p.A[r], c_p.b[r], c_p.Ea[r]);
  if (type == 3) kf += arrhenius(lnT, invT, c_p.A2[r], c_p.b2[r], c_p.Ea2[r]);
  if (type > 3) {
    double cc = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) cc += c[l] * c_p.tb[r][l];
    if (type == 4) {
      kf *= cc;
    } else {
      const double kf_low = arrhenius(lnT, invT, c_p.A2[r], c_p.b2[r], c_p.Ea2[r]);
      const double kf_high = kf;
      const double pr = kf_low * cc / kf_high;
      double F = 1.0;
      if (type > 5) {
        double f_cent = (1 - c_p.troe_alpha[r]) * exp(-t / c_p.troe_t3[r]) + c_p.troe_alpha[r] * exp(-t / c_p.troe_t1[r]);
        if (type == 7) f_cent += exp(-c_p.troe_t2[r] / t);
        const double logFc = log10(f_cent);
        const double cc2 = -0.4 - 0.67 * logFc;
        const double nn = 0.75 - 1.27 * logFc;
        const double logPr = log10(pr);
        const double tempo = (logPr + cc2) / (nn - 0.14 * (logPr + cc2));
        const double pp = logFc / (1.0 + tempo * tempo);
        F = pow(10.0, pp);
      }
      kf = kf_high * pr / (1.0 + pr) * F;
    }
  }
  double kb = 0;
  if (type == 2) {
    kb = arrhenius(lnT, invT, c_p.A2[r], c_p.b2[r], c_p.Ea2[r]);
  } else if (type != 0) {
    double dg = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) dg += g[l] * (c_p.nub[r][l] - c_p.nuf[r][l]);
    // kf / (temp_t^order exp(-dg)) as one exponential
    kb = kf * exp(dg - c_p.reac_order[r] * ln_temp_t);
  }
  // species in increasing order, as the reference's loop
  q1 = 1.0;
  q2 = 1.0;
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    const int nf = c_p.nuf[r][l], nb = c_p.nub[r][l];
    if (nf) q1 *= ipow(c[l], nf);
    if (nb && type != 0) q2 *= ipow(c[l], nb);
  }
  q1 *= kf;
  if (type != 0) q2 *= kb; else q2 = 0.0;
}

// concentrations in mol/cm^3 and the Gibbs terms shared by all reactions
template <int NS>
__device__ __forceinline__ void chemistry_setup(double rho, double t, const double *Y, double *c, double *g,
                                                double &lnT, double &invT, double &ln_temp_t) {
#pragma unroll
  for (int l = 0; l < NS; ++l) c[l] = rho * Y[l] * c_p.imw[l] * 1e-3;
  if (c_p.need_gibbs) gibbs_div_rt<NS>(t, g);
  constexpr double temp_p = p_atm / R_u * 1e-3;
  const double temp_t = temp_p / t;
  lnT = log(t);
  invT = 1.0 / t;
  ln_temp_t = log(temp_t);
}

// omega[NS] in kg/(m^3 s) at density rho, temperature t, mass fractions Y
template <int NS>
__device__ __forceinline__ void chemistry_omega(double rho, double t, const double *Y, double *omega) {
  double c[NS], g[NS];
  double lnT, invT, ln_temp_t;
  chemistry_setup<NS>(rho, t, Y, c, g, lnT, invT, ln_temp_t);
  double cre[NS], des[NS];
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    cre[l] = 0;
    des[l] = 0;
  }
  const int nr = c_p.n_reac;
  for (int r = 0; r < nr; ++r) {
    double q1, q2;
    reaction_q<NS>(r, t, lnT, invT, ln_temp_t, c, g, q1, q2);
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      const int nf = c_p.nuf[r][l], nb = c_p.nub[r][l];
      if (nf | nb) {
        cre[l] += q2 * nf + q1 * nb;
        des[l] += q1 * nf + q2 * nb;
      }
    }
  }
#pragma unroll
  for (int l = 0; l < NS; ++l) omega[l] = cre[l] * (c_p.mw[l] * 1e+3) - des[l] * (c_p.mw[l] * 1e+3);
}

// Rates of progress of all reactions plus omega and its destruction part
// omega_d (chemical_source, FiniteRateChem.cu:178-194): the inputs of the
// chemical Jacobians.
template <int NS>
__device__ __forceinline__ void chemistry_rates(double rho, double t, const double *Y, double *q1, double *q2,
                                                double *omega, double *omega_d) {
  double c[NS], g[NS];
  double lnT, invT, ln_temp_t;
  chemistry_setup<NS>(rho, t, Y, c, g, lnT, invT, ln_temp_t);
  double cre[NS], des[NS];
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    cre[l] = 0;
    des[l] = 0;
  }
  const int nr = c_p.n_reac;
  for (int r = 0; r < nr; ++r) {
    reaction_q<NS>(r, t, lnT, invT, ln_temp_t, c, g, q1[r], q2[r]);
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      const int nf = c_p.nuf[r][l], nb = c_p.nub[r][l];
      if (nf | nb) {
        cre[l] += q2[r] * nf + q1[r] * nb;
        des[l] += q1[r] * nf + q2[r] * nb;
      }
    }
  }
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    omega[l] = cre[l] * (c_p.mw[l] * 1e+3) - des[l] * (c_p.mw[l] * 1e+3);
    omega_d[l] = des[l] * (c_p.mw[l] * 1e+3);
  }
}

// d omega_m / d (rho Y_n), row-major m * NS + n (compute_chem_src_jacobian,
// FiniteRateChem.cu:196-216): q in mol/(cm^3 s); columns of absent species
// (Y_n <= 1e-25) are zero
template <int NS>
__device__ __forceinline__ void chemistry_jacobian(double rho, const double *Y, const double *q1, const double *q2,
                                                   double *J) {
  const int nr = c_p.n_reac;
#pragma unroll 1
  for (int m = 0; m < NS; ++m) {
#pragma unroll 1
    for (int n = 0; n < NS; ++n) {
      double zz = 0;
      if (Y[n] > 1e-25) {
        for (int r = 0; r < nr; ++r)
          zz += (c_p.nub[r][m] - c_p.nuf[r][m]) * (c_p.nuf[r][n] * q1[r] - c_p.nub[r][n] * q2[r]);
        zz /= rho * Y[n];
      }
      J[m * NS + n] = c_p.mw[m] * zz * 1e+3;
    }
  }
}

// Column-pivoted Crout LU factorisation in place (A row-major NS x NS) in
// the operation order of solve_chem_system (FiniteRateChem.cu:324-419)
template <int NS>
__device__ __forceinline__ void lu_factor(double *A, int *ipiv) {
#pragma unroll 1
  for (int n = 0; n < NS; ++n) {
    int ik = n;
    for (int m = n; m < NS; ++m) {
      for (int t = 0; t < n; ++t) A[m * NS + n] -= A[m * NS + t] * A[t * NS + n];
      if (fabs(A[m * NS + n]) > fabs(A[ik * NS + n])) ik = m;
    }
    ipiv[n] = ik;
    if (ik != n) {
      for (int t = 0; t < NS; ++t) {
        const double mid = A[ik * NS + t];
        A[ik * NS + t] = A[n * NS + t];
        A[n * NS + t] = mid;
      }
    }
    for (int p = n + 1; p < NS; ++p)
      for (int t = 0; t < n; ++t) A[n * NS + p] -= A[n * NS + t] * A[t * NS + p];
    for (int m = n + 1; m < NS; ++m) A[m * NS + n] /= A[n * NS + n];
  }
}

// b <- A^-1 b with the factors and pivots of lu_factor
template <int NS>
__device__ __forceinline__ void lu_apply(const double *A, const int *ipiv, double *b) {
#pragma unroll 1
  for (int m = 0; m < NS; ++m) {
    const int t = ipiv[m];
    if (t != m) {
      const double mid = b[t];
      b[t] = b[m];
      b[m] = mid;
    }
  }
#pragma unroll 1
  for (int m = 1; m < NS; ++m)
    for (int t = 0; t < m; ++t) b[m] -= A[m * NS + t] * b[t];
  b[NS - 1] /= A[NS * NS - 1];
#pragma unroll 1
  for (int m = NS - 2; m >= 0; --m) {
    for (int t = m + 1; t < NS; ++t) b[m] -= A[m * NS + t] * b[t];
    b[m] /= A[m * NS + m];
  }
}

template <int NS>
__device__ __forceinline__ void lu_solve(double *A, double *b) {
  int ipiv[NS];
  lu_factor<NS>(A, ipiv);
  lu_apply<NS>(A, ipiv, b);
}


// The FP64 point-implicit chemistry integrator of one state over dt at
// constant density and internal energy (no single reference function: it
// composes finite_rate_chemistry, compute_chem_src_jacobian and
// solve_chem_system, FiniteRateChem.cu:7-419, with the energy / temperature
// relation of compute_temperature_and_pressure, FieldOperation.cu:3-39):
//   rho from p = rho R_u T sum(Y/W); omega, J = d omega / d(rho Y) at (T, Y);
//   d(rho Y) = (I - dt J)^-1 dt omega; Y' = Y + d(rho Y) / rho;
//   T' solves e(T', Y') = e(T, Y), e = sum Y h(T) - R_u T sum(Y/W), by Newton
//   to |1 - T1/T| <= 1e-13 (at most 100 iterations; the reference's 1e-3
//   tolerance would leave kelvin-sized errors in an integrator that arbitrates the surrogate).
// Returns dY (NS) and dT; `iters` is the Newton count (0 if it failed).
template <int NS>
__device__ __forceinline__ void point_implicit_increment(double T, double p, const double *Y, double dt, double *dY,
                                                         double &dT, int &iters) {
  double mwinv = 0;
#pragma unroll
  for (int l = 0; l < NS; ++l) mwinv += Y[l] * c_p.imw[l];
  const double rho = p / (R_u * T * mwinv);
  double q1[OSTC_MAX_REAC], q2[OSTC_MAX_REAC], om[NS], od[NS];
  chemistry_rates<NS>(rho, T, Y, q1, q2, om, od);
  double A[NS * NS], b[NS];
  chemistry_jacobian<NS>(rho, Y, q1, q2, A);
#pragma unroll 1
  for (int m = 0; m < NS; ++m)
    for (int n = 0; n < NS; ++n) A[m * NS + n] = m == n ? 1.0 - dt * A[m * NS + n] : -dt * A[m * NS + n];
#pragma unroll
  for (int l = 0; l < NS; ++l) b[l] = dt * om[l];
  lu_solve<NS>(A, b);
  double Y1[NS], h[NS], cp[NS];
  enthalpy<NS>(T, h);
  double e0 = 0, mwinv1 = 0;
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    dY[l] = b[l] / rho;
    Y1[l] = Y[l] + dY[l];
    e0 += Y[l] * h[l];
    mwinv1 += Y1[l] * c_p.imw[l];
  }
  e0 -= R_u * T * mwinv;
  const double R1 = R_u * mwinv1;
  double t = T;
  iters = 0;
  for (int it = 1; it <= 100; ++it) {
    enthalpy_cp<NS, false>(t, h, cp);
    double hs = 0, cps = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      hs += Y1[l] * h[l];
      cps += Y1[l] * cp[l];
    }
    const double t1 = t - (hs - R1 * t - e0) / (cps - R1);
    const double err = fabs(1 - t1 / t);
    t = t1;
    if (err <= 1e-13) {
      iters = it;
      break;
    }
  }
  dT = t - T;
}

// compute_viscosity (Transport.cu:112-145): the mixture's Wilke viscosity at
// temperature T for mass fractions Y, the transport kernel's formula below
// with the viscosity alone (the SST wall and initial turbulent viscosity)
template <int NS>
__device__ __forceinline__ double mixture_viscosity(double T, const double *Y) {
  double mw_inv = 0;
#pragma unroll
  for (int l = 0; l < NS; ++l) mw_inv += Y[l] * c_p.imw[l];
  const double mw_total = 1.0 / mw_inv;
  double X[NS], vis[NS], svis[NS], rsvis[NS];
  const double sqT = sqrt(T);
  const double Tm145 = exp(-0.145 * log(T));
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    X[l] = Y[l] * mw_total * c_p.imw[l];
    const double t_dl = T * c_p.LJ_inv[l] + 0.5;
    const double ci = 1.147 * (Tm145 * c_p.LJm145[l]) + 1.0 / (t_dl * t_dl);
    vis[l] = c_p.vis_coeff[l] * sqT / ci;
    svis[l] = sqrt(vis[l]);
    rsvis[l] = 1.0 / svis[l];
  }
  double viscosity = 0;
#pragma unroll
  for (int m = 0; m < NS; ++m) {
    double vt = 0;
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      double pf = 1.0;
      if (m != n) {
        const double num = 1 + svis[m] * rsvis[n] * c_p.WjWi4[m][n];
        pf = num * num * c_p.sqWW8[m][n];
      }
      vt += pf * X[n];
    }
    viscosity += vis[m] * X[m] / vt;
  }
  return viscosity;
}

// mixture transport at one state (Transport.cu:40-109)
template <int NS>
__device__ __forceinline__ void mixture_transport(double T, double mw_total, const double *Y, const double *cp,
                                                  double rho, double p, double &mu, double &kappa, double *rhoD) {
  // T^-0.145 once; (T c)^-0.145 = T^-0.145 c^-0.145 with c^-0.145 from the host
  double X[NS], vis[NS], svis[NS], rsvis[NS];
  const double sqT = sqrt(T);
  const double Tm145 = exp(-0.145 * log(T));
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    X[l] = Y[l] * mw_total * c_p.imw[l];
    const double t_dl = T * c_p.LJ_inv[l] + 0.5;
    const double ci = 1.147 * (Tm145 * c_p.LJm145[l]) + 1.0 / (t_dl * t_dl);
    vis[l] = c_p.vis_coeff[l] * sqT / ci;
    svis[l] = sqrt(vis[l]);
    rsvis[l] = 1.0 / svis[l];
  }
  double viscosity = 0, conductivity = 0;
#pragma unroll
  for (int m = 0; m < NS; ++m) {
    double vt = 0;
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      double pf = 1.0;
      if (m != n) {  // sqrt(vis_m / vis_n) = sqrt(vis_m) / sqrt(vis_n)
        const double num = 1 + svis[m] * rsvis[n] * c_p.WjWi4[m][n];
        pf = num * num * c_p.sqWW8[m][n];
      }
      vt += pf * X[n];
    }
    const double ct = 1.065 * vt - 0.065 * X[m];
    viscosity += vis[m] * X[m] / vt;
    const double lambda = vis[m] * (cp[m] + 1.25 * c_p.Rmw[m]);
    conductivity += lambda * X[m] / ct;
  }
  mu = viscosity;
  kappa = conductivity;
  // 1 / D_mn = Omega_D / (bdc T^1.5 / p), Omega_D = t_red^-0.145 + (t_red + 0.5)^-2
  const double inv_t32p = p / (T * sqT);
  double dinv[NS][NS];
#pragma unroll
  for (int m = 0; m < NS; ++m) {
#pragma unroll
    for (int n = m + 1; n < NS; ++n) {
      const double tr = T * c_p.kbe[m][n] + 0.5;
      const double od = Tm145 * c_p.kbem145[m][n] + 1.0 / (tr * tr);
      const double di = od * c_p.inv_bdc[m][n] * inv_t32p;
      dinv[m][n] = di;
      dinv[n][m] = di;
    }
  }
  constexpr double eps = 1e-12;
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    double num = 0, den = 0;
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      if (l != n) {
        num += (X[n] + eps) * c_p.mw[n];
        den += (X[n] + eps) * dinv[l][n];
      }
    }
    rhoD[l] = rho * num / (den * mw_total);
  }
}

}  // namespace ostc
