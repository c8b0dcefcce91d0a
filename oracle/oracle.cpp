// oracle.cpp — CPU restatement (test infrastructure) of the OpenSTC-dev RHS and
// RK3 path. Every function cites the reference file:line whose arithmetic it
// restates; operation order is kept so that results agree with the reference
// functions compiled as host code to the last few ulps.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <cstdio>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double R_u = 8314.462618;       // src/Constants.h:17
constexpr double p_atm = 101325;          // src/Constants.h:23
constexpr double gamma_air = 1.4;         // src/Constants.h:21
constexpr double mw_air = 28.9647;        // src/Constants.h:27
constexpr int MAXS = OSTC_MAX_SPEC;
constexpr int MAXR = OSTC_MAX_REAC;

// ---------------------------------------------------------------------------
// array views in the ggxl ColMajor layout (src/gxl_lib/Array.hpp:146-194)
// ---------------------------------------------------------------------------
struct View {
  double *p = nullptr;
  long disp2 = 0, disp1 = 0, dispt = 0, sz = 0;
  View() = default;
  View(double *ptr, int mx, int my, int mz, int g) : p(ptr) {
    disp2 = mx + 2 * g;
    disp1 = (long)(my + 2 * g) * disp2;
    dispt = (disp1 + disp2 + 1) * g;
    sz = (long)(mx + 2 * g) * (my + 2 * g) * (mz + 2 * g);
  }
  double &operator()(int i, int j, int k, int l = 0) const {
    return p[(long)k * disp1 + (long)j * disp2 + i + dispt + (long)l * sz];
  }
};

// gxl::Matrix<real,3,3,1>: int bias + pad, then 9 doubles (src/gxl_lib/Matrix.hpp:214-233)
struct MetricView {
  const unsigned char *p = nullptr;
  long disp2 = 0, disp1 = 0, dispt = 0;
  MetricView() = default;
  MetricView(const void *ptr, int mx, int my, int mz, int g) : p((const unsigned char *)ptr) {
    disp2 = mx + 2 * g;
    disp1 = (long)(my + 2 * g) * disp2;
    dispt = (disp1 + disp2 + 1) * g;
  }
  // m(d, c) with d, c 1-based as in the reference: row d = (xi, eta, zeta)
  const double *at(int i, int j, int k) const {
    return (const double *)(p + 80 * ((long)k * disp1 + (long)j * disp2 + i + dispt) + 8);
  }
};

struct Z {  // a zone with views
  const ostc_zone *z;
  int mx, my, mz, ngg;
  View bv, sv, cv, qn, dq, jac, vel, a, mach, mul, kappa, rhoD, gam, cp, dt_local, bv_last, mut, ttc, wall, tsj;
  MetricView metric;
  explicit Z(const ostc_zone *zz) : z(zz), mx(zz->mx), my(zz->my), mz(zz->mz), ngg(zz->ngg) {
    const int g = ngg;
    bv = View(zz->bv, mx, my, mz, g);
    sv = View(zz->sv, mx, my, mz, g);
    cv = View(zz->cv, mx, my, mz, g);
    qn = View(zz->qn, mx, my, mz, g);
    dq = View(zz->dq, mx, my, mz, zz->dq_ngg);
    jac = View(const_cast<double *>(zz->jac), mx, my, mz, g);
    vel = View(zz->vel, mx, my, mz, g);
    a = View(zz->acoustic_speed, mx, my, mz, g);
    mach = View(zz->mach, mx, my, mz, g);
    mul = View(zz->mul, mx, my, mz, g);
    kappa = View(zz->thermal_conductivity, mx, my, mz, g);
    rhoD = View(zz->rho_D, mx, my, mz, g);
    gam = View(zz->gamma, mx, my, mz, g);
    cp = View(zz->cp, mx, my, mz, g);
    mut = View(zz->mut, mx, my, mz, g);
    ttc = View(zz->turb_therm_cond, mx, my, mz, g);
    wall = View(zz->wall_distance, mx, my, mz, g);
    tsj = View(zz->turb_src_jac, mx, my, mz, 0);
    dt_local = View(zz->dt_local, mx, my, mz, 0);
    bv_last = View(zz->bv_last, mx, my, mz, 0);
    metric = MetricView(zz->metric, mx, my, mz, g);
  }
};

inline double coeff(const double *tab, int i, int c) { return tab[i * 7 + c]; }

// ---------------------------------------------------------------------------
// thermodynamics: src/Thermo.cu:5-79
// ---------------------------------------------------------------------------
void enthalpy(const ostc_param *P, double t, double *h) {  // Thermo.cu:5-23
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  for (int i = 0; i < P->n_spec; ++i) {
    if (t < P->t_low[i]) {
      const double tt = P->t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      const double *c = P->low_temp_coeff;
      h[i] = coeff(c, i, 0) * tt + 0.5 * coeff(c, i, 1) * tt2 + coeff(c, i, 2) * tt3 / 3 +
             0.25 * coeff(c, i, 3) * tt4 + 0.2 * coeff(c, i, 4) * tt5 + coeff(c, i, 5);
      const double cpv = coeff(c, i, 0) + coeff(c, i, 1) * tt + coeff(c, i, 2) * tt2 +
                         coeff(c, i, 3) * tt3 + coeff(c, i, 4) * tt4;
      h[i] += cpv * (t - tt);
    } else {
      const double *c = t < P->t_mid[i] ? P->low_temp_coeff : P->high_temp_coeff;
      h[i] = coeff(c, i, 0) * t + 0.5 * coeff(c, i, 1) * t2 + coeff(c, i, 2) * t3 / 3 +
             0.25 * coeff(c, i, 3) * t4 + 0.2 * coeff(c, i, 4) * t5 + coeff(c, i, 5);
    }
    h[i] *= R_u / P->mw[i];
  }
}

void enthalpy_and_cp(const ostc_param *P, double t, double *h, double *cp) {  // Thermo.cu:25-45
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  for (int i = 0; i < P->n_spec; ++i) {
    if (t < P->t_low[i]) {
      const double tt = P->t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      const double *c = P->low_temp_coeff;
      h[i] = coeff(c, i, 0) * tt + 0.5 * coeff(c, i, 1) * tt2 + coeff(c, i, 2) * tt3 / 3 +
             0.25 * coeff(c, i, 3) * tt4 + 0.2 * coeff(c, i, 4) * tt5 + coeff(c, i, 5);
      cp[i] = coeff(c, i, 0) + coeff(c, i, 1) * tt + coeff(c, i, 2) * tt2 + coeff(c, i, 3) * tt3 +
              coeff(c, i, 4) * tt4;
      h[i] += cp[i] * (t - tt);
    } else {
      const double *c = t < P->t_mid[i] ? P->low_temp_coeff : P->high_temp_coeff;
      h[i] = coeff(c, i, 0) * t + 0.5 * coeff(c, i, 1) * t2 + coeff(c, i, 2) * t3 / 3 +
             0.25 * coeff(c, i, 3) * t4 + 0.2 * coeff(c, i, 4) * t5 + coeff(c, i, 5);
      cp[i] = coeff(c, i, 0) + coeff(c, i, 1) * t + coeff(c, i, 2) * t2 + coeff(c, i, 3) * t3 +
              coeff(c, i, 4) * t4;
    }
    h[i] *= R_u / P->mw[i];
    cp[i] *= R_u / P->mw[i];
  }
}

void cp_only(const ostc_param *P, double t, double *cp) {  // Thermo.cu:47-61
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t;
  for (int i = 0; i < P->n_spec; ++i) {
    if (t < P->t_low[i]) {
      const double tt = P->t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
      const double *c = P->low_temp_coeff;
      cp[i] = coeff(c, i, 0) + coeff(c, i, 1) * tt + coeff(c, i, 2) * tt2 + coeff(c, i, 3) * tt3 +
              coeff(c, i, 4) * tt4;
    } else {
      const double *c = t < P->t_mid[i] ? P->low_temp_coeff : P->high_temp_coeff;
      cp[i] = coeff(c, i, 0) + coeff(c, i, 1) * t + coeff(c, i, 2) * t2 + coeff(c, i, 3) * t3 +
              coeff(c, i, 4) * t4;
    }
    cp[i] *= R_u / P->mw[i];
  }
}

void gibbs_div_rt(const ostc_param *P, double t, double *g) {  // Thermo.cu:63-79
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t_inv = 1 / t, log_t = std::log(t);
  for (int i = 0; i < P->n_spec; ++i) {
    if (t < P->t_low[i]) {
      const double tt = P->t_low[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt_inv = 1 / tt, log_tt = std::log(tt);
      const double *c = P->low_temp_coeff;
      g[i] = coeff(c, i, 0) * (1.0 - log_tt) - 0.5 * coeff(c, i, 1) * tt - coeff(c, i, 2) * tt2 / 6.0 -
             coeff(c, i, 3) * tt3 / 12.0 - coeff(c, i, 4) * tt4 * 0.05 + coeff(c, i, 5) * tt_inv -
             coeff(c, i, 6);
    } else {
      const double *c = t < P->t_mid[i] ? P->low_temp_coeff : P->high_temp_coeff;
      g[i] = coeff(c, i, 0) * (1.0 - log_t) - 0.5 * coeff(c, i, 1) * t - coeff(c, i, 2) * t2 / 6.0 -
             coeff(c, i, 3) * t3 / 12.0 - coeff(c, i, 4) * t4 * 0.05 + coeff(c, i, 5) * t_inv -
             coeff(c, i, 6);
    }
  }
}

// ---------------------------------------------------------------------------
// transport: src/Transport.cu:6-145
// ---------------------------------------------------------------------------
double sutherland(double t) {  // Transport.cu:6-9
  return 1.716e-5 * std::pow(t / 273, 1.5) * (273 + 111) / (t + 111);
}

double omega_d(double t_red) {  // Transport.cu:142-145
  return 1.0 / std::pow(t_red, 0.145) + 1.0 / ((t_red + 0.5) * (t_red + 0.5));
}

// compute_viscosity (Transport.cu:112-145): the Wilke viscosity of a mixture
// at temperature T (the SST wall and the initial turbulent viscosity)
double mixture_viscosity(const ostc_param *P, double temperature, const double *Y) {
  const int ns = P->n_spec;
  const double *mw = P->mw;
  double mw_total = 0;
  for (int l = 0; l < ns; ++l) mw_total += Y[l] / mw[l];
  mw_total = 1 / mw_total;
  double X[MAXS], vis[MAXS];
  for (int l = 0; l < ns; ++l) {
    X[l] = Y[l] * mw_total / mw[l];
    const double t_dl = temperature * P->LJ_potent_inv[l];
    const double ci = 1.147 * std::pow(t_dl, -0.145) + std::pow(t_dl + 0.5, -2);
    vis[l] = P->vis_coeff[l] * std::sqrt(temperature) / ci;
  }
  double viscosity = 0;
  for (int m = 0; m < ns; ++m) {
    double vis_temp = 0;
    for (int n = 0; n < ns; ++n) {
      double pf = 1.0;
      if (m != n) {
        const double num = 1 + std::sqrt(vis[m] / vis[n]) * P->WjDivWi_to_One4th[m * ns + n];
        pf = num * num * P->sqrt_WiDivWjPl1Mul8[m * ns + n];
      }
      vis_temp += pf * X[n];
    }
    viscosity += vis[m] * X[m] / vis_temp;
  }
  return viscosity;
}

// compute_transport_property (Transport.cu:40-109): mu, kappa, rho*D_k
void transport(const ostc_param *P, double temperature, double mw_total, const double *Y,
               const double *cp, double rho, double pressure, double *mu_out, double *kappa_out,
               double *rhoD) {
  const int ns = P->n_spec;
  const double *mw = P->mw;
  double X[MAXS], vis[MAXS], d_ij[MAXS * MAXS];
  for (int l = 0; l < ns; ++l) {
    X[l] = Y[l] * mw_total / mw[l];
    const double t_dl = temperature * P->LJ_potent_inv[l];
    const double ci = 1.147 * std::pow(t_dl, -0.145) + std::pow(t_dl + 0.5, -2);
    vis[l] = P->vis_coeff[l] * std::sqrt(temperature) / ci;
  }
  double viscosity = 0, conductivity = 0;
  for (int m = 0; m < ns; ++m) {
    double vis_temp = 0;
    for (int n = 0; n < ns; ++n) {
      double pf = 1.0;
      if (m != n) {
        const double num = 1 + std::sqrt(vis[m] / vis[n]) * P->WjDivWi_to_One4th[m * ns + n];
        pf = num * num * P->sqrt_WiDivWjPl1Mul8[m * ns + n];
      }
      vis_temp += pf * X[n];
    }
    const double cond_temp = 1.065 * vis_temp - 0.065 * X[m];
    viscosity += vis[m] * X[m] / vis_temp;
    const double lambda = vis[m] * (cp[m] + 1.25 * R_u / mw[m]);
    conductivity += lambda * X[m] / cond_temp;
  }
  *mu_out = viscosity;
  *kappa_out = conductivity;
  const double t32p = temperature * std::sqrt(temperature) / pressure;
  for (int m = 0; m < ns; ++m) {
    for (int n = m + 1; n < ns; ++n) {
      const double t_red = temperature * P->kb_over_eps_jk[m * ns + n];
      d_ij[m * ns + n] = P->binary_diffusivity_coeff[m * ns + n] * t32p / omega_d(t_red);
      d_ij[n * ns + m] = d_ij[m * ns + n];
    }
  }
  constexpr double eps = 1e-12;
  for (int l = 0; l < ns; ++l) {
    double num = 0, den = 0;
    for (int n = 0; n < ns; ++n) {
      if (l != n) {
        num += (X[n] + eps) * mw[n];
        den += (X[n] + eps) / d_ij[l * ns + n];
      }
    }
    rhoD[l] = rho * num / (den * mw_total);
  }
}

// ---------------------------------------------------------------------------
// finite-rate chemistry: src/FiniteRateChem.cu:7-194
// ---------------------------------------------------------------------------
double arrhenius(double t, double A, double b, double Ea) {  // FiniteRateChem.cu:110-112
  return A * std::pow(t, b) * std::exp(-Ea / t);
}

void chemistry_omega(const ostc_param *P, double density, double t, const double *Y,
                     double *omega, double *q1o, double *q2o, double *odo = nullptr) {  // FiniteRateChem.cu:7-63
  const int ns = P->n_spec, nr = P->n_reac;
  double c[MAXS] = {0};
  for (int l = 0; l < ns; ++l) c[l] = density * Y[l] / P->mw[l] * 1e-3;
  double kf[MAXR] = {0}, kb[MAXR] = {0};
  // forward_reaction_rate, FiniteRateChem.cu:65-108
  for (int i = 0; i < nr; ++i) {
    kf[i] = arrhenius(t, P->A[i], P->b[i], P->Ea[i]);
    const int type = P->reac_type[i];
    if (type == 3) kf[i] += arrhenius(t, P->A2[i], P->b2[i], P->Ea2[i]);
    if (type > 3) {
      double cc = 0;
      for (int l = 0; l < ns; ++l) cc += c[l] * P->third_body_coeff[i * ns + l];
      if (type == 4) {
        kf[i] *= cc;
      } else {
        const double kf_low = arrhenius(t, P->A2[i], P->b2[i], P->Ea2[i]);
        const double kf_high = kf[i];
        const double pr = kf_low * cc / kf_high;
        double F = 1.0;
        if (type > 5) {
          double f_cent = (1 - P->troe_alpha[i]) * std::exp(-t / P->troe_t3[i]) +
                          P->troe_alpha[i] * std::exp(-t / P->troe_t1[i]);
          if (type == 7) f_cent += std::exp(-P->troe_t2[i] / t);
          const double logFc = std::log10(f_cent);
          const double cc2 = -0.4 - 0.67 * logFc;
          const double n = 0.75 - 1.27 * logFc;
          const double logPr = std::log10(pr);
          const double tempo = (logPr + cc2) / (n - 0.14 * (logPr + cc2));
          const double pp = logFc / (1.0 + tempo * tempo);
          F = std::pow(10, pp);
        }
        kf[i] = kf_high * pr / (1.0 + pr) * F;
      }
    }
  }
  // backward_reaction_rate, FiniteRateChem.cu:114-149
  int n_gibbs = nr;
  for (int i = 0; i < nr; ++i) {
    if (P->reac_type[i] == 0) {
      kb[i] = 0;
      --n_gibbs;
    } else if (P->reac_type[i] == 2) {
      kb[i] = arrhenius(t, P->A2[i], P->b2[i], P->Ea2[i]);
      --n_gibbs;
    }
  }
  if (n_gibbs >= 1) {
    double g[MAXS] = {0};
    gibbs_div_rt(P, t, g);
    constexpr double temp_p = p_atm / R_u * 1e-3;
    const double temp_t = temp_p / t;
    for (int i = 0; i < nr; ++i) {
      if (P->reac_type[i] != 2 && P->reac_type[i] != 0) {
        double dg = 0;
        for (int l = 0; l < ns; ++l) dg += g[l] * (P->stoi_b[i * ns + l] - P->stoi_f[i * ns + l]);
        const double kc = std::pow(temp_t, P->reac_order[i]) * std::exp(-dg);
        kb[i] = kf[i] / kc;
      }
    }
  }
  // rate_of_progress, FiniteRateChem.cu:151-176
  double q1[MAXR], q2[MAXR];
  for (int i = 0; i < nr; ++i) {
    if (P->reac_type[i] != 0) {
      q1[i] = 1.0;
      q2[i] = 1.0;
      for (int j = 0; j < ns; ++j) {
        q1[i] *= std::pow(c[j], P->stoi_f[i * ns + j]);
        q2[i] *= std::pow(c[j], P->stoi_b[i * ns + j]);
      }
      q1[i] *= kf[i];
      q2[i] *= kb[i];
    } else {
      q1[i] = 1.0;
      q2[i] = 0.0;
      for (int j = 0; j < ns; ++j) q1[i] *= std::pow(c[j], P->stoi_f[i * ns + j]);
      q1[i] *= kf[i];
    }
  }
  // chemical_source, FiniteRateChem.cu:178-194
  for (int i = 0; i < ns; ++i) {
    double creation = 0, od = 0;
    for (int j = 0; j < nr; ++j) {
      creation += q2[j] * P->stoi_f[j * ns + i] + q1[j] * P->stoi_b[j * ns + i];
      od += q1[j] * P->stoi_f[j * ns + i] + q2[j] * P->stoi_b[j * ns + i];
    }
    creation *= P->mw[i] * 1e+3;
    od *= P->mw[i] * 1e+3;
    omega[i] = creation - od;
    if (odo) odo[i] = od;
  }
  if (q1o) for (int i = 0; i < nr; ++i) q1o[i] = q1[i];
  if (q2o) for (int i = 0; i < nr; ++i) q2o[i] = q2[i];
}

// ---------------------------------------------------------------------------
// reconstruction: src/Reconstruction.cu:5-46, src/Reconstruction.cuh:20-72,
// src/Limiter.cuh:13-16 (minmod with sgn(0)=+1, src/gxl_lib/Math.hpp:13-15)
// ---------------------------------------------------------------------------
inline int sgn(double a) { return a < 0 ? -1 : 1; }
inline double minmod(double a, double b) {
  return 0.5 * (sgn(a) + sgn(b)) * std::min(std::abs(a), std::abs(b));
}

// pv: rows of nv values, row index = point; pv_l/pv_r get nv + 2 values
void reconstruct(const ostc_param *P, const double *pv, double *pl, double *pr, int is, int nv) {
  switch (P->reconstruction) {
    case 2: {
      constexpr double kappa = 1.0 / 3.0;
      for (int l = 0; l < nv; ++l) {
        const double di = pv[is * nv + l] - pv[(is - 1) * nv + l];
        const double di1 = pv[(is + 1) * nv + l] - pv[is * nv + l];
        const double di2 = pv[(is + 2) * nv + l] - pv[(is + 1) * nv + l];
        const double dnl = minmod(di, di1), dpl = minmod(di1, di);
        const double dnr = minmod(di1, di2), dpr = minmod(di2, di1);
        pl[l] = pv[is * nv + l] + 0.25 * ((1 - kappa) * dnl + (1 + kappa) * dpl);
        pr[l] = pv[(is + 1) * nv + l] - 0.25 * ((1 - kappa) * dpr + (1 + kappa) * dnr);
      }
      break;
    }
    case 3:
      for (int l = 0; l < nv; ++l) {
        const double di = pv[is * nv + l] - pv[(is - 1) * nv + l];
        const double di1 = pv[(is + 1) * nv + l] - pv[is * nv + l];
        const double di2 = pv[(is + 2) * nv + l] - pv[(is + 1) * nv + l];
        pl[l] = pv[is * nv + l] + 0.5 * minmod(di, di1);
        pr[l] = pv[(is + 1) * nv + l] - 0.5 * minmod(di1, di2);
      }
      break;
    default:
      for (int l = 0; l < nv; ++l) {
        pl[l] = pv[is * nv + l];
        pr[l] = pv[(is + 1) * nv + l];
      }
  }
  if (P->mix_model != OSTC_MIX_AIR) {
    double el = 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]);
    double er = 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
    const int ns = P->n_spec;
    double mwl = 0, mwr = 0;
    for (int l = 0; l < ns; ++l) {
      mwl += pl[5 + l] / P->mw[l];
      mwr += pr[5 + l] / P->mw[l];
    }
    const double tl = pl[4] / (pl[0] * R_u * mwl);
    const double tr = pr[4] / (pr[0] * R_u * mwr);
    double hl[MAXS], hr[MAXS], cpl_i[MAXS], cpr_i[MAXS];
    enthalpy_and_cp(P, tl, hl, cpl_i);
    enthalpy_and_cp(P, tr, hr, cpr_i);
    double cpl = 0, cpr = 0, cvl = 0, cvr = 0;
    for (int l = 0; l < ns; ++l) {
      cpl += cpl_i[l] * pl[l + 5];
      cpr += cpr_i[l] * pr[l + 5];
      cvl += pl[l + 5] * (cpl_i[l] - R_u / P->mw[l]);
      cvr += pr[l + 5] * (cpr_i[l] - R_u / P->mw[l]);
      el += hl[l] * pl[l + 5];
      er += hr[l] * pr[l + 5];
    }
    pl[nv] = pl[0] * el - pl[4];
    pr[nv] = pr[0] * er - pr[4];
    pl[nv + 1] = cpl / cvl;
    pr[nv + 1] = cpr / cvr;
  } else {
    const double el = 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]);
    const double er = 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
    pl[nv] = el * pl[0] + pl[4] / (gamma_air - 1);
    pr[nv] = er * pr[0] + pr[4] / (gamma_air - 1);
  }
}

// ---------------------------------------------------------------------------
// Riemann fluxes. met: 3 metric components per point of the line, jac: per point
// ---------------------------------------------------------------------------
// AUSM+: src/AusmP.cu:6-94
void ausm_plus(const ostc_param *P, const double *pl, const double *pr, const double *met,
               const double *jac, int is, double *fci) {
  const double *ml = &met[is * 3], *mr = &met[(is + 1) * 3];
  const double jl = jac[is], jr = jac[is + 1];
  const double k1 = 0.5 * (jl * ml[0] + jr * mr[0]);
  const double k2 = 0.5 * (jl * ml[1] + jr * mr[1]);
  const double k3 = 0.5 * (jl * ml[2] + jr * mr[2]);
  const double gk = std::sqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const double ul = (k1 * pl[1] + k2 * pl[2] + k3 * pl[3]) / gk;
  const double ur = (k1 * pr[1] + k2 * pr[2] + k3 * pr[3]) / gk;
  const double p_l = pl[4], p_r = pr[4], rl = pl[0], rr = pr[0];
  const int nv = P->n_var;
  double gl = gamma_air, gr = gamma_air;
  if (P->mix_model != OSTC_MIX_AIR) {
    gl = pl[nv + 1];
    gr = pr[nv + 1];
  }
  const double c = 0.5 * (std::sqrt(gl * p_l / rl) + std::sqrt(gr * p_r / rr));
  const double mlm = ul / c, mrm = ur / c;
  double mlp, mrn, plp, prn;
  constexpr double alpha = 3 / 16.0;
  if (std::abs(mlm) > 1) {
    mlp = 0.5 * (mlm + std::abs(mlm));
    plp = mlp / mlm;
  } else {
    const double a = (mlm + 1) * (mlm + 1) * 0.25;
    const double b = (mlm * mlm - 1) * (mlm * mlm - 1);
    mlp = a + 0.125 * b;
    plp = a * (2 - mlm) + alpha * mlm * b;
  }
  if (std::abs(mrm) > 1) {
    mrn = 0.5 * (mrm - std::abs(mrm));
    prn = mrn / mrm;
  } else {
    const double a = (mrm - 1) * (mrm - 1) * 0.25;
    const double b = (mrm * mrm - 1) * (mrm * mrm - 1);
    mrn = -a - 0.125 * b;
    prn = a * (2 + mrm) - alpha * mrm * b;
  }
  const double p_coeff = plp * p_l + prn * p_r;
  const double m_half = mlp + mrn;
  const double mpos = 0.5 * (m_half + std::abs(m_half));
  const double mneg = 0.5 * (m_half - std::abs(m_half));
  const double mass = c * (rl * mpos + rr * mneg);
  const double co = mass * gk;
  const double *q = mass >= 0 ? pl : pr;
  fci[0] = co;
  fci[1] = co * q[1] + p_coeff * k1;
  fci[2] = co * q[2] + p_coeff * k2;
  fci[3] = co * q[3] + p_coeff * k3;
  fci[4] = co * (q[nv] + q[4]) / q[0];
  for (int l = 5; l < nv; ++l) fci[l] = co * q[l];
}

// HLLC: src/HLLC.cu:10-143
void hllc(const ostc_param *P, const double *pl, const double *pr, const double *met,
          const double *jac, int is, double *fci) {
  const int nv = P->n_var;
  const double rlc = std::sqrt(pl[0]) / (std::sqrt(pl[0]) + std::sqrt(pr[0]));
  const double rrc = std::sqrt(pr[0]) / (std::sqrt(pl[0]) + std::sqrt(pr[0]));
  const double ut = pl[1] * rlc + pr[1] * rrc;
  const double vt = pl[2] * rlc + pr[2] * rrc;
  const double wt = pl[3] * rlc + pr[3] * rrc;
  const double hl = (pl[nv] + pl[4]) / pl[0];
  const double hr = (pr[nv] + pr[4]) / pr[0];
  const double ht = hl * rlc + hr * rrc;
  const double ekt = 0.5 * (ut * ut + vt * vt + wt * wt);
  double gamma = gamma_air, c_tilde = 0;
  double svm[MAXS + 4] = {0};
  for (int l = 0; l < nv - 5; ++l) svm[l] = rlc * pl[l + 5] + rrc * pr[l + 5];
  if (P->mix_model == OSTC_MIX_AIR) {
    c_tilde = std::sqrt((gamma - 1) * (ht - ekt));
  } else {
    double mw_inv = 0;
    for (int l = 0; l < P->n_spec; ++l) mw_inv += svm[l] / P->mw[l];
    const double tl = pl[4] / pl[0];
    const double tr = pr[4] / pr[0];
    const double t = (rlc * tl + rrc * tr) / (R_u * mw_inv);
    double h_i[MAXS], cp_i[MAXS];
    enthalpy_and_cp(P, t, h_i, cp_i);
    double cvv = 0, cpp = 0;
    for (int l = 0; l < P->n_spec; ++l) {
      cpp += cp_i[l] * svm[l];
      cvv += svm[l] * (cp_i[l] - R_u / P->mw[l]);
    }
    gamma = cpp / cvv;
    c_tilde = std::sqrt(gamma * R_u * mw_inv * t);
  }
  const double kx = 0.5 * (met[is * 3] + met[(is + 1) * 3]);
  const double ky = 0.5 * (met[is * 3 + 1] + met[(is + 1) * 3 + 1]);
  const double kz = 0.5 * (met[is * 3 + 2] + met[(is + 1) * 3 + 2]);
  const double gradK = std::sqrt(kx * kx + ky * ky + kz * kz);
  const double Ub = (kx * ut + ky * vt + kz * wt) / gradK;
  const double jac_ave = 0.5 * (jac[is] + jac[is + 1]);
  double gl = gamma_air, gr = gamma_air;
  if (P->mix_model != OSTC_MIX_AIR) {
    gl = pl[nv + 1];
    gr = pr[nv + 1];
  }
  const double Ul = kx * pl[1] + ky * pl[2] + kz * pl[3];
  const double cl = std::sqrt(gl * pl[4] / pl[0]);
  const double sl = std::min(Ul / gradK - cl, Ub - c_tilde);
  if (sl >= 0) {
    const double rhoUk = pl[0] * Ul;
    fci[0] = jac_ave * rhoUk;
    fci[1] = jac_ave * (rhoUk * pl[1] + pl[4] * kx);
    fci[2] = jac_ave * (rhoUk * pl[2] + pl[4] * ky);
    fci[3] = jac_ave * (rhoUk * pl[3] + pl[4] * kz);
    fci[4] = jac_ave * ((pl[nv] + pl[4]) * Ul);
    for (int l = 5; l < nv; ++l) fci[l] = jac_ave * rhoUk * pl[l];
    return;
  }
  const double Ur = kx * pr[1] + ky * pr[2] + kz * pr[3];
  const double cr = std::sqrt(gr * pr[4] / pr[0]);
  const double sr = std::max(Ur / gradK + cr, Ub + c_tilde);
  if (sr < 0) {
    const double rhoUk = pr[0] * Ur;
    fci[0] = jac_ave * rhoUk;
    fci[1] = jac_ave * (rhoUk * pr[1] + pr[4] * kx);
    fci[2] = jac_ave * (rhoUk * pr[2] + pr[4] * ky);
    fci[3] = jac_ave * (rhoUk * pr[3] + pr[4] * kz);
    fci[4] = jac_ave * ((pr[nv] + pr[4]) * Ur);
    for (int l = 5; l < nv; ++l) fci[l] = jac_ave * rhoUk * pr[l];
    return;
  }
  const double sm = ((pr[0] * Ur * (sr - Ur / gradK) - pl[0] * Ul * (sl - Ul / gradK)) / gradK + pl[4] - pr[4]) /
                    (pr[0] * (sr - Ur / gradK) - pl[0] * (sl - Ul / gradK));
  const double pm = pl[0] * (sl - Ul / gradK) * (sm - Ul / gradK) + pl[4];
  if (sm >= 0) {
    const double pC = 1.0 / (sl - sm);
    const double Q = jac_ave * pC * sm * (sl * gradK - Ul) * pl[0];
    fci[0] = Q;
    const double dP = (sl * pm - sm * pl[4]) * pC * jac_ave;
    fci[1] = Q * pl[1] + dP * kx;
    fci[2] = Q * pl[2] + dP * ky;
    fci[3] = Q * pl[3] + dP * kz;
    fci[4] = Q * pl[nv] / pl[0] + pC * jac_ave * (sl * pm * sm * gradK - sm * pl[4] * Ul);
    for (int l = 5; l < nv; ++l) fci[l] = Q * pl[l];
  } else {
    const double pC = 1.0 / (sr - sm);
    const double Q = jac_ave * pC * sm * (sr * gradK - Ur) * pr[0];
    fci[0] = Q;
    const double dP = (sr * pm - sm * pr[4]) * pC * jac_ave;
    fci[1] = Q * pr[1] + dP * kx;
    fci[2] = Q * pr[2] + dP * ky;
    fci[3] = Q * pr[3] + dP * kz;
    fci[4] = Q * pr[nv] / pr[0] + pC * jac_ave * (sr * pm * sm * gradK - sm * pr[4] * Ur);
    for (int l = 5; l < nv; ++l) fci[l] = Q * pr[l];
  }
}

// Lax-Friedrichs, air only: src/LaxFriedrichs.cu:13-49
void lax_friedrichs(const ostc_param *P, const double *pl, const double *pr, const double *met,
                    const double *jac, int is, double *fci) {
  const int nv = P->n_var;
  const double kx = 0.5 * (met[is * 3] + met[(is + 1) * 3]);
  const double ky = 0.5 * (met[is * 3 + 1] + met[(is + 1) * 3 + 1]);
  const double kz = 0.5 * (met[is * 3 + 2] + met[(is + 1) * 3 + 2]);
  const double gradK = std::sqrt(kx * kx + ky * ky + kz * kz);
  const double Ukl = pl[1] * kx + pl[2] * ky + pl[3] * kz;
  const double Ukr = pr[1] * kx + pr[2] * ky + pr[3] * kz;
  const double cl = std::sqrt(gamma_air * pl[4] / pl[0]);
  const double cr = std::sqrt(gamma_air * pr[4] / pr[0]);
  const double sr = std::max(std::abs(Ukl) + cl * gradK, std::abs(Ukr) + cr * gradK);
  const double hj = 0.5 * 0.5 * (jac[is] + jac[is + 1]);
  const double rUl = pl[0] * Ukl, rUr = pr[0] * Ukr;
  fci[0] = (rUl + rUr - sr * (pr[0] - pl[0])) * hj;
  fci[1] = (rUl * pl[1] + rUr * pr[1] + kx * (pl[4] + pr[4]) - sr * (pr[1] * pr[0] - pl[1] * pl[0])) * hj;
  fci[2] = (rUl * pl[2] + rUr * pr[2] + ky * (pl[4] + pr[4]) - sr * (pr[2] * pr[0] - pl[2] * pl[0])) * hj;
  fci[3] = (rUl * pl[3] + rUr * pr[3] + kz * (pl[4] + pr[4]) - sr * (pr[3] * pr[0] - pl[3] * pl[0])) * hj;
  fci[4] = ((pl[nv] + pl[4]) * Ukl + (pr[nv] + pr[4]) * Ukr - sr * (pr[nv] - pl[nv])) * hj;
}

// Roe flux-difference splitting with the Harten entropy fix: compute_half_sum_left_right_flux
// (Roe.cu:339-375) + Roe_compute_half_point_flux (Roe.cu:186-337). delta: entropy-fix width per point.
void roe_flux(const ostc_param *P, const double *pl, const double *pr, const double *met, const double *jac,
              const double *delta, int is, double *fc) {
  const int nv = P->n_var;
  double JacKx = jac[is] * met[is * 3], JacKy = jac[is] * met[is * 3 + 1], JacKz = jac[is] * met[is * 3 + 2];
  double Uk = pl[1] * JacKx + pl[2] * JacKy + pl[3] * JacKz;
  double coeff = Uk * pl[0];
  fc[0] = 0.5 * coeff;
  fc[1] = 0.5 * (coeff * pl[1] + pl[4] * JacKx);
  fc[2] = 0.5 * (coeff * pl[2] + pl[4] * JacKy);
  fc[3] = 0.5 * (coeff * pl[3] + pl[4] * JacKz);
  fc[4] = 0.5 * Uk * (pl[4] + pl[nv]);
  for (int l = 5; l < nv; ++l) fc[l] = 0.5 * coeff * pl[l];
  JacKx = jac[is + 1] * met[(is + 1) * 3];
  JacKy = jac[is + 1] * met[(is + 1) * 3 + 1];
  JacKz = jac[is + 1] * met[(is + 1) * 3 + 2];
  Uk = pr[1] * JacKx + pr[2] * JacKy + pr[3] * JacKz;
  coeff = Uk * pr[0];
  fc[0] += 0.5 * coeff;
  fc[1] += 0.5 * (coeff * pr[1] + pr[4] * JacKx);
  fc[2] += 0.5 * (coeff * pr[2] + pr[4] * JacKy);
  fc[3] += 0.5 * (coeff * pr[3] + pr[4] * JacKz);
  fc[4] += 0.5 * Uk * (pr[4] + pr[nv]);
  for (int l = 5; l < nv; ++l) fc[l] += 0.5 * coeff * pr[l];

  const double dl = std::sqrt(pl[0]), dr = std::sqrt(pr[0]);
  const double inv_den = 1.0 / (dl + dr);
  const double u = (dl * pl[1] + dr * pr[1]) * inv_den;
  const double v = (dl * pl[2] + dr * pr[2]) * inv_den;
  const double w = (dl * pl[3] + dr * pr[3]) * inv_den;
  const double ek = 0.5 * (u * u + v * v + w * w);
  const double hl = (pl[nv] + pl[4]) / pl[0], hr = (pr[nv] + pr[4]) / pr[0];
  const double h = (dl * hl + dr * hr) * inv_den;
  double gamma = gamma_air;
  double c = std::sqrt((gamma - 1) * (h - ek));
  double mw = mw_air;
  double svm[MAXS + 4] = {0}, h_i[MAXS] = {0};
  for (int l = 0; l < nv - 5; ++l) svm[l] = (dl * pl[l + 5] + dr * pr[l + 5]) * inv_den;
  if (P->mix_model != OSTC_MIX_AIR) {
    double mw_inv = 0;
    for (int l = 0; l < P->n_spec; ++l) mw_inv += svm[l] / P->mw[l];
    const double tl = pl[4] / pl[0], tr = pr[4] / pr[0];
    const double t = (dl * tl + dr * tr) * inv_den / (R_u * mw_inv);
    double cp_i[MAXS];
    enthalpy_and_cp(P, t, h_i, cp_i);
    double cv = 0, cp = 0;
    for (int l = 0; l < P->n_spec; ++l) {
      cp += cp_i[l] * svm[l];
      cv += svm[l] * (cp_i[l] - R_u / P->mw[l]);
    }
    gamma = cp / cv;
    c = std::sqrt(gamma * R_u * mw_inv * t);
    mw = 1.0 / mw_inv;
  }
  double kx = 0.5 * (met[is * 3] + met[(is + 1) * 3]);
  double ky = 0.5 * (met[is * 3 + 1] + met[(is + 1) * 3 + 1]);
  double kz = 0.5 * (met[is * 3 + 2] + met[(is + 1) * 3 + 2]);
  const double gradK = std::sqrt(kx * kx + ky * ky + kz * kz);
  Uk = kx * u + ky * v + kz * w;
  double ch[3] = {Uk - gradK * c, Uk, Uk + gradK * c};
  const double dfix = 0.5 * (delta[is] + delta[is + 1]);
  for (double &cc : ch) {
    cc = std::abs(cc);
    if (cc < dfix) cc = 0.5 * (cc * cc / dfix + dfix);
  }
  kx /= gradK;
  ky /= gradK;
  kz /= gradK;
  Uk /= gradK;
  const double jac_ave = 0.5 * (jac[is] + jac[is + 1]);
  double dq[5 + MAXS + 4] = {0};
  dq[0] = jac_ave * (pr[0] - pl[0]);
  for (int l = 1; l < nv; ++l) dq[l] = jac_ave * (pr[0] * pr[l] - pl[0] * pl[l]);
  dq[4] = jac_ave * (pr[nv] - pl[nv]);
  double c1 = (gamma - 1) * (ek * dq[0] - u * dq[1] - v * dq[2] - w * dq[3] + dq[4]) / (c * c);
  double c2 = (kx * dq[1] + ky * dq[2] + kz * dq[3] - Uk * dq[0]) / c;
  for (int l = 0; l < P->n_spec; ++l) c1 += (mw / P->mw[l] - h_i[l] * (gamma - 1) / (c * c)) * dq[l + 5];
  double c3 = dq[0] - c1;
  double L[5 + MAXS + 4] = {0};
  L[0] = 0.5 * (c1 - c2);
  L[1] = kx * c3 - ((kz * v - ky * w) * dq[0] - kz * dq[2] + ky * dq[3]) / c;
  L[2] = ky * c3 - ((kx * w - kz * u) * dq[0] - kx * dq[3] + kz * dq[1]) / c;
  L[3] = kz * c3 - ((ky * u - kx * v) * dq[0] - ky * dq[1] + kx * dq[2]) / c;
  L[4] = 0.5 * (c1 + c2);
  for (int l = 0; l < P->n_scalar; ++l) L[l + 5] = dq[l + 5] - svm[l] * dq[0];
  double *b = dq;
  b[0] = -ch[0] * L[0];
  for (int l = 1; l < nv; ++l) b[l] = -ch[1] * L[l];
  b[4] = -ch[2] * L[4];
  const double c0 = kx * b[1] + ky * b[2] + kz * b[3];
  c1 = c0 + b[0] + b[4];
  c2 = c * (b[4] - b[0]);
  c3 = 0;
  for (int l = 0; l < P->n_spec; ++l) c3 += (h_i[l] - mw / P->mw[l] * c * c / (gamma - 1)) * b[l + 5];
  fc[0] += 0.5 * c1;
  fc[1] += 0.5 * (u * c1 + kx * c2 - c * (kz * b[2] - ky * b[3]));
  fc[2] += 0.5 * (v * c1 + ky * c2 - c * (kx * b[3] - kz * b[1]));
  fc[3] += 0.5 * (w * c1 + kz * c2 - c * (ky * b[1] - kx * b[2]));
  fc[4] += 0.5 * (h * c1 + Uk * c2 - c * c * c0 / (gamma - 1) +
                  c * ((kz * v - ky * w) * b[1] + (kx * w - kz * u) * b[2] + (ky * u - kx * v) * b[3]) + c3);
  for (int l = 0; l < nv - 5; ++l) fc[5 + l] += 0.5 * (b[l + 5] + svm[l] * c1);
}

void riemann(const ostc_param *P, const double *pl, const double *pr, const double *met,
             const double *jac, int is, double *fci) {  // InviscidScheme.cu:137-150
  switch (P->inviscid_scheme) {
    case 1: lax_friedrichs(P, pl, pr, met, jac, is, fci); break;
    case 4: hllc(P, pl, pr, met, jac, is, fci); break;
    default: ausm_plus(P, pl, pr, met, jac, is, fci); break;  // 3 and (quirk A1) 2
  }
}

// ---------------------------------------------------------------------------
// AWENO-5 for air: src/AWENO.cu:17-206. cvl rows hold n_var conservative
// values followed by p and T (row stride nv + 2).
// ---------------------------------------------------------------------------
void weno5_values(const double *v, double *vm, double *vp);

void weno5(const double *L, const double *cv, int stride, int is, int row, double *vm, double *vp) {
  double v[6] = {0};
  for (int i = -2; i < 4; ++i) {
    const double *U = &cv[(is + i) * stride];
    for (int j = 0; j < 5; ++j) v[i + 2] += L[row * 5 + j] * U[j];
  }
  weno5_values(v, vm, vp);
}

// the WENO5 pair (left state of face is+1/2 from points is-2..is+2, right
// state from is-1..is+3) of six point values v[0..5] = points is-2..is+3
void weno5_values(const double *v, double *vm, double *vp) {
  double v0 = 0.125 * (3 * v[0] - 10 * v[1] + 15 * v[2]);
  double v1 = 0.125 * (-v[1] + 6 * v[2] + 3 * v[3]);
  double v2 = 0.125 * (3 * v[2] + 6 * v[3] - v[4]);
  constexpr double t13 = 13.0 / 12;
  double b0 = t13 * (v[0] + v[2] - 2 * v[1]) * (v[0] + v[2] - 2 * v[1]) +
              0.25 * (v[0] + 3 * v[2] - 4 * v[1]) * (v[0] + 3 * v[2] - 4 * v[1]);
  double b1 = t13 * (v[1] + v[3] - 2 * v[2]) * (v[1] + v[3] - 2 * v[2]) + 0.25 * (v[3] - v[1]) * (v[3] - v[1]);
  double b2 = t13 * (v[2] + v[4] - 2 * v[3]) * (v[2] + v[4] - 2 * v[3]) +
              0.25 * (3 * v[2] + v[4] - 4 * v[3]) * (3 * v[2] + v[4] - 4 * v[3]);
  double tau = (b0 - b2) * (b0 - b2);
  constexpr double eps = 1e-6, d0 = 1.0 / 16, d1 = 5.0 / 8, d2 = 5.0 / 16;
  double a0 = d0 + d0 * tau / ((eps + b0) * (eps + b0));
  double a1 = d1 + d1 * tau / ((eps + b1) * (eps + b1));
  double a2 = d2 + d2 * tau / ((eps + b2) * (eps + b2));
  *vm = (a0 * v0 + a1 * v1 + a2 * v2) / (a0 + a1 + a2);
  v0 = v1;
  v1 = v2;
  v2 = 0.125 * (15 * v[3] - 10 * v[4] + 3 * v[5]);
  b0 = t13 * (v[1] + v[3] - 2 * v[2]) * (v[1] + v[3] - 2 * v[2]) +
       0.25 * (v[1] + 3 * v[3] - 4 * v[2]) * (v[1] + 3 * v[3] - 4 * v[2]);
  b1 = t13 * (v[2] + v[4] - 2 * v[3]) * (v[2] + v[4] - 2 * v[3]) + 0.25 * (v[4] - v[2]) * (v[4] - v[2]);
  b2 = t13 * (v[3] + v[5] - 2 * v[4]) * (v[3] + v[5] - 2 * v[4]) +
       0.25 * (3 * v[3] + v[5] - 4 * v[4]) * (3 * v[3] + v[5] - 4 * v[4]);
  tau = (b0 - b2) * (b0 - b2);
  a0 = d2 + d2 * tau / ((eps + b0) * (eps + b0));
  a1 = d1 + d1 * tau / ((eps + b1) * (eps + b1));
  a2 = d0 + d0 * tau / ((eps + b2) * (eps + b2));
  *vp = (a0 * v0 + a1 * v1 + a2 * v2) / (a0 + a1 + a2);
}

void aweno_interpolation(const ostc_param *P, const double *cv, double *pl, double *pr, int is,
                         const double *met) {
  const int nv = P->n_var;
  const int st = nv + 2;
  const double *cl = &cv[is * st], *cr = &cv[(is + 1) * st];
  const double rlc = std::sqrt(cl[0]) / (std::sqrt(cl[0]) + std::sqrt(cr[0]));
  const double rrc = std::sqrt(cr[0]) / (std::sqrt(cl[0]) + std::sqrt(cr[0]));
  const double um = rlc * cl[1] / cl[0] + rrc * cr[1] / cr[0];
  const double vm = rlc * cl[2] / cl[0] + rrc * cr[2] / cr[0];
  const double wm = rlc * cl[3] / cl[0] + rrc * cr[3] / cr[0];
  const double ekm = 0.5 * (um * um + vm * vm + wm * wm);
  constexpr double gm1 = gamma_air - 1;
  const double hl = (cl[4] + cl[nv]) / cl[0];
  const double hr = (cr[4] + cr[nv]) / cr[0];
  const double hm = rlc * hl + rrc * hr;
  const double cm2 = gm1 * (hm - ekm);
  const double cm = std::sqrt(cm2);
  double kx = 0.5 * (met[is * 3] + met[(is + 1) * 3]);
  double ky = 0.5 * (met[is * 3 + 1] + met[(is + 1) * 3 + 1]);
  double kz = 0.5 * (met[is * 3 + 2] + met[(is + 1) * 3 + 2]);
  const double gK = std::sqrt(kx * kx + ky * ky + kz * kz);
  kx /= gK;
  ky /= gK;
  kz /= gK;
  const double Uk = kx * um + ky * vm + kz * wm;
  const double alpha = gm1 * ekm;
  double L[25];
  L[0] = (alpha + Uk * cm) / cm2 * 0.5;
  L[1] = -(gm1 * um + kx * cm) / cm2 * 0.5;
  L[2] = -(gm1 * vm + ky * cm) / cm2 * 0.5;
  L[3] = -(gm1 * wm + kz * cm) / cm2 * 0.5;
  L[4] = gm1 / cm2 * 0.5;
  L[5] = kx * (1 - alpha / cm2) - (kz * vm - ky * wm) / cm;
  L[6] = kx * gm1 * um / cm2;
  L[7] = (kx * gm1 * vm + kz * cm) / cm2;
  L[8] = (kx * gm1 * wm - ky * cm) / cm2;
  L[9] = -kx * gm1 / cm2;
  L[10] = ky * (1 - alpha / cm2) - (kx * wm - kz * um) / cm;
  L[11] = (ky * gm1 * um - kz * cm) / cm2;
  L[12] = ky * gm1 * vm / cm2;
  L[13] = (ky * gm1 * wm + kx * cm) / cm2;
  L[14] = -ky * gm1 / cm2;
  L[15] = kz * (1 - alpha / cm2) - (ky * um - kx * vm) / cm;
  L[16] = (kz * gm1 * um + ky * cm) / cm2;
  L[17] = (kz * gm1 * vm - kx * cm) / cm2;
  L[18] = kz * gm1 * wm / cm2;
  L[19] = -kz * gm1 / cm2;
  L[20] = (alpha - Uk * cm) / cm2 * 0.5;
  L[21] = -(gm1 * um - kx * cm) / cm2 * 0.5;
  L[22] = -(gm1 * vm - ky * cm) / cm2 * 0.5;
  L[23] = -(gm1 * wm - kz * cm) / cm2 * 0.5;
  L[24] = gm1 / cm2 * 0.5;
  double vplus[5] = {0}, vminus[5] = {0};
  if (P->reconstruction == 4) {
    // the reference passes n_var = 5 to WENO5 and so reads rows of stride 7
    // (quirk A3), which is the true stride n_var + 2 without turbulence scalars
    for (int l = 0; l < 5; ++l) weno5(L, cv, st, is, l, &vminus[l], &vplus[l]);
  }
  double R[25];
  R[0] = 1.0; R[1] = kx; R[2] = ky; R[3] = kz; R[4] = 1.0;
  R[5] = um - kx * cm; R[6] = kx * um; R[7] = ky * um - kz * cm; R[8] = kz * um + ky * cm; R[9] = um + kx * cm;
  R[10] = vm - ky * cm; R[11] = kx * vm + kz * cm; R[12] = ky * vm; R[13] = kz * vm - kx * cm; R[14] = vm + ky * cm;
  R[15] = wm - kz * cm; R[16] = kx * wm - ky * cm; R[17] = ky * wm + kx * cm; R[18] = kz * wm; R[19] = wm + kz * cm;
  R[20] = hm - Uk * cm;
  R[21] = kx * alpha / gm1 + (kz * vm - ky * wm) * cm;
  R[22] = ky * alpha / gm1 + (kx * wm - kz * um) * cm;
  R[23] = kz * alpha / gm1 + (ky * um - kx * vm) * cm;
  R[24] = hm + Uk * cm;
  double ql[5], qr[5];
  for (int m = 0; m < 5; ++m) {
    ql[m] = 0;
    qr[m] = 0;
    for (int n = 0; n < 5; ++n) {
      ql[m] += R[m * 5 + n] * vminus[n];
      qr[m] += R[m * 5 + n] * vplus[n];
    }
  }
  pl[0] = ql[0];
  pl[1] = ql[1] / ql[0];
  pl[2] = ql[2] / ql[0];
  pl[3] = ql[3] / ql[0];
  pl[4] = gm1 * (ql[4] - 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]) * ql[0]);
  pl[nv] = ql[4];
  pr[0] = qr[0];
  pr[1] = qr[1] / qr[0];
  pr[2] = qr[2] / qr[0];
  pr[3] = qr[3] / qr[0];
  pr[4] = gm1 * (qr[4] - 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]) * qr[0]);
  pr[nv] = qr[4];
  // SST scalars (not in the reference's AWENO, quirk A3): component-wise WENO5
  // of rho k, rho omega, divided by the reconstructed densities
  for (int l = 5; l < nv; ++l) {
    double v[6], sm = 0, sp = 0;
    for (int i = -2; i < 4; ++i) v[i + 2] = cv[(is + i) * st + l];
    if (P->reconstruction == 4) weno5_values(v, &sm, &sp);
    pl[l] = sm / ql[0];
    pr[l] = sp / qr[0];
  }
}

// optional per-variable max |face flux| (conditioning scale of dq), see oracle_flux_scale
double *g_flux_scale = nullptr;
inline void note_scale(const double *F, int nv) {
  if (!g_flux_scale) return;
  for (int l = 0; l < nv; ++l) {
    const double a = std::abs(F[l]);
#pragma omp critical(flux_scale)
    if (a > g_flux_scale[l]) g_flux_scale[l] = a;
  }
}

// index helpers for "direction d, position s along the line, (a,b) the other two"
inline void line_ijk(int d, int s, int a, int b, int &i, int &j, int &k) {
  if (d == 0) { i = s; j = a; k = b; }
  else if (d == 1) { i = a; j = s; k = b; }
  else { i = a; j = b; k = s; }
}

// ---------------------------------------------------------------------------
// inviscid terms: compute_convective_term_pv_1D (InviscidScheme.cu:48-158),
// compute_convective_term_aweno_1D (InviscidScheme.cu:207-311) and
// CDSPart1D<Air> (AWENO.cu:213-264). One call processes one direction.
// ---------------------------------------------------------------------------
void inviscid_direction(const ostc_param *P, Z &Zn, int d) {
  const int ext[3] = {Zn.mx, Zn.my, Zn.mz};
  const int n = ext[d], ngg = Zn.ngg;
  const int oa = d == 0 ? 1 : 0, ob = d == 2 ? 1 : 2;
  const int na = ext[oa], nb = ext[ob];
  const int nv = P->n_var;
  const bool aweno = P->inviscid_type == 1;
  const bool roe = P->inviscid_type == 2;
  const int nrow = aweno ? nv + 2 : nv;
  const int npt = n + 2 * ngg;  // line points -ngg .. n+ngg-1 at index s+ngg
#pragma omp parallel
  {
    std::vector<double> rows(npt * nrow), met(npt * 3), jac(npt), fc((n + 1) * nv), f(npt * nv), delta(npt);
    double pl[MAXS + 11], pr[MAXS + 11];
#pragma omp for collapse(2) schedule(static)
    for (int b = 0; b < nb; ++b) {
      for (int a = 0; a < na; ++a) {
        for (int s = -ngg; s < n + ngg; ++s) {
          int i, j, k;
          line_ijk(d, s, a, b, i, j, k);
          const int is = s + ngg;
          if (aweno) {
            for (int l = 0; l < nv; ++l) rows[is * nrow + l] = Zn.cv(i, j, k, l);
            rows[is * nrow + nv] = Zn.bv(i, j, k, 4);
            rows[is * nrow + nv + 1] = Zn.bv(i, j, k, 5);
          } else {
            for (int l = 0; l < 5; ++l) rows[is * nrow + l] = Zn.bv(i, j, k, l);
            for (int l = 0; l < P->n_scalar; ++l) rows[is * nrow + 5 + l] = Zn.sv(i, j, k, l);
          }
          const double *m = Zn.metric.at(i, j, k);
          for (int c = 0; c < 3; ++c) met[is * 3 + c] = m[3 * d + c];
          jac[is] = Zn.jac(i, j, k);
          if (roe && s >= -1 && s <= n) {  // compute_entropy_fix_delta on [-1, m] (Roe.cu:61-85)
            const double u = Zn.bv(i, j, k, 1), v = Zn.bv(i, j, k, 2), w = Zn.bv(i, j, k, 3);
            const double U = std::abs(u * m[0] + v * m[1] + w * m[2]);
            const double V = std::abs(u * m[3] + v * m[4] + w * m[5]);
            const double W = std::abs(u * m[6] + v * m[7] + w * m[8]);
            const double kx = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
            const double ky = std::sqrt(m[3] * m[3] + m[4] * m[4] + m[5] * m[5]);
            const double kz = std::sqrt(m[6] * m[6] + m[7] * m[7] + m[8] * m[8]);
            if (Zn.mz == 1)  // param->dim == 2 (Roe.cu:79-81)
              delta[is] = P->entropy_fix_factor * (U + V + Zn.a(i, j, k) * 0.5 * (kx + ky));
            else
              delta[is] = P->entropy_fix_factor * (U + V + W + Zn.a(i, j, k) * (kx + ky + kz) / 3.0);
          }
        }
        // face fluxes for s = -1 .. n-1 (face between s and s+1), stored at s+1
        for (int s = -1; s < n; ++s) {
          const int is = s + ngg;
          if (aweno)
            aweno_interpolation(P, rows.data(), pl, pr, is, met.data());
          else
            reconstruct(P, rows.data(), pl, pr, is, nv);
          if (roe)
            roe_flux(P, pl, pr, met.data(), jac.data(), delta.data(), is, &fc[(s + 1) * nv]);
          else
            riemann(P, pl, pr, met.data(), jac.data(), is, &fc[(s + 1) * nv]);
          note_scale(&fc[(s + 1) * nv], nv);
        }
        for (int s = 0; s < n; ++s) {
          int i, j, k;
          line_ijk(d, s, a, b, i, j, k);
          for (int l = 0; l < nv; ++l) Zn.dq(i, j, k, l) -= fc[(s + 1) * nv + l] - fc[s * nv + l];
        }
        if (aweno) {
          // physical fluxes for s in [-ngg, n - ngg) (AWENO.cu:228-249)
          for (int s = -ngg; s < n - ngg; ++s) {
            int i, j, k;
            line_ijk(d, s, a, b, i, j, k);
            const double *m = Zn.metric.at(i, j, k);
            const double kx = m[3 * d], ky = m[3 * d + 1], kz = m[3 * d + 2];
            const double jc = Zn.jac(i, j, k);
            const double u = Zn.bv(i, j, k, 1), v = Zn.bv(i, j, k, 2), w = Zn.bv(i, j, k, 3);
            const double Uk = kx * u + ky * v + kz * w;
            const double rUk = Zn.bv(i, j, k, 0) * Uk;
            const double p = Zn.bv(i, j, k, 4);
            double *fi = &f[(s + ngg) * nv];
            fi[0] = rUk * jc;
            fi[1] = jc * (rUk * u + kx * p);
            fi[2] = jc * (rUk * v + ky * p);
            fi[3] = jc * (rUk * w + kz * p);
            fi[4] = jc * Uk * (Zn.cv(i, j, k, 4) + p);
            for (int l = 5; l < nv; ++l) fi[l] = jc * (rUk * Zn.sv(i, j, k, l - 5));  // SST scalars
          }
          // central correction only on [0, n - 2 ngg) (quirk A4)
          constexpr double c1 = 19.0 / 3840, c2 = -13.0 / 320, c3 = 17.0 / 256;
          for (int s = 0; s < n - 2 * ngg; ++s) {
            int i, j, k;
            line_ijk(d, s, a, b, i, j, k);
            const int is = s + ngg;
            for (int l = 0; l < nv; ++l) {
              Zn.dq(i, j, k, l) -= c1 * (f[(is + 3) * nv + l] - f[(is - 3) * nv + l]) +
                                   c2 * (f[(is + 2) * nv + l] - f[(is - 2) * nv + l]) +
                                   c3 * (f[(is + 1) * nv + l] - f[(is - 1) * nv + l]);
            }
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// viscous face flux, laminar: compute_{fv,gv,hv}_2nd_order (ViscousScheme.cuh:22-821)
// for the face between p0 = (i,j,k) and p1 = p0 + e_d.
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// k-omega SST, air (SST.cu:8-247, SST.cuh:12-45)
// ---------------------------------------------------------------------------
inline bool is_sst(const ostc_param *P) { return P->turbulence && P->rans_model == 2; }

namespace sst {
constexpr double beta_star = 0.09, sqrt_beta_star = 0.3, kappa = 0.41;
constexpr double sigma_k1 = 0.85, sigma_omega1 = 0.5, beta_1 = 0.0750, a_1 = 0.31;
constexpr double gamma1 = beta_1 / beta_star - sigma_omega1 * kappa * kappa / sqrt_beta_star;
constexpr double sigma_k2 = 1, sigma_omega2 = 0.856, beta_2 = 0.0828;
constexpr double gamma2 = beta_2 / beta_star - sigma_omega2 * kappa * kappa / sqrt_beta_star;
constexpr double delta_sigma_k = sigma_k1 - sigma_k2, delta_sigma_omega = sigma_omega1 - sigma_omega2;
constexpr double delta_beta = beta_1 - beta_2, delta_gamma = gamma1 - gamma2;

// 0.5 * (xi_c (V(i+1)-V(i-1)) + eta_c (V(j+1)-V(j-1)) + zeta_c (V(k+1)-V(k-1))), SST.cu:52-69
double grad(const Z &Zn, const View &V, int l, const double *m, int c, int i, int j, int k) {
  return 0.5 * (m[c] * (V(i + 1, j, k, l) - V(i - 1, j, k, l)) + m[3 + c] * (V(i, j + 1, k, l) - V(i, j - 1, k, l)) +
                m[6 + c] * (V(i, j, k + 1, l) - V(i, j, k - 1, l)));
}

// it: the plane of k in sv (n_spec; omega follows)
double compute_mut(const Z &Zn, int it, int i, int j, int k, double mul) {  // SST.cu:44-97
  const double *m = Zn.metric.at(i, j, k);
  const double u_y = grad(Zn, Zn.bv, 1, m, 1, i, j, k), u_z = grad(Zn, Zn.bv, 1, m, 2, i, j, k);
  const double v_x = grad(Zn, Zn.bv, 2, m, 0, i, j, k), v_z = grad(Zn, Zn.bv, 2, m, 2, i, j, k);
  const double w_x = grad(Zn, Zn.bv, 3, m, 0, i, j, k), w_y = grad(Zn, Zn.bv, 3, m, 1, i, j, k);
  const double density = Zn.bv(i, j, k, 0), tke = Zn.sv(i, j, k, it), omega = Zn.sv(i, j, k, it + 1);
  const double rhoK = density * tke;
  const double vorticity =
      std::sqrt((v_x - u_y) * (v_x - u_y) + (w_x - u_z) * (w_x - u_z) + (w_y - v_z) * (w_y - v_z));
  double f2 = 1;
  const double dy = Zn.wall(i, j, k);
  if (dy > 1e-25) {
    const double param1 = 2 * std::sqrt(tke) / (0.09 * omega * dy);
    const double param2 = 500 * mul / (density * dy * dy * omega);
    const double arg2 = std::max(param1, param2);
    f2 = std::tanh(arg2 * arg2);
  }
  double mut = 0;
  const double denominator = std::max(a_1 * omega, vorticity * f2);
  if (denominator > 1e-25) mut = a_1 * rhoK / denominator;
  return mut;
}

double wilcox(double Mt) {  // SST.cu:24-31
  constexpr double Mt0 = 0.25;
  return Mt - Mt0 > 0 ? beta_star * 2 * (Mt * Mt - Mt0 * Mt0) : 0.0;
}
double zeman(double Mt, double gammaP1) {  // SST.cu:33-42
  const double Mt0 = 0.25 * std::sqrt(2.0 / gammaP1);
  const double DMt = Mt - Mt0;
  if (DMt > 0) {
    constexpr double Lambda2 = 0.66 * 0.66;
    return beta_star * 0.75 * (1 - std::exp(-0.5 * gammaP1 * DMt * DMt / Lambda2));
  }
  return 0.0;
}

// compute_source_and_mut (SST.cu:99-247) + the turbulent conductivity (SourceTerm.cuh:19-27)
void source_and_mut(const ostc_param *P, Z &Zn, int i, int j, int k) {
  const int it = P->n_spec;  // k, omega planes it, it + 1; dq rows 5 + it, 6 + it (i_turb_cv)
  const double *m = Zn.metric.at(i, j, k);
  const View &bv = Zn.bv, &sv = Zn.sv;
  const double u_x = grad(Zn, bv, 1, m, 0, i, j, k), u_y = grad(Zn, bv, 1, m, 1, i, j, k);
  const double u_z = grad(Zn, bv, 1, m, 2, i, j, k);
  const double v_x = grad(Zn, bv, 2, m, 0, i, j, k), v_y = grad(Zn, bv, 2, m, 1, i, j, k);
  const double v_z = grad(Zn, bv, 2, m, 2, i, j, k);
  const double w_x = grad(Zn, bv, 3, m, 0, i, j, k), w_y = grad(Zn, bv, 3, m, 1, i, j, k);
  const double w_z = grad(Zn, bv, 3, m, 2, i, j, k);
  const double density = bv(i, j, k, 0);
  const double omega = sv(i, j, k, it + 1);
  const double k_x = grad(Zn, sv, it, m, 0, i, j, k), k_y = grad(Zn, sv, it, m, 1, i, j, k);
  const double k_z = grad(Zn, sv, it, m, 2, i, j, k);
  const double omega_x = grad(Zn, sv, it + 1, m, 0, i, j, k), omega_y = grad(Zn, sv, it + 1, m, 1, i, j, k);
  const double omega_z = grad(Zn, sv, it + 1, m, 2, i, j, k);
  const double inter_var = 2 * density * sigma_omega2 / omega * (k_x * omega_x + k_y * omega_y + k_z * omega_z);
  const double tke = sv(i, j, k, it);
  const double rhoK = density * tke;
  const double vorticity =
      std::sqrt((v_x - u_y) * (v_x - u_y) + (w_x - u_z) * (w_x - u_z) + (w_y - v_z) * (w_y - v_z));
  double f1 = 1, f2 = 1;
  const double dy = Zn.wall(i, j, k);
  if (dy > 1e-25) {
    const double param1 = std::sqrt(tke) / (0.09 * omega * dy);
    const double d2 = dy * dy;
    const double param2 = 500 * Zn.mul(i, j, k) / (density * d2 * omega);
    const double arg2 = std::max(2 * param1, param2);
    f2 = std::tanh(arg2 * arg2);
    const double CDkomega = std::max(1e-20, inter_var);
    const double param3 = 4 * density * sigma_omega2 * tke / (CDkomega * d2);
    const double arg1 = std::min(std::max(param1, param2), param3);
    f1 = std::tanh(arg1 * arg1 * arg1 * arg1);
  }
  double mut = 0;
  const double denominator = std::max(a_1 * omega, vorticity * f2);
  if (denominator > 1e-25) mut = a_1 * rhoK / denominator;
  Zn.mut(i, j, k) = mut;
  double beta = beta_2 + delta_beta * f1;
  double betaStar = beta_star;
  if (const int correction = P->compressibility_correction) {
    const double gam = it > 0 ? Zn.gam(i, j, k) : gamma_air;  // SST.cu:195-199
    const double Mt = std::sqrt(2 * tke / (gam * bv(i, j, k, 4) / density));
    double c;
    switch (correction) {
      case 1: c = wilcox(Mt); break;
      case 2: c = beta_star * Mt * Mt; break;
      default: c = zeman(Mt, gam + 1.0); break;
    }
    betaStar += c;
    beta -= c;
  }
  if (mut > 1e-25) {
    const double divU = u_x + v_y + w_z;
    const double divU2 = divU * divU;
    double prod_k = mut * (2 * (u_x * u_x + v_y * v_y + w_z * w_z) - 2.0 / 3 * divU2 + (u_y + v_x) * (u_y + v_x) +
                           (u_z + w_x) * (u_z + w_x) + (v_z + w_y) * (v_z + w_y)) -
                    2.0 / 3 * rhoK * divU;
    const double prod_k2 = mut * vorticity * vorticity;
    if (prod_k > 10 * prod_k2) prod_k = prod_k2;
    const double diss_k = betaStar * rhoK * omega;
    const double jac = Zn.jac(i, j, k);
    Zn.dq(i, j, k, 5 + it) += jac * (prod_k - diss_k);
    const double gamma = gamma2 + delta_gamma * f1;
    const double prod_omega = gamma * density / mut * prod_k + (1 - f1) * inter_var;
    const double diss_omega = beta * density * omega * omega;
    Zn.dq(i, j, k, 6 + it) += jac * (prod_omega - diss_omega);
  }
  if (P->turb_implicit == 1 && Zn.tsj.p) {  // SST.cu:243-246
    Zn.tsj(i, j, k, 0) = -2 * betaStar * omega;
    Zn.tsj(i, j, k, 1) = -2 * beta * omega;
  }
  constexpr double cpa = gamma_air * R_u / mw_air / (gamma_air - 1);
  Zn.ttc(i, j, k) = Zn.mut(i, j, k) * (it > 0 ? Zn.cp(i, j, k) : cpa) / P->Prt;
}
}  // namespace sst

void viscous_face(const ostc_param *P, const Z &Zn, int d, int i, int j, int k, double *fv) {
  const int e[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  const int i1 = i + e[d][0], j1 = j + e[d][1], k1 = k + e[d][2];
  const double *m = Zn.metric.at(i, j, k), *m1 = Zn.metric.at(i1, j1, k1);
  double mm[9];
  for (int c = 0; c < 9; ++c) mm[c] = 0.5 * (m[c] + m1[c]);
  const double xi_x = mm[0], xi_y = mm[1], xi_z = mm[2];
  const double eta_x = mm[3], eta_y = mm[4], eta_z = mm[5];
  const double zeta_x = mm[6], zeta_y = mm[7], zeta_z = mm[8];
  // derivative of a field along the three computational directions at the face
  auto der = [&](const View &V, int l, double out[3]) {
    for (int c = 0; c < 3; ++c) {
      if (c == d) {
        out[c] = V(i1, j1, k1, l) - V(i, j, k, l);
      } else {
        const int di = e[c][0], dj = e[c][1], dk = e[c][2];
        out[c] = 0.25 * (V(i + di, j + dj, k + dk, l) - V(i - di, j - dj, k - dk, l) +
                         V(i1 + di, j1 + dj, k1 + dk, l) - V(i1 - di, j1 - dj, k1 - dk, l));
      }
    }
  };
  double du[3], dv[3], dw[3], dt[3];
  der(Zn.bv, 1, du);
  der(Zn.bv, 2, dv);
  der(Zn.bv, 3, dw);
  der(Zn.bv, 5, dt);
  const double u_x = du[0] * xi_x + du[1] * eta_x + du[2] * zeta_x;
  const double u_y = du[0] * xi_y + du[1] * eta_y + du[2] * zeta_y;
  const double u_z = du[0] * xi_z + du[1] * eta_z + du[2] * zeta_z;
  const double v_x = dv[0] * xi_x + dv[1] * eta_x + dv[2] * zeta_x;
  const double v_y = dv[0] * xi_y + dv[1] * eta_y + dv[2] * zeta_y;
  const double v_z = dv[0] * xi_z + dv[1] * eta_z + dv[2] * zeta_z;
  const double w_x = dw[0] * xi_x + dw[1] * eta_x + dw[2] * zeta_x;
  const double w_y = dw[0] * xi_y + dw[1] * eta_y + dw[2] * zeta_y;
  const double w_z = dw[0] * xi_z + dw[1] * eta_z + dw[2] * zeta_z;
  const double mul = 0.5 * (Zn.mul(i, j, k) + Zn.mul(i1, j1, k1));
  const bool turb = is_sst(P);
  const double mut = turb ? 0.5 * (Zn.mut(i, j, k) + Zn.mut(i1, j1, k1)) : 0.0;
  const double viscosity = mul + mut;
  double tau_xx = viscosity * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
  double tau_yy = viscosity * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
  double tau_zz = viscosity * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
  if (turb) {  // ViscousScheme.cuh:82-95
    constexpr double delta_d = 1e-3;
    const double dy_div_delta = std::min(0.5 * (Zn.wall(i, j, k) + Zn.wall(i1, j1, k1)) / delta_d, 1.0);
    const double twoThirdrhoKm =
        -2.0 / 3 * 0.5 *
        (Zn.bv(i, j, k, 0) * Zn.sv(i, j, k, P->n_spec) + Zn.bv(i1, j1, k1, 0) * Zn.sv(i1, j1, k1, P->n_spec)) *
        dy_div_delta;
    tau_xx += twoThirdrhoKm;
    tau_yy += twoThirdrhoKm;
    tau_zz += twoThirdrhoKm;
  }
  const double tau_xy = viscosity * (u_y + v_x);
  const double tau_xz = viscosity * (u_z + w_x);
  const double tau_yz = viscosity * (v_z + w_y);
  const double kxj = 0.5 * (m[3 * d] * Zn.jac(i, j, k) + m1[3 * d] * Zn.jac(i1, j1, k1));
  const double kyj = 0.5 * (m[3 * d + 1] * Zn.jac(i, j, k) + m1[3 * d + 1] * Zn.jac(i1, j1, k1));
  const double kzj = 0.5 * (m[3 * d + 2] * Zn.jac(i, j, k) + m1[3 * d + 2] * Zn.jac(i1, j1, k1));
  fv[0] = 0;
  fv[1] = kxj * tau_xx + kyj * tau_xy + kzj * tau_xz;
  fv[2] = kxj * tau_xy + kyj * tau_yy + kzj * tau_yz;
  fv[3] = kxj * tau_xz + kyj * tau_yz + kzj * tau_zz;
  const double um = 0.5 * (Zn.bv(i, j, k, 1) + Zn.bv(i1, j1, k1, 1));
  const double vm = 0.5 * (Zn.bv(i, j, k, 2) + Zn.bv(i1, j1, k1, 2));
  const double wm = 0.5 * (Zn.bv(i, j, k, 3) + Zn.bv(i1, j1, k1, 3));
  const double t_x = dt[0] * xi_x + dt[1] * eta_x + dt[2] * zeta_x;
  const double t_y = dt[0] * xi_y + dt[1] * eta_y + dt[2] * zeta_y;
  const double t_z = dt[0] * xi_z + dt[1] * eta_z + dt[2] * zeta_z;
  double cond = 0.5 * (Zn.kappa(i, j, k) + Zn.kappa(i1, j1, k1));
  if (turb) cond += 0.5 * (Zn.ttc(i, j, k) + Zn.ttc(i1, j1, k1));
  fv[4] = um * fv[1] + vm * fv[2] + wm * fv[3] + cond * (kxj * t_x + kyj * t_y + kzj * t_z);
  if (P->mix_model != OSTC_MIX_AIR) {
    const int ns = P->n_spec;
    double diff[MAXS], yk[MAXS], ddf[MAXS];
    double sum_gy_w = 0, sum_rDY = 0, corr = 0, mw_tot = 0;
    for (int l = 0; l < ns; ++l) {
      yk[l] = 0.5 * (Zn.sv(i, j, k, l) + Zn.sv(i1, j1, k1, l));
      diff[l] = 0.5 * (Zn.rhoD(i, j, k, l) + Zn.rhoD(i1, j1, k1, l));
      if (turb) diff[l] += mut / P->Sct;  // turbulent diffusivity (ViscousScheme.cuh:122-125)
      double dy[3];
      der(Zn.sv, l, dy);
      const double y_x = dy[0] * xi_x + dy[1] * eta_x + dy[2] * zeta_x;
      const double y_y = dy[0] * xi_y + dy[1] * eta_y + dy[2] * zeta_y;
      const double y_z = dy[0] * xi_z + dy[1] * eta_z + dy[2] * zeta_z;
      const double g = kxj * y_x + kyj * y_y + kzj * y_z;
      ddf[l] = g;
      corr += diff[l] * g;
      sum_gy_w += g / P->mw[l];
      mw_tot += yk[l] / P->mw[l];
      sum_rDY += diff[l] * yk[l];
    }
    mw_tot = 1.0 / mw_tot;
    corr -= mw_tot * sum_rDY * sum_gy_w;
    if (P->gradPInDiffusionFlux) {
      double dp[3];
      der(Zn.bv, 4, dp);
      const double p_x = dp[0] * xi_x + dp[1] * eta_x + dp[2] * zeta_x;
      const double p_y = dp[0] * xi_y + dp[1] * eta_y + dp[2] * zeta_y;
      const double p_z = dp[0] * xi_z + dp[1] * eta_z + dp[2] * zeta_z;
      const double gp = (kxj * p_x + kyj * p_y + kzj * p_z) / (0.5 * (Zn.bv(i1, j1, k1, 4) + Zn.bv(i, j, k, 4)));
      for (int l = 0; l < ns; ++l) {
        ddf[l] += (mw_tot / P->mw[l] - 1) * yk[l] * gp;
        corr += (mw_tot / P->mw[l] - 1) * yk[l] * gp * diff[l];
      }
    }
    double h[MAXS];
    const double tm = 0.5 * (Zn.bv(i, j, k, 5) + Zn.bv(i1, j1, k1, 5));
    enthalpy(P, tm, h);
    for (int l = 0; l < ns; ++l) {
      const double flux = diff[l] * (ddf[l] - mw_tot * yk[l] * sum_gy_w) - yk[l] * corr;
      fv[5 + l] = flux;
      fv[4] += h[l] * flux;
    }
  }
  if (turb) {  // k and omega diffusion, ViscousScheme.cuh:200-251
    const int it = P->n_spec;
    double dk[3], dw[3];
    der(Zn.sv, it, dk);
    der(Zn.sv, it + 1, dw);
    const double k_x = dk[0] * xi_x + dk[1] * eta_x + dk[2] * zeta_x;
    const double k_y = dk[0] * xi_y + dk[1] * eta_y + dk[2] * zeta_y;
    const double k_z = dk[0] * xi_z + dk[1] * eta_z + dk[2] * zeta_z;
    const double omega_x = dw[0] * xi_x + dw[1] * eta_x + dw[2] * zeta_x;
    const double omega_y = dw[0] * xi_y + dw[1] * eta_y + dw[2] * zeta_y;
    const double omega_z = dw[0] * xi_z + dw[1] * eta_z + dw[2] * zeta_z;
    const double wall_dist = 0.5 * (Zn.wall(i, j, k) + Zn.wall(i1, j1, k1));
    double f1 = 1;
    if (wall_dist > 1e-25) {
      const double km = 0.5 * (Zn.sv(i, j, k, it) + Zn.sv(i1, j1, k1, it));
      const double omegam = 0.5 * (Zn.sv(i, j, k, it + 1) + Zn.sv(i1, j1, k1, it + 1));
      const double param1 = std::sqrt(km) / (0.09 * omegam * wall_dist);
      const double rhom = 0.5 * (Zn.bv(i, j, k, 0) + Zn.bv(i1, j1, k1, 0));
      const double d2 = wall_dist * wall_dist;
      const double param2 = 500 * mul / (rhom * d2 * omegam);
      const double CDkomega =
          std::max(1e-20, 2 * rhom * sst::sigma_omega2 / omegam * (k_x * omega_x + k_y * omega_y + k_z * omega_z));
      const double param3 = 4 * rhom * sst::sigma_omega2 * km / (CDkomega * d2);
      const double arg1 = std::min(std::max(param1, param2), param3);
      f1 = std::tanh(arg1 * arg1 * arg1 * arg1);
    }
    const double sigma_k = sst::sigma_k2 + sst::delta_sigma_k * f1;
    const double sigma_omega = sst::sigma_omega2 + sst::delta_sigma_omega * f1;
    fv[5 + it] = (mul + mut * sigma_k) * (kxj * k_x + kyj * k_y + kzj * k_z);
    fv[6 + it] = (mul + mut * sigma_omega) * (kxj * omega_x + kyj * omega_y + kzj * omega_z);
  }
}

void viscous_direction(const ostc_param *P, Z &Zn, int d) {  // SchemeSelector.cuh:71-157
  const int ext[3] = {Zn.mx, Zn.my, Zn.mz};
  const int n = ext[d];
  const int oa = d == 0 ? 1 : 0, ob = d == 2 ? 1 : 2;
  const int na = ext[oa], nb = ext[ob];
  const int nv = P->n_var;
#pragma omp parallel
  {
    std::vector<double> fv((n + 1) * nv);
#pragma omp for collapse(2) schedule(static)
    for (int b = 0; b < nb; ++b) {
      for (int a = 0; a < na; ++a) {
        for (int s = -1; s < n; ++s) {
          int i, j, k;
          line_ijk(d, s, a, b, i, j, k);
          viscous_face(P, Zn, d, i, j, k, &fv[(s + 1) * nv]);
          note_scale(&fv[(s + 1) * nv], nv);
        }
        for (int s = 0; s < n; ++s) {
          int i, j, k;
          line_ijk(d, s, a, b, i, j, k);
          for (int l = 0; l < nv; ++l) Zn.dq(i, j, k, l) += fv[(s + 1) * nv + l] - fv[s * nv + l];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// field operations: src/FieldOperation.cuh:18-146, src/FieldOperation.cu:3-39
// ---------------------------------------------------------------------------
void total_energy(const ostc_param *P, Z &Zn, int i, int j, int k) {  // FieldOperation.cuh:18-41
  const double V2 = Zn.bv(i, j, k, 1) * Zn.bv(i, j, k, 1) + Zn.bv(i, j, k, 2) * Zn.bv(i, j, k, 2) +
                    Zn.bv(i, j, k, 3) * Zn.bv(i, j, k, 3);
  double E = 0.5 * V2;
  if (P->mix_model != OSTC_MIX_AIR) {
    double h[MAXS];
    enthalpy(P, Zn.bv(i, j, k, 5), h);
    for (int l = 0; l < P->n_spec; ++l) E += h[l] * Zn.sv(i, j, k, l);
    E *= Zn.bv(i, j, k, 0);
    E -= Zn.bv(i, j, k, 4);
  } else {
    E *= Zn.bv(i, j, k, 0);
    E += Zn.bv(i, j, k, 4) / (gamma_air - 1);
  }
  Zn.cv(i, j, k, 4) = E;
  Zn.vel(i, j, k) = std::sqrt(V2);
}

void cv_from_bv_point(const ostc_param *P, Z &Zn, int i, int j, int k) {  // FieldOperation.cuh:81-110
  const double rho = Zn.bv(i, j, k, 0);
  Zn.cv(i, j, k, 0) = rho;
  Zn.cv(i, j, k, 1) = rho * Zn.bv(i, j, k, 1);
  Zn.cv(i, j, k, 2) = rho * Zn.bv(i, j, k, 2);
  Zn.cv(i, j, k, 3) = rho * Zn.bv(i, j, k, 3);
  for (int l = 0; l < P->n_scalar; ++l) Zn.cv(i, j, k, 5 + l) = rho * Zn.sv(i, j, k, l);
  total_energy(P, Zn, i, j, k);
}

void temperature_and_pressure(const ostc_param *P, Z &Zn, int i, int j, int k, double E) {
  const int ns = P->n_spec;
  double mw = 0;
  for (int l = 0; l < ns; ++l) mw += Zn.sv(i, j, k, l) / P->mw[l];
  mw = 1 / mw;
  const double R = R_u / mw;
  const double e = E / Zn.bv(i, j, k, 0) -
                   0.5 * (Zn.bv(i, j, k, 1) * Zn.bv(i, j, k, 1) + Zn.bv(i, j, k, 2) * Zn.bv(i, j, k, 2) +
                          Zn.bv(i, j, k, 3) * Zn.bv(i, j, k, 3));
  double err = 1, t = Zn.bv(i, j, k, 5);
  int iter = 0;
  double h_i[MAXS], cp_i[MAXS];
  while (err > 1e-3 && iter++ < 1000) {
    enthalpy_and_cp(P, t, h_i, cp_i);
    double cpt = 0, h = 0;
    for (int l = 0; l < ns; ++l) {
      cpt += cp_i[l] * Zn.sv(i, j, k, l);
      h += h_i[l] * Zn.sv(i, j, k, l);
    }
    const double et = h - R * t;
    const double cvv = cpt - R;
    const double t1 = t - (et - e) / cvv;
    err = std::abs(1 - t1 / t);
    t = t1;
  }
  Zn.bv(i, j, k, 5) = t;
  Zn.bv(i, j, k, 4) = Zn.bv(i, j, k, 0) * t * R;
}

void properties_point(const ostc_param *P, Z &Zn, int i, int j, int k) {  // FieldOperation.cuh:112-146
  const double T = Zn.bv(i, j, k, 5);
  if (P->mix_model != OSTC_MIX_AIR) {
    const int ns = P->n_spec;
    double mw = 0, cpt = 0, cvv = 0, cp[MAXS], Y[MAXS], rD[MAXS];
    cp_only(P, T, cp);
    for (int l = 0; l < ns; ++l) {
      Y[l] = Zn.sv(i, j, k, l);
      mw += Y[l] / P->mw[l];
      cpt += Y[l] * cp[l];
      cvv += Y[l] * (cp[l] - R_u / P->mw[l]);
    }
    mw = 1 / mw;
    Zn.cp(i, j, k) = cpt;
    Zn.gam(i, j, k) = cpt / cvv;
    Zn.a(i, j, k) = std::sqrt(Zn.gam(i, j, k) * R_u * T / mw);
    double mu, kap;
    transport(P, T, mw, Y, cp, Zn.bv(i, j, k, 0), Zn.bv(i, j, k, 4), &mu, &kap, rD);
    Zn.mul(i, j, k) = mu;
    Zn.kappa(i, j, k) = kap;
    for (int l = 0; l < ns; ++l) Zn.rhoD(i, j, k, l) = rD[l];
  } else {
    constexpr double c_temp = gamma_air * R_u / mw_air;
    constexpr double cpa = gamma_air * R_u / mw_air / (gamma_air - 1);
    Zn.a(i, j, k) = std::sqrt(c_temp * T);
    Zn.mul(i, j, k) = sutherland(T);
    Zn.kappa(i, j, k) = Zn.mul(i, j, k) * cpa / P->Pr;
  }
  Zn.mach(i, j, k) = Zn.vel(i, j, k) / Zn.a(i, j, k);
}

// ---------------------------------------------------------------------------
// boundary conditions: src/BoundCond.cuh:52-189 (symmetry, outflow, inflow)
// ---------------------------------------------------------------------------
void bc_symmetry(const ostc_param *P, Z &Zn, const ostc_bc_face &b) {  // BoundCond.cuh:52-118
  int dir[3] = {0, 0, 0};
  dir[b.face] = b.direction;
  for (int k = b.range_start[2]; k <= b.range_end[2]; ++k)
    for (int j = b.range_start[1]; j <= b.range_end[1]; ++j)
      for (int i = b.range_start[0]; i <= b.range_end[0]; ++i) {
        const int ii0 = i - dir[0], ij0 = j - dir[1], ik0 = k - dir[2];
        const double *m = Zn.metric.at(i, j, k);
        double kx = m[3 * b.face], ky = m[3 * b.face + 1], kz = m[3 * b.face + 2];
        const double km = std::sqrt(kx * kx + ky * ky + kz * kz);
        kx /= km;
        ky /= km;
        kz /= km;
        const double u1 = Zn.bv(ii0, ij0, ik0, 1), v1 = Zn.bv(ii0, ij0, ik0, 2), w1 = Zn.bv(ii0, ij0, ik0, 3);
        double uk = kx * u1 + ky * v1 + kz * w1;
        const double ut = u1 - kx * uk, vt = v1 - ky * uk, wt = w1 - kz * uk;
        Zn.bv(i, j, k, 1) = ut;
        Zn.bv(i, j, k, 2) = vt;
        Zn.bv(i, j, k, 3) = wt;
        Zn.vel(i, j, k) = std::sqrt(ut * ut + vt * vt + wt * wt);
        Zn.bv(i, j, k, 0) = Zn.bv(ii0, ij0, ik0, 0);
        Zn.bv(i, j, k, 4) = Zn.bv(ii0, ij0, ik0, 4);
        Zn.bv(i, j, k, 5) = Zn.bv(ii0, ij0, ik0, 5);
        for (int l = 0; l < P->n_scalar; ++l) Zn.sv(i, j, k, l) = Zn.sv(ii0, ij0, ik0, l);
        for (int g = 1; g <= Zn.ngg; ++g) {
          const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
          const int ii = i - g * dir[0], ij = j - g * dir[1], ik = k - g * dir[2];
          Zn.bv(gi, gj, gk, 0) = Zn.bv(ii, ij, ik, 0);
          const double u = Zn.bv(ii, ij, ik, 1), v = Zn.bv(ii, ij, ik, 2), w = Zn.bv(ii, ij, ik, 3);
          uk = kx * u + ky * v + kz * w;
          Zn.bv(gi, gj, gk, 1) = u - 2 * uk * kx;
          Zn.bv(gi, gj, gk, 2) = v - 2 * uk * ky;
          Zn.bv(gi, gj, gk, 3) = w - 2 * uk * kz;
          Zn.vel(gi, gj, gk) = std::sqrt(Zn.bv(gi, gj, gk, 1) * Zn.bv(gi, gj, gk, 1) +
                                         Zn.bv(gi, gj, gk, 2) * Zn.bv(gi, gj, gk, 2) +
                                         Zn.bv(gi, gj, gk, 3) * Zn.bv(gi, gj, gk, 3));
          Zn.bv(gi, gj, gk, 4) = Zn.bv(ii, ij, ik, 4);
          Zn.bv(gi, gj, gk, 5) = Zn.bv(ii, ij, ik, 5);
          for (int l = 0; l < P->n_scalar; ++l) Zn.sv(gi, gj, gk, l) = Zn.sv(ii, ij, ik, l);
          if (is_sst(P)) Zn.mut(gi, gj, gk) = Zn.mut(ii, ij, ik);
        }
      }
}

void bc_outflow(const ostc_param *P, Z &Zn, const ostc_bc_face &b, int with_cv) {  // BoundCond.cuh:120-150
  int dir[3] = {0, 0, 0};
  dir[b.face] = b.direction;
  for (int k = b.range_start[2]; k <= b.range_end[2]; ++k)
    for (int j = b.range_start[1]; j <= b.range_end[1]; ++j)
      for (int i = b.range_start[0]; i <= b.range_end[0]; ++i)
        for (int g = 1; g <= Zn.ngg; ++g) {
          const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
          for (int l = 0; l < 6; ++l) Zn.bv(gi, gj, gk, l) = Zn.bv(i, j, k, l);
          for (int l = 0; l < P->n_scalar; ++l) Zn.sv(gi, gj, gk, l) = Zn.sv(i, j, k, l);
          if (is_sst(P)) Zn.mut(gi, gj, gk) = Zn.mut(i, j, k);
          if (with_cv) cv_from_bv_point(P, Zn, gi, gj, gk);
        }
}

void bc_inflow(const ostc_param *P, Z &Zn, const ostc_bc_face &b, int with_cv) {  // BoundCond.cuh:152-210
  int dir[3] = {0, 0, 0};
  dir[b.face] = b.direction;
  auto set = [&](int i, int j, int k) {
    Zn.bv(i, j, k, 0) = b.density;
    Zn.bv(i, j, k, 1) = b.u;
    Zn.bv(i, j, k, 2) = b.v;
    Zn.bv(i, j, k, 3) = b.w;
    Zn.bv(i, j, k, 4) = b.pressure;
    Zn.bv(i, j, k, 5) = b.temperature;
    for (int l = 0; l < P->n_scalar; ++l) Zn.sv(i, j, k, l) = b.sv[l];
    if (is_sst(P)) Zn.mut(i, j, k) = b.mut;
  };
  for (int k = b.range_start[2]; k <= b.range_end[2]; ++k)
    for (int j = b.range_start[1]; j <= b.range_end[1]; ++j)
      for (int i = b.range_start[0]; i <= b.range_end[0]; ++i) {
        set(i, j, k);
        Zn.vel(i, j, k) = b.velocity;
        if (with_cv) cv_from_bv_point(P, Zn, i, j, k);
        for (int g = 1; g <= Zn.ngg; ++g) {
          const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
          set(gi, gj, gk);
          if (with_cv) cv_from_bv_point(P, Zn, gi, gj, gk);
        }
      }
}

// no-slip wall, laminar (BoundCond.cuh:415-526)
void bc_wall(const ostc_param *P, Z &Zn, const ostc_bc_face &b, int with_cv) {
  int dir[3] = {0, 0, 0};
  dir[b.face] = b.direction;
  const int ns = P->n_spec;
  for (int k = b.range_start[2]; k <= b.range_end[2]; ++k)
    for (int j = b.range_start[1]; j <= b.range_end[1]; ++j)
      for (int i = b.range_start[0]; i <= b.range_end[0]; ++i) {
        const int ii = i - dir[0], ij = j - dir[1], ik = k - dir[2];
        double t_wall = b.wall_temperature;
        if (!b.wall_isothermal) t_wall = Zn.bv(ii, ij, ik, 5);
        const double p = Zn.bv(ii, ij, ik, 4);
        double mw = mw_air;
        if (P->mix_model != OSTC_MIX_AIR) {
          mw = 0;
          for (int l = 0; l < ns; ++l) {
            Zn.sv(i, j, k, l) = Zn.sv(ii, ij, ik, l);
            mw += Zn.sv(i, j, k, l) / P->mw[l];
          }
          mw = 1 / mw;
        }
        const double rho_wall = p * mw / (t_wall * R_u);
        Zn.bv(i, j, k, 0) = rho_wall;
        Zn.bv(i, j, k, 1) = 0;
        Zn.bv(i, j, k, 2) = 0;
        Zn.bv(i, j, k, 3) = 0;
        Zn.bv(i, j, k, 4) = p;
        Zn.bv(i, j, k, 5) = t_wall;
        Zn.vel(i, j, k) = 0;
        if (is_sst(P)) {  // BoundCond.cuh:471-484; the mixture's viscosity at the wall species
          double Yw[MAXS];
          for (int l = 0; l < ns; ++l) Yw[l] = Zn.sv(i, j, k, l);
          const double mu_wall = ns > 0 ? mixture_viscosity(P, t_wall, Yw) : sutherland(t_wall);
          const double dy = Zn.wall(ii, ij, ik);
          Zn.sv(i, j, k, ns) = 0;
          Zn.sv(i, j, k, ns + 1) =
              dy > 1e-25 ? 60 * mu_wall / (rho_wall * sst::beta_1 * dy * dy) : Zn.sv(ii, ij, ik, ns + 1);
        }
        if (with_cv) cv_from_bv_point(P, Zn, i, j, k);
        for (int g = 1; g <= Zn.ngg; ++g) {
          const int ai = i - g * dir[0], aj = j - g * dir[1], ak = k - g * dir[2];
          const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
          const double u_i = Zn.bv(ai, aj, ak, 1), v_i = Zn.bv(ai, aj, ak, 2), w_i = Zn.bv(ai, aj, ak, 3);
          const double p_i = Zn.bv(ai, aj, ak, 4), t_i = Zn.bv(ai, aj, ak, 5);
          double t_g = t_i;
          if (b.wall_isothermal) {
            t_g = 2 * t_wall - t_i;
            if (t_g <= 0.1 * t_wall) t_g = t_wall;
          }
          if (P->mix_model != OSTC_MIX_AIR) {
            mw = 0;
            for (int l = 0; l < ns; ++l) {
              Zn.sv(gi, gj, gk, l) = Zn.sv(ai, aj, ak, l);
              mw += Zn.sv(gi, gj, gk, l) / P->mw[l];
            }
            mw = 1 / mw;
          }
          Zn.bv(gi, gj, gk, 0) = p_i * mw / (t_g * R_u);
          Zn.bv(gi, gj, gk, 1) = -u_i;
          Zn.bv(gi, gj, gk, 2) = -v_i;
          Zn.bv(gi, gj, gk, 3) = -w_i;
          Zn.bv(gi, gj, gk, 4) = p_i;
          Zn.bv(gi, gj, gk, 5) = t_g;
          if (is_sst(P)) {  // BoundCond.cuh:536-541
            Zn.sv(gi, gj, gk, ns) = 0;
            Zn.sv(gi, gj, gk, ns + 1) = Zn.sv(i, j, k, ns + 1);
            Zn.mut(gi, gj, gk) = 0;
          }
          if (with_cv) cv_from_bv_point(P, Zn, gi, gj, gk);
        }
      }
}

// Riemann-invariant far field (BoundCond.cuh:212-413); never recomputes cv
void bc_farfield(const ostc_param *P, Z &Zn, const ostc_bc_face &b) {
  int dir[3] = {0, 0, 0};
  dir[b.face] = b.direction;
  const int ns = P->n_spec, nsc = P->n_scalar;
  for (int k = b.range_start[2]; k <= b.range_end[2]; ++k)
    for (int j = b.range_start[1]; j <= b.range_end[1]; ++j)
      for (int i = b.range_start[0]; i <= b.range_end[0]; ++i) {
        const double *m = Zn.metric.at(i, j, k);
        double nx = m[3 * b.face], ny = m[3 * b.face + 1], nz = m[3 * b.face + 2];
        const double gni = b.direction / std::sqrt(nx * nx + ny * ny + nz * nz);
        nx *= gni;
        ny *= gni;
        nz *= gni;
        const double u_b = Zn.bv(i, j, k, 1), v_b = Zn.bv(i, j, k, 2), w_b = Zn.bv(i, j, k, 3);
        const double u_face = nx * u_b + ny * v_b + nz * w_b;
        double gamma_b = gamma_air, mw = mw_air, sv_b[MAXS + 4] = {0}, cp[MAXS];
        // the point's own scalars; for air with SST the reference leaves sv_b
        // unset on subsonic outflow (BoundCond.cuh:244, 330-336), where these are kept
        for (int l = 0; l < nsc; ++l) sv_b[l] = Zn.sv(i, j, k, l);
        const bool turb = is_sst(P);
        if (P->mix_model != OSTC_MIX_AIR) {
          gamma_b = Zn.gam(i, j, k);
          double mw_inv = 0;
          for (int l = 0; l < ns; ++l) mw_inv += sv_b[l] / P->mw[l];
          mw = 1.0 / mw_inv;
        }
        const double p_b = Zn.bv(i, j, k, 4), rho_b = Zn.bv(i, j, k, 0);
        const double a_b = std::sqrt(gamma_b * p_b / rho_b);
        const double mach_b = u_face / a_b;
        auto set = [&](int gi, int gj, int gk, double rho, double u, double v, double w, double p, double T,
                       const double *svv) {
          Zn.bv(gi, gj, gk, 0) = rho;
          Zn.bv(gi, gj, gk, 1) = u;
          Zn.bv(gi, gj, gk, 2) = v;
          Zn.bv(gi, gj, gk, 3) = w;
          Zn.bv(gi, gj, gk, 4) = p;
          Zn.bv(gi, gj, gk, 5) = T;
          for (int l = 0; l < nsc; ++l) Zn.sv(gi, gj, gk, l) = svv[l];
        };
        if (mach_b <= -1) {
          set(i, j, k, b.density, b.u, b.v, b.w, b.pressure, b.temperature, b.sv);
          if (turb) Zn.mut(i, j, k) = b.mut;
          Zn.vel(i, j, k) = std::sqrt(b.u * b.u + b.v * b.v + b.w * b.w);
          for (int g = 1; g <= Zn.ngg; ++g) {
            set(i + g * dir[0], j + g * dir[1], k + g * dir[2], b.density, b.u, b.v, b.w, b.pressure, b.temperature,
                b.sv);
            if (turb) Zn.mut(i + g * dir[0], j + g * dir[1], k + g * dir[2]) = b.mut;
          }
        } else if (mach_b >= 1) {
          for (int g = 1; g <= Zn.ngg; ++g) {
            const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
            for (int l = 0; l < 6; ++l) Zn.bv(gi, gj, gk, l) = Zn.bv(i, j, k, l);
            for (int l = 0; l < nsc; ++l) Zn.sv(gi, gj, gk, l) = Zn.sv(i, j, k, l);
            if (turb) Zn.mut(gi, gj, gk) = Zn.mut(i, j, k);
          }
        } else {
          const double r_pos = u_face + 2 * a_b / (gamma_b - 1);
          const double u_inf = b.u * nx + b.v * ny + b.w * nz;
          const double r_neg = u_inf - 2 * b.acoustic_speed / (b.specific_heat_ratio - 1);
          const double Un = 0.5 * (r_pos + r_neg);
          double s_b, rho = 0, p = 0, T = 0, u, v, w;
          double mut_b = 0;
          if (turb) mut_b = (P->mix_model == OSTC_MIX_AIR ? mach_b <= 0 : mach_b < 0) ? b.mut : Zn.mut(i, j, k);
          if (P->mix_model == OSTC_MIX_AIR) {
            const double c_b = 0.25 * (gamma_air - 1) * (r_pos - r_neg);
            if (mach_b <= 0) {
              s_b = b.entropy;
              u = b.u + (Un - u_inf) * nx;
              v = b.v + (Un - u_inf) * ny;
              w = b.w + (Un - u_inf) * nz;
              for (int l = 0; l < nsc; ++l) sv_b[l] = b.sv[l];
            } else {
              s_b = p_b / std::pow(rho_b, gamma_air);
              u = u_b + (Un - u_face) * nx;
              v = v_b + (Un - u_face) * ny;
              w = w_b + (Un - u_face) * nz;
            }
            rho = std::pow(c_b * c_b / (gamma_air * s_b), 1 / (gamma_air - 1));
            p = rho * c_b * c_b / gamma_air;
            T = p * mw_air / (rho * R_u);
          } else {
            if (mach_b < 0) {
              u = b.u + (Un - u_inf) * nx;
              v = b.v + (Un - u_inf) * ny;
              w = b.w + (Un - u_inf) * nz;
              for (int l = 0; l < nsc; ++l) sv_b[l] = b.sv[l];
              mw = b.mw;
            } else {
              u = u_b + (Un - u_face) * nx;
              v = v_b + (Un - u_face) * ny;
              w = w_b + (Un - u_face) * nz;
            }
            double gamma = gamma_air, err = 1, gamma_last;
            for (int it = 0; it < 100 && err > 1e-4; ++it) {
              gamma_last = gamma;
              const double c_b = 0.25 * (gamma - 1) * (r_pos - r_neg);
              s_b = mach_b <= 0 ? b.entropy : p_b / std::pow(rho_b, gamma);
              rho = std::pow(c_b * c_b / (gamma * s_b), 1 / (gamma - 1));
              p = rho * c_b * c_b / gamma;
              T = p * mw / (rho * R_u);
              cp_only(P, T, cp);
              double cp_tot = 0;
              for (int l = 0; l < ns; ++l) cp_tot += cp[l] * sv_b[l];
              gamma = cp_tot / (cp_tot - R_u / mw);
              err = std::abs(1 - gamma / gamma_last);
            }
          }
          set(i, j, k, rho, u, v, w, p, T, sv_b);
          if (turb) Zn.mut(i, j, k) = mut_b;
          Zn.vel(i, j, k) = std::sqrt(u * u + v * v + w * w);
          for (int g = 1; g <= Zn.ngg; ++g) {
            set(i + g * dir[0], j + g * dir[1], k + g * dir[2], rho, u, v, w, p, T, sv_b);
            if (turb) Zn.mut(i + g * dir[0], j + g * dir[1], k + g * dir[2]) = mut_b;
          }
        }
      }
}

// back pressure (BoundCond.cuh:636-671)
void bc_back_pressure(const ostc_param *P, Z &Zn, const ostc_bc_face &b, int with_cv) {
  int dir[3] = {0, 0, 0};
  dir[b.face] = b.direction;
  for (int k = b.range_start[2]; k <= b.range_end[2]; ++k)
    for (int j = b.range_start[1]; j <= b.range_end[1]; ++j)
      for (int i = b.range_start[0]; i <= b.range_end[0]; ++i)
        for (int g = 1; g <= Zn.ngg; ++g) {
          const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
          for (int l = 0; l < 4; ++l) Zn.bv(gi, gj, gk, l) = Zn.bv(i, j, k, l);
          Zn.bv(gi, gj, gk, 4) = b.pressure;
          Zn.bv(gi, gj, gk, 5) = Zn.bv(i, j, k, 5);
          for (int l = 0; l < P->n_scalar; ++l) Zn.sv(gi, gj, gk, l) = Zn.sv(i, j, k, l);
          if (is_sst(P)) Zn.mut(gi, gj, gk) = Zn.mut(i, j, k);
          if (with_cv) cv_from_bv_point(P, Zn, gi, gj, gk);
        }
}

// subsonic inflow from total conditions, air (BoundCond.cuh:528-634)
void bc_subsonic_inflow(const ostc_param *P, Z &Zn, const ostc_bc_face &b, int with_cv) {
  int dir[3] = {0, 0, 0};
  dir[b.face] = b.direction;
  for (int k = b.range_start[2]; k <= b.range_end[2]; ++k)
    for (int j = b.range_start[1]; j <= b.range_end[1]; ++j)
      for (int i = b.range_start[0]; i <= b.range_end[0]; ++i) {
        const double *m = Zn.metric.at(i, j, k);
        double nx = m[3 * b.face], ny = m[3 * b.face + 1], nz = m[3 * b.face + 2];
        const double gni = b.direction / std::sqrt(nx * nx + ny * ny + nz * nz);
        nx *= gni;
        ny *= gni;
        nz *= gni;
        const double rho0 = Zn.bv(i, j, k, 0), u0 = Zn.bv(i, j, k, 1), v0 = Zn.bv(i, j, k, 2), w0 = Zn.bv(i, j, k, 3);
        const double p0 = Zn.bv(i, j, k, 4);
        const double u_face = nx * u0 + ny * v0 + nz * w0;
        const double a = std::sqrt(gamma_air * p0 / rho0);
        const double r_neg = std::abs(u_face) - 2 * a / (gamma_air - 1);
        const double hti = p0 / rho0 * gamma_air / (gamma_air - 1) + 0.5 * (u0 * u0 + v0 * v0 + w0 * w0);
        constexpr double qa = 1 + 2.0 / (gamma_air - 1);
        const double qb = 2 * r_neg;
        const double qc = (gamma_air - 1) * (0.5 * r_neg * r_neg - hti);
        const double delta = qb * qb - 4 * qa * qc;
        double a_new = a;
        if (delta >= 0) {
          const double ap = (-qb + std::sqrt(delta)) / (2 * qa), am = (-qb - std::sqrt(delta)) / (2 * qa);
          a_new = ap > am ? ap : am;
        }
        const double u_new = r_neg + 2 * a_new / (gamma_air - 1);
        const double mach = u_new / a_new;
        const double p = b.total_pressure * std::pow(1 + 0.5 * (gamma_air - 1) * mach * mach, -gamma_air / (gamma_air - 1));
        const double T = b.total_temperature * std::pow(p / b.total_pressure, (gamma_air - 1) / gamma_air);
        const double rho = p * mw_air / (T * R_u);
        for (int g = 1; g <= Zn.ngg; ++g) {
          const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
          Zn.bv(gi, gj, gk, 0) = rho;
          Zn.bv(gi, gj, gk, 1) = u_new * b.u;
          Zn.bv(gi, gj, gk, 2) = u_new * b.v;
          Zn.bv(gi, gj, gk, 3) = u_new * b.w;
          Zn.bv(gi, gj, gk, 4) = p;
          Zn.bv(gi, gj, gk, 5) = T;
          const double u_bar = Zn.bv(gi, gj, gk, 1) * nx + Zn.bv(gi, gj, gk, 2) * ny + Zn.bv(gi, gj, gk, 3) * nz;
          for (int l = 0; l < P->n_scalar; ++l) Zn.sv(gi, gj, gk, l) = u_bar > 0 ? Zn.sv(i, j, k, l) : b.sv[l];
          if (is_sst(P)) Zn.mut(gi, gj, gk) = Zn.mut(i, j, k);
          if (with_cv) cv_from_bv_point(P, Zn, gi, gj, gk);
        }
      }
}

// periodic (no reference counterpart): ghost layers wrap from the opposite side
void bc_periodic(const ostc_param *P, Z &Zn, const ostc_bc_face &b, int with_cv) {
  const int ext[3] = {Zn.mx, Zn.my, Zn.mz};
  const int n = ext[b.face];
  int dir[3] = {0, 0, 0};
  dir[b.face] = b.direction;
  for (int k = b.range_start[2]; k <= b.range_end[2]; ++k)
    for (int j = b.range_start[1]; j <= b.range_end[1]; ++j)
      for (int i = b.range_start[0]; i <= b.range_end[0]; ++i)
        for (int g = 1; g <= Zn.ngg; ++g) {
          const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
          int si = gi, sj = gj, sk = gk;
          int *s = b.face == 0 ? &si : (b.face == 1 ? &sj : &sk);
          *s -= b.direction * n;
          for (int l = 0; l < 6; ++l) Zn.bv(gi, gj, gk, l) = Zn.bv(si, sj, sk, l);
          for (int l = 0; l < P->n_scalar; ++l) Zn.sv(gi, gj, gk, l) = Zn.sv(si, sj, sk, l);
          if (is_sst(P)) Zn.mut(gi, gj, gk) = Zn.mut(si, sj, sk);
          Zn.vel(gi, gj, gk) = Zn.vel(si, sj, sk);
          if (with_cv)
            for (int l = 0; l < P->n_var; ++l) Zn.cv(gi, gj, gk, l) = Zn.cv(si, sj, sk, l);
        }
}

std::vector<ostc_interface> g_ifaces;

// inner_communication (DataCommunication.cuh:58-110) for one interface
void interface_exchange(const ostc_param *P, Z &Zs, Z &Zt, const ostc_interface &f, int with_cv) {
  const int plane = f.direction > 0 ? f.range_start[f.face] : f.range_end[f.face];
  for (int n2 = 0; n2 < f.n_point[2]; ++n2)
    for (int n1 = 0; n1 < f.n_point[1]; ++n1)
      for (int n0 = 0; n0 < f.n_point[0]; ++n0) {
        const int n[3] = {n0, n1, n2};
        int idx[3], d[3], it[3];
        for (int a = 0; a < 3; ++a) {
          d[a] = f.loop_dir[a] * n[a];
          idx[a] = f.range_start[a] + d[a];
        }
        for (int a = 0; a < 3; ++a) it[a] = f.target_start[a] + f.target_loop_dir[a] * d[f.src_tar[a]];
        if (idx[f.face] == plane) {
          for (int l = 0; l < 6; ++l) {
            const double ave = 0.5 * (Zt.bv(it[0], it[1], it[2], l) + Zs.bv(idx[0], idx[1], idx[2], l));
            Zs.bv(idx[0], idx[1], idx[2], l) = ave;
            Zt.bv(it[0], it[1], it[2], l) = ave;
          }
          for (int l = 0; l < P->n_scalar; ++l) {
            const double ave = 0.5 * (Zt.sv(it[0], it[1], it[2], l) + Zs.sv(idx[0], idx[1], idx[2], l));
            Zs.sv(idx[0], idx[1], idx[2], l) = ave;
            Zt.sv(it[0], it[1], it[2], l) = ave;
          }
          const double u = Zs.bv(idx[0], idx[1], idx[2], 1), v = Zs.bv(idx[0], idx[1], idx[2], 2),
                       w = Zs.bv(idx[0], idx[1], idx[2], 3);
          const double vel = std::sqrt(u * u + v * v + w * w);
          Zs.vel(idx[0], idx[1], idx[2]) = vel;
          Zt.vel(it[0], it[1], it[2]) = vel;
        } else {
          for (int l = 0; l < 6; ++l) Zs.bv(idx[0], idx[1], idx[2], l) = Zt.bv(it[0], it[1], it[2], l);
          for (int l = 0; l < P->n_scalar; ++l) Zs.sv(idx[0], idx[1], idx[2], l) = Zt.sv(it[0], it[1], it[2], l);
        }
        if (with_cv) cv_from_bv_point(P, Zs, idx[0], idx[1], idx[2]);
      }
}

// operator-split chemistry (config chem_mode != 0) takes the source out of the RHS
bool g_skip_source = false;

void compute_rhs_zone(const ostc_param *P, Z &Zn) {
  const long nint = (long)Zn.mx * Zn.my * Zn.mz;
  const int nv = P->n_var;
  // cudaMemset(dq, 0) (RK.cuh:110): dq carries dq_ngg ghosts
  const View &dq = Zn.dq;
  std::fill(dq.p, dq.p + dq.sz * nv, 0.0);
  (void)nint;
  // compute_source<mix, Laminar>: finite-rate chemistry (SourceTerm.cuh:11-37)
  if (P->mix_model == OSTC_MIX_FR && P->n_reac > 0 && !g_skip_source) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Zn.mz; ++k)
      for (int j = 0; j < Zn.my; ++j)
        for (int i = 0; i < Zn.mx; ++i) {
          double Y[MAXS], om[MAXS];
          for (int l = 0; l < P->n_spec; ++l) Y[l] = Zn.sv(i, j, k, l);
          chemistry_omega(P, Zn.bv(i, j, k, 0), Zn.bv(i, j, k, 5), Y, om, nullptr, nullptr);
          for (int l = 0; l < P->n_spec; ++l) Zn.dq(i, j, k, l + 5) += Zn.jac(i, j, k) * om[l];
        }
  }
  // compute_source<Air, SST>: mut, turbulent conductivity, k and omega sources
  if (is_sst(P)) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Zn.mz; ++k)
      for (int j = 0; j < Zn.my; ++j)
        for (int i = 0; i < Zn.mx; ++i) sst::source_and_mut(P, Zn, i, j, k);
  }
  // inviscid: x, y, then z when 3-D (InviscidScheme.cu:23-45, 176-204)
  inviscid_direction(P, Zn, 0);
  inviscid_direction(P, Zn, 1);
  if (Zn.mz > 1) inviscid_direction(P, Zn, 2);
  // viscous: x, y, z (SchemeSelector.cuh:49-69)
  if (P->viscous_scheme != 0) {
    viscous_direction(P, Zn, 0);
    viscous_direction(P, Zn, 1);
    if (Zn.mz > 1) viscous_direction(P, Zn, 2);
  }
}


// ---------------------------------------------------------------------------
// steady path: SteadySim.cuh:15-137 with its implicit treatments
// ---------------------------------------------------------------------------
// compute_chem_src_jacobian (FiniteRateChem.cu:196-216), row-major m*ns+n
void chem_jacobian(const ostc_param *P, double rho, const double *Y, const double *q1, const double *q2,
                   double *J) {
  const int ns = P->n_spec, nr = P->n_reac;
  for (int m = 0; m < ns; ++m)
    for (int n = 0; n < ns; ++n) {
      double zz = 0;
      if (Y[n] > 1e-25) {
        for (int r = 0; r < nr; ++r)
          zz += (P->stoi_b[r * ns + m] - P->stoi_f[r * ns + m]) *
                (P->stoi_f[r * ns + n] * q1[r] - P->stoi_b[r * ns + n] * q2[r]);
        zz /= rho * Y[n];
      }
      J[m * ns + n] = P->mw[m] * zz * 1e+3;
    }
}

// solve_chem_system (FiniteRateChem.cu:324-419): column-pivoted LU, then solve
void lu_factor(double *A, int *ipiv, int dim) {
  for (int n = 0; n < dim; ++n) {
    int ik = n;
    for (int m = n; m < dim; ++m) {
      for (int t = 0; t < n; ++t) A[m * dim + n] -= A[m * dim + t] * A[t * dim + n];
      if (std::abs(A[m * dim + n]) > std::abs(A[ik * dim + n])) ik = m;
    }
    ipiv[n] = ik;
    if (ik != n)
      for (int t = 0; t < dim; ++t) std::swap(A[ik * dim + t], A[n * dim + t]);
    for (int p = n + 1; p < dim; ++p)
      for (int t = 0; t < n; ++t) A[n * dim + p] -= A[n * dim + t] * A[t * dim + p];
    for (int m = n + 1; m < dim; ++m) A[m * dim + n] /= A[n * dim + n];
  }
}
void lu_apply(const double *A, const int *ipiv, double *b, int dim) {
  for (int m = 0; m < dim; ++m)
    if (ipiv[m] != m) std::swap(b[ipiv[m]], b[m]);
  for (int m = 1; m < dim; ++m)
    for (int t = 0; t < m; ++t) b[m] -= A[m * dim + t] * b[t];
  b[dim - 1] /= A[dim * dim - 1];
  for (int m = dim - 2; m >= 0; --m) {
    for (int t = m + 1; t < dim; ++t) b[m] -= A[m * dim + t] * b[t];
    b[m] /= A[m * dim + m];
  }
}

// local_time_step (TimeAdvanceFunc.cuh:50-100): dt_local and the inviscid
// spectral radii (3 per interior point)
void local_time_step_zone(const ostc_param *P, Z &Zn, std::vector<double> &isr) {
  const int dim = Zn.mz == 1 ? 2 : 3;
  isr.assign(3 * (size_t)Zn.mx * Zn.my * Zn.mz, 0.0);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < Zn.mz; ++k)
    for (int j = 0; j < Zn.my; ++j)
      for (int i = 0; i < Zn.mx; ++i) {
        const double *m = Zn.metric.at(i, j, k);
        const double gx = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
        const double ge = std::sqrt(m[3] * m[3] + m[4] * m[4] + m[5] * m[5]);
        const double gz = std::sqrt(m[6] * m[6] + m[7] * m[7] + m[8] * m[8]);
        const double u = Zn.bv(i, j, k, 1), v = Zn.bv(i, j, k, 2), w = Zn.bv(i, j, k, 3);
        const double U = u * m[0] + v * m[1] + w * m[2];
        const double V = u * m[3] + v * m[4] + w * m[5];
        const double W = u * m[6] + v * m[7] + w * m[8];
        const double a = Zn.a(i, j, k);
        const size_t q = 3 * (((size_t)k * Zn.my + j) * Zn.mx + i);
        isr[q] = std::abs(U) + a * gx;
        isr[q + 1] = std::abs(V) + a * ge;
        isr[q + 2] = dim == 3 ? std::abs(W) + a * gz : 0.0;
        const double sri = isr[q] + isr[q + 1] + isr[q + 2];
        double gamma = gamma_air;
        if (P->mix_model != OSTC_MIX_AIR) gamma = Zn.gam(i, j, k);
        const double c1 = std::max(gamma, 4.0 / 3.0) / Zn.bv(i, j, k, 0);
        double c2 = Zn.mul(i, j, k) / P->Pr;
        if (is_sst(P)) c2 += Zn.mut(i, j, k) / P->Prt;
        double srv = gx * gx + ge * ge;
        if (dim == 3) srv += gz * gz;
        srv *= c1 * c2;
        Zn.dt_local(i, j, k) = P->cfl / (sri + srv);
      }
}

// rates, omega_d and (optionally) the full Jacobian at one cell
void cell_chemistry(const ostc_param *P, Z &Zn, int i, int j, int k, double *Y, double &rho, double *J,
                    double *od) {
  const int ns = P->n_spec;
  rho = Zn.bv(i, j, k, 0);
  for (int l = 0; l < ns; ++l) Y[l] = Zn.sv(i, j, k, l);
  double om[MAXS], q1[MAXR], q2[MAXR];
  chemistry_omega(P, rho, Zn.bv(i, j, k, 5), Y, om, q1, q2, od);
  if (J) chem_jacobian(P, rho, Y, q1, q2, J);
}

// EPI / DA of the explicit steady step (FiniteRateChem.cu:234-256, 421-432)
void chem_implicit_zone(const ostc_param *P, Z &Zn) {
  const int ns = P->n_spec;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < Zn.mz; ++k)
    for (int j = 0; j < Zn.my; ++j)
      for (int i = 0; i < Zn.mx; ++i) {
        double Y[MAXS], J[MAXS * MAXS], od[MAXS], rho;
        const double dt = Zn.dt_local(i, j, k);
        if (P->chemSrcMethod == 1) {
          cell_chemistry(P, Zn, i, j, k, Y, rho, J, od);
          for (int m = 0; m < ns; ++m)
            for (int n = 0; n < ns; ++n) J[m * ns + n] = m == n ? 1.0 - dt * J[m * ns + n] : -dt * J[m * ns + n];
          double b[MAXS];
          int ipiv[MAXS];
          for (int l = 0; l < ns; ++l) b[l] = Zn.dq(i, j, k, 5 + l);
          lu_factor(J, ipiv, ns);
          lu_apply(J, ipiv, b, ns);
          for (int l = 0; l < ns; ++l) Zn.dq(i, j, k, 5 + l) = b[l];
        } else if (P->chemSrcMethod == 2) {
          cell_chemistry(P, Zn, i, j, k, Y, rho, nullptr, od);
          for (int l = 0; l < ns; ++l) {
            const double jd = Y[l] > 1e-25 ? -od[l] / (Y[l] * rho) : 0.0;
            Zn.dq(i, j, k, 5 + l) /= 1 - dt * jd;
          }
        }
      }
}

// update_bv (FieldOperation.cuh:221-296)
void update_bv_zone(const ostc_param *P, Z &Zn) {
  const int ns = P->n_spec;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < Zn.mz; ++k)
    for (int j = 0; j < Zn.my; ++j)
      for (int i = 0; i < Zn.mx; ++i) {
        const double rho_n = Zn.bv(i, j, k, 0);
        const double u_n = Zn.bv(i, j, k, 1), v_n = Zn.bv(i, j, k, 2), w_n = Zn.bv(i, j, k, 3);
        double E = 0.5 * (u_n * u_n + v_n * v_n + w_n * w_n);
        if (P->mix_model != OSTC_MIX_AIR) {
          double h[MAXS];
          enthalpy(P, Zn.bv(i, j, k, 5), h);
          for (int l = 0; l < ns; ++l) E += h[l] * Zn.sv(i, j, k, l);
          E *= rho_n;
          E -= Zn.bv(i, j, k, 4);
        } else {
          E *= rho_n;
          E += Zn.bv(i, j, k, 4) / (gamma_air - 1);
        }
        const double dtj = Zn.dt_local(i, j, k) / Zn.jac(i, j, k);
        Zn.bv(i, j, k, 0) += Zn.dq(i, j, k, 0) * dtj;
        const double ri = 1.0 / Zn.bv(i, j, k, 0);
        Zn.bv(i, j, k, 1) = ri * (rho_n * Zn.bv(i, j, k, 1) + Zn.dq(i, j, k, 1) * dtj);
        Zn.bv(i, j, k, 2) = ri * (rho_n * Zn.bv(i, j, k, 2) + Zn.dq(i, j, k, 2) * dtj);
        if (Zn.mz == 1)
          Zn.bv(i, j, k, 3) = 0;
        else
          Zn.bv(i, j, k, 3) = ri * (rho_n * Zn.bv(i, j, k, 3) + Zn.dq(i, j, k, 3) * dtj);
        const double Et = E + Zn.dq(i, j, k, 4) * dtj;
        for (int l = 0; l < P->n_scalar; ++l)
          Zn.sv(i, j, k, l) = ri * (rho_n * Zn.sv(i, j, k, l) + Zn.dq(i, j, k, 5 + l) * dtj);
        const double V2 = Zn.bv(i, j, k, 1) * Zn.bv(i, j, k, 1) + Zn.bv(i, j, k, 2) * Zn.bv(i, j, k, 2) +
                          Zn.bv(i, j, k, 3) * Zn.bv(i, j, k, 3);
        if (P->mix_model != OSTC_MIX_AIR) {
          temperature_and_pressure(P, Zn, i, j, k, Et);
        } else {
          Zn.bv(i, j, k, 4) = (gamma_air - 1) * (Et - 0.5 * Zn.bv(i, j, k, 0) * V2);
          Zn.bv(i, j, k, 5) = Zn.bv(i, j, k, 4) * mw_air * ri / R_u;
        }
        Zn.vel(i, j, k) = std::sqrt(V2);
      }
}

// compute_jacobian_times_dq (DPLUR.cuh:81-140) at (i,j,k), direction dir
void jacobian_times_dq(const ostc_param *P, Z &Zn, const View &dqv, int i, int j, int k, int dir, double lam,
                       double *out) {
  const int ns = P->n_spec;
  const double *m = Zn.metric.at(i, j, k);
  const double kx = m[3 * dir], ky = m[3 * dir + 1], kz = m[3 * dir + 2];
  const double u = Zn.bv(i, j, k, 1), v = Zn.bv(i, j, k, 2), w = Zn.bv(i, j, k, 3);
  const double U = kx * u + ky * v + kz * w;
  const double lmd1 = U + lam;
  const double e = 0.5 * Zn.vel(i, j, k) * Zn.vel(i, j, k);
  double gamma = gamma_air, b3 = 0, b4 = 0, h = 0;
  if (P->mix_model == OSTC_MIX_AIR) {
    h = gamma / (gamma - 1) * Zn.bv(i, j, k, 4) / Zn.bv(i, j, k, 0) + e;
  } else {
    const double t = Zn.bv(i, j, k, 5);
    double hk[MAXS];
    enthalpy(P, t, hk);
    gamma = Zn.gam(i, j, k);
    for (int l = 0; l < ns; ++l) {
      b3 += R_u * t / P->mw[l] * dqv(i, j, k, 5 + l);
      b4 += hk[l] * dqv(i, j, k, 5 + l);
      h += Zn.sv(i, j, k, l) * hk[l];
    }
    b3 *= gamma;
    b4 *= gamma - 1;
    h += e;
  }
  const double b1 = kx * dqv(i, j, k, 1) + ky * dqv(i, j, k, 2) + kz * dqv(i, j, k, 3) - U * dqv(i, j, k, 0);
  const double b2 = (gamma - 1) * (e * dqv(i, j, k, 0) - u * dqv(i, j, k, 1) - v * dqv(i, j, k, 2) -
                                   w * dqv(i, j, k, 3) + dqv(i, j, k, 4));
  out[0] = b1 + lmd1 * dqv(i, j, k, 0);
  out[1] = u * b1 + kx * b2 + lmd1 * dqv(i, j, k, 1) + kx * (b3 - b4);
  out[2] = v * b1 + ky * b2 + lmd1 * dqv(i, j, k, 2) + ky * (b3 - b4);
  out[3] = w * b1 + kz * b2 + lmd1 * dqv(i, j, k, 3) + kz * (b3 - b4);
  out[4] = h * b1 + U * b2 + lmd1 * dqv(i, j, k, 4) + U * (b3 - b4);
  for (int l = 0; l < P->n_scalar; ++l) out[5 + l] = lmd1 * dqv(i, j, k, 5 + l) + Zn.sv(i, j, k, l) * b1;
}

// DPLUR (DPLUR.cuh:14-314, DPLUR.cu:5-52) on one block
void dplur_zone(const ostc_config *c, const ostc_param *P, Z &Zn, const std::vector<double> &isr,
                const ostc_bc_face *f, int n_faces, int block) {
  const int nv = P->n_var, ns = P->n_spec;
  const int g = Zn.z->dq_ngg;
  const size_t nq = (size_t)(Zn.mx + 2 * g) * (Zn.my + 2 * g) * (Zn.mz + 2 * g) * nv;
  std::vector<double> dq0v(nq, 0.0), dqkv(nq, 0.0);
  View dq0(dq0v.data(), Zn.mx, Zn.my, Zn.mz, g), dqk(dqkv.data(), Zn.mx, Zn.my, Zn.mz, g);
  const bool chem = P->mix_model == OSTC_MIX_FR && P->n_reac > 0;
  auto R = [&](int i, int j, int k, int d) { return isr[3 * (((size_t)k * Zn.my + j) * Zn.mx + i) + d]; };
  // compute_DQ_0
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < Zn.mz; ++k)
    for (int j = 0; j < Zn.my; ++j)
      for (int i = 0; i < Zn.mx; ++i) {
        const double dt = Zn.dt_local(i, j, k);
        for (int l = 0; l < nv; ++l) Zn.dq(i, j, k, l) *= dt;
        const double diag = 1 + dt * (R(i, j, k, 0) + R(i, j, k, 1) + R(i, j, k, 2));
        for (int l = 0; l < 5; ++l) Zn.dq(i, j, k, l) /= diag;
        if (ns > 0) {
          if (chem && P->chemSrcMethod == 1) {
            double Y[MAXS], J[MAXS * MAXS], od[MAXS], rho, b[MAXS];
            int ipiv[MAXS];
            cell_chemistry(P, Zn, i, j, k, Y, rho, J, od);
            for (int m = 0; m < ns; ++m)
              for (int n = 0; n < ns; ++n) J[m * ns + n] = m == n ? diag - dt * J[m * ns + n] : -dt * J[m * ns + n];
            for (int l = 0; l < ns; ++l) b[l] = Zn.dq(i, j, k, 5 + l);
            lu_factor(J, ipiv, ns);
            lu_apply(J, ipiv, b, ns);
            for (int l = 0; l < ns; ++l) Zn.dq(i, j, k, 5 + l) = b[l];
          } else if (chem && P->chemSrcMethod == 2) {
            double Y[MAXS], od[MAXS], rho;
            cell_chemistry(P, Zn, i, j, k, Y, rho, nullptr, od);
            for (int l = 0; l < ns; ++l) {
              const double jd = Y[l] > 1e-25 ? -od[l] / (Y[l] * rho) : 0.0;
              Zn.dq(i, j, k, 5 + l) /= diag - dt * jd;
            }
          } else {
            for (int l = 5; l < 5 + ns; ++l) Zn.dq(i, j, k, l) /= diag;
          }
        }
        if (is_sst(P)) {  // DPLUR.cuh:72-84, SST.cu:249-258 (rows i_turb_cv, +1)
          for (int t = 0; t < 2; ++t)
            Zn.dq(i, j, k, 5 + ns + t) /= P->turb_implicit == 1 ? diag - dt * Zn.tsj(i, j, k, t) : diag;
        }
        for (int l = 0; l < nv; ++l) dq0(i, j, k, l) = Zn.dq(i, j, k, l);
      }
  for (int it = 0; it < c->DPLUR_inner_step; ++it) {
    // set_wall_dq_to_0 (DPLUR.cu:33-52)
    for (int q = 0; q < n_faces; ++q) {
      if (f[q].block != block || f[q].type_label != OSTC_BC_WALL) continue;
      for (int k = f[q].range_start[2]; k <= f[q].range_end[2]; ++k)
        for (int j = f[q].range_start[1]; j <= f[q].range_end[1]; ++j)
          for (int i = f[q].range_start[0]; i <= f[q].range_end[0]; ++i) {
            if (i < -g || j < -g || k < -g || i >= Zn.mx + g || j >= Zn.my + g || k >= Zn.mz + g) continue;
            for (int l = 0; l < nv; ++l) Zn.dq(i, j, k, l) = 0;
          }
    }
    // DPLUR_inner_iteration (DPLUR.cuh:161-280)
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Zn.mz; ++k)
      for (int j = 0; j < Zn.my; ++j)
        for (int i = 0; i < Zn.mx; ++i) {
          double tot[MAXS + 5] = {0}, cj[MAXS + 5];
          auto add = [&](double s) {
            for (int l = 0; l < nv; ++l) tot[l] += s * cj[l];
          };
          if (i > 0) { jacobian_times_dq(P, Zn, Zn.dq, i - 1, j, k, 0, R(i - 1, j, k, 0), cj); add(0.5); }
          if (j > 0) { jacobian_times_dq(P, Zn, Zn.dq, i, j - 1, k, 1, R(i, j - 1, k, 1), cj); add(0.5); }
          if (k > 0) { jacobian_times_dq(P, Zn, Zn.dq, i, j, k - 1, 2, R(i, j, k - 1, 2), cj); add(0.5); }
          if (i != Zn.mx - 1) {
            jacobian_times_dq(P, Zn, Zn.dq, i + 1, j, k, 0, -R(i + 1, j, k, 0), cj);
            for (int l = 0; l < nv; ++l) tot[l] -= 0.5 * cj[l];
          }
          if (j != Zn.my - 1) {
            jacobian_times_dq(P, Zn, Zn.dq, i, j + 1, k, 1, -R(i, j + 1, k, 1), cj);
            for (int l = 0; l < nv; ++l) tot[l] -= 0.5 * cj[l];
          }
          if (k != Zn.mz - 1) {
            jacobian_times_dq(P, Zn, Zn.dq, i, j, k + 1, 2, -R(i, j, k + 1, 2), cj);
            for (int l = 0; l < nv; ++l) tot[l] -= 0.5 * cj[l];
          }
          const double dt = Zn.dt_local(i, j, k);
          const double diag = 1 + dt * (R(i, j, k, 0) + R(i, j, k, 1) + R(i, j, k, 2));
          for (int l = 0; l < 5; ++l) dqk(i, j, k, l) = dq0(i, j, k, l) + dt * tot[l] / diag;
          if (ns > 0) {
            if (chem && P->chemSrcMethod == 1) {
              double Y[MAXS], J[MAXS * MAXS], od[MAXS], rho, b[MAXS];
              int ipiv[MAXS];
              cell_chemistry(P, Zn, i, j, k, Y, rho, J, od);
              for (int m = 0; m < ns; ++m)
                for (int n = 0; n < ns; ++n)
                  J[m * ns + n] = m == n ? diag - dt * J[m * ns + n] : -dt * J[m * ns + n];
              for (int l = 0; l < ns; ++l) b[l] = tot[5 + l] * dt;
              lu_factor(J, ipiv, ns);
              lu_apply(J, ipiv, b, ns);
              for (int l = 0; l < ns; ++l) dqk(i, j, k, 5 + l) = dq0(i, j, k, 5 + l) + b[l];
            } else if (chem && P->chemSrcMethod == 2) {
              double Y[MAXS], od[MAXS], rho;
              cell_chemistry(P, Zn, i, j, k, Y, rho, nullptr, od);
              for (int l = 0; l < ns; ++l) {
                const double jd = Y[l] > 1e-25 ? -od[l] / (Y[l] * rho) : 0.0;
                dqk(i, j, k, 5 + l) = dq0(i, j, k, 5 + l) + dt * tot[5 + l] / (diag - dt * jd);
              }
            } else {
              for (int l = 5; l < 5 + ns; ++l) dqk(i, j, k, l) = dq0(i, j, k, l) + dt * tot[l] / diag;
            }
          }
          if (is_sst(P)) {  // DPLUR.cuh:262-276, SST.cu:260-273 (rows i_turb_cv, +1)
            for (int t = 0; t < 2; ++t)
              dqk(i, j, k, 5 + ns + t) =
                  dq0(i, j, k, 5 + ns + t) +
                  dt * tot[5 + ns + t] / (P->turb_implicit == 1 ? diag - dt * Zn.tsj(i, j, k, t) : diag);
          }
        }
    // dq <- dqk over the interior (the ghost layer of dq is never read)
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Zn.mz; ++k)
      for (int j = 0; j < Zn.my; ++j)
        for (int i = 0; i < Zn.mx; ++i)
          for (int l = 0; l < nv; ++l) Zn.dq(i, j, k, l) = dqk(i, j, k, l);
  }
  // convert_dq_back_to_dqDt (DPLUR.cu:5-17)
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < Zn.mz; ++k)
    for (int j = 0; j < Zn.my; ++j)
      for (int i = 0; i < Zn.mx; ++i) {
        const double dt = Zn.dt_local(i, j, k);
        for (int l = 0; l < nv; ++l) Zn.dq(i, j, k, l) /= dt;
      }
}

}  // namespace

// ===========================================================================
// extern "C" API
// ===========================================================================
extern "C" {

void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int oracle_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int oracle_compute_cv_from_bv(const ostc_param *P, ostc_zone *z) {
  Z Zn(z);
  const int g = Zn.ngg;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = -g; k < Zn.mz + g; ++k)
    for (int j = -g; j < Zn.my + g; ++j)
      for (int i = -g; i < Zn.mx + g; ++i) cv_from_bv_point(P, Zn, i, j, k);
  return 0;
}

int oracle_flux_scale(const ostc_param *P, ostc_zone *z, double *scale) {
  for (int l = 0; l < P->n_var; ++l) scale[l] = 0;
  g_flux_scale = scale;
  const int st = oracle_compute_rhs(P, z);
  g_flux_scale = nullptr;
  return st;
}

int oracle_compute_rhs(const ostc_param *P, ostc_zone *z) {
  if (P->inviscid_type == 1 && P->mix_model != OSTC_MIX_AIR) return OSTC_ERR_UNSUPPORTED;  // A2
  if (P->inviscid_scheme == 1 && P->mix_model != OSTC_MIX_AIR) return OSTC_ERR_UNSUPPORTED;
  Z Zn(z);
  compute_rhs_zone(P, Zn);
  return 0;
}

double oracle_global_time_step(const ostc_param *P, ostc_zone *zones, int n_zones) {
  double dt = 1e+6;  // TimeAdvanceFunc.cu:156
  for (int b = 0; b < n_zones; ++b) {
    Z Zn(&zones[b]);
    const int dim = Zn.mz == 1 ? 2 : 3;
    double dtb = 1e+6;  // min_of_arr seed, TimeAdvanceFunc.cu:190
#pragma omp parallel for collapse(2) reduction(min : dtb) schedule(static)
    for (int k = 0; k < Zn.mz; ++k)
      for (int j = 0; j < Zn.my; ++j)
        for (int i = 0; i < Zn.mx; ++i) {  // local_time_step, TimeAdvanceFunc.cuh:50-100
          const double *m = Zn.metric.at(i, j, k);
          const double gx = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
          const double ge = std::sqrt(m[3] * m[3] + m[4] * m[4] + m[5] * m[5]);
          const double gz = std::sqrt(m[6] * m[6] + m[7] * m[7] + m[8] * m[8]);
          const double u = Zn.bv(i, j, k, 1), v = Zn.bv(i, j, k, 2), w = Zn.bv(i, j, k, 3);
          const double U = u * m[0] + v * m[1] + w * m[2];
          const double V = u * m[3] + v * m[4] + w * m[5];
          const double W = u * m[6] + v * m[7] + w * m[8];
          const double a = Zn.a(i, j, k);
          const double r0 = std::abs(U) + a * gx, r1 = std::abs(V) + a * ge;
          const double r2 = dim == 3 ? std::abs(W) + a * gz : 0.0;
          const double sri = r0 + r1 + r2;
          double gamma = gamma_air;
          if (P->mix_model != OSTC_MIX_AIR) gamma = Zn.gam(i, j, k);
          const double c1 = std::max(gamma, 4.0 / 3.0) / Zn.bv(i, j, k, 0);
          double c2 = Zn.mul(i, j, k) / P->Pr;
          if (is_sst(P)) c2 += Zn.mut(i, j, k) / P->Prt;
          double srv = gx * gx + ge * ge;
          if (dim == 3) srv += gz * gz;
          srv *= c1 * c2;
          const double dtl = P->cfl / (sri + srv);
          if (Zn.z->dt_local) Zn.dt_local(i, j, k) = dtl;
          dtb = std::min(dtb, dtl);
        }
    dt = std::min(dt, dtb);
  }
  return dt;
}

int oracle_update_cv_and_bv_rk(const ostc_param *P, ostc_zone *z, double dt, int rk) {
  static const double A[3] = {1.0, 0.75, 1.0 / 3.0}, B[3] = {0.0, 0.25, 2.0 / 3.0},
                      C[3] = {1.0, 0.25, 2.0 / 3.0};  // RK.cuh:11-13
  Z Zn(z);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < Zn.mz; ++k)
    for (int j = 0; j < Zn.my; ++j)
      for (int i = 0; i < Zn.mx; ++i) {
        const double dtj = dt / Zn.jac(i, j, k);
        for (int l = 0; l < P->n_var; ++l)
          Zn.cv(i, j, k, l) = A[rk] * Zn.qn(i, j, k, l) + B[rk] * Zn.cv(i, j, k, l) + C[rk] * dtj * Zn.dq(i, j, k, l);
        if (Zn.mz == 1) Zn.cv(i, j, k, 3) = 0;
        Zn.bv(i, j, k, 0) = Zn.cv(i, j, k, 0);
        const double ri = 1.0 / Zn.cv(i, j, k, 0);
        Zn.bv(i, j, k, 1) = Zn.cv(i, j, k, 1) * ri;
        Zn.bv(i, j, k, 2) = Zn.cv(i, j, k, 2) * ri;
        Zn.bv(i, j, k, 3) = Zn.cv(i, j, k, 3) * ri;
        double vel = Zn.bv(i, j, k, 1) * Zn.bv(i, j, k, 1) + Zn.bv(i, j, k, 2) * Zn.bv(i, j, k, 2) +
                     Zn.bv(i, j, k, 3) * Zn.bv(i, j, k, 3);
        for (int l = 0; l < P->n_scalar; ++l) Zn.sv(i, j, k, l) = Zn.cv(i, j, k, 5 + l) * ri;
        if (P->mix_model != OSTC_MIX_AIR) {
          temperature_and_pressure(P, Zn, i, j, k, Zn.cv(i, j, k, 4));
        } else {
          Zn.bv(i, j, k, 4) = (gamma_air - 1) * (Zn.cv(i, j, k, 4) - 0.5 * Zn.bv(i, j, k, 0) * vel);
          Zn.bv(i, j, k, 5) = Zn.bv(i, j, k, 4) * mw_air * ri / R_u;
        }
        Zn.vel(i, j, k) = std::sqrt(vel);
      }
  return 0;
}

int oracle_apply_boundary_conditions(const ostc_param *P, ostc_zone *zones, int n_zones,
                                     const ostc_bc_face *f, int n_faces, int with_cv) {
  // priority order of BoundCond.cuh:673-822: farfield, outflow, back pressure,
  // inflow, subsonic inflow, symmetry, wall; periodic wraps last.
  static const int order[] = {OSTC_BC_FARFIELD, OSTC_BC_OUTFLOW, OSTC_BC_BACK_PRESSURE, OSTC_BC_INFLOW,
                              OSTC_BC_SUBSONIC_INFLOW, OSTC_BC_SYMMETRY, OSTC_BC_WALL, OSTC_BC_PERIODIC};
  for (int t : order) {
    for (int q = 0; q < n_faces; ++q) {
      if (f[q].type_label != t) continue;
      if (f[q].block < 0 || f[q].block >= n_zones) return OSTC_ERR_INVALID_ARG;
      Z Zn(&zones[f[q].block]);
      switch (t) {
        case OSTC_BC_OUTFLOW: bc_outflow(P, Zn, f[q], with_cv); break;
        case OSTC_BC_INFLOW: bc_inflow(P, Zn, f[q], with_cv); break;
        case OSTC_BC_SYMMETRY: bc_symmetry(P, Zn, f[q]); break;  // ignores with_cv (quirk A5)
        case OSTC_BC_PERIODIC: bc_periodic(P, Zn, f[q], with_cv); break;
        case OSTC_BC_WALL: bc_wall(P, Zn, f[q], with_cv); break;
        case OSTC_BC_FARFIELD: bc_farfield(P, Zn, f[q]); break;
        case OSTC_BC_BACK_PRESSURE: bc_back_pressure(P, Zn, f[q], with_cv); break;
        case OSTC_BC_SUBSONIC_INFLOW: bc_subsonic_inflow(P, Zn, f[q], with_cv); break;
      }
    }
  }

  return 0;
}

int oracle_set_interfaces(const ostc_interface *f, int n) {
  g_ifaces.assign(f, f + (n > 0 ? n : 0));
  return 0;
}

int oracle_data_communication(const ostc_param *P, ostc_zone *zones, int n_zones, int with_cv) {
  for (int b = 0; b < n_zones; ++b)
    for (const auto &f : g_ifaces) {
      if (f.block != b) continue;
      if (f.target < 0 || f.target >= n_zones) return OSTC_ERR_INVALID_ARG;
      Z Zs(&zones[b]), Zt(&zones[f.target]);
      interface_exchange(P, Zs, Zt, f, with_cv);
    }
  return 0;
}

// eliminate_k_gradient (FieldOperation.cuh:372-400) on a 2-D block (mz == 1):
// the k ghost planes of bv, sv (and cv) copy the plane k = 0 over the whole
// ghosted (i, j) range
int oracle_eliminate_k_gradient(const ostc_param *P, ostc_zone *z, int with_cv) {
  Z Zn(z);
  if (Zn.mz != 1) return 0;
  const int g = Zn.ngg;
  for (int j = -g; j < Zn.my + g; ++j)
    for (int i = -g; i < Zn.mx + g; ++i)
      for (int k = 1; k <= g; ++k) {
        for (int l = 0; l < 6; ++l) Zn.bv(i, j, k, l) = Zn.bv(i, j, -k, l) = Zn.bv(i, j, 0, l);
        for (int l = 0; l < P->n_scalar; ++l) Zn.sv(i, j, k, l) = Zn.sv(i, j, -k, l) = Zn.sv(i, j, 0, l);
        if (with_cv)
          for (int l = 0; l < P->n_var; ++l) Zn.cv(i, j, k, l) = Zn.cv(i, j, -k, l) = Zn.cv(i, j, 0, l);
      }
  return 0;
}

int oracle_update_physical_properties(const ostc_param *P, ostc_zone *z) {
  Z Zn(z);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = -1; k <= Zn.mz; ++k)
    for (int j = -1; j <= Zn.my; ++j)
      for (int i = -1; i <= Zn.mx; ++i) properties_point(P, Zn, i, j, k);
  return 0;
}

int oracle_initialize(const ostc_config *c, const ostc_param *P, ostc_zone *zones, int n_zones,
                      const ostc_bc_face *f, int n_faces) {
  (void)c;
  // Driver::initialize_computation (Driver.cu:39-98): on 2-D blocks the k
  // ghost planes first, BCs without cv, velocity everywhere, interfaces,
  // properties; then RK3_bv pre-loop (RK.cuh:40-49).
  for (int b = 0; b < n_zones; ++b) oracle_eliminate_k_gradient(P, &zones[b], 0);
  int st = oracle_apply_boundary_conditions(P, zones, n_zones, f, n_faces, 0);
  if (st) return st;
  for (int b = 0; b < n_zones; ++b) {
    Z Zn(&zones[b]);
    const int g = Zn.ngg;
    for (int k = -g; k < Zn.mz + g; ++k)
      for (int j = -g; j < Zn.my + g; ++j)
        for (int i = -g; i < Zn.mx + g; ++i)
          Zn.vel(i, j, k) = std::sqrt(Zn.bv(i, j, k, 1) * Zn.bv(i, j, k, 1) + Zn.bv(i, j, k, 2) * Zn.bv(i, j, k, 2) +
                                      Zn.bv(i, j, k, 3) * Zn.bv(i, j, k, 3));
    if (is_sst(P))  // initialize_mut over [-1, m] (FieldOperation.cuh:175-195)
      for (int k = -1; k <= Zn.mz; ++k)
        for (int j = -1; j <= Zn.my; ++j)
          for (int i = -1; i <= Zn.mx; ++i) {
            // Sutherland's viscosity for air, the mixture's (compute_viscosity) with species
            double Y[MAXS];
            for (int l = 0; l < P->n_spec; ++l) Y[l] = Zn.sv(i, j, k, l);
            const double T = Zn.bv(i, j, k, 5);
            const double mul = P->n_spec > 0 ? mixture_viscosity(P, T, Y) : sutherland(T);
            Zn.mut(i, j, k) = sst::compute_mut(Zn, P->n_spec, i, j, k, mul);
          }
  }
  oracle_data_communication(P, zones, n_zones, 0);
  for (int b = 0; b < n_zones; ++b) oracle_update_physical_properties(P, &zones[b]);
  for (int b = 0; b < n_zones; ++b) oracle_compute_cv_from_bv(P, &zones[b]);
  return 0;
}

int oracle_rk3_steps(const ostc_config *c, const ostc_param *P, ostc_zone *zones, int n_zones,
                     const ostc_bc_face *f, int n_faces, int n_steps, double *res_hist, double *dt_hist) {
  if (c->chem_mode == 2) return OSTC_ERR_UNSUPPORTED;  // the oracle checks the surrogate through chem_mode 1
  struct SkipGuard {
    explicit SkipGuard(bool on) { g_skip_source = on; }
    ~SkipGuard() { g_skip_source = false; }
  } guard(c->chem_mode != 0);
  for (int step = 0; step < n_steps; ++step) {
    long n_total = 0;
    std::vector<std::vector<double>> last(n_zones);
    for (int b = 0; b < n_zones; ++b) {  // store_last_step (TimeAdvanceFunc.cu:6-17)
      Z Zn(&zones[b]);
      const long n = (long)Zn.mx * Zn.my * Zn.mz;
      n_total += n;
      last[b].resize(4 * n);
      long q = 0;
      for (int k = 0; k < Zn.mz; ++k)
        for (int j = 0; j < Zn.my; ++j)
          for (int i = 0; i < Zn.mx; ++i, ++q) {
            last[b][q] = Zn.bv(i, j, k, 0);
            last[b][q + n] = Zn.vel(i, j, k);
            last[b][q + 2 * n] = Zn.bv(i, j, k, 4);
            last[b][q + 3 * n] = Zn.bv(i, j, k, 5);
          }
      // qn <- cv over the whole ghosted array (RK.cuh:101-104)
      std::memcpy(Zn.qn.p, Zn.cv.p, sizeof(double) * Zn.cv.sz * P->n_var);
    }
    double dt = c->dt;
    for (int rk = 0; rk < 3; ++rk) {
      for (int b = 0; b < n_zones; ++b) {
        int st = oracle_compute_rhs(P, &zones[b]);
        if (st) return st;
      }
      if (!c->fixed_time_step) dt = oracle_global_time_step(P, zones, n_zones);
      for (int b = 0; b < n_zones; ++b) oracle_update_cv_and_bv_rk(P, &zones[b], dt, rk);
      int st = oracle_apply_boundary_conditions(P, zones, n_zones, f, n_faces, 1);
      if (st) return st;
      oracle_data_communication(P, zones, n_zones, 1);
      for (int b = 0; b < n_zones; ++b) oracle_eliminate_k_gradient(P, &zones[b], 1);  // 2-D (RK.cuh:147-153)
      for (int b = 0; b < n_zones; ++b) oracle_update_physical_properties(P, &zones[b]);
    }
    if (c->chem_mode == 1) {
      // operator-split chemistry: the point-implicit integrator over the step's dt
      // at constant density and internal energy, then BCs, interfaces, properties
      for (int b = 0; b < n_zones; ++b) {
        Z Zn(&zones[b]);
        const int ns = P->n_spec;
        const long n = (long)Zn.mx * Zn.my * Zn.mz;
        std::vector<double> T(n), p(n), Y(ns * n), dts(n, dt), dY(ns * n), dT(n);
        long q = 0;
        for (int k = 0; k < Zn.mz; ++k)
          for (int j = 0; j < Zn.my; ++j)
            for (int i = 0; i < Zn.mx; ++i, ++q) {
              T[q] = Zn.bv(i, j, k, 5);
              p[q] = Zn.bv(i, j, k, 4);
              for (int l = 0; l < ns; ++l) Y[l * n + q] = Zn.sv(i, j, k, l);
            }
        oracle_chem_point_implicit(P, (int)n, T.data(), p.data(), Y.data(), dts.data(), dY.data(), dT.data());
        q = 0;
        for (int k = 0; k < Zn.mz; ++k)
          for (int j = 0; j < Zn.my; ++j)
            for (int i = 0; i < Zn.mx; ++i, ++q) {
              const double rho = Zn.bv(i, j, k, 0);
              double mwinv = 0;
              for (int l = 0; l < ns; ++l) {
                const double y = Zn.sv(i, j, k, l) + dY[l * n + q];
                Zn.sv(i, j, k, l) = y;
                Zn.cv(i, j, k, 5 + l) = rho * y;
                mwinv += y / P->mw[l];
              }
              const double t = Zn.bv(i, j, k, 5) + dT[q];
              Zn.bv(i, j, k, 5) = t;
              Zn.bv(i, j, k, 4) = rho * R_u * mwinv * t;
            }
      }
      int st = oracle_apply_boundary_conditions(P, zones, n_zones, f, n_faces, 1);
      if (st) return st;
      oracle_data_communication(P, zones, n_zones, 1);
      for (int b = 0; b < n_zones; ++b) oracle_eliminate_k_gradient(P, &zones[b], 1);  // 2-D (RK.cuh:147-153)
      for (int b = 0; b < n_zones; ++b) oracle_update_physical_properties(P, &zones[b]);
    }
    if (dt_hist) dt_hist[step] = dt;
    if (res_hist) {  // compute_square_of_dbv + reductions (Residual.cuh:57-111)
      double res[4] = {0, 0, 0, 0};
      for (int b = 0; b < n_zones; ++b) {
        Z Zn(&zones[b]);
        const long n = (long)Zn.mx * Zn.my * Zn.mz;
        long q = 0;
        for (int k = 0; k < Zn.mz; ++k)
          for (int j = 0; j < Zn.my; ++j)
            for (int i = 0; i < Zn.mx; ++i, ++q) {
              const double d0 = Zn.bv(i, j, k, 0) - last[b][q];
              const double d1 = Zn.vel(i, j, k) - last[b][q + n];
              const double d2 = Zn.bv(i, j, k, 4) - last[b][q + 2 * n];
              const double d3 = Zn.bv(i, j, k, 5) - last[b][q + 3 * n];
              res[0] += d0 * d0;
              res[1] += d1 * d1;
              res[2] += d2 * d2;
              res[3] += d3 * d3;
            }
      }
      for (int l = 0; l < 4; ++l) res_hist[4 * step + l] = std::sqrt(res[l] / (double)n_total);
    }
  }
  return 0;
}


int oracle_steady_steps(const ostc_config *c, const ostc_param *P, ostc_zone *zones, int n_zones,
                        const ostc_bc_face *f, int n_faces, int n_steps, double *res_hist) {
  // the loop body of steady_simulation (SteadySim.cuh:51-126)
  if (P->inviscid_type == 1) return OSTC_ERR_UNSUPPORTED;  // quirk A6
  for (int step = 0; step < n_steps; ++step) {
    long n_total = 0;
    std::vector<std::vector<double>> last(n_zones);
    if (res_hist)
      for (int b = 0; b < n_zones; ++b) {  // store_last_step (TimeAdvanceFunc.cu:6-17)
        Z Zn(&zones[b]);
        const long n = (long)Zn.mx * Zn.my * Zn.mz;
        n_total += n;
        last[b].resize(4 * n);
        long q = 0;
        for (int k = 0; k < Zn.mz; ++k)
          for (int j = 0; j < Zn.my; ++j)
            for (int i = 0; i < Zn.mx; ++i, ++q) {
              last[b][q] = Zn.bv(i, j, k, 0);
              last[b][q + n] = Zn.vel(i, j, k);
              last[b][q + 2 * n] = Zn.bv(i, j, k, 4);
              last[b][q + 3 * n] = Zn.bv(i, j, k, 5);
            }
      }
    for (int b = 0; b < n_zones; ++b) {
      int st = oracle_compute_rhs(P, &zones[b]);
      if (st) return st;
      Z Zn(&zones[b]);
      std::vector<double> isr;
      local_time_step_zone(P, Zn, isr);
      if (c->implicit_method == 1) {
        dplur_zone(c, P, Zn, isr, f, n_faces, b);
      } else {
        if (P->mix_model == OSTC_MIX_FR && P->n_reac > 0 && P->chemSrcMethod != 0) chem_implicit_zone(P, Zn);
        if (is_sst(P) && P->turb_implicit == 1) {  // implicit_treat_for_SST (SST.cu:8-22)
          for (int k = 0; k < Zn.mz; ++k)
            for (int j = 0; j < Zn.my; ++j)
              for (int i = 0; i < Zn.mx; ++i) {
                const double dt = Zn.dt_local(i, j, k);
                Zn.dq(i, j, k, P->i_turb_cv) /= 1 - dt * Zn.tsj(i, j, k, 0);
                Zn.dq(i, j, k, P->i_turb_cv + 1) /= 1 - dt * Zn.tsj(i, j, k, 1);
              }
        }
      }
      update_bv_zone(P, Zn);
    }
    int st = oracle_apply_boundary_conditions(P, zones, n_zones, f, n_faces, 0);
    if (st) return st;
    oracle_data_communication(P, zones, n_zones, 0);
    for (int b = 0; b < n_zones; ++b) oracle_eliminate_k_gradient(P, &zones[b], 0);  // 2-D (SteadySim.cuh:101-107)
    for (int b = 0; b < n_zones; ++b) oracle_update_physical_properties(P, &zones[b]);
    if (res_hist) {
      double res[4] = {0, 0, 0, 0};
      for (int b = 0; b < n_zones; ++b) {
        Z Zn(&zones[b]);
        const long n = (long)Zn.mx * Zn.my * Zn.mz;
        long q = 0;
        for (int k = 0; k < Zn.mz; ++k)
          for (int j = 0; j < Zn.my; ++j)
            for (int i = 0; i < Zn.mx; ++i, ++q) {
              const double d0 = Zn.bv(i, j, k, 0) - last[b][q];
              const double d1 = Zn.vel(i, j, k) - last[b][q + n];
              const double d2 = Zn.bv(i, j, k, 4) - last[b][q + 2 * n];
              const double d3 = Zn.bv(i, j, k, 5) - last[b][q + 3 * n];
              res[0] += d0 * d0;
              res[1] += d1 * d1;
              res[2] += d2 * d2;
              res[3] += d3 * d3;
            }
      }
      for (int l = 0; l < 4; ++l) res_hist[4 * step + l] = std::sqrt(res[l] / (double)n_total);
    }
  }
  return 0;
}


int oracle_chem_point_implicit(const ostc_param *P, int n, const double *T, const double *p, const double *Y,
                               const double *dt, double *dY, double *dT) {
  // the point-implicit chemistry integrator of ostc_chem_point_implicit:
  // omega and J (FiniteRateChem.cu:7-216), the LU solve of solve_chem_system
  // (FiniteRateChem.cu:324-419), T' at constant e by the Newton update of
  // compute_temperature_and_pressure (FieldOperation.cu:3-39) run to 1e-13
  if (P->mix_model != OSTC_MIX_FR || P->n_reac <= 0) return OSTC_ERR_INVALID_ARG;
  const int ns = P->n_spec;
#pragma omp parallel for schedule(static)
  for (int q = 0; q < n; ++q) {
    double y[MAXS], mwinv = 0;
    for (int l = 0; l < ns; ++l) {
      y[l] = Y[(long)l * n + q];
      mwinv += y[l] / P->mw[l];
    }
    const double rho = p[q] / (R_u * T[q] * mwinv);
    double om[MAXS], q1[MAXR], q2[MAXR], od[MAXS], J[MAXS * MAXS], b[MAXS];
    int ipiv[MAXS];
    chemistry_omega(P, rho, T[q], y, om, q1, q2, od);
    chem_jacobian(P, rho, y, q1, q2, J);
    for (int m = 0; m < ns; ++m)
      for (int c = 0; c < ns; ++c) J[m * ns + c] = m == c ? 1.0 - dt[q] * J[m * ns + c] : -dt[q] * J[m * ns + c];
    for (int l = 0; l < ns; ++l) b[l] = dt[q] * om[l];
    lu_factor(J, ipiv, ns);
    lu_apply(J, ipiv, b, ns);
    double y1[MAXS], h[MAXS], cp[MAXS], e0 = 0, mwinv1 = 0;
    enthalpy(P, T[q], h);
    for (int l = 0; l < ns; ++l) {
      dY[(long)l * n + q] = b[l] / rho;
      y1[l] = y[l] + b[l] / rho;
      e0 += y[l] * h[l];
      mwinv1 += y1[l] / P->mw[l];
    }
    e0 -= R_u * T[q] * mwinv;
    const double R1 = R_u * mwinv1;
    double t = T[q];
    bool ok = false;
    for (int it = 1; it <= 100; ++it) {
      enthalpy_and_cp(P, t, h, cp);
      double hs = 0, cps = 0;
      for (int l = 0; l < ns; ++l) {
        hs += y1[l] * h[l];
        cps += y1[l] * cp[l];
      }
      const double t1 = t - (hs - R1 * t - e0) / (cps - R1);
      const double err = std::abs(1 - t1 / t);
      t = t1;
      if (err <= 1e-13) {
        ok = true;
        break;
      }
    }
    dT[q] = ok ? t - T[q] : std::numeric_limits<double>::quiet_NaN();
  }
  return 0;
}

int oracle_chemical_source(const ostc_param *P, double rho, double T, const double *Y, double *omega) {
  chemistry_omega(P, rho, T, Y, omega, nullptr, nullptr);
  return 0;
}

int oracle_enthalpy_cp(const ostc_param *P, double T, double *h, double *cp) {
  enthalpy_and_cp(P, T, h, cp);
  return 0;
}

int oracle_transport(const ostc_param *P, double rho, double p_, double T, const double *Y, double *mu,
                     double *kappa, double *rhoD) {
  double cp[MAXS], mw = 0;
  cp_only(P, T, cp);
  for (int l = 0; l < P->n_spec; ++l) mw += Y[l] / P->mw[l];
  mw = 1 / mw;
  transport(P, T, mw, Y, cp, rho, p_, mu, kappa, rhoD);
  return 0;
}

}  // extern "C"
