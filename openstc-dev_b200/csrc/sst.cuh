// sst.cuh — Menter k-omega SST on the device: turbulent viscosity, the k and
// omega source terms with the optional compressibility corrections
// (SST.cu:8-247, SST.cuh:12-45), the turbulent parts of the viscous face
// flux (ViscousScheme.cuh:82-95, 111-113, 200-251) and of the wall boundary
// (BoundCond.cuh:471-484, 536-541). NS species before them: sv holds k and
// omega in its planes NS and NS + 1, dq and cv in their planes 5 + NS and
// 6 + NS (i_turb_cv, DParameter.cu).
#pragma once
#include "common.cuh"

namespace ostc {
namespace sst {

constexpr double beta_star = 0.09, sqrt_beta_star = 0.3, kappa = 0.41;
constexpr double sigma_k1 = 0.85, sigma_omega1 = 0.5, beta_1 = 0.0750, a_1 = 0.31;
constexpr double gamma1 = beta_1 / beta_star - sigma_omega1 * kappa * kappa / sqrt_beta_star;
constexpr double sigma_k2 = 1, sigma_omega2 = 0.856, beta_2 = 0.0828;
constexpr double gamma2 = beta_2 / beta_star - sigma_omega2 * kappa * kappa / sqrt_beta_star;
constexpr double delta_sigma_k = sigma_k1 - sigma_k2, delta_sigma_omega = sigma_omega1 - sigma_omega2;
constexpr double delta_beta = beta_1 - beta_2, delta_gamma = gamma1 - gamma2;

// Wilcox (SST.cu:24-31) and Zeman (SST.cu:33-42) corrections of beta*
__device__ __forceinline__ double wilcox(double Mt) {
  constexpr double Mt0 = 0.25;
  return Mt - Mt0 > 0 ? beta_star * 2 * (Mt * Mt - Mt0 * Mt0) : 0.0;
}
__device__ __forceinline__ double zeman(double Mt, double gammaP1) {
  const double Mt0 = 0.25 * sqrt(2.0 / gammaP1);
  const double DMt = Mt - Mt0;
  if (DMt > 0) {
    constexpr double Lambda2 = 0.66 * 0.66;
    const double F_Mt = 1 - exp(-0.5 * gammaP1 * DMt * DMt / Lambda2);
    return beta_star * 0.75 * F_Mt;
  }
  return 0.0;
}

// central difference 0.5 * (xi_c d_xi + eta_c d_eta + zeta_c d_zeta) of a
// plane at point g (the gradient form of SST.cu:52-69); m = the point's metric
struct Grad {
  double dxi, deta, dzeta;
  __device__ __forceinline__ double c(const double *m, int comp) const {
    return 0.5 * (m[comp] * dxi + m[3 + comp] * deta + m[6 + comp] * dzeta);
  }
};
__device__ __forceinline__ Grad diffs(const DevZone &z, const double *base, int g) {
  return {base[g + 1] - base[g - 1], base[g + z.d2] - base[g - z.d2], base[g + z.d1] - base[g - z.d1]};
}

// SST::compute_mut (SST.cu:44-97): the initial turbulent viscosity of a point
template <int NS>
__device__ __forceinline__ double mut_point(const DevZone &z, int g, double mul) {
  double m[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) m[c] = z.met[c * z.sz + g];
  const Grad gu = diffs(z, z.bv + z.sz, g), gv = diffs(z, z.bv + 2 * z.sz, g), gw = diffs(z, z.bv + 3 * z.sz, g);
  const double u_y = gu.c(m, 1), u_z = gu.c(m, 2);
  const double v_x = gv.c(m, 0), v_z = gv.c(m, 2);
  const double w_x = gw.c(m, 0), w_y = gw.c(m, 1);
  const double density = z.bv[g];
  const double tke = z.sv[NS * z.sz + g];
  const double rhoK = density * tke;
  const double omega = z.sv[(NS + 1) * z.sz + g];
  const double vorticity = sqrt((v_x - u_y) * (v_x - u_y) + (w_x - u_z) * (w_x - u_z) + (w_y - v_z) * (w_y - v_z));
  double f2 = 1;
  const double dy = z.wall[g];
  if (dy > 1e-25) {
    const double param1 = 2 * sqrt(tke) / (0.09 * omega * dy);
    const double param2 = 500 * mul / (density * dy * dy * omega);
    const double arg2 = fmax(param1, param2);
    f2 = tanh(arg2 * arg2);
  }
  double mut = 0;
  const double denominator = fmax(a_1 * omega, vorticity * f2);
  if (denominator > 1e-25) mut = a_1 * rhoK / denominator;
  return mut;
}

// SST::compute_source_and_mut (SST.cu:99-247) at interior point g: mut, the k
// and omega sources (zero when mut <= 1e-25) and the diagonal source Jacobian
// (-2 beta* omega, -2 beta omega) the steady path's implicit treatment uses
template <int NS>
__device__ __forceinline__ void source_point(const DevZone &z, int g, double &mut_out, double &src_k,
                                             double &src_w, double &jac_k, double &jac_w) {
  double m[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) m[c] = z.met[c * z.sz + g];
  const Grad gu = diffs(z, z.bv + z.sz, g), gv = diffs(z, z.bv + 2 * z.sz, g), gw = diffs(z, z.bv + 3 * z.sz, g);
  const double u_x = gu.c(m, 0), u_y = gu.c(m, 1), u_z = gu.c(m, 2);
  const double v_x = gv.c(m, 0), v_y = gv.c(m, 1), v_z = gv.c(m, 2);
  const double w_x = gw.c(m, 0), w_y = gw.c(m, 1), w_z = gw.c(m, 2);
  const double density = z.bv[g];
  const double omega = z.sv[(NS + 1) * z.sz + g];
  const Grad gk = diffs(z, z.sv + NS * z.sz, g), go = diffs(z, z.sv + (NS + 1) * z.sz, g);
  const double k_x = gk.c(m, 0), k_y = gk.c(m, 1), k_z = gk.c(m, 2);
  const double omega_x = go.c(m, 0), omega_y = go.c(m, 1), omega_z = go.c(m, 2);
  const double inter_var = 2 * density * sigma_omega2 / omega * (k_x * omega_x + k_y * omega_y + k_z * omega_z);
  const double tke = z.sv[NS * z.sz + g];
  const double rhoK = density * tke;
  const double vorticity = sqrt((v_x - u_y) * (v_x - u_y) + (w_x - u_z) * (w_x - u_z) + (w_y - v_z) * (w_y - v_z));
  double f1 = 1, f2 = 1;
  const double dy = z.wall[g];
  if (dy > 1e-25) {
    const double param1 = sqrt(tke) / (0.09 * omega * dy);
    const double d2 = dy * dy;
    const double param2 = 500 * z.mul[g] / (density * d2 * omega);
    const double arg2 = fmax(2 * param1, param2);
    f2 = tanh(arg2 * arg2);
    const double CDkomega = fmax(1e-20, inter_var);
    const double param3 = 4 * density * sigma_omega2 * tke / (CDkomega * d2);
    const double arg1 = fmin(fmax(param1, param2), param3);
    f1 = tanh(arg1 * arg1 * arg1 * arg1);
  }
  double mut = 0;
  const double denominator = fmax(a_1 * omega, vorticity * f2);
  if (denominator > 1e-25) mut = a_1 * rhoK / denominator;
  mut_out = mut;
  double beta = beta_2 + delta_beta * f1;
  double betaStar = beta_star;
  if (c_p.comp_corr) {  // the mixture's gamma when there are species (SST.cu:195-199)
    const double gam = NS > 0 ? z.gam[g] : gamma_air;
    const double Mt = sqrt(2 * tke / (gam * z.bv[4 * z.sz + g] / density));
    double corr;
    switch (c_p.comp_corr) {
      case 1: corr = wilcox(Mt); break;
      case 2: corr = beta_star * Mt * Mt; break;
      default: corr = zeman(Mt, gam + 1.0); break;
    }
    betaStar += corr;
    beta -= corr;
  }
  jac_k = -2 * betaStar * omega;
  jac_w = -2 * beta * omega;
  src_k = 0;
  src_w = 0;
  if (mut > 1e-25) {
    const double divU = u_x + v_y + w_z;
    const double divU2 = divU * divU;
    double prod_k = mut * (2 * (u_x * u_x + v_y * v_y + w_z * w_z) - 2.0 / 3 * divU2 + (u_y + v_x) * (u_y + v_x) +
                           (u_z + w_x) * (u_z + w_x) + (v_z + w_y) * (v_z + w_y)) -
                    2.0 / 3 * rhoK * divU;
    const double prod_k2 = mut * vorticity * vorticity;
    if (prod_k > 10 * prod_k2) prod_k = prod_k2;
    const double diss_k = betaStar * rhoK * omega;
    const double jac = z.jac[g];
    src_k = jac * (prod_k - diss_k);
    const double gamma = gamma2 + delta_gamma * f1;
    const double prod_omega = gamma * density / mut * prod_k + (1 - f1) * inter_var;
    const double diss_omega = beta * density * omega * omega;
    src_w = jac * (prod_omega - diss_omega);
  }
}

}  // namespace sst
}  // namespace ostc
