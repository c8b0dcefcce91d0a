// face.cuh — per-face inviscid and viscous fluxes and the per-cell AWENO
// central correction, as device functions of one thread.
//
// A face of direction DIR lies between the cell at ghosted index gi and the
// cell at gi + sd (sd = the stride along DIR). The primitive and scalar values
// of the face's stencil come through a cell accessor: PlaneCells reads the
// ColMajor planes through the read-only path (threads of a warp always differ
// in i, so every load is a coalesced 32-wide row); TileCells reads the cells
// of the CTA's sweep plane from its shared-memory tile and only the cells
// across that plane from HBM. Metrics and transport properties are read from
// the planes in both cases.
#pragma once
#include "common.cuh"
#include "sst.cuh"
#include "thermo.cuh"

namespace ostc {

template <int DIR>
__device__ __forceinline__ int dir_stride(const DevZone &z) {
  return DIR == 0 ? 1 : (DIR == 1 ? z.d2 : z.d1);
}

__device__ __forceinline__ double bvl(const DevZone &z, int g, int l) { return ld(z.bv + l * z.isz + g); }
__device__ __forceinline__ double svl(const DevZone &z, int g, int l) { return ld(z.sv + l * z.isz + g); }
__device__ __forceinline__ double cvl(const DevZone &z, int g, int l) { return ld(z.cv + l * z.isz + g); }
__device__ __forceinline__ double met(const DevZone &z, int g, int c) { return ld(z.met + c * z.isz + g); }

// Cell accessors of one face: bv(l, n, a, b) / sv(l, n, a, b) is plane l at
// n steps along the face normal (n = 0: the cell before the face, 1: the cell
// after it) and a, b steps along the face's two tangential directions (TA,
// TB of viscous_face: for the x sweep a = j, b = k; for y, a = i, b = k; for
// z, a = i, b = j). Every call site passes literal steps, so the tile
// accessor's choice between shared memory and HBM is resolved at compile time.
struct PlaneCells {
  const double *bvp, *svp, *metp, *jacp, *mulp, *kappap, *rhodp, *mutp, *ttcp, *wallp;
  int isz, g0, sn, sa, sb;
  // the cell's index: the face's first cell, then the step along the normal,
  // then the tangential step
  __device__ __forceinline__ double at(const double *plane, int n, int a, int b) const {
    const double *q = plane + (g0 + n * sn);
    return ld(a != 0 ? q + a * sa : (b != 0 ? q + b * sb : q));
  }
  __device__ __forceinline__ double bv(int l, int n, int a = 0, int b = 0) const {
    return at(bvp + l * isz, n, a, b);
  }
  __device__ __forceinline__ double sv(int l, int n, int a = 0, int b = 0) const {
    return at(svp + l * isz, n, a, b);
  }
  // metric, Jacobian and transport properties of the face's cells n = 0, 1
  __device__ __forceinline__ double met(int c, int n) const { return ld(metp + c * isz + (g0 + n * sn)); }
  __device__ __forceinline__ double jac(int n) const { return ld(jacp + (g0 + n * sn)); }
  __device__ __forceinline__ double mul(int n) const { return ld(mulp + (g0 + n * sn)); }
  __device__ __forceinline__ double kappa(int n) const { return ld(kappap + (g0 + n * sn)); }
  __device__ __forceinline__ double rhod(int l, int n) const { return ld(rhodp + l * isz + (g0 + n * sn)); }
  __device__ __forceinline__ double mut(int n) const { return ld(mutp + (g0 + n * sn)); }
  __device__ __forceinline__ double ttc(int n) const { return ld(ttcp + (g0 + n * sn)); }
  __device__ __forceinline__ double wall(int n) const { return ld(wallp + (g0 + n * sn)); }
};

template <int DIR>
__device__ __forceinline__ PlaneCells plane_cells(const DevZone &z, int g0) {
  // tangential strides: TA = j for the x sweep, else i; TB = j for the z sweep, else k
  const int sa = DIR == 0 ? z.d2 : 1;
  const int sb = DIR == 2 ? z.d2 : z.d1;
  return PlaneCells{z.bv,   z.sv,  z.met, z.jac, z.mul, z.kappa, z.rhoD, z.mut, z.ttc, z.wall,
                    z.isz, g0,    dir_stride<DIR>(z),  sa,    sb};
}

// The state tile holds, for the CTA's sweep plane (b = 0), bv planes 0..5 then
// the sv planes, each as a [row][column] array: t points at the thread's own
// cell of plane 0, TN / TA are the tile strides of one step along n / a, TV
// the tile stride of one plane (compile-time, so every tile read is one
// shared-memory load at a constant offset from t); cells across the plane
// (b != 0) come from HBM. The cell tile holds the metric, Jacobian and
// transport planes of the faces' own cells (QN: stride of one step along n,
// QV: stride of one plane), in the order of StagedPlanes.
enum StagedPlanes { Q_MET = 0, Q_JAC = 9, Q_MUL = 10, Q_KAPPA = 11, Q_MUT = 12, Q_TTC = 13, Q_WALL = 14 };
template <int NT>
constexpr int q_rhod() { return NT > 0 ? 15 : 12; }  // first rhoD plane

template <int TN, int TA, int TV, int QN, int QV, int RD>
struct TileCells {
  PlaneCells p;
  const double *t, *q;
  __device__ __forceinline__ double bv(int l, int n, int a = 0, int b = 0) const {
    return b != 0 ? p.bv(l, n, a, b) : t[l * TV + n * TN + a * TA];
  }
  __device__ __forceinline__ double sv(int l, int n, int a = 0, int b = 0) const {
    return b != 0 ? p.sv(l, n, a, b) : t[(6 + l) * TV + n * TN + a * TA];
  }
  __device__ __forceinline__ double met(int c, int n) const { return q[(Q_MET + c) * QV + n * QN]; }
  __device__ __forceinline__ double jac(int n) const { return q[Q_JAC * QV + n * QN]; }
  __device__ __forceinline__ double mul(int n) const { return q[Q_MUL * QV + n * QN]; }
  __device__ __forceinline__ double kappa(int n) const { return q[Q_KAPPA * QV + n * QN]; }
  __device__ __forceinline__ double rhod(int l, int n) const { return q[(RD + l) * QV + n * QN]; }
  __device__ __forceinline__ double mut(int n) const { return q[Q_MUT * QV + n * QN]; }
  __device__ __forceinline__ double ttc(int n) const { return q[Q_TTC * QV + n * QN]; }
  __device__ __forceinline__ double wall(int n) const { return q[Q_WALL * QV + n * QN]; }
};

// 0.5 * (sgn(a) + sgn(b)) * min(|a|, |b|) with sgn(x) = (x < 0 ? -1 : 1)
// (Limiter.cuh:13-16), written without the integer sum and its conversion:
// the product is exactly +m, -m or +0, so the result is bit-identical;
// symmetric in a and b
__device__ __forceinline__ double minmod(double a, double b) {
  const double m = fmin(fabs(a), fabs(b));
  const bool na = a < 0, nb = b < 0;
  return na != nb ? 0.0 : (na ? -m : m);
}

// ---------------------------------------------------------------------------
// Riemann solvers on reconstructed states (pl/pr: NV primitive values, then
// total energy at NV and gamma at NV+1). Output: NV face fluxes.
// ---------------------------------------------------------------------------
// AUSM+ (AusmP.cu:6-94); k1..k3: jac-weighted face metric
template <int NV, bool MIXG>
__device__ __forceinline__ void ausm_plus(const double *pl, const double *pr, double k1, double k2, double k3,
                                          double *F) {
  const double gk = sqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const double ul = (k1 * pl[1] + k2 * pl[2] + k3 * pl[3]) / gk;
  const double ur = (k1 * pr[1] + k2 * pr[2] + k3 * pr[3]) / gk;
  const double gl = MIXG ? pl[NV + 1] : gamma_air, gr = MIXG ? pr[NV + 1] : gamma_air;
  const double c = 0.5 * (sqrt(gl * pl[4] / pl[0]) + sqrt(gr * pr[4] / pr[0]));
  const double mlm = ul / c, mrm = ur / c;
  double mlp, mrn, plp, prn;
  constexpr double alpha = 3 / 16.0;
  if (fabs(mlm) > 1) {
    mlp = 0.5 * (mlm + fabs(mlm));
    plp = mlp / mlm;
  } else {
    const double a = (mlm + 1) * (mlm + 1) * 0.25;
    const double b = (mlm * mlm - 1) * (mlm * mlm - 1);
    mlp = a + 0.125 * b;
    plp = a * (2 - mlm) + alpha * mlm * b;
  }
  if (fabs(mrm) > 1) {
    mrn = 0.5 * (mrm - fabs(mrm));
    prn = mrn / mrm;
  } else {
    const double a = (mrm - 1) * (mrm - 1) * 0.25;
    const double b = (mrm * mrm - 1) * (mrm * mrm - 1);
    mrn = -a - 0.125 * b;
    prn = a * (2 + mrm) - alpha * mrm * b;
  }
  const double pc = plp * pl[4] + prn * pr[4];
  const double mh = mlp + mrn;
  const double mass = c * (pl[0] * 0.5 * (mh + fabs(mh)) + pr[0] * 0.5 * (mh - fabs(mh)));
  const double co = mass * gk;
  const bool left = mass >= 0;
  const double q0 = left ? pl[0] : pr[0], q1 = left ? pl[1] : pr[1], q2 = left ? pl[2] : pr[2];
  const double q3 = left ? pl[3] : pr[3], q4 = left ? pl[4] : pr[4], qe = left ? pl[NV] : pr[NV];
  F[0] = co;
  F[1] = co * q1 + pc * k1;
  F[2] = co * q2 + pc * k2;
  F[3] = co * q3 + pc * k3;
  F[4] = co * (qe + q4) / q0;
#pragma unroll
  for (int l = 5; l < NV; ++l) F[l] = co * (left ? pl[l] : pr[l]);
}

// HLLC (HLLC.cu:10-143); kx..kz: face-averaged metric, jac_ave: face Jacobian
template <int NV, int NS>
__device__ __forceinline__ void hllc(const double *pl, const double *pr, double kx, double ky, double kz,
                                     double jac_ave, double *F) {
  const double sl0 = sqrt(pl[0]), sr0 = sqrt(pr[0]);
  const double rlc = sl0 / (sl0 + sr0), rrc = sr0 / (sl0 + sr0);
  const double ut = pl[1] * rlc + pr[1] * rrc;
  const double vt = pl[2] * rlc + pr[2] * rrc;
  const double wt = pl[3] * rlc + pr[3] * rrc;
  const double hl = (pl[NV] + pl[4]) / pl[0], hr = (pr[NV] + pr[4]) / pr[0];
  const double ht = hl * rlc + hr * rrc;
  const double ekt = 0.5 * (ut * ut + vt * vt + wt * wt);
  double c_tilde;
  if constexpr (NS == 0) {
    c_tilde = sqrt((gamma_air - 1) * (ht - ekt));
  } else {
    double svm[NS], mw_inv = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      svm[l] = rlc * pl[l + 5] + rrc * pr[l + 5];
      mw_inv += svm[l] * c_p.imw[l];
    }
    const double t = (rlc * (pl[4] / pl[0]) + rrc * (pr[4] / pr[0])) / (R_u * mw_inv);
    double h_i[NS], cp_i[NS];
    enthalpy_cp<NS>(t, h_i, cp_i);
    double cvv = 0, cpp = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      cpp += cp_i[l] * svm[l];
      cvv += svm[l] * (cp_i[l] - c_p.Rmw[l]);
    }
    c_tilde = sqrt(cpp / cvv * R_u * mw_inv * t);
  }
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  const double Ub = (kx * ut + ky * vt + kz * wt) / gradK;
  const double gl = NS > 0 ? pl[NV + 1] : gamma_air, gr = NS > 0 ? pr[NV + 1] : gamma_air;
  const double Ul = kx * pl[1] + ky * pl[2] + kz * pl[3];
  const double cl = sqrt(gl * pl[4] / pl[0]);
  const double sl = fmin(Ul / gradK - cl, Ub - c_tilde);
  const double Ur = kx * pr[1] + ky * pr[2] + kz * pr[3];
  const double cr = sqrt(gr * pr[4] / pr[0]);
  const double sr = fmax(Ur / gradK + cr, Ub + c_tilde);
  if (sl >= 0 || sr < 0) {
    const double *q = sl >= 0 ? pl : pr;
    const double U = sl >= 0 ? Ul : Ur;
    const double rhoUk = q[0] * U;
    F[0] = jac_ave * rhoUk;
    F[1] = jac_ave * (rhoUk * q[1] + q[4] * kx);
    F[2] = jac_ave * (rhoUk * q[2] + q[4] * ky);
    F[3] = jac_ave * (rhoUk * q[3] + q[4] * kz);
    F[4] = jac_ave * ((q[NV] + q[4]) * U);
#pragma unroll
    for (int l = 5; l < NV; ++l) F[l] = jac_ave * rhoUk * q[l];
    return;
  }
  const double sm = ((pr[0] * Ur * (sr - Ur / gradK) - pl[0] * Ul * (sl - Ul / gradK)) / gradK + pl[4] - pr[4]) /
                    (pr[0] * (sr - Ur / gradK) - pl[0] * (sl - Ul / gradK));
  const double pm = pl[0] * (sl - Ul / gradK) * (sm - Ul / gradK) + pl[4];
  const bool lft = sm >= 0;
  const double *q = lft ? pl : pr;
  const double s = lft ? sl : sr, U = lft ? Ul : Ur;
  const double pC = 1.0 / (s - sm);
  const double Q = jac_ave * pC * sm * (s * gradK - U) * q[0];
  F[0] = Q;
  const double dP = (s * pm - sm * q[4]) * pC * jac_ave;
  F[1] = Q * q[1] + dP * kx;
  F[2] = Q * q[2] + dP * ky;
  F[3] = Q * q[3] + dP * kz;
  F[4] = Q * q[NV] / q[0] + pC * jac_ave * (s * pm * sm * gradK - sm * q[4] * U);
#pragma unroll
  for (int l = 5; l < NV; ++l) F[l] = Q * q[l];
}

// Lax-Friedrichs, air only (LaxFriedrichs.cu:13-49)
template <int NV>
__device__ __forceinline__ void lax_friedrichs(const double *pl, const double *pr, double kx, double ky, double kz,
                                               double jac_ave, double *F) {
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  const double Ukl = pl[1] * kx + pl[2] * ky + pl[3] * kz;
  const double Ukr = pr[1] * kx + pr[2] * ky + pr[3] * kz;
  const double cl = sqrt(gamma_air * pl[4] / pl[0]), cr = sqrt(gamma_air * pr[4] / pr[0]);
  const double sr = fmax(fabs(Ukl) + cl * gradK, fabs(Ukr) + cr * gradK);
  const double hj = 0.5 * jac_ave;
  const double rUl = pl[0] * Ukl, rUr = pr[0] * Ukr;
  F[0] = (rUl + rUr - sr * (pr[0] - pl[0])) * hj;
  F[1] = (rUl * pl[1] + rUr * pr[1] + kx * (pl[4] + pr[4]) - sr * (pr[1] * pr[0] - pl[1] * pl[0])) * hj;
  F[2] = (rUl * pl[2] + rUr * pr[2] + ky * (pl[4] + pr[4]) - sr * (pr[2] * pr[0] - pl[2] * pl[0])) * hj;
  F[3] = (rUl * pl[3] + rUr * pr[3] + kz * (pl[4] + pr[4]) - sr * (pr[3] * pr[0] - pl[3] * pl[0])) * hj;
  F[4] = ((pl[NV] + pl[4]) * Ukl + (pr[NV] + pr[4]) * Ukr - sr * (pr[NV] - pl[NV])) * hj;
}

// dispatch on the inviscid_scheme tag (InviscidScheme.cu:137-150; Roe -> AUSM+, quirk A1)
template <int NV, int NS, class Cells>
__device__ __forceinline__ void riemann(const double *pl, const double *pr, const Cells &c, int DIR, double *F) {
  const double j0 = c.jac(0), j1 = c.jac(1);
  const double m0x = c.met(3 * DIR, 0), m0y = c.met(3 * DIR + 1, 0), m0z = c.met(3 * DIR + 2, 0);
  const double m1x = c.met(3 * DIR, 1), m1y = c.met(3 * DIR + 1, 1), m1z = c.met(3 * DIR + 2, 1);
  const int sch = c_p.inviscid_scheme;
  if (sch == 4) {
    hllc<NV, NS>(pl, pr, 0.5 * (m0x + m1x), 0.5 * (m0y + m1y), 0.5 * (m0z + m1z), 0.5 * (j0 + j1), F);
  } else if (sch == 1 && NS == 0) {
    lax_friedrichs<NV>(pl, pr, 0.5 * (m0x + m1x), 0.5 * (m0y + m1y), 0.5 * (m0z + m1z), 0.5 * (j0 + j1), F);
  } else {
    ausm_plus<NV, (NS > 0)>(pl, pr, 0.5 * (j0 * m0x + j1 * m1x), 0.5 * (j0 * m0y + j1 * m1y),
                            0.5 * (j0 * m0z + j1 * m1z), F);
  }
}

// ---------------------------------------------------------------------------
// primitive-variable reconstruction face (InviscidScheme.cu:48-158 +
// Reconstruction.cu:5-46 + Reconstruction.cuh:20-72)
// ---------------------------------------------------------------------------
// NT: turbulence scalars (k, omega) after the NS species, reconstructed alike
template <int NS, int NT, class Cells>
__device__ __forceinline__ void reconstruct_pv_c(const Cells &c, double *pl, double *pr) {
  constexpr int NV = 5 + NS + NT;
  const int rec = c_p.reconstruction;
  // variable l of the reconstruction: bv 0..4 (rho, u, v, w, p), then the scalars
  auto val = [&](int l, int n) { return l < 5 ? c.bv(l, n) : c.sv(l - 5, n); };
#pragma unroll
  for (int l = 0; l < NV; ++l) {
    const double v0 = val(l, 0), v1 = val(l, 1);
    if (rec == 2 || rec == 3) {
      const double vm = val(l, -1), v2 = val(l, 2);
      const double di = v0 - vm, di1 = v1 - v0, di2 = v2 - v1;
      if (rec == 2) {
        constexpr double kappa = 1.0 / 3.0;
        const double ml = minmod(di, di1), mr = minmod(di2, di1);  // = minmod(di1, di), minmod(di1, di2)
        pl[l] = v0 + 0.25 * ((1 - kappa) * ml + (1 + kappa) * ml);
        pr[l] = v1 - 0.25 * ((1 - kappa) * mr + (1 + kappa) * mr);
      } else {
        pl[l] = v0 + 0.5 * minmod(di, di1);
        pr[l] = v1 - 0.5 * minmod(di1, di2);
      }
    } else {
      pl[l] = v0;
      pr[l] = v1;
    }
  }
  if constexpr (NS > 0) {
    double el = 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]);
    double er = 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
    double mwl = 0, mwr = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      mwl += pl[5 + l] * c_p.imw[l];
      mwr += pr[5 + l] * c_p.imw[l];
    }
    const double tl = pl[4] / (pl[0] * R_u * mwl), tr = pr[4] / (pr[0] * R_u * mwr);
    double cpl = 0, cpr = 0, cvl = 0, cvr = 0;
    {
      double h[NS], cp[NS];
      enthalpy_cp<NS>(tl, h, cp);
#pragma unroll
      for (int l = 0; l < NS; ++l) {
        cpl += cp[l] * pl[l + 5];
        cvl += pl[l + 5] * (cp[l] - c_p.Rmw[l]);
        el += h[l] * pl[l + 5];
      }
    }
    {
      double h[NS], cp[NS];
      enthalpy_cp<NS>(tr, h, cp);
#pragma unroll
      for (int l = 0; l < NS; ++l) {
        cpr += cp[l] * pr[l + 5];
        cvr += pr[l + 5] * (cp[l] - c_p.Rmw[l]);
        er += h[l] * pr[l + 5];
      }
    }
    pl[NV] = pl[0] * el - pl[4];
    pr[NV] = pr[0] * er - pr[4];
    pl[NV + 1] = cpl / cvl;
    pr[NV + 1] = cpr / cvr;
  } else {
    pl[NV] = 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]) * pl[0] + pl[4] / (gamma_air - 1);
    pr[NV] = 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]) * pr[0] + pr[4] / (gamma_air - 1);
    pl[NV + 1] = gamma_air;
    pr[NV + 1] = gamma_air;
  }
}

template <int NS, int DIR, int NT = 0>
__device__ __forceinline__ void reconstruct_pv(const DevZone &z, int g0, double *pl, double *pr) {
  reconstruct_pv_c<NS, NT>(plane_cells<DIR>(z, g0), pl, pr);
}

template <int NS, int DIR, int NT, class Cells>
__device__ __forceinline__ void inviscid_face_pv(const Cells &c, double *F) {
  constexpr int NV = 5 + NS + NT;
  double pl[NV + 2], pr[NV + 2];
  reconstruct_pv_c<NS, NT>(c, pl, pr);
  riemann<NV, NS>(pl, pr, c, DIR, F);
}

// Harten entropy-fix width at one point (compute_entropy_fix_delta, Roe.cu:61-85): the 3-D
// form, or for 2-D blocks (mz == 1) the form without W and kz;
// evaluated here at the two points of a face instead of a separate pass and array
__device__ __forceinline__ double entropy_fix_delta(const DevZone &z, int g) {
  const double u = bvl(z, g, 1), v = bvl(z, g, 2), w = bvl(z, g, 3);
  double m[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) m[c] = met(z, g, c);
  const double U = fabs(u * m[0] + v * m[1] + w * m[2]);
  const double V = fabs(u * m[3] + v * m[4] + w * m[5]);
  const double W = fabs(u * m[6] + v * m[7] + w * m[8]);
  const double kx = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
  const double ky = sqrt(m[3] * m[3] + m[4] * m[4] + m[5] * m[5]);
  const double kz = sqrt(m[6] * m[6] + m[7] * m[7] + m[8] * m[8]);
  if (z.mz == 1) return c_p.entropy_fix_factor * (U + V + ld(z.a + g) * 0.5 * (kx + ky));
  return c_p.entropy_fix_factor * (U + V + W + ld(z.a + g) * (kx + ky + kz) * (1.0 / 3));
}

// Roe flux-difference splitting (Roe_compute_half_point_flux + compute_half_sum_left_right_flux,
// Roe.cu:186-375)
template <int NS, int DIR>
__device__ __forceinline__ void inviscid_face_roe(const DevZone &z, int g0, double *F) {
  constexpr int NV = 5 + NS;
  const int g1 = g0 + dir_stride<DIR>(z);
  double pl[NV + 2], pr[NV + 2];
  reconstruct_pv<NS, DIR>(z, g0, pl, pr);
  const double j0 = ld(z.jac + g0), j1 = ld(z.jac + g1);
  const double m0x = met(z, g0, 3 * DIR), m0y = met(z, g0, 3 * DIR + 1), m0z = met(z, g0, 3 * DIR + 2);
  const double m1x = met(z, g1, 3 * DIR), m1y = met(z, g1, 3 * DIR + 1), m1z = met(z, g1, 3 * DIR + 2);
  {  // half sum of the left and right physical fluxes, each with its own point's metric
    double Jx = j0 * m0x, Jy = j0 * m0y, Jz = j0 * m0z;
    double Uk = pl[1] * Jx + pl[2] * Jy + pl[3] * Jz;
    double co = Uk * pl[0];
    F[0] = 0.5 * co;
    F[1] = 0.5 * (co * pl[1] + pl[4] * Jx);
    F[2] = 0.5 * (co * pl[2] + pl[4] * Jy);
    F[3] = 0.5 * (co * pl[3] + pl[4] * Jz);
    F[4] = 0.5 * Uk * (pl[4] + pl[NV]);
#pragma unroll
    for (int l = 5; l < NV; ++l) F[l] = 0.5 * co * pl[l];
    Jx = j1 * m1x;
    Jy = j1 * m1y;
    Jz = j1 * m1z;
    Uk = pr[1] * Jx + pr[2] * Jy + pr[3] * Jz;
    co = Uk * pr[0];
    F[0] += 0.5 * co;
    F[1] += 0.5 * (co * pr[1] + pr[4] * Jx);
    F[2] += 0.5 * (co * pr[2] + pr[4] * Jy);
    F[3] += 0.5 * (co * pr[3] + pr[4] * Jz);
    F[4] += 0.5 * Uk * (pr[4] + pr[NV]);
#pragma unroll
    for (int l = 5; l < NV; ++l) F[l] += 0.5 * co * pr[l];
  }
  const double dl = sqrt(pl[0]), dr = sqrt(pr[0]);
  const double inv_den = 1.0 / (dl + dr);
  const double u = (dl * pl[1] + dr * pr[1]) * inv_den;
  const double v = (dl * pl[2] + dr * pr[2]) * inv_den;
  const double w = (dl * pl[3] + dr * pr[3]) * inv_den;
  const double ek = 0.5 * (u * u + v * v + w * w);
  const double hl = (pl[NV] + pl[4]) / pl[0], hr = (pr[NV] + pr[4]) / pr[0];
  const double h = (dl * hl + dr * hr) * inv_den;
  double gamma = gamma_air;
  double c = sqrt((gamma - 1) * (h - ek));
  double mw = mw_air;
  double svm[NS > 0 ? NS : 1], h_i[NS > 0 ? NS : 1];
  if constexpr (NS > 0) {
    double mw_inv = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      svm[l] = (dl * pl[l + 5] + dr * pr[l + 5]) * inv_den;
      mw_inv += svm[l] * c_p.imw[l];
    }
    const double tl = pl[4] / pl[0], tr = pr[4] / pr[0];
    const double t = (dl * tl + dr * tr) * inv_den / (R_u * mw_inv);
    double cp_i[NS];
    enthalpy_cp<NS>(t, h_i, cp_i);
    double cv = 0, cp = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      cp += cp_i[l] * svm[l];
      cv += svm[l] * (cp_i[l] - c_p.Rmw[l]);
    }
    gamma = cp / cv;
    c = sqrt(gamma * R_u * mw_inv * t);
    mw = 1.0 / mw_inv;
  }
  double kx = 0.5 * (m0x + m1x), ky = 0.5 * (m0y + m1y), kz = 0.5 * (m0z + m1z);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  double Uk = kx * u + ky * v + kz * w;
  double ch[3] = {Uk - gradK * c, Uk, Uk + gradK * c};
  const double dfix = 0.5 * (entropy_fix_delta(z, g0) + entropy_fix_delta(z, g1));
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    ch[q] = fabs(ch[q]);
    if (ch[q] < dfix) ch[q] = 0.5 * (ch[q] * ch[q] / dfix + dfix);
  }
  kx /= gradK;
  ky /= gradK;
  kz /= gradK;
  Uk /= gradK;
  const double jac_ave = 0.5 * (j0 + j1);
  double dq[NV];
  dq[0] = jac_ave * (pr[0] - pl[0]);
#pragma unroll
  for (int l = 1; l < NV; ++l) dq[l] = jac_ave * (pr[0] * pr[l] - pl[0] * pl[l]);
  dq[4] = jac_ave * (pr[NV] - pl[NV]);
  double c1 = (gamma - 1) * (ek * dq[0] - u * dq[1] - v * dq[2] - w * dq[3] + dq[4]) / (c * c);
  double c2 = (kx * dq[1] + ky * dq[2] + kz * dq[3] - Uk * dq[0]) / c;
#pragma unroll
  for (int l = 0; l < NS; ++l) c1 += (mw * c_p.imw[l] - h_i[l] * (gamma - 1) / (c * c)) * dq[l + 5];
  double c3 = dq[0] - c1;
  double b[NV];
  {
    double L[NV];
    L[0] = 0.5 * (c1 - c2);
    L[1] = kx * c3 - ((kz * v - ky * w) * dq[0] - kz * dq[2] + ky * dq[3]) / c;
    L[2] = ky * c3 - ((kx * w - kz * u) * dq[0] - kx * dq[3] + kz * dq[1]) / c;
    L[3] = kz * c3 - ((ky * u - kx * v) * dq[0] - ky * dq[1] + kx * dq[2]) / c;
    L[4] = 0.5 * (c1 + c2);
#pragma unroll
    for (int l = 0; l < NS; ++l) L[l + 5] = dq[l + 5] - svm[l] * dq[0];
    b[0] = -ch[0] * L[0];
#pragma unroll
    for (int l = 1; l < NV; ++l) b[l] = -ch[1] * L[l];
    b[4] = -ch[2] * L[4];
  }
  const double c0 = kx * b[1] + ky * b[2] + kz * b[3];
  c1 = c0 + b[0] + b[4];
  c2 = c * (b[4] - b[0]);
  c3 = 0;
#pragma unroll
  for (int l = 0; l < NS; ++l) c3 += (h_i[l] - mw * c_p.imw[l] * c * c / (gamma - 1)) * b[l + 5];
  F[0] += 0.5 * c1;
  F[1] += 0.5 * (u * c1 + kx * c2 - c * (kz * b[2] - ky * b[3]));
  F[2] += 0.5 * (v * c1 + ky * c2 - c * (kx * b[3] - kz * b[1]));
  F[3] += 0.5 * (w * c1 + kz * c2 - c * (ky * b[1] - kx * b[2]));
  F[4] += 0.5 * (h * c1 + Uk * c2 - c * c * c0 / (gamma - 1) +
                 c * ((kz * v - ky * w) * b[1] + (kx * w - kz * u) * b[2] + (ky * u - kx * v) * b[3]) + c3);
#pragma unroll
  for (int l = 0; l < NS; ++l) F[5 + l] += 0.5 * (b[l + 5] + svm[l] * c1);
}

// ---------------------------------------------------------------------------
// AWENO-5 characteristic face, air only (AWENO.cu:17-206). The characteristic
// rows are processed one at a time so that only one row of the left
// eigenvector matrix is live.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void weno5_pair(const double v[6], double &vminus, double &vplus) {
  constexpr double t13 = 13.0 / 12, eps = 1e-6, d0 = 1.0 / 16, d1 = 5.0 / 8, d2 = 5.0 / 16;
  double v0 = 0.125 * (3 * v[0] - 10 * v[1] + 15 * v[2]);
  double v1 = 0.125 * (-v[1] + 6 * v[2] + 3 * v[3]);
  double v2 = 0.125 * (3 * v[2] + 6 * v[3] - v[4]);
  double b0 = t13 * (v[0] + v[2] - 2 * v[1]) * (v[0] + v[2] - 2 * v[1]) +
              0.25 * (v[0] + 3 * v[2] - 4 * v[1]) * (v[0] + 3 * v[2] - 4 * v[1]);
  double b1 = t13 * (v[1] + v[3] - 2 * v[2]) * (v[1] + v[3] - 2 * v[2]) + 0.25 * (v[3] - v[1]) * (v[3] - v[1]);
  double b2 = t13 * (v[2] + v[4] - 2 * v[3]) * (v[2] + v[4] - 2 * v[3]) +
              0.25 * (3 * v[2] + v[4] - 4 * v[3]) * (3 * v[2] + v[4] - 4 * v[3]);
  double tau = (b0 - b2) * (b0 - b2);
  double a0 = d0 + d0 * tau / ((eps + b0) * (eps + b0));
  double a1 = d1 + d1 * tau / ((eps + b1) * (eps + b1));
  double a2 = d2 + d2 * tau / ((eps + b2) * (eps + b2));
  vminus = (a0 * v0 + a1 * v1 + a2 * v2) / (a0 + a1 + a2);
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
  vplus = (a0 * v0 + a1 * v1 + a2 * v2) / (a0 + a1 + a2);
}

// NT = 2 (SST): k and omega are not part of the reference's AWENO (quirk A3:
// its WENO5 reads a 5-variable row stride); here their conservative values
// rho k, rho omega are reconstructed component by component with the same
// WENO5 weights and divided by the characteristically reconstructed density.
template <int DIR, int NT = 0>
__device__ __forceinline__ void inviscid_face_aweno(const DevZone &z, int g0, double *F) {
  constexpr double gm1 = gamma_air - 1;
  constexpr int NV = 5 + NT;
  const int sd = dir_stride<DIR>(z);
  double U[6][5];
#pragma unroll
  for (int s = 0; s < 6; ++s)
#pragma unroll
    for (int l = 0; l < 5; ++l) U[s][l] = cvl(z, g0 + (s - 2) * sd, l);
  const double pL = bvl(z, g0, 4), pR = bvl(z, g0 + sd, 4);
  const double *cl = U[2], *cr = U[3];
  const double sl0 = sqrt(cl[0]), sr0 = sqrt(cr[0]);
  const double rlc = sl0 / (sl0 + sr0), rrc = sr0 / (sl0 + sr0);
  const double um = rlc * cl[1] / cl[0] + rrc * cr[1] / cr[0];
  const double vm = rlc * cl[2] / cl[0] + rrc * cr[2] / cr[0];
  const double wm = rlc * cl[3] / cl[0] + rrc * cr[3] / cr[0];
  const double ekm = 0.5 * (um * um + vm * vm + wm * wm);
  const double hm = rlc * ((cl[4] + pL) / cl[0]) + rrc * ((cr[4] + pR) / cr[0]);
  const double cm2 = gm1 * (hm - ekm);
  const double cm = sqrt(cm2);
  const int g1 = g0 + sd;
  double kx = 0.5 * (met(z, g0, 3 * DIR) + met(z, g1, 3 * DIR));
  double ky = 0.5 * (met(z, g0, 3 * DIR + 1) + met(z, g1, 3 * DIR + 1));
  double kz = 0.5 * (met(z, g0, 3 * DIR + 2) + met(z, g1, 3 * DIR + 2));
  const double gK = sqrt(kx * kx + ky * ky + kz * kz);
  kx /= gK;
  ky /= gK;
  kz /= gK;
  const double Uk = kx * um + ky * vm + kz * wm;
  const double alpha = gm1 * ekm;
  double ql[5] = {0, 0, 0, 0, 0}, qr[5] = {0, 0, 0, 0, 0};
  if (c_p.reconstruction == 4) {
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double L[5];
      switch (r) {
        case 0:
          L[0] = (alpha + Uk * cm) / cm2 * 0.5;
          L[1] = -(gm1 * um + kx * cm) / cm2 * 0.5;
          L[2] = -(gm1 * vm + ky * cm) / cm2 * 0.5;
          L[3] = -(gm1 * wm + kz * cm) / cm2 * 0.5;
          L[4] = gm1 / cm2 * 0.5;
          break;
        case 1:
          L[0] = kx * (1 - alpha / cm2) - (kz * vm - ky * wm) / cm;
          L[1] = kx * gm1 * um / cm2;
          L[2] = (kx * gm1 * vm + kz * cm) / cm2;
          L[3] = (kx * gm1 * wm - ky * cm) / cm2;
          L[4] = -kx * gm1 / cm2;
          break;
        case 2:
          L[0] = ky * (1 - alpha / cm2) - (kx * wm - kz * um) / cm;
          L[1] = (ky * gm1 * um - kz * cm) / cm2;
          L[2] = ky * gm1 * vm / cm2;
          L[3] = (ky * gm1 * wm + kx * cm) / cm2;
          L[4] = -ky * gm1 / cm2;
          break;
        case 3:
          L[0] = kz * (1 - alpha / cm2) - (ky * um - kx * vm) / cm;
          L[1] = (kz * gm1 * um + ky * cm) / cm2;
          L[2] = (kz * gm1 * vm - kx * cm) / cm2;
          L[3] = kz * gm1 * wm / cm2;
          L[4] = -kz * gm1 / cm2;
          break;
        default:
          L[0] = (alpha - Uk * cm) / cm2 * 0.5;
          L[1] = -(gm1 * um - kx * cm) / cm2 * 0.5;
          L[2] = -(gm1 * vm - ky * cm) / cm2 * 0.5;
          L[3] = -(gm1 * wm - kz * cm) / cm2 * 0.5;
          L[4] = gm1 / cm2 * 0.5;
      }
      double v[6];
#pragma unroll
      for (int s = 0; s < 6; ++s) {
        double acc = 0;
#pragma unroll
        for (int j = 0; j < 5; ++j) acc += L[j] * U[s][j];
        v[s] = acc;
      }
      double vmn, vpl;
      weno5_pair(v, vmn, vpl);
      // column r of the right eigenvector matrix (AWENO.cu:98-122)
      double Rc[5];
      switch (r) {
        case 0: Rc[0] = 1.0; Rc[1] = um - kx * cm; Rc[2] = vm - ky * cm; Rc[3] = wm - kz * cm; Rc[4] = hm - Uk * cm; break;
        case 1: Rc[0] = kx; Rc[1] = kx * um; Rc[2] = kx * vm + kz * cm; Rc[3] = kx * wm - ky * cm;
                Rc[4] = kx * alpha / gm1 + (kz * vm - ky * wm) * cm; break;
        case 2: Rc[0] = ky; Rc[1] = ky * um - kz * cm; Rc[2] = ky * vm; Rc[3] = ky * wm + kx * cm;
                Rc[4] = ky * alpha / gm1 + (kx * wm - kz * um) * cm; break;
        case 3: Rc[0] = kz; Rc[1] = kz * um + ky * cm; Rc[2] = kz * vm - kx * cm; Rc[3] = kz * wm;
                Rc[4] = kz * alpha / gm1 + (ky * um - kx * vm) * cm; break;
        default: Rc[0] = 1.0; Rc[1] = um + kx * cm; Rc[2] = vm + ky * cm; Rc[3] = wm + kz * cm; Rc[4] = hm + Uk * cm;
      }
#pragma unroll
      for (int m = 0; m < 5; ++m) {
        ql[m] += Rc[m] * vmn;
        qr[m] += Rc[m] * vpl;
      }
    }
  }
  double pl[NV + 2], pr[NV + 2];
  pl[0] = ql[0];
  pl[1] = ql[1] / ql[0];
  pl[2] = ql[2] / ql[0];
  pl[3] = ql[3] / ql[0];
  pl[4] = gm1 * (ql[4] - 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]) * ql[0]);
  pl[NV] = ql[4];
  pl[NV + 1] = gamma_air;
  pr[0] = qr[0];
  pr[1] = qr[1] / qr[0];
  pr[2] = qr[2] / qr[0];
  pr[3] = qr[3] / qr[0];
  pr[4] = gm1 * (qr[4] - 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]) * qr[0]);
  pr[NV] = qr[4];
  pr[NV + 1] = gamma_air;
#pragma unroll
  for (int t = 0; t < NT; ++t) {  // componentwise WENO5 of rho k, rho omega
    double v[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) v[s] = cvl(z, g0 + (s - 2) * sd, 5 + t);
    double vmn = 0, vpl = 0;
    if (c_p.reconstruction == 4) weno5_pair(v, vmn, vpl);
    pl[5 + t] = vmn / ql[0];
    pr[5 + t] = vpl / qr[0];
  }
  riemann<NV, 0>(pl, pr, plane_cells<DIR>(z, g0), DIR, F);
}

// physical flux of the AWENO central correction at one point (AWENO.cu:236-249);
// NT turbulence scalars: jac * rho U s
template <int DIR, int NT = 0>
__device__ __forceinline__ void cds_point_flux(const DevZone &z, int g, double *f) {
  const double kx = met(z, g, 3 * DIR), ky = met(z, g, 3 * DIR + 1), kz = met(z, g, 3 * DIR + 2);
  const double jac = ld(z.jac + g);
  const double u = bvl(z, g, 1), v = bvl(z, g, 2), w = bvl(z, g, 3);
  const double Uk = kx * u + ky * v + kz * w;
  const double rUk = bvl(z, g, 0) * Uk;
  const double p = bvl(z, g, 4);
  f[0] = rUk * jac;
  f[1] = jac * (rUk * u + kx * p);
  f[2] = jac * (rUk * v + ky * p);
  f[3] = jac * (rUk * w + kz * p);
  f[4] = jac * Uk * (cvl(z, g, 4) + p);
#pragma unroll
  for (int t = 0; t < NT; ++t) f[5 + t] = jac * (rUk * svl(z, g, t));
}

// sum_m c_m (f(c+m) - f(c-m)), m = 3, 2, 1 (AWENO.cu:257-263)
template <int DIR, int NT = 0>
__device__ __forceinline__ void cds_correction(const DevZone &z, int g, double *corr) {
  constexpr int NC = 5 + NT;
  const int sd = dir_stride<DIR>(z);
  constexpr double c1 = 19.0 / 3840, c2 = -13.0 / 320, c3 = 17.0 / 256;
  double fp[NC], fm[NC], d3[NC], d2[NC];
  cds_point_flux<DIR, NT>(z, g + 3 * sd, fp);
  cds_point_flux<DIR, NT>(z, g - 3 * sd, fm);
#pragma unroll
  for (int l = 0; l < NC; ++l) d3[l] = fp[l] - fm[l];
  cds_point_flux<DIR, NT>(z, g + 2 * sd, fp);
  cds_point_flux<DIR, NT>(z, g - 2 * sd, fm);
#pragma unroll
  for (int l = 0; l < NC; ++l) d2[l] = fp[l] - fm[l];
  cds_point_flux<DIR, NT>(z, g + sd, fp);
  cds_point_flux<DIR, NT>(z, g - sd, fm);
#pragma unroll
  for (int l = 0; l < NC; ++l) corr[l] = c1 * d3[l] + c2 * d2[l] + c3 * (fp[l] - fm[l]);
}

// ---------------------------------------------------------------------------
// viscous face flux (ViscousScheme.cuh:22-821, compute_{f,g,h}v_2nd_order);
// NT = 2: the SST terms (turbulent viscosity and conductivity, the -2/3 rho k
// normal stresses, k and omega diffusion with the F1 blend)
// ---------------------------------------------------------------------------
template <int NS, int DIR, int NT, class Cells>
__device__ __forceinline__ void viscous_face(const Cells &cc, double *F) {
  constexpr int NV = 5 + NS + NT;
  // tangential directions
  constexpr int TA = DIR == 0 ? 1 : 0, TB = DIR == 2 ? 1 : 2;
  double mm[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) mm[c] = 0.5 * (cc.met(c, 0) + cc.met(c, 1));
  // derivative along (normal, ta, tb) ordered as (xi, eta, zeta); v(n, a, b) is the variable's cell value
  auto der = [&](auto v, double out[3]) {
    const double dn = v(1, 0, 0) - v(0, 0, 0);
    const double da = 0.25 * (v(0, 1, 0) - v(0, -1, 0) + v(1, 1, 0) - v(1, -1, 0));
    const double db = 0.25 * (v(0, 0, 1) - v(0, 0, -1) + v(1, 0, 1) - v(1, 0, -1));
    out[DIR] = dn;
    out[TA] = da;
    out[TB] = db;
  };
  auto bvv = [&](int l) { return [&cc, l](int n, int a, int b) { return cc.bv(l, n, a, b); }; };
  auto svv = [&](int l) { return [&cc, l](int n, int a, int b) { return cc.sv(l, n, a, b); }; };
  double du[3], dv[3], dw[3], dt[3];
  der(bvv(1), du);
  der(bvv(2), dv);
  der(bvv(3), dw);
  der(bvv(5), dt);
  const double u_x = du[0] * mm[0] + du[1] * mm[3] + du[2] * mm[6];
  const double u_y = du[0] * mm[1] + du[1] * mm[4] + du[2] * mm[7];
  const double u_z = du[0] * mm[2] + du[1] * mm[5] + du[2] * mm[8];
  const double v_x = dv[0] * mm[0] + dv[1] * mm[3] + dv[2] * mm[6];
  const double v_y = dv[0] * mm[1] + dv[1] * mm[4] + dv[2] * mm[7];
  const double v_z = dv[0] * mm[2] + dv[1] * mm[5] + dv[2] * mm[8];
  const double w_x = dw[0] * mm[0] + dw[1] * mm[3] + dw[2] * mm[6];
  const double w_y = dw[0] * mm[1] + dw[1] * mm[4] + dw[2] * mm[7];
  const double w_z = dw[0] * mm[2] + dw[1] * mm[5] + dw[2] * mm[8];
  const double mul = 0.5 * (cc.mul(0) + cc.mul(1));
  const double mut = NT > 0 ? 0.5 * (cc.mut(0) + cc.mut(1)) : 0.0;
  const double mu = NT > 0 ? mul + mut : mul;
  double txx = mu * (4 * u_x - 2 * v_y - 2 * w_z) * (1.0 / 3);
  double tyy = mu * (4 * v_y - 2 * u_x - 2 * w_z) * (1.0 / 3);
  double tzz = mu * (4 * w_z - 2 * u_x - 2 * v_y) * (1.0 / 3);
  const double txy = mu * (u_y + v_x), txz = mu * (u_z + w_x), tyz = mu * (v_z + w_y);
  if constexpr (NT > 0) {  // ViscousScheme.cuh:82-95
    constexpr double delta_d = 1e-3;
    const double dy_div_delta = fmin(0.5 * (cc.wall(0) + cc.wall(1)) / delta_d, 1.0);
    const double twoThirdrhoKm =
        -2.0 / 3 * 0.5 * (cc.bv(0, 0) * cc.sv(NS, 0) + cc.bv(0, 1) * cc.sv(NS, 1)) * dy_div_delta;
    txx += twoThirdrhoKm;
    tyy += twoThirdrhoKm;
    tzz += twoThirdrhoKm;
  }
  const double j0 = cc.jac(0), j1 = cc.jac(1);
  const double kxj = 0.5 * (cc.met(3 * DIR, 0) * j0 + cc.met(3 * DIR, 1) * j1);
  const double kyj = 0.5 * (cc.met(3 * DIR + 1, 0) * j0 + cc.met(3 * DIR + 1, 1) * j1);
  const double kzj = 0.5 * (cc.met(3 * DIR + 2, 0) * j0 + cc.met(3 * DIR + 2, 1) * j1);
  F[0] = 0;
  F[1] = kxj * txx + kyj * txy + kzj * txz;
  F[2] = kxj * txy + kyj * tyy + kzj * tyz;
  F[3] = kxj * txz + kyj * tyz + kzj * tzz;
  const double um = 0.5 * (cc.bv(1, 0) + cc.bv(1, 1));
  const double vm = 0.5 * (cc.bv(2, 0) + cc.bv(2, 1));
  const double wm = 0.5 * (cc.bv(3, 0) + cc.bv(3, 1));
  const double t_x = dt[0] * mm[0] + dt[1] * mm[3] + dt[2] * mm[6];
  const double t_y = dt[0] * mm[1] + dt[1] * mm[4] + dt[2] * mm[7];
  const double t_z = dt[0] * mm[2] + dt[1] * mm[5] + dt[2] * mm[8];
  double cond = 0.5 * (cc.kappa(0) + cc.kappa(1));
  if constexpr (NT > 0) cond += 0.5 * (cc.ttc(0) + cc.ttc(1));
  F[4] = um * F[1] + vm * F[2] + wm * F[3] + cond * (kxj * t_x + kyj * t_y + kzj * t_z);
  if constexpr (NS > 0) {
    double yk[NS], diff[NS], ddf[NS];
    double sgw = 0, srdy = 0, corr = 0, mwt = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      yk[l] = 0.5 * (cc.sv(l, 0) + cc.sv(l, 1));
      diff[l] = 0.5 * (cc.rhod(l, 0) + cc.rhod(l, 1));
      if constexpr (NT > 0) diff[l] += mut / c_p.Sct;  // turbulent diffusivity (ViscousScheme.cuh:122-125)
      double dy[3];
      der(svv(l), dy);
      const double y_x = dy[0] * mm[0] + dy[1] * mm[3] + dy[2] * mm[6];
      const double y_y = dy[0] * mm[1] + dy[1] * mm[4] + dy[2] * mm[7];
      const double y_z = dy[0] * mm[2] + dy[1] * mm[5] + dy[2] * mm[8];
      const double g = kxj * y_x + kyj * y_y + kzj * y_z;
      ddf[l] = g;
      corr += diff[l] * g;
      sgw += g * c_p.imw[l];
      mwt += yk[l] * c_p.imw[l];
      srdy += diff[l] * yk[l];
    }
    mwt = 1.0 / mwt;
    corr -= mwt * srdy * sgw;
    if (c_p.gradP) {
      double dp[3];
      der(bvv(4), dp);
      const double p_x = dp[0] * mm[0] + dp[1] * mm[3] + dp[2] * mm[6];
      const double p_y = dp[0] * mm[1] + dp[1] * mm[4] + dp[2] * mm[7];
      const double p_z = dp[0] * mm[2] + dp[1] * mm[5] + dp[2] * mm[8];
      const double gp = (kxj * p_x + kyj * p_y + kzj * p_z) / (0.5 * (cc.bv(4, 1) + cc.bv(4, 0)));
#pragma unroll
      for (int l = 0; l < NS; ++l) {
        ddf[l] += (mwt * c_p.imw[l] - 1) * yk[l] * gp;
        corr += (mwt * c_p.imw[l] - 1) * yk[l] * gp * diff[l];
      }
    }
    double h[NS];
    enthalpy<NS>(0.5 * (cc.bv(5, 0) + cc.bv(5, 1)), h);
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      const double flux = diff[l] * (ddf[l] - mwt * yk[l] * sgw) - yk[l] * corr;
      F[5 + l] = flux;
      F[4] += h[l] * flux;
    }
  }
  if constexpr (NT > 0) {  // k and omega diffusion (ViscousScheme.cuh:200-251)
    double dk[3], dw[3];
    der(svv(NS), dk);
    der(svv(NS + 1), dw);
    const double k_x = dk[0] * mm[0] + dk[1] * mm[3] + dk[2] * mm[6];
    const double k_y = dk[0] * mm[1] + dk[1] * mm[4] + dk[2] * mm[7];
    const double k_z = dk[0] * mm[2] + dk[1] * mm[5] + dk[2] * mm[8];
    const double omega_x = dw[0] * mm[0] + dw[1] * mm[3] + dw[2] * mm[6];
    const double omega_y = dw[0] * mm[1] + dw[1] * mm[4] + dw[2] * mm[7];
    const double omega_z = dw[0] * mm[2] + dw[1] * mm[5] + dw[2] * mm[8];
    const double wall_dist = 0.5 * (cc.wall(0) + cc.wall(1));
    double f1 = 1;
    if (wall_dist > 1e-25) {
      const double km = 0.5 * (cc.sv(NS, 0) + cc.sv(NS, 1));
      const double omegam = 0.5 * (cc.sv(NS + 1, 0) + cc.sv(NS + 1, 1));
      const double param1 = sqrt(km) / (0.09 * omegam * wall_dist);
      const double rhom = 0.5 * (cc.bv(0, 0) + cc.bv(0, 1));
      const double d2 = wall_dist * wall_dist;
      const double param2 = 500 * mul / (rhom * d2 * omegam);
      const double CDkomega =
          fmax(1e-20, 2 * rhom * sst::sigma_omega2 / omegam * (k_x * omega_x + k_y * omega_y + k_z * omega_z));
      const double param3 = 4 * rhom * sst::sigma_omega2 * km / (CDkomega * d2);
      const double arg1 = fmin(fmax(param1, param2), param3);
      f1 = tanh(arg1 * arg1 * arg1 * arg1);
    }
    const double sigma_k = sst::sigma_k2 + sst::delta_sigma_k * f1;
    const double sigma_omega = sst::sigma_omega2 + sst::delta_sigma_omega * f1;
    F[5 + NS] = (mul + mut * sigma_k) * (kxj * k_x + kyj * k_y + kzj * k_z);
    F[6 + NS] = (mul + mut * sigma_omega) * (kxj * omega_x + kyj * omega_y + kzj * omega_z);
  }
  (void)NV;
}

}  // namespace ostc
