// common.cuh — device-side data model of the B200 RHS/RK3 path.
//
// DevZone is the kernel-side view of one block of the reference's DZone
// (src/Field.h:13-71): base pointers of the ColMajor planes plus the three
// stride sets in use (ghosted arrays, dq-like arrays, interior-only arrays).
// DevParam holds the scalar tags and species/reaction tables of the
// reference's DParameter (src/DParameter.cuh:13-92) in __constant__ memory,
// where every warp reads them with uniform addresses.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/ostc.h"

namespace ostc {

constexpr double R_u = 8314.462618;  // universal gas constant, J/(kmol K)
constexpr double p_atm = 101325;
constexpr double gamma_air = 1.4;
constexpr double mw_air = 28.9647;
constexpr int MAXS = OSTC_MAX_SPEC;
constexpr int MAXR = OSTC_MAX_REAC;

struct DevParam {
  int n_var, n_scalar, n_spec, n_reac;
  int mix, inviscid_scheme, reconstruction, limiter, inviscid_type, viscous_scheme;
  int chemSrcMethod, gradP, dimension, turbulence, need_gibbs, sst;  // sst: k-omega SST scalars in sv
  int comp_corr, turb_implicit;  // SST: compressibility correction 0..3; point-implicit k, omega sources (steady)
  double Pr, Prt, Sct, Sc, cfl, entropy_fix_factor;
  double mw[MAXS], imw[MAXS], Rmw[MAXS];           // W_k, 1/W_k, R_u/W_k
  double lo[MAXS][7], hi[MAXS][7];                 // NASA-7 low / high ranges
  double t_low[MAXS], t_mid[MAXS];
  double LJ_inv[MAXS], vis_coeff[MAXS];
  double WjWi4[MAXS][MAXS], sqWW8[MAXS][MAXS];     // Wilke mixing constants
  double bdc[MAXS][MAXS], kbe[MAXS][MAXS];         // binary diffusion constants
  // derived on the host so that one pow(T, -0.145) per point serves all
  // species and pairs: (T c)^-0.145 = T^-0.145 c^-0.145
  double LJm145[MAXS];                             // LJ_inv^-0.145
  double kbem145[MAXS][MAXS];                      // kb_over_eps^-0.145
  double inv_bdc[MAXS][MAXS];                      // 1 / binary_diffusivity_coeff
  int reac_type[MAXR], reac_order[MAXR];
  signed char nuf[MAXR][MAXS], nub[MAXR][MAXS];    // stoichiometric coefficients
  double A[MAXR], b[MAXR], Ea[MAXR], A2[MAXR], b2[MAXR], Ea2[MAXR];
  double tb[MAXR][MAXS];                           // third-body efficiencies
  double troe_alpha[MAXR], troe_t3[MAXR], troe_t1[MAXR], troe_t2[MAXR];
};

// c_p (the __constant__ DevParam) is defined in kernels.cu before the
// physics headers that read it are included.

struct DevZone {
  int mx, my, mz, ngg;
  // ghosted arrays (g = ngg)
  int d2, d1, dt_;  // disp2, disp1, dispt
  long long sz;
  // dq-like arrays (g = dq_ngg)
  int q2, q1, qt;
  long long qsz;
  // interior arrays (g = 0)
  int n2, n1;
  long long nsz;
  double *bv, *sv, *cv, *qn, *dq;
  double *vel, *a, *mach, *mul, *kappa, *rhoD, *gam, *cp, *mut, *ttc, *wall;
  double *dt_local, *bv_last;
  double *isr;  // inviscid spectral radii, 3 interior planes (steady path; null otherwise)
  double *tsj;  // SST source Jacobian diagonal, 2 interior planes (steady path with turb_implicit; else null)
  const double *jac;
  const double *met;  // 9 SoA planes (context-owned copy), ghosted layout
  int block_id;
  // sz and qsz as 32-bit ints for the flux kernels' index arithmetic (every
  // plane offset of a block is below 2^31: checked at ostc_create)
  int isz, iqsz;
  // bit 0 (kZoneBulk): the ghosted row length is even and every plane the
  // staged flux kernels copy starts on a 16-byte boundary, so that their tile
  // rows can move as 16-byte-aligned bulk copies
  int flags;
};

constexpr int kZoneBulk = 1;

__device__ __forceinline__ int gidx(const DevZone &z, int i, int j, int k) {
  return k * z.d1 + j * z.d2 + i + z.dt_;
}
__device__ __forceinline__ int qidx(const DevZone &z, int i, int j, int k) {
  return k * z.q1 + j * z.q2 + i + z.qt;
}
__device__ __forceinline__ int nidx(const DevZone &z, int i, int j, int k) {
  return k * z.n1 + j * z.n2 + i;
}

// read-only load through the non-coherent path
template <typename T>
__device__ __forceinline__ T ld(const T *p) { return __ldg(p); }

// error word written by kernels (first failing cell), read by ostc_get_error
struct DevError {
  int status;
  int block, i, j, k;
};

}  // namespace ostc
