// kernels.cu — sm_100a kernels of the RHS / RK3 stage (the flux kernels,
// flux_dir in flux.cuh, are built in flux0.cu, flux9.cu, flux0t.cu and flux9t.cu).
//
//  source_kernel<NS>      finite-rate chemistry or SST source, starts dq (SourceTerm.cuh:11-37)
//  update_rk_kernel<NS>   SSPRK3 stage update, cv -> bv/sv, T and p (RK.cuh:197-253)
//  properties_kernel<NS>  cp, gamma, a, mu, kappa, rho*D, Mach over [-1, m] (FieldOperation.cuh:112-146)
//  cv_from_bv_kernel<NS>  conservative from primitive, ghosts included (FieldOperation.cuh:43-79)
//  dt_kernel<NS>          local time step + block min + atomic min (TimeAdvanceFunc.cuh:50-100, .cu:155-201)
//  bc_*_kernel            boundary conditions (BoundCond.cuh:52-210) and periodic wrap
//  waves_kernel<NS,KIND>  every boundary face (KIND 0) or interface (KIND 1) of a call in
//                         one cooperative launch, waves apart by a bounded grid barrier
//  residual kernels       store_last_step / square of d(bv) / deterministic sums (Residual.cuh:57-161)
#include <cstdio>

#include "common.cuh"

namespace ostc {
// this unit's copy of the run parameters (written by upload_param)
static __constant__ DevParam c_p;
}

#include "chem.cuh"
#include "mech_h2air9.cuh"
#include "face.cuh"
#include "kernels.cuh"
#include "thermo.cuh"

namespace ostc {

// the zones of tile-table launches (upload_zones)
static __constant__ DevZone c_zones[kMaxTableZones];

// ---------------------------------------------------------------------------
// per-cell kernels
// ---------------------------------------------------------------------------
// SPEC = 1: the mechanism-specialised chemistry (mech_h2air9.cuh), for
// contexts whose mechanism has that structure
template <int NS, int SPEC>
__device__ __forceinline__ void source_cells(const DevZone &z, const int bx, const int by, const int bz) {
  constexpr int NV = 5 + NS;
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k = bz;
  if (i >= z.mx || j >= z.my) return;
  const int g = gidx(z, i, j, k);
  double *dq = z.dq + qidx(z, i, j, k);
#pragma unroll
  for (int l = 0; l < 5; ++l) dq[l * z.qsz] = 0;
  if (c_p.sst) {  // SST::compute_source_and_mut and the turbulent conductivity (SourceTerm.cuh:19-27)
    double mut, sk, sw, jk, jw;
    sst::source_point<NS>(z, g, mut, sk, sw, jk, jw);
    z.mut[g] = mut;
    if (c_p.turb_implicit == 1 && z.tsj) {  // SST.cu:243-246
      const int n = nidx(z, i, j, k);
      z.tsj[n] = jk;
      z.tsj[z.nsz + n] = jw;
    }
    constexpr double cpa = gamma_air * R_u / mw_air / (gamma_air - 1);
    z.ttc[g] = mut * (NS > 0 ? z.cp[g] : cpa) / c_p.Prt;  // the mixture's cp (SourceTerm.cuh:21-23)
    dq[(5 + NS) * z.qsz] = sk;
    dq[(6 + NS) * z.qsz] = sw;
  }
  if constexpr (NS > 0) {
    double Y[NS], om[NS];
#pragma unroll
    for (int l = 0; l < NS; ++l) Y[l] = svl(z, g, l);
    if constexpr (SPEC == 1 && NS == mech_h2air9::NS)
      mech_h2air9::omega(bvl(z, g, 0), bvl(z, g, 5), Y, om);
    else
      chemistry_omega<NS>(bvl(z, g, 0), bvl(z, g, 5), Y, om);
    const double jc = ld(z.jac + g);
#pragma unroll
    for (int l = 0; l < NS; ++l) dq[(5 + l) * z.qsz] = jc * om[l];
  }
  (void)NV;
}

template <int NS, int SPEC>
__global__ void __launch_bounds__(256) source_kernel(DevZone z) {
  source_cells<NS, SPEC>(z, blockIdx.x, blockIdx.y, blockIdx.z);
}


// batched FP64 point-implicit chemistry integrator (point_implicit_increment)
// over n states held as SoA device arrays: Y and dY are [NS][n]
template <int NS>
__global__ void __launch_bounds__(128) chem_integrator_kernel(int n, const double *T, const double *p, const double *Y,
                                                              const double *dt, double *dY, double *dT) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  if constexpr (NS > 0) {
    double y[NS], d[NS], dtq;
    int it;
#pragma unroll
    for (int l = 0; l < NS; ++l) y[l] = Y[(long long)l * n + q];
    point_implicit_increment<NS>(T[q], p[q], y, dt[q], d, dtq, it);
#pragma unroll
    for (int l = 0; l < NS; ++l) dY[(long long)l * n + q] = d[l];
    dT[q] = it ? dtq : __longlong_as_double(0x7ff8000000000000ll);  // NaN marks a failed Newton solve
  }
}


// operator-split chemistry on a block: gather the interior states as SoA
// arrays (T, p, Y [NS][n], dt), and scatter the increments back at constant
// density and internal energy (Y, T, p, the species cv; rho E unchanged)
template <int NS>
__global__ void __launch_bounds__(256) chem_gather_kernel(DevZone z, const double *dt_dev, double dt_fixed, double *T,
                                                          double *p, double *Y, double *dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= z.mx || j >= z.my) return;
  const int g = gidx(z, i, j, k);
  const long long q = nidx(z, i, j, k), n = z.nsz;
  T[q] = z.bv[5 * z.sz + g];
  p[q] = z.bv[4 * z.sz + g];
#pragma unroll
  for (int l = 0; l < NS; ++l) Y[l * n + q] = z.sv[l * z.sz + g];
  dt[q] = dt_dev ? *dt_dev : dt_fixed;
}

template <int NS>
__global__ void __launch_bounds__(256) chem_scatter_kernel(DevZone z, const double *dY, const double *dT) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= z.mx || j >= z.my) return;
  if constexpr (NS > 0) {
    const int g = gidx(z, i, j, k);
    const long long q = nidx(z, i, j, k), n = z.nsz;
    const double rho = z.bv[g];
    double mwinv = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      const double y = z.sv[l * z.sz + g] + dY[l * n + q];
      z.sv[l * z.sz + g] = y;
      z.cv[(5 + l) * z.sz + g] = rho * y;
      mwinv += y * c_p.imw[l];
    }
    const double t = z.bv[5 * z.sz + g] + dT[q];
    z.bv[5 * z.sz + g] = t;
    z.bv[4 * z.sz + g] = rho * R_u * mwinv * t;
  }
}

static __global__ void chem_stats_kernel(long long *stats, long long n, const int *count) {
  stats[0] += n;
  if (count) stats[1] += *count;
}

__constant__ double c_rk_a[3] = {1.0, 0.75, 1.0 / 3.0};
__constant__ double c_rk_b[3] = {0.0, 0.25, 2.0 / 3.0};
__constant__ double c_rk_c[3] = {1.0, 0.25, 2.0 / 3.0};

template <int NS>
__device__ __forceinline__ void update_rk_cells(const DevZone &z, const int bx, const int by, const int bz, double dt_in, const double *dt_dev, int rk) {
  constexpr int NV = 5 + NS;
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k = bz;
  if (i >= z.mx || j >= z.my) return;
  const double dt = dt_dev ? *dt_dev : dt_in;
  const int g = gidx(z, i, j, k);
  const int q = qidx(z, i, j, k);
  const double a = c_rk_a[rk], b = c_rk_b[rk], c = c_rk_c[rk];
  const double dtj = dt / z.jac[g];
  double cv[NV];
#pragma unroll
  for (int l = 0; l < NV; ++l) {
    cv[l] = a * z.qn[l * z.sz + g] + b * z.cv[l * z.sz + g] + c * dtj * z.dq[l * z.qsz + q];
  }
  if (z.mz == 1) cv[3] = 0;
#pragma unroll
  for (int l = 0; l < NV; ++l) z.cv[l * z.sz + g] = cv[l];
  const double rho = cv[0];
  const double ri = 1.0 / rho;
  // scalars after the species (SST k, omega): cv update and sv = cv / rho (RK.cuh:209-235)
  for (int l = NV; l < c_p.n_var; ++l) {
    const double c_l = a * z.qn[l * z.sz + g] + b * z.cv[l * z.sz + g] + c * dtj * z.dq[l * z.qsz + q];
    z.cv[l * z.sz + g] = c_l;
    z.sv[(l - 5) * z.sz + g] = c_l * ri;
  }
  const double u = cv[1] * ri, v = cv[2] * ri, w = cv[3] * ri;
  z.bv[g] = rho;
  z.bv[z.sz + g] = u;
  z.bv[2 * z.sz + g] = v;
  z.bv[3 * z.sz + g] = w;
  const double V2 = u * u + v * v + w * w;
  if constexpr (NS == 0) {
    const double p = (gamma_air - 1) * (cv[4] - 0.5 * rho * V2);
    z.bv[4 * z.sz + g] = p;
    z.bv[5 * z.sz + g] = p * mw_air * ri / R_u;
  } else {
    double Y[NS];
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      Y[l] = cv[5 + l] * ri;
      z.sv[l * z.sz + g] = Y[l];
    }
    // compute_temperature_and_pressure (FieldOperation.cu:3-39)
    double mw = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) mw += Y[l] * c_p.imw[l];
    mw = 1 / mw;
    const double R = R_u / mw;
    const double e = cv[4] / rho - 0.5 * V2;
    double err = 1, t = z.bv[5 * z.sz + g];
    int iter = 0;
    while (err > 1e-3 && iter++ < 1000) {
      double h[NS], cp[NS];
      enthalpy_cp<NS, false>(t, h, cp);
      double cpt = 0, hh = 0;
#pragma unroll
      for (int l = 0; l < NS; ++l) {
        cpt += cp[l] * Y[l];
        hh += h[l] * Y[l];
      }
      const double t1 = t - (hh - R * t - e) / (cpt - R);
      err = fabs(1 - t1 / t);
      t = t1;
    }
    z.bv[5 * z.sz + g] = t;
    z.bv[4 * z.sz + g] = rho * t * R;
  }
  z.vel[g] = sqrt(V2);
}

template <int NS>
__global__ void __launch_bounds__(256) update_rk_kernel(DevZone z, double dt_in, const double *dt_dev, int rk) {
  update_rk_cells<NS>(z, blockIdx.x, blockIdx.y, blockIdx.z, dt_in, dt_dev, rk);
}

template <int NS>
__device__ __forceinline__ void properties_cells(const DevZone &z, const int bx, const int by, const int bz) {
  const int i = bx * blockDim.x + threadIdx.x - 1;
  const int j = by * blockDim.y + threadIdx.y - 1;
  const int k = bz - 1;
  if (i > z.mx || j > z.my) return;
  const int g = gidx(z, i, j, k);
  const double T = z.bv[5 * z.sz + g];
  double a;
  if constexpr (NS == 0) {
    constexpr double c_temp = gamma_air * R_u / mw_air;
    constexpr double cpa = gamma_air * R_u / mw_air / (gamma_air - 1);
    a = sqrt(c_temp * T);
    const double mu = sutherland(T);
    z.mul[g] = mu;
    z.kappa[g] = mu * cpa / c_p.Pr;
  } else {
    double Y[NS], cp[NS], rD[NS];
    cp_only<NS>(T, cp);
    double mw = 0, cpt = 0, cvv = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      Y[l] = z.sv[l * z.sz + g];
      mw += Y[l] * c_p.imw[l];
      cpt += Y[l] * cp[l];
      cvv += Y[l] * (cp[l] - c_p.Rmw[l]);
    }
    mw = 1 / mw;
    const double gam = cpt / cvv;
    z.cp[g] = cpt;
    z.gam[g] = gam;
    a = sqrt(gam * R_u * T / mw);
    double mu, kap;
    mixture_transport<NS>(T, mw, Y, cp, z.bv[g], z.bv[4 * z.sz + g], mu, kap, rD);
    z.mul[g] = mu;
    z.kappa[g] = kap;
#pragma unroll
    for (int l = 0; l < NS; ++l) z.rhoD[l * z.sz + g] = rD[l];
  }
  z.a[g] = a;
  z.mach[g] = z.vel[g] / a;
}

template <int NS>
__global__ void __launch_bounds__(256) properties_kernel(DevZone z) {
  properties_cells<NS>(z, blockIdx.x, blockIdx.y, blockIdx.z);
}

// initialize_mut (FieldOperation.cuh:175-195) over [-1, m]: the SST turbulent
// viscosity from the initial field, with Sutherland's viscosity for air or
// the mixture's Wilke viscosity (compute_viscosity)
template <int NS>
__device__ __forceinline__ void init_mut_cells(const DevZone &z, const int bx, const int by, const int bz) {
  const int i = bx * blockDim.x + threadIdx.x - 1;
  const int j = by * blockDim.y + threadIdx.y - 1;
  const int k = bz - 1;
  if (i > z.mx || j > z.my) return;
  const int g = gidx(z, i, j, k);
  const double T = z.bv[5 * z.sz + g];
  double mul;
  if constexpr (NS > 0) {
    double Y[NS];
#pragma unroll
    for (int l = 0; l < NS; ++l) Y[l] = z.sv[l * z.sz + g];
    mul = mixture_viscosity<NS>(T, Y);
  } else {
    mul = sutherland(T);
  }
  z.mut[g] = sst::mut_point<NS>(z, g, mul);
}

template <int NS>
__global__ void __launch_bounds__(256) init_mut_kernel(DevZone z) {
  init_mut_cells<NS>(z, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <int NS>
__device__ __forceinline__ void cv_from_bv_point(const DevZone &z, int g) {
  const double rho = z.bv[g], u = z.bv[z.sz + g], v = z.bv[2 * z.sz + g], w = z.bv[3 * z.sz + g];
  const double p = z.bv[4 * z.sz + g];
  z.cv[g] = rho;
  z.cv[z.sz + g] = rho * u;
  z.cv[2 * z.sz + g] = rho * v;
  z.cv[3 * z.sz + g] = rho * w;
  for (int l = NS; l < c_p.n_scalar; ++l) z.cv[(5 + l) * z.sz + g] = rho * z.sv[l * z.sz + g];  // SST k, omega
  const double V2 = u * u + v * v + w * w;
  double E = 0.5 * V2;
  if constexpr (NS == 0) {
    E *= rho;
    E += p / (gamma_air - 1);
  } else {
    double h[NS];
    enthalpy<NS>(z.bv[5 * z.sz + g], h);
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      const double Y = z.sv[l * z.sz + g];
      z.cv[(5 + l) * z.sz + g] = rho * Y;
      E += h[l] * Y;
    }
    E *= rho;
    E -= p;
  }
  z.cv[4 * z.sz + g] = E;
  z.vel[g] = sqrt(V2);
}

template <int NS>
__device__ __forceinline__ void cv_from_bv_cells(const DevZone &z, const int bx, const int by, const int bz) {
  const int i = bx * blockDim.x + threadIdx.x - z.ngg;
  const int j = by * blockDim.y + threadIdx.y - z.ngg;
  const int k = bz - z.ngg;
  if (i >= z.mx + z.ngg || j >= z.my + z.ngg) return;
  cv_from_bv_point<NS>(z, gidx(z, i, j, k));
}

template <int NS>
__global__ void __launch_bounds__(256) cv_from_bv_kernel(DevZone z) {
  cv_from_bv_cells<NS>(z, blockIdx.x, blockIdx.y, blockIdx.z);
}

__device__ __forceinline__ void velocity_cells(const DevZone &z, const int bx, const int by, const int bz) {
  const int i = bx * blockDim.x + threadIdx.x - z.ngg;
  const int j = by * blockDim.y + threadIdx.y - z.ngg;
  const int k = bz - z.ngg;
  if (i >= z.mx + z.ngg || j >= z.my + z.ngg) return;
  const int g = gidx(z, i, j, k);
  const double u = z.bv[z.sz + g], v = z.bv[2 * z.sz + g], w = z.bv[3 * z.sz + g];
  z.vel[g] = sqrt(u * u + v * v + w * w);
}

static __global__ void __launch_bounds__(256) velocity_kernel(DevZone z) {
  velocity_cells(z, blockIdx.x, blockIdx.y, blockIdx.z);
}

// local time step and global minimum; dt_bits holds the IEEE bits of a
// positive double, whose unsigned order equals the numeric order
template <int NS>
__device__ __forceinline__ void dt_cells(const DevZone &z, const int bx, const int by, const int bz, unsigned long long *dt_bits) {
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k = bz;
  double dtl = 1e6;
  if (i < z.mx && j < z.my) {
    const int g = gidx(z, i, j, k);
    double m[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) m[c] = met(z, g, c);
    const double gx = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    const double ge = sqrt(m[3] * m[3] + m[4] * m[4] + m[5] * m[5]);
    const double gz = sqrt(m[6] * m[6] + m[7] * m[7] + m[8] * m[8]);
    const double u = bvl(z, g, 1), v = bvl(z, g, 2), w = bvl(z, g, 3);
    const double U = u * m[0] + v * m[1] + w * m[2];
    const double V = u * m[3] + v * m[4] + w * m[5];
    const double W = u * m[6] + v * m[7] + w * m[8];
    const double a = ld(z.a + g);
    const bool d3 = z.mz > 1;
    const double sri = (fabs(U) + a * gx) + (fabs(V) + a * ge) + (d3 ? fabs(W) + a * gz : 0.0);
    const double gamma = NS == 0 ? gamma_air : ld(z.gam + g);
    const double c1 = fmax(gamma, 4.0 / 3.0) / bvl(z, g, 0);
    double c2 = ld(z.mul + g) / c_p.Pr;
    if (c_p.sst) c2 += ld(z.mut + g) / c_p.Prt;
    double srv = gx * gx + ge * ge;
    if (d3) srv += gz * gz;
    srv *= c1 * c2;
    dtl = c_p.cfl / (sri + srv);
    if (z.dt_local) z.dt_local[nidx(z, i, j, k)] = dtl;
    if (z.isr) {  // the radii DPLUR reuses (TimeAdvanceFunc.cuh:72-77)
      const int n = nidx(z, i, j, k);
      z.isr[n] = fabs(U) + a * gx;
      z.isr[z.nsz + n] = fabs(V) + a * ge;
      z.isr[2 * z.nsz + n] = d3 ? fabs(W) + a * gz : 0.0;
    }
  }
  // warp then block min
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dtl = fmin(dtl, __shfl_xor_sync(0xffffffffu, dtl, o));
  __shared__ double wmin[32];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  if ((tid & 31) == 0) wmin[tid >> 5] = dtl;
  __syncthreads();
  if (tid < 32) {
    const int nw = (blockDim.x * blockDim.y + 31) / 32;
    double v = tid < nw ? wmin[tid] : 1e6;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (tid == 0) atomicMin(dt_bits, (unsigned long long)__double_as_longlong(v));
  }
  __syncthreads();  // wmin is reused by the next tile of a tile-table launch
}

template <int NS>
__global__ void __launch_bounds__(256) dt_kernel(DevZone z, unsigned long long *dt_bits) {
  dt_cells<NS>(z, blockIdx.x, blockIdx.y, blockIdx.z, dt_bits);
}

static __global__ void dt_reset_kernel(unsigned long long *dt_bits) {
  *dt_bits = (unsigned long long)__double_as_longlong(1e6);
}

// ---------------------------------------------------------------------------
// boundary conditions. One thread per boundary point of the face range.
// ---------------------------------------------------------------------------
template <int NS>
__device__ __forceinline__ void bc_outflow_point(const DevZone &z, const BcFace &b, int with_cv, int i, int j, int k) {  // BoundCond.cuh:120-150
  const int g = gidx(z, i, j, k);
  const int step = b.dir_stride;
  for (int gg = 1; gg <= z.ngg; ++gg) {
    const int gi = g + gg * step;
    for (int l = 0; l < 6; ++l) z.bv[l * z.sz + gi] = z.bv[l * z.sz + g];
    for (int l = 0; l < c_p.n_scalar; ++l) z.sv[l * z.sz + gi] = z.sv[l * z.sz + g];
    if (c_p.sst) z.mut[gi] = z.mut[g];
    if (with_cv) cv_from_bv_point<NS>(z, gi);
  }
}

template <int NS>
__device__ __forceinline__ void bc_inflow_point(const DevZone &z, const BcFace &b, int with_cv, int i, int j, int k) {  // BoundCond.cuh:152-210
  const int g = gidx(z, i, j, k);
  const int step = b.dir_stride;
  for (int gg = 0; gg <= z.ngg; ++gg) {
    const int gi = g + gg * step;
    z.bv[gi] = b.density;
    z.bv[z.sz + gi] = b.u;
    z.bv[2 * z.sz + gi] = b.v;
    z.bv[3 * z.sz + gi] = b.w;
    z.bv[4 * z.sz + gi] = b.pressure;
    z.bv[5 * z.sz + gi] = b.temperature;
    for (int l = 0; l < c_p.n_scalar; ++l) z.sv[l * z.sz + gi] = b.sv[l];
    if (c_p.sst) z.mut[gi] = b.mut;
    if (gg == 0) z.vel[gi] = b.velocity;
    if (with_cv) {
      // compute_cv_from_bv_1_point also rewrites vel from bv (FieldOperation.cuh:40)
      cv_from_bv_point<NS>(z, gi);
    }
  }
}

static __device__ __forceinline__ void bc_symmetry_point(const DevZone &z, const BcFace &b, int, int i, int j, int k) {  // BoundCond.cuh:52-118
  const int g = gidx(z, i, j, k);
  const int step = b.dir_stride;
  const int gin = g - step;
  double kx = z.met[(3 * b.face) * z.sz + g], ky = z.met[(3 * b.face + 1) * z.sz + g];
  double kz = z.met[(3 * b.face + 2) * z.sz + g];
  const double km = sqrt(kx * kx + ky * ky + kz * kz);
  kx /= km;
  ky /= km;
  kz /= km;
  const double u1 = z.bv[z.sz + gin], v1 = z.bv[2 * z.sz + gin], w1 = z.bv[3 * z.sz + gin];
  double uk = kx * u1 + ky * v1 + kz * w1;
  const double ut = u1 - kx * uk, vt = v1 - ky * uk, wt = w1 - kz * uk;
  z.bv[z.sz + g] = ut;
  z.bv[2 * z.sz + g] = vt;
  z.bv[3 * z.sz + g] = wt;
  z.vel[g] = sqrt(ut * ut + vt * vt + wt * wt);
  z.bv[g] = z.bv[gin];
  z.bv[4 * z.sz + g] = z.bv[4 * z.sz + gin];
  z.bv[5 * z.sz + g] = z.bv[5 * z.sz + gin];
  for (int l = 0; l < c_p.n_scalar; ++l) z.sv[l * z.sz + g] = z.sv[l * z.sz + gin];
  for (int gg = 1; gg <= z.ngg; ++gg) {
    const int go = g + gg * step, gi = g - gg * step;
    z.bv[go] = z.bv[gi];
    const double u = z.bv[z.sz + gi], v = z.bv[2 * z.sz + gi], w = z.bv[3 * z.sz + gi];
    uk = kx * u + ky * v + kz * w;
    const double uo = u - 2 * uk * kx, vo = v - 2 * uk * ky, wo = w - 2 * uk * kz;
    z.bv[z.sz + go] = uo;
    z.bv[2 * z.sz + go] = vo;
    z.bv[3 * z.sz + go] = wo;
    z.vel[go] = sqrt(uo * uo + vo * vo + wo * wo);
    z.bv[4 * z.sz + go] = z.bv[4 * z.sz + gi];
    z.bv[5 * z.sz + go] = z.bv[5 * z.sz + gi];
    for (int l = 0; l < c_p.n_scalar; ++l) z.sv[l * z.sz + go] = z.sv[l * z.sz + gi];
    if (c_p.sst) z.mut[go] = z.mut[gi];
  }
}

// periodic wrap (no reference counterpart): ghost layer gg of this face takes
// the point n cells back along the face normal
static __device__ __forceinline__ void bc_periodic_point(const DevZone &z, const BcFace &b, int with_cv, int i, int j, int k) {
  const int g = gidx(z, i, j, k);
  for (int gg = 1; gg <= z.ngg; ++gg) {
    const int go = g + gg * b.dir_stride;
    const int gs = go - b.period_stride;
    for (int l = 0; l < 6; ++l) z.bv[l * z.sz + go] = z.bv[l * z.sz + gs];
    for (int l = 0; l < c_p.n_scalar; ++l) z.sv[l * z.sz + go] = z.sv[l * z.sz + gs];
    if (c_p.sst) z.mut[go] = z.mut[gs];
    z.vel[go] = z.vel[gs];
    if (with_cv)
      for (int l = 0; l < c_p.n_var; ++l) z.cv[l * z.sz + go] = z.cv[l * z.sz + gs];
  }
}

// isothermal / adiabatic no-slip wall (BoundCond.cuh:415-541); with SST, k = 0
// on the wall and in the ghosts, omega = 60 mu_w / (rho_w beta_1 d^2) from the
// wall distance d of the first interior point, mut = 0 in the ghosts
template <int NS>
__device__ __forceinline__ void bc_wall_point(const DevZone &z, const BcFace &b, int with_cv, int i, int j, int k) {
  const int g = gidx(z, i, j, k);
  const int step = b.dir_stride;
  const int gin = g - step;
  double t_wall = b.wall_temperature;
  if (!b.wall_isothermal) t_wall = z.bv[5 * z.sz + gin];
  const double p = z.bv[4 * z.sz + gin];
  double mw = mw_air;
  if constexpr (NS > 0) {
    mw = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      z.sv[l * z.sz + g] = z.sv[l * z.sz + gin];
      mw += z.sv[l * z.sz + g] * c_p.imw[l];
    }
    mw = 1 / mw;
  }
  const double rho_wall = p * mw / (t_wall * R_u);
  z.bv[g] = rho_wall;
  z.bv[z.sz + g] = 0;
  z.bv[2 * z.sz + g] = 0;
  z.bv[3 * z.sz + g] = 0;
  z.bv[4 * z.sz + g] = p;
  z.bv[5 * z.sz + g] = t_wall;
  z.vel[g] = 0;
  if (c_p.sst) {  // BoundCond.cuh:471-485: mu at the wall temperature (the mixture's at the wall species)
    double mu_wall;
    if constexpr (NS > 0) {
      double Y[NS];
#pragma unroll
      for (int l = 0; l < NS; ++l) Y[l] = z.sv[l * z.sz + g];
      mu_wall = mixture_viscosity<NS>(t_wall, Y);
    } else {
      mu_wall = sutherland(t_wall);
    }
    const double dy = z.wall[gin];
    z.sv[NS * z.sz + g] = 0;
    z.sv[(NS + 1) * z.sz + g] =
        dy > 1e-25 ? 60 * mu_wall / (rho_wall * sst::beta_1 * dy * dy) : z.sv[(NS + 1) * z.sz + gin];
  }
  if (with_cv) cv_from_bv_point<NS>(z, g);
  for (int gg = 1; gg <= z.ngg; ++gg) {
    const int gi = g - gg * step, go = g + gg * step;
    const double u_i = z.bv[z.sz + gi], v_i = z.bv[2 * z.sz + gi], w_i = z.bv[3 * z.sz + gi];
    const double p_i = z.bv[4 * z.sz + gi], t_i = z.bv[5 * z.sz + gi];
    double t_g = t_i;
    if (b.wall_isothermal) {
      t_g = 2 * t_wall - t_i;
      if (t_g <= 0.1 * t_wall) t_g = t_wall;
    }
    if constexpr (NS > 0) {
      mw = 0;
#pragma unroll
      for (int l = 0; l < NS; ++l) {
        z.sv[l * z.sz + go] = z.sv[l * z.sz + gi];
        mw += z.sv[l * z.sz + go] * c_p.imw[l];
      }
      mw = 1 / mw;
    }
    z.bv[go] = p_i * mw / (t_g * R_u);
    z.bv[z.sz + go] = -u_i;
    z.bv[2 * z.sz + go] = -v_i;
    z.bv[3 * z.sz + go] = -w_i;
    z.bv[4 * z.sz + go] = p_i;
    z.bv[5 * z.sz + go] = t_g;
    if (c_p.sst) {
      z.sv[NS * z.sz + go] = 0;
      z.sv[(NS + 1) * z.sz + go] = z.sv[(NS + 1) * z.sz + g];
      z.mut[go] = 0;
    }
    if (with_cv) cv_from_bv_point<NS>(z, go);
  }
}

// Riemann-invariant far field (BoundCond.cuh:212-413); like the reference, it
// never recomputes cv. The mixture's gamma iteration, unbounded in the
// reference, stops after 100 sweeps here.
template <int NS>
__device__ __forceinline__ void bc_farfield_point(const DevZone &z, const BcFace &b, int, int i, int j, int k) {
  const int g = gidx(z, i, j, k);
  const int step = b.dir_stride;
  double nx = z.met[(3 * b.face) * z.sz + g], ny = z.met[(3 * b.face + 1) * z.sz + g];
  double nz = z.met[(3 * b.face + 2) * z.sz + g];
  const double gni = b.direction / sqrt(nx * nx + ny * ny + nz * nz);
  nx *= gni;
  ny *= gni;
  nz *= gni;
  const double u_b = z.bv[z.sz + g], v_b = z.bv[2 * z.sz + g], w_b = z.bv[3 * z.sz + g];
  const double u_face = nx * u_b + ny * v_b + nz * w_b;
  double gamma_b = gamma_air, mw = mw_air;
  // boundary scalars start from the point's own; for air with SST the
  // reference leaves them unset on subsonic outflow (uninitialised sv_b,
  // BoundCond.cuh:244, 330-336), where the point's own values are kept here
  double sv_b[NS + 2];
  for (int l = 0; l < c_p.n_scalar && l < NS + 2; ++l) sv_b[l] = z.sv[l * z.sz + g];
  if constexpr (NS > 0) {
    double mw_inv = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) mw_inv += sv_b[l] * c_p.imw[l];
    gamma_b = z.gam[g];
    mw = 1.0 / mw_inv;
  }
  const double p_b = z.bv[4 * z.sz + g], rho_b = z.bv[g];
  const double a_b = sqrt(gamma_b * p_b / rho_b);
  const double mach_b = u_face / a_b;
  auto fill = [&](double rho, double u, double v, double w, double p, double T, const double *svv, double mut,
                  bool node) {
    for (int gg = node ? 0 : 1; gg <= z.ngg; ++gg) {
      const int go = g + gg * step;
      z.bv[go] = rho;
      z.bv[z.sz + go] = u;
      z.bv[2 * z.sz + go] = v;
      z.bv[3 * z.sz + go] = w;
      z.bv[4 * z.sz + go] = p;
      z.bv[5 * z.sz + go] = T;
      for (int l = 0; l < c_p.n_scalar; ++l) z.sv[l * z.sz + go] = svv[l];
      if (c_p.sst) z.mut[go] = mut;
    }
    if (node) z.vel[g] = sqrt(u * u + v * v + w * w);
  };
  if (mach_b <= -1) {
    fill(b.density, b.u, b.v, b.w, b.pressure, b.temperature, b.sv, b.mut, true);
  } else if (mach_b >= 1) {
    for (int gg = 1; gg <= z.ngg; ++gg) {
      const int go = g + gg * step;
      for (int l = 0; l < 6; ++l) z.bv[l * z.sz + go] = z.bv[l * z.sz + g];
      for (int l = 0; l < c_p.n_scalar; ++l) z.sv[l * z.sz + go] = z.sv[l * z.sz + g];
      if (c_p.sst) z.mut[go] = z.mut[g];
    }
  } else {
    const double r_pos = u_face + 2 * a_b / (gamma_b - 1);
    const double u_inf = b.u * nx + b.v * ny + b.w * nz;
    const double r_neg = u_inf - 2 * b.acoustic_speed / (b.specific_heat_ratio - 1);
    const double Un = 0.5 * (r_pos + r_neg);
    double s_b, rho, p, T, u, v, w;
    const double mut_b = mach_b <= 0 && (NS == 0 || mach_b < 0) ? b.mut : (c_p.sst ? z.mut[g] : 0.0);
    if constexpr (NS == 0) {
      const double c_b = 0.25 * (gamma_air - 1) * (r_pos - r_neg);
      if (mach_b <= 0) {
        s_b = b.entropy;
        u = b.u + (Un - u_inf) * nx;
        v = b.v + (Un - u_inf) * ny;
        w = b.w + (Un - u_inf) * nz;
        for (int l = 0; l < c_p.n_scalar && l < NS + 2; ++l) sv_b[l] = b.sv[l];
      } else {
        s_b = p_b / pow(rho_b, gamma_air);
        u = u_b + (Un - u_face) * nx;
        v = v_b + (Un - u_face) * ny;
        w = w_b + (Un - u_face) * nz;
      }
      rho = pow(c_b * c_b / (gamma_air * s_b), 1 / (gamma_air - 1));
      p = rho * c_b * c_b / gamma_air;
      T = p * mw_air / (rho * R_u);
      fill(rho, u, v, w, p, T, sv_b, mut_b, true);
    } else {
      if (mach_b < 0) {
        u = b.u + (Un - u_inf) * nx;
        v = b.v + (Un - u_inf) * ny;
        w = b.w + (Un - u_inf) * nz;
        for (int l = 0; l < c_p.n_scalar && l < NS + 2; ++l) sv_b[l] = b.sv[l];  // species, k, omega
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
        s_b = mach_b <= 0 ? b.entropy : p_b / pow(rho_b, gamma);
        rho = pow(c_b * c_b / (gamma * s_b), 1 / (gamma - 1));
        p = rho * c_b * c_b / gamma;
        T = p * mw / (rho * R_u);
        double cp[NS];
        cp_only<NS>(T, cp);
        double cp_tot = 0;
#pragma unroll
        for (int l = 0; l < NS; ++l) cp_tot += cp[l] * sv_b[l];
        gamma = cp_tot / (cp_tot - R_u / mw);
        err = fabs(1 - gamma / gamma_last);
      }
      fill(rho, u, v, w, p, T, sv_b, mut_b, true);
    }
  }
}

// back pressure: extrapolate all but p (BoundCond.cuh:636-671)
template <int NS>
__device__ __forceinline__ void bc_back_pressure_point(const DevZone &z, const BcFace &b, int with_cv, int i, int j, int k) {
  const int g = gidx(z, i, j, k);
  for (int gg = 1; gg <= z.ngg; ++gg) {
    const int go = g + gg * b.dir_stride;
    for (int l = 0; l < 4; ++l) z.bv[l * z.sz + go] = z.bv[l * z.sz + g];
    z.bv[4 * z.sz + go] = b.pressure;
    z.bv[5 * z.sz + go] = z.bv[5 * z.sz + g];
    for (int l = 0; l < c_p.n_scalar; ++l) z.sv[l * z.sz + go] = z.sv[l * z.sz + g];
    if (c_p.sst) z.mut[go] = z.mut[g];
    if (with_cv) cv_from_bv_point<NS>(z, go);
  }
}

// subsonic inflow from total conditions, air (BoundCond.cuh:528-634)
static __device__ __forceinline__ void bc_subsonic_inflow_point(const DevZone &z, const BcFace &b, int with_cv, int i, int j, int k) {
  const int g = gidx(z, i, j, k);
  double nx = z.met[(3 * b.face) * z.sz + g], ny = z.met[(3 * b.face + 1) * z.sz + g];
  double nz = z.met[(3 * b.face + 2) * z.sz + g];
  const double gni = b.direction / sqrt(nx * nx + ny * ny + nz * nz);
  nx *= gni;
  ny *= gni;
  nz *= gni;
  const double rho0 = z.bv[g], u0 = z.bv[z.sz + g], v0 = z.bv[2 * z.sz + g], w0 = z.bv[3 * z.sz + g];
  const double p0 = z.bv[4 * z.sz + g];
  const double u_face = nx * u0 + ny * v0 + nz * w0;
  const double a = sqrt(gamma_air * p0 / rho0);
  const double r_neg = fabs(u_face) - 2 * a / (gamma_air - 1);
  const double hti = p0 / rho0 * gamma_air / (gamma_air - 1) + 0.5 * (u0 * u0 + v0 * v0 + w0 * w0);
  constexpr double qa = 1 + 2.0 / (gamma_air - 1);
  const double qb = 2 * r_neg;
  const double qc = (gamma_air - 1) * (0.5 * r_neg * r_neg - hti);
  const double delta = qb * qb - 4 * qa * qc;
  double a_new = a;
  if (delta >= 0) {
    const double ap = (-qb + sqrt(delta)) / (2 * qa), am = (-qb - sqrt(delta)) / (2 * qa);
    a_new = ap > am ? ap : am;
  }
  const double u_new = r_neg + 2 * a_new / (gamma_air - 1);
  const double mach = u_new / a_new;
  const double p = b.total_pressure * pow(1 + 0.5 * (gamma_air - 1) * mach * mach, -gamma_air / (gamma_air - 1));
  const double T = b.total_temperature * pow(p / b.total_pressure, (gamma_air - 1) / gamma_air);
  const double rho = p * mw_air / (T * R_u);
  for (int gg = 1; gg <= z.ngg; ++gg) {
    const int go = g + gg * b.dir_stride;
    z.bv[go] = rho;
    z.bv[z.sz + go] = u_new * b.u;
    z.bv[2 * z.sz + go] = u_new * b.v;
    z.bv[3 * z.sz + go] = u_new * b.w;
    z.bv[4 * z.sz + go] = p;
    z.bv[5 * z.sz + go] = T;
    const double u_bar = z.bv[z.sz + go] * nx + z.bv[2 * z.sz + go] * ny + z.bv[3 * z.sz + go] * nz;
    for (int l = 0; l < c_p.n_scalar; ++l) z.sv[l * z.sz + go] = u_bar > 0 ? z.sv[l * z.sz + g] : b.sv[l];
    if (c_p.sst) z.mut[go] = z.mut[g];
    if (with_cv) cv_from_bv_point<0>(z, go);
  }
}

// per-face kernels: the launch of one face's points (launch_bc)
#define OSTC_BC_KERNEL(name, point)                                      \
  __global__ void name(DevZone z, BcFace b, int with_cv) {               \
    const int i = b.rs[0] + blockIdx.x * blockDim.x + threadIdx.x;       \
    const int j = b.rs[1] + blockIdx.y * blockDim.y + threadIdx.y;       \
    const int k = b.rs[2] + blockIdx.z;                                  \
    if (i > b.re[0] || j > b.re[1] || k > b.re[2]) return;               \
    point(z, b, with_cv, i, j, k);                                       \
  }
template <int NS>
OSTC_BC_KERNEL(bc_outflow_kernel, bc_outflow_point<NS>)
template <int NS>
OSTC_BC_KERNEL(bc_inflow_kernel, bc_inflow_point<NS>)
static OSTC_BC_KERNEL(bc_symmetry_kernel, bc_symmetry_point)
static OSTC_BC_KERNEL(bc_periodic_kernel, bc_periodic_point)
template <int NS>
OSTC_BC_KERNEL(bc_wall_kernel, bc_wall_point<NS>)
template <int NS>
OSTC_BC_KERNEL(bc_farfield_kernel, bc_farfield_point<NS>)
template <int NS>
OSTC_BC_KERNEL(bc_back_pressure_kernel, bc_back_pressure_point<NS>)
static OSTC_BC_KERNEL(bc_subsonic_inflow_kernel, bc_subsonic_inflow_point)
#undef OSTC_BC_KERNEL

// one point of a boundary face of any type (the face records of the wave
// launches carry the type)
template <int NS>
__device__ __forceinline__ void bc_point(const DevZone &z, const BcFace &b, int with_cv, int i, int j, int k) {
  switch (b.type) {
    case OSTC_BC_OUTFLOW: bc_outflow_point<NS>(z, b, with_cv, i, j, k); break;
    case OSTC_BC_INFLOW: bc_inflow_point<NS>(z, b, with_cv, i, j, k); break;
    case OSTC_BC_SYMMETRY: bc_symmetry_point(z, b, with_cv, i, j, k); break;
    case OSTC_BC_WALL: bc_wall_point<NS>(z, b, with_cv, i, j, k); break;
    case OSTC_BC_FARFIELD: bc_farfield_point<NS>(z, b, with_cv, i, j, k); break;
    case OSTC_BC_BACK_PRESSURE: bc_back_pressure_point<NS>(z, b, with_cv, i, j, k); break;
    case OSTC_BC_SUBSONIC_INFLOW: bc_subsonic_inflow_point(z, b, with_cv, i, j, k); break;
    case OSTC_BC_PERIODIC: bc_periodic_point(z, b, with_cv, i, j, k); break;
    default: break;
  }
}

// 1-to-1 interface (inner_communication, DataCommunication.cuh:58-110): ghosts
// take the partner's values, the coincident plane the average of both blocks
template <int NS>
__device__ __forceinline__ void interface_point(const DevZone &z, const DevZone &t, const Iface &f, int with_cv,
                                                int n0, int n1, int n2) {
  const int n[3] = {n0, n1, n2};
  int idx[3], d[3], it[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    d[a] = f.ld[a] * n[a];
    idx[a] = f.rs[a] + d[a];
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) it[a] = f.ts[a] + f.tld[a] * d[f.st[a]];
  const int g = gidx(z, idx[0], idx[1], idx[2]);
  const int gt = gidx(t, it[0], it[1], it[2]);
  const int plane = f.direction > 0 ? f.rs[f.face] : f.rs[f.face] + f.ld[f.face] * (f.np[f.face] - 1);
  if (idx[f.face] == plane) {
    for (int l = 0; l < 6; ++l) {
      const double ave = 0.5 * (t.bv[l * t.sz + gt] + z.bv[l * z.sz + g]);
      z.bv[l * z.sz + g] = ave;
      t.bv[l * t.sz + gt] = ave;
    }
    for (int l = 0; l < c_p.n_scalar; ++l) {
      const double ave = 0.5 * (t.sv[l * t.sz + gt] + z.sv[l * z.sz + g]);
      z.sv[l * z.sz + g] = ave;
      t.sv[l * t.sz + gt] = ave;
    }
    const double u = z.bv[z.sz + g], v = z.bv[2 * z.sz + g], w = z.bv[3 * z.sz + g];
    const double vel = sqrt(u * u + v * v + w * w);
    z.vel[g] = vel;
    t.vel[gt] = vel;
  } else {
    for (int l = 0; l < 6; ++l) z.bv[l * z.sz + g] = t.bv[l * t.sz + gt];
    for (int l = 0; l < c_p.n_scalar; ++l) z.sv[l * z.sz + g] = t.sv[l * t.sz + gt];
  }
  if (with_cv) cv_from_bv_point<NS>(z, g);
}

template <int NS>
__global__ void interface_kernel(DevZone z, DevZone t, Iface f, int with_cv) {
  const int n0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int n1 = blockIdx.y * blockDim.y + threadIdx.y;
  const int n2 = blockIdx.z;
  if (n0 >= f.np[0] || n1 >= f.np[1] || n2 >= f.np[2]) return;
  interface_point<NS>(z, t, f, with_cv, n0, n1, n2);
}

// ---------------------------------------------------------------------------
// the waves of one call in one cooperative launch: boundary faces (KIND 0,
// every priority level's faces, then the periodic ones) or interfaces (KIND
// 1, in the order of data_communication). The faces of a wave touch disjoint
// cells; every CTA walks wave w's tiles and then waits at a grid barrier until
// all CTAs have finished wave w, so wave w + 1 reads what wave w wrote. The
// barrier counts arrivals in the context's WaveSync. Each wait is bounded by
// the global timer: a CTA whose wait runs out sets abort (every other wait
// then ends at once) and timed_out, which the host reads after the step; the
// waves after it are not computed. The last CTA to leave resets the counters
// for the next launch on the stream.
// ---------------------------------------------------------------------------
constexpr unsigned long long kWaveWaitNs = 1000000000ull;  // 1 s

__device__ __forceinline__ unsigned long long wave_clock() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// thread (0, 0) of a CTA: arrive, then wait until `target` arrivals in all
__device__ __forceinline__ bool wave_barrier(WaveSync *s, unsigned target) {
  __threadfence();  // this CTA's writes of the wave before its arrival
  atomicAdd(&s->arrive, 1u);
  const bool held = *(volatile int *)&s->hold != 0;
  const unsigned long long t0 = wave_clock();
  for (unsigned it = 0;; ++it) {
    unsigned a;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(a) : "l"(&s->arrive) : "memory");
    if (a >= target && !held) {
      __threadfence();
      return true;
    }
    if (*(volatile int *)&s->abort) return false;
    if ((it & 15) == 15 && wave_clock() - t0 > kWaveWaitNs) {
      atomicExch(&s->timed_out, 1);
      atomicExch(&s->abort, 1);
      return false;
    }
    if (it >= 4) __nanosleep(64);  // fewer polls of the one counter every CTA waits on
  }
}

template <int NS, int KIND>
__global__ void __launch_bounds__(256) waves_kernel(const void *records, const int4 *tiles, const int *ends,
                                                    int n_waves, int with_cv, WaveSync *sync) {
  __shared__ int go_on;
  const bool lead = threadIdx.x == 0 && threadIdx.y == 0;
  int begin = 0;
  for (int w = 0; w < n_waves; ++w) {
    const int end = ends[w];
    for (int q = begin + blockIdx.x; q < end; q += gridDim.x) {
      const int4 c = tiles[q];
      // a tile spans the face's two tangential axes (32 along the first, 8
      // along the second) at one layer along its normal (wave_axes)
      const int u = c.y * 32 + threadIdx.x, v = c.z * 8 + threadIdx.y, w = c.w;
      if constexpr (KIND == 0) {
        const BcFace &b = static_cast<const BcFace *>(records)[c.x];
        const int f = b.face;
        const int i = b.rs[0] + (f == 0 ? w : u);
        const int j = b.rs[1] + (f == 1 ? w : (f == 0 ? u : v));
        const int k = b.rs[2] + (f == 2 ? w : v);
        if (i <= b.re[0] && j <= b.re[1] && k <= b.re[2]) bc_point<NS>(c_zones[b.zone], b, with_cv, i, j, k);
      } else {
        // an interface normal to i (a few layers along i, the fastest index):
        // each warp covers 4 layers x 8 points along j, so that the layers of
        // a row share their sectors; the other faces as the boundary faces
        const Iface &f = static_cast<const Iface *>(records)[c.x];
        const int nf = f.face;
        int n0, n1, n2;
        if (nf == 0) {
          n0 = c.w * 4 + (threadIdx.x & 3);
          n1 = c.y * 8 + (threadIdx.x >> 2);
          n2 = c.z * 8 + threadIdx.y;
        } else {
          n0 = u, n1 = nf == 1 ? w : v, n2 = nf == 2 ? w : v;
        }
        if (n0 < f.np[0] && n1 < f.np[1] && n2 < f.np[2])
          interface_point<NS>(c_zones[f.zone], c_zones[f.target], f, with_cv, n0, n1, n2);
      }
    }
    begin = end;
    if (w + 1 < n_waves) {
      __syncthreads();
      if (lead) go_on = wave_barrier(sync, (unsigned)(w + 1) * gridDim.x) ? 1 : 0;
      __syncthreads();
      if (!go_on) break;
    }
  }
  if (lead) {
    __threadfence();
    if (atomicAdd(&sync->done, 1u) == gridDim.x - 1) {
      // every CTA has left its last wait: reset for the next launch
      sync->arrive = 0;
      sync->abort = 0;
      __threadfence();
      sync->done = 0;
    }
  }
}

// ---------------------------------------------------------------------------
// residual: store_last_step (TimeAdvanceFunc.cu:6-17), square of the change
// and deterministic two-level sums (Residual.cuh:57-111, Residual.cu:49-89)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void store_last_cells(const DevZone &z, const int bx, const int by, const int bz) {
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k = bz;
  if (i >= z.mx || j >= z.my) return;
  const int g = gidx(z, i, j, k), n = nidx(z, i, j, k);
  z.bv_last[n] = z.bv[g];
  z.bv_last[z.nsz + n] = z.vel[g];
  z.bv_last[2 * z.nsz + n] = z.bv[4 * z.sz + g];
  z.bv_last[3 * z.nsz + n] = z.bv[5 * z.sz + g];
}

static __global__ void store_last_kernel(DevZone z) {
  store_last_cells(z, blockIdx.x, blockIdx.y, blockIdx.z);
}

// one partial sum of the 4 squared changes per CTA (256 threads, grid-stride)
// bad (optional): the state check of the residual epilogue. The reference
// stops when its residual is NaN (Residual.cuh:153-158); here every cell whose
// density or pressure is not positive, or whose residual terms are NaN, offers
// the key (step << 44 | block << 34 | interior cell index; the step of the
// call, at most 2^20 - 1, and a block below 1024) to an atomic minimum, so the
// host learns the first failing cell of the earliest step.
static __global__ void __launch_bounds__(256) residual_partial_kernel(DevZone z, double *partial, unsigned long long *bad,
                                                               const int *step, int block) {
  const long long n = (long long)z.mx * z.my * z.mz;
  double s[4] = {0, 0, 0, 0};
  for (long long q = blockIdx.x * 256ll + threadIdx.x; q < n; q += 256ll * gridDim.x) {
    const int i = (int)(q % z.mx);
    const int j = (int)((q / z.mx) % z.my);
    const int k = (int)(q / ((long long)z.mx * z.my));
    const int g = gidx(z, i, j, k);
    const double d0 = z.bv[g] - z.bv_last[q];
    const double d1 = z.vel[g] - z.bv_last[z.nsz + q];
    const double d2 = z.bv[4 * z.sz + g] - z.bv_last[2 * z.nsz + q];
    const double d3 = z.bv[5 * z.sz + g] - z.bv_last[3 * z.nsz + q];
    if (bad && !(z.bv[g] > 0 && z.bv[4 * z.sz + g] > 0 && d0 == d0 && d1 == d1 && d2 == d2 && d3 == d3)) {
      const unsigned long long st = step ? (unsigned long long)min(*step, (1 << 20) - 1) : 0ull;
      atomicMin(bad, (st << 44) | ((unsigned long long)(block & 1023) << 34) | (unsigned long long)q);
    }
    s[0] += d0 * d0;
    s[1] += d1 * d1;
    s[2] += d2 * d2;
    s[3] += d3 * d3;
  }
  __shared__ double red[4][256];
#pragma unroll
  for (int l = 0; l < 4; ++l) red[l][threadIdx.x] = s[l];
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o)
#pragma unroll
      for (int l = 0; l < 4; ++l) red[l][threadIdx.x] += red[l][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int l = 0; l < 4; ++l) partial[blockIdx.x * 4 + l] = red[l][0];
}

// sums n_part partials (fixed order) of every zone and writes sqrt(sum / n_total)
static __global__ void residual_final_kernel(const double *partial, int n_part, double n_total, double *out) {
  const int l = threadIdx.x;
  if (l >= 4) return;
  double s = 0;
  for (int p = 0; p < n_part; ++p) s += partial[p * 4 + l];
  out[l] = sqrt(s / n_total);
}

// ---------------------------------------------------------------------------
// tile-table form of the per-cell kernels: a persistent grid of 32 x 8
// CTAs walks {zone, bx, by, bz} tiles of every zone (zones in c_zones)
// ---------------------------------------------------------------------------
template <class Op>
__global__ void __launch_bounds__(256) cells_table_kernel(const int4 *tiles, int n_tiles, Op op) {
  for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    const int4 c = tiles[t];
    op(c_zones[c.x], c.y, c.z, c.w);
  }
}

template <int NS, int SPEC>
struct SourceOp {
  __device__ void operator()(const DevZone &z, int bx, int by, int bz) const { source_cells<NS, SPEC>(z, bx, by, bz); }
};
template <int NS>
struct UpdateOp {
  double dt;
  const double *dt_dev;
  int rk;
  __device__ void operator()(const DevZone &z, int bx, int by, int bz) const {
    update_rk_cells<NS>(z, bx, by, bz, dt, dt_dev, rk);
  }
};
template <int NS>
struct PropertiesOp {
  __device__ void operator()(const DevZone &z, int bx, int by, int bz) const { properties_cells<NS>(z, bx, by, bz); }
};
template <int NS>
struct CvOp {
  __device__ void operator()(const DevZone &z, int bx, int by, int bz) const { cv_from_bv_cells<NS>(z, bx, by, bz); }
};
struct VelocityOp {
  __device__ void operator()(const DevZone &z, int bx, int by, int bz) const { velocity_cells(z, bx, by, bz); }
};
template <int NS>
struct DtOp {
  unsigned long long *dt_bits;
  __device__ void operator()(const DevZone &z, int bx, int by, int bz) const { dt_cells<NS>(z, bx, by, bz, dt_bits); }
};
struct StoreLastOp {
  __device__ void operator()(const DevZone &z, int bx, int by, int bz) const { store_last_cells(z, bx, by, bz); }
};
template <int NS>
struct InitMutOp {
  __device__ void operator()(const DevZone &z, int bx, int by, int bz) const { init_mut_cells<NS>(z, bx, by, bz); }
};

}  // namespace ostc

#include "steady.cuh"
#include "surrogate.cuh"

namespace ostc {

// ---------------------------------------------------------------------------
// host-side launchers (kernels.cuh)
// ---------------------------------------------------------------------------
namespace {
dim3 plane_grid(int nx, int ny, int nz, dim3 blk) {
  return dim3((nx + blk.x - 1) / blk.x, (ny + blk.y - 1) / blk.y, nz);
}

// persistent launch of cells_table_kernel<Op>: every resident CTA slot, at most one per tile
template <class Op>
cudaError_t launch_table(const CellTable &tab, const Op &op, cudaStream_t s) {
  if (tab.n <= 0) return cudaSuccess;
  int per_sm = 0, dev = 0, sms = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cells_table_kernel<Op>, 256, 0);
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const int slots = per_sm * sms;
  if (slots <= 0) return cudaErrorInvalidConfiguration;
  cells_table_kernel<Op><<<tab.n < slots ? tab.n : slots, dim3(32, 8), 0, s>>>(tab.tiles, tab.n, op);
  return cudaGetLastError();
}
}  // namespace

#ifndef OSTC_NS_UNIT
cudaError_t upload_zones(const DevZone *z, int n, cudaStream_t s) {
  if (n < 0 || n > kMaxTableZones) return cudaErrorInvalidValue;
  cudaError_t e = n ? cudaMemcpyToSymbolAsync(c_zones, z, sizeof(DevZone) * n, 0, cudaMemcpyHostToDevice, s)
                    : cudaSuccess;
  if (e == cudaSuccess) e = upload_zones_flux0(z, n, s);
  if (e == cudaSuccess) e = upload_zones_flux9(z, n, s);
  if (e == cudaSuccess) e = upload_zones_flux0t(z, n, s);
  if (e == cudaSuccess) e = upload_zones_flux9t(z, n, s);
  if (e == cudaSuccess) e = upload_zones_ns_a(z, n, s);
  if (e == cudaSuccess) e = upload_zones_flux_ns_a(z, n, s);
  if (e == cudaSuccess) e = upload_zones_ns_b(z, n, s);
  if (e == cudaSuccess) e = upload_zones_flux_ns_b(z, n, s);
  if (e == cudaSuccess) e = upload_zones_ns_c(z, n, s);
  if (e == cudaSuccess) e = upload_zones_flux_ns_c(z, n, s);
  if (e == cudaSuccess) e = upload_zones_ns_d(z, n, s);
  if (e == cudaSuccess) e = upload_zones_flux_ns_d(z, n, s);
  return e;
}
#endif  // OSTC_NS_UNIT

template <int NS>
cudaError_t launch_cells_table(CellOp op, const CellTable &tab, const CellArgs &a, cudaStream_t s) {
  switch (op) {
    case CellOp::Source:
      return a.spec ? launch_table(tab, SourceOp<NS, 1>{}, s) : launch_table(tab, SourceOp<NS, 0>{}, s);
    case CellOp::UpdateRK: return launch_table(tab, UpdateOp<NS>{a.dt, a.dt_dev, a.rk}, s);
    case CellOp::Properties: return launch_table(tab, PropertiesOp<NS>{}, s);
    case CellOp::CvFromBv: return launch_table(tab, CvOp<NS>{}, s);
    case CellOp::Velocity: return launch_table(tab, VelocityOp{}, s);
    case CellOp::Dt: return launch_table(tab, DtOp<NS>{a.dt_bits}, s);
    case CellOp::StoreLast: return launch_table(tab, StoreLastOp{}, s);
    case CellOp::InitMut: return launch_table(tab, InitMutOp<NS>{}, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int NS>
cudaError_t launch_cells(CellOp op, const DevZone &z, const CellArgs &a, cudaStream_t s) {
  const dim3 blk(32, 8);
  switch (op) {
    case CellOp::Source:
      if (a.spec)
        source_kernel<NS, 1><<<plane_grid(z.mx, z.my, z.mz, blk), blk, 0, s>>>(z);
      else
        source_kernel<NS, 0><<<plane_grid(z.mx, z.my, z.mz, blk), blk, 0, s>>>(z);
      break;
    case CellOp::UpdateRK:
      update_rk_kernel<NS><<<plane_grid(z.mx, z.my, z.mz, blk), blk, 0, s>>>(z, a.dt, a.dt_dev, a.rk);
      break;
    case CellOp::Properties:
      properties_kernel<NS><<<plane_grid(z.mx + 2, z.my + 2, z.mz + 2, blk), blk, 0, s>>>(z);
      break;
    case CellOp::InitMut:
      init_mut_kernel<NS><<<plane_grid(z.mx + 2, z.my + 2, z.mz + 2, blk), blk, 0, s>>>(z);
      break;
    case CellOp::CvFromBv:
      cv_from_bv_kernel<NS>
          <<<plane_grid(z.mx + 2 * z.ngg, z.my + 2 * z.ngg, z.mz + 2 * z.ngg, blk), blk, 0, s>>>(z);
      break;
    case CellOp::Velocity:
      velocity_kernel<<<plane_grid(z.mx + 2 * z.ngg, z.my + 2 * z.ngg, z.mz + 2 * z.ngg, blk), blk, 0, s>>>(z);
      break;
    case CellOp::Dt:
      dt_kernel<NS><<<plane_grid(z.mx, z.my, z.mz, blk), blk, 0, s>>>(z, a.dt_bits);
      break;
    case CellOp::DtReset:
      dt_reset_kernel<<<1, 1, 0, s>>>(a.dt_bits);
      break;
    case CellOp::StoreLast:
      store_last_kernel<<<plane_grid(z.mx, z.my, z.mz, blk), blk, 0, s>>>(z);
      break;
    case CellOp::ResidualPartial:
      residual_partial_kernel<<<a.n_part, 256, 0, s>>>(z, a.partial, a.bad, a.step, a.block);
      break;
  }
  return cudaGetLastError();
}

#ifndef OSTC_NS_UNIT
cudaError_t launch_residual_final(const double *partial, int n_part, double n_total, double *out, cudaStream_t s) {
  residual_final_kernel<<<1, 32, 0, s>>>(partial, n_part, n_total, out);
  return cudaGetLastError();
}
#endif  // OSTC_NS_UNIT

// 2-D blocks (mz == 1): eliminate_k_gradient (FieldOperation.cuh:372-400).
// Every ghost plane k = +-1 .. +-ngg of bv, sv (and cv) becomes a copy of the
// plane k = 0, over the whole ghosted (i, j) range, so every difference
// across k vanishes.
static __global__ void eliminate_k_kernel(DevZone z, int with_cv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x - z.ngg;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - z.ngg;
  if (i >= z.mx + z.ngg || j >= z.my + z.ngg) return;
  const int g0 = gidx(z, i, j, 0);
  const long long S = z.sz;
  for (int k = 1; k <= z.ngg; ++k) {
    const int gp = g0 + k * z.d1, gm = g0 - k * z.d1;
    for (int l = 0; l < 6; ++l) z.bv[l * S + gp] = z.bv[l * S + gm] = z.bv[l * S + g0];
    for (int l = 0; l < c_p.n_scalar; ++l) z.sv[l * S + gp] = z.sv[l * S + gm] = z.sv[l * S + g0];
    if (with_cv)
      for (int l = 0; l < c_p.n_var; ++l) z.cv[l * S + gp] = z.cv[l * S + gm] = z.cv[l * S + g0];
  }
}

#ifndef OSTC_NS_UNIT
cudaError_t launch_eliminate_k(const DevZone &z, int with_cv, cudaStream_t s) {
  if (z.mz != 1) return cudaSuccess;
  const dim3 blk(32, 8);
  const dim3 grid((z.mx + 2 * z.ngg + 31) / 32, (z.my + 2 * z.ngg + 7) / 8);
  eliminate_k_kernel<<<grid, blk, 0, s>>>(z, with_cv);
  return cudaGetLastError();
}
#endif  // OSTC_NS_UNIT

template <int NS>
cudaError_t launch_bc(const DevZone &z, const BcFace &b, int with_cv, cudaStream_t s) {
  const int n0 = b.re[0] - b.rs[0] + 1, n1 = b.re[1] - b.rs[1] + 1, n2 = b.re[2] - b.rs[2] + 1;
  const dim3 blk(n0 >= 32 ? 32 : (n0 >= 8 ? 8 : 1), n1 >= 8 ? 8 : 1);
  const dim3 grid((n0 + blk.x - 1) / blk.x, (n1 + blk.y - 1) / blk.y, n2);
  switch (b.type) {
    case OSTC_BC_OUTFLOW: bc_outflow_kernel<NS><<<grid, blk, 0, s>>>(z, b, with_cv); break;
    case OSTC_BC_INFLOW: bc_inflow_kernel<NS><<<grid, blk, 0, s>>>(z, b, with_cv); break;
    case OSTC_BC_SYMMETRY: bc_symmetry_kernel<<<grid, blk, 0, s>>>(z, b, with_cv); break;
    case OSTC_BC_PERIODIC: bc_periodic_kernel<<<grid, blk, 0, s>>>(z, b, with_cv); break;
    case OSTC_BC_WALL: bc_wall_kernel<NS><<<grid, blk, 0, s>>>(z, b, with_cv); break;
    case OSTC_BC_FARFIELD: bc_farfield_kernel<NS><<<grid, blk, 0, s>>>(z, b, with_cv); break;
    case OSTC_BC_BACK_PRESSURE: bc_back_pressure_kernel<NS><<<grid, blk, 0, s>>>(z, b, with_cv); break;
    case OSTC_BC_SUBSONIC_INFLOW: bc_subsonic_inflow_kernel<<<grid, blk, 0, s>>>(z, b, with_cv); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// the waves of one call (waves_kernel): one cooperative launch of at most
// every resident CTA slot and at most the largest wave's tiles (the barrier
// needs every CTA resident at once, which a cooperative launch guarantees)
template <int NS, int KIND>
static cudaError_t launch_waves(const void *records, const WavePlan &p, int with_cv, WaveSync *sync, cudaStream_t s) {
  if (p.n_waves <= 0 || p.max_tiles <= 0) return cudaSuccess;
  if (!records || !p.tiles || !p.ends || !sync) return cudaErrorInvalidValue;
  int per_sm = 0, dev = 0, sms = 0, coop = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, waves_kernel<NS, KIND>, 256, 0);
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  if (e != cudaSuccess) return e;
  const int slots = per_sm * sms;
  if (slots < 1) return cudaErrorInvalidConfiguration;
  const int grid = p.max_tiles < slots ? p.max_tiles : slots;
  if (!coop) return cudaErrorNotSupported;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(32, 8);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  e = cudaLaunchKernelEx(&cfg, waves_kernel<NS, KIND>, records, p.tiles, p.ends, p.n_waves, with_cv, sync);
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <int NS>
cudaError_t launch_bc_waves(const BcFace *faces, const WavePlan &p, int with_cv, WaveSync *sync, cudaStream_t s) {
  return launch_waves<NS, 0>(faces, p, with_cv, sync, s);
}

template <int NS>
cudaError_t launch_interface_waves(const Iface *faces, const WavePlan &p, int with_cv, WaveSync *sync, cudaStream_t s) {
  return launch_waves<NS, 1>(faces, p, with_cv, sync, s);
}

template <int NS>
cudaError_t launch_interface(const DevZone &self, const DevZone &tar, const Iface &f, int with_cv, cudaStream_t s) {
  // launch shape of data_communication (DataCommunication.cuh:36-45)
  const dim3 blk(f.np[0] <= 2 * self.ngg + 1 ? 1 : 16, f.np[1] <= 2 * self.ngg + 1 ? 1 : 16);
  const dim3 grid((f.np[0] + blk.x - 1) / blk.x, (f.np[1] + blk.y - 1) / blk.y, f.np[2]);
  interface_kernel<NS><<<grid, blk, 0, s>>>(self, tar, f, with_cv);
  return cudaGetLastError();
}

template <int NS>
cudaError_t launch_steady(SteadyOp op, const DevZone &z, const SteadyArgs &a, const BcFace *wall, cudaStream_t s) {
  const dim3 blk(32, 8), blk4(32, 4);
  switch (op) {
    case SteadyOp::ChemImplicit:
      chem_implicit_kernel<NS><<<plane_grid(z.mx, z.my, z.mz, blk4), blk4, 0, s>>>(z);
      break;
    case SteadyOp::UpdateBv:
      update_bv_kernel<NS><<<plane_grid(z.mx, z.my, z.mz, blk), blk, 0, s>>>(z);
      break;
    case SteadyOp::TurbImplicit:
      turb_implicit_kernel<<<plane_grid(z.mx, z.my, z.mz, blk), blk, 0, s>>>(z);
      break;
    case SteadyOp::DplurDq0:
      dplur_dq0_kernel<NS><<<plane_grid(z.mx, z.my, z.mz, blk4), blk4, 0, s>>>(z, a);
      break;
    case SteadyOp::DplurSweep:
      dplur_sweep_kernel<NS><<<plane_grid(z.mx, z.my, z.mz, blk4), blk4, 0, s>>>(z, a);
      break;
    case SteadyOp::DplurFinish:
      dplur_finish_kernel<NS><<<plane_grid(z.mx, z.my, z.mz, blk), blk, 0, s>>>(z, a.dq_in);
      break;
    case SteadyOp::WallDqZero: {
      if (!wall) return cudaErrorInvalidValue;
      const BcFace &b = *wall;
      const int n0 = b.re[0] - b.rs[0] + 1, n1 = b.re[1] - b.rs[1] + 1, n2 = b.re[2] - b.rs[2] + 1;
      const dim3 wb(n0 >= 32 ? 32 : (n0 >= 8 ? 8 : 1), n1 >= 8 ? 8 : 1);
      wall_dq_zero_kernel<NS><<<dim3((n0 + wb.x - 1) / wb.x, (n1 + wb.y - 1) / wb.y, n2), wb, 0, s>>>(
          z, b, a.dq_out);
      break;
    }
  }
  return cudaGetLastError();
}

template <int NS>
cudaError_t launch_chem_integrator(int n, const double *T, const double *p, const double *Y, const double *dt,
                                   double *dY, double *dT, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  chem_integrator_kernel<NS><<<(n + 127) / 128, 128, 0, s>>>(n, T, p, Y, dt, dY, dT);
  return cudaGetLastError();
}

template <int NS>
cudaError_t launch_chem_surrogate(const mlp::Net &net, int n, const double *T, const double *p, const double *Y,
                                  const double *dt, double *dY, double *dT, const ChemScratch &w, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if constexpr (NS != mlp::NIN - 3) {
    return cudaErrorInvalidValue;
  } else {
    // the network kernel's shared-memory attribute is set by prepare_chem_surrogate
    int dev = 0, sms = 148;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(w.count, 0, sizeof(int), s)) != cudaSuccess) return e;
    const int cb = (n + 255) / 256, cells_grid = cb < 16 * sms ? cb : 16 * sms;
    chem_features_kernel<NS><<<cells_grid, 256, 0, s>>>(n, T, p, Y, dt, net.scale, net.checks, w.x, w.env);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int tiles = (n + tc::ROWS - 1) / tc::ROWS;
    surrogate_chem_kernel<<<tiles < sms ? tiles : sms, tc::THREADS, tc::SM_BYTES, s>>>(net, w.x, w.y, n, w.err);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    chem_checks_kernel<NS><<<cells_grid, 256, 0, s>>>(n, T, Y, dt, w.y, w.env, net.scale, net.checks, dY, dT, w.list,
                                                      w.count);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int fb = (n + 127) / 128;
    chem_fallback_kernel<NS><<<fb < 8 * sms ? fb : 8 * sms, 128, 0, s>>>(w.list, w.count, n, T, p, Y, dt, dY, dT);
    return cudaGetLastError();
  }
}

template <int NS>
cudaError_t launch_chem_split(int op, const DevZone &z, const double *dt_dev, double dt_fixed, double *buf,
                              long long *stats, const int *count, cudaStream_t s) {
  // buf: T [n], p [n], Y [NS][n], dt [n], dY [NS][n], dT [n]
  const long long n = z.nsz;
  double *T = buf, *p = T + n, *Y = p + n, *dt = Y + NS * n, *dY = dt + n, *dT = dY + NS * n;
  const dim3 blk(32, 8);
  if (op == 0) {
    chem_gather_kernel<NS><<<plane_grid(z.mx, z.my, z.mz, blk), blk, 0, s>>>(z, dt_dev, dt_fixed, T, p, Y, dt);
  } else if (op == 1) {
    chem_scatter_kernel<NS><<<plane_grid(z.mx, z.my, z.mz, blk), blk, 0, s>>>(z, dY, dT);
  } else {
    chem_stats_kernel<<<1, 1, 0, s>>>(stats, n, count);
  }
  return cudaGetLastError();
}

#ifndef OSTC_NS_UNIT
cudaError_t prepare_chem_surrogate() {
  return cudaFuncSetAttribute(surrogate_chem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SM_BYTES);
}

bool mechanism_is_h2air9(const int *reac_type, const int *stoi_f, const int *stoi_b, const int *reac_order, int nr,
                         int ns) {
  using namespace mech_h2air9;
  if (nr != NR || ns != NS || !reac_type || !stoi_f || !stoi_b || !reac_order) return false;
  for (int r = 0; r < NR; ++r) {
    if (reac_type[r] != mech_h2air9::reac_type[r] || reac_order[r] != mech_h2air9::reac_order[r]) return false;
    for (int l = 0; l < NS; ++l)
      if (stoi_f[r * NS + l] != mech_h2air9::stoi_f[r][l] || stoi_b[r * NS + l] != mech_h2air9::stoi_b[r][l])
        return false;
  }
  return true;
}

// any staged-flux tile wait that ran out, over all flux units (flags cleared)
cudaError_t stage_timeouts(int *any) {
  cudaError_t (*const fns[])(int *) = {stage_timeout_flux0,     stage_timeout_flux9,     stage_timeout_flux0t,
                                        stage_timeout_flux9t,    stage_timeout_flux_ns_a, stage_timeout_flux_ns_b,
                                        stage_timeout_flux_ns_c, stage_timeout_flux_ns_d};
  *any = 0;
  for (auto fn : fns) {
    int f = 0;
    const cudaError_t e = fn(&f);
    if (e != cudaSuccess) return e;
    *any |= f;
  }
  return cudaSuccess;
}

// this unit's parameters and those of the flux units (flux0.cu, flux9.cu)
cudaError_t upload_param(const DevParam &p, cudaStream_t s) {
  cudaError_t e = cudaMemcpyToSymbolAsync(c_p, &p, sizeof(DevParam), 0, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = upload_param_flux0(p, s);
  if (e == cudaSuccess) e = upload_param_flux9(p, s);
  if (e == cudaSuccess) e = upload_param_flux0t(p, s);
  if (e == cudaSuccess) e = upload_param_flux9t(p, s);
  if (e == cudaSuccess) e = upload_param_ns_a(p, s);
  if (e == cudaSuccess) e = upload_param_flux_ns_a(p, s);
  if (e == cudaSuccess) e = upload_param_ns_b(p, s);
  if (e == cudaSuccess) e = upload_param_flux_ns_b(p, s);
  if (e == cudaSuccess) e = upload_param_ns_c(p, s);
  if (e == cudaSuccess) e = upload_param_flux_ns_c(p, s);
  if (e == cudaSuccess) e = upload_param_ns_d(p, s);
  if (e == cudaSuccess) e = upload_param_flux_ns_d(p, s);
  return e;
}
#endif  // OSTC_NS_UNIT

#define OSTC_INSTANTIATE(NS)                                                                                  \
  template cudaError_t launch_cells<NS>(CellOp, const DevZone &, const CellArgs &, cudaStream_t);            \
  template cudaError_t launch_cells_table<NS>(CellOp, const CellTable &, const CellArgs &, cudaStream_t);    \
  template cudaError_t launch_bc<NS>(const DevZone &, const BcFace &, int, cudaStream_t);                    \
  template cudaError_t launch_bc_waves<NS>(const BcFace *, const WavePlan &, int, WaveSync *, cudaStream_t);   \
  template cudaError_t launch_interface_waves<NS>(const Iface *, const WavePlan &, int, WaveSync *, cudaStream_t); \
  template cudaError_t launch_interface<NS>(const DevZone &, const DevZone &, const Iface &, int, cudaStream_t); \
  template cudaError_t launch_steady<NS>(SteadyOp, const DevZone &, const SteadyArgs &, const BcFace *, cudaStream_t); \
  template cudaError_t launch_chem_integrator<NS>(int, const double *, const double *, const double *, const double *, \
                                                  double *, double *, cudaStream_t);                                  \
  template cudaError_t launch_chem_surrogate<NS>(const mlp::Net &, int, const double *, const double *, const double *, \
                                                 const double *, double *, double *, const ChemScratch &, cudaStream_t); \
  template cudaError_t launch_chem_split<NS>(int, const DevZone &, const double *, double, double *, long long *,        \
                                             const int *, cudaStream_t);

#ifndef OSTC_NS_UNIT
OSTC_INSTANTIATE(0)
OSTC_INSTANTIATE(9)
#else
// a unit of further species counts (kernels_ns*.cu): OSTC_NS_LIST(X) names
// them, OSTC_NS_UNIT the unit; its own parameter and zone copies are written
// through upload_param_<unit> / upload_zones_<unit>
OSTC_NS_LIST(OSTC_INSTANTIATE)
#define OSTC_CAT2(a, b) a##b
#define OSTC_CAT(a, b) OSTC_CAT2(a, b)
cudaError_t OSTC_CAT(upload_param_, OSTC_NS_UNIT)(const DevParam &p, cudaStream_t s) {
  return cudaMemcpyToSymbolAsync(c_p, &p, sizeof(DevParam), 0, cudaMemcpyHostToDevice, s);
}
cudaError_t OSTC_CAT(upload_zones_, OSTC_NS_UNIT)(const DevZone *z, int n, cudaStream_t s) {
  if (n < 0 || n > kMaxTableZones) return cudaErrorInvalidValue;
  return n ? cudaMemcpyToSymbolAsync(c_zones, z, sizeof(DevZone) * n, 0, cudaMemcpyHostToDevice, s) : cudaSuccess;
}
#endif

}  // namespace ostc
