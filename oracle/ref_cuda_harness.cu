// ref_cuda_harness.cu — drives the REFERENCE's own CUDA kernels (compiled
// for sm_100a from the reference sources by oracle/build_ref.sh) on the same
// inputs as the B200 path. Test and measurement infrastructure: the tight
// GPU oracle of the parity tests and the "reference CUDA build" timing.
//
// It rebuilds what Driver<mix,turb> sets up (src/Driver.cu:10-35,
// src/Field.cu:133-251, src/DParameter.cu:7-159) from ostc_param /
// ostc_zone host data, and repeats the per-step sequence of RK3_bv
// (src/RK.cuh:89-170) calling the reference's launchers and kernels:
// compute_source, compute_inviscid_flux, compute_viscous_flux,
// local_time_step + min_of_arr, update_cv_and_bv_rk, the apply_* boundary
// kernels in the priority order of DBoundCond::apply_boundary_conditions
// (src/BoundCond.cuh:673-822) with its launch shapes, and
// update_physical_properties. Everything runs on the legacy default stream
// with the reference's implicit synchronisations (the per-stage dt D2H copy).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <unistd.h>
#include <vector>

// include order of the reference's own translation units (RK.cuh needs the
// I/O managers and the time-advance helpers declared first)
#include "Define.h"
#include "DParameter.cuh"
#include "Field.h"
#include "Mesh.h"
#include "Parameter.h"
#include "BoundCond.cuh"
#include "FieldOperation.cuh"
#include "DataCommunication.cuh"
#include "TimeAdvanceFunc.cuh"
#include "IOManager.h"
#include "RK.cuh"
#include "Residual.cuh"
#include "DPLUR.cuh"
#include "FiniteRateChem.cuh"
#include "SchemeSelector.cuh"
#include "SourceTerm.cuh"
#include "../include/ostc.h"
#include "../include/ostc_reference_shim.h"

using namespace cfd;

namespace cfd {
// defined in DPLUR.cu without a header declaration
__global__ void set_dq_to_0(const DParameter *param, DZone *zone, integer i_face);
}  // namespace cfd

namespace {

struct RefCtx {  // one block
  ostc_config cfg{};
  int mix = 0, n_var = 5, n_scalar = 0, n_spec = 0, ngg = 2, mx = 0, my = 0, mz = 0;
  Parameter *parameter = nullptr;
  Block *block = nullptr;
  DZone h{};
  DZone *d_zone = nullptr;
  DParameter h_param{};
  DParameter *d_param = nullptr;
  std::vector<Boundary> faces;
  std::vector<int> face_inflow;  // index into inflows, or -1
  std::vector<Inflow *> d_inflows;
  std::vector<double *> d_inflow_sv;
  std::vector<void *> d_cond;  // per face: device Wall / FarField / SubsonicInflow / BackPressure
  std::vector<InnerFace> inner;  // host copies of this block's 1-to-1 faces
  std::vector<int> inner_target;
};

struct RefMulti {  // all blocks of a run
  ostc_config cfg{};
  int mix = 0;
  int sst = 0;  // k-omega SST (Driver<Air, SST> or Driver<FR, SST>)
  std::vector<RefCtx *> blk;
};

template <typename T>
T *dcopy(const T *src, size_t n) {
  T *d = nullptr;
  cudaMalloc(&d, n * sizeof(T));
  cudaMemcpy(d, src, n * sizeof(T), cudaMemcpyHostToDevice);
  return d;
}

template <typename M, typename T>
void fill_matrix(M &m, const T *src, int r, int c) {
  m.init_with_size(r, c);
  cudaMemcpy(m.data(), src, sizeof(T) * r * c, cudaMemcpyHostToDevice);
}

size_t plane(int mx, int my, int mz, int g) { return (size_t)(mx + 2 * g) * (my + 2 * g) * (mz + 2 * g); }

// the reference's per-cell launch shape: {8, 8, 4}, or {16, 16, 1} for 2-D
// problems (RK.cuh:25-30, SteadySim.cuh:27-31)
dim3 tpb_for(int mz) { return mz == 1 ? dim3{16, 16, 1} : dim3{8, 8, 4}; }

// eliminate_k_gradient on every block of a 2-D problem (RK.cuh:147-153,
// SteadySim.cuh:101-107, Driver.cu:54-60)
template <bool with_cv>
void eliminate_k(RefMulti &m) {
  if (m.blk.empty() || m.blk[0]->mz != 1) return;
  const dim3 tpb = tpb_for(1);
  for (RefCtx *c : m.blk) {
    const int ng_1 = 2 * c->ngg - 1;
    dim3 BPG{(unsigned)((c->mx + ng_1) / tpb.x + 1), (unsigned)((c->my + ng_1) / tpb.y + 1), 1};
    eliminate_k_gradient<with_cv><<<BPG, tpb>>>(c->d_zone, c->d_param);
  }
}

void build_param(RefCtx &c, const ostc_param *p) {
  DParameter &d = c.h_param;
  d.dim = c.mz == 1 ? 2 : 3;  // DParameter.cu:9 from the mesh dimension (Mesh.cpp:612-614)
  d.n_var = p->n_var;
  d.n_scalar = p->n_scalar;
  d.n_scalar_transported = p->n_scalar;
  d.n_spec = p->n_spec;
  d.i_turb_cv = 5 + p->n_spec;
  d.inviscid_scheme = p->inviscid_scheme;
  d.reconstruction = p->reconstruction;
  d.limiter = p->limiter;
  d.entropy_fix_factor = p->entropy_fix_factor;
  d.viscous_scheme = p->viscous_scheme;
  d.rans_model = p->turbulence ? p->rans_model : 0;
  d.turb_implicit = p->turbulence ? p->turb_implicit : 0;
  d.compressibility_correction = p->turbulence ? p->compressibility_correction : 0;
  d.chemSrcMethod = p->chemSrcMethod;
  d.n_reac = p->mix_model == OSTC_MIX_FR ? p->n_reac : 0;
  d.Pr = p->Pr;
  d.cfl = p->cfl;
  d.gradPInDiffusionFlux = p->gradPInDiffusionFlux != 0;
  d.Sc = p->Sc;
  d.Prt = p->Prt;
  d.Sct = p->Sct;
  const int ns = p->n_spec;
  if (ns > 0) {
    d.mw = dcopy(p->mw, ns);
    fill_matrix(d.high_temp_coeff, p->high_temp_coeff, ns, 7);
    fill_matrix(d.low_temp_coeff, p->low_temp_coeff, ns, 7);
    d.t_low = dcopy(p->t_low, ns);
    d.t_mid = dcopy(p->t_mid, ns);
    d.t_high = dcopy(p->t_high ? p->t_high : p->t_mid, ns);
    d.LJ_potent_inv = dcopy(p->LJ_potent_inv, ns);
    d.vis_coeff = dcopy(p->vis_coeff, ns);
    fill_matrix(d.WjDivWi_to_One4th, p->WjDivWi_to_One4th, ns, ns);
    fill_matrix(d.sqrt_WiDivWjPl1Mul8, p->sqrt_WiDivWjPl1Mul8, ns, ns);
    fill_matrix(d.binary_diffusivity_coeff, p->binary_diffusivity_coeff, ns, ns);
    fill_matrix(d.kb_over_eps_jk, p->kb_over_eps_jk, ns, ns);
  }
  const int nr = d.n_reac;
  if (nr > 0) {
    d.reac_type = dcopy(p->reac_type, nr);
    fill_matrix(d.stoi_f, p->stoi_f, nr, ns);
    fill_matrix(d.stoi_b, p->stoi_b, nr, ns);
    d.reac_order = dcopy(p->reac_order, nr);
    d.A = dcopy(p->A, nr);
    d.b = dcopy(p->b, nr);
    d.Ea = dcopy(p->Ea, nr);
    d.A2 = dcopy(p->A2, nr);
    d.b2 = dcopy(p->b2, nr);
    d.Ea2 = dcopy(p->Ea2, nr);
    fill_matrix(d.third_body_coeff, p->third_body_coeff, nr, ns);
    d.troe_alpha = dcopy(p->troe_alpha, nr);
    d.troe_t3 = dcopy(p->troe_t3, nr);
    d.troe_t1 = dcopy(p->troe_t1, nr);
    d.troe_t2 = dcopy(p->troe_t2, nr);
  }
  cudaMalloc(&c.d_param, sizeof(DParameter));
  cudaMemcpy(c.d_param, &c.h_param, sizeof(DParameter), cudaMemcpyHostToDevice);
}

void build_zone(RefCtx &c, const ostc_zone *z, const ostc_param *p) {
  DZone &h = c.h;
  const int mx = z->mx, my = z->my, mz = z->mz, g = z->ngg;
  h.mx = mx;
  h.my = my;
  h.mz = mz;
  h.ngg = g;
  const size_t P = plane(mx, my, mz, g);
  h.jac.allocate_memory(mx, my, mz, g);
  cudaMemcpy(h.jac.data(), z->jac, sizeof(double) * P, cudaMemcpyHostToDevice);
  h.metric.allocate_memory(mx, my, mz, g);
  static_assert(sizeof(gxl::Matrix<real, 3, 3, 1>) == 80, "metric record");
  cudaMemcpy(h.metric.data(), z->metric, 80 * P, cudaMemcpyHostToDevice);
  h.cv.allocate_memory(mx, my, mz, p->n_var, g);
  h.bv.allocate_memory(mx, my, mz, 6, g);
  cudaMemcpy(h.bv.data(), z->bv, sizeof(double) * P * 6, cudaMemcpyHostToDevice);
  h.bv_last.allocate_memory(mx, my, mz, 4, 0);
  h.vel.allocate_memory(mx, my, mz, g);
  h.acoustic_speed.allocate_memory(mx, my, mz, g);
  h.mach.allocate_memory(mx, my, mz, g);
  h.mul.allocate_memory(mx, my, mz, g);
  h.thermal_conductivity.allocate_memory(mx, my, mz, g);
  h.sv.allocate_memory(mx, my, mz, p->n_scalar, g);
  if (p->n_scalar) cudaMemcpy(h.sv.data(), z->sv, sizeof(double) * P * p->n_scalar, cudaMemcpyHostToDevice);
  h.rho_D.allocate_memory(mx, my, mz, p->n_spec, g);
  if (p->turbulence) {  // SST arrays (Field.cu:196-207); the wall distance is an input here
    h.wall_distance.allocate_memory(mx, my, mz, g);
    cudaMemcpy(h.wall_distance.data(), z->wall_distance, sizeof(double) * P, cudaMemcpyHostToDevice);
    h.mut.allocate_memory(mx, my, mz, g);
    cudaMemset(h.mut.data(), 0, sizeof(double) * P);
    h.turb_therm_cond.allocate_memory(mx, my, mz, g);
    cudaMemset(h.turb_therm_cond.data(), 0, sizeof(double) * P);
    if (p->turb_implicit == 1) h.turb_src_jac.allocate_memory(mx, my, mz, 2, 0);
  }
  if (p->n_spec > 0) {
    h.gamma.allocate_memory(mx, my, mz, g);
    h.cp.allocate_memory(mx, my, mz, g);
    if (p->mix_model == OSTC_MIX_FR) {
      if (p->chemSrcMethod == 1)
        h.chem_src_jac.allocate_memory(mx, my, mz, p->n_spec * p->n_spec, 0);
      else if (p->chemSrcMethod == 2)
        h.chem_src_jac.allocate_memory(mx, my, mz, p->n_spec, 0);
    }
  }
  // DPLUR: one ghost layer on dq, dq0, dqk and the spectral radii (Field.cu:209-221)
  const bool dplur = c.cfg.steady && c.cfg.implicit_method == 1;
  h.dq.allocate_memory(mx, my, mz, p->n_var, dplur ? 1 : 0);
  h.inv_spectr_rad.allocate_memory(mx, my, mz, dplur ? 1 : 0);
  h.visc_spectr_rad.allocate_memory(mx, my, mz, dplur ? 1 : 0);
  if (dplur) {
    h.dq0.allocate_memory(mx, my, mz, p->n_var, 1);
    h.dqk.allocate_memory(mx, my, mz, p->n_var, 1);
  }
  h.dt_local.allocate_memory(mx, my, mz, 0);
  h.unphysical.allocate_memory(mx, my, mz, 0);
  h.qn.allocate_memory(mx, my, mz, p->n_var, g);
  if (p->inviscid_scheme == 2) h.entropy_fix_delta.allocate_memory(mx, my, mz, 1);  // Field.cu:223-226
  h.boundary = nullptr;
  if (!c.faces.empty()) h.boundary = dcopy(c.faces.data(), c.faces.size());
  h.innerface = nullptr;
  if (!c.inner.empty()) h.innerface = dcopy(c.inner.data(), c.inner.size());
  cudaMalloc(&c.d_zone, sizeof(DZone));
  cudaMemcpy(c.d_zone, &h, sizeof(DZone), cudaMemcpyHostToDevice);
}

// one kernel launch per face, launch shape of DBoundCond::apply_boundary_conditions
template <MixtureModel mix, class Turb, bool with_cv>
void apply_bcs(RefCtx &c) {
  const int order[] = {4, 6, 9, 5, 7, 3, 2};
  for (int t : order) {
    for (size_t q = 0; q < c.faces.size(); ++q) {
      const Boundary &f = c.faces[q];
      if (f.type_label != t) continue;
      uint tpb[3], bpg[3];
      for (int j = 0; j < 3; ++j) {
        const int n = f.range_end[j] - f.range_start[j] + 1;
        tpb[j] = n <= (2 * c.ngg + 1) ? 1 : 16;
        bpg[j] = (n - 1) / tpb[j] + 1;
      }
      dim3 TPB{tpb[0], tpb[1], tpb[2]}, BPG{bpg[0], bpg[1], bpg[2]};
      switch (t) {
        case 6: apply_outflow<mix, Turb, with_cv><<<BPG, TPB>>>(c.d_zone, (integer)q, c.d_param); break;
        case 5:
          apply_inflow<mix, Turb, with_cv><<<BPG, TPB>>>(c.d_zone, c.d_inflows[c.face_inflow[q]], (integer)q,
                                                              c.d_param);
          break;
        case 3: apply_symmetry<mix, Turb, with_cv><<<BPG, TPB>>>(c.d_zone, (integer)q, c.d_param); break;
        case 2:
          apply_wall<mix, Turb, with_cv><<<BPG, TPB>>>(c.d_zone, (Wall *)c.d_cond[q], c.d_param, (integer)q);
          break;
        case 4:
          apply_farfield<mix, Turb, with_cv><<<BPG, TPB>>>(c.d_zone, (FarField *)c.d_cond[q], (integer)q,
                                                                c.d_param);
          break;
        case 7:
          apply_subsonic_inflow<mix, Turb, with_cv><<<BPG, TPB>>>(c.d_zone, (SubsonicInflow *)c.d_cond[q],
                                                                       c.d_param, (integer)q);
          break;
        case 9:
          apply_back_pressure<mix, Turb, with_cv><<<BPG, TPB>>>(c.d_zone, (BackPressure *)c.d_cond[q], c.d_param,
                                                                     (integer)q);
          break;
        default: break;
      }
    }
  }
}

// data_communication (DataCommunication.cuh:27-56), inner faces only: one
// inner_communication launch per face of every block, in block order
template <MixtureModel mix, class Turb, bool with_cv>
void communicate(RefMulti &m) {
  for (RefCtx *c : m.blk) {
    for (size_t l = 0; l < c->inner.size(); ++l) {
      const InnerFace &fc = c->inner[l];
      uint tpb[3], bpg[3];
      for (int j = 0; j < 3; ++j) {
        tpb[j] = fc.n_point[j] <= (2 * c->ngg + 1) ? 1 : 16;
        bpg[j] = (fc.n_point[j] - 1) / tpb[j] + 1;
      }
      dim3 TPB{tpb[0], tpb[1], tpb[2]}, BPG{bpg[0], bpg[1], bpg[2]};
      RefCtx *t = m.blk[c->inner_target[l]];
      inner_communication<mix, Turb, with_cv><<<BPG, TPB>>>(c->d_zone, t->d_zone, (integer)l, c->d_param);
    }
  }
}

template <MixtureModel mix, class Turb>
void initialize(RefMulti &m) {
  // Driver::initialize_computation (Driver.cu:39-98) + RK3_bv pre-loop (RK.cuh:40-49)
  const dim3 tpb = tpb_for(m.blk[0]->mz);
  eliminate_k<false>(m);
  for (RefCtx *c : m.blk) apply_bcs<mix, Turb, false>(*c);
  for (RefCtx *c : m.blk) {
    const int ng_1 = 2 * c->ngg - 1;
    dim3 bpg{(unsigned)((c->mx + ng_1) / tpb.x + 1), (unsigned)((c->my + ng_1) / tpb.y + 1),
             (unsigned)((c->mz + ng_1) / tpb.z + 1)};
    compute_velocity<<<bpg, tpb>>>(c->d_zone);
    if constexpr (TurbMethod<Turb>::hasMut) initialize_mut<mix, Turb><<<bpg, tpb>>>(c->d_zone, c->d_param);
  }
  cudaDeviceSynchronize();
  communicate<mix, Turb, false>(m);
  cudaDeviceSynchronize();
  for (RefCtx *c : m.blk) {
    const int ng_1 = 2 * c->ngg - 1;
    dim3 bpg{(unsigned)((c->mx + ng_1) / tpb.x + 1), (unsigned)((c->my + ng_1) / tpb.y + 1),
             (unsigned)((c->mz + ng_1) / tpb.z + 1)};
    update_physical_properties<mix><<<bpg, tpb>>>(c->d_zone, c->d_param);
  }
  cudaDeviceSynchronize();
  for (RefCtx *c : m.blk) {
    const int ng_1 = 2 * c->ngg - 1;
    dim3 bpg{(unsigned)((c->mx + ng_1) / tpb.x + 1), (unsigned)((c->my + ng_1) / tpb.y + 1),
             (unsigned)((c->mz + ng_1) / tpb.z + 1)};
    dim3 bpg0{(unsigned)((c->mx - 1) / tpb.x + 1), (unsigned)((c->my - 1) / tpb.y + 1),
              (unsigned)((c->mz - 1) / tpb.z + 1)};
    store_last_step<<<bpg0, tpb>>>(c->d_zone);
    compute_cv_from_bv<mix, Turb><<<bpg, tpb>>>(c->d_zone, c->d_param);
  }
  cudaDeviceSynchronize();
}

template <MixtureModel mix, class Turb>
void rhs(RefCtx &c) {
  const dim3 tpb = tpb_for(c.mz);
  dim3 bpg{(unsigned)((c.mx - 1) / tpb.x + 1), (unsigned)((c.my - 1) / tpb.y + 1), (unsigned)((c.mz - 1) / tpb.z + 1)};
  cudaMemset(c.h.dq.data(), 0, c.h.dq.size() * c.n_var * sizeof(real));
  compute_source<mix, Turb><<<bpg, tpb>>>(c.d_zone, c.d_param);
  compute_inviscid_flux<mix, Turb>(*c.block, c.d_zone, c.d_param, c.n_var, *c.parameter);
  compute_viscous_flux<mix, Turb>(*c.block, c.d_zone, c.d_param, c.n_var);
}

double block_dt(RefCtx &c) {  // one block of global_time_step (TimeAdvanceFunc.cu:155-182)
  constexpr integer TPB{128};
  int num_sms, per_sm;
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, min_of_arr, TPB, 0);
  const integer size = c.mx * c.my * c.mz;
  const int n_blocks = std::min(per_sm * num_sms, (size + TPB - 1) / TPB);
  min_of_arr<<<n_blocks, TPB>>>(c.h.dt_local.data(), size);
  min_of_arr<<<1, TPB>>>(c.h.dt_local.data(), n_blocks);
  double dt_block;
  cudaMemcpy(&dt_block, c.h.dt_local.data(), sizeof(real), cudaMemcpyDeviceToHost);
  return dt_block;
}

// one block of compute_residual (Residual.cuh:57-111): the summed squares
void block_residual(RefCtx &c, double *r) {
  const dim3 tpb = tpb_for(c.mz);
  dim3 bpg{(unsigned)((c.mx - 1) / tpb.x + 1), (unsigned)((c.my - 1) / tpb.y + 1), (unsigned)((c.mz - 1) / tpb.z + 1)};
  compute_square_of_dbv<<<bpg, tpb>>>(c.d_zone);
  constexpr integer TPB{128};
  int num_sms, per_sm;
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reduction_of_dv_squared, TPB, 0);
  const integer size = c.mx * c.my * c.mz;
  const int n_blocks = std::min(per_sm * num_sms, (size + TPB - 1) / TPB);
  reduction_of_dv_squared<<<n_blocks, TPB>>>(c.h.bv_last.data(), size);
  reduction_of_dv_squared<<<1, TPB>>>(c.h.bv_last.data(), n_blocks);
  cudaMemcpy(r, c.h.bv_last.data(), 4 * sizeof(real), cudaMemcpyDeviceToHost);
}

template <MixtureModel mix, class Turb>
int steps(RefMulti &m, int n, double *res_hist, double *dt_hist) {
  // the body of RK3_bv's while loop (RK.cuh:89-170), all blocks
  const dim3 tpb = tpb_for(m.blk[0]->mz);
  auto bpg = [&](RefCtx *c, int e) {
    return dim3{(unsigned)((c->mx + e) / tpb.x + 1), (unsigned)((c->my + e) / tpb.y + 1),
                (unsigned)((c->mz + e) / tpb.z + 1)};
  };
  double n_total = 0;
  for (RefCtx *c : m.blk) n_total += (double)c->mx * c->my * c->mz;
  double dt = m.cfg.fixed_time_step ? m.cfg.dt : 1e+6;
  for (int s = 0; s < n; ++s) {
    if (res_hist)
      for (RefCtx *c : m.blk) store_last_step<<<bpg(c, -1), tpb>>>(c->d_zone);
    for (RefCtx *c : m.blk)
      cudaMemcpy(c->h.qn.data(), c->h.cv.data(), c->h.cv.size() * sizeof(real) * c->n_var, cudaMemcpyDeviceToDevice);
    for (integer rk = 0; rk < 3; ++rk) {
      for (RefCtx *c : m.blk) rhs<mix, Turb>(*c);
      if (!m.cfg.fixed_time_step) {
        for (RefCtx *c : m.blk) local_time_step<mix, Turb><<<bpg(c, -1), tpb>>>(c->d_zone, c->d_param);
        dt = 1e+6;
        for (RefCtx *c : m.blk) dt = std::min(dt, block_dt(*c));
      }
      for (RefCtx *c : m.blk) {
        update_cv_and_bv_rk<mix, Turb><<<bpg(c, -1), tpb>>>(c->d_zone, c->d_param, dt, rk);
        apply_bcs<mix, Turb, true>(*c);
      }
      communicate<mix, Turb, true>(m);
      eliminate_k<true>(m);
      for (RefCtx *c : m.blk) update_physical_properties<mix><<<bpg(c, 1), tpb>>>(c->d_zone, c->d_param);
    }
    if (res_hist) {
      double acc[4] = {0, 0, 0, 0};
      for (RefCtx *c : m.blk) {
        double r[4];
        block_residual(*c, r);
        for (int l = 0; l < 4; ++l) acc[l] += r[l];
      }
      for (int l = 0; l < 4; ++l) res_hist[4 * s + l] = std::sqrt(acc[l] / n_total);
    }
    if (dt_hist) dt_hist[s] = dt;
  }
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? 0 : 2;
}


// implicit_treatment (ImplicitTreatmentHPP.cuh:8-52) for one block; DPLUR's
// host loop (DPLUR.cuh:283-312) with set_wall_dq_to_0 (DPLUR.cu:33-52) over
// this block's wall faces
template <MixtureModel mix, class Turb>
void implicit_treatment_block(RefMulti &m, RefCtx &c) {
  const dim3 tpb = tpb_for(c.mz);
  dim3 bpg{(unsigned)((c.mx - 1) / tpb.x + 1), (unsigned)((c.my - 1) / tpb.y + 1), (unsigned)((c.mz - 1) / tpb.z + 1)};
  if (m.cfg.implicit_method == 0) {
    if constexpr (mix == MixtureModel::FR) {
      if (c.h_param.n_reac > 0 && c.h_param.chemSrcMethod == 1) EPI<<<bpg, tpb>>>(c.d_zone, c.n_spec);
      if (c.h_param.n_reac > 0 && c.h_param.chemSrcMethod == 2) DA<<<bpg, tpb>>>(c.d_zone, c.n_spec);
    }
    if constexpr (TurbMethod<Turb>::hasImplicitTreat)
      if (c.h_param.turb_implicit == 1) implicit_treat_for_SST<<<bpg, tpb>>>(c.d_zone, c.d_param);
    return;
  }
  compute_DQ_0<mix, Turb><<<bpg, tpb>>>(c.d_zone, c.d_param);
  const size_t mem = c.h.dq.size() * c.n_var * sizeof(real);
  cudaMemcpy(c.h.dq0.data(), c.h.dq.data(), mem, cudaMemcpyDeviceToDevice);
  for (int it = 0; it < m.cfg.DPLUR_inner_step; ++it) {
    for (size_t q = 0; q < c.faces.size(); ++q) {
      if (c.faces[q].type_label != 2) continue;
      const Boundary &hf = c.faces[q];
      uint tp[3], bp[3];
      for (int j = 0; j < 3; ++j) {
        const int n = hf.range_end[j] - hf.range_start[j] + 1;
        tp[j] = n <= (2 * c.ngg + 1) ? 1 : 16;
        bp[j] = (n - 1) / tp[j] + 1;
      }
      set_dq_to_0<<<dim3{bp[0], bp[1], bp[2]}, dim3{tp[0], tp[1], tp[2]}>>>(c.d_param, c.d_zone, (integer)q);
    }
    DPLUR_inner_iteration<mix, Turb><<<bpg, tpb>>>(c.d_param, c.d_zone);
    cudaMemcpy(c.h.dq.data(), c.h.dqk.data(), mem, cudaMemcpyDeviceToDevice);
  }
  convert_dq_back_to_dqDt<<<bpg, tpb>>>(c.d_zone, c.d_param);
}

template <MixtureModel mix, class Turb>
int steady_steps(RefMulti &m, int n, double *res_hist) {
  // the loop body of steady_simulation (SteadySim.cuh:51-126), all blocks
  const dim3 tpb = tpb_for(m.blk[0]->mz);
  auto bpg = [&](RefCtx *c, int e) {
    return dim3{(unsigned)((c->mx + e) / tpb.x + 1), (unsigned)((c->my + e) / tpb.y + 1),
                (unsigned)((c->mz + e) / tpb.z + 1)};
  };
  double n_total = 0;
  for (RefCtx *c : m.blk) n_total += (double)c->mx * c->my * c->mz;
  for (int s = 0; s < n; ++s) {
    if (res_hist)
      for (RefCtx *c : m.blk) store_last_step<<<bpg(c, -1), tpb>>>(c->d_zone);
    for (RefCtx *c : m.blk) {
      rhs<mix, Turb>(*c);
      local_time_step<mix, Turb><<<bpg(c, -1), tpb>>>(c->d_zone, c->d_param);
      implicit_treatment_block<mix, Turb>(m, *c);
      update_bv<mix, Turb><<<bpg(c, -1), tpb>>>(c->d_zone, c->d_param);
      apply_bcs<mix, Turb, false>(*c);
    }
    communicate<mix, Turb, false>(m);
    eliminate_k<false>(m);
    for (RefCtx *c : m.blk) update_physical_properties<mix><<<bpg(c, 1), tpb>>>(c->d_zone, c->d_param);
    if (res_hist) {
      double acc[4] = {0, 0, 0, 0};
      for (RefCtx *c : m.blk) {
        double r[4];
        block_residual(*c, r);
        for (int l = 0; l < 4; ++l) acc[l] += r[l];
      }
      for (int l = 0; l < 4; ++l) res_hist[4 * s + l] = std::sqrt(acc[l] / n_total);
    }
  }
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? 0 : 2;
}

// one block: its DZone, DParameter, boundary records and condition structs;
// f holds this block's faces only (their index is the reference's i_face)
RefCtx *make_block(const ostc_config *cfg, const ostc_param *p, const ostc_zone *z,
                   const std::vector<ostc_bc_face> &f, const std::vector<ostc_interface> &inner, int *status) {
  auto *c = new RefCtx;
  c->cfg = *cfg;
  c->mix = p->mix_model;
  c->n_var = p->n_var;
  c->n_scalar = p->n_scalar;
  c->n_spec = p->n_spec;
  c->ngg = z->ngg;
  c->mx = z->mx;
  c->my = z->my;
  c->mz = z->mz;
  c->parameter = new Parameter(std::string("/dev/null"));
  c->parameter->update_parameter("inviscid_type", p->inviscid_type);
  c->parameter->update_parameter("n_spec", p->n_spec);
  c->block = new Block(z->mx, z->my, z->mz, z->ngg, 0);
  const int nf = (int)f.size();
  for (int q = 0; q < nf; ++q) {
    const int t = f[q].type_label;
    if (t != 2 && t != 3 && t != 4 && t != 5 && t != 6 && t != 7 && t != 9) {
      delete c;
      *status = 5;  // the reference has no periodic boundary (quirk A13)
      return nullptr;
    }
    Boundary b;
    for (int d = 0; d < 3; ++d) {
      b.range_start[d] = f[q].range_start[d];
      b.range_end[d] = f[q].range_end[d];
    }
    b.type_label = f[q].type_label;
    b.face = f[q].face;
    b.direction = f[q].direction;
    c->faces.push_back(b);
    c->face_inflow.push_back(-1);
    c->d_cond.push_back(nullptr);
    // the condition structs have no default constructor: fill zeroed records of their layout
    double *dsv_c = nullptr;
    if ((t == 4 || t == 7) && p->n_scalar) dsv_c = dcopy(f[q].sv, p->n_scalar);
    if (t == 2) {
      alignas(Wall) unsigned char buf[sizeof(Wall)];
      std::memset(buf, 0, sizeof(buf));
      Wall *wl = reinterpret_cast<Wall *>(buf);
      wl->label = 2;
      wl->thermal_type = f[q].wall_isothermal ? Wall::ThermalType::isothermal : Wall::ThermalType::adiabatic;
      wl->temperature = f[q].wall_temperature;
      c->d_cond.back() = dcopy(wl, 1);
    } else if (t == 4) {
      alignas(FarField) unsigned char buf[sizeof(FarField)];
      std::memset(buf, 0, sizeof(buf));
      FarField *ff = reinterpret_cast<FarField *>(buf);
      ff->label = 4;
      ff->pressure = f[q].pressure;
      ff->temperature = f[q].temperature;
      ff->velocity = f[q].velocity;
      ff->density = f[q].density;
      ff->u = f[q].u;
      ff->v = f[q].v;
      ff->w = f[q].w;
      ff->acoustic_speed = f[q].acoustic_speed;
      ff->entropy = f[q].entropy;
      ff->sv = dsv_c;
      ff->mw = f[q].mw;
      ff->mut = f[q].mut;
      ff->specific_heat_ratio = f[q].specific_heat_ratio;
      c->d_cond.back() = dcopy(ff, 1);
    } else if (t == 7) {
      alignas(SubsonicInflow) unsigned char buf[sizeof(SubsonicInflow)];
      std::memset(buf, 0, sizeof(buf));
      SubsonicInflow *si = reinterpret_cast<SubsonicInflow *>(buf);
      si->label = 7;
      si->total_pressure = f[q].total_pressure;
      si->total_temperature = f[q].total_temperature;
      si->u = f[q].u;
      si->v = f[q].v;
      si->w = f[q].w;
      si->sv = dsv_c;
      si->mut = f[q].mut;
      c->d_cond.back() = dcopy(si, 1);
    } else if (t == 9) {
      alignas(BackPressure) unsigned char buf[sizeof(BackPressure)];
      std::memset(buf, 0, sizeof(buf));
      BackPressure *bp = reinterpret_cast<BackPressure *>(buf);
      bp->label = 9;
      bp->pressure = f[q].pressure;
      c->d_cond.back() = dcopy(bp, 1);
    }
    if (f[q].type_label == 5) {
      // cfd::Inflow has no default constructor; fill a zeroed record of its layout
      alignas(Inflow) unsigned char buf[sizeof(Inflow)];
      std::memset(buf, 0, sizeof(buf));
      Inflow *in = reinterpret_cast<Inflow *>(buf);
      in->label = 5;
      in->density = f[q].density;
      in->u = f[q].u;
      in->v = f[q].v;
      in->w = f[q].w;
      in->pressure = f[q].pressure;
      in->temperature = f[q].temperature;
      in->velocity = f[q].velocity;
      in->mut = f[q].mut;
      double *dsv = nullptr;
      if (p->n_scalar) dsv = dcopy(f[q].sv, p->n_scalar);
      in->sv = dsv;
      c->d_inflow_sv.push_back(dsv);
      c->d_inflows.push_back(dcopy(in, 1));
      c->face_inflow.back() = (int)c->d_inflows.size() - 1;
    }
  }
  // InnerFace after register_boundary (Mesh.cpp:34-178); no default constructor either
  for (const ostc_interface &s : inner) {
    alignas(InnerFace) unsigned char buf[sizeof(InnerFace)];
    std::memset(buf, 0, sizeof(buf));
    InnerFace *fc = reinterpret_cast<InnerFace *>(buf);
    for (int d = 0; d < 3; ++d) {
      fc->range_start[d] = s.range_start[d];
      fc->range_end[d] = s.range_end[d];
      fc->target_start[d] = s.target_start[d];
      fc->loop_dir[d] = s.loop_dir[d];
      fc->target_loop_dir[d] = s.target_loop_dir[d];
      fc->src_tar[d] = s.src_tar[d];
      fc->n_point[d] = s.n_point[d];
    }
    fc->face = s.face;
    fc->direction = s.direction;
    fc->target_block = s.target;
    c->inner.push_back(*fc);
    c->inner_target.push_back(s.target);
  }
  build_param(*c, p);
  build_zone(*c, z, p);
  *status = 0;
  return c;
}

}  // namespace

extern "C" {

// all blocks of a run: faces[q].block and ifaces[q].block pick the block
int ref_create_multi(const ostc_config *cfg, const ostc_param *p, const ostc_zone *z, int nz, const ostc_bc_face *f,
                     int nf, const ostc_interface *ifc, int nif, void **out) {
  if (!cfg || !p || !z || !out || nz < 1) return 1;
  if (p->mix_model != OSTC_MIX_AIR && p->mix_model != OSTC_MIX_FR) return 5;
  if (p->turbulence && p->rans_model != 2) return 5;
  for (int q = 0; q < nf; ++q)
    if (f[q].block < 0 || f[q].block >= nz) return 1;
  for (int q = 0; q < nif; ++q)
    if (ifc[q].block < 0 || ifc[q].block >= nz || ifc[q].target < 0 || ifc[q].target >= nz) return 1;
  auto *m = new RefMulti;
  m->cfg = *cfg;
  m->mix = p->mix_model;
  m->sst = p->turbulence ? 1 : 0;
  for (int b = 0; b < nz; ++b) {
    std::vector<ostc_bc_face> fb;
    std::vector<ostc_interface> ib;
    for (int q = 0; q < nf; ++q)
      if (f[q].block == b) fb.push_back(f[q]);
    for (int q = 0; q < nif; ++q)
      if (ifc[q].block == b) ib.push_back(ifc[q]);
    int st = 0;
    RefCtx *c = make_block(cfg, p, z + b, fb, ib, &st);
    if (!c) {
      delete m;
      return st;
    }
    m->blk.push_back(c);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return 2;
  *out = m;
  return 0;
}

int ref_create(const ostc_config *cfg, const ostc_param *p, const ostc_zone *z, const ostc_bc_face *f, int nf,
               void **out) {
  if (!z) return 1;
  for (int q = 0; q < nf; ++q)
    if (f[q].block != 0) return 1;
  return ref_create_multi(cfg, p, z, 1, f, nf, nullptr, 0, out);
}

int ref_initialize(void *h) {
  auto *m = (RefMulti *)h;
  if (m->sst && m->mix != OSTC_MIX_AIR)
    initialize<MixtureModel::FR, SST>(*m);
  else if (m->sst)
    initialize<MixtureModel::Air, SST>(*m);
  else if (m->mix == OSTC_MIX_AIR)
    initialize<MixtureModel::Air, Laminar>(*m);
  else
    initialize<MixtureModel::FR, Laminar>(*m);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int ref_rhs(void *h) {
  auto *m = (RefMulti *)h;
  for (RefCtx *c : m->blk) {
    if (m->sst && m->mix != OSTC_MIX_AIR)
      rhs<MixtureModel::FR, SST>(*c);
    else if (m->sst)
      rhs<MixtureModel::Air, SST>(*c);
    else if (m->mix == OSTC_MIX_AIR)
      rhs<MixtureModel::Air, Laminar>(*c);
    else
      rhs<MixtureModel::FR, Laminar>(*c);
  }
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

int ref_steps(void *h, int n, double *res_hist, double *dt_hist) {
  auto *m = (RefMulti *)h;
  if (m->sst && m->mix != OSTC_MIX_AIR) return steps<MixtureModel::FR, SST>(*m, n, res_hist, dt_hist);
  if (m->sst) return steps<MixtureModel::Air, SST>(*m, n, res_hist, dt_hist);
  return m->mix == OSTC_MIX_AIR ? steps<MixtureModel::Air, Laminar>(*m, n, res_hist, dt_hist)
                                : steps<MixtureModel::FR, Laminar>(*m, n, res_hist, dt_hist);
}

int ref_steady_steps(void *h, int n, double *res_hist) {
  auto *m = (RefMulti *)h;
  if (!m->cfg.steady) return 1;
  if (m->sst && m->mix != OSTC_MIX_AIR) return steady_steps<MixtureModel::FR, SST>(*m, n, res_hist);
  if (m->sst) return steady_steps<MixtureModel::Air, SST>(*m, n, res_hist);
  return m->mix == OSTC_MIX_AIR ? steady_steps<MixtureModel::Air, Laminar>(*m, n, res_hist)
                                : steady_steps<MixtureModel::FR, Laminar>(*m, n, res_hist);
}

// device time of n steps (CUDA events around the loop, as bench.py does for ours)
double ref_time_steps(void *h, int n) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaDeviceSynchronize();
  cudaEventRecord(e0);
  if (ref_steps(h, n, nullptr, nullptr)) return -1;
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms;
}

// copy a DZone array of block b to the host: name in {bv, sv, cv, dq, mul,
// thermal_conductivity, vel, acoustic_speed, rho_D}
int ref_download_block(void *h, int b, const char *name, double *dst) {
  auto *m = (RefMulti *)h;
  if (b < 0 || b >= (int)m->blk.size()) return 1;
  RefCtx *c = m->blk[b];
  DZone &z = c->h;
  const size_t P = plane(c->mx, c->my, c->mz, c->ngg);
  const size_t I = plane(c->mx, c->my, c->mz, 0);
  const void *src = nullptr;
  size_t n = 0;
  if (!strcmp(name, "bv")) src = z.bv.data(), n = 6 * P;
  else if (!strcmp(name, "sv")) src = z.sv.data(), n = c->n_scalar * P;
  else if (!strcmp(name, "cv")) src = z.cv.data(), n = c->n_var * P;
  else if (!strcmp(name, "dq"))  // one ghost layer under DPLUR (Field.cu:209-221)
    src = z.dq.data(), n = c->n_var * plane(c->mx, c->my, c->mz, c->cfg.steady && c->cfg.implicit_method == 1 ? 1 : 0);
  else if (!strcmp(name, "mul")) src = z.mul.data(), n = P;
  else if (!strcmp(name, "thermal_conductivity")) src = z.thermal_conductivity.data(), n = P;
  else if (!strcmp(name, "vel")) src = z.vel.data(), n = P;
  else if (!strcmp(name, "acoustic_speed")) src = z.acoustic_speed.data(), n = P;
  else if (!strcmp(name, "rho_D")) src = z.rho_D.data(), n = c->n_spec * P;
  else if (!strcmp(name, "mut") && z.mut.data()) src = z.mut.data(), n = P;
  else if (!strcmp(name, "turb_therm_cond") && z.turb_therm_cond.data()) src = z.turb_therm_cond.data(), n = P;
  else return 1;
  return cudaMemcpy(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : 2;
}

int ref_download(void *h, const char *name, double *dst) { return ref_download_block(h, 0, name, dst); }

// block b's device arrays as an ostc_zone, through the maintainer's shim
// (include/ostc_reference_shim.h) compiled against the reference's Field.h
int ref_zone_view(void *h, int b, ostc_zone *out) {
  auto *m = (RefMulti *)h;
  if (!out || b < 0 || b >= (int)m->blk.size()) return 1;
  RefCtx *c = m->blk[b];
  *out = ostc_from_reference::to_ostc(c->h, c->cfg.steady && c->cfg.implicit_method == 1 ? 1 : 0);
  return 0;
}

// Block::compute_jac_metric (Mesh.cpp:259-521), the reference's own host code,
// on caller coordinates with ngg+1 ghost layers (x, y, z in the ghosted
// layout of gxl::Array3D): fills jac (ngg ghosts) and the 80-byte metric
// records (ngg ghosts). Host only; the grid must have positive Jacobians (the
// reference logs and copies a neighbour otherwise).
int ref_metric(int mx, int my, int mz, int ngg, const double *x, const double *y, const double *z, double *jac_out,
               void *metric_out) {
  if (mx < 1 || my < 1 || mz < 1 || ngg < 1 || !x || !y || !z || !jac_out || !metric_out) return 1;
  Block b(mx, my, mz, ngg, 0);
  const size_t nc = plane(mx, my, mz, ngg + 1), np = plane(mx, my, mz, ngg);
  std::memcpy(b.x.data(), x, nc * sizeof(double));
  std::memcpy(b.y.data(), y, nc * sizeof(double));
  std::memcpy(b.z.data(), z, nc * sizeof(double));
  b.compute_jac_metric(0);
  std::memcpy(jac_out, b.jacobian.data(), np * sizeof(double));
  std::memcpy(metric_out, b.metric.data(), np * sizeof(gxl::Matrix<real, 3, 3, 1>));
  return 0;
}

// the reference's own Mesh (src/Mesh.cpp:550-588): its grid, boundary and
// inner-face files read from dir/input_files (grid   0.grd, boundary   0.txt,
// inner   0.txt), faces registered, ghost grid, metrics. Host only.
struct RefMesh {
  Parameter *parameter = nullptr;
  Mesh *mesh = nullptr;
};

int ref_mesh_read(const char *dir, int ngg, double grid_scale, void **out) {
  if (!dir || !out || ngg < 1) return 1;
  char old[4096];
  if (!getcwd(old, sizeof(old))) return 2;
  // the Parameter keys Mesh reads, in the reference's setup-file syntax
  const std::string pfile = "/tmp/ostc_ref_mesh_param_" + std::to_string((long)getpid()) + ".txt";
  {
    FILE *f = std::fopen(pfile.c_str(), "w");
    if (!f) return 2;
    std::fprintf(f, "int ngg = %d\nint n_proc = 1\nint myid = 0\nbool parallel = 0\nreal gridScale = %.17g\n", ngg,
                 grid_scale);
    std::fclose(f);
  }
  if (chdir(dir) != 0) return 2;
  auto *m = new RefMesh;
  m->parameter = new Parameter(pfile);
  m->mesh = new Mesh(*m->parameter);
  if (chdir(old) != 0) return 2;
  std::remove(pfile.c_str());
  *out = m;
  return 0;
}

int ref_mesh_counts(void *h, int *n_block, int *dimension) {
  auto *m = (RefMesh *)h;
  *n_block = m->mesh->n_block;
  *dimension = m->mesh->dimension;
  return 0;
}

// extents, and x, y, z / jac / metric with ngg ghost layers (any pointer may be NULL)
int ref_mesh_block(void *h, int b, int *dims, double *x, double *y, double *z, double *jac, void *metric) {
  auto *m = (RefMesh *)h;
  if (b < 0 || b >= m->mesh->n_block) return 1;
  Block &B = (*m->mesh)[b];
  dims[0] = B.mx, dims[1] = B.my, dims[2] = B.mz;
  const int g = B.ngg;
  const size_t np = plane(B.mx, B.my, B.mz, g);
  if (x) std::memcpy(x, B.x.data(), np * sizeof(double));
  if (y) std::memcpy(y, B.y.data(), np * sizeof(double));
  if (z) std::memcpy(z, B.z.data(), np * sizeof(double));
  if (jac) std::memcpy(jac, B.jacobian.data(), np * sizeof(double));
  if (metric) std::memcpy(metric, B.metric.data(), np * sizeof(gxl::Matrix<real, 3, 3, 1>));
  return 0;
}

// the registered boundary faces of block b: 9 ints each (range_start[3],
// range_end[3], face, direction, type_label); *n the count (out may be NULL)
int ref_mesh_boundaries(void *h, int b, int *n, int *out) {
  auto *m = (RefMesh *)h;
  Block &B = (*m->mesh)[b];
  *n = (int)B.boundary.size();
  if (out)
    for (size_t q = 0; q < B.boundary.size(); ++q) {
      const Boundary &f = B.boundary[q];
      int *o = out + 9 * q;
      for (int a = 0; a < 3; ++a) o[a] = f.range_start[a], o[3 + a] = f.range_end[a];
      o[6] = f.face, o[7] = f.direction, o[8] = f.type_label;
    }
  return 0;
}

// the registered inner faces of block b: 25 ints each (range_start[3],
// range_end[3], target_start[3], loop_dir[3], target_loop_dir[3], src_tar[3],
// n_point[3], face, direction, target_block, target_face)
int ref_mesh_inner(void *h, int b, int *n, int *out) {
  auto *m = (RefMesh *)h;
  Block &B = (*m->mesh)[b];
  *n = (int)B.inner_face.size();
  if (out)
    for (size_t q = 0; q < B.inner_face.size(); ++q) {
      const InnerFace &f = B.inner_face[q];
      int *o = out + 25 * q;
      for (int a = 0; a < 3; ++a) {
        o[a] = f.range_start[a], o[3 + a] = f.range_end[a], o[6 + a] = f.target_start[a];
        o[9 + a] = f.loop_dir[a], o[12 + a] = f.target_loop_dir[a], o[15 + a] = f.src_tar[a], o[18 + a] = f.n_point[a];
      }
      o[21] = f.face, o[22] = f.direction, o[23] = f.target_block, o[24] = f.target_face;
    }
  return 0;
}

// bytes of device memory the reference arrays of this run hold
double ref_device_bytes(void *h) {
  auto *m = (RefMulti *)h;
  double b = 0;
  for (RefCtx *c : m->blk) {
    const double P = (double)plane(c->mx, c->my, c->mz, c->ngg), I = (double)plane(c->mx, c->my, c->mz, 0);
    b += 8 * P * (1 + 10 + c->n_var * 2 + 6 + c->n_scalar + 5 + c->n_spec) + 8 * I * (4 + c->n_var + 5);
    if (c->mix == OSTC_MIX_FR && c->h_param.chemSrcMethod == 1) b += 8 * I * c->n_spec * c->n_spec;
  }
  return b;
}

}  // extern "C"
