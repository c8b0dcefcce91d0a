/*
 * oracle.h — CPU oracle for the OpenSTC-dev RHS, RK3 and steady time-advance paths.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain FP64 restatement of the
 * reference's algorithm on HOST arrays laid out exactly like the device
 * arrays of include/ostc.h (same ostc_zone / ostc_param / ostc_bc_face
 * structs, but every pointer is a host pointer). Only tests/, the smoke()
 * check and bench.py's cpu_baseline / reference legs may load it; the
 * product library never links or calls it.
 *
 * Parity: this port is pinned against the reference itself. The reference
 * sources are compiled unchanged for sm_100a (oracle/build_ref.sh ->
 * oracle/_ref/libostc_ref_cuda.so, driven by oracle/ref_cuda_harness.cu);
 * the GPU tests compare this port with that build case by case, and
 * tests/golden/make_golden.py stores the build's outputs on small seeded
 * cases as golden vectors (tests/golden/*.npz) that tests/test_golden_cpu.py
 * checks this port against without a GPU.
 */
#ifndef OSTC_ORACLE_H
#define OSTC_ORACLE_H
#include "../include/ostc.h"

#ifdef __cplusplus
extern "C" {
#endif

/* compute_cv_from_bv over [-ngg, m+ngg) (src/FieldOperation.cuh:43-79) */
int oracle_compute_cv_from_bv(const ostc_param *p, ostc_zone *z);
/* memset(dq) + compute_source + inviscid + viscous (src/RK.cuh:110-116) */
int oracle_compute_rhs(const ostc_param *p, ostc_zone *z);
/* same as oracle_compute_rhs, and scale[l] = max |face flux| of variable l:
 * the magnitude whose differences form dq_l (its conditioning scale) */
int oracle_flux_scale(const ostc_param *p, ostc_zone *z, double *scale);
/* local_time_step on every zone, then the global minimum (capped at 1e6) */
double oracle_global_time_step(const ostc_param *p, ostc_zone *zones, int n_zones);
/* update_cv_and_bv_rk (src/RK.cuh:197-253) */
int oracle_update_cv_and_bv_rk(const ostc_param *p, ostc_zone *z, double dt, int rk);
/* BCs in the reference priority order, then periodic faces */
int oracle_apply_boundary_conditions(const ostc_param *p, ostc_zone *zones, int n_zones,
                                     const ostc_bc_face *f, int n_faces, int with_cv);
/* update_physical_properties over [-1, m] (src/FieldOperation.cuh:112-146) */
int oracle_update_physical_properties(const ostc_param *p, ostc_zone *z);
/* 2-D blocks: the k ghost planes copy k = 0 (no-op when mz > 1) */
int oracle_eliminate_k_gradient(const ostc_param *p, ostc_zone *z, int with_cv);
/* Driver::initialize_computation + RK3_bv pre-loop */
int oracle_initialize(const ostc_config *c, const ostc_param *p, ostc_zone *zones, int n_zones,
                      const ostc_bc_face *f, int n_faces);
/* n RK3 steps; res_hist: 4 per step (RMS of d rho, d|V|, d p, d T), dt_hist: 1 per step */
int oracle_rk3_steps(const ostc_config *c, const ostc_param *p, ostc_zone *zones, int n_zones,
                     const ostc_bc_face *f, int n_faces, int n_steps,
                     double *res_hist, double *dt_hist);
/* n steady iterations (SteadySim.cuh:51-126): RHS, local dt, EPI/DA or
 * DPLUR (c->implicit_method, c->DPLUR_inner_step), update_bv, BCs and
 * interfaces without cv, properties; res_hist: 4 per step or NULL */
int oracle_steady_steps(const ostc_config *c, const ostc_param *p, ostc_zone *zones, int n_zones,
                        const ostc_bc_face *f, int n_faces, int n_steps, double *res_hist);
/* 1-to-1 interfaces used by oracle_initialize / oracle_rk3_steps (copied) */
int oracle_set_interfaces(const ostc_interface *f, int n);
/* data_communication over the registered interfaces (DataCommunication.cuh:27-110) */
int oracle_data_communication(const ostc_param *p, ostc_zone *zones, int n_zones, int with_cv);
/* point-implicit chemistry step of n states (host SoA arrays; Y, dY are
 * [n_spec][n]), as ostc_chem_point_implicit */
int oracle_chem_point_implicit(const ostc_param *p, int n, const double *T, const double *p_,
                               const double *Y, const double *dt, double *dY, double *dT);
/* chemistry source of one state (omega[n_spec], kg/m3/s), for known-answer tests */
int oracle_chemical_source(const ostc_param *p, double rho, double T, const double *Y,
                           double *omega);
/* NASA-7 enthalpy and cp per species (J/kg, J/kg/K) */
int oracle_enthalpy_cp(const ostc_param *p, double T, double *h, double *cp);
/* mixture viscosity/conductivity/rho*D of one state */
int oracle_transport(const ostc_param *p, double rho, double p_, double T, const double *Y,
                     double *mu, double *kappa, double *rhoD);
/* OpenMP threads the oracle uses (0 = library default) */
void oracle_set_threads(int n);
int oracle_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
