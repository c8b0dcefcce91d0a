/*
 * ostc.h — C ABI of the B200-native right-hand-side and time-advance path of
 * the OpenSTC-dev structured-grid compressible reacting-flow solver.
 *
 * The ABI keeps the reference's device data model so that the path is a
 * drop-in for the per-stage calls made by RK3_bv (src/RK.cuh:107-161):
 *
 *   - every field array is a ColMajor ggxl::VectorField3D / Array3D
 *     (src/gxl_lib/Array.hpp:128-194): one plane per variable, i fastest,
 *     element (i,j,k,l) at  k*disp1 + j*disp2 + i + dispt + l*sz  with
 *     disp2 = mx+2g, disp1 = (my+2g)*disp2, dispt = (disp1+disp2+1)*g,
 *     sz = (mx+2g)(my+2g)(mz+2g), g = the array's own ghost count;
 *   - the metric is the reference's gxl::Matrix<double,3,3,1> per point
 *     (src/gxl_lib/Matrix.hpp:214-233): an int bias, 4 bytes of padding and
 *     9 doubles, 80 bytes per point; row d (0 = xi, 1 = eta, 2 = zeta) holds
 *     (d_x, d_y, d_z);
 *   - scheme selection uses the reference's setup-file tags
 *     (input_files/setup/2_scheme.txt, decoded in src/Parameter.cpp:165-218).
 *
 * All pointers in ostc_zone are DEVICE pointers owned by the caller (the
 * reference's Field::h_ptr members, src/Field.cu:133-251). Species and
 * reaction tables in ostc_param are HOST pointers copied at ostc_create.
 *
 * Every entry point returns an ostc_status; none aborts. Work is enqueued on
 * the stream passed in; no entry point below synchronises the host unless
 * its comment says so. The library keeps the run parameters and the zone
 * table of the context used last in constant memory and uploads them when
 * a call on another context comes first; an operator called into a caller's
 * stream capture at that moment returns OSTC_ERR_INVALID_ARG (a captured
 * upload would take effect only when the graph runs).
 */
#ifndef OSTC_H
#define OSTC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------------------- */
/* status codes                                                            */
/* ----------------------------------------------------------------------- */
typedef enum ostc_status {
  OSTC_OK = 0,
  OSTC_ERR_INVALID_ARG = 1,   /* bad pointer, size, tag or combination      */
  OSTC_ERR_CUDA = 2,          /* a CUDA runtime call failed                 */
  OSTC_ERR_TIMEOUT = 3,       /* a bounded device wait gave up              */
  OSTC_ERR_NONPHYSICAL = 4,   /* NaN / non-positive density or pressure     */
  OSTC_ERR_UNSUPPORTED = 5,   /* scheme combination not built               */
  OSTC_ERR_NO_DEVICE = 6,     /* no CUDA device visible                     */
  OSTC_ERR_IO = 7             /* a file could not be opened, read or written */
} ostc_status;

/* Mixture model, same meaning as cfd::MixtureModel (src/Define.h:19-25).  */
enum { OSTC_MIX_AIR = 0, OSTC_MIX_MIXTURE = 1, OSTC_MIX_FR = 2 };

/* Boundary labels, same numbers as the reference (src/BoundCond.h:4-11).
 * OSTC_BC_PERIODIC has no counterpart in the reference (quirk A13): it
 * wraps ghost layers from the opposite face of the same block.            */
enum {
  OSTC_BC_WALL = 2, OSTC_BC_SYMMETRY = 3, OSTC_BC_FARFIELD = 4,
  OSTC_BC_INFLOW = 5, OSTC_BC_OUTFLOW = 6, OSTC_BC_SUBSONIC_INFLOW = 7,
  OSTC_BC_BACK_PRESSURE = 9, OSTC_BC_PERIODIC = 100
};

#define OSTC_MAX_SPEC 20   /* MAX_SPEC_NUMBER of the reference build      */
#define OSTC_MAX_REAC 50   /* MAX_REAC_NUMBER of the reference build      */

/* ----------------------------------------------------------------------- */
/* data model                                                              */
/* ----------------------------------------------------------------------- */

/* One grid block: the device arrays of cfd::DZone (src/Field.h:13-71).
 * Arrays with "g=ngg" carry the block's ghost layers, "g=0" none,
 * "g=dq_ngg" the dq ghost count (0 for RK3, 1 for DPLUR, src/Field.cu:203-212).
 * Unused arrays may be NULL (see ostc_zone_required()).                    */
typedef struct ostc_zone {
  int mx, my, mz, ngg;       /* interior extents and ghost count           */
  int dq_ngg;                /* ghosts of dq/dq0/dqk/spectral radii: 0 or 1 */
  int reserved_;
  const double *x, *y, *z;   /* g=ngg; only read by ostc_metric_from_grid   */
  const double *jac;         /* g=ngg                                        */
  const void *metric;        /* g=ngg, 80-byte gxl::Matrix<real,3,3,1>      */
  double *wall_distance;     /* g=ngg (SST)                                  */
  double *cv;                /* g=ngg, n_var planes                          */
  double *bv;                /* g=ngg, 6 planes: rho,u,v,w,p,T               */
  double *sv;                /* g=ngg, n_scalar planes: Y_k, k, omega        */
  double *bv_last;           /* g=0, 4 planes (residual)                     */
  double *vel, *acoustic_speed, *mach, *mul, *thermal_conductivity; /* g=ngg */
  double *rho_D;             /* g=ngg, n_spec planes                         */
  double *gamma, *cp;        /* g=ngg (mixtures)                             */
  double *chem_src_jac;      /* g=0, n_spec^2 (EPI) or n_spec (DA) planes    */
  double *mut, *turb_therm_cond; /* g=ngg (SST)                              */
  double *turb_src_jac;      /* g=0, 2 planes (SST implicit)                 */
  double *dq, *dq0, *dqk;    /* g=dq_ngg, n_var planes                       */
  double *inv_spectr_rad;    /* g=dq_ngg, 3 interleaved doubles per point    */
  double *visc_spectr_rad;   /* g=dq_ngg                                     */
  double *dt_local;          /* g=0                                          */
  double *entropy_fix_delta; /* g=1 (Roe)                                    */
  double *qn;                /* g=ngg, n_var planes (RK3)                    */
} ostc_zone;

/* Scheme tags and physical tables: the fields of cfd::DParameter
 * (src/DParameter.cuh:13-92) plus the derived tags of
 * Parameter::deduce_known_info (src/Parameter.cpp:165-218).
 * Table pointers are HOST pointers, row-major, copied by ostc_create.      */
typedef struct ostc_param {
  int mix_model;             /* OSTC_MIX_*                                   */
  int turbulence;            /* 0 laminar, 1 RANS (SST when rans_model==2)   */
  int n_var, n_scalar, n_spec, n_reac, i_turb_cv;
  int inviscid_scheme;       /* 1 LF, 2 Roe, 3 AUSM+, 4 HLLC                 */
  int reconstruction;        /* 1 first order, 2 MUSCL, 3 NND2, 4 WENO5      */
  int limiter;               /* 0 minmod                                     */
  int inviscid_type;         /* derived: 0 pv, 1 AWENO, 2 Roe (Parameter.cpp:193-198) */
  int viscous_scheme;        /* viscous_order: 0 inviscid, 2 central         */
  int rans_model, turb_implicit, compressibility_correction;
  int chemSrcMethod;         /* 0 explicit, 1 EPI, 2 DA                      */
  int gradPInDiffusionFlux;
  int dimension;             /* 2 or 3                                       */
  double entropy_fix_factor, Pr, Prt, Sct, Sc, cfl;
  /* species tables */
  const double *mw;          /* [n_spec]                                     */
  const double *high_temp_coeff, *low_temp_coeff; /* [n_spec][7]           */
  const double *t_low, *t_mid, *t_high;           /* [n_spec]              */
  const double *LJ_potent_inv, *vis_coeff;        /* [n_spec]              */
  const double *WjDivWi_to_One4th, *sqrt_WiDivWjPl1Mul8; /* [n_spec][n_spec] */
  const double *binary_diffusivity_coeff, *kb_over_eps_jk; /* [n_spec][n_spec] */
  /* reaction tables */
  const int *reac_type;                 /* [n_reac] labels 0..7             */
  const int *stoi_f, *stoi_b;           /* [n_reac][n_spec]                 */
  const int *reac_order;                /* [n_reac]                         */
  const double *A, *b, *Ea, *A2, *b2, *Ea2; /* [n_reac]                     */
  const double *third_body_coeff;       /* [n_reac][n_spec]                 */
  const double *troe_alpha, *troe_t3, *troe_t1, *troe_t2; /* [n_reac]       */
} ostc_param;

/* One boundary face of one block: cfd::Boundary (src/Mesh.h:9-31) after
 * register_boundary (ranges already widened by ngg on tangential axes; wall
 * faces trimmed back by ngg as DBoundCond::initialize_bc_on_GPU does,
 * src/BoundCond.cu:369-387), with the state of its condition (src/BoundCond.h). */
typedef struct ostc_bc_face {
  int block;                 /* zone index                                   */
  int type_label;            /* OSTC_BC_*                                    */
  int face;                  /* 0 i, 1 j, 2 k                                */
  int direction;             /* -1 on the min face, +1 on the max face       */
  int range_start[3], range_end[3]; /* inclusive                            */
  /* inflow / farfield state (cfd::Inflow, src/BoundCond.h:23-44)           */
  double density, u, v, w, pressure, temperature, velocity, mut;
  double sv[OSTC_MAX_SPEC + 4];
  /* wall (cfd::Wall): isothermal flag and temperature                       */
  int wall_isothermal;
  double wall_temperature;
  /* farfield (cfd::FarField, src/BoundCond.h:65-87): free-stream sound speed,
   * entropy p/rho^gamma, gamma and molar mass; subsonic inflow
   * (cfd::SubsonicInflow): total pressure and temperature, u/v/w = direction;
   * back pressure (cfd::BackPressure): the pressure field above             */
  double acoustic_speed, entropy, specific_heat_ratio, mw;
  double total_pressure, total_temperature;
} ostc_bc_face;

/* One 1-to-1 interface of a block with a block of the same context:
 * cfd::InnerFace (src/Mesh.h:33-58) after InnerFace::register_boundary
 * (src/Mesh.cpp:34-178). range_* spans the ghost layers and the coincident
 * face plane along `face`; point n of the range (n = 0..n_point-1 per axis)
 * is idx = range_start + loop_dir*n, and its partner in `target` is
 * target_start[a] + target_loop_dir[a] * (loop_dir*n)[src_tar[a]].        */
typedef struct ostc_interface {
  int block, target;
  int face, direction;
  int range_start[3], range_end[3];
  int target_start[3];
  int loop_dir[3], target_loop_dir[3], src_tar[3];
  int n_point[3];
} ostc_interface;

/* Options of the time-advance path (the relevant keys of 2_scheme.txt). */
typedef struct ostc_config {
  int steady;                /* 0 unsteady (RK3), 1 steady                   */
  int temporal_scheme;       /* 3 SSPRK3                                     */
  int implicit_method;       /* 0 explicit, 1 DPLUR                          */
  int DPLUR_inner_step;
  int fixed_time_step;       /* 1: dt given; 0: CFL dt each stage (quirk A12) */
  double dt;
  int output_screen;         /* residual cadence, RK.cuh:94                 */
  int compat;                /* 1: replicate reference quirks (Appendix A)   */
  int chem_mode;             /* RK3 chemistry: 0 source term in the RHS (the
                              * reference, explicit); 1 operator split: the
                              * FP64 point-implicit integrator over each
                              * step's dt after the three stages; 2 split
                              * with the learned surrogate and FP64 fallback
                              * (ostc_set_chem_surrogate)                    */
} ostc_config;

typedef struct ostc_ctx ostc_ctx;

/* ----------------------------------------------------------------------- */
/* lifecycle                                                               */
/* ----------------------------------------------------------------------- */

/* Build a context over n_zones caller-owned blocks. Replaces the setup half
 * of Driver<mix,turb> (src/Driver.cu:10-35): copies the DParameter tables
 * and BC data to the device and repacks the 80-byte metric into SoA planes
 * (immutable input). Synchronises the device once.                        */
ostc_status ostc_create(const ostc_config *cfg, const ostc_param *param,
                        const ostc_zone *zones, int n_zones,
                        const ostc_bc_face *faces, int n_faces,
                        ostc_ctx **out);
ostc_status ostc_destroy(ostc_ctx *ctx);

/* Which optional ostc_zone arrays the given param/config needs (bit mask in
 * the order of ostc_zone's pointer members starting at bit 0 = x).         */
uint64_t ostc_zone_required(const ostc_config *cfg, const ostc_param *param);

/* Attach the 1-to-1 interfaces between the context's blocks (replaces any
 * previous set; resets the cached step graphs). Used by ostc_initialize,
 * ostc_data_communication and every RK3 stage.                             */
ostc_status ostc_set_interfaces(ostc_ctx *ctx, const ostc_interface *faces, int n_faces);

/* Last error recorded on the context: status, CUDA error code, and the
 * first failing block/cell when the status is OSTC_ERR_NONPHYSICAL.        */
ostc_status ostc_get_error(const ostc_ctx *ctx, int *cuda_error, int *block,
                           int *i, int *j, int *k);

/* ----------------------------------------------------------------------- */
/* operator API: one call per reference operator of the RK3 stage         */
/* ----------------------------------------------------------------------- */

/* compute_cv_from_bv<mix,turb> over [-ngg, m+ngg) (src/FieldOperation.cuh:43-79). */
ostc_status ostc_compute_cv_from_bv(ostc_ctx *ctx, void *stream);

/* cudaMemset(dq) + compute_source + compute_inviscid_flux +
 * compute_viscous_flux (src/RK.cuh:110-116): the right-hand side of every
 * block into dq, in fused sm_100a kernels.                                 */
ostc_status ostc_compute_rhs(ostc_ctx *ctx, void *stream);

/* local_time_step (src/TimeAdvanceFunc.cuh:50-100) + global_time_step
 * (src/TimeAdvanceFunc.cu:155-201) as one fused kernel with an on-device
 * min; the result stays in device memory (ostc_dt_device) unless dt_host is
 * non-NULL, in which case this call synchronises the stream.              */
ostc_status ostc_global_time_step(ostc_ctx *ctx, double *dt_host, void *stream);
const double *ostc_dt_device(const ostc_ctx *ctx);

/* update_cv_and_bv_rk (src/RK.cuh:197-253) for SSPRK3 stage rk in {0,1,2}.
 * dt < 0 reads the device dt written by ostc_global_time_step.            */
ostc_status ostc_update_cv_and_bv_rk(ostc_ctx *ctx, double dt, int rk, void *stream);

/* DBoundCond::apply_boundary_conditions<mix,turb,with_cv> in the reference's
 * priority order (src/BoundCond.cuh:673-822), plus periodic faces.        */
ostc_status ostc_apply_boundary_conditions(ostc_ctx *ctx, int with_cv, void *stream);

/* data_communication<mix,turb,with_cv> for same-device 1-to-1 interfaces
 * (src/DataCommunication.cuh:27-110): ghost layers take the partner block's
 * values, the coincident plane takes the average of both blocks (quirk A10).
 * A no-op without interfaces.                                              */
ostc_status ostc_data_communication(ostc_ctx *ctx, int with_cv, void *stream);

/* update_physical_properties<mix> over [-1, m] (src/FieldOperation.cuh:112-146). */
ostc_status ostc_update_physical_properties(ostc_ctx *ctx, void *stream);

/* ----------------------------------------------------------------------- */
/* per-step epilogues of the RK3 loop (src/RK.cuh:164-180)                  */
/* ----------------------------------------------------------------------- */
/* Every step of ostc_rk3_steps ends with physical_time += dt of its last
 * stage and step += 1 (both reset by ostc_initialize); this returns them
 * (synchronises the device; either pointer may be NULL).                   */
ostc_status ostc_physical_time(ostc_ctx *ctx, double *time, int *step);
/* Resuming a run from a checkpoint (the reference's restart: solution_time of
 * the flow-field file, read_flowfield, Initialize.cuh:64-243, and the step of
 * step.txt): after restoring bv / sv in the caller's arrays and calling
 * ostc_initialize, sets the physical time and step count the following steps
 * continue from.                                                           */
ostc_status ostc_set_physical_time(ostc_ctx *ctx, double time, int step);

/* Monitor points (Monitor.cu:196-251, record_monitor_data): after every step
 * the bv planes bv_label[0..n_bv) (0 rho, 1 u, 2 v, 3 w, 4 p, 5 T) and the sv
 * planes sv_label[0..n_sv) (species, then k, omega) at the interior points
 * (block[p], i[p], j[p], k[p]), followed by the physical time, go to a device
 * ring of `capacity` steps. n_points = 0 removes the monitor. Resets the
 * cached step graphs.                                                       */
ostc_status ostc_set_monitor(ostc_ctx *ctx, int n_points, const int *block, const int *i, const int *j,
                             const int *k, int n_bv, const int *bv_label, int n_sv, const int *sv_label,
                             int capacity);
/* Copies the ring to the HOST array out[(p * capacity + s) * (n_bv + n_sv + 1)
 * + v] and restarts it (Monitor::output_data); *n_recorded = the steps
 * recorded since the last call (at most capacity; ring slot s = step index
 * modulo capacity). Synchronises the device.                               */
ostc_status ostc_get_monitor(ostc_ctx *ctx, double *out, int *n_recorded);

/* Statistics (StatisticsCollector.cu:14-52): on = 1 starts per-cell sums over
 * the interior of every block, for each step after start_step (and after this
 * call): rho, u, v, w, p, T and their squares (sum12, 12 planes), cubes and
 * fourth powers (sum34, 12 planes), uv, uw, vw (3 planes) and the mass
 * fractions (n_spec planes). on = 0 frees them. Resets the cached graphs.   */
ostc_status ostc_set_statistics(ostc_ctx *ctx, int on, int start_step);
/* The sums of one block to HOST arrays (each may be NULL; interior layout,
 * g = 0) and the number of samples summed into them (counted on the device,
 * so it stays exact when ostc_set_physical_time moves the step count after
 * statistics were switched on). Synchronises the device.                  */
ostc_status ostc_get_statistics(ostc_ctx *ctx, int block, double *sum12, double *sum34, double *sum_rs,
                                double *sum_yk, int *n_collected);

/* ---- grid pre-processing: the reference's grid and boundary files ------- */
/* A mesh read on the host as cfd::Mesh reads it (src/Mesh.cpp:550-588) from
 * the text grid file (input_files/grid/grid N.grd: block count, mx my mz per
 * block, then x, y, z of each block with i fastest), the boundary file
 * (boundary N.txt: per block a face count, then i1 i2 j1 j2 k1 k2 label) and
 * the inner-face file (inner N.txt; NULL: no interfaces): faces and 1-to-1
 * interfaces registered as Boundary / InnerFace::register_boundary
 * (src/Mesh.cpp:14-178), coordinates scaled by grid_scale, ghost grid
 * extrapolated, copied across interfaces and completed at edges and corners
 * (init_ghost_grid, src/Mesh.cpp:789-987), and the Jacobian and metrics of
 * ostc_metric_from_grid. Host only; one process (no parallel-interface
 * file). OSTC_ERR_IO: a file is missing or malformed.                      */
typedef struct ostc_mesh ostc_mesh;
ostc_status ostc_mesh_read(const char *grid_file, const char *boundary_file, const char *inner_file, int ngg,
                           double grid_scale, ostc_mesh **out);
ostc_status ostc_mesh_destroy(ostc_mesh *m);
/* counts: blocks, dimension (2 when the first block has mz == 1), boundary
 * faces and interfaces over all blocks (each may be NULL)                   */
ostc_status ostc_mesh_sizes(const ostc_mesh *m, int *n_blocks, int *dimension, int *n_faces, int *n_interfaces);
/* one block: its extents and, where non-NULL, HOST arrays with ngg ghost
 * layers (the ostc_zone layout) of x, y, z, the Jacobian and the 80-byte
 * metric records                                                            */
ostc_status ostc_mesh_block(const ostc_mesh *m, int b, int *mx, int *my, int *mz, double *x, double *y, double *z,
                            double *jac, void *metric);
/* the registered boundary faces of all blocks, block by block in file order:
 * block, type_label (the file's label), face, direction and ranges; the
 * condition's state is left zero, and wall faces are not yet trimmed (the
 * boundary-condition set-up does both, src/BoundCond.cu:167-416)           */
ostc_status ostc_mesh_faces(const ostc_mesh *m, ostc_bc_face *faces);
/* the registered interfaces of all blocks, block by block in file order,
 * ready for ostc_set_interfaces                                             */
ostc_status ostc_mesh_interfaces(const ostc_mesh *m, ostc_interface *faces);

/* ---- restart and output: the reference's flow-field file --------------- */
/* Writes the context's flow field to `path` in the layout of
 * FieldIO::print_field (src/FieldIO.h:44-560), the file the reference
 * restarts from (output/field/flowfield.plt): Tecplot binary V112, one
 * ordered zone "zone b" per block with the solution time, nodal FP64 values
 * over [-ngg_out, m + ngg_out) per axis of x, y, z, density, u, v, w,
 * pressure, temperature, mach, the species (named by species_names, n_spec
 * HOST strings), and tke, omega, mut with SST, each with its min / max in the
 * zone header. x, y, z: HOST arrays per block with the block's ngg ghost
 * layers (the reference's Block::x); the flow data are copied from the
 * blocks' device arrays (mach as the properties last computed it).
 * Synchronises the device; OSTC_ERR_IO when the file cannot be written.    */
ostc_status ostc_write_flowfield(ostc_ctx *ctx, const char *path, const double *const *x,
                                 const double *const *y, const double *const *z,
                                 const char *const *species_names, int ngg_out, double solution_time);
/* Reads such a file into the blocks' bv and sv device arrays as
 * read_flowfield (src/Initialize.cuh:64-243): variables are matched by name,
 * case-insensitive, as identify_variable_labels (src/Initialize.cuh:
 * 246-310) does: DENSITY / ROE / RHO, U, V, W, P / PRESSURE, T / TEMPERATURE,
 * the species names, and K / TKE, OMEGA with SST; others are skipped. A zone
 * may hold fewer ghost layers than its block ((file extent - m) / 2); the
 * values it does not cover keep theirs. *found (optional) gets bit 0 when
 * species were in the file and bit 1 when k and omega were (the reference
 * then initialises what is missing from the inflow, src/Initialize.cuh:
 * 195-214; here the caller does), *solution_time (optional) the zones' time
 * (for ostc_set_physical_time). Call ostc_initialize afterwards.
 * Synchronises the device.                                                 */
ostc_status ostc_read_flowfield(ostc_ctx *ctx, const char *path, const char *const *species_names,
                                double *solution_time, int *found);

/* eliminate_k_gradient<with_cv> (src/FieldOperation.cuh:372-400): on 2-D
 * blocks (mz == 1) every k ghost plane of bv, sv (and cv when with_cv) takes
 * the values of the plane k = 0 over the whole ghosted (i, j) range, so
 * nothing varies across k. A no-op for 3-D blocks. The drivers below call it
 * where the reference does: before the boundary conditions of the
 * initialisation (src/Driver.cu:54-60), and after the interface exchange of
 * every RK3 stage (src/RK.cuh:147-153, with cv) and steady step
 * (src/SteadySim.cuh:101-107, without).
 * 2-D problems: every block has mz == 1 (the reference takes the dimension
 * from its first block, src/Mesh.cpp:612-614); the z fluxes are skipped
 * (src/InviscidScheme.cu:34, src/SchemeSelector.cuh:64), the time step and
 * the Roe entropy fix drop their zeta terms (src/TimeAdvanceFunc.cuh:60-93,
 * src/Roe.cu:79-81), and the stage update zeroes rho w (src/RK.cuh:213-215). */
ostc_status ostc_eliminate_k_gradient(ostc_ctx *ctx, int with_cv, void *stream);

/* ----------------------------------------------------------------------- */
/* fused drivers                                                           */
/* ----------------------------------------------------------------------- */

/* Driver::initialize_computation (src/Driver.cu:39-98) followed by the
 * pre-loop of RK3_bv (src/RK.cuh:40-49). Also re-reads the metric records
 * (so they may be written after ostc_create).                             */
ostc_status ostc_initialize(ostc_ctx *ctx, void *stream);

/* One SSPRK3 stage: RHS, dt (if CFL), update, BCs, interfaces, properties. */
ostc_status ostc_rk3_stage(ostc_ctx *ctx, int rk, void *stream);

/* n_steps full RK3 steps (the body of the while loop in RK3_bv,
 * src/RK.cuh:89-170), captured once as a CUDA graph and replayed.
 * If res_hist is non-NULL it receives 4 doubles per step (the RMS change of
 * rho, |V|, p, T, src/Residual.cuh:57-161, unnormalised) and dt_hist one dt
 * per step; both synchronise the stream at the end. With either history the
 * residual epilogue also checks the state of every interior cell after each
 * step (the reference stops on a NaN residual, src/Residual.cuh:153-158):
 * a non-positive or NaN density or pressure, or a NaN residual term, makes
 * the call return OSTC_ERR_NONPHYSICAL after all n_steps, and ostc_get_error
 * reports the first such cell (earliest step, then lowest block, then lowest
 * k, j, i). The histories are still written.                              */
ostc_status ostc_rk3_steps(ostc_ctx *ctx, int n_steps, double *res_hist,
                           double *dt_hist, void *stream);

/* ---- steady path (cfg.steady = 1; src/SteadySim.cuh:15-137) ------------ */

/* local_time_step (src/TimeAdvanceFunc.cuh:50-100) on every block: per-cell
 * dt_local (zone.dt_local, required when steady) and the inviscid spectral
 * radii DPLUR reuses (kept in context-owned planes; zone.inv_spectr_rad and
 * zone.visc_spectr_rad are not written).                                   */
ostc_status ostc_local_time_step(ostc_ctx *ctx, void *stream);

/* implicit_treatment (src/ImplicitTreatmentHPP.cuh:8-52) on every block.
 * implicit_method 0: point-implicit chemistry of the explicit steady step,
 * EPI (chemSrcMethod 1, src/FiniteRateChem.cu:234-256) or DA (2,
 * src/FiniteRateChem.cu:421-432), applied to the species rows of dq.
 * implicit_method 1: DPLUR (src/DPLUR.cuh:283-312) with DPLUR_inner_step
 * Jacobi sweeps, wall dq set to 0 before each sweep, no exchange between
 * blocks inside the sweeps; zone.dq0 / zone.dqk are used when given, else
 * the context allocates them. The chemical Jacobian is rebuilt from the
 * state inside the kernels (zone.chem_src_jac is neither read nor written);
 * DPLUR keeps the LU factors of (diag I - dt J) for its sweeps.            */
ostc_status ostc_implicit_treatment(ostc_ctx *ctx, void *stream);

/* update_bv (src/FieldOperation.cuh:221-296): bv, sv (and T, p by the
 * Newton solve of src/FieldOperation.cu:3-39) from dq * dt_local / jac.   */
ostc_status ostc_update_bv(ostc_ctx *ctx, void *stream);

/* n_steps steady iterations (the loop body of steady_simulation,
 * src/SteadySim.cuh:51-126: RHS, local dt, implicit treatment, update_bv,
 * BCs and interfaces without cv, properties), captured as a CUDA graph.
 * res_hist and the state check as for ostc_rk3_steps; the caller tests
 * convergence on res_hist.                                                 */
ostc_status ostc_steady_steps(ostc_ctx *ctx, int n_steps, double *res_hist, void *stream);

/* ---- FP64 point-implicit chemistry integrator -------------------------- */

/* One point-implicit step of the finite-rate chemistry of each of n states
 * at constant density and internal energy: rho from (T, p, Y), omega and
 * J = d omega / d(rho Y) as compute_chem_src_jacobian builds them
 * (src/FiniteRateChem.cu:7-216), d(rho Y) = (I - dt J)^-1 dt omega with the
 * column-pivoted LU of solve_chem_system (src/FiniteRateChem.cu:324-419),
 * Y' = Y + d(rho Y)/rho, and T' from e(T', Y') = e(T, Y) by the Newton
 * iteration of compute_temperature_and_pressure (src/FieldOperation.cu:
 * 3-39) run to a relative 1e-13. The reference has no single function for
 * this composition; it is the labeller, fallback and arbiter of the chemistry
 * surrogate. All pointers are DEVICE arrays: T, p, dt, dT of n doubles, Y
 * and dY of n_spec x n (species-major). dT is NaN where the Newton solve did
 * not converge. Needs a context with a finite-rate mechanism.              */
ostc_status ostc_chem_point_implicit(ostc_ctx *ctx, int n, const double *T, const double *p,
                                     const double *Y, const double *dt, double *dY, double *dT,
                                     void *stream);

/* ---- chemistry surrogate: network and training ------------------------- */
/* A 12-256-256-256-10 perceptron with SiLU activations that maps the
 * standardised features of a cell state (log T, log p, 9 transformed Y_k,
 * log dt) to the standardised increments (9 dY_k, dT) of
 * ostc_chem_point_implicit. BF16 weights and activations, FP32 accumulation
 * on the tensor cores, FP32 master weights, Adam. No reference counterpart:
 * the reference integrates chemistry only with the FP64 path above.        */
typedef struct ostc_surrogate ostc_surrogate;
#define OSTC_SURR_IN 12
#define OSTC_SURR_OUT 10
#define OSTC_SURR_HIDDEN 256
#define OSTC_SURR_PARAMS 137482  /* W1[256][12] b1 W2[256][256] b2 W3 b3 W4[10][256] b4[10] */

/* He-uniform weights from a seeded generator, zero biases; buffers for
 * training batches of up to max_batch rows. Allocates device memory.      */
ostc_status ostc_surrogate_create(int max_batch, unsigned long long seed, ostc_surrogate **out);
ostc_status ostc_surrogate_destroy(ostc_surrogate *s);
/* Feature / target scaling (HOST arrays): x_std = (x - in_mean) / in_std,
 * z = out_mean + out_std * net(x_std), and the predicted rate (increment
 * per unit dt) is r0 sinh(z) where out_r0 > 0 (out_r0 NULL or 0: r = z);
 * in_min / in_max bound the training envelope in raw feature units (states
 * outside it take the FP64 path).                                          */
ostc_status ostc_surrogate_set_scaling(ostc_surrogate *s, const double *in_mean, const double *in_std,
                                       const double *out_mean, const double *out_std,
                                       const double *in_min, const double *in_max, const double *out_r0);
/* FP32 master parameters in the flat order of OSTC_SURR_PARAMS (HOST).
 * set_params also resets the Adam moments.                                */
ostc_status ostc_surrogate_get_params(const ostc_surrogate *s, float *host_out);
ostc_status ostc_surrogate_set_params(ostc_surrogate *s, const float *host_in);
/* Network on n standardised rows: xs [n][12] -> ys [n][10] (DEVICE).     */
ostc_status ostc_surrogate_forward(ostc_surrogate *s, const float *xs, int n, float *ys, void *stream);
/* The same network on the tcgen05 tensor cores (128-row tiles, TMEM
 * accumulators; the inference kernel of the chemistry surrogate) on n
 * standardised rows; synchronises. OSTC_ERR_TIMEOUT if a bounded wait on the
 * tensor cores ran out (the outputs are then undefined).                  */
ostc_status ostc_surrogate_forward_tc(ostc_surrogate *s, const float *xs, int n, float *ys, void *stream);
/* Gradients of the mean squared error over n rows (xs, ys DEVICE) in the
 * flat parameter order (grad_host, HOST) and the loss; synchronises.      */
ostc_status ostc_surrogate_gradients(ostc_surrogate *s, const float *xs, const float *ys, int n,
                                     float *grad_host, float *loss_host, void *stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) at learning rate lr on n rows;
 * loss_dev (DEVICE, optional) receives the batch's sum of squared errors. */
ostc_status ostc_surrogate_train_step(ostc_surrogate *s, const float *xs, const float *ys, int n, float lr,
                                      float *loss_dev, void *stream);

/* Acceptance tests of the surrogate's increments: n_elem (<= 4) elements
 * with counts elem_counts[e][n_spec] and atomic masses elem_mass[e]; an
 * increment is rejected when an element's mass fraction changes by more
 * than tol_elem, or when the internal energy at constant density changes
 * by more than tol_T kelvin worth of cv (HOST arrays).                     */
ostc_status ostc_surrogate_set_checks(ostc_surrogate *s, int n_elem, int n_spec, const double *elem_counts,
                                      const double *elem_mass, double tol_elem, double tol_T);

/* The learned chemistry step of n states (DEVICE arrays laid out as for
 * ostc_chem_point_implicit): features, training-envelope test, the network
 * on the tensor cores, element and energy checks; every state that fails a
 * test is redone by the FP64 point-implicit integrator. n_fallback (HOST,
 * optional) receives the number of redone states and makes the call
 * synchronise; OSTC_ERR_TIMEOUT then reports a bounded tensor-core wait that
 * ran out. Needs the 9-species finite-rate context of the surrogate.       */
ostc_status ostc_chem_surrogate(ostc_ctx *ctx, ostc_surrogate *sur, int n, const double *T, const double *p,
                                const double *Y, const double *dt, double *dY, double *dT, int *n_fallback,
                                void *stream);

/* Diagnostic of the timeout path, for callers that test their error
 * handling: with on = 1 the tensor-core kernels launched afterwards for s
 * (ostc_surrogate_forward_tc, ostc_chem_surrogate) withhold the completion
 * signal of their first matrix product, so their bounded wait for it runs
 * out after about one second and the call returns OSTC_ERR_TIMEOUT. The
 * kernels still drain their in-flight work and free their tensor memory, so
 * the device stays usable; on = 0 restores normal operation. Steps captured
 * in graphs before the call keep the setting they were captured with.
 * No reference counterpart.                                                */
ostc_status ostc_surrogate_inject_timeout(ostc_surrogate *s, int on);

/* The surrogate used by chem_mode 2 (the context keeps the pointer; the
 * surrogate must outlive it). Resets the cached step graphs.               */
ostc_status ostc_set_chem_surrogate(ostc_ctx *ctx, ostc_surrogate *sur);
/* Totals of the split chemistry since the context was created: states
 * integrated and states the surrogate handed to the FP64 fallback (HOST
 * outputs; synchronises the stream).                                       */
ostc_status ostc_chem_stats(ostc_ctx *ctx, long long *states, long long *fallbacks, void *stream);

/* The chemistry source of the RHS has a second, generated form for the
 * 9-species / 19-reaction H2-air mechanism's structure (straight-line code
 * from openstc-dev_b200/gen_mechanism.py; rate parameters still come from
 * ostc_param). ostc_create selects it when the mechanism's reaction types,
 * stoichiometry and orders match; on = 0 forces the generic form, on = 1
 * returns OSTC_ERR_INVALID_ARG for another mechanism. No reference
 * counterpart: the reference always runs the generic loops.               */
ostc_status ostc_use_generated_chemistry(ostc_ctx *ctx, int on);

/* Metric and Jacobian from grid coordinates that carry ngg+1 ghost layers
 * (x,y,z as host arrays with ghost count ngg+1), as Block::compute_jac_metric
 * (src/Mesh.cpp:259-521). Host-only helper: fills host jac (g=ngg) and host
 * metric (80-byte records, g=ngg). Returns OSTC_ERR_NONPHYSICAL on a
 * non-positive interior Jacobian. mz == 1 is a 2-D block: its k ghost nodes
 * sit at z(i,j,0) + k, as the reference's grid reader puts them
 * (src/Mesh.cpp:840-854); otherwise mz >= 3.                               */
ostc_status ostc_metric_from_grid(int mx, int my, int mz, int ngg,
                                  const double *x, const double *y, const double *z,
                                  double *jac_out, void *metric_out);

/* Tile shape of the flux kernel of direction dir (0 x, 1 y, 2 z): rows of
 * 32 threads per CTA (1, 2, 4 or 8) and chunks marched per CTA; rows may be
 * OR-ed with (2 << 8) or (3 << 8) to select the builds limited to 128 or 80
 * registers (two or three 256-thread CTAs per SM), or with (4 << 8) / (5 << 8)
 * for the builds limited to 168 / 96 registers (three / five CTAs of at most
 * 4 rows per SM). OR-ing (1 << 16) selects the staged kernels (rows = 8
 * only, 128 registers): before its faces are computed a CTA copies with
 * cp.async into shared memory the primitive and scalar values of the cells of
 * its sweep plane that they read (with the reconstruction halo along the
 * sweep) and the metric, Jacobian and transport properties of the faces' own
 * cells; only the cells across the plane are read from HBM by the faces. Built
 * for the primitive-variable and Roe faces, not AWENO (launches then fail with
 * OSTC_ERR_CUDA). Results are bit-identical to the plane kernels.
 * dir 3, 4, 5: a tile for a separate viscous-flux kernel of direction
 * dir - 3; with one set, a viscous flow runs the inviscid flux (tile of dir
 * - 3) and the viscous flux as two kernels instead of the fused one. rows = 0
 * there returns to the fused kernel (get_tile reports 0, 0 then).
 * Set by the autotuner (openstc-dev_b200/ostc.py:
 * Solver.autotune) or by hand; resets the cached graphs.                  */
ostc_status ostc_set_tile(ostc_ctx *ctx, int dir, int rows, int chunks);
ostc_status ostc_get_tile(const ostc_ctx *ctx, int dir, int *rows, int *chunks);

/* The flux autotuner (no reference counterpart: the reference launches fixed
 * block shapes, InviscidScheme.cu / ViscousScheme.cuh). For each direction it
 * times, with CUDA events on `stream` (warmup + reps launches each), every
 * tile of rows {2,4,8} (x) or {4,8} (y, z) x chunks 1, 2, 4, .. up to the
 * first block's extent x register budgets 1..5, and the staged kernels (8
 * rows; not for AWENO); for a viscous flow also the separate inviscid and
 * viscous kernels, each tuned on its own, which replace the fused kernel when
 * their sum is faster. Sets the winners (ostc_set_tile) and, if ms_out is not
 * null, writes the chosen device ms per launch of each direction (3 floats).
 * Only dq is written, so the flow state is left as it was. Synchronises.    */
ostc_status ostc_autotune(ostc_ctx *ctx, int warmup, int reps, void *stream, float *ms_out);

/* Batched multi-block launches. on = 1: every block of the context is
 * processed by one persistent launch per kernel (flux of each direction,
 * source, stage update, properties, time step, conservative variables): the
 * grid fills the device's resident CTA slots and walks a device tile table
 * of {block, tile} entries built from the blocks' extents and the flux tile
 * shapes. Results are identical to the per-block launches (on = 0): every
 * cell sees the same operations in the same order. Default: on for 2 to 64
 * blocks, off for one (a single block whose boundary faces hold at most
 * 2^17 points still takes the one-launch boundary faces below, which small,
 * launch-bound faces favour). Batched, ostc_apply_boundary_conditions is one
 * cooperative launch over
 * every face in the per-face order (priority levels of BoundCond.cuh:673-822,
 * then the periodic wraps), ostc_data_communication one over every interface
 * in their order (DataCommunication.cuh:30-49). Each splits its faces into
 * waves of faces whose footprints do not meet (a face goes one wave after
 * the last earlier face whose footprint meets its own: for interfaces own
 * range and plane, partner's range and plane), with a grid barrier between
 * waves, so the results are the per-face ones bit for bit. A barrier wait is
 * bounded (about one second); one that runs out makes the next check of a
 * call with histories return OSTC_ERR_TIMEOUT. At most 64 blocks:
 * OSTC_ERR_UNSUPPORTED beyond. No reference counterpart: the reference
 * launches every kernel per block and face (RK.cuh:107-161).              */
ostc_status ostc_set_batching(ostc_ctx *ctx, int on);
ostc_status ostc_get_batching(const ostc_ctx *ctx, int *on);
/* Diagnostic for failure handling: with on = 1 the grid barriers of the
 * batched boundary-face and interface launches withhold their release, so
 * each launch with more than one wave waits about one second, stops, and
 * the next ostc_rk3_steps / ostc_steady_steps with histories returns
 * OSTC_ERR_TIMEOUT (the waves after the first were not computed); on = 0
 * restores normal operation. Synchronises the device. No reference
 * counterpart.                                                              */
ostc_status ostc_inject_wave_timeout(ostc_ctx *ctx, int on);

/* Launch one kernel family on every block (timing and autotuning aid):
 * OSTC_OP_FLUX (arg = direction, accumulates into dq; arg + 3: the inviscid
 * flux kernel alone, arg + 6: the viscous flux kernel alone), OSTC_OP_SOURCE,
 * OSTC_OP_PROPERTIES, OSTC_OP_UPDATE (arg = rk stage), OSTC_OP_DT,
 * OSTC_OP_BC (arg = with_cv). No reference counterpart: the reference
 * launches these only from its stage loop (src/RK.cuh:107-161).            */
enum { OSTC_OP_FLUX = 0, OSTC_OP_SOURCE = 1, OSTC_OP_PROPERTIES = 2, OSTC_OP_UPDATE = 3, OSTC_OP_DT = 4,
       OSTC_OP_BC = 5 };
ostc_status ostc_launch_op(ostc_ctx *ctx, int op, int arg, void *stream);

/* Number of kernel nodes in the CUDA graph of one RK3 step, or of one steady
 * iteration for a steady context (with or without the residual epilogue);
 * captures the graph if it does not exist yet.                             */
ostc_status ostc_step_kernel_count(ostc_ctx *ctx, int with_hist, int *count);

/* Residual of one block without any device allocation. No counterpart in
 * the reference: for callers that cannot allocate device memory when the
 * residual is wanted (a host solver that reserves its whole device budget at
 * start-up, or one sharing a fixed memory pool with other codes). Writes to
 * res_out (DEVICE pointer, 4 doubles) sqrt(sum(d^2)/cells) of rho, |V|, p, T
 * between zone->bv_last (written by store_last_step at the start of a step)
 * and the current zone->bv / zone->vel: the same quantity as the residual
 * history of ostc_rk3_steps. Partial sums go to a fixed array in the
 * library's own device memory (OSTC_NOALLOC_MAX_PARTIALS x 4 doubles =
 * 512 KiB, held on every GPU that loads the library until exit); blocks of
 * more than OSTC_NOALLOC_MAX_CELLS cells are rejected with
 * OSTC_ERR_INVALID_ARG. Every call made outside a stream capture looks up the
 * array's address on the current device; a call made while its stream is
 * being captured uses the address found by the last such call and returns
 * OSTC_ERR_INVALID_ARG when there was none, so make a first call on each
 * device before any capture. All calls share the array: calls that overlap
 * on the GPU race.                                                         */
#define OSTC_NOALLOC_MAX_PARTIALS 16384
#define OSTC_NOALLOC_MAX_CELLS (OSTC_NOALLOC_MAX_PARTIALS * 2048LL)
ostc_status ostc_compute_residual_noalloc(const ostc_zone *zone, double *res_out, void *stream);

/* Library version string. */
const char *ostc_version(void);

#ifdef __cplusplus
}
#endif
#endif /* OSTC_H */
