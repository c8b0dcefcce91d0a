// kernels.cuh — host-side launch interface of kernels.cu.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "mlp.cuh"

namespace ostc {

// launch shape of one flux-direction kernel: R rows of 32 threads, C chunks per segment
struct TileShape {
  int rows;
  int chunks;
  int minb = 1;  // register budget: 1 (<=255 regs), 2 (<=128) or 3 (<=80) CTAs of 256 threads per SM,
                 // 4 (<=168 regs) or 5 (<=96 regs) with CTAs of at most 128 threads
  // viscous flow: vrows > 0 splits the face flux into an inviscid kernel
  // (the shape above) and a viscous kernel of this shape
  int vrows = 0;
  int vchunks = 1;
  int vminb = 1;
  // 1: the staged kernels (flux_dir_staged: the cells a CTA's faces read
  // copied into shared-memory tiles first), 0: cells read from the planes
  int staged = 0;
  int vstaged = 0;
};

// tile-table launches: all zones of a context in one persistent launch per
// kernel; the zones live in a __constant__ table of each kernel unit
constexpr int kMaxTableZones = 64;

// a device array of {zone, bx, by, bz} CTA tiles
struct FluxTable {
  const int4 *tiles = nullptr;
  int n = 0;
  int n_bulk = 0;  // flux tables: the leading tiles, of zones with kZoneBulk
};
using CellTable = FluxTable;

// grid of one flux-direction kernel over a zone of mx x my x mz cells
inline dim3 flux_grid(int mx, int my, int mz, int dir, int R, int C) {
  if (dir == 0) {
    const int S = 32 * C - 1;
    return dim3((mx + S - 1) / S, (my + R - 1) / R, mz);
  }
  const int S = R * C - 1;
  if (dir == 1) return dim3((mx + 31) / 32, (my + S - 1) / S, mz);
  return dim3((mx + 31) / 32, my, (mz + S - 1) / S);
}

// one boundary face as the kernels see it
struct BcFace {
  int type, face, direction;
  int zone;  // index of the face's zone in the context (tile-table launches)
  int rs[3], re[3];
  int dir_stride;     // ghosted-index stride of one step along the outward normal
  int period_stride;  // periodic: ghosted-index stride of n cells along the normal
  double density, u, v, w, pressure, temperature, velocity, mut;
  double sv[OSTC_MAX_SPEC + 4];
  int wall_isothermal;
  double wall_temperature;
  double acoustic_speed, entropy, specific_heat_ratio, mw;
  double total_pressure, total_temperature;
};

struct Iface {
  int face, direction;
  int rs[3], ts[3], ld[3], tld[3], st[3], np[3];
  int zone, target;  // the face's zone and its partner's in the context (tile-table launches)
};

enum class CellOp { Source, UpdateRK, Properties, CvFromBv, Velocity, Dt, DtReset, StoreLast, ResidualPartial, InitMut };

struct CellArgs {
  double dt = 0;
  const double *dt_dev = nullptr;
  int rk = 0;
  unsigned long long *dt_bits = nullptr;
  double *partial = nullptr;
  int n_part = 0;
  unsigned long long *bad = nullptr;  // ResidualPartial: first non-physical cell (key, atomic minimum)
  const int *step = nullptr;          // ResidualPartial: device step counter of the key
  int block = 0;                      // ResidualPartial: zone index of the key
  int spec = 0;  // Source: use the mechanism-specialised chemistry
};

// the steady path (steady.cuh)
enum class SteadyOp { ChemImplicit, UpdateBv, DplurDq0, DplurSweep, DplurFinish, WallDqZero, TurbImplicit };
struct SteadyArgs {
  const double *dq_in = nullptr;  // DPLUR sweep: current iterate (dq layout)
  double *dq_out = nullptr;       // DPLUR sweep: next iterate
  double *dq0 = nullptr;          // DPLUR: dq after compute_DQ_0 (dq layout)
  double *lu = nullptr;           // DPLUR + EPI: NS*NS interior planes of LU factors
  unsigned char *piv = nullptr;   // DPLUR + EPI: NS interior planes of pivot rows
  double *da = nullptr;           // DPLUR + DA: NS interior planes of diag - dt J_ll
  int final_div = 0;              // DPLUR sweep: write (dq0 + ...) / dt_local into dq_out
};

// part 0: the face flux of the flow; 1: its inviscid half alone; 2: its
// viscous half alone (flux.cuh: launch_flux_t). tab = nullptr: zone z alone;
// else tab[0] (shape t) and tab[1] (viscous shape) hold the tiles of every
// zone of the uploaded table and z is not used
// NT: turbulence scalars after the NS species (0, or 2 for SST with NS = 0);
// built in flux0.cu (NS 0, NT 0), flux9.cu (9, 0), flux0t.cu (0, 2) and flux9t.cu (9, 2)
template <int NS, int NT>
cudaError_t launch_flux_nt(const DevZone &z, int inv, int dir, const TileShape &t, const FluxTable *tab,
                           int accumulate, int viscous, int part, cudaStream_t s);
template <int NS>
cudaError_t launch_cells(CellOp op, const DevZone &z, const CellArgs &a, cudaStream_t s);
// the per-cell kernels of Source, UpdateRK, Properties, CvFromBv, Velocity,
// Dt and StoreLast over a tile table of (32 x 8)-thread tiles; the table's
// extents per zone: interior (mx, my, mz) for Source, UpdateRK, Dt,
// StoreLast; (mx+2, my+2, mz+2) for Properties and InitMut; ghosted for
// CvFromBv, Velocity
template <int NS>
cudaError_t launch_cells_table(CellOp op, const CellTable &tab, const CellArgs &a, cudaStream_t s);
// the zone tables of every kernel unit
cudaError_t upload_zones(const DevZone *z, int n, cudaStream_t s);
cudaError_t upload_zones_flux0(const DevZone *z, int n, cudaStream_t s);   // flux0.cu
cudaError_t upload_zones_flux9(const DevZone *z, int n, cudaStream_t s);   // flux9.cu
cudaError_t upload_zones_flux0t(const DevZone *z, int n, cudaStream_t s);  // flux0t.cu
cudaError_t upload_zones_flux9t(const DevZone *z, int n, cudaStream_t s);  // flux9t.cu
// staged flux kernels: whether a tile wait ran out since the last read (the
// flag is cleared), per flux unit and over all of them (kernels.cu)
cudaError_t stage_timeout_flux0(int *flag);
cudaError_t stage_timeout_flux9(int *flag);
cudaError_t stage_timeout_flux0t(int *flag);
cudaError_t stage_timeout_flux9t(int *flag);
cudaError_t stage_timeout_flux_ns_a(int *flag);
cudaError_t stage_timeout_flux_ns_b(int *flag);
cudaError_t stage_timeout_flux_ns_c(int *flag);
cudaError_t stage_timeout_flux_ns_d(int *flag);
cudaError_t stage_timeouts(int *any);
template <int NS>
cudaError_t launch_bc(const DevZone &z, const BcFace &b, int with_cv, cudaStream_t s);
// The waves of one call (boundary faces or interfaces over every zone; device
// records, zones in the tile-table zone table): tiles {record, a, b, c} of a
// face's points (32 along its first tangential axis and 8 along the second at
// one layer along its normal; interfaces normal to i: 4 layers x 8 x 8), wave
// after wave; ends[w] is the end of wave w in tiles. One cooperative launch
// walks all waves with a grid barrier between them.
struct WavePlan {
  const int4 *tiles = nullptr;
  const int *ends = nullptr;  // device, n_waves entries
  int n_waves = 0;
  int max_tiles = 0;          // tiles of the largest wave (grid bound)
};
// the grid barrier of a wave launch (device memory of the context, zeroed
// once): arrivals, CTAs that have left, the abort flag of a wait that ran
// out, timed_out, which stays set until the host reads and clears it, and
// hold, a diagnostic the host sets to withhold every barrier's release (its
// waits then run out: ostc_inject_wave_timeout)
struct WaveSync {
  unsigned arrive, done;
  int abort, timed_out, hold, pad;
};
template <int NS>
cudaError_t launch_bc_waves(const BcFace *faces, const WavePlan &p, int with_cv, WaveSync *sync, cudaStream_t s);
template <int NS>
cudaError_t launch_interface_waves(const Iface *faces, const WavePlan &p, int with_cv, WaveSync *sync, cudaStream_t s);
template <int NS>
cudaError_t launch_interface(const DevZone &self, const DevZone &tar, const Iface &f, int with_cv, cudaStream_t s);
template <int NS>
cudaError_t launch_steady(SteadyOp op, const DevZone &z, const SteadyArgs &a, const BcFace *wall, cudaStream_t s);
template <int NS>
cudaError_t launch_chem_integrator(int n, const double *T, const double *p, const double *Y, const double *dt,
                                   double *dY, double *dT, cudaStream_t s);
template <int NS>
cudaError_t launch_chem_surrogate(const mlp::Net &net, int n, const double *T, const double *p, const double *Y,
                                  const double *dt, double *dY, double *dT, const ChemScratch &w, cudaStream_t s);
// split chemistry of a block: op 0 gathers the interior states into buf,
// 1 scatters the increments back, 2 adds the block's counts to stats
template <int NS>
cudaError_t launch_chem_split(int op, const DevZone &z, const double *dt_dev, double dt_fixed, double *buf,
                              long long *stats, const int *count, cudaStream_t s);
cudaError_t prepare_chem_surrogate();
cudaError_t launch_residual_final(const double *partial, int n_part, double n_total, double *out, cudaStream_t s);

// per-step epilogues (epilogue.cu): step count and physical time, monitor
// points, statistics sums
struct MonitorSet {
  int n = 0, nbv = 0, nsv = 0, cap = 0;
  int4 *pts = nullptr;       // {block, i, j, k} per point
  int *labels = nullptr;     // nbv bv planes, then nsv sv planes
  double *data = nullptr;    // [n][cap][nbv + nsv + 1]
  int *counter = nullptr;    // records since the last read (ring position = counter % cap)
  const double *time = nullptr;
};
struct StatSums {
  double *s12 = nullptr, *s34 = nullptr, *srs = nullptr, *syk = nullptr;  // 12, 12, 3, n_spec interior planes
  int *count = nullptr;  // samples summed (device)
};
cudaError_t launch_step_clock(int *step, double *time, const double *dt_dev, double dt_fixed, cudaStream_t s);
cudaError_t launch_monitor(const DevZone &z, int blk, const MonitorSet &m, cudaStream_t s);
cudaError_t launch_monitor_advance(int *counter, cudaStream_t s);
cudaError_t launch_statistics(const DevZone &z, const int *step, int start, const StatSums &st, int ns,
                              cudaStream_t s);
// 2-D blocks: copy the plane k = 0 into every k ghost plane (no-op when mz > 1)
cudaError_t launch_eliminate_k(const DevZone &z, int with_cv, cudaStream_t s);
cudaError_t upload_param(const DevParam &p, cudaStream_t s);
cudaError_t upload_param_flux0(const DevParam &p, cudaStream_t s);   // flux0.cu
cudaError_t upload_param_flux9(const DevParam &p, cudaStream_t s);   // flux9.cu
cudaError_t upload_param_flux0t(const DevParam &p, cudaStream_t s);  // flux0t.cu
cudaError_t upload_param_flux9t(const DevParam &p, cudaStream_t s);  // flux9t.cu
// the units of the other species counts, 1..OSTC_MAX_SPEC
cudaError_t upload_param_ns_a(const DevParam &p, cudaStream_t s);       // kernels_ns_a.cu
cudaError_t upload_zones_ns_a(const DevZone *z, int n, cudaStream_t s);
cudaError_t upload_param_flux_ns_a(const DevParam &p, cudaStream_t s);  // flux_ns_a.cu
cudaError_t upload_zones_flux_ns_a(const DevZone *z, int n, cudaStream_t s);
cudaError_t upload_param_ns_b(const DevParam &p, cudaStream_t s);       // kernels_ns_b.cu
cudaError_t upload_zones_ns_b(const DevZone *z, int n, cudaStream_t s);
cudaError_t upload_param_flux_ns_b(const DevParam &p, cudaStream_t s);  // flux_ns_b.cu
cudaError_t upload_zones_flux_ns_b(const DevZone *z, int n, cudaStream_t s);
cudaError_t upload_param_ns_c(const DevParam &p, cudaStream_t s);       // kernels_ns_c.cu
cudaError_t upload_zones_ns_c(const DevZone *z, int n, cudaStream_t s);
cudaError_t upload_param_flux_ns_c(const DevParam &p, cudaStream_t s);  // flux_ns_c.cu
cudaError_t upload_zones_flux_ns_c(const DevZone *z, int n, cudaStream_t s);
cudaError_t upload_param_ns_d(const DevParam &p, cudaStream_t s);       // kernels_ns_d.cu
cudaError_t upload_zones_ns_d(const DevZone *z, int n, cudaStream_t s);
cudaError_t upload_param_flux_ns_d(const DevParam &p, cudaStream_t s);  // flux_ns_d.cu
cudaError_t upload_zones_flux_ns_d(const DevZone *z, int n, cudaStream_t s);
// every species count with a build: 0 (air), 1..OSTC_MAX_SPEC
constexpr int kMaxBuiltSpecies = OSTC_MAX_SPEC;
// whether a mechanism has the structure of the generated mech_h2air9.cuh
bool mechanism_is_h2air9(const int *reac_type, const int *stoi_f, const int *stoi_b, const int *reac_order, int nr,
                         int ns);

}  // namespace ostc
