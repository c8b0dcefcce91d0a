// api.cu — the C ABI of include/ostc.h: context, operator entry points,
// fused RK3 stage and the CUDA-graph step driver.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <type_traits>
#include <vector>

#include "../host/flowfield.h"
#include "common.cuh"
#include "kernels.cuh"

using namespace ostc;

#define OSTC_VERSION_STRING "openstc-b200 0.1 (sm_100a)"

struct GraphEntry {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

struct ostc_ctx {
  ostc_config cfg{};
  ostc_param prm{};
  DevParam dp{};
  int ns = 0;  // compile-time species count selecting the kernel instantiation
  int nt = 0;  // turbulence scalars after the species (2 with SST)
  bool has_source = false;
  int spec_ok = 0;    // the mechanism has the structure of the generated chemistry code
  int spec_mech = 0;  // ... and the source kernel uses it
  std::vector<ostc_zone> zones;
  std::vector<DevZone> dz;
  std::vector<double *> met_soa;
  std::vector<BcFace> faces;
  std::vector<int> face_zone;
  std::vector<Iface> ifaces;
  std::vector<int> iface_zone, iface_target;
  TileShape tile[3] = {{4, 4, 1}, {8, 2, 1}, {8, 2, 1}};
  // tile-table launches (ostc_set_batching): every zone in one persistent
  // launch per kernel; tables of the interior, properties and ghosted cell
  // ranges and of each flux direction (shape of tile[d], viscous shape)
  int batched = 0;
  int4 *tab_dev = nullptr;
  size_t tab_cap = 0;
  // boundary faces and interfaces in waves (one cooperative launch per call
  // over every zone): on by default for up to kMaxTableZones zones, one block
  // included; ostc_set_batching switches it with the tile tables. The face
  // and interface records on the device, the two wave plans (their tiles in
  // tab_dev, their ends in wave_ends_dev) and the grid barriers (two WaveSync)
  int face_batched = 0;
  BcFace *faces_dev = nullptr;
  Iface *ifaces_dev = nullptr;
  size_t ifaces_cap = 0;
  WavePlan bc_plan, if_plan;
  int *wave_ends_dev = nullptr;
  size_t wave_ends_cap = 0;
  WaveSync *wave_sync = nullptr;
  CellTable cell_tab[3];
  FluxTable flux_tab[3][2];
  unsigned long long *dt_bits = nullptr;  // device dt (as bits)
  double *res_partial = nullptr;          // [n_part_total][4]
  int n_part_per_zone = 0;
  double *hist_res = nullptr, *hist_dt = nullptr;  // device history buffers
  int *hist_counter = nullptr;
  int hist_cap = 0;
  // state check of the residual epilogue: key of the first non-physical cell
  // (step of the call << 44 | zone << 34 | interior cell index), all ones when none
  unsigned long long *bad_key = nullptr;
  double n_total = 0;
  std::map<int, GraphEntry> graphs;  // key: with_residual (+2 for the steady step)
  // per-step epilogues of the RK3 loop: step count and physical time (one int, one
  // double), monitor points, statistics sums (per zone)
  int *ep_step = nullptr;
  double *ep_time = nullptr;
  MonitorSet mon;
  int stat_on = 0, stat_start = 0;
  std::vector<StatSums> stats;
  // steady path: spectral radii (3 interior planes), DPLUR buffers (dq layout),
  // DPLUR point-implicit chemistry (LU factors + pivots, or DA divisors)
  std::vector<double *> isr, dq0, dqk, lu, da;
  std::vector<unsigned char *> piv;
  std::vector<void *> owned;  // allocations of this context to free
  // split chemistry (chem_mode 1, 2): SoA staging of the largest block and totals
  ostc_surrogate *sur = nullptr;
  double *chem_buf = nullptr;
  long long *chem_stats = nullptr;
  long long max_cells = 0;
  ostc_status last = OSTC_OK;
  int last_cuda = 0;
  int err_block = -1, err_i = 0, err_j = 0, err_k = 0, err_step = -1;
};

namespace {

const ostc_ctx *g_uploaded = nullptr;

ostc_status fail(ostc_ctx *c, ostc_status s, cudaError_t e = cudaSuccess) {
  if (c) {
    c->last = s;
    c->last_cuda = (int)e;
  }
  return s;
}

#define CK(expr)                                         \
  do {                                                   \
    cudaError_t e_ = (expr);                             \
    if (e_ != cudaSuccess) return fail(ctx, OSTC_ERR_CUDA, e_); \
  } while (0)

// the run parameters and zone table of ctx in every kernel unit's constant
// memory, uploaded when another context (or none) was the last one uploaded.
// Not inside a stream capture: an upload captured into a graph would happen
// only when the graph runs, while later calls took it as done (ensure_graph
// uploads before it captures).
ostc_status ensure_param(ostc_ctx *ctx, cudaStream_t s) {
  if (g_uploaded != ctx) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(s, &cap));
    if (cap != cudaStreamCaptureStatusNone) return fail(ctx, OSTC_ERR_INVALID_ARG);
    CK(upload_param(ctx->dp, s));
    if (ctx->batched || ctx->face_batched) CK(upload_zones(ctx->dz.data(), (int)ctx->dz.size(), s));
    g_uploaded = ctx;
  }
  return OSTC_OK;
}

// the tile tables of ctx (cell ranges and flux segments of every zone),
// rebuilt when batching is switched on or a tile shape changes
ostc_status build_tables(ostc_ctx *ctx) {
  std::vector<int4> all;
  std::vector<std::pair<size_t, size_t>> spans;  // [begin, end) of each table in `all`
  std::vector<size_t> flux_bulk_tiles;           // per flux table: its leading tiles of kZoneBulk zones
  auto cells = [&](int ext_add_xy, bool ghosted) {
    const size_t b0 = all.size();
    for (size_t b = 0; b < ctx->dz.size(); ++b) {
      const DevZone &z = ctx->dz[b];
      const int add = ghosted ? 2 * z.ngg : ext_add_xy;
      const int ex = z.mx + add, ey = z.my + add, ez = z.mz + add;
      const int gx = (ex + 31) / 32, gy = (ey + 7) / 8;
      for (int bz = 0; bz < ez; ++bz)
        for (int by = 0; by < gy; ++by)
          for (int bx = 0; bx < gx; ++bx) all.push_back(make_int4((int)b, bx, by, bz));
    }
    spans.push_back({b0, all.size()});
  };
  cells(0, false);  // interior
  cells(2, false);  // properties: [-1, m]
  cells(0, true);   // ghosted
  for (int d = 0; d < 3; ++d)
    for (int v = 0; v < 2; ++v) {
      const size_t b0 = all.size();
      const TileShape &t = ctx->tile[d];
      const int R = v ? t.vrows : t.rows, C = v ? t.vchunks : t.chunks;
      // the tiles of zones with kZoneBulk first, then the others: the staged
      // kernels walk the two parts with their bulk-copy and 8-byte builds
      size_t nb = 0;
      if (R > 0)
        for (int pass = 0; pass < 2; ++pass)
          for (size_t b = 0; b < ctx->dz.size(); ++b) {
            const DevZone &z = ctx->dz[b];
            if (d == 2 && z.mz <= 1) continue;
            if (((z.flags & kZoneBulk) != 0) != (pass == 0)) continue;
            const dim3 g = flux_grid(z.mx, z.my, z.mz, d, R, C);
            for (unsigned bz = 0; bz < g.z; ++bz)
              for (unsigned by = 0; by < g.y; ++by)
                for (unsigned bx = 0; bx < g.x; ++bx) all.push_back(make_int4((int)b, bx, by, bz));
            if (pass == 0) nb += (size_t)g.x * g.y * g.z;
          }
      spans.push_back({b0, all.size()});
      flux_bulk_tiles.push_back(nb);
    }
  // the tiles of a face of n[0] x n[1] x n[2] points with normal axis f in a
  // wave: 32 points along its first tangential axis, 8 along the second, one
  // layer along the normal (waves_kernel maps them back)
  auto wave_tiles = [&](int rec, int f, const int n[3]) {
    const int a = f == 0 ? 1 : 0, b = f == 2 ? 1 : 2;
    for (int tc = 0; tc < n[f]; ++tc)
      for (int tb = 0; tb < (n[b] + 7) / 8; ++tb)
        for (int ta = 0; ta < (n[a] + 31) / 32; ++ta) all.push_back(make_int4(rec, ta, tb, tc));
  };
  // boundary faces in the per-face order of apply_boundary_conditions
  // (priority levels of BoundCond.cuh:673-822, each level's faces in order,
  // then the periodic wraps), split into waves: a face goes one wave after
  // the last earlier face of its zone that writes a cell it reads or writes,
  // or reads a cell it writes, so every such pair keeps the per-face order and
  // the faces of a wave touch disjoint cells. Footprints along the normal:
  // writes from the boundary layer (types that set it) or the first ghost
  // layer out to ngg ghosts; reads from the boundary layer ngg layers inward
  // (periodic: the layers one period back from its ghosts); tangentially the
  // face's ranges.
  std::vector<std::pair<size_t, size_t>> bc_spans;
  {
    struct Box {
      int lo[3], hi[3];
    };
    auto boxes = [&](const BcFace &b, Box &W, Box &R) {
      const int f = b.face, d = b.direction, g = ctx->dz[b.zone].ngg, bi = b.rs[f];
      for (int a = 0; a < 3; ++a) W.lo[a] = R.lo[a] = b.rs[a], W.hi[a] = R.hi[a] = b.re[a];
      const bool sets_boundary = b.type == OSTC_BC_INFLOW || b.type == OSTC_BC_SYMMETRY || b.type == OSTC_BC_WALL ||
                                 b.type == OSTC_BC_FARFIELD;
      const int wa = sets_boundary ? bi : bi + d, wb = bi + d * g;
      int ra = bi, rb = bi - d * g;
      if (b.type == OSTC_BC_PERIODIC) {  // go = g + gg * dir_stride reads go - period_stride
        const int ext[3] = {ctx->dz[b.zone].mx, ctx->dz[b.zone].my, ctx->dz[b.zone].mz};
        ra = bi + d - d * ext[f], rb = bi + d * g - d * ext[f];
      }
      W.lo[f] = std::min(wa, wb), W.hi[f] = std::max(wa, wb);
      R.lo[f] = std::min(ra, rb), R.hi[f] = std::max(ra, rb);
    };
    auto meet = [](const Box &x, const Box &y) {
      for (int a = 0; a < 3; ++a)
        if (x.hi[a] < y.lo[a] || y.hi[a] < x.lo[a]) return false;
      return true;
    };
    static const int order[] = {OSTC_BC_FARFIELD,        OSTC_BC_OUTFLOW,  OSTC_BC_BACK_PRESSURE, OSTC_BC_INFLOW,
                                OSTC_BC_SUBSONIC_INFLOW, OSTC_BC_SYMMETRY, OSTC_BC_WALL,          OSTC_BC_PERIODIC};
    std::vector<int> qs, wave;
    std::vector<Box> W, R;
    for (int t : order)
      for (size_t q = 0; q < ctx->faces.size(); ++q) {
        if (ctx->faces[q].type != t) continue;
        Box w, r;
        boxes(ctx->faces[q], w, r);
        int wv = 0;
        for (size_t p = 0; p < qs.size(); ++p) {
          if (ctx->faces[qs[p]].zone != ctx->faces[q].zone) continue;
          if (meet(w, W[p]) || meet(w, R[p]) || meet(W[p], r)) wv = std::max(wv, wave[p] + 1);
        }
        qs.push_back((int)q), wave.push_back(wv), W.push_back(w), R.push_back(r);
      }
    const int n_waves = qs.empty() ? 0 : *std::max_element(wave.begin(), wave.end()) + 1;
    for (int wv = 0; wv < n_waves; ++wv) {
      const size_t b0 = all.size();
      for (size_t p = 0; p < qs.size(); ++p) {
        if (wave[p] != wv) continue;
        const BcFace &b = ctx->faces[qs[p]];
        const int n[3] = {b.re[0] - b.rs[0] + 1, b.re[1] - b.rs[1] + 1, b.re[2] - b.rs[2] + 1};
        wave_tiles(qs[p], b.face, n);
      }
      bc_spans.push_back({b0, all.size()});
    }
  }
  // interfaces in the order of data_communication (block by block, each
  // block's faces in order; DataCommunication.cuh:30-49), split into waves
  // the same way: a face goes one wave after the last earlier face that writes
  // a cell it reads or writes, or reads a cell it writes. A face writes its
  // own range in its zone and the coincident plane in its partner's, and
  // reads the partner's range and its own plane.
  std::vector<std::pair<size_t, size_t>> if_spans;
  {
    struct ZBox {
      int zone, lo[3], hi[3];
    };
    auto meet = [](const ZBox &x, const ZBox &y) {
      if (x.zone != y.zone) return false;
      for (int a = 0; a < 3; ++a)
        if (x.hi[a] < y.lo[a] || y.hi[a] < x.lo[a]) return false;
      return true;
    };
    struct Foot {
      ZBox w[2], r[2];
    };
    auto foot = [&](const Iface &f) {
      Foot o;
      ZBox self{f.zone, {}, {}}, tar{f.target, {}, {}};
      for (int d = 0; d < 3; ++d) {
        const int a = f.rs[d], b = f.rs[d] + f.ld[d] * (f.np[d] - 1);
        self.lo[d] = std::min(a, b), self.hi[d] = std::max(a, b);
        const int span = f.np[f.st[d]] - 1;
        const int ta = f.ts[d], tb = f.ts[d] + f.tld[d] * f.ld[f.st[d]] * span;
        tar.lo[d] = std::min(ta, tb), tar.hi[d] = std::max(ta, tb);
      }
      // the coincident plane: n[face] fixed where idx[face] == plane
      const int plane = f.direction > 0 ? f.rs[f.face] : f.rs[f.face] + f.ld[f.face] * (f.np[f.face] - 1);
      const int nf = (plane - f.rs[f.face]) / f.ld[f.face];
      ZBox sp = self, tp = tar;
      sp.lo[f.face] = sp.hi[f.face] = plane;
      for (int d = 0; d < 3; ++d)
        if (f.st[d] == f.face) tp.lo[d] = tp.hi[d] = f.ts[d] + f.tld[d] * f.ld[f.face] * nf;
      o.w[0] = self, o.w[1] = tp, o.r[0] = tar, o.r[1] = sp;
      return o;
    };
    auto conflict = [&](const Foot &x, const Foot &y) {
      for (const ZBox &a : x.w) {
        for (const ZBox &b : y.w)
          if (meet(a, b)) return true;
        for (const ZBox &b : y.r)
          if (meet(a, b)) return true;
      }
      for (const ZBox &a : y.w)
        for (const ZBox &b : x.r)
          if (meet(a, b)) return true;
      return false;
    };
    std::vector<int> qs, wave;
    std::vector<Foot> fs;
    for (size_t b = 0; b < ctx->dz.size(); ++b)
      for (size_t q = 0; q < ctx->ifaces.size(); ++q) {
        if (ctx->iface_zone[q] != (int)b) continue;
        const Foot f = foot(ctx->ifaces[q]);
        int wv = 0;
        for (size_t p = 0; p < qs.size(); ++p)
          if (conflict(f, fs[p])) wv = std::max(wv, wave[p] + 1);
        qs.push_back((int)q), wave.push_back(wv), fs.push_back(f);
      }
    const int n_waves = qs.empty() ? 0 : *std::max_element(wave.begin(), wave.end()) + 1;
    for (int wv = 0; wv < n_waves; ++wv) {
      const size_t b0 = all.size();
      for (size_t p = 0; p < qs.size(); ++p) {
        if (wave[p] != wv) continue;
        const Iface &f = ctx->ifaces[qs[p]];
        if (f.face == 0) {  // tiles of 4 layers x 8 (j) x 8 (k) points
          for (int tc = 0; tc < (f.np[0] + 3) / 4; ++tc)
            for (int tb = 0; tb < (f.np[2] + 7) / 8; ++tb)
              for (int ta = 0; ta < (f.np[1] + 7) / 8; ++ta) all.push_back(make_int4(qs[p], ta, tb, tc));
        } else {
          wave_tiles(qs[p], f.face, f.np);
        }
      }
      if_spans.push_back({b0, all.size()});
    }
    if (ctx->ifaces.size() > ctx->ifaces_cap) {
      cudaFree(ctx->ifaces_dev);
      ctx->ifaces_dev = nullptr;
      ctx->ifaces_cap = 0;
      CK(cudaMalloc(&ctx->ifaces_dev, sizeof(Iface) * ctx->ifaces.size()));
      ctx->ifaces_cap = ctx->ifaces.size();
    }
    if (!ctx->ifaces.empty())
      CK(cudaMemcpy(ctx->ifaces_dev, ctx->ifaces.data(), sizeof(Iface) * ctx->ifaces.size(), cudaMemcpyHostToDevice));
  }
  if (!ctx->faces.empty() && !ctx->faces_dev) {
    CK(cudaMalloc(&ctx->faces_dev, sizeof(BcFace) * ctx->faces.size()));
    CK(cudaMemcpy(ctx->faces_dev, ctx->faces.data(), sizeof(BcFace) * ctx->faces.size(), cudaMemcpyHostToDevice));
  }
  if (all.size() > (size_t)INT32_MAX) return fail(ctx, OSTC_ERR_UNSUPPORTED);
  if (all.size() > ctx->tab_cap) {
    cudaFree(ctx->tab_dev);
    ctx->tab_dev = nullptr;
    ctx->tab_cap = 0;
    CK(cudaMalloc(&ctx->tab_dev, sizeof(int4) * all.size()));
    ctx->tab_cap = all.size();
  }
  if (!all.empty()) CK(cudaMemcpy(ctx->tab_dev, all.data(), sizeof(int4) * all.size(), cudaMemcpyHostToDevice));
  auto table = [&](size_t q) {
    FluxTable t;
    t.tiles = ctx->tab_dev + spans[q].first;
    t.n = (int)(spans[q].second - spans[q].first);
    return t;
  };
  for (int c = 0; c < 3; ++c) ctx->cell_tab[c] = table(c);
  for (int d = 0; d < 3; ++d)
    for (int v = 0; v < 2; ++v) {
      ctx->flux_tab[d][v] = table(3 + 2 * d + v);
      ctx->flux_tab[d][v].n_bulk = (int)flux_bulk_tiles[2 * d + v];
    }
  // the wave plans: tiles from the first wave's on, ends relative to it; the
  // boundary plan's ends first in wave_ends_dev, then the interfaces'
  std::vector<int> ends;
  auto plan = [&](const std::vector<std::pair<size_t, size_t>> &sp, WavePlan &p) {
    p = WavePlan{};
    if (sp.empty()) return;
    p.tiles = ctx->tab_dev + sp.front().first;
    p.n_waves = (int)sp.size();
    for (const auto &w : sp) {
      ends.push_back((int)(w.second - sp.front().first));
      p.max_tiles = std::max(p.max_tiles, (int)(w.second - w.first));
    }
  };
  plan(bc_spans, ctx->bc_plan);
  plan(if_spans, ctx->if_plan);
  if (ends.size() > ctx->wave_ends_cap) {
    cudaFree(ctx->wave_ends_dev);
    ctx->wave_ends_dev = nullptr;
    ctx->wave_ends_cap = 0;
    CK(cudaMalloc(&ctx->wave_ends_dev, sizeof(int) * ends.size()));
    ctx->wave_ends_cap = ends.size();
  }
  if (!ends.empty())
    CK(cudaMemcpy(ctx->wave_ends_dev, ends.data(), sizeof(int) * ends.size(), cudaMemcpyHostToDevice));
  if (ctx->bc_plan.n_waves) ctx->bc_plan.ends = ctx->wave_ends_dev;
  if (ctx->if_plan.n_waves) ctx->if_plan.ends = ctx->wave_ends_dev + ctx->bc_plan.n_waves;
  if (!ctx->wave_sync) {
    CK(cudaMalloc(&ctx->wave_sync, 2 * sizeof(WaveSync)));
    CK(cudaMemset(ctx->wave_sync, 0, 2 * sizeof(WaveSync)));
  }
  return OSTC_OK;
}

// one per-cell kernel family over every zone: a tile-table launch when
// batched (table: 0 interior, 1 properties range, 2 ghosted), else one
// launch per zone
ostc_status cells_all(ostc_ctx *ctx, CellOp op, int table, const CellArgs &a, cudaStream_t s);

template <typename F>
cudaError_t dispatch_ns(int ns, F &&f) {
  // every species count has a build: 0 and 9 in kernels.cu / flux0.cu / flux9.cu, the others in
  // kernels_ns_*.cu / flux_ns_*.cu
  static_assert(OSTC_MAX_SPEC == 20, "one case per species count");
  switch (ns) {
    case 0: return f(std::integral_constant<int, 0>{});
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 5: return f(std::integral_constant<int, 5>{});
    case 6: return f(std::integral_constant<int, 6>{});
    case 7: return f(std::integral_constant<int, 7>{});
    case 8: return f(std::integral_constant<int, 8>{});
    case 9: return f(std::integral_constant<int, 9>{});
    case 10: return f(std::integral_constant<int, 10>{});
    case 11: return f(std::integral_constant<int, 11>{});
    case 12: return f(std::integral_constant<int, 12>{});
    case 13: return f(std::integral_constant<int, 13>{});
    case 14: return f(std::integral_constant<int, 14>{});
    case 15: return f(std::integral_constant<int, 15>{});
    case 16: return f(std::integral_constant<int, 16>{});
    case 17: return f(std::integral_constant<int, 17>{});
    case 18: return f(std::integral_constant<int, 18>{});
    case 19: return f(std::integral_constant<int, 19>{});
    case 20: return f(std::integral_constant<int, 20>{});
    default: return cudaErrorInvalidValue;
  }
}

// the flux kernels of the context's build: species count and turbulence scalars
cudaError_t flux_launch(const ostc_ctx *ctx, const DevZone &z, int d, const FluxTable *tab, int accumulate, int part,
                        cudaStream_t s) {
  const int inv = ctx->prm.inviscid_type;
  const int vis = ctx->prm.viscous_scheme != 0;
  if (ctx->nt == 2)
    return ctx->ns == 9 ? launch_flux_nt<9, 2>(z, inv, d, ctx->tile[d], tab, accumulate, vis, part, s)
                        : launch_flux_nt<0, 2>(z, inv, d, ctx->tile[d], tab, accumulate, vis, part, s);
  return dispatch_ns(ctx->ns, [&](auto n) {
    return launch_flux_nt<decltype(n)::value, 0>(z, inv, d, ctx->tile[d], tab, accumulate, vis, part, s);
  });
}

ostc_status cells_all(ostc_ctx *ctx, CellOp op, int table, const CellArgs &a, cudaStream_t s) {
  if (ctx->batched) {
    CK(dispatch_ns(ctx->ns, [&](auto n) {
      return launch_cells_table<decltype(n)::value>(op, ctx->cell_tab[table], a, s);
    }));
    return OSTC_OK;
  }
  for (auto &z : ctx->dz) CK(dispatch_ns(ctx->ns, [&](auto n) { return launch_cells<decltype(n)::value>(op, z, a, s); }));
  return OSTC_OK;
}

// repack the reference's 80-byte gxl::Matrix<real,3,3,1> records into 9 planes
__global__ void repack_metric_kernel(const unsigned char *src, double *dst, long long n) {
  const long long q = blockIdx.x * 256ll + threadIdx.x;
  if (q >= n) return;
  const double *m = (const double *)(src + 80 * q + 8);
#pragma unroll
  for (int c = 0; c < 9; ++c) dst[c * n + q] = m[c];
}

__global__ void step_end_kernel(const double *partial, int n_part, double n_total, const double *dt_dev,
                                double dt_fixed, double *hist_res, double *hist_dt, int *counter, int cap) {
  if (threadIdx.x != 0) return;
  const int s = *counter;
  if (s < cap) {
    if (hist_res && partial) {
      for (int l = 0; l < 4; ++l) {
        double acc = 0;
        for (int p = 0; p < n_part; ++p) acc += partial[p * 4 + l];
        hist_res[s * 4 + l] = sqrt(acc / n_total);
      }
    }
    if (hist_dt) hist_dt[s] = dt_dev ? *dt_dev : dt_fixed;
  }
  *counter = s + 1;
}

void fill_devzone(const ostc_zone &z, DevZone &d) {
  d.mx = z.mx;
  d.my = z.my;
  d.mz = z.mz;
  d.ngg = z.ngg;
  auto strides = [&](int g, int &s2, int &s1, int &st, long long &sz) {
    s2 = z.mx + 2 * g;
    s1 = (z.my + 2 * g) * s2;
    st = (s1 + s2 + 1) * g;
    sz = (long long)(z.mx + 2 * g) * (z.my + 2 * g) * (z.mz + 2 * g);
  };
  strides(z.ngg, d.d2, d.d1, d.dt_, d.sz);
  strides(z.dq_ngg, d.q2, d.q1, d.qt, d.qsz);
  int dummy;
  strides(0, d.n2, d.n1, dummy, d.nsz);
  d.isz = (int)d.sz;
  d.iqsz = (int)d.qsz;
  d.bv = z.bv;
  d.sv = z.sv;
  d.cv = z.cv;
  d.qn = z.qn;
  d.dq = z.dq;
  d.vel = z.vel;
  d.a = z.acoustic_speed;
  d.mach = z.mach;
  d.mul = z.mul;
  d.kappa = z.thermal_conductivity;
  d.rhoD = z.rho_D;
  d.gam = z.gamma;
  d.cp = z.cp;
  d.mut = z.mut;
  d.ttc = z.turb_therm_cond;
  d.wall = z.wall_distance;
  d.dt_local = z.dt_local;
  d.bv_last = z.bv_last;
  d.isr = nullptr;
  d.tsj = z.turb_src_jac;
  d.jac = z.jac;
}

// kZoneBulk when the ghosted row length (and so the plane size) is even and the
// planes the staged flux kernels copy start on 16-byte boundaries
static int zone_flags(const DevZone &d) {
  auto a16 = [](const void *p) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  const bool ok = d.d2 % 2 == 0 && d.isz % 2 == 0 && a16(d.bv) && a16(d.sv) && a16(d.met) && a16(d.jac) &&
                  a16(d.mul) && a16(d.kappa) && a16(d.rhoD) && a16(d.mut) && a16(d.ttc) && a16(d.wall);
  return ok ? kZoneBulk : 0;
}

ostc_status validate(const ostc_config *cfg, const ostc_param *p, const ostc_zone *zones, int n_zones,
                     const ostc_bc_face *faces, int n_faces) {
  if (!cfg || !p || !zones || n_zones <= 0 || (n_faces > 0 && !faces)) return OSTC_ERR_INVALID_ARG;
  const bool sst = p->turbulence != 0;
  if (sst) {
    // k-omega SST (rans_model 2): air or the 9-species mixtures (Driver<Air|Mixture|FR, SST>,
    // main.cu:25-96), primitive-variable reconstruction with AUSM+ or HLLC (and AWENO for air)
    if (p->rans_model != 2) return OSTC_ERR_UNSUPPORTED;
    if (cfg->chem_mode != 0) return OSTC_ERR_UNSUPPORTED;
    if (p->mix_model != OSTC_MIX_AIR && p->mix_model != OSTC_MIX_MIXTURE && p->mix_model != OSTC_MIX_FR)
      return OSTC_ERR_UNSUPPORTED;
    if (p->mix_model != OSTC_MIX_AIR && p->n_spec != 9) return OSTC_ERR_UNSUPPORTED;
    if (p->mix_model == OSTC_MIX_FR && (p->n_reac < 0 || p->n_reac > OSTC_MAX_REAC)) return OSTC_ERR_INVALID_ARG;
    if (p->turb_implicit != 0 && p->turb_implicit != 1) return OSTC_ERR_INVALID_ARG;
    // primitive-variable reconstruction with AUSM+ / HLLC, or AWENO (its Roe tag runs AUSM+, A1) with AUSM+ / HLLC
    const bool pv = p->inviscid_type == 0 && (p->inviscid_scheme == 3 || p->inviscid_scheme == 4);
    const bool aweno = p->inviscid_type == 1 && p->inviscid_scheme >= 2 && p->inviscid_scheme <= 4;
    if (!pv && !aweno) return OSTC_ERR_UNSUPPORTED;
    if (p->viscous_scheme == 0) return OSTC_ERR_UNSUPPORTED;
    const int ns = p->mix_model == OSTC_MIX_AIR ? 0 : p->n_spec;
    if (p->n_spec != ns || p->n_scalar != ns + 2 || p->n_var != 7 + ns || p->i_turb_cv != 5 + ns)
      return OSTC_ERR_INVALID_ARG;
    if (p->compressibility_correction < 0 || p->compressibility_correction > 3) return OSTC_ERR_INVALID_ARG;
    if (!(p->Prt > 0)) return OSTC_ERR_INVALID_ARG;
  } else if (p->mix_model == OSTC_MIX_AIR) {
    if (p->n_spec != 0 || p->n_var != 5 || p->n_scalar != 0) return OSTC_ERR_INVALID_ARG;
  } else if (p->mix_model == OSTC_MIX_MIXTURE || p->mix_model == OSTC_MIX_FR) {
    // any mechanism up to MAX_SPEC_NUMBER species (CMakeLists.txt:13-19)
    if (p->n_spec < 1 || p->n_spec > OSTC_MAX_SPEC) return OSTC_ERR_INVALID_ARG;
    if (p->n_var != 5 + p->n_spec || p->n_scalar != p->n_spec) return OSTC_ERR_INVALID_ARG;
    if (p->mix_model == OSTC_MIX_FR && (p->n_reac < 0 || p->n_reac > OSTC_MAX_REAC)) return OSTC_ERR_INVALID_ARG;
  } else {
    return OSTC_ERR_UNSUPPORTED;
  }
  if (p->inviscid_type == 1 && p->mix_model != OSTC_MIX_AIR) return OSTC_ERR_UNSUPPORTED;  // quirk A2
  if (p->inviscid_type == 1 && p->reconstruction != 4) return OSTC_ERR_INVALID_ARG;
  if (p->inviscid_type == 0 && p->inviscid_scheme == 1 && p->mix_model != OSTC_MIX_AIR) return OSTC_ERR_UNSUPPORTED;
  if (p->inviscid_type == 2 && p->inviscid_scheme != 2) return OSTC_ERR_INVALID_ARG;
  if (p->inviscid_scheme < 1 || p->inviscid_scheme > 4) return OSTC_ERR_INVALID_ARG;
  if (p->limiter != 0) return OSTC_ERR_INVALID_ARG;
  if (cfg->chem_mode < 0 || cfg->chem_mode > 2) return OSTC_ERR_INVALID_ARG;
  if (cfg->chem_mode != 0) {
    if (cfg->steady || p->mix_model != OSTC_MIX_FR || p->n_reac <= 0) return OSTC_ERR_INVALID_ARG;
    if (cfg->chem_mode == 2 && p->n_spec != 9) return OSTC_ERR_UNSUPPORTED;  // the surrogate's species count
  }
  if (cfg->steady) {
    if (cfg->implicit_method != 0 && cfg->implicit_method != 1) return OSTC_ERR_UNSUPPORTED;
    if (cfg->implicit_method == 1 && cfg->DPLUR_inner_step < 0) return OSTC_ERR_INVALID_ARG;
    // quirk A6: the reference's steady path never computes cv, which AWENO reads
    if (p->inviscid_type == 1) return OSTC_ERR_UNSUPPORTED;
    if (p->chemSrcMethod < 0 || p->chemSrcMethod > 2) return OSTC_ERR_INVALID_ARG;
  } else if (cfg->temporal_scheme != 3) {
    return OSTC_ERR_UNSUPPORTED;
  }
  if (!(p->cfl > 0) && !cfg->fixed_time_step) return OSTC_ERR_INVALID_ARG;
  const int need_ngg = p->inviscid_type == 1 ? 3 : 2;
  for (int b = 0; b < n_zones; ++b) {
    const ostc_zone &z = zones[b];
    if (z.mx < 2 || z.my < 2 || z.mz < 1 || z.ngg < need_ngg || z.dq_ngg < 0 || z.dq_ngg > 1)
      return OSTC_ERR_INVALID_ARG;
    // the problem is 2-D when the first block has mz == 1 (Mesh.cpp:612-614); every block alike
    if ((z.mz == 1) != (zones[0].mz == 1)) return OSTC_ERR_INVALID_ARG;
    if (!z.bv || !z.cv || !z.qn || !z.dq || !z.jac || !z.metric || !z.vel || !z.acoustic_speed || !z.mach ||
        !z.mul || !z.thermal_conductivity)
      return OSTC_ERR_INVALID_ARG;
    if (p->n_spec > 0 && (!z.sv || !z.rho_D || !z.gamma || !z.cp)) return OSTC_ERR_INVALID_ARG;
    if (sst && (!z.sv || !z.mut || !z.turb_therm_cond || !z.wall_distance)) return OSTC_ERR_INVALID_ARG;
    if (cfg->steady && !z.dt_local) return OSTC_ERR_INVALID_ARG;
    if (cfg->steady && cfg->implicit_method == 1 && z.dq_ngg != 1) return OSTC_ERR_INVALID_ARG;  // Field.cu:213-221
    // int32 ghosted index space
    const double np = (double)(z.mx + 2 * z.ngg) * (z.my + 2 * z.ngg) * (z.mz + 2 * z.ngg);
    if (np * std::max(p->n_var, 6) >= 2147483647.0) return OSTC_ERR_INVALID_ARG;
  }
  for (int q = 0; q < n_faces; ++q) {
    const ostc_bc_face &f = faces[q];
    if (f.block < 0 || f.block >= n_zones || f.face < 0 || f.face > 2 || (f.direction != 1 && f.direction != -1))
      return OSTC_ERR_INVALID_ARG;
    const ostc_zone &z = zones[f.block];
    const int ext[3] = {z.mx, z.my, z.mz};
    for (int d = 0; d < 3; ++d) {
      if (f.range_start[d] > f.range_end[d]) return OSTC_ERR_INVALID_ARG;
      if (d == f.face) {
        const int want = f.direction < 0 ? 0 : ext[d] - 1;
        if (f.range_start[d] != want || f.range_end[d] != want) return OSTC_ERR_INVALID_ARG;
      } else if (f.range_start[d] < -z.ngg || f.range_end[d] > ext[d] - 1 + z.ngg) {
        return OSTC_ERR_INVALID_ARG;
      }
    }
    switch (f.type_label) {
      case OSTC_BC_INFLOW:
      case OSTC_BC_OUTFLOW:
      case OSTC_BC_SYMMETRY:
      case OSTC_BC_WALL:
      case OSTC_BC_FARFIELD:
      case OSTC_BC_BACK_PRESSURE: break;
      case OSTC_BC_SUBSONIC_INFLOW:
        if (p->n_spec > 0) return OSTC_ERR_UNSUPPORTED;  // air only (BoundCond.cpp:300-305)
        break;
      case OSTC_BC_PERIODIC:
        if (ext[f.face] < z.ngg) return OSTC_ERR_INVALID_ARG;
        break;
      default: return OSTC_ERR_UNSUPPORTED;
    }
  }
  return OSTC_OK;
}

void build_devparam(const ostc_param *p, DevParam &d) {
  std::memset(&d, 0, sizeof(d));
  d.n_var = p->n_var;
  d.n_scalar = p->n_scalar;
  d.n_spec = p->n_spec;
  d.n_reac = p->mix_model == OSTC_MIX_FR ? p->n_reac : 0;
  d.mix = p->mix_model;
  d.inviscid_scheme = p->inviscid_scheme;
  d.reconstruction = p->reconstruction;
  d.limiter = p->limiter;
  d.inviscid_type = p->inviscid_type;
  d.viscous_scheme = p->viscous_scheme;
  d.chemSrcMethod = p->chemSrcMethod;
  d.gradP = p->gradPInDiffusionFlux;
  d.dimension = p->dimension;
  d.turbulence = p->turbulence;
  d.sst = p->turbulence && p->rans_model == 2 ? 1 : 0;
  d.comp_corr = d.sst ? p->compressibility_correction : 0;
  d.turb_implicit = d.sst ? p->turb_implicit : 0;
  d.Pr = p->Pr;
  d.Prt = p->Prt;
  d.Sct = p->Sct;
  d.Sc = p->Sc;
  d.cfl = p->cfl;
  d.entropy_fix_factor = p->entropy_fix_factor;
  const int ns = p->n_spec;
  for (int i = 0; i < ns; ++i) {
    d.mw[i] = p->mw[i];
    d.imw[i] = 1.0 / p->mw[i];
    d.Rmw[i] = R_u / p->mw[i];
    for (int c = 0; c < 7; ++c) {
      d.lo[i][c] = p->low_temp_coeff[i * 7 + c];
      d.hi[i][c] = p->high_temp_coeff[i * 7 + c];
    }
    d.t_low[i] = p->t_low[i];
    d.t_mid[i] = p->t_mid[i];
    d.LJ_inv[i] = p->LJ_potent_inv[i];
    d.vis_coeff[i] = p->vis_coeff[i];
    d.LJm145[i] = std::pow(p->LJ_potent_inv[i], -0.145);
    for (int j = 0; j < ns; ++j) {
      d.kbem145[i][j] = i == j ? 0.0 : std::pow(p->kb_over_eps_jk[i * ns + j], -0.145);
      d.inv_bdc[i][j] = i == j ? 0.0 : 1.0 / p->binary_diffusivity_coeff[i * ns + j];
      d.WjWi4[i][j] = p->WjDivWi_to_One4th[i * ns + j];
      d.sqWW8[i][j] = p->sqrt_WiDivWjPl1Mul8[i * ns + j];
      d.bdc[i][j] = p->binary_diffusivity_coeff[i * ns + j];
      d.kbe[i][j] = p->kb_over_eps_jk[i * ns + j];
    }
  }
  for (int r = 0; r < d.n_reac; ++r) {
    d.reac_type[r] = p->reac_type[r];
    d.reac_order[r] = p->reac_order[r];
    d.A[r] = p->A[r];
    d.b[r] = p->b[r];
    d.Ea[r] = p->Ea[r];
    d.A2[r] = p->A2[r];
    d.b2[r] = p->b2[r];
    d.Ea2[r] = p->Ea2[r];
    d.troe_alpha[r] = p->troe_alpha[r];
    d.troe_t3[r] = p->troe_t3[r];
    d.troe_t1[r] = p->troe_t1[r];
    d.troe_t2[r] = p->troe_t2[r];
    for (int l = 0; l < ns; ++l) {
      d.nuf[r][l] = (signed char)p->stoi_f[r * ns + l];
      d.nub[r][l] = (signed char)p->stoi_b[r * ns + l];
      d.tb[r][l] = p->third_body_coeff[r * ns + l];
    }
    if (d.reac_type[r] != 0 && d.reac_type[r] != 2) d.need_gibbs = 1;
  }
}

// default tile shapes: enough CTAs for ~4 per SM, as few re-computed faces as possible
void default_tiles(ostc_ctx *c) {
  const DevZone &z = c->dz[0];
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long target = 4ll * sms;
  // x: rows 4, chunks so a segment spans the line, unless that leaves too few CTAs
  {
    int R = 4, C = (z.mx + 1 + 31) / 32;
    while (C > 1 && (long long)((z.mx + 32 * C - 2) / (32 * C - 1)) * ((z.my + R - 1) / R) * z.mz < target) --C;
    c->tile[0] = {R, std::max(C, 1), 1};
  }
  for (int d = 1; d < 3; ++d) {
    const int n = d == 1 ? z.my : z.mz;
    const int other = d == 1 ? z.mz : z.my;
    int R = 8, C = (n + 1 + R - 1) / R;
    while (C > 1 && (long long)((z.mx + 31) / 32) * other * ((n + R * C - 2) / (R * C - 1)) < target) --C;
    c->tile[d] = {R, std::max(C, 1), 1};
  }
}

cudaStream_t S(void *s) { return (cudaStream_t)s; }

// the metric is immutable input: its SoA copy is refreshed at create and at
// every initialize, so callers may fill the 80-byte records after ostc_create
ostc_status repack_metrics(ostc_ctx *ctx, cudaStream_t s) {
  for (size_t b = 0; b < ctx->dz.size(); ++b) {
    const long long n = ctx->dz[b].sz;
    repack_metric_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
        (const unsigned char *)ctx->zones[b].metric, ctx->met_soa[b], n);
    CK(cudaGetLastError());
  }
  return OSTC_OK;
}

}  // namespace

// ===========================================================================
extern "C" {

const char *ostc_version(void) { return OSTC_VERSION_STRING; }

uint64_t ostc_zone_required(const ostc_config *cfg, const ostc_param *p) {
  // bit order = pointer members of ostc_zone starting at x
  enum { X, Y, Z_, JAC, MET, WALL, CV, BV, SV, BVL, VEL, A, MACH, MUL, KAP, RHOD, GAM, CP, CHEM, MUT, TTC, TSJ,
         DQ, DQ0, DQK, ISR, VSR, DTL, EFD, QN };
  uint64_t m = (1ull << JAC) | (1ull << MET) | (1ull << CV) | (1ull << BV) | (1ull << VEL) | (1ull << A) |
               (1ull << MACH) | (1ull << MUL) | (1ull << KAP) | (1ull << DQ) | (1ull << QN);
  if (p && p->n_spec > 0) m |= (1ull << SV) | (1ull << RHOD) | (1ull << GAM) | (1ull << CP);
  if (cfg && cfg->output_screen > 0) m |= (1ull << BVL);
  return m;
}

ostc_status ostc_create(const ostc_config *cfg, const ostc_param *param, const ostc_zone *zones, int n_zones,
                        const ostc_bc_face *faces, int n_faces, ostc_ctx **out) {
  if (!out) return OSTC_ERR_INVALID_ARG;
  *out = nullptr;
  ostc_status st = validate(cfg, param, zones, n_zones, faces, n_faces);
  if (st != OSTC_OK) return st;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return OSTC_ERR_NO_DEVICE;
  std::unique_ptr<ostc_ctx> c(new ostc_ctx);
  ostc_ctx *ctx = c.get();
  c->cfg = *cfg;
  c->prm = *param;
  build_devparam(param, c->dp);
  c->ns = param->n_spec;
  c->nt = c->dp.sst ? 2 : 0;
  c->has_source = param->mix_model == OSTC_MIX_FR && c->dp.n_reac > 0;
  c->spec_ok = c->has_source && mechanism_is_h2air9(param->reac_type, param->stoi_f, param->stoi_b,
                                                    param->reac_order, param->n_reac, param->n_spec)
                   ? 1
                   : 0;
  c->spec_mech = c->spec_ok;
  c->zones.assign(zones, zones + n_zones);
  c->dz.resize(n_zones);
  for (int b = 0; b < n_zones; ++b) {
    fill_devzone(zones[b], c->dz[b]);
    c->dz[b].block_id = b;
    double *soa = nullptr;
    CK(cudaMalloc(&soa, sizeof(double) * 9 * c->dz[b].sz));
    c->met_soa.push_back(soa);
    c->dz[b].met = soa;
    c->dz[b].flags = zone_flags(c->dz[b]);
    c->n_total += (double)zones[b].mx * zones[b].my * zones[b].mz;
  }
  for (int q = 0; q < n_faces; ++q) {
    const ostc_bc_face &f = faces[q];
    const DevZone &z = c->dz[f.block];
    BcFace b{};
    b.type = f.type_label;
    b.face = f.face;
    b.direction = f.direction;
    for (int d = 0; d < 3; ++d) {
      b.rs[d] = f.range_start[d];
      b.re[d] = f.range_end[d];
    }
    const int unit = f.face == 0 ? 1 : (f.face == 1 ? z.d2 : z.d1);
    b.dir_stride = f.direction * unit;
    const int ext[3] = {z.mx, z.my, z.mz};
    b.period_stride = f.direction * unit * ext[f.face];
    b.density = f.density;
    b.u = f.u;
    b.v = f.v;
    b.w = f.w;
    b.pressure = f.pressure;
    b.temperature = f.temperature;
    b.velocity = f.velocity;
    b.mut = f.mut;
    for (int l = 0; l < OSTC_MAX_SPEC + 4; ++l) b.sv[l] = f.sv[l];
    b.wall_isothermal = f.wall_isothermal;
    b.wall_temperature = f.wall_temperature;
    b.acoustic_speed = f.acoustic_speed;
    b.entropy = f.entropy;
    b.specific_heat_ratio = f.specific_heat_ratio;
    b.mw = f.mw;
    b.total_pressure = f.total_pressure;
    b.total_temperature = f.total_temperature;
    b.zone = f.block;
    c->faces.push_back(b);
    c->face_zone.push_back(f.block);
  }
  if ((st = repack_metrics(ctx, nullptr))) return st;
  if (cfg->steady) {
    auto alloc = [&](size_t bytes) -> void * {
      void *p = nullptr;
      if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
      c->owned.push_back(p);
      return p;
    };
    const int nv = param->n_var, ns = param->n_spec;
    const bool dplur = cfg->implicit_method == 1;
    const bool chem = param->mix_model == OSTC_MIX_FR && c->dp.n_reac > 0;
    for (int b = 0; b < n_zones; ++b) {
      DevZone &z = c->dz[b];
      double *isr = (double *)alloc(sizeof(double) * 3 * z.nsz);
      if (!isr) return fail(ctx, OSTC_ERR_CUDA, cudaErrorMemoryAllocation);
      z.isr = isr;
      c->isr.push_back(isr);
      if (c->dp.sst && c->dp.turb_implicit == 1 && !z.tsj) {  // SST source Jacobian, 2 interior planes
        z.tsj = (double *)alloc(sizeof(double) * 2 * z.nsz);
        if (!z.tsj) return fail(ctx, OSTC_ERR_CUDA, cudaErrorMemoryAllocation);
      }
      double *d0 = nullptr, *dk = nullptr, *lu = nullptr, *da = nullptr;
      unsigned char *pv = nullptr;
      if (dplur) {
        d0 = zones[b].dq0 ? zones[b].dq0 : (double *)alloc(sizeof(double) * nv * z.qsz);
        dk = zones[b].dqk ? zones[b].dqk : (double *)alloc(sizeof(double) * nv * z.qsz);
        if (!d0 || !dk) return fail(ctx, OSTC_ERR_CUDA, cudaErrorMemoryAllocation);
        if (chem && param->chemSrcMethod == 1) {
          lu = (double *)alloc(sizeof(double) * ns * ns * z.nsz);
          pv = (unsigned char *)alloc((size_t)ns * z.nsz);
          if (!lu || !pv) return fail(ctx, OSTC_ERR_CUDA, cudaErrorMemoryAllocation);
        } else if (chem && param->chemSrcMethod == 2) {
          da = (double *)alloc(sizeof(double) * ns * z.nsz);
          if (!da) return fail(ctx, OSTC_ERR_CUDA, cudaErrorMemoryAllocation);
        }
      }
      c->dq0.push_back(d0);
      c->dqk.push_back(dk);
      c->lu.push_back(lu);
      c->piv.push_back(pv);
      c->da.push_back(da);
    }
  }
  if (cfg->chem_mode != 0) {
    for (auto &z : c->dz) c->max_cells = std::max(c->max_cells, (long long)z.nsz);
    const size_t per = 2 * (size_t)param->n_spec + 4;  // T p Y dt dY dT
    CK(cudaMalloc(&c->chem_buf, sizeof(double) * per * c->max_cells));
    c->owned.push_back(c->chem_buf);
    CK(cudaMalloc(&c->chem_stats, sizeof(long long) * 2));
    c->owned.push_back(c->chem_stats);
    CK(cudaMemset(c->chem_stats, 0, sizeof(long long) * 2));
  }
  CK(cudaMalloc(&c->dt_bits, sizeof(unsigned long long)));
  c->n_part_per_zone = 148 * 2;
  CK(cudaMalloc(&c->res_partial, sizeof(double) * 4 * c->n_part_per_zone * n_zones));
  CK(cudaMalloc(&c->hist_counter, sizeof(int)));
  CK(cudaMalloc(&c->bad_key, sizeof(unsigned long long)));
  CK(cudaMalloc(&c->ep_step, sizeof(int)));
  CK(cudaMalloc(&c->ep_time, sizeof(double)));
  CK(cudaMemset(c->ep_step, 0, sizeof(int)));
  CK(cudaMemset(c->ep_time, 0, sizeof(double)));
  CK(cudaDeviceSynchronize());
  default_tiles(ctx);
  // several blocks: one tile-table launch per kernel over all of them, the
  // boundary faces and interfaces in waves. One block: its faces in one wave
  // launch when they are small (launch-bound: 43 K face points of a 128 x 128
  // x 8 block, 0.042 ms per set against 0.056 face by face), else one launch
  // per face, whose per-type kernels run the large faces faster (406 K points
  // of a 256^3 block: 0.45 ms per set against 0.58)
  long long face_points = 0;
  for (const BcFace &b : c->faces)
    face_points += (long long)(b.re[0] - b.rs[0] + 1) * (b.re[1] - b.rs[1] + 1) * (b.re[2] - b.rs[2] + 1);
  constexpr long long kOneBlockWavePoints = 1 << 17;
  if (n_zones > 1 && n_zones <= kMaxTableZones) {
    c->batched = 1;
    c->face_batched = 1;
    if ((st = build_tables(ctx))) return st;
  } else if (n_zones == 1 && !c->faces.empty() && face_points <= kOneBlockWavePoints) {
    c->face_batched = 1;
    if ((st = build_tables(ctx))) return st;
  }
  *out = c.release();
  return OSTC_OK;
}

ostc_status ostc_destroy(ostc_ctx *ctx) {
  if (!ctx) return OSTC_ERR_INVALID_ARG;
  cudaDeviceSynchronize();
  for (auto &kv : ctx->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  for (double *p : ctx->met_soa) cudaFree(p);
  for (void *p : ctx->owned) cudaFree(p);
  cudaFree(ctx->dt_bits);
  cudaFree(ctx->tab_dev);
  cudaFree(ctx->faces_dev);
  cudaFree(ctx->ifaces_dev);
  cudaFree(ctx->wave_ends_dev);
  cudaFree(ctx->wave_sync);
  cudaFree(ctx->res_partial);
  cudaFree(ctx->hist_counter);
  cudaFree(ctx->bad_key);
  cudaFree(ctx->hist_res);
  cudaFree(ctx->hist_dt);
  cudaFree(ctx->ep_step);
  cudaFree(ctx->ep_time);
  cudaFree(ctx->mon.pts);
  cudaFree(ctx->mon.labels);
  cudaFree(ctx->mon.data);
  cudaFree(ctx->mon.counter);
  for (auto &st : ctx->stats) {
    cudaFree(st.s12);
    cudaFree(st.count);
  }
  if (g_uploaded == ctx) g_uploaded = nullptr;
  delete ctx;
  return OSTC_OK;
}

ostc_status ostc_get_error(const ostc_ctx *ctx, int *cuda_error, int *block, int *i, int *j, int *k) {
  if (!ctx) return OSTC_ERR_INVALID_ARG;
  if (cuda_error) *cuda_error = ctx->last_cuda;
  if (block) *block = ctx->err_block;
  if (i) *i = ctx->err_i;
  if (j) *j = ctx->err_j;
  if (k) *k = ctx->err_k;
  return ctx->last;
}

const double *ostc_dt_device(const ostc_ctx *ctx) { return ctx ? (const double *)ctx->dt_bits : nullptr; }

ostc_status ostc_compute_cv_from_bv(ostc_ctx *ctx, void *stream) {
  if (!ctx) return OSTC_ERR_INVALID_ARG;
  if (ensure_param(ctx, S(stream))) return ctx->last;
  return cells_all(ctx, CellOp::CvFromBv, 2, {}, S(stream));
}

ostc_status ostc_compute_rhs(ostc_ctx *ctx, void *stream) {
  if (!ctx) return OSTC_ERR_INVALID_ARG;
  if (ensure_param(ctx, S(stream))) return ctx->last;
  // the source kernel: finite-rate chemistry and / or the SST source with mut
  const bool source = (ctx->has_source && ctx->cfg.chem_mode == 0) || ctx->nt > 0;
  CellArgs src;
  src.spec = ctx->spec_mech;
  if (ctx->batched) {
    // every zone per launch: the same per-cell order (source, x, y, z) as below
    for (auto &z : ctx->dz)
      if (z.qt != 0) CK(cudaMemsetAsync(z.dq, 0, sizeof(double) * z.qsz * ctx->prm.n_var, S(stream)));
    const bool acc = ctx->dz[0].qt != 0 || source;
    if (source) {
      ostc_status st = cells_all(ctx, CellOp::Source, 0, src, S(stream));
      if (st) return st;
    }
    for (int d = 0; d < 3; ++d)
      CK(flux_launch(ctx, ctx->dz[0], d, ctx->flux_tab[d], (acc || d > 0) ? 1 : 0, 0, S(stream)));
    return OSTC_OK;
  }
  for (auto &z : ctx->dz) {
    if (z.qt != 0) CK(cudaMemsetAsync(z.dq, 0, sizeof(double) * z.qsz * ctx->prm.n_var, S(stream)));
    bool acc = z.qt != 0;
    if (source) {
      CK(dispatch_ns(ctx->ns, [&](auto n) { return launch_cells<decltype(n)::value>(CellOp::Source, z, src, S(stream)); }));
      acc = true;
    }
    for (int d = 0; d < (z.mz > 1 ? 3 : 2); ++d)
      CK(flux_launch(ctx, z, d, nullptr, (acc || d > 0) ? 1 : 0, 0, S(stream)));
  }
  return OSTC_OK;
}

ostc_status ostc_global_time_step(ostc_ctx *ctx, double *dt_host, void *stream) {
  if (!ctx) return OSTC_ERR_INVALID_ARG;
  if (ensure_param(ctx, S(stream))) return ctx->last;
  CellArgs a;
  a.dt_bits = ctx->dt_bits;
  CK(launch_cells<0>(CellOp::DtReset, ctx->dz[0], a, S(stream)));
  ostc_status st = cells_all(ctx, CellOp::Dt, 0, a, S(stream));
  if (st) return st;
  if (dt_host) {
    CK(cudaMemcpyAsync(dt_host, ctx->dt_bits, sizeof(double), cudaMemcpyDeviceToHost, S(stream)));
    CK(cudaStreamSynchronize(S(stream)));
  }
  return OSTC_OK;
}

ostc_status ostc_update_cv_and_bv_rk(ostc_ctx *ctx, double dt, int rk, void *stream) {
  if (!ctx || rk < 0 || rk > 2) return OSTC_ERR_INVALID_ARG;
  if (ensure_param(ctx, S(stream))) return ctx->last;
  CellArgs a;
  a.dt = dt;
  a.dt_dev = dt < 0 ? (const double *)ctx->dt_bits : nullptr;
  a.rk = rk;
  return cells_all(ctx, CellOp::UpdateRK, 0, a, S(stream));
}

ostc_status ostc_apply_boundary_conditions(ostc_ctx *ctx, int with_cv, void *stream) {
  if (!ctx) return OSTC_ERR_INVALID_ARG;
  if (ensure_param(ctx, S(stream))) return ctx->last;
  // priority order of BoundCond.cuh:673-822; periodic wraps after all others
  static const int order[] = {OSTC_BC_FARFIELD, OSTC_BC_OUTFLOW, OSTC_BC_BACK_PRESSURE, OSTC_BC_INFLOW,
                              OSTC_BC_SUBSONIC_INFLOW, OSTC_BC_SYMMETRY, OSTC_BC_WALL, OSTC_BC_PERIODIC};
  if (ctx->face_batched) {
    // every face in the per-face order's waves, one cooperative launch (build_tables)
    CK(dispatch_ns(ctx->ns, [&](auto n) {
      return launch_bc_waves<decltype(n)::value>(ctx->faces_dev, ctx->bc_plan, with_cv, ctx->wave_sync, S(stream));
    }));
    return OSTC_OK;
  }
  for (int t : order) {
    for (size_t q = 0; q < ctx->faces.size(); ++q) {
      if (ctx->faces[q].type != t) continue;
      const DevZone &z = ctx->dz[ctx->face_zone[q]];
      CK(dispatch_ns(ctx->ns, [&](auto n) { return launch_bc<decltype(n)::value>(z, ctx->faces[q], with_cv, S(stream)); }));
    }
  }
  return OSTC_OK;
}

ostc_status ostc_data_communication(ostc_ctx *ctx, int with_cv, void *stream) {
  if (!ctx) return OSTC_ERR_INVALID_ARG;
  if (ctx->ifaces.empty()) return OSTC_OK;
  if (ensure_param(ctx, S(stream))) return ctx->last;
  if (ctx->face_batched) {  // the waves of build_tables, one cooperative launch over all zones
    CK(dispatch_ns(ctx->ns, [&](auto n) {
      return launch_interface_waves<decltype(n)::value>(ctx->ifaces_dev, ctx->if_plan, with_cv, ctx->wave_sync + 1,
                                                        S(stream));
    }));
    return OSTC_OK;
  }
  // per block, per face, in order (DataCommunication.cuh:30-49)
  for (size_t b = 0; b < ctx->dz.size(); ++b)
    for (size_t q = 0; q < ctx->ifaces.size(); ++q) {
      if (ctx->iface_zone[q] != (int)b) continue;
      const DevZone &z = ctx->dz[b], &t = ctx->dz[ctx->iface_target[q]];
      CK(dispatch_ns(ctx->ns, [&](auto n) {
        return launch_interface<decltype(n)::value>(z, t, ctx->ifaces[q], with_cv, S(stream));
      }));
    }
  return OSTC_OK;
}

ostc_status ostc_set_interfaces(ostc_ctx *ctx, const ostc_interface *f, int n) {
  if (!ctx || n < 0 || (n > 0 && !f)) return OSTC_ERR_INVALID_ARG;
  std::vector<Iface> v;
  std::vector<int> zb, tb;
  const int nz = (int)ctx->zones.size();
  for (int q = 0; q < n; ++q) {
    const ostc_interface &a = f[q];
    if (a.block < 0 || a.block >= nz || a.target < 0 || a.target >= nz || a.face < 0 || a.face > 2 ||
        (a.direction != 1 && a.direction != -1))
      return OSTC_ERR_INVALID_ARG;
    const ostc_zone &z = ctx->zones[a.block], &t = ctx->zones[a.target];
    const int ez[3] = {z.mx, z.my, z.mz}, et[3] = {t.mx, t.my, t.mz};
    Iface g{};
    g.face = a.face;
    g.direction = a.direction;
    for (int d = 0; d < 3; ++d) {
      if (a.n_point[d] < 1 || (a.loop_dir[d] != 1 && a.loop_dir[d] != -1) ||
          (a.target_loop_dir[d] != 1 && a.target_loop_dir[d] != -1) || a.src_tar[d] < 0 || a.src_tar[d] > 2)
        return OSTC_ERR_INVALID_ARG;
      g.rs[d] = a.range_start[d];
      g.ts[d] = a.target_start[d];
      g.ld[d] = a.loop_dir[d];
      g.tld[d] = a.target_loop_dir[d];
      g.st[d] = a.src_tar[d];
      g.np[d] = a.n_point[d];
    }
    // every point of the range and of its partner must lie inside the ghosted arrays
    for (int d = 0; d < 3; ++d) {
      const int lo = std::min(g.rs[d], g.rs[d] + g.ld[d] * (g.np[d] - 1));
      const int hi = std::max(g.rs[d], g.rs[d] + g.ld[d] * (g.np[d] - 1));
      if (lo < -z.ngg || hi > ez[d] - 1 + z.ngg) return OSTC_ERR_INVALID_ARG;
      const int span = g.np[g.st[d]] - 1;
      const int tlo = std::min(g.ts[d], g.ts[d] + g.tld[d] * g.ld[g.st[d]] * span);
      const int thi = std::max(g.ts[d], g.ts[d] + g.tld[d] * g.ld[g.st[d]] * span);
      if (tlo < -t.ngg || thi > et[d] - 1 + t.ngg) return OSTC_ERR_INVALID_ARG;
    }
    g.zone = a.block;
    g.target = a.target;
    v.push_back(g);
    zb.push_back(a.block);
    tb.push_back(a.target);
  }
  ctx->ifaces.swap(v);
  ctx->iface_zone.swap(zb);
  ctx->iface_target.swap(tb);
  for (auto &kv : ctx->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  ctx->graphs.clear();
  if (ctx->batched || ctx->face_batched) return build_tables(ctx);  // the interface waves
  return OSTC_OK;
}

ostc_status ostc_eliminate_k_gradient(ostc_ctx *ctx, int with_cv, void *stream) {
  if (!ctx) return OSTC_ERR_INVALID_ARG;
  if (ensure_param(ctx, S(stream))) return ctx->last;
  for (auto &z : ctx->dz) CK(launch_eliminate_k(z, with_cv, S(stream)));
  return OSTC_OK;
}

ostc_status ostc_update_physical_properties(ostc_ctx *ctx, void *stream) {
  if (!ctx) return OSTC_ERR_INVALID_ARG;
  if (ensure_param(ctx, S(stream))) return ctx->last;
  return cells_all(ctx, CellOp::Properties, 1, {}, S(stream));
}

ostc_status ostc_initialize(ostc_ctx *ctx, void *stream) {
  if (!ctx) return OSTC_ERR_INVALID_ARG;
  ostc_status st;
  if ((st = repack_metrics(ctx, S(stream)))) return st;
  // a fresh run: step 0 at physical time 0
  CK(cudaMemsetAsync(ctx->ep_step, 0, sizeof(int), S(stream)));
  CK(cudaMemsetAsync(ctx->ep_time, 0, sizeof(double), S(stream)));
  // 2-D: the k ghost planes copy the plane k = 0 first (Driver.cu:54-60)
  if ((st = ostc_eliminate_k_gradient(ctx, 0, stream))) return st;
  if ((st = ostc_apply_boundary_conditions(ctx, 0, stream))) return st;
  if (ensure_param(ctx, S(stream))) return ctx->last;
  if ((st = cells_all(ctx, CellOp::Velocity, 2, {}, S(stream)))) return st;
  // SST: the initial turbulent viscosity over [-1, m] (Driver.cu:69-78)
  if (ctx->nt > 0 && (st = cells_all(ctx, CellOp::InitMut, 1, {}, S(stream)))) return st;
  if ((st = ostc_data_communication(ctx, 0, stream))) return st;
  if ((st = ostc_update_physical_properties(ctx, stream))) return st;
  return ostc_compute_cv_from_bv(ctx, stream);
}

ostc_status ostc_rk3_stage(ostc_ctx *ctx, int rk, void *stream) {
  if (!ctx || rk < 0 || rk > 2) return OSTC_ERR_INVALID_ARG;
  ostc_status st;
  if ((st = ostc_compute_rhs(ctx, stream))) return st;
  double dt = ctx->cfg.dt;
  if (!ctx->cfg.fixed_time_step) {
    if ((st = ostc_global_time_step(ctx, nullptr, stream))) return st;
    dt = -1;
  }
  if ((st = ostc_update_cv_and_bv_rk(ctx, dt, rk, stream))) return st;
  if ((st = ostc_apply_boundary_conditions(ctx, 1, stream))) return st;
  if ((st = ostc_data_communication(ctx, 1, stream))) return st;
  if ((st = ostc_eliminate_k_gradient(ctx, 1, stream))) return st;  // 2-D only (RK.cuh:147-153)
  return ostc_update_physical_properties(ctx, stream);
}

// one full step as enqueued work (captured into a graph by ostc_rk3_steps)
static ostc_status enqueue_step(ostc_ctx *ctx, bool with_hist, cudaStream_t s) {
  ostc_status st;
  if (with_hist && (st = cells_all(ctx, CellOp::StoreLast, 0, {}, s))) return st;
  for (auto &z : ctx->dz)
    CK(cudaMemcpyAsync(z.qn, z.cv, sizeof(double) * z.sz * ctx->prm.n_var, cudaMemcpyDeviceToDevice, s));
  for (int rk = 0; rk < 3; ++rk)
    if ((st = ostc_rk3_stage(ctx, rk, s))) return st;
  if (ctx->cfg.chem_mode != 0) {
    // operator-split chemistry over the step's dt (the last stage's dt, quirk A12)
    if (ctx->cfg.chem_mode == 2 && !ctx->sur) return fail(ctx, OSTC_ERR_INVALID_ARG);
    const double *dt_dev = ctx->cfg.fixed_time_step ? nullptr : (const double *)ctx->dt_bits;
    constexpr int NS_SUR = mlp::NIN - 3;  // the surrogate's species count
    const int ns = ctx->prm.n_spec;
    for (auto &z : ctx->dz) {
      // the staging layout of launch_chem_split: T, p, Y [ns][n], dt, dY [ns][n], dT
      const long long n = z.nsz;
      double *T = ctx->chem_buf, *p = T + n, *Y = p + n, *dt = Y + ns * n, *dY = dt + n, *dT = dY + ns * n;
      int *count = nullptr;
      CK(dispatch_ns(ctx->ns, [&](auto m) {
        return launch_chem_split<decltype(m)::value>(0, z, dt_dev, ctx->cfg.dt, ctx->chem_buf, nullptr, nullptr, s);
      }));
      if (ctx->cfg.chem_mode == 1) {
        CK(dispatch_ns(ctx->ns, [&](auto m) {
          return launch_chem_integrator<decltype(m)::value>((int)n, T, p, Y, dt, dY, dT, s);
        }));
      } else {
        ChemScratch w;
        CK(surrogate_scratch(ctx->sur, (int)n, &w));
        count = w.count;
        CK(launch_chem_surrogate<NS_SUR>(*surrogate_net(ctx->sur), (int)n, T, p, Y, dt, dY, dT, w, s));
      }
      CK(dispatch_ns(ctx->ns, [&](auto m) {
        return launch_chem_split<decltype(m)::value>(2, z, nullptr, 0, nullptr, ctx->chem_stats, count, s);
      }));
      CK(dispatch_ns(ctx->ns, [&](auto m) {
        return launch_chem_split<decltype(m)::value>(1, z, nullptr, 0, ctx->chem_buf, nullptr, nullptr, s);
      }));
    }
    if ((st = ostc_apply_boundary_conditions(ctx, 1, s))) return st;
    if ((st = ostc_data_communication(ctx, 1, s))) return st;
    if ((st = ostc_eliminate_k_gradient(ctx, 1, s))) return st;
    if ((st = ostc_update_physical_properties(ctx, s))) return st;
  }
  if (with_hist) {
    CellArgs a;
    a.n_part = ctx->n_part_per_zone;
    a.bad = ctx->bad_key;
    a.step = ctx->hist_counter;
    for (size_t b = 0; b < ctx->dz.size(); ++b) {
      a.partial = ctx->res_partial + 4 * ctx->n_part_per_zone * b;
      a.block = (int)b;
      CK(launch_cells<0>(CellOp::ResidualPartial, ctx->dz[b], a, s));
    }
    step_end_kernel<<<1, 32, 0, s>>>(ctx->res_partial, ctx->n_part_per_zone * (int)ctx->dz.size(), ctx->n_total,
                                     ctx->cfg.fixed_time_step ? nullptr : (const double *)ctx->dt_bits, ctx->cfg.dt,
                                     ctx->hist_res, ctx->hist_dt, ctx->hist_counter, ctx->hist_cap);
    CK(cudaGetLastError());
  }
  // epilogues (RK.cuh:164-180): physical_time += dt of the last stage, then the
  // monitor points and the statistics sums of the step
  CK(launch_step_clock(ctx->ep_step, ctx->ep_time,
                       ctx->cfg.fixed_time_step ? nullptr : (const double *)ctx->dt_bits, ctx->cfg.dt, s));
  if (ctx->mon.n > 0) {
    for (size_t b = 0; b < ctx->dz.size(); ++b) CK(launch_monitor(ctx->dz[b], (int)b, ctx->mon, s));
    CK(launch_monitor_advance(ctx->mon.counter, s));
  }
  if (ctx->stat_on)
    for (size_t b = 0; b < ctx->dz.size(); ++b)
      CK(launch_statistics(ctx->dz[b], ctx->ep_step, ctx->stat_start, ctx->stats[b], ctx->prm.n_spec, s));
  return OSTC_OK;
}

static ostc_status ensure_hist(ostc_ctx *ctx, int n_steps) {
  if (n_steps <= ctx->hist_cap) return OSTC_OK;
  cudaFree(ctx->hist_res);
  cudaFree(ctx->hist_dt);
  ctx->hist_res = ctx->hist_dt = nullptr;
  CK(cudaMalloc(&ctx->hist_res, sizeof(double) * 4 * n_steps));
  CK(cudaMalloc(&ctx->hist_dt, sizeof(double) * n_steps));
  ctx->hist_cap = n_steps;
  // cached graphs captured the old buffers
  for (auto &kv : ctx->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  ctx->graphs.clear();
  return OSTC_OK;
}

static ostc_status enqueue_steady_step(ostc_ctx *ctx, bool with_hist, cudaStream_t s);

static ostc_status ensure_graph(ostc_ctx *ctx, bool hist, GraphEntry **out, bool steady = false) {
  GraphEntry &ge = ctx->graphs[(hist ? 1 : 0) + (steady ? 2 : 0)];
  if (!ge.exec) {
    // parameters and zones uploaded now, so that the capture holds no upload
    // (every launch of the graph is preceded by ensure_param on its stream)
    if (g_uploaded != ctx) {
      if (ensure_param(ctx, nullptr)) return ctx->last;
      CK(cudaStreamSynchronize(nullptr));
    }
    // a legacy default stream cannot be captured: capture on a private stream
    cudaStream_t cs;
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    ostc_status st = steady ? enqueue_steady_step(ctx, hist, cs) : enqueue_step(ctx, hist, cs);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (st != OSTC_OK || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return st != OSTC_OK ? st : fail(ctx, OSTC_ERR_CUDA, e);
    }
    e = cudaGraphInstantiate(&ge.exec, g, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      ge.exec = nullptr;
      return fail(ctx, OSTC_ERR_CUDA, e);
    }
    ge.graph = g;
  }
  *out = &ge;
  return OSTC_OK;
}

// after a synchronised call with histories: the first non-physical cell found by
// the residual epilogue, if any, becomes OSTC_ERR_NONPHYSICAL with its zone and
// cell (ostc_get_error) and the step of the call it was found in (err_step)
static ostc_status check_state(ostc_ctx *ctx, unsigned long long key) {
  // a staged flux kernel that gave up waiting for its tile (bounded wait) left
  // its faces uncomputed: the steps are not valid
  int late = 0;
  CK(stage_timeouts(&late));
  // likewise a wave launch whose grid barrier ran out (the waves after it
  // were not computed); the flags are cleared for the next steps
  if (ctx->wave_sync) {
    WaveSync ws[2];
    CK(cudaMemcpy(ws, ctx->wave_sync, sizeof(ws), cudaMemcpyDeviceToHost));
    if (ws[0].timed_out || ws[1].timed_out) {
      const int zero = 0;
      for (int k = 0; k < 2; ++k)
        CK(cudaMemcpy(&ctx->wave_sync[k].timed_out, &zero, sizeof(int), cudaMemcpyHostToDevice));
      late = 1;
    }
  }
  if (late) return fail(ctx, OSTC_ERR_TIMEOUT);
  if (key == ~0ull) return OSTC_OK;
  const long long q = (long long)(key & ((1ull << 34) - 1));
  const int b = (int)((key >> 34) & 1023);
  if (b >= (int)ctx->dz.size()) return fail(ctx, OSTC_ERR_NONPHYSICAL);
  const DevZone &z = ctx->dz[b];
  ctx->err_block = b;
  ctx->err_i = (int)(q % z.mx);
  ctx->err_j = (int)((q / z.mx) % z.my);
  ctx->err_k = (int)(q / ((long long)z.mx * z.my));
  ctx->err_step = (int)(key >> 44);
  return fail(ctx, OSTC_ERR_NONPHYSICAL);
}

ostc_status ostc_rk3_steps(ostc_ctx *ctx, int n_steps, double *res_hist, double *dt_hist, void *stream) {
  if (!ctx || n_steps < 0) return OSTC_ERR_INVALID_ARG;
  if (ctx->cfg.steady) return OSTC_ERR_INVALID_ARG;
  cudaStream_t s = S(stream);
  const bool hist = res_hist || dt_hist;
  ostc_status st;
  if (hist && (st = ensure_hist(ctx, n_steps))) return st;
  if (ensure_param(ctx, s)) return ctx->last;
  if (hist) CK(cudaMemsetAsync(ctx->hist_counter, 0, sizeof(int), s));
  if (hist) CK(cudaMemsetAsync(ctx->bad_key, 0xff, sizeof(unsigned long long), s));
  GraphEntry *ge = nullptr;
  if ((st = ensure_graph(ctx, hist, &ge))) return st;
  for (int i = 0; i < n_steps; ++i) CK(cudaGraphLaunch(ge->exec, s));
  if (hist) {
    unsigned long long key = ~0ull;
    if (res_hist) CK(cudaMemcpyAsync(res_hist, ctx->hist_res, sizeof(double) * 4 * n_steps, cudaMemcpyDeviceToHost, s));
    if (dt_hist) CK(cudaMemcpyAsync(dt_hist, ctx->hist_dt, sizeof(double) * n_steps, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&key, ctx->bad_key, sizeof(key), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return check_state(ctx, key);
  }
  return OSTC_OK;
}

// ---------------------------------------------------------------------------
// steady path (SteadySim.cuh:15-137)
// ---------------------------------------------------------------------------
ostc_status ostc_local_time_step(ostc_ctx *ctx, void *stream) {
  if (!ctx || !ctx->cfg.steady) return OSTC_ERR_INVALID_ARG;
  if (ensure_param(ctx, S(stream))) return ctx->last;
  CellArgs a;
  a.dt_bits = ctx->dt_bits;
  CK(launch_cells<0>(CellOp::DtReset, ctx->dz[0], a, S(stream)));
  for (auto &z : ctx->dz)
    CK(dispatch_ns(ctx->ns, [&](auto n) { return launch_cells<decltype(n)::value>(CellOp::Dt, z, a, S(stream)); }));
  return OSTC_OK;
}

ostc_status ostc_implicit_treatment(ostc_ctx *ctx, void *stream) {
  if (!ctx || !ctx->cfg.steady) return OSTC_ERR_INVALID_ARG;
  if (ensure_param(ctx, S(stream))) return ctx->last;
  cudaStream_t s = S(stream);
  if (ctx->cfg.implicit_method == 0) {
    // ImplicitTreatmentHPP.cuh:11-48: the chemistry's EPI / DA, then SST's point-implicit k, omega sources
    if (ctx->has_source && ctx->prm.chemSrcMethod != 0)
      for (auto &z : ctx->dz)
        CK(dispatch_ns(ctx->ns, [&](auto n) {
          return launch_steady<decltype(n)::value>(SteadyOp::ChemImplicit, z, SteadyArgs{}, nullptr, s);
        }));
    if (ctx->dp.sst && ctx->dp.turb_implicit == 1)
      for (auto &z : ctx->dz) CK(launch_steady<0>(SteadyOp::TurbImplicit, z, SteadyArgs{}, nullptr, s));
    return OSTC_OK;
  }
  // DPLUR (DPLUR.cuh:283-312): no exchange between blocks inside the sweeps (quirk A11)
  for (size_t b = 0; b < ctx->dz.size(); ++b) {
    const DevZone &z = ctx->dz[b];
    SteadyArgs a;
    a.dq0 = ctx->dq0[b];
    a.lu = ctx->lu[b];
    a.piv = ctx->piv[b];
    a.da = ctx->da[b];
    CK(dispatch_ns(ctx->ns, [&](auto n) { return launch_steady<decltype(n)::value>(SteadyOp::DplurDq0, z, a, nullptr, s); }));
    double *cur = z.dq, *nxt = ctx->dqk[b];
    for (int it = 0; it < ctx->cfg.DPLUR_inner_step; ++it) {
      for (size_t q = 0; q < ctx->faces.size(); ++q) {
        if (ctx->face_zone[q] != (int)b || ctx->faces[q].type != OSTC_BC_WALL) continue;
        SteadyArgs w;
        w.dq_out = cur;
        CK(dispatch_ns(ctx->ns, [&](auto n) {
          return launch_steady<decltype(n)::value>(SteadyOp::WallDqZero, z, w, &ctx->faces[q], s);
        }));
      }
      a.dq_in = cur;
      a.dq_out = nxt;
      CK(dispatch_ns(ctx->ns, [&](auto n) { return launch_steady<decltype(n)::value>(SteadyOp::DplurSweep, z, a, nullptr, s); }));
      std::swap(cur, nxt);
    }
    a.dq_in = cur;
    CK(dispatch_ns(ctx->ns, [&](auto n) { return launch_steady<decltype(n)::value>(SteadyOp::DplurFinish, z, a, nullptr, s); }));
  }
  return OSTC_OK;
}

ostc_status ostc_update_bv(ostc_ctx *ctx, void *stream) {
  if (!ctx || !ctx->cfg.steady) return OSTC_ERR_INVALID_ARG;
  if (ensure_param(ctx, S(stream))) return ctx->last;
  for (auto &z : ctx->dz)
    CK(dispatch_ns(ctx->ns, [&](auto n) {
      return launch_steady<decltype(n)::value>(SteadyOp::UpdateBv, z, SteadyArgs{}, nullptr, S(stream));
    }));
  return OSTC_OK;
}

static ostc_status enqueue_steady_step(ostc_ctx *ctx, bool with_hist, cudaStream_t s) {
  ostc_status st;
  if (with_hist)
    for (auto &z : ctx->dz) CK(launch_cells<0>(CellOp::StoreLast, z, {}, s));
  if ((st = ostc_compute_rhs(ctx, s))) return st;
  if ((st = ostc_local_time_step(ctx, s))) return st;
  if ((st = ostc_implicit_treatment(ctx, s))) return st;
  if ((st = ostc_update_bv(ctx, s))) return st;
  if ((st = ostc_apply_boundary_conditions(ctx, 0, s))) return st;
  if ((st = ostc_data_communication(ctx, 0, s))) return st;
  if ((st = ostc_eliminate_k_gradient(ctx, 0, s))) return st;  // 2-D only (SteadySim.cuh:101-107)
  if ((st = ostc_update_physical_properties(ctx, s))) return st;
  if (with_hist) {
    CellArgs a;
    a.n_part = ctx->n_part_per_zone;
    a.bad = ctx->bad_key;
    a.step = ctx->hist_counter;
    for (size_t b = 0; b < ctx->dz.size(); ++b) {
      a.partial = ctx->res_partial + 4 * ctx->n_part_per_zone * b;
      a.block = (int)b;
      CK(launch_cells<0>(CellOp::ResidualPartial, ctx->dz[b], a, s));
    }
    step_end_kernel<<<1, 32, 0, s>>>(ctx->res_partial, ctx->n_part_per_zone * (int)ctx->dz.size(), ctx->n_total,
                                     nullptr, 0.0, ctx->hist_res, nullptr, ctx->hist_counter, ctx->hist_cap);
    CK(cudaGetLastError());
  }
  return OSTC_OK;
}

ostc_status ostc_steady_steps(ostc_ctx *ctx, int n_steps, double *res_hist, void *stream) {
  if (!ctx || n_steps < 0 || !ctx->cfg.steady) return OSTC_ERR_INVALID_ARG;
  cudaStream_t s = S(stream);
  const bool hist = res_hist != nullptr;
  ostc_status st;
  if (hist && (st = ensure_hist(ctx, n_steps))) return st;
  if (ensure_param(ctx, s)) return ctx->last;
  if (hist) CK(cudaMemsetAsync(ctx->hist_counter, 0, sizeof(int), s));
  if (hist) CK(cudaMemsetAsync(ctx->bad_key, 0xff, sizeof(unsigned long long), s));
  GraphEntry *ge = nullptr;
  if ((st = ensure_graph(ctx, hist, &ge, true))) return st;
  for (int i = 0; i < n_steps; ++i) CK(cudaGraphLaunch(ge->exec, s));
  if (hist) {
    unsigned long long key = ~0ull;
    CK(cudaMemcpyAsync(res_hist, ctx->hist_res, sizeof(double) * 4 * n_steps, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&key, ctx->bad_key, sizeof(key), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return check_state(ctx, key);
  }
  return OSTC_OK;
}

ostc_status ostc_chem_point_implicit(ostc_ctx *ctx, int n, const double *T, const double *p, const double *Y,
                                     const double *dt, double *dY, double *dT, void *stream) {
  if (!ctx || n < 0 || (n > 0 && (!T || !p || !Y || !dt || !dY || !dT))) return OSTC_ERR_INVALID_ARG;
  if (!ctx->has_source) return OSTC_ERR_INVALID_ARG;  // needs a finite-rate mechanism
  if (ensure_param(ctx, S(stream))) return ctx->last;
  CK(dispatch_ns(ctx->ns, [&](auto m) {
    return launch_chem_integrator<decltype(m)::value>(n, T, p, Y, dt, dY, dT, S(stream));
  }));
  return OSTC_OK;
}

ostc_status ostc_use_generated_chemistry(ostc_ctx *ctx, int on) {
  if (!ctx) return OSTC_ERR_INVALID_ARG;
  if (on && !ctx->spec_ok) return OSTC_ERR_INVALID_ARG;
  ctx->spec_mech = on ? 1 : 0;
  for (auto &kv : ctx->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  ctx->graphs.clear();
  return OSTC_OK;
}

ostc_status ostc_set_chem_surrogate(ostc_ctx *ctx, ostc_surrogate *sur) {
  if (!ctx || !sur) return OSTC_ERR_INVALID_ARG;
  if (!ctx->has_source || ctx->ns != mlp::NIN - 3) return OSTC_ERR_INVALID_ARG;
  // everything a captured step needs is set up here, outside any capture
  CK(prepare_chem_surrogate());
  ChemScratch w;
  long long cells = 1;
  for (auto &z : ctx->dz) cells = std::max(cells, (long long)z.nsz);
  if (cells > 2147483647ll) return OSTC_ERR_INVALID_ARG;
  CK(surrogate_scratch(sur, (int)cells, &w));
  ctx->sur = sur;
  for (auto &kv : ctx->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  ctx->graphs.clear();
  return OSTC_OK;
}

ostc_status ostc_chem_stats(ostc_ctx *ctx, long long *states, long long *fallbacks, void *stream) {
  if (!ctx || !states || !fallbacks) return OSTC_ERR_INVALID_ARG;
  long long h[2] = {0, 0};
  if (ctx->chem_stats) {
    CK(cudaMemcpyAsync(h, ctx->chem_stats, sizeof(h), cudaMemcpyDeviceToHost, S(stream)));
    CK(cudaStreamSynchronize(S(stream)));
  }
  *states = h[0];
  *fallbacks = h[1];
  return OSTC_OK;
}

ostc_status ostc_chem_surrogate(ostc_ctx *ctx, ostc_surrogate *sur, int n, const double *T, const double *p,
                                const double *Y, const double *dt, double *dY, double *dT, int *n_fallback,
                                void *stream) {
  if (!ctx || !sur || n < 0 || (n > 0 && (!T || !p || !Y || !dt || !dY || !dT))) return OSTC_ERR_INVALID_ARG;
  if (!ctx->has_source || ctx->ns != mlp::NIN - 3) return OSTC_ERR_INVALID_ARG;
  if (ensure_param(ctx, S(stream))) return ctx->last;
  CK(prepare_chem_surrogate());
  ChemScratch w;
  CK(surrogate_scratch(sur, n > 0 ? n : 1, &w));
  CK(cudaMemsetAsync(w.err, 0, sizeof(int), S(stream)));
  CK(launch_chem_surrogate<mlp::NIN - 3>(*surrogate_net(sur), n, T, p, Y, dt, dY, dT, w, S(stream)));
  if (n_fallback) {
    int h[2] = {0, 0};
    CK(cudaMemcpyAsync(&h[0], w.count, sizeof(int), cudaMemcpyDeviceToHost, S(stream)));
    CK(cudaMemcpyAsync(&h[1], w.err, sizeof(int), cudaMemcpyDeviceToHost, S(stream)));
    CK(cudaStreamSynchronize(S(stream)));
    *n_fallback = h[0];
    if (h[1]) return fail(ctx, OSTC_ERR_TIMEOUT);
  }
  return OSTC_OK;
}

// one kernel family on every block, for per-kernel timing and the autotuner
ostc_status ostc_launch_op(ostc_ctx *ctx, int op, int arg, void *stream) {
  if (!ctx) return OSTC_ERR_INVALID_ARG;
  if (ensure_param(ctx, S(stream))) return ctx->last;
  const int inv = ctx->prm.inviscid_type;
  const int vis = ctx->prm.viscous_scheme != 0;
  switch (op) {
    case OSTC_OP_FLUX: {
      // arg 0..2: the direction's face flux; 3..5: its inviscid kernel alone; 6..8: its viscous kernel alone
      if (arg < 0 || arg > 8) return OSTC_ERR_INVALID_ARG;
      const int d = arg % 3, part = arg / 3;
      if (part == 2 && !vis) return OSTC_ERR_INVALID_ARG;
      if (ctx->batched) {
        CK(flux_launch(ctx, ctx->dz[0], d, ctx->flux_tab[d], 1, part, S(stream)));
        return OSTC_OK;
      }
      for (auto &z : ctx->dz)
        if (d < 2 || z.mz > 1) CK(flux_launch(ctx, z, d, nullptr, 1, part, S(stream)));  // 2-D: no z flux
      return OSTC_OK;
    }
    case OSTC_OP_SOURCE: {
      CellArgs src;
      src.spec = ctx->spec_mech;
      return cells_all(ctx, CellOp::Source, 0, src, S(stream));
    }
    case OSTC_OP_PROPERTIES: return ostc_update_physical_properties(ctx, stream);
    case OSTC_OP_UPDATE: return ostc_update_cv_and_bv_rk(ctx, ctx->cfg.fixed_time_step ? ctx->cfg.dt : -1, arg, stream);
    case OSTC_OP_DT: return ostc_global_time_step(ctx, nullptr, stream);
    case OSTC_OP_BC: return ostc_apply_boundary_conditions(ctx, arg, stream);
    default: return OSTC_ERR_INVALID_ARG;
  }
}

// kernel launches in one captured step: an RK3 step, or a steady iteration for
// a steady context (captures the graph if needed)
ostc_status ostc_step_kernel_count(ostc_ctx *ctx, int with_hist, int *count) {
  if (!ctx || !count) return OSTC_ERR_INVALID_ARG;
  ostc_status st;
  if (with_hist && (st = ensure_hist(ctx, 1))) return st;
  GraphEntry *ge = nullptr;
  if ((st = ensure_graph(ctx, with_hist != 0, &ge, ctx->cfg.steady != 0))) return st;
  size_t n = 0;
  CK(cudaGraphGetNodes(ge->graph, nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n);
  CK(cudaGraphGetNodes(ge->graph, nodes.data(), &n));
  int k = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    CK(cudaGraphNodeGetType(nd, &t));
    if (t == cudaGraphNodeTypeKernel) ++k;
  }
  *count = k;
  return OSTC_OK;
}

static void drop_graphs(ostc_ctx *ctx) {
  for (auto &kv : ctx->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  ctx->graphs.clear();
}

ostc_status ostc_set_monitor(ostc_ctx *ctx, int n_points, const int *block, const int *i, const int *j, const int *k,
                             int n_bv, const int *bv_label, int n_sv, const int *sv_label, int capacity) {
  if (!ctx || n_points < 0) return OSTC_ERR_INVALID_ARG;
  MonitorSet m;
  if (n_points > 0) {
    if (!block || !i || !j || !k || n_bv < 0 || n_sv < 0 || n_bv + n_sv < 1 || capacity < 1 ||
        (n_bv > 0 && !bv_label) || (n_sv > 0 && !sv_label))
      return OSTC_ERR_INVALID_ARG;
    std::vector<int4> pts(n_points);
    for (int p = 0; p < n_points; ++p) {
      if (block[p] < 0 || block[p] >= (int)ctx->dz.size()) return OSTC_ERR_INVALID_ARG;
      const DevZone &z = ctx->dz[block[p]];
      if (i[p] < 0 || i[p] >= z.mx || j[p] < 0 || j[p] >= z.my || k[p] < 0 || k[p] >= z.mz) return OSTC_ERR_INVALID_ARG;
      pts[p] = make_int4(block[p], i[p], j[p], k[p]);
    }
    std::vector<int> labels;
    for (int l = 0; l < n_bv; ++l) {
      if (bv_label[l] < 0 || bv_label[l] > 5) return OSTC_ERR_INVALID_ARG;
      labels.push_back(bv_label[l]);
    }
    for (int l = 0; l < n_sv; ++l) {
      if (sv_label[l] < 0 || sv_label[l] >= ctx->prm.n_scalar) return OSTC_ERR_INVALID_ARG;
      labels.push_back(sv_label[l]);
    }
    m.n = n_points, m.nbv = n_bv, m.nsv = n_sv, m.cap = capacity;
    const size_t nd = (size_t)n_points * capacity * (n_bv + n_sv + 1);
    CK(cudaMalloc(&m.pts, sizeof(int4) * n_points));
    CK(cudaMalloc(&m.labels, sizeof(int) * labels.size()));
    CK(cudaMalloc(&m.data, sizeof(double) * nd));
    CK(cudaMalloc(&m.counter, sizeof(int)));
    CK(cudaMemcpy(m.pts, pts.data(), sizeof(int4) * n_points, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(m.labels, labels.data(), sizeof(int) * labels.size(), cudaMemcpyHostToDevice));
    CK(cudaMemset(m.data, 0, sizeof(double) * nd));
    CK(cudaMemset(m.counter, 0, sizeof(int)));
    m.time = ctx->ep_time;
  }
  CK(cudaDeviceSynchronize());
  cudaFree(ctx->mon.pts);
  cudaFree(ctx->mon.labels);
  cudaFree(ctx->mon.data);
  cudaFree(ctx->mon.counter);
  ctx->mon = m;
  drop_graphs(ctx);
  return OSTC_OK;
}

ostc_status ostc_get_monitor(ostc_ctx *ctx, double *out, int *n_recorded) {
  if (!ctx || !n_recorded || (ctx->mon.n > 0 && !out)) return OSTC_ERR_INVALID_ARG;
  *n_recorded = 0;
  if (ctx->mon.n == 0) return OSTC_OK;
  CK(cudaDeviceSynchronize());
  int c = 0;
  CK(cudaMemcpy(&c, ctx->mon.counter, sizeof(int), cudaMemcpyDeviceToHost));
  const size_t nd = (size_t)ctx->mon.n * ctx->mon.cap * (ctx->mon.nbv + ctx->mon.nsv + 1);
  CK(cudaMemcpy(out, ctx->mon.data, sizeof(double) * nd, cudaMemcpyDeviceToHost));
  CK(cudaMemset(ctx->mon.counter, 0, sizeof(int)));  // Monitor::output_data restarts the ring
  *n_recorded = c < ctx->mon.cap ? c : ctx->mon.cap;
  return OSTC_OK;
}

ostc_status ostc_physical_time(ostc_ctx *ctx, double *time, int *step) {
  if (!ctx) return OSTC_ERR_INVALID_ARG;
  CK(cudaDeviceSynchronize());
  if (time) CK(cudaMemcpy(time, ctx->ep_time, sizeof(double), cudaMemcpyDeviceToHost));
  if (step) CK(cudaMemcpy(step, ctx->ep_step, sizeof(int), cudaMemcpyDeviceToHost));
  return OSTC_OK;
}

ostc_status ostc_set_physical_time(ostc_ctx *ctx, double time, int step) {
  if (!ctx || step < 0 || !(time >= 0)) return OSTC_ERR_INVALID_ARG;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(ctx->ep_time, &time, sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->ep_step, &step, sizeof(int), cudaMemcpyHostToDevice));
  return OSTC_OK;
}

ostc_status ostc_set_statistics(ostc_ctx *ctx, int on, int start_step) {
  if (!ctx || (on != 0 && on != 1) || start_step < 0) return OSTC_ERR_INVALID_ARG;
  CK(cudaDeviceSynchronize());
  for (auto &st : ctx->stats) {
    cudaFree(st.s12);
    cudaFree(st.count);
  }
  ctx->stats.clear();
  ctx->stat_on = 0;
  if (on) {
    const int ns = ctx->prm.n_spec;
    for (auto &z : ctx->dz) {
      StatSums st;
      const size_t n = (size_t)z.nsz, planes = 27 + ns;
      CK(cudaMalloc(&st.s12, sizeof(double) * planes * n));
      CK(cudaMemset(st.s12, 0, sizeof(double) * planes * n));
      CK(cudaMalloc(&st.count, sizeof(int)));
      CK(cudaMemset(st.count, 0, sizeof(int)));
      st.s34 = st.s12 + 12 * n;
      st.srs = st.s34 + 12 * n;
      st.syk = st.srs + 3 * n;
      ctx->stats.push_back(st);
    }
    // sums from the step after start_step (StatisticsCollector: step > start), and never for
    // steps taken before this call
    int cur = 0;
    CK(cudaMemcpy(&cur, ctx->ep_step, sizeof(int), cudaMemcpyDeviceToHost));
    ctx->stat_on = 1;
    ctx->stat_start = start_step > cur ? start_step : cur;
  }
  drop_graphs(ctx);
  return OSTC_OK;
}

ostc_status ostc_get_statistics(ostc_ctx *ctx, int block, double *sum12, double *sum34, double *sum_rs,
                                double *sum_yk, int *n_collected) {
  if (!ctx || !ctx->stat_on || block < 0 || block >= (int)ctx->dz.size()) return OSTC_ERR_INVALID_ARG;
  CK(cudaDeviceSynchronize());
  const size_t n = (size_t)ctx->dz[block].nsz;
  const StatSums &st = ctx->stats[block];
  if (sum12) CK(cudaMemcpy(sum12, st.s12, sizeof(double) * 12 * n, cudaMemcpyDeviceToHost));
  if (sum34) CK(cudaMemcpy(sum34, st.s34, sizeof(double) * 12 * n, cudaMemcpyDeviceToHost));
  if (sum_rs) CK(cudaMemcpy(sum_rs, st.srs, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
  if (sum_yk && ctx->prm.n_spec > 0)
    CK(cudaMemcpy(sum_yk, st.syk, sizeof(double) * ctx->prm.n_spec * n, cudaMemcpyDeviceToHost));
  if (n_collected) CK(cudaMemcpy(n_collected, st.count, sizeof(int), cudaMemcpyDeviceToHost));
  return OSTC_OK;
}

// ---------------------------------------------------------------------------
// restart / output files (FieldIO::print_field, read_flowfield)
// ---------------------------------------------------------------------------
static std::vector<std::string> species_list(const ostc_ctx *ctx, const char *const *names) {
  std::vector<std::string> v;
  for (int l = 0; l < ctx->prm.n_spec; ++l) v.emplace_back(names[l] ? names[l] : "");
  return v;
}

ostc_status ostc_write_flowfield(ostc_ctx *ctx, const char *path, const double *const *x, const double *const *y,
                                 const double *const *z, const char *const *species_names, int ngg_out,
                                 double solution_time) {
  if (!ctx || !path || !x || !y || !z || ngg_out < 0) return OSTC_ERR_INVALID_ARG;
  const int ns = ctx->prm.n_spec, nsc = ctx->prm.n_scalar;
  const bool sst = ctx->nt > 0;
  if (ns > 0 && !species_names) return OSTC_ERR_INVALID_ARG;
  const size_t nb = ctx->zones.size();
  for (size_t b = 0; b < nb; ++b)
    if (!x[b] || !y[b] || !z[b] || ngg_out > ctx->zones[b].ngg || !ctx->zones[b].mach) return OSTC_ERR_INVALID_ARG;
  CK(cudaDeviceSynchronize());
  std::vector<std::vector<double>> hbv(nb), hsv(nb), hmach(nb), hmut(nb);
  std::vector<ostc_io::PltBlock> blocks(nb);
  for (size_t b = 0; b < nb; ++b) {
    const ostc_zone &z0 = ctx->zones[b];
    const size_t sz = (size_t)(z0.mx + 2 * z0.ngg) * (z0.my + 2 * z0.ngg) * (z0.mz + 2 * z0.ngg);
    hbv[b].resize(6 * sz);
    hmach[b].resize(sz);
    CK(cudaMemcpy(hbv[b].data(), z0.bv, 6 * sz * sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(hmach[b].data(), z0.mach, sz * sizeof(double), cudaMemcpyDeviceToHost));
    if (nsc > 0) {
      hsv[b].resize(nsc * sz);
      CK(cudaMemcpy(hsv[b].data(), z0.sv, nsc * sz * sizeof(double), cudaMemcpyDeviceToHost));
    }
    if (sst) {
      hmut[b].resize(sz);
      CK(cudaMemcpy(hmut[b].data(), z0.mut, sz * sizeof(double), cudaMemcpyDeviceToHost));
    }
    ostc_io::PltBlock &B = blocks[b];
    B.mx = z0.mx, B.my = z0.my, B.mz = z0.mz, B.ngg = z0.ngg;
    B.x = x[b], B.y = y[b], B.z = z[b];
    B.bv = hbv[b].data(), B.mach = hmach[b].data();
    B.sv = nsc > 0 ? hsv[b].data() : nullptr;
    B.mut = sst ? hmut[b].data() : nullptr;
  }
  const int r = ostc_io::write_plt(path, blocks, species_list(ctx, species_names), sst, ngg_out, solution_time);
  return r == 0 ? OSTC_OK : fail(ctx, OSTC_ERR_IO);
}

ostc_status ostc_read_flowfield(ostc_ctx *ctx, const char *path, const char *const *species_names,
                                double *solution_time, int *found) {
  if (!ctx || !path) return OSTC_ERR_INVALID_ARG;
  const int ns = ctx->prm.n_spec, nsc = ctx->prm.n_scalar;
  if (ns > 0 && !species_names) return OSTC_ERR_INVALID_ARG;
  const size_t nb = ctx->zones.size();
  CK(cudaDeviceSynchronize());
  // the variables the file does not hold keep their values
  std::vector<std::vector<double>> hbv(nb), hsv(nb);
  std::vector<ostc_io::PltBlock> blocks(nb);
  for (size_t b = 0; b < nb; ++b) {
    const ostc_zone &z0 = ctx->zones[b];
    const size_t sz = (size_t)(z0.mx + 2 * z0.ngg) * (z0.my + 2 * z0.ngg) * (z0.mz + 2 * z0.ngg);
    hbv[b].resize(6 * sz);
    CK(cudaMemcpy(hbv[b].data(), z0.bv, 6 * sz * sizeof(double), cudaMemcpyDeviceToHost));
    if (nsc > 0) {
      hsv[b].resize(nsc * sz);
      CK(cudaMemcpy(hsv[b].data(), z0.sv, nsc * sz * sizeof(double), cudaMemcpyDeviceToHost));
    }
    ostc_io::PltBlock &B = blocks[b];
    B.mx = z0.mx, B.my = z0.my, B.mz = z0.mz, B.ngg = z0.ngg;
    B.bv_out = hbv[b].data();
    B.sv_out = nsc > 0 ? hsv[b].data() : nullptr;
  }
  const int r = ostc_io::read_plt(path, blocks, species_list(ctx, species_names), ctx->nt > 0, solution_time, found);
  if (r == 3) return fail(ctx, OSTC_ERR_INVALID_ARG);
  if (r != 0) return fail(ctx, OSTC_ERR_IO);
  for (size_t b = 0; b < nb; ++b) {
    const ostc_zone &z0 = ctx->zones[b];
    CK(cudaMemcpy(z0.bv, hbv[b].data(), hbv[b].size() * sizeof(double), cudaMemcpyHostToDevice));
    if (nsc > 0) CK(cudaMemcpy(z0.sv, hsv[b].data(), hsv[b].size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  return OSTC_OK;
}

// tile-shape control for the autotuner: dir 0..2
ostc_status ostc_set_tile(ostc_ctx *ctx, int dir, int rows, int chunks) {
  if (!ctx || dir < 0 || dir > 5) return OSTC_ERR_INVALID_ARG;
  // rows may carry the register budget and the staged kernels in its upper
  // bits: rows | (minb << 8) | (staged << 16), staged 1 = the staged kernels
  const int minb = (rows >> 8) & 0xff;
  const int staged = (rows >> 16) & 0xff;
  rows &= 0xff;
  TileShape &t = ctx->tile[dir % 3];
  if (dir > 2 && rows == 0) {  // back to the fused kernel
    t.vrows = 0;
  } else {
    if (chunks < 1 || chunks > 4096 || minb < 0 || minb > 5 || staged > 1) return OSTC_ERR_INVALID_ARG;
    // the staged kernels are built for 128 registers and CTAs of 8 rows
    if (staged && (minb > 2 || rows != 8)) return OSTC_ERR_INVALID_ARG;
    if (!(rows == 1 || rows == 2 || rows == 4 || rows == 8)) return OSTC_ERR_INVALID_ARG;
    if (minb >= 4 && rows > 4) return OSTC_ERR_INVALID_ARG;  // the 168- and 96-register builds take <= 128 threads
    if (dir > 2) {
      t.vrows = rows, t.vchunks = chunks, t.vminb = staged ? 2 : (minb < 1 ? 1 : minb), t.vstaged = staged;
    } else {
      t.rows = rows, t.chunks = chunks, t.minb = staged ? 2 : (minb < 1 ? 1 : minb), t.staged = staged;
    }
  }
  for (auto &kv : ctx->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  ctx->graphs.clear();
  if (ctx->batched || ctx->face_batched) return build_tables(ctx);
  return OSTC_OK;
}

ostc_status ostc_set_batching(ostc_ctx *ctx, int on) {
  if (!ctx || (on != 0 && on != 1)) return OSTC_ERR_INVALID_ARG;
  if (on && ctx->dz.size() > (size_t)kMaxTableZones) return OSTC_ERR_UNSUPPORTED;
  ctx->batched = on;
  ctx->face_batched = on;
  for (auto &kv : ctx->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  ctx->graphs.clear();
  g_uploaded = nullptr;  // the next launch uploads this context's zone table
  return on ? build_tables(ctx) : OSTC_OK;
}

ostc_status ostc_inject_wave_timeout(ostc_ctx *ctx, int on) {
  if (!ctx || (on != 0 && on != 1)) return OSTC_ERR_INVALID_ARG;
  if (!ctx->wave_sync) return OSTC_ERR_INVALID_ARG;  // no batched faces on this context
  CK(cudaDeviceSynchronize());
  for (int k = 0; k < 2; ++k) CK(cudaMemcpy(&ctx->wave_sync[k].hold, &on, sizeof(int), cudaMemcpyHostToDevice));
  return OSTC_OK;
}

ostc_status ostc_get_batching(const ostc_ctx *ctx, int *on) {
  if (!ctx || !on) return OSTC_ERR_INVALID_ARG;
  *on = ctx->batched;
  return OSTC_OK;
}

// the flux autotuner: device ms of one launch of flux op `arg` (0..8, as
// ostc_launch_op) at the current tiles, or a negative value when this tile
// setting cannot run for the scheme (a staged kernel for AWENO, a tile past a
// CTA's shared memory); CUDA events on the stream, after `warmup` launches
static float time_flux(ostc_ctx *ctx, int arg, int warmup, int reps, cudaStream_t s) {
  if (ostc_launch_op(ctx, OSTC_OP_FLUX, arg, s) != OSTC_OK) {
    cudaGetLastError();
    return -1.f;
  }
  for (int i = 0; i < warmup; ++i)
    if (ostc_launch_op(ctx, OSTC_OP_FLUX, arg, s) != OSTC_OK) return -1.f;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return -1.f;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return -1.f;
  }
  float ms = -1.f;
  bool ok = cudaEventRecord(e0, s) == cudaSuccess;
  for (int i = 0; ok && i < reps; ++i) ok = ostc_launch_op(ctx, OSTC_OP_FLUX, arg, s) == OSTC_OK;
  if (ok && cudaEventRecord(e1, s) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
      cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
    ms /= reps;
  else
    ms = -1.f;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms;
}

ostc_status ostc_autotune(ostc_ctx *ctx, int warmup, int reps, void *stream, float *ms_out) {
  if (!ctx || warmup < 0 || reps < 1) return OSTC_ERR_INVALID_ARG;
  cudaStream_t s = S(stream);
  if (ensure_param(ctx, s)) return ctx->last;
  const DevZone &z0 = ctx->dz[0];
  const int ext[3] = {z0.mx, z0.my, z0.mz};
  const bool viscous = ctx->prm.viscous_scheme != 0;
  const bool staged_ok = ctx->prm.reconstruction != 4;  // AWENO has no staged build
  struct Cand {
    int rows, chunks;
  };
  for (int d = 0; d < 3; ++d) {
    // tile candidates: rows x chunks (doubling up to the direction's extent)
    // x register budgets, and the staged kernels (8 rows, 128 registers)
    auto cands = [&](int min_budget) {
      std::vector<Cand> out;
      const int rows_list[3] = {2, 4, 8};
      for (int ri = d == 0 ? 0 : 1; ri < 3; ++ri) {
        const int R = rows_list[ri], span = d == 0 ? 32 : R;
        const int cmax = std::min(64, std::max(1, (ext[d] + 1 + span - 1) / span));
        for (int c = 1;; c *= 2) {
          const int cc = std::min(c, cmax);
          for (int b = min_budget; b <= 5; ++b) {
            if (b >= 4 && R > 4) continue;
            out.push_back({R | (b > 1 ? b << 8 : 0), cc});
          }
          if (staged_ok && R == 8) out.push_back({R | (2 << 8) | (1 << 16), cc});
          if (c >= cmax) break;
        }
      }
      return out;
    };
    if (ostc_set_tile(ctx, d + 3, 0, 0) != OSTC_OK) return ctx->last;
    float best = -1.f;
    Cand bf{}, bi{}, bv{};
    for (const Cand &c : cands(1)) {
      if (ostc_set_tile(ctx, d, c.rows, c.chunks) != OSTC_OK) continue;
      const float t = time_flux(ctx, d, warmup, reps, s);
      if (t >= 0 && (best < 0 || t < best)) best = t, bf = c;
    }
    if (best < 0) return fail(ctx, OSTC_ERR_CUDA);
    bool split = false;
    if (viscous) {
      // the separate inviscid and viscous kernels, each tuned on its own
      float ti = -1.f, tv = -1.f;
      for (const Cand &c : cands(2)) {
        if (ostc_set_tile(ctx, d, c.rows, c.chunks) != OSTC_OK) continue;
        const float a = time_flux(ctx, d + 3, warmup, reps, s);
        if (a >= 0 && (ti < 0 || a < ti)) ti = a, bi = c;
        if (ostc_set_tile(ctx, d + 3, c.rows, c.chunks) != OSTC_OK) continue;
        const float b = time_flux(ctx, d + 6, warmup, reps, s);
        if (b >= 0 && (tv < 0 || b < tv)) tv = b, bv = c;
      }
      if (ti >= 0 && tv >= 0 && ti + tv < best) best = ti + tv, split = true;
    }
    ostc_status st = split ? ostc_set_tile(ctx, d, bi.rows, bi.chunks) : ostc_set_tile(ctx, d, bf.rows, bf.chunks);
    if (st == OSTC_OK) st = split ? ostc_set_tile(ctx, d + 3, bv.rows, bv.chunks) : ostc_set_tile(ctx, d + 3, 0, 0);
    if (st != OSTC_OK) return st;
    if (ms_out) ms_out[d] = best;
  }
  return OSTC_OK;
}

ostc_status ostc_get_tile(const ostc_ctx *ctx, int dir, int *rows, int *chunks) {
  if (!ctx || dir < 0 || dir > 5 || !rows || !chunks) return OSTC_ERR_INVALID_ARG;
  const TileShape &t = ctx->tile[dir % 3];
  if (dir > 2) {
    *rows = t.vrows == 0 ? 0 : (t.vrows | (t.vminb > 1 ? (t.vminb << 8) : 0) | (t.vstaged << 16));
    *chunks = t.vrows == 0 ? 0 : t.vchunks;
    return OSTC_OK;
  }
  *rows = t.rows | (t.minb > 1 ? (t.minb << 8) : 0) | (t.staged << 16);
  *chunks = t.chunks;
  return OSTC_OK;
}

}  // extern "C"
