// flux.cuh — the per-direction flux kernel family flux_dir<NS,INV,DIR,MINB,PART>
// and its launchers. Included by one translation unit per species count or
// group of counts (flux0.cu, flux9.cu, flux0t.cu, flux9t.cu, flux_ns_*.cu) so
// the builds compile in parallel; each unit holds its own copy of the
// __constant__ parameters (uploaded by upload_param).
//
// Flux kernels march along the sweep direction: a CTA owns a segment of
// S = R*C - 1 cells of 32 (or R) lines, computes the R*C faces that bound
// them chunk by chunk, and carries the last face flux of each chunk into the
// next, so every face is evaluated once and dq is touched once per direction
// (InviscidScheme.cu, AWENO.cu, ViscousScheme.cuh).
#pragma once
#include "face.cuh"
#include "kernels.cuh"

namespace ostc {

// ---------------------------------------------------------------------------
// flux kernels
// ---------------------------------------------------------------------------
// PART 0: inviscid and (when `viscous`) viscous flux of the face;
// PART 1: the inviscid flux alone; PART 2: the viscous flux alone
// NT: turbulence scalars after the species (2 for SST; primitive-variable
// or AWENO reconstruction)
// Cells: the face's cell accessor (PlaneCells or TileCells, face.cuh); the
// AWENO and Roe faces read their cells from the planes
template <int NS, int INV, int DIR, int PART, int NT, class Cells>
__device__ __forceinline__ void face_total(const DevZone &z, const Cells &c, int g0, bool viscous, double *G) {
  constexpr int NV = 5 + NS + NT;
  static_assert(NT == 0 || INV != 2, "turbulence scalars: primitive-variable or AWENO reconstruction");
  if constexpr (PART == 2) {
    viscous_face<NS, DIR, NT>(c, G);
    return;
  }
  double Fi[NV];
  if constexpr (INV == 1)
    inviscid_face_aweno<DIR, NT>(z, g0, Fi);
  else if constexpr (INV == 2)
    inviscid_face_roe<NS, DIR>(z, g0, Fi);
  else
    inviscid_face_pv<NS, DIR, NT>(c, Fi);
  if (PART == 0 && viscous) {
    double Fv[NV];
    viscous_face<NS, DIR, NT>(c, Fv);
#pragma unroll
    for (int l = 0; l < NV; ++l) G[l] = Fv[l] - Fi[l];
  } else {
#pragma unroll
    for (int l = 0; l < NV; ++l) G[l] = -Fi[l];
  }
}

// register budget of a flux build: MINB 1..3 = that many resident CTAs of 256
// threads per SM (255, 128 or 80 registers); MINB 4 = three CTAs of at most
// 128 threads (168 registers, 12 warps per SM); MINB 5 = five CTAs of at most
// 128 threads (96 registers, 20 warps per SM)
template <int MINB>
struct FluxBounds {
  static constexpr int threads = MINB >= 4 ? 128 : 256;
  static constexpr int blocks = MINB == 4 ? 3 : MINB;
};

// PART selects the fused face flux or one of its halves (face_total); the
// viscous half (PART 2) does not depend on INV and is built for INV 0 only
// the work of one CTA: segment (bx, by, bz) of zone z
template <int NS, int INV, int DIR, int PART, int NT>
__device__ __forceinline__ void flux_tile(const DevZone &z, const int bx, const int by, const int bz, int nchunk,
                                          int accumulate, int viscous) {
  constexpr int NV = 5 + NS + NT;
  constexpr bool CDS = INV == 1 && PART != 2;  // AWENO's central correction belongs to the inviscid flux
  const int lane = threadIdx.x, row = threadIdx.y, R = blockDim.y;
  const int n = DIR == 0 ? z.mx : (DIR == 1 ? z.my : z.mz);
  const int cds_limit = n - 2 * z.ngg;  // quirk A4: no central correction on the last 2*ngg cells
  const bool vis = viscous != 0;
  if constexpr (DIR == 0) {
    const int S = 32 * nchunk - 1;
    const int c0 = bx * S;
    const int j = by * R + row, k = bz;
    const bool line_ok = j < z.my;
    // the last face flux of the previous chunk of each row (lane 31 -> lane 0)
    __shared__ double carry[8][NV];
    if (lane == 31)
#pragma unroll
      for (int l = 0; l < NV; ++l) carry[row][l] = 0;
    __syncwarp();
    for (int ch = 0; ch < nchunk; ++ch) {
      const int f = c0 - 1 + 32 * ch + lane;
      const bool active = line_ok && f <= n - 1;
      double G[NV];
      if (active) {
        const int g = gidx(z, f, j, k);
        face_total<NS, INV, DIR, PART, NT>(z, plane_cells<DIR>(z, g), g, vis, G);
      } else {
#pragma unroll
        for (int l = 0; l < NV; ++l) G[l] = 0;
      }
      double Gm[NV];
#pragma unroll
      for (int l = 0; l < NV; ++l) {
        const double up = __shfl_up_sync(0xffffffffu, G[l], 1);
        Gm[l] = lane == 0 ? carry[row][l] : up;
      }
      __syncwarp();
      if (lane == 31)
#pragma unroll
        for (int l = 0; l < NV; ++l) carry[row][l] = G[l];
      __syncwarp();
      if (active && f >= c0 && f >= 0) {
        double corr[5 + NT] = {};
        if constexpr (CDS) {
          if (f < cds_limit) cds_correction<DIR, NT>(z, gidx(z, f, j, k), corr);
        }
        double *dq = z.dq + qidx(z, f, j, k);
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          double d = G[l] - Gm[l];
          if (CDS && l < 5 + NT) d -= corr[l];
          if (accumulate)
            dq[l * z.iqsz] += d;
          else
            dq[l * z.iqsz] = d;
        }
      }
    }
  } else {
    extern __shared__ double sG[];  // [R+1][NV][32]
    const int S = R * nchunk - 1;
    const int i = bx * 32 + lane;
    const int c0 = (DIR == 1 ? by : bz) * S;
    const int j_fixed = by, k_fixed = bz;
    const bool col_ok = i < z.mx;
    for (int ch = 0; ch < nchunk; ++ch) {
      const int f = c0 - 1 + R * ch + row;
      const bool active = col_ok && f <= n - 1;
      const int ci = i, cj = DIR == 1 ? f : j_fixed, ck = DIR == 2 ? f : k_fixed;
      double G[NV];
      if (active) {
        const int g = gidx(z, ci, cj, ck);
        face_total<NS, INV, DIR, PART, NT>(z, plane_cells<DIR>(z, g), g, vis, G);
      } else {
#pragma unroll
        for (int l = 0; l < NV; ++l) G[l] = 0;
      }
#pragma unroll
      for (int l = 0; l < NV; ++l) sG[((row + 1) * NV + l) * 32 + lane] = G[l];
      __syncthreads();
      if (active && f >= c0 && f >= 0 && !(ch == 0 && row == 0)) {
        double corr[5 + NT] = {};
        if constexpr (CDS) {
          if (f < cds_limit) cds_correction<DIR, NT>(z, gidx(z, ci, cj, ck), corr);
        }
        double *dq = z.dq + qidx(z, ci, cj, ck);
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          double d = G[l] - sG[(row * NV + l) * 32 + lane];
          if (CDS && l < 5 + NT) d -= corr[l];
          if (accumulate)
            dq[l * z.iqsz] += d;
          else
            dq[l * z.iqsz] = d;
        }
      }
      __syncthreads();
      if (row == 0) {
#pragma unroll
        for (int l = 0; l < NV; ++l) sG[l * 32 + lane] = sG[(R * NV + l) * 32 + lane];
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// staged flux kernels: the cells of the CTA's sweep plane that its faces read
// (the chunk's faces plus the reconstruction halo along the sweep and one cell
// on each side along the in-plane tangential direction) are copied into a
// shared-memory tile with cp.async before the faces are computed; with two
// tile buffers the copy of the next chunk overlaps the faces of this one.
// The faces then read their in-plane stencil from the tile (TileCells) and only
// the cells across the plane, the metrics and the transport properties from
// HBM. Same arithmetic as the plane kernels, so the results are bit-identical.
//
// Tile of one chunk, per variable (bv 0..5, then sv 0..NS+NT-1), for CTAs of
// R = 8 rows:
//   x sweep: [R + 2 rows j0-1 .. j0+R][35 cells F-1 .. F+33 along i]
//   y / z sweep: [R + 3 rows F-1 .. F+R+1 along j / k][34 cells i0-1 .. i0+32]
// with F the chunk's first face (face f lies between cells f and f+1).
// ---------------------------------------------------------------------------
// Tile geometry of a staged CTA of SR = 8 rows of 32 threads (compile-time, so
// that every tile read is a shared-memory load at a constant offset and the
// copy loops divide by constants). A tile row holds W (state) or QW (cell)
// cells starting at column `shift` of a slot of WS / QWS doubles: slots are
// 16-byte multiples, so that a row copied in bulk from a 16-byte boundary of
// HBM (shift = 1 when the row's first cell is not on one) lands aligned.
constexpr int SR = 8;
template <int DIR>
struct StageGeom {
  static constexpr int W = DIR == 0 ? 35 : 34;           // state tile: cells per row
  static constexpr int WS = 36;                          // state tile: row slot
  static constexpr int TR = DIR == 0 ? SR + 2 : SR + 3;  // state tile: rows per variable
  static constexpr int TV = TR * WS;                     // state tile: stride of one variable
  static constexpr int QW = DIR == 0 ? 33 : 32;          // cell tile: cells per row
  static constexpr int QWS = 34;                         // cell tile: row slot
  static constexpr int QR = DIR == 0 ? SR : SR + 1;      // cell tile: rows per plane
  static constexpr int QV = QR * QWS;                    // cell tile: stride of one plane
  static_assert(W + 1 <= WS && QW + 1 <= QWS && WS % 2 == 0 && QWS % 2 == 0, "row slots hold a shifted row");
};

// planes of the cell tile: the metric and Jacobian, and for viscous faces the
// transport properties (with the SST planes when NT > 0)
template <int NS, int NT>
__host__ __device__ constexpr int stage_q_planes(bool viscous) {
  return viscous ? q_rhod<NT>() + NS : Q_JAC + 1;
}

// doubles of dynamic shared memory: state tile, cell tile and (y / z sweeps)
// the carried face flux; the y / z face-flux exchange reuses the state tile
template <int NS, int NT, int DIR>
__host__ __device__ constexpr size_t stage_smem_doubles(bool viscous) {
  return (size_t)(6 + NS + NT) * StageGeom<DIR>::TV + (size_t)stage_q_planes<NS, NT>(viscous) * StageGeom<DIR>::QV +
         (DIR == 0 ? 0 : (size_t)(5 + NS + NT) * 32);
}

__device__ __forceinline__ void stage_cp8(double *dst, const double *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void stage_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void stage_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// the CTA's tile mbarrier (bulk copies signal their bytes on it; one arrival
// per chunk by thread 0 after every copying thread has announced its bytes)
__device__ __forceinline__ void stage_bar_init(unsigned bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void stage_expect(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void stage_arrive(unsigned bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// one row: `bytes` (a multiple of 16) from a 16-byte-aligned global address to
// a 16-byte-aligned shared address, completion counted on the mbarrier
__device__ __forceinline__ void stage_bulk(double *dst, const double *src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
constexpr unsigned long long kStageWaitNs = 1000000000ull;  // 1 s of the global timer per tile wait
// bounded wait for the mbarrier phase `parity`; false when the time ran out
__device__ __forceinline__ bool stage_bar_wait(unsigned bar, unsigned parity) {
  unsigned long long t0;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t0));
  for (unsigned it = 0;; ++it) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 31) == 31) {
      unsigned long long t;
      asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
      if (t - t0 > kStageWaitNs) return false;
    }
  }
}

// set when a staged flux CTA gave up waiting for its tile (read and cleared
// by the unit's host accessor, stage_timeout_read)
static __device__ int g_stage_timeout;

// host side: this unit's timeout flag, cleared after the read
static cudaError_t stage_timeout_read(int *flag) {
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_stage_timeout, sizeof(int));
  if (e == cudaSuccess && v) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(g_stage_timeout, &zero, sizeof(int));
  }
  *flag = v;
  return e;
}

// base pointer of plane p of the cell tile (StagedPlanes order)
template <int NT>
__device__ __forceinline__ const double *stage_q_plane(const DevZone &z, int p) {
  if (p < Q_JAC) return z.met + p * z.isz;
  if (p == Q_JAC) return z.jac;
  if (p == Q_MUL) return z.mul;
  if (p == Q_KAPPA) return z.kappa;
  if (NT > 0 && p == Q_MUT) return z.mut;
  if (NT > 0 && p == Q_TTC) return z.ttc;
  if (NT > 0 && p == Q_WALL) return z.wall;
  return z.rhoD + (p - q_rhod<NT>()) * z.isz;
}

// copy one tile row of `w` cells starting at ghosted index gi of `plane` into
// its slot `dst` (the row's first cell at dst[shift]). Bulk: one thread copies
// `slot` cells from gi - shift, 16-byte aligned at both ends and inside the
// plane, else the row falls back to 8-byte cp.async by the same thread.
// Returns the bytes announced on the mbarrier.
__device__ __forceinline__ unsigned stage_row_bulk(const double *plane, int isz, int gi, int w, int slot, int shift,
                                                   double *dst, unsigned bar, int i0, int lo, int hi) {
  const int start = gi - shift;
  const double *src = plane + start;
  if (start >= 0 && start + slot <= isz && (reinterpret_cast<uintptr_t>(src) & 15) == 0 &&
      (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
    const unsigned bytes = (unsigned)slot * 8u;
    stage_expect(bar, bytes);
    stage_bulk(dst, src, bytes, bar);
    return bytes;
  }
  for (int c = 0; c < w; ++c)
    if (i0 + c >= lo && i0 + c < hi) stage_cp8(dst + shift + c, plane + gi + c);
  return 0;
}

// issue the copies of one chunk's tiles: the state tile (bv, sv of the chunk's
// cells with the reconstruction halo along the sweep and one cell on each side
// in-plane) and the cell tile (metric, Jacobian, properties of the faces' own
// cells). Rows outside the block's ghosted extent are not copied, nor (8-byte
// path) cells outside it: no face that is computed reads them. o1, o2: the
// CTA's fixed coordinates (x sweep: j0 = first row, k; y sweep: i0 = first
// column, k; z sweep: i0, j). Bulk path (zone flag kZoneBulk): thread t copies
// rows t, t + 256, ... of both tiles, one bulk copy each; 8-byte path: warp w
// copies rows w, w + 8, ..., one cp.async per cell and lane. sshift / qshift:
// the tile column of a state / cell row's first cell.
template <int NS, int NT, int DIR, bool BULK>
__device__ __forceinline__ void stage_issue(const DevZone &z, double *tile, double *qtile, int nq, int F, int o1,
                                            int o2, int sshift, int qshift, unsigned bar) {
  using G = StageGeom<DIR>;
  constexpr int NVAR = 6 + NS + NT, NT_S = NVAR * G::TR;
  const int lane = threadIdx.x;
  const int g = z.ngg;
  auto in_i = [&](int i) { return i >= -g && i < z.mx + g; };
  auto rows_ok = [&](int j, int k) { return j >= -g && j < z.my + g && k >= -g && k < z.mz + g; };
  // state row r of variable var: first cell x (F-1, j0-1+r, k); y (i0-1, F-1+r, k); z (i0-1, j, F-1+r)
  const int si0 = DIR == 0 ? F - 1 : o1 - 1;
  auto srow = [&](int rr, const double *&plane, int &gi) {
    const int var = rr / G::TR, r = rr - var * G::TR;
    const int j = DIR == 0 ? o1 - 1 + r : (DIR == 1 ? F - 1 + r : o2);
    const int k = DIR == 2 ? F - 1 + r : o2;
    if (!rows_ok(j, k)) return false;
    plane = var < 6 ? z.bv + var * z.isz : z.sv + (var - 6) * z.isz;
    gi = gidx(z, si0, j, k);
    return true;
  };
  // cell row r of plane p: first cell x (F, j0+r, k); y (i0, F+r, k); z (i0, j, F+r)
  const int qi0 = DIR == 0 ? F : o1;
  auto qrow = [&](int rr, const double *&plane, int &gi) {
    const int p = rr / G::QR, r = rr - p * G::QR;
    const int j = DIR == 0 ? o1 + r : (DIR == 1 ? F + r : o2);
    const int k = DIR == 2 ? F + r : o2;
    if (!rows_ok(j, k)) return false;
    plane = stage_q_plane<NT>(z, p);
    gi = gidx(z, qi0, j, k);
    return true;
  };
  if constexpr (BULK) {
    const int tid = threadIdx.y * 32 + lane;
    for (int rr = tid; rr < NT_S + nq * G::QR; rr += 32 * SR) {
      const double *plane;
      int gi;
      if (rr < NT_S) {
        if (srow(rr, plane, gi))
          stage_row_bulk(plane, z.isz, gi, G::W, G::WS, sshift, tile + rr * G::WS, bar, si0, -g, z.mx + g);
      } else {
        const int q = rr - NT_S;
        if (qrow(q, plane, gi))
          stage_row_bulk(plane, z.isz, gi, G::QW, G::QWS, qshift, qtile + q * G::QWS, bar, qi0, -g, z.mx + g);
      }
    }
  } else {
    const bool s0 = in_i(si0 + lane), s1 = lane + 32 < G::W && in_i(si0 + lane + 32);
#pragma unroll 2
    for (int rr = threadIdx.y; rr < NT_S; rr += SR) {
      const double *plane;
      int gi;
      if (!srow(rr, plane, gi)) continue;
      double *dst = tile + rr * G::WS + sshift;
      if (s0) stage_cp8(dst + lane, plane + gi + lane);
      if (s1) stage_cp8(dst + lane + 32, plane + gi + lane + 32);
    }
    const bool q0 = in_i(qi0 + lane), q1 = lane + 32 < G::QW && in_i(qi0 + lane + 32);
#pragma unroll 2
    for (int rr = threadIdx.y; rr < nq * G::QR; rr += SR) {
      const double *plane;
      int gi;
      if (!qrow(rr, plane, gi)) continue;
      double *dst = qtile + rr * G::QWS + qshift;
      if (q0) stage_cp8(dst + lane, plane + gi + lane);
      if (q1) stage_cp8(dst + lane + 32, plane + gi + lane + 32);
    }
  }
  stage_commit();
}

// one segment (bx, by, bz) of zone z; BULK: the tiles move as bulk copies (the
// zone has kZoneBulk), else as 8-byte cp.async; bar: the CTA's initialised tile
// mbarrier, phase: its current phase parity (advanced per bulk chunk). Returns
// false when a tile wait ran out (CTA-uniform; the kernel then stops).
template <int NS, int INV, int DIR, int PART, int NT, bool BULK>
__device__ __forceinline__ bool flux_tile_staged(const DevZone &z, const int bx, const int by, const int bz,
                                                 int nchunk, int accumulate, int viscous, double *smem, unsigned bar,
                                                 unsigned &phase) {
  using Geo = StageGeom<DIR>;
  constexpr int NV = 5 + NS + NT, NVAR = 6 + NS + NT, R = SR;
  static_assert(INV != 1, "AWENO reads its cells (and the central correction's) from the planes");
  const int lane = threadIdx.x, row = threadIdx.y;
  const int n = DIR == 0 ? z.mx : (DIR == 1 ? z.my : z.mz);
  const bool vis = viscous != 0;
  const int nq = stage_q_planes<NS, NT>(PART == 2 || (PART == 0 && vis));
  double *tile = smem;                                  // state tile; y / z: then the chunk's face fluxes
  double *qtile = smem + (size_t)NVAR * Geo::TV;        // cell tile
  double *cG = qtile + (size_t)nq * Geo::QV;            // y / z: [NV][32] last face flux of the previous chunk
  // segment geometry, as in flux_tile
  const int S = DIR == 0 ? 32 * nchunk - 1 : R * nchunk - 1;
  const int c0 = (DIR == 0 ? bx : (DIR == 1 ? by : bz)) * S;
  constexpr int span = DIR == 0 ? 32 : R;
  const int o1 = DIR == 0 ? by * R : bx * 32, o2 = DIR == 0 ? bz : (DIR == 1 ? bz : by);
  __shared__ double carry[R][NV];  // x sweep: the last face flux of the previous chunk of each row
  if (DIR == 0 && lane == 31)
#pragma unroll
    for (int l = 0; l < NV; ++l) carry[row][l] = 0;
  for (int ch = 0; ch < nchunk; ++ch) {
    const int F = c0 - 1 + span * ch;
    // tile columns of the rows' first cells: with bulk copies each row starts on
    // a 16-byte boundary, which (even row and plane lengths) the parity of the
    // first cell's index decides alike for every row of a tile
    const int si0 = DIR == 0 ? F - 1 : o1 - 1;
    const int sshift = BULK ? (si0 + z.dt_) & 1 : 0, qshift = BULK ? (si0 + 1 + z.dt_) & 1 : 0;
    stage_issue<NS, NT, DIR, BULK>(z, tile, qtile, nq, F, o1, o2, sshift, qshift, bar);
    stage_wait_all();
    if constexpr (BULK) {
      __syncthreads();  // every copying thread has announced its bytes
      if (threadIdx.x == 0 && threadIdx.y == 0) stage_arrive(bar);
      const bool late = !stage_bar_wait(bar, phase);
      if (__syncthreads_or(late)) {
        // give up: record it, let the copies in flight land (bounded) and stop
        if (threadIdx.x == 0 && threadIdx.y == 0) atomicExch(&g_stage_timeout, 1);
        stage_bar_wait(bar, phase);
        return false;
      }
      phase ^= 1u;
    } else {
      __syncthreads();
    }
    // this thread's face and cell
    const int f = F + (DIR == 0 ? lane : row);
    const int i = DIR == 0 ? f : bx * 32 + lane;
    const int j = DIR == 0 ? by * R + row : (DIR == 1 ? f : by);
    const int k = DIR == 2 ? f : bz;
    const bool active = (DIR == 0 ? j < z.my : i < z.mx) && f <= n - 1;
    double G[NV];
    if (active) {
      const int g = gidx(z, i, j, k);
      const TileCells<DIR == 0 ? 1 : Geo::WS, DIR == 0 ? Geo::WS : 1, Geo::TV, DIR == 0 ? 1 : Geo::QWS, Geo::QV,
                      q_rhod<NT>()>
          tc{plane_cells<DIR>(z, g), tile + (row + 1) * Geo::WS + lane + 1 + sshift,
             qtile + row * Geo::QWS + lane + qshift};
      face_total<NS, INV, DIR, PART, NT>(z, tc, g, vis, G);
    } else {
#pragma unroll
      for (int l = 0; l < NV; ++l) G[l] = 0;
    }
    if constexpr (DIR == 0) {
      double Gm[NV];
#pragma unroll
      for (int l = 0; l < NV; ++l) {
        const double up = __shfl_up_sync(0xffffffffu, G[l], 1);
        Gm[l] = lane == 0 ? carry[row][l] : up;
      }
      __syncwarp();
      if (lane == 31)
#pragma unroll
        for (int l = 0; l < NV; ++l) carry[row][l] = G[l];
      __syncwarp();
      if (active && f >= c0 && f >= 0) {
        double *dq = z.dq + qidx(z, i, j, k);
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          const double d = G[l] - Gm[l];
          if (accumulate)
            dq[l * z.iqsz] += d;
          else
            dq[l * z.iqsz] = d;
        }
      }
      // every face of the chunk has read the tiles (ordered before the next
      // chunk's asynchronous copies into them) before they are refilled
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
    } else {
      __syncthreads();  // every face has read the tiles: the state tile now takes the face fluxes
      double *sG = tile;  // [R][NV][32]
#pragma unroll
      for (int l = 0; l < NV; ++l) sG[(row * NV + l) * 32 + lane] = G[l];
      __syncthreads();
      if (active && f >= c0 && f >= 0 && !(ch == 0 && row == 0)) {
        double *dq = z.dq + qidx(z, i, j, k);
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          const double gm = row == 0 ? cG[l * 32 + lane] : sG[((row - 1) * NV + l) * 32 + lane];
          const double d = G[l] - gm;
          if (accumulate)
            dq[l * z.iqsz] += d;
          else
            dq[l * z.iqsz] = d;
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();  // the previous chunk's carried flux and the exchange are read
      if (row == R - 1)
#pragma unroll
        for (int l = 0; l < NV; ++l) cG[l * 32 + lane] = G[l];
    }
  }
  if constexpr (DIR != 0) __syncthreads();  // the carried flux of this tile is written before a next tile starts
  return true;
}

// the CTA's tile mbarrier, initialised once per launch
__device__ __forceinline__ unsigned stage_bar_setup(unsigned long long *bar_mem) {
  const unsigned bar = (unsigned)__cvta_generic_to_shared(bar_mem);
  if (threadIdx.x == 0 && threadIdx.y == 0) stage_bar_init(bar);
  __syncthreads();
  return bar;
}

// BULK: every zone the launch walks has kZoneBulk (the launcher checks)
template <int NS, int INV, int DIR, int MINB, int PART, int NT, bool BULK>
__global__ void __launch_bounds__(FluxBounds<MINB>::threads, FluxBounds<MINB>::blocks)
    flux_dir_staged(DevZone z, int nchunk, int accumulate, int viscous) {
  extern __shared__ __align__(16) double smem[];
  __shared__ unsigned long long bar_mem;
  const unsigned bar = stage_bar_setup(&bar_mem);
  unsigned phase = 0;
  flux_tile_staged<NS, INV, DIR, PART, NT, BULK>(z, blockIdx.x, blockIdx.y, blockIdx.z, nchunk, accumulate, viscous,
                                                 smem, bar, phase);
}

template <int NS, int INV, int DIR, int MINB, int PART, int NT, bool BULK>
__global__ void __launch_bounds__(FluxBounds<MINB>::threads, FluxBounds<MINB>::blocks)
    flux_dir_staged_table(const int4 *tiles, int n_tiles, int nchunk, int accumulate, int viscous) {
  extern __shared__ __align__(16) double smem[];
  __shared__ unsigned long long bar_mem;
  const unsigned bar = stage_bar_setup(&bar_mem);
  unsigned phase = 0;
  for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    const int4 c = tiles[t];
    if (!flux_tile_staged<NS, INV, DIR, PART, NT, BULK>(c_zones[c.x], c.y, c.z, c.w, nchunk, accumulate, viscous,
                                                        smem, bar, phase))
      return;
  }
}

template <int NS, int INV, int DIR, int MINB, int PART, int NT>
__global__ void __launch_bounds__(FluxBounds<MINB>::threads, FluxBounds<MINB>::blocks)
    flux_dir(DevZone z, int nchunk, int accumulate, int viscous) {
  flux_tile<NS, INV, DIR, PART, NT>(z, blockIdx.x, blockIdx.y, blockIdx.z, nchunk, accumulate, viscous);
}

// all zones of the context in one launch: a persistent grid walks the tile
// table of {zone, bx, by, bz} segments (zones in c_zones)
template <int NS, int INV, int DIR, int MINB, int PART, int NT>
__global__ void __launch_bounds__(FluxBounds<MINB>::threads, FluxBounds<MINB>::blocks)
    flux_dir_table(const int4 *tiles, int n_tiles, int nchunk, int accumulate, int viscous) {
  for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    const int4 c = tiles[t];
    flux_tile<NS, INV, DIR, PART, NT>(c_zones[c.x], c.y, c.z, c.w, nchunk, accumulate, viscous);
  }
}

// ---------------------------------------------------------------------------
// host-side launchers (kernels.cuh)
// ---------------------------------------------------------------------------
template <int NS, int INV, int DIR, int MINB, int PART, int NT>
static cudaError_t launch_flux_m(const DevZone &z, const TileShape &t, const FluxTable *tab, int accumulate,
                                 int viscous, cudaStream_t s) {
  constexpr int NV = 5 + NS + NT;
  const int R = t.rows, C = t.chunks;
  if (32 * R > FluxBounds<MINB>::threads) return cudaErrorInvalidConfiguration;
  const dim3 blk(32, R);
  const size_t smem = DIR == 0 ? 0 : sizeof(double) * (R + 1) * NV * 32;
  if (smem > 48 * 1024) {
    cudaError_t e = tab ? cudaFuncSetAttribute(flux_dir_table<NS, INV, DIR, MINB, PART, NT>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                        : cudaFuncSetAttribute(flux_dir<NS, INV, DIR, MINB, PART, NT>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  if (smem > 0) {
    // carve out only the shared memory of the CTAs the register budget lets an SM hold
    // (plus the 1 KB the driver reserves per CTA): the rest of the 256 KB stays L1, which
    // serves the stencil's re-reads (the default sizes the carveout for the shared-memory
    // limit alone)
    int per_sm = 0;
    cudaError_t e = tab ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                              &per_sm, flux_dir_table<NS, INV, DIR, MINB, PART, NT>, 32 * R, smem)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, flux_dir<NS, INV, DIR, MINB, PART, NT>,
                                                                        32 * R, smem);
    if (e != cudaSuccess) return e;
    const size_t need = (size_t)per_sm * (smem + 1024);
    int pct = (int)((need * 100 + 228 * 1024 - 1) / (228 * 1024));
    pct = pct < 1 ? 1 : (pct > 100 ? 100 : pct);
    e = tab ? cudaFuncSetAttribute(flux_dir_table<NS, INV, DIR, MINB, PART, NT>,
                                   cudaFuncAttributePreferredSharedMemoryCarveout, pct)
            : cudaFuncSetAttribute(flux_dir<NS, INV, DIR, MINB, PART, NT>,
                                   cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    if (e != cudaSuccess) return e;
  }
  if (!tab) {
    flux_dir<NS, INV, DIR, MINB, PART, NT><<<flux_grid(z.mx, z.my, z.mz, DIR, R, C), blk, smem, s>>>(z, C, accumulate,
                                                                                                 viscous);
    return cudaGetLastError();
  }
  if (tab->n <= 0) return cudaSuccess;
  // persistent grid: every resident CTA slot of the device, no more than there are tiles
  int per_sm = 0, dev = 0, sms = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, flux_dir_table<NS, INV, DIR, MINB, PART, NT>,
                                                                32 * R, smem);
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const int slots = per_sm * sms;
  if (slots <= 0) return cudaErrorInvalidConfiguration;
  const int grid = tab->n < slots ? tab->n : slots;
  flux_dir_table<NS, INV, DIR, MINB, PART, NT><<<grid, blk, smem, s>>>(tab->tiles, tab->n, C, accumulate, viscous);
  return cudaGetLastError();
}

// the staged kernels (CTAs of 8 rows, 128-register budget): dynamic shared
// memory = state tile + cell tile (+ the y / z sweep's carried face flux),
// checked against the 227 KB a CTA may use; the carveout is sized for the CTAs
// that fit
template <int NS, int INV, int DIR, int PART, int NT, bool BULK>
static cudaError_t launch_flux_sb(const DevZone &z, const TileShape &t, const FluxTable *tab, int accumulate,
                                  int viscous, cudaStream_t s) {
  constexpr int NV = 5 + NS + NT, MINB = 2, R = SR;
  const int C = t.chunks;
  if (t.rows != SR) return cudaErrorInvalidConfiguration;
  const bool vis_planes = PART == 2 || (PART == 0 && viscous);
  const size_t smem = sizeof(double) * stage_smem_doubles<NS, NT, DIR>(vis_planes);
  if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  const void *fn = tab ? (const void *)flux_dir_staged_table<NS, INV, DIR, MINB, PART, NT, BULK>
                       : (const void *)flux_dir_staged<NS, INV, DIR, MINB, PART, NT, BULK>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * R, smem);
  if (e != cudaSuccess) return e;
  if (per_sm <= 0) return cudaErrorInvalidConfiguration;
  {
    const size_t need = (size_t)per_sm * (smem + SR * NV * 8 + 1024);
    int pct = (int)((need * 100 + 228 * 1024 - 1) / (228 * 1024));
    pct = pct < 1 ? 1 : (pct > 100 ? 100 : pct);
    e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    if (e != cudaSuccess) return e;
  }
  const dim3 blk(32, R);
  if (!tab) {
    flux_dir_staged<NS, INV, DIR, MINB, PART, NT, BULK><<<flux_grid(z.mx, z.my, z.mz, DIR, R, C), blk, smem, s>>>(
        z, C, accumulate, viscous);
    return cudaGetLastError();
  }
  if (tab->n <= 0) return cudaSuccess;
  int dev = 0, sms = 0;
  e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const int slots = per_sm * sms;
  const int grid = tab->n < slots ? tab->n : slots;
  flux_dir_staged_table<NS, INV, DIR, MINB, PART, NT, BULK><<<grid, blk, smem, s>>>(tab->tiles, tab->n, C, accumulate,
                                                                              viscous);
  return cudaGetLastError();
}

// the bulk-copy build for zones with kZoneBulk, the 8-byte one for the others:
// a tile table holds the tiles of the bulk zones first (n_bulk), so it is
// walked by one launch of each build over its part (zones are independent)
template <int NS, int INV, int DIR, int PART, int NT>
static cudaError_t launch_flux_s(const DevZone &z, const TileShape &t, const FluxTable *tab, int accumulate,
                                 int viscous, cudaStream_t s) {
  if (!tab) {
    return (z.flags & kZoneBulk) ? launch_flux_sb<NS, INV, DIR, PART, NT, true>(z, t, nullptr, accumulate, viscous, s)
                                 : launch_flux_sb<NS, INV, DIR, PART, NT, false>(z, t, nullptr, accumulate, viscous, s);
  }
  const FluxTable tb{tab->tiles, tab->n_bulk, tab->n_bulk}, tc{tab->tiles + tab->n_bulk, tab->n - tab->n_bulk, 0};
  cudaError_t e = cudaSuccess;
  if (tb.n > 0) e = launch_flux_sb<NS, INV, DIR, PART, NT, true>(z, t, &tb, accumulate, viscous, s);
  if (e == cudaSuccess && tc.n > 0) e = launch_flux_sb<NS, INV, DIR, PART, NT, false>(z, t, &tc, accumulate, viscous, s);
  return e;
}

template <int NS, int INV, int DIR, int PART, int NT>
static cudaError_t launch_flux_p(const DevZone &z, const TileShape &t, const FluxTable *tab, int accumulate,
                                 int viscous, cudaStream_t s) {
  if (t.staged) {
    if constexpr (INV == 1) {
      return cudaErrorInvalidConfiguration;  // AWENO reads its cells from the planes
    } else {
      return launch_flux_s<NS, INV, DIR, PART, NT>(z, t, tab, accumulate, viscous, s);
    }
  }
#ifdef OSTC_FLUX_REDUCED
  // the units of further species counts build the 128-register budget only
  return launch_flux_m<NS, INV, DIR, 2, PART, NT>(z, t, tab, accumulate, viscous, s);
#else
  switch (t.minb) {
    case 5: return launch_flux_m<NS, INV, DIR, 5, PART, NT>(z, t, tab, accumulate, viscous, s);
    case 4: return launch_flux_m<NS, INV, DIR, 4, PART, NT>(z, t, tab, accumulate, viscous, s);
    case 3: return launch_flux_m<NS, INV, DIR, 3, PART, NT>(z, t, tab, accumulate, viscous, s);
    case 2: return launch_flux_m<NS, INV, DIR, 2, PART, NT>(z, t, tab, accumulate, viscous, s);
    default: return launch_flux_m<NS, INV, DIR, 1, PART, NT>(z, t, tab, accumulate, viscous, s);
  }
#endif
}

// part 0: the face flux of the flow — the fused kernel, or (viscous flow with
// a viscous tile set) the inviscid half followed by the viscous half, which
// accumulates; part 1: the inviscid half alone; part 2: the viscous half
// alone (tile t.vrows/vchunks/vminb, or t when no viscous tile is set).
// With tables (tab[0] for the shape t, tab[1] for the viscous shape) every
// zone of the context is processed by one launch per kernel.
template <int NS, int INV, int DIR, int NT>
static cudaError_t launch_flux_t(const DevZone &z, const TileShape &t, const FluxTable *tab, int accumulate,
                                 int viscous, int part, cudaStream_t s) {
  TileShape tv = t;
  if (t.vrows) {
    tv.rows = t.vrows, tv.chunks = t.vchunks, tv.minb = t.vminb, tv.staged = t.vstaged;
  }
  const FluxTable *tp = tab ? &tab[0] : nullptr;
  const FluxTable *tq = tab ? (t.vrows ? &tab[1] : &tab[0]) : nullptr;
  if (part == 1) return launch_flux_p<NS, INV, DIR, 1, NT>(z, t, tp, accumulate, 0, s);
  if (part == 2) return launch_flux_p<NS, 0, DIR, 2, NT>(z, tv, tq, accumulate, 1, s);
  if (!viscous || t.vrows == 0) return launch_flux_p<NS, INV, DIR, 0, NT>(z, t, tp, accumulate, viscous, s);
  cudaError_t e = launch_flux_p<NS, INV, DIR, 1, NT>(z, t, tp, accumulate, 0, s);
  if (e != cudaSuccess) return e;
  return launch_flux_p<NS, 0, DIR, 2, NT>(z, tv, tq, 1, 1, s);
}

template <int NS, int NT>
cudaError_t launch_flux_nt(const DevZone &z, int inv, int dir, const TileShape &t, const FluxTable *tab, int accumulate,
                           int viscous, int part, cudaStream_t s) {
  if constexpr (NT > 0) {
    if constexpr (NS == 0) {
      if (inv == 1) {  // AWENO (air) with the scalars reconstructed component-wise
        switch (dir) {
          case 0: return launch_flux_t<NS, 1, 0, NT>(z, t, tab, accumulate, viscous, part, s);
          case 1: return launch_flux_t<NS, 1, 1, NT>(z, t, tab, accumulate, viscous, part, s);
          default: return launch_flux_t<NS, 1, 2, NT>(z, t, tab, accumulate, viscous, part, s);
        }
      }
    }
    if (inv != 0) return cudaErrorInvalidValue;  // no Roe with turbulence scalars
    switch (dir) {
      case 0: return launch_flux_t<NS, 0, 0, NT>(z, t, tab, accumulate, viscous, part, s);
      case 1: return launch_flux_t<NS, 0, 1, NT>(z, t, tab, accumulate, viscous, part, s);
      default: return launch_flux_t<NS, 0, 2, NT>(z, t, tab, accumulate, viscous, part, s);
    }
  } else {
    if constexpr (NS == 0) {
      if (inv == 1) {
        switch (dir) {
          case 0: return launch_flux_t<0, 1, 0, 0>(z, t, tab, accumulate, viscous, part, s);
          case 1: return launch_flux_t<0, 1, 1, 0>(z, t, tab, accumulate, viscous, part, s);
          default: return launch_flux_t<0, 1, 2, 0>(z, t, tab, accumulate, viscous, part, s);
        }
      }
    }
    if (inv == 2) {
      switch (dir) {
        case 0: return launch_flux_t<NS, 2, 0, 0>(z, t, tab, accumulate, viscous, part, s);
        case 1: return launch_flux_t<NS, 2, 1, 0>(z, t, tab, accumulate, viscous, part, s);
        default: return launch_flux_t<NS, 2, 2, 0>(z, t, tab, accumulate, viscous, part, s);
      }
    }
    switch (dir) {
      case 0: return launch_flux_t<NS, 0, 0, 0>(z, t, tab, accumulate, viscous, part, s);
      case 1: return launch_flux_t<NS, 0, 1, 0>(z, t, tab, accumulate, viscous, part, s);
      default: return launch_flux_t<NS, 0, 2, 0>(z, t, tab, accumulate, viscous, part, s);
    }
  }
}

}  // namespace ostc
