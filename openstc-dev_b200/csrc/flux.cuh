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
    viscous_face<NS, DIR, NT>(z, c, g0, G);
    return;
  }
  double Fi[NV];
  if constexpr (INV == 1)
    inviscid_face_aweno<DIR, NT>(z, g0, Fi);
  else if constexpr (INV == 2)
    inviscid_face_roe<NS, DIR>(z, g0, Fi);
  else
    inviscid_face_pv<NS, DIR, NT>(z, c, g0, Fi);
  if (PART == 0 && viscous) {
    double Fv[NV];
    viscous_face<NS, DIR, NT>(z, c, g0, Fv);
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
// Tile of one chunk, per variable (bv 0..5, then sv 0..NS+NT-1):
//   x sweep: [R + 2 rows j0-1 .. j0+R][35 cells F-1 .. F+33 along i]
//   y / z sweep: [R + 3 rows F-1 .. F+R+1 along j / k][34 cells i0-1 .. i0+32]
// with F the chunk's first face (face f lies between cells f and f+1).
// ---------------------------------------------------------------------------
template <int DIR>
struct StageGeom {
  static constexpr int W = DIR == 0 ? 35 : 34;
  __host__ __device__ static constexpr int rows(int R) { return DIR == 0 ? R + 2 : R + 3; }
};

template <int NS, int NT, int DIR>
__host__ __device__ constexpr size_t stage_tile_doubles(int R) {
  return (size_t)(6 + NS + NT) * StageGeom<DIR>::rows(R) * StageGeom<DIR>::W;
}

__device__ __forceinline__ void stage_cp8(double *dst, const double *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void stage_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void stage_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// issue the copies of one chunk's tile: warp w copies tile rows w, w + R, ...
// o1, o2: the CTA's fixed coordinates (x sweep: j0 = first row, k; y sweep:
// i0 = first column, k; z sweep: i0, j)
// (one row = W consecutive cells of one variable); cells outside the block's
// ghosted extent are not copied (no face that is computed reads them)
template <int NS, int NT, int DIR>
__device__ __forceinline__ void stage_issue(const DevZone &z, double *tile, int F, int o1, int o2) {
  constexpr int NVAR = 6 + NS + NT, W = StageGeom<DIR>::W;
  const int R = blockDim.y, TR = StageGeom<DIR>::rows(R);
  const int lane = threadIdx.x;
  const int g = z.ngg;
  for (int rr = threadIdx.y; rr < NVAR * TR; rr += R) {
    const int var = rr / TR, r = rr - var * TR;
    // first cell of the tile row: x sweep (F-1, j0-1+r, k); y (i0-1, F-1+r, k); z (i0-1, j, F-1+r)
    const int i0 = DIR == 0 ? F - 1 : o1 - 1;
    const int j = DIR == 0 ? o1 - 1 + r : (DIR == 1 ? F - 1 + r : o2);
    const int k = DIR == 2 ? F - 1 + r : o2;
    if (j < -g || j >= z.my + g || k < -g || k >= z.mz + g) continue;
    const double *src = (var < 6 ? z.bv + var * z.isz : z.sv + (var - 6) * z.isz) + gidx(z, i0, j, k);
    double *dst = tile + rr * W;
    for (int c = lane; c < W; c += 32) {
      const int i = i0 + c;
      if (i >= -g && i < z.mx + g) stage_cp8(dst + c, src + c);
    }
  }
  stage_commit();
}

template <int NS, int INV, int DIR, int PART, int NT>
__device__ __forceinline__ void flux_tile_staged(const DevZone &z, const int bx, const int by, const int bz,
                                                 int nchunk, int accumulate, int viscous, int nbuf, double *smem) {
  constexpr int NV = 5 + NS + NT;
  constexpr int W = StageGeom<DIR>::W;
  static_assert(INV != 1, "AWENO reads its cells (and the central correction's) from the planes");
  const int lane = threadIdx.x, row = threadIdx.y, R = blockDim.y;
  const int n = DIR == 0 ? z.mx : (DIR == 1 ? z.my : z.mz);
  const int TR = StageGeom<DIR>::rows(R);
  const int tv = TR * W;                          // tile stride of one variable
  const size_t tsz = stage_tile_doubles<NS, NT, DIR>(R);
  const bool vis = viscous != 0;
  // segment geometry, as in flux_tile
  const int S = DIR == 0 ? 32 * nchunk - 1 : R * nchunk - 1;
  const int c0 = (DIR == 0 ? bx : (DIR == 1 ? by : bz)) * S;
  const int span = DIR == 0 ? 32 : R;
  // tile origin arguments of stage_issue: x (j0, k); y (i0, k); z (i0, j)
  const int o1 = DIR == 0 ? by * R : bx * 32, o2 = DIR == 0 ? bz : (DIR == 1 ? bz : by);
  __shared__ double carry[8][NV];  // x sweep: the last face flux of the previous chunk of each row
  double *sG = smem + (size_t)nbuf * tsz;  // y / z sweep: [R+1][NV][32] face fluxes of the chunk
  if (DIR == 0 && lane == 31)
#pragma unroll
    for (int l = 0; l < NV; ++l) carry[row][l] = 0;
  if (nbuf == 2) stage_issue<NS, NT, DIR>(z, smem, c0 - 1, o1, o2);
  for (int ch = 0; ch < nchunk; ++ch) {
    const int F = c0 - 1 + span * ch;
    double *tile = smem + (nbuf == 2 ? (size_t)(ch & 1) * tsz : 0);
    if (nbuf == 2) {
      if (ch + 1 < nchunk) {
        stage_issue<NS, NT, DIR>(z, smem + (size_t)((ch + 1) & 1) * tsz, F + span, o1, o2);
        stage_wait<1>();
      } else {
        stage_wait<0>();
      }
    } else {
      stage_issue<NS, NT, DIR>(z, tile, F, o1, o2);
      stage_wait<0>();
    }
    __syncthreads();
    // this thread's face and cell
    const int f = F + (DIR == 0 ? lane : row);
    const int i = DIR == 0 ? f : bx * 32 + lane;
    const int j = DIR == 0 ? by * R + row : (DIR == 1 ? f : by);
    const int k = DIR == 2 ? f : bz;
    const bool active = (DIR == 0 ? j < z.my : i < z.mx) && f <= n - 1;
    double G[NV];
    if (active) {
      const int g = gidx(z, i, j, k);
      const TileCells tc{plane_cells<DIR>(z, g), tile + (row + 1) * W + lane + 1, DIR == 0 ? 1 : W, DIR == 0 ? W : 1,
                         tv};
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
      __syncthreads();  // every face of the chunk has read the tile before it is refilled
    } else {
#pragma unroll
      for (int l = 0; l < NV; ++l) sG[((row + 1) * NV + l) * 32 + lane] = G[l];
      __syncthreads();
      if (active && f >= c0 && f >= 0 && !(ch == 0 && row == 0)) {
        double *dq = z.dq + qidx(z, i, j, k);
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          const double d = G[l] - sG[(row * NV + l) * 32 + lane];
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

template <int NS, int INV, int DIR, int MINB, int PART, int NT>
__global__ void __launch_bounds__(FluxBounds<MINB>::threads, FluxBounds<MINB>::blocks)
    flux_dir_staged(DevZone z, int nchunk, int accumulate, int viscous, int nbuf) {
  extern __shared__ double smem[];
  flux_tile_staged<NS, INV, DIR, PART, NT>(z, blockIdx.x, blockIdx.y, blockIdx.z, nchunk, accumulate, viscous, nbuf,
                                           smem);
}

template <int NS, int INV, int DIR, int MINB, int PART, int NT>
__global__ void __launch_bounds__(FluxBounds<MINB>::threads, FluxBounds<MINB>::blocks)
    flux_dir_staged_table(const int4 *tiles, int n_tiles, int nchunk, int accumulate, int viscous, int nbuf) {
  extern __shared__ double smem[];
  for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    const int4 c = tiles[t];
    flux_tile_staged<NS, INV, DIR, PART, NT>(c_zones[c.x], c.y, c.z, c.w, nchunk, accumulate, viscous, nbuf, smem);
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

// the staged kernels (128-register budget): dynamic shared memory = nbuf
// tiles (+ the y / z sweep's face-flux exchange), checked against the 227 KB a
// CTA may use; the carveout is sized for the CTAs that fit
template <int NS, int INV, int DIR, int PART, int NT>
static cudaError_t launch_flux_s(const DevZone &z, const TileShape &t, int nbuf, const FluxTable *tab,
                                 int accumulate, int viscous, cudaStream_t s) {
  constexpr int NV = 5 + NS + NT, MINB = 2;
  const int R = t.rows, C = t.chunks;
  if (32 * R > FluxBounds<MINB>::threads || R > 8 || (nbuf != 1 && nbuf != 2)) return cudaErrorInvalidConfiguration;
  const size_t smem = sizeof(double) * ((size_t)nbuf * stage_tile_doubles<NS, NT, DIR>(R) +
                                        (DIR == 0 ? 0 : (size_t)(R + 1) * NV * 32));
  if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  const void *fn = tab ? (const void *)flux_dir_staged_table<NS, INV, DIR, MINB, PART, NT>
                       : (const void *)flux_dir_staged<NS, INV, DIR, MINB, PART, NT>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * R, smem);
  if (e != cudaSuccess) return e;
  if (per_sm <= 0) return cudaErrorInvalidConfiguration;
  {
    const size_t need = (size_t)per_sm * (smem + 8 * NV * 8 + 1024);
    int pct = (int)((need * 100 + 228 * 1024 - 1) / (228 * 1024));
    pct = pct < 1 ? 1 : (pct > 100 ? 100 : pct);
    e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    if (e != cudaSuccess) return e;
  }
  const dim3 blk(32, R);
  if (!tab) {
    flux_dir_staged<NS, INV, DIR, MINB, PART, NT><<<flux_grid(z.mx, z.my, z.mz, DIR, R, C), blk, smem, s>>>(
        z, C, accumulate, viscous, nbuf);
    return cudaGetLastError();
  }
  if (tab->n <= 0) return cudaSuccess;
  int dev = 0, sms = 0;
  e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const int slots = per_sm * sms;
  const int grid = tab->n < slots ? tab->n : slots;
  flux_dir_staged_table<NS, INV, DIR, MINB, PART, NT><<<grid, blk, smem, s>>>(tab->tiles, tab->n, C, accumulate,
                                                                              viscous, nbuf);
  return cudaGetLastError();
}

template <int NS, int INV, int DIR, int PART, int NT>
static cudaError_t launch_flux_p(const DevZone &z, const TileShape &t, const FluxTable *tab, int accumulate,
                                 int viscous, cudaStream_t s) {
  if (t.staged) {
    if constexpr (INV == 1) {
      return cudaErrorInvalidConfiguration;  // AWENO reads its cells from the planes
    } else {
      return launch_flux_s<NS, INV, DIR, PART, NT>(z, t, t.staged, tab, accumulate, viscous, s);
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
