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
template <int NS, int INV, int DIR, int PART, int NT>
__device__ __forceinline__ void face_total(const DevZone &z, int g0, bool viscous, double *G) {
  constexpr int NV = 5 + NS + NT;
  static_assert(NT == 0 || INV != 2, "turbulence scalars: primitive-variable or AWENO reconstruction");
  if constexpr (PART == 2) {
    viscous_face<NS, DIR, NT>(z, g0, G);
    return;
  }
  double Fi[NV];
  if constexpr (INV == 1)
    inviscid_face_aweno<DIR, NT>(z, g0, Fi);
  else if constexpr (INV == 2)
    inviscid_face_roe<NS, DIR>(z, g0, Fi);
  else
    inviscid_face_pv<NS, DIR, NT>(z, g0, Fi);
  if (PART == 0 && viscous) {
    double Fv[NV];
    viscous_face<NS, DIR, NT>(z, g0, Fv);
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
        face_total<NS, INV, DIR, PART, NT>(z, gidx(z, f, j, k), vis, G);
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
        face_total<NS, INV, DIR, PART, NT>(z, gidx(z, ci, cj, ck), vis, G);
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

template <int NS, int INV, int DIR, int PART, int NT>
static cudaError_t launch_flux_p(const DevZone &z, const TileShape &t, const FluxTable *tab, int accumulate,
                                 int viscous, cudaStream_t s) {
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
  const TileShape tv = t.vrows ? TileShape{t.vrows, t.vchunks, t.vminb} : TileShape{t.rows, t.chunks, t.minb};
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
