// flux_ns_b.cu — the flux kernel family (flux.cuh) for mechanisms of
// 6, 7, 8, 10 species, in its 128-register budget only (the
// 9-species unit flux9.cu carries every budget the autotuner chooses from).
#include "common.cuh"

namespace ostc {
// this unit's copy of the run parameters (written by upload_param) and of
// the zone table of tile-table launches (written by upload_zones)
static __constant__ DevParam c_p;
}  // namespace ostc

#include "kernels.cuh"

namespace ostc {
static __constant__ DevZone c_zones[kMaxTableZones];
}  // namespace ostc

#define OSTC_FLUX_REDUCED
#include "flux.cuh"

namespace ostc {

template cudaError_t launch_flux_nt<6, 0>(const DevZone &, int, int, const TileShape &, const FluxTable *, int,
                                           int, int, cudaStream_t);
template cudaError_t launch_flux_nt<7, 0>(const DevZone &, int, int, const TileShape &, const FluxTable *, int,
                                           int, int, cudaStream_t);
template cudaError_t launch_flux_nt<8, 0>(const DevZone &, int, int, const TileShape &, const FluxTable *, int,
                                           int, int, cudaStream_t);
template cudaError_t launch_flux_nt<10, 0>(const DevZone &, int, int, const TileShape &, const FluxTable *, int,
                                           int, int, cudaStream_t);

cudaError_t upload_param_flux_ns_b(const DevParam &p, cudaStream_t s) {
  return cudaMemcpyToSymbolAsync(c_p, &p, sizeof(DevParam), 0, cudaMemcpyHostToDevice, s);
}

// this unit's staged-kernel timeout flag (read and cleared)
cudaError_t stage_timeout_flux_ns_b(int *flag) { return stage_timeout_read(flag); }

cudaError_t upload_zones_flux_ns_b(const DevZone *z, int n, cudaStream_t s) {
  if (n < 0 || n > kMaxTableZones) return cudaErrorInvalidValue;
  return n ? cudaMemcpyToSymbolAsync(c_zones, z, sizeof(DevZone) * n, 0, cudaMemcpyHostToDevice, s) : cudaSuccess;
}

}  // namespace ostc
