// flux0t.cu — the flux kernel family (flux.cuh) built for air with the two SST scalars (k, omega).
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

#include "flux.cuh"

namespace ostc {

template cudaError_t launch_flux_nt<0, 2>(const DevZone &, int, int, const TileShape &, const FluxTable *, int,
                                            int, int, cudaStream_t);

cudaError_t upload_param_flux0t(const DevParam &p, cudaStream_t s) {
  return cudaMemcpyToSymbolAsync(c_p, &p, sizeof(DevParam), 0, cudaMemcpyHostToDevice, s);
}

// this unit's staged-kernel timeout flag (read and cleared)
cudaError_t stage_timeout_flux0t(int *flag) { return stage_timeout_read(flag); }

cudaError_t upload_zones_flux0t(const DevZone *z, int n, cudaStream_t s) {
  if (n < 0 || n > kMaxTableZones) return cudaErrorInvalidValue;
  return n ? cudaMemcpyToSymbolAsync(c_zones, z, sizeof(DevZone) * n, 0, cudaMemcpyHostToDevice, s) : cudaSuccess;
}

}  // namespace ostc
