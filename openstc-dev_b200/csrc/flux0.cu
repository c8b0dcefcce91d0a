// flux0.cu — the flux kernel family (flux.cuh) built for NS = 0 species.
#include "common.cuh"

namespace ostc {
// this unit's copy of the run parameters (written by upload_param)
static __constant__ DevParam c_p;
}  // namespace ostc

#include "flux.cuh"

namespace ostc {

template cudaError_t launch_flux<0>(const DevZone &, int, int, const TileShape &, int, int, int, cudaStream_t);

cudaError_t upload_param_flux0(const DevParam &p, cudaStream_t s) {
  return cudaMemcpyToSymbolAsync(c_p, &p, sizeof(DevParam), 0, cudaMemcpyHostToDevice, s);
}

}  // namespace ostc
