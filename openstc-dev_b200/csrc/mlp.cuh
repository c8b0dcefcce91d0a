// mlp.cuh — shapes and device parameters of the chemistry surrogate network
// (12-256-256-256-10 perceptron, SiLU), shared by the training kernels
// (mlp.cu) and the fused inference kernel (surrogate.cuh).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/ostc.h"

struct ostc_surrogate;

namespace ostc {
namespace mlp {

constexpr int NIN = 12;    // features: log T, log p, 9 transformed Y_k, log dt
constexpr int KIN = 16;    // the first layer's K, padded to one MMA K-step
constexpr int NH = 256;    // hidden width
constexpr int NOUT = 10;   // dY_k (9) and dT, standardised
constexpr int NOUTP = 16;  // the last layer's N, padded

// flat padded parameter layout: W1[256][16] b1[256] W2[256][256] b2 W3 b3 W4[16][256] b4[16]
constexpr long long OFF_W1 = 0, OFF_B1 = OFF_W1 + (long long)NH * KIN, OFF_W2 = OFF_B1 + NH,
                    OFF_B2 = OFF_W2 + (long long)NH * NH, OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + (long long)NH * NH,
                    OFF_W4 = OFF_B3 + NH, OFF_B4 = OFF_W4 + (long long)NOUTP * NH, NPAR = OFF_B4 + NOUTP;

// feature / target scaling (doubles): means, standard deviations, the
// training envelope (min / max of the raw features) and the target
// transform: with r0 > 0 the network learns z = asinh(rate / r0), so small
// rates keep relative precision and large ones are compressed
// logarithmically; rate = r0 sinh(mean + std * y)
enum {
  SC_IN_MEAN = 0,
  SC_IN_STD = SC_IN_MEAN + NIN,
  SC_IN_MIN = SC_IN_STD + NIN,
  SC_IN_MAX = SC_IN_MIN + NIN,
  SC_OUT_MEAN = SC_IN_MAX + NIN,
  SC_OUT_STD = SC_OUT_MEAN + NOUT,
  SC_OUT_R0 = SC_OUT_STD + NOUT,  // > 0: the target is asinh(rate / r0)
  SCALE_COUNT = SC_OUT_R0 + NOUT
};

// acceptance tests of a surrogate increment (device copy in the surrogate)
struct Checks {
  int n_elem = 0;
  double a[4][OSTC_MAX_SPEC] = {};  // element counts per species
  double m[4] = {};                 // element atomic masses (kg/kmol)
  double tol_el = 1e-4;             // largest element mass fraction imbalance
  double tol_T = 1.0;               // largest implied temperature error (K)
};

struct Net {
  const Checks *checks = nullptr;  // device
  __nv_bfloat16 *wb = nullptr;  // BF16 copy of every parameter (padded layout)
  float *wf = nullptr;          // FP32 master parameters (padded layout; biases are read from here)
  double *scale = nullptr;      // SCALE_COUNT doubles
  int withhold_commit = 0;      // diagnostic (ostc_surrogate_inject_timeout): tensor-core waits run out
  __device__ __host__ const __nv_bfloat16 *w1() const { return wb + OFF_W1; }
  __device__ __host__ const __nv_bfloat16 *w2() const { return wb + OFF_W2; }
  __device__ __host__ const __nv_bfloat16 *w3() const { return wb + OFF_W3; }
  __device__ __host__ const __nv_bfloat16 *w4() const { return wb + OFF_W4; }
  __device__ __host__ const float *b1() const { return wf + OFF_B1; }
  __device__ __host__ const float *b2() const { return wf + OFF_B2; }
  __device__ __host__ const float *b3() const { return wf + OFF_B3; }
  __device__ __host__ const float *b4() const { return wf + OFF_B4; }
};

}  // namespace mlp

// the device parameters of a surrogate (mlp.cu), for the inference path
const mlp::Net *surrogate_net(const ostc_surrogate *s);
// per-call scratch of the surrogate chemistry step, for at least n states
// (grown on demand): the fallback list and its counter, the error word, the
// standardised BF16 feature rows [n][16], the network's outputs [n][10] and
// the training-envelope flags [n]
struct ChemScratch {
  int *list = nullptr, *count = nullptr, *err = nullptr;
  __nv_bfloat16 *x = nullptr;
  float *y = nullptr;
  unsigned char *env = nullptr;
};
cudaError_t surrogate_scratch(ostc_surrogate *s, int n, ChemScratch *out);

}  // namespace ostc
