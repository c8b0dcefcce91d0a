// kernels_ns_d.cu — the per-cell, boundary, interface, steady and chemistry
// kernels of kernels.cu built for mechanisms of 16, 17, 18, 19, 20 species, so that
// any mechanism up to OSTC_MAX_SPEC runs with its species count as a
// compile-time constant (per-species arrays in registers).
#define OSTC_NS_UNIT ns_d
#define OSTC_NS_LIST(X) X(16) X(17) X(18) X(19) X(20)
#include "kernels.cu"
