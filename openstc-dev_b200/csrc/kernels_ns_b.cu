// kernels_ns_b.cu — the per-cell, boundary, interface, steady and chemistry
// kernels of kernels.cu built for mechanisms of 6, 7, 8, 10 species, so that
// any mechanism up to OSTC_MAX_SPEC runs with its species count as a
// compile-time constant (per-species arrays in registers).
#define OSTC_NS_UNIT ns_b
#define OSTC_NS_LIST(X) X(6) X(7) X(8) X(10)
#include "kernels.cu"
