// kernels_ns_a.cu — the per-cell, boundary, interface, steady and chemistry
// kernels of kernels.cu built for mechanisms of 1, 2, 3, 4, 5 species, so that
// any mechanism up to OSTC_MAX_SPEC runs with its species count as a
// compile-time constant (per-species arrays in registers).
#define OSTC_NS_UNIT ns_a
#define OSTC_NS_LIST(X) X(1) X(2) X(3) X(4) X(5)
#include "kernels.cu"
