// kernels_ns_c.cu — the per-cell, boundary, interface, steady and chemistry
// kernels of kernels.cu built for mechanisms of 11, 12, 13, 14, 15 species, so that
// any mechanism up to OSTC_MAX_SPEC runs with its species count as a
// compile-time constant (per-species arrays in registers).
#define OSTC_NS_UNIT ns_c
#define OSTC_NS_LIST(X) X(11) X(12) X(13) X(14) X(15)
#include "kernels.cu"
