// Strict-arithmetic kernels: compiled with --fmad=false so that every FP64
// expression rounds as the reference's CPU build (-ffp-contract=off) does.
#define EU_STRICT 1
#define EU3D_NS strict
#include "eu3d_kernels_impl.cuh"
