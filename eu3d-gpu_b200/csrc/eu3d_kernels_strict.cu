// Strict-arithmetic kernels: compiled with --fmad=false, with the reference's
// expression forms everywhere, so every FP64 operation rounds as the
// reference's CPU build (-ffp-contract=off) does.
#define EU_EXACT_CHEM 1
#define EU_EXACT_FLUX 1
#define EU3D_NS strict
#include "eu3d_kernels_impl.cuh"
