// Mixed-precision kernels (EU_PREC_MIXED): FP32 MUSCL/AUSM with the
// division-light limiter, FP64 conserved update, state recovery and kinetics
// with FMA contraction and the fast FP64 forms of the thermo and rate
// expressions (mixture-polynomial temperature Newton, exp-of-sums rates).
// These round differently from the reference's expressions at the 1e-15
// level, far below the FP32 flux error the mode already accepts. Cells whose
// predicted Nchem is large are advanced one warp per cell.
#define EU_EXACT_FLUX 0
// cells with a large Nchem go to the warp-per-cell kinetics (k_react_heavy)
#define EU_HEAVY_QUEUE 1
#define EU3D_NS mixed
#include "eu3d_kernels_impl.cuh"
