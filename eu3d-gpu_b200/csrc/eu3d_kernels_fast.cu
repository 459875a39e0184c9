// Fast-arithmetic kernels: FMA contraction and reciprocal forms allowed.
#define EU3D_NS fast
#include "eu3d_kernels_impl.cuh"
