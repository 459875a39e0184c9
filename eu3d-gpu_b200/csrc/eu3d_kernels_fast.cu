// Fast-arithmetic kernels: FMA contraction allowed, division-light flux
// reconstruction. The thermo/rate expressions keep the reference's forms by
// default (they cost the same here once the mechanism is specialised); build
// with -DEU_FAST_CHEM to use the exp-of-sums rate and mixture-polynomial forms.
#ifndef EU_FAST_CHEM
#define EU_EXACT_CHEM 1
#endif
#ifndef EU_EXACT_FLUX
#define EU_EXACT_FLUX 0
#endif
#define EU3D_NS fast
#include "eu3d_kernels_impl.cuh"
