// eu3d_launch.hpp — host-side launch interface of the kernel translation
// units. Each arithmetic flavour (strict: no FMA, rounds as the reference's
// CPU build; fast: FMA allowed) is compiled into its own namespace.
#pragma once

#include <cuda_runtime.h>

#include "eu3d_types.h"

namespace eu3d {

struct LaunchArgs {
    const DevMech *mech; // host copy, passed to kernels by value
    DevGrid g;
    DevState st;
    const double *dt_dev;
    int max_substeps;
    int precision; // eu_precision
    int chemistry; // eu_chemistry
    int spec;      // 1: tables are bitwise H2_JA919, use the generated rate code
    cudaStream_t stream;
};

bool sizes_supported(int ns, int nr);

#define EU3D_DECLARE_LAUNCHERS(NSP)                                                                \
    namespace NSP {                                                                                \
    cudaError_t launch_boundary(const LaunchArgs &a);                                              \
    cudaError_t launch_flux_update(const LaunchArgs &a);                                           \
    cudaError_t launch_recover_react(const LaunchArgs &a, bool react);                             \
    cudaError_t launch_derived(const LaunchArgs &a, int which, double *out);                       \
    cudaError_t launch_set_value(double *dst, double v, cudaStream_t s);                           \
    }

EU3D_DECLARE_LAUNCHERS(strict)
EU3D_DECLARE_LAUNCHERS(fast)

} // namespace eu3d
