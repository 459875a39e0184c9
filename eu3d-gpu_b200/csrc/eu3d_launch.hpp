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
    int sms;       // multiprocessors of the device (fixed grids of the queue kernels)
    int flux_ci;   // nodes each flux block marches along x (autotuned; 0: 16)
    int recover_block; // threads per block of the recovery kernels, 32..128 (autotuned; 0: 128)
    int recover_minb;  // register target of the learned-mode recovery: 3, 4, 5 or 6 blocks per SM (0: 4)
    cudaStream_t stream;
};

bool sizes_supported(int ns, int nr);

// The launchers of one arithmetic flavour, so the host picks a flavour once.
struct Launchers {
    cudaError_t (*boundary)(const LaunchArgs &a);
    cudaError_t (*flux_update)(const LaunchArgs &a);
    cudaError_t (*recover_react)(const LaunchArgs &a, bool react);
    cudaError_t (*derived)(const LaunchArgs &a, int which, double *out);
    cudaError_t (*recover_classify)(const LaunchArgs &a, const LearnedParams &lp);
    cudaError_t (*learned_features)(const LaunchArgs &a, const LearnedParams &lp);
    cudaError_t (*learned_apply)(const LaunchArgs &a, const LearnedParams &lp);
    cudaError_t (*react_queue)(const LaunchArgs &a, const int *queue, int *count, int counter);
    cudaError_t (*react_heavy)(const LaunchArgs &a, int blocks);
    cudaError_t (*materialize)(const LaunchArgs &a);
    cudaError_t (*learned_route)(const LaunchArgs &a, const LearnedParams &lp);
    // a batch's shared kinetics stage over the instances of tab[0..n)
    cudaError_t (*react_queue_batch)(const LaunchArgs &a, const BatchCell *tab, int n, int *next, int counter);
    cudaError_t (*react_heavy_batch)(const LaunchArgs &a, const BatchCell *tab, int n, int *next, int blocks);
};

#define EU3D_DECLARE_LAUNCHERS(NSP)                                                                \
    namespace NSP {                                                                                \
    cudaError_t launch_boundary(const LaunchArgs &a);                                              \
    cudaError_t launch_flux_update(const LaunchArgs &a);                                           \
    cudaError_t launch_recover_react(const LaunchArgs &a, bool react);                             \
    cudaError_t launch_derived(const LaunchArgs &a, int which, double *out);                       \
    cudaError_t launch_set_value(double *dst, double v, cudaStream_t s);                           \
    cudaError_t launch_rk_combine(const LaunchArgs &a, const double *cs0, double ca, double cb);   \
    cudaError_t launch_cfl(const LaunchArgs &a, double cfl, unsigned long long *slot, double *time); \
    cudaError_t launch_recover_classify(const LaunchArgs &a, const LearnedParams &lp);             \
    cudaError_t launch_learned_features(const LaunchArgs &a, const LearnedParams &lp);             \
    cudaError_t launch_learned_apply(const LaunchArgs &a, const LearnedParams &lp);                \
    cudaError_t launch_learned_route(const LaunchArgs &a, const LearnedParams &lp);                \
    cudaError_t launch_react_queue(const LaunchArgs &a, const int *queue, int *count, int counter); \
    cudaError_t launch_state_from_tpy(const LaunchArgs &a, long long n, const double *T,           \
                                      const double *p, const double *Y, double *cs, double *E);    \
    cudaError_t launch_chem_samples(const LaunchArgs &a, long long n, double *cs, double *T,       \
                                    double *E, const double *dt, int *nchem);                      \
    cudaError_t launch_react_heavy(const LaunchArgs &a, int blocks);                               \
    cudaError_t launch_react_queue_batch(const LaunchArgs &a, const BatchCell *tab, int n, int *next, \
                                         int counter);                                             \
    cudaError_t launch_react_heavy_batch(const LaunchArgs &a, const BatchCell *tab, int n, int *next, \
                                         int blocks);                                              \
    cudaError_t launch_materialize(const LaunchArgs &a);                                           \
    cudaError_t launch_to_f32(const double *src, float *dst, long long n, cudaStream_t s);          \
    cudaError_t launch_halo(const LaunchArgs &a, int nf, int face, bool pack, void *msg);           \
    extern const Launchers launchers;                                                              \
    }

EU3D_DECLARE_LAUNCHERS(strict)
EU3D_DECLARE_LAUNCHERS(fast)
EU3D_DECLARE_LAUNCHERS(mixed)

} // namespace eu3d
