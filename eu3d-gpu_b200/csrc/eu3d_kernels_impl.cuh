// eu3d_kernels_impl.cuh — launchers for one arithmetic flavour. Included once
// by eu3d_kernels_strict.cu (--fmad=false, exact forms) and once by
// eu3d_kernels_fast.cu, with EU3D_NS naming the namespace.
#pragma once

#include <algorithm>

#include "eu3d_attr.hpp"
#include "eu3d_kernels.cuh"
#include "eu3d_launch.hpp"

namespace eu3d {
namespace EU3D_NS {

namespace {

template <int NS, int NR>
cudaError_t boundary_t(const LaunchArgs &a)
{
    const DevGrid &g = a.g;
    const long long n = 2LL * g.bc * ((long long)g.nj * g.nk + (long long)g.ni * g.nk + (long long)g.ni * g.nj);
    const int threads = 256;
    const long long blocks = (n + threads - 1) / threads;
    k_boundary<NS><<<dim3((unsigned)blocks), threads, 0, a.stream>>>(*a.mech, g, a.st);
    return cudaGetLastError();
}

// FP64 reconstruction: the reference's divisions (EU_EXACT_FLUX=1) or the
// division-light limiter form.
constexpr bool kStrictFlux = EU_EXACT_FLUX != 0;

template <int NS, typename R, bool kStrict>
cudaError_t flux_launch(const LaunchArgs &a, const R *prim)
{
    const DevGrid &g = a.g;
    const size_t smem = flux_smem_bytes<NS, R>();
    static SmemLimit limit; // per instantiation, per device
    const cudaError_t e = limit.ensure(k_flux_update<NS, R, kStrict>, smem);
    if (e != cudaSuccess)
        return e;
    const dim3 block(kFluxTK, kFluxTJ);
    const int ci = a.flux_ci > 0 ? a.flux_ci : 16;
    const dim3 grid((g.nk + kFluxTK - 1) / kFluxTK, (g.nj + kFluxTJ - 1) / kFluxTJ, (g.ni + ci - 1) / ci);
    k_flux_update<NS, R, kStrict><<<grid, block, smem, a.stream>>>(g, a.st, prim, a.dt_dev, ci);
    return cudaGetLastError();
}

template <int NS, typename R, bool kStrict>
cudaError_t tiled_flux_launch(const LaunchArgs &a, const R *prim)
{
    const DevGrid &g = a.g;
    const size_t smem = tiled_flux_smem_bytes<NS, R>();
    static SmemLimit limit; // per instantiation, per device
    const cudaError_t e = limit.ensure(k_flux_update_tiled<NS, R, kStrict>, smem);
    if (e != cudaSuccess)
        return e;
    const dim3 block(kTileK, TileShape<R>::Warps);
    const int ci = a.flux_ci > 0 ? a.flux_ci : 16;
    const dim3 grid((g.nk + kTileK - 1) / kTileK, (g.nj + TileShape<R>::J - 1) / TileShape<R>::J,
                    (g.ni + ci - 1) / ci);
    k_flux_update_tiled<NS, R, kStrict><<<grid, block, smem, a.stream>>>(g, a.st, prim, a.dt_dev, ci);
    return cudaGetLastError();
}

// Grids thin in z: one thread per (j, k) column.
constexpr int kThinNk = 16;

template <int NS, typename R, bool kStrict>
cudaError_t cols_flux_launch(const LaunchArgs &a, const R *prim)
{
    const DevGrid &g = a.g;
    const int ci = a.flux_ci > 0 ? a.flux_ci : 16;
    const dim3 grid(unsigned((g.nj * g.nk + 127) / 128), unsigned((g.ni + ci - 1) / ci));
    k_flux_update_cols<NS, R, kStrict><<<grid, 128, 0, a.stream>>>(g, a.st, prim, a.dt_dev, ci);
    return cudaGetLastError();
}

template <int NS, int NR>
cudaError_t flux_t(const LaunchArgs &a)
{
    if (a.g.nk < kThinNk) {
        if (a.precision == 1)
            return cols_flux_launch<NS, float, false>(a, a.st.prim32);
        return cols_flux_launch<NS, double, kStrictFlux>(a, a.st.prim);
    }
    // mixed precision: FP32 reconstruction and AUSM (always the division-light
    // forms); FP64: the reference's forms (strict) or the division-light
    // limiter (fast). Both plane-tiled.
    if (a.precision == 1)
        return tiled_flux_launch<NS, float, false>(a, a.st.prim32);
    return tiled_flux_launch<NS, double, kStrictFlux>(a, a.st.prim);
}

template <int NS, int NR>
cudaError_t react_t(const LaunchArgs &a, bool react)
{
    const DevGrid &g = a.g;
    const long long n = (long long)g.ni * g.nj * g.nk;
    const int threads = a.recover_block > 0 ? a.recover_block : 128;
    const long long blocks = (n + threads - 1) / threads;
    const dim3 grid((unsigned)blocks);
    if (!react)
        k_recover_react<NS, NR, false, TableRates<NS, NR>><<<grid, threads, 0, a.stream>>>(*a.mech, g, a.st, a.dt_dev,
                                                                                           a.max_substeps);
    else if (a.spec == 1 && NS == Mech_JA919::NS && NR == Mech_JA919::NR) {
        // register target (autotuned): 2, 3 or 4 resident blocks per SM
        if (a.recover_minb == 4)
            k_recover_react<NS, NR, true, Mech_JA919, 4><<<grid, threads, 0, a.stream>>>(*a.mech, g, a.st, a.dt_dev,
                                                                                       a.max_substeps);
        else if (a.recover_minb == 3)
            k_recover_react<NS, NR, true, Mech_JA919, 3><<<grid, threads, 0, a.stream>>>(*a.mech, g, a.st, a.dt_dev,
                                                                                       a.max_substeps);
        else
            k_recover_react<NS, NR, true, Mech_JA919, 2><<<grid, threads, 0, a.stream>>>(*a.mech, g, a.st, a.dt_dev,
                                                                                       a.max_substeps);
    } else
        k_recover_react<NS, NR, true, TableRates<NS, NR>><<<grid, threads, 0, a.stream>>>(*a.mech, g, a.st, a.dt_dev,
                                                                                          a.max_substeps);
    return cudaGetLastError();
}

template <int NS, int NR>
cudaError_t derived_t(const LaunchArgs &a, int which, double *out)
{
    const int threads = 256;
    const long long blocks = (a.g.n3 + threads - 1) / threads;
    k_derived<NS><<<dim3((unsigned)blocks), threads, 0, a.stream>>>(*a.mech, a.g, a.st, which, out);
    return cudaGetLastError();
}

template <int NS, int NR>
cudaError_t materialize_t(const LaunchArgs &a)
{
    if (!a.st.prim32)
        return cudaSuccess;
    k_materialize<NS><<<dim3(unsigned((a.g.n3 + 127) / 128)), 128, 0, a.stream>>>(*a.mech, a.g, a.st);
    return cudaGetLastError();
}

template <int NS, int NR>
cudaError_t classify_t(const LaunchArgs &a, const LearnedParams &lp)
{
    const long long n = (long long)a.g.ni * a.g.nj * a.g.nk;
    const int threads = a.recover_block > 0 ? a.recover_block : 128;
    const dim3 grid(unsigned((n + threads - 1) / threads));
    switch (a.recover_minb) {
    case 3: k_recover_classify<NS, 3><<<grid, threads, 0, a.stream>>>(*a.mech, a.g, a.st, lp); break;
    case 5: k_recover_classify<NS, 5><<<grid, threads, 0, a.stream>>>(*a.mech, a.g, a.st, lp); break;
    case 6: k_recover_classify<NS, 6><<<grid, threads, 0, a.stream>>>(*a.mech, a.g, a.st, lp); break;
    default: k_recover_classify<NS, 4><<<grid, threads, 0, a.stream>>>(*a.mech, a.g, a.st, lp); break;
    }
    return cudaGetLastError();
}

// The learned-chemistry kernels run on fixed grids that read the queue lengths
// on the device, so a step needs no host-side count and can be captured.
inline unsigned queue_grid(const LaunchArgs &a, int per_sm) { return unsigned((a.sms > 0 ? a.sms : 148) * per_sm); }

template <int NS, int NR>
cudaError_t features_t(const LaunchArgs &a, const LearnedParams &lp)
{
    k_learned_features<NS><<<dim3(queue_grid(a, 8)), 128, 0, a.stream>>>(*a.mech, a.g, a.st, lp, a.dt_dev);
    return cudaGetLastError();
}

template <int NS, int NR>
cudaError_t apply_t(const LaunchArgs &a, const LearnedParams &lp)
{
    k_learned_apply<NS><<<dim3(queue_grid(a, 8)), 128, 0, a.stream>>>(*a.mech, a.g, a.st, lp);
    return cudaGetLastError();
}

// count[0]: queue length, count[1]: cells taken so far (zero at launch)
template <int NS, int NR>
cudaError_t react_queue_t(const LaunchArgs &a, const int *queue, int *count, int counter)
{
    const dim3 grid(queue_grid(a, 4));
    if (a.spec == 1 && NS == Mech_JA919::NS && NR == Mech_JA919::NR)
        k_react_queue<NS, Mech_JA919><<<grid, 128, 0, a.stream>>>(*a.mech, a.g, a.st, queue, count, a.dt_dev,
                                                                  a.max_substeps, counter);
    else
        k_react_queue<NS, TableRates<NS, NR>><<<grid, 128, 0, a.stream>>>(*a.mech, a.g, a.st, queue, count,
                                                                          a.dt_dev, a.max_substeps, counter);
    return cudaGetLastError();
}

template <int NS, int NR>
cudaError_t route_t(const LaunchArgs &a, const LearnedParams &lp)
{
    const dim3 grid(queue_grid(a, 4));
    if (a.spec == 1 && NS == Mech_JA919::NS && NR == Mech_JA919::NR)
        k_learned_route<NS, Mech_JA919><<<grid, 128, 0, a.stream>>>(*a.mech, a.g, a.st, lp, a.dt_dev, a.max_substeps);
    else
        k_learned_route<NS, TableRates<NS, NR>><<<grid, 128, 0, a.stream>>>(*a.mech, a.g, a.st, lp, a.dt_dev,
                                                                            a.max_substeps);
    return cudaGetLastError();
}

template <int NS, int NR>
cudaError_t state_from_tpy_t(const LaunchArgs &a, long long n, const double *T, const double *p, const double *Y,
                             double *cs, double *E)
{
    if (n <= 0)
        return cudaSuccess;
    k_state_from_tpy<NS><<<dim3(unsigned((n + 127) / 128)), 128, 0, a.stream>>>(*a.mech, n, T, p, Y, cs, E);
    return cudaGetLastError();
}

template <int NS, int NR>
cudaError_t chem_samples_t(const LaunchArgs &a, long long n, double *cs, double *T, double *E, const double *dt,
                           int *nchem)
{
    if (n <= 0)
        return cudaSuccess;
    const dim3 grid(unsigned((n + 127) / 128));
    if (a.spec == 1 && NS == Mech_JA919::NS && NR == Mech_JA919::NR)
        k_chem_samples<NS, Mech_JA919><<<grid, 128, 0, a.stream>>>(*a.mech, n, cs, T, E, dt, nchem, a.max_substeps,
                                                                   a.st.counters);
    else
        k_chem_samples<NS, TableRates<NS, NR>><<<grid, 128, 0, a.stream>>>(*a.mech, n, cs, T, E, dt, nchem,
                                                                           a.max_substeps, a.st.counters);
    return cudaGetLastError();
}

template <int NS, int NR>
cudaError_t heavy_t(const LaunchArgs &a, int blocks)
{
    k_react_heavy<NS, NR><<<dim3(unsigned(blocks)), 128, 0, a.stream>>>(*a.mech, a.g, a.st, a.dt_dev,
                                                                         a.max_substeps);
    return cudaGetLastError();
}

// The batch's shared kinetics stage: the stiff-fallback queues, then the
// deferred cells, of every instance in tab[0..n) drained by one fixed grid
// each (next[0] and next[1] zero at launch). a: any member's arguments (the
// mechanism, flavour and substep cap are the same over the table).
template <int NS, int NR>
cudaError_t react_queue_batch_t(const LaunchArgs &a, const BatchCell *tab, int n, int *next, int counter)
{
    const dim3 grid(queue_grid(a, 4));
    if (a.spec == 1 && NS == Mech_JA919::NS && NR == Mech_JA919::NR)
        k_react_queue_batch<NS, Mech_JA919><<<grid, 128, 0, a.stream>>>(*a.mech, tab, n, next, a.max_substeps,
                                                                        counter);
    else
        k_react_queue_batch<NS, TableRates<NS, NR>><<<grid, 128, 0, a.stream>>>(*a.mech, tab, n, next,
                                                                                a.max_substeps, counter);
    return cudaGetLastError();
}

template <int NS, int NR>
cudaError_t heavy_batch_t(const LaunchArgs &a, const BatchCell *tab, int n, int *next, int blocks)
{
    k_react_heavy_batch<NS, NR><<<dim3(unsigned(blocks)), 128, 0, a.stream>>>(*a.mech, tab, n, next + 1,
                                                                               a.max_substeps);
    return cudaGetLastError();
}

} // namespace

// Supported (NS, NR): the repository mechanism H2_JA919 (9 species, 19
// reactions), the one the reference's parser reads.
#define EU3D_DISPATCH(fn, ...)                                                                     \
    switch (a.mech->ns * 100 + a.mech->nr) {                                                        \
    case 919:                                                                                      \
        return fn<9, 19>(__VA_ARGS__);                                                             \
    default:                                                                                       \
        return cudaErrorInvalidValue;                                                              \
    }

cudaError_t launch_boundary(const LaunchArgs &a) { EU3D_DISPATCH(boundary_t, a) }
cudaError_t launch_flux_update(const LaunchArgs &a) { EU3D_DISPATCH(flux_t, a) }
cudaError_t launch_recover_react(const LaunchArgs &a, bool react) { EU3D_DISPATCH(react_t, a, react) }
cudaError_t launch_derived(const LaunchArgs &a, int which, double *out) { EU3D_DISPATCH(derived_t, a, which, out) }
cudaError_t launch_materialize(const LaunchArgs &a) { EU3D_DISPATCH(materialize_t, a) }
cudaError_t launch_to_f32(const double *src, float *dst, long long n, cudaStream_t s)
{
    if (n <= 0)
        return cudaSuccess;
    k_to_f32<<<dim3(unsigned(std::min<long long>((n + 255) / 256, 148LL * 16))), 256, 0, s>>>(src, dst, n);
    return cudaGetLastError();
}

cudaError_t launch_recover_classify(const LaunchArgs &a, const LearnedParams &lp) { EU3D_DISPATCH(classify_t, a, lp) }
cudaError_t launch_learned_features(const LaunchArgs &a, const LearnedParams &lp) { EU3D_DISPATCH(features_t, a, lp) }
cudaError_t launch_learned_apply(const LaunchArgs &a, const LearnedParams &lp) { EU3D_DISPATCH(apply_t, a, lp) }
cudaError_t launch_learned_route(const LaunchArgs &a, const LearnedParams &lp) { EU3D_DISPATCH(route_t, a, lp) }
cudaError_t launch_react_queue(const LaunchArgs &a, const int *queue, int *count, int counter)
{
    EU3D_DISPATCH(react_queue_t, a, queue, count, counter)
}
cudaError_t launch_state_from_tpy(const LaunchArgs &a, long long n, const double *T, const double *p, const double *Y,
                                  double *cs, double *E)
{
    EU3D_DISPATCH(state_from_tpy_t, a, n, T, p, Y, cs, E)
}
cudaError_t launch_chem_samples(const LaunchArgs &a, long long n, double *cs, double *T, double *E, const double *dt,
                                int *nchem)
{
    EU3D_DISPATCH(chem_samples_t, a, n, cs, T, E, dt, nchem)
}

cudaError_t launch_react_heavy(const LaunchArgs &a, int blocks) { EU3D_DISPATCH(heavy_t, a, blocks) }
cudaError_t launch_react_queue_batch(const LaunchArgs &a, const BatchCell *tab, int n, int *next, int counter)
{
    EU3D_DISPATCH(react_queue_batch_t, a, tab, n, next, counter)
}
cudaError_t launch_react_heavy_batch(const LaunchArgs &a, const BatchCell *tab, int n, int *next, int blocks)
{
    EU3D_DISPATCH(heavy_batch_t, a, tab, n, next, blocks)
}

cudaError_t launch_cfl(const LaunchArgs &a, double cfl, unsigned long long *slot, double *time)
{
    const long long n = (long long)a.g.ni * a.g.nj * a.g.nk;
    const unsigned blocks = unsigned(std::min<long long>((n + 255) / 256, (long long)(a.sms > 0 ? a.sms : 148) * 8));
    k_cfl_min<<<blocks, 256, 0, a.stream>>>(a.g, a.st, slot);
    k_cfl_finish<<<1, 1, 0, a.stream>>>(slot, cfl, const_cast<double *>(a.dt_dev), time);
    return cudaGetLastError();
}

// face 0: x low, 1: x high; pack: planes -> msg, else msg -> ghost planes.
cudaError_t launch_halo(const LaunchArgs &a, int nf, int face, bool pack, void *msg)
{
    const DevGrid &g = a.g;
    const long long plane = (long long)g.ny * g.nz;
    int first, step;
    if (pack) {
        first = face == 0 ? g.bc + 1 : g.ni + g.bc - 2;
        step = face == 0 ? 1 : -1;
    } else {
        first = face == 0 ? g.bc - 1 : g.ni + g.bc;
        step = face == 0 ? -1 : 1;
    }
    const long long total = (long long)nf * g.bc * plane;
    const unsigned blocks = unsigned(std::min<long long>((total + 255) / 256, (long long)(a.sms > 0 ? a.sms : 148) * 8));
    if (a.st.prim32)
        k_halo_copy<float><<<blocks, 256, 0, a.stream>>>(a.st.prim32, static_cast<float *>(msg), nf, g.bc, g.n3, plane,
                                                       first, step, pack);
    else
        k_halo_copy<double><<<blocks, 256, 0, a.stream>>>(a.st.prim, static_cast<double *>(msg), nf, g.bc, g.n3, plane,
                                                        first, step, pack);
    return cudaGetLastError();
}

cudaError_t launch_rk_combine(const LaunchArgs &a, const double *cs0, double ca, double cb)
{
    const long long n = (long long)a.g.ni * a.g.nj * a.g.nk;
    const unsigned blocks = unsigned(std::min<long long>((n + 255) / 256, (long long)(a.sms > 0 ? a.sms : 148) * 8));
    k_rk_combine<<<blocks, 256, 0, a.stream>>>(a.g, a.st.cs, cs0, a.mech->ns + 4, ca, cb);
    return cudaGetLastError();
}

cudaError_t launch_set_value(double *dst, double v, cudaStream_t s)
{
    k_set_value<<<1, 1, 0, s>>>(dst, v);
    return cudaGetLastError();
}

const Launchers launchers = {&launch_boundary,         &launch_flux_update,      &launch_recover_react,
                             &launch_derived,          &launch_recover_classify, &launch_learned_features,
                             &launch_learned_apply,    &launch_react_queue,      &launch_react_heavy,
                             &launch_materialize,      &launch_learned_route,    &launch_react_queue_batch,
                             &launch_react_heavy_batch};

#undef EU3D_DISPATCH

} // namespace EU3D_NS
} // namespace eu3d
