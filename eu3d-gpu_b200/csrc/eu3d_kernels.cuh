// eu3d_kernels.cuh — the timestep kernels, templated on the species and
// reaction counts. Instantiated twice: eu3d_kernels_strict.cu (--fmad=false,
// EU_EXACT_CHEM/EU_EXACT_FLUX) and eu3d_kernels_fast.cu.
#pragma once

#include "eu3d_device.cuh"
#include "eu3d_mech_JA919.cuh"

#ifndef EU3D_NS
#error "define EU3D_NS (the arithmetic flavour's namespace) before including eu3d_kernels.cuh"
#endif

// Kernels live in a per-flavour namespace: the strict and fast translation
// units instantiate the same templates with different arithmetic, and their
// host-side symbols must not merge at link time.
namespace eu3d {
namespace EU3D_NS {

// ---------------------------------------------------------------- ghosts
// Flowfield::FieldBoundary_3dRSBI (src/Flowfield.cpp:593-807) on the ghost
// layers the stencils read: x faces over interior (j,k), y faces over interior
// (i,k), z faces over interior (i,j). One thread per ghost node.
//   x low/high: zero-gradient mirror copy      (:597-641)
//   y low: symmetry, V reflected, rho/H/Gamma rebuilt from mirrored T, p, Y (:647-679)
//   y high: zero-gradient mirror copy          (:684-705)
//   z low/high: mirror copy with W reflected   (:710-802)
template <int NS>
__global__ void __launch_bounds__(256) k_boundary(const __grid_constant__ DevMech m, const DevGrid g,
                                                  const DevState st)
{
    const int bc = g.bc, ni = g.ni, nj = g.nj, nk = g.nk;
    const long long nxf = 2LL * bc * nj * nk, nyf = 2LL * bc * ni * nk, nzf = 2LL * bc * ni * nj;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nxf + nyf + nzf)
        return;
    const long long n3 = g.n3;
    long long dst, src;
    double sv = 1, sw = 1;
    bool rebuild = false;
    if (t < nxf) {
        const int k = bc + int(t % nk);
        const int j = bc + int((t / nk) % nj);
        const int q = int(t / ((long long)nk * nj)); // 0 .. 2bc-1
        const int i = q < bc ? q : ni + q;           // ghost index
        const int si = q < bc ? 2 * bc - 1 - i : 2 * (ni + bc) - 1 - i;
        dst = cell_index(g, i, j, k);
        src = cell_index(g, si, j, k);
    } else if (t < nxf + nyf) {
        t -= nxf;
        const int k = bc + int(t % nk);
        const int i = bc + int((t / nk) % ni);
        const int q = int(t / ((long long)nk * ni));
        const int j = q < bc ? q : nj + q;
        const int sj = q < bc ? 2 * bc - 1 - j : 2 * (nj + bc) - 1 - j;
        dst = cell_index(g, i, j, k);
        src = cell_index(g, i, sj, k);
        if (q < bc) {
            sv = -1;
            rebuild = true;
        }
    } else {
        t -= nxf + nyf;
        const int j = bc + int(t % nj);
        const int i = bc + int((t / nj) % ni);
        const int q = int(t / ((long long)nj * ni));
        const int k = q < bc ? q : nk + q;
        const int sk = q < bc ? 2 * bc - 1 - k : 2 * (nk + bc) - 1 - k;
        dst = cell_index(g, i, j, k);
        src = cell_index(g, i, j, sk);
        sw = -1;
    }
    double v[7 + NS];
#pragma unroll
    for (int f = 0; f < 7 + NS; ++f) v[f] = st.prim[f * n3 + src];
    v[kV] = sv * v[kV];
    v[kW] = sw * v[kW];
    const double T = st.T[src];
    if (rebuild) {
        const TPow p = make_tpow(T, true);
        double rg = 0, cp = 0, h = 0, e = 0;
        double Cpi[NS], Hi[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            Cpi[s] = cp_species<NS>(m, p, m.ri[s], s);
            Hi[s] = h_species<NS>(m, p, m.ri[s], s);
        }
#pragma unroll
        for (int s = 0; s < NS; ++s) rg += v[kY0 + s] * m.ri[s];
        const double Rgas = rg * 1000;
        v[kD] = v[kP] / (T * Rgas);
#pragma unroll
        for (int s = 0; s < NS; ++s) cp += Cpi[s] * v[kY0 + s];
#pragma unroll
        for (int s = 0; s < NS; ++s) h += v[kY0 + s] * Hi[s];
        (void)e;
        const double Cp = cp * 1000;
        v[kH] = h * 1000;
        v[kG] = Cp / (Cp - Rgas);
    }
    st.T[dst] = T;
#pragma unroll
    for (int f = 0; f < 7 + NS; ++f) {
        st.prim[f * n3 + dst] = v[f];
        if (st.prim32)
            st.prim32[f * n3 + dst] = float(v[f]);
    }
}

// ----------------------------------------------------------------- fluxes

// Face flux between cell c and c + stride along DIR, from the primitive planes
// (FP64 or FP32 copies): MUSCL_2 on every primitive, then AUSM+.
template <int NS, int DIR, typename R, bool kStrict>
__device__ __forceinline__ void face_flux(const R *__restrict__ prim, long long n3, long long c, long long stride,
                                          R (&F)[NS + 4])
{
    R L[7], Rt[7], YL[NS], YR[NS];
#pragma unroll
    for (int f = 0; f < 7; ++f) {
        const R *a = prim + f * n3 + c;
        muscl<R, kStrict>(__ldg(a - stride), __ldg(a), __ldg(a + stride), __ldg(a + 2 * stride), L[f], Rt[f]);
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const R *a = prim + (kY0 + s) * n3 + c;
        muscl<R, kStrict>(__ldg(a - stride), __ldg(a), __ldg(a + stride), __ldg(a + 2 * stride), YL[s], YR[s]);
    }
    ausm<NS, DIR, R, kStrict, R>(L, Rt, YL, YR, F);
}

// Flux divergence and the Euler-explicit update (TimeAdv::EE, src/TimeAdv.cpp:42-56,
// then CS += RHS, src/Flowfield.cpp:1350-1354) with every face flux formed once.
//
// A block owns a kFluxTJ x kFluxTK tile of (j, k) columns and marches along x
// over kFluxCI nodes. The x-face flux at i-1/2 stays in registers from the
// previous node; the y- and z-face fluxes of the current plane go through
// shared memory (row 0 / column 0 hold the faces below the tile, computed by
// warp 0 and by eight lanes of warp 1). RHS keeps the reference's order
// -dt/dx (F+ - F-) - dt/dy (G+ - G-) - dt/dz (Q+ - Q-), accumulated in FP64.
constexpr int kFluxTK = 32, kFluxTJ = 8, kFluxCI = 16;

template <int NS, typename R>
constexpr size_t flux_smem_bytes()
{
    return sizeof(R) * (NS + 4) * ((kFluxTJ + 1) * kFluxTK + kFluxTJ * (kFluxTK + 1));
}

template <int NS, typename R, bool kStrict>
__global__ void __launch_bounds__(kFluxTK *kFluxTJ, 1)
    k_flux_update(const DevGrid g, const DevState st, const R *__restrict__ prim, const double *__restrict__ dt_dev)
{
    constexpr int NV = NS + 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R(*sG)[kFluxTJ + 1][kFluxTK] = reinterpret_cast<R(*)[kFluxTJ + 1][kFluxTK]>(smem_raw);
    R(*sQ)[kFluxTJ][kFluxTK + 1] =
        reinterpret_cast<R(*)[kFluxTJ][kFluxTK + 1]>(smem_raw + sizeof(R) * NV * (kFluxTJ + 1) * kFluxTK);

    const int tx = threadIdx.x, ty = threadIdx.y;
    const int k0 = blockIdx.x * kFluxTK, j0 = blockIdx.y * kFluxTJ;
    const int k = g.bc + k0 + tx, j = g.bc + j0 + ty;
    const bool valid = (k0 + tx < g.nk) && (j0 + ty < g.nj);
    const int i_begin = g.bc + blockIdx.z * kFluxCI;
    const int i_end = min(i_begin + kFluxCI, g.bc + g.ni);
    const long long n3 = g.n3, sx = (long long)g.ny * g.nz, sy = g.nz;
    const double dt = *dt_dev;
    const double cy = valid ? dt / (g.y[j] - g.y[j - 1]) : 0.0;
    const double cz = valid ? dt / (g.z[k] - g.z[k - 1]) : 0.0;
    // lanes of warp 1 that form the z faces below the tile, one per row
    const int zrow = tx;
    const bool zlow = (ty == 1) && (tx < kFluxTJ) && (j0 + zrow < g.nj) && (k0 < g.nk);

    R Fm[NV];
    if (valid)
        face_flux<NS, 0, R, kStrict>(prim, n3, cell_index(g, i_begin - 1, j, k), sx, Fm);
    for (int i = i_begin; i < i_end; ++i) {
        const long long c = cell_index(g, i, j, k);
        R Fp[NV];
        if (valid) {
            face_flux<NS, 0, R, kStrict>(prim, n3, c, sx, Fp);
            {
                R G[NV];
                face_flux<NS, 1, R, kStrict>(prim, n3, c, sy, G);
#pragma unroll
                for (int q = 0; q < NV; ++q) sG[q][ty + 1][tx] = G[q];
            }
            {
                R Q[NV];
                face_flux<NS, 2, R, kStrict>(prim, n3, c, 1, Q);
#pragma unroll
                for (int q = 0; q < NV; ++q) sQ[q][ty][tx + 1] = Q[q];
            }
            if (ty == 0) {
                R G[NV];
                face_flux<NS, 1, R, kStrict>(prim, n3, c - sy, sy, G);
#pragma unroll
                for (int q = 0; q < NV; ++q) sG[q][0][tx] = G[q];
            }
        }
        if (zlow) {
            R Q[NV];
            face_flux<NS, 2, R, kStrict>(prim, n3, cell_index(g, i, g.bc + j0 + zrow, g.bc + k0 - 1), 1, Q);
#pragma unroll
            for (int q = 0; q < NV; ++q) sQ[q][zrow][0] = Q[q];
        }
        __syncthreads();
        if (valid) {
            const double cx = -dt / (g.x[i] - g.x[i - 1]);
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                const double rhs = cx * (double(Fp[q]) - double(Fm[q])) -
                                   cy * (double(sG[q][ty + 1][tx]) - double(sG[q][ty][tx])) -
                                   cz * (double(sQ[q][ty][tx + 1]) - double(sQ[q][ty][tx]));
                st.cs[q * n3 + c] = st.cs[q * n3 + c] + rhs;
                Fm[q] = Fp[q];
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------- recovery + kinetics

template <int NS>
__device__ __forceinline__ void store_cell(const DevMech &m, const DevState &st, long long n3, long long c,
                                           const CellState<NS> &cell)
{
    double P, H, G;
    finish_primitives<NS>(m, cell, P, H, G);
    const double v[7] = {P, cell.D, cell.U, cell.V, cell.W, H, G};
#pragma unroll
    for (int f = 0; f < 7; ++f) st.prim[f * n3 + c] = v[f];
#pragma unroll
    for (int s = 0; s < NS; ++s) st.prim[(kY0 + s) * n3 + c] = cell.Y[s];
    if (st.prim32) {
#pragma unroll
        for (int f = 0; f < 7; ++f) st.prim32[f * n3 + c] = float(v[f]);
#pragma unroll
        for (int s = 0; s < NS; ++s) st.prim32[(kY0 + s) * n3 + c] = float(cell.Y[s]);
    }
#pragma unroll
    for (int q = 0; q < NS + 4; ++q) st.cs[q * n3 + c] = cell.cs[q];
    st.T[c] = cell.T;
    st.E[c] = cell.E;
    if (!(isfinite(cell.D) && isfinite(cell.T)))
        atomicAdd(&st.counters[kCntNonfinite], 1ULL);
}

// Post-advection state recovery (Flowfield::Update_after_Adv ->
// Update_after_CS, src/Flowfield.cpp:1579-1617), Nchem prediction
// (Reaction::TrapezoidPrediction, src/Reaction.cpp:865-942) and the Nchem
// trapezoid substeps with state recovery after each (src/Euler.cpp:462-493,
// src/Reaction.cpp:562-805, src/Flowfield.cpp:1521-1536). The prediction's
// rate evaluation is reused by the first substep: both evaluate the same
// expression on the same state. One thread per interior node.
// Rate evaluation from the runtime tables (any mechanism of these sizes).
template <int NS_, int NR_>
struct TableRates {
    static constexpr int NS = NS_, NR = NR_;
    __device__ __forceinline__ static void rates(const DevMech &m, double T, const double (&mc)[NS], SpeciesRates<NS> &k)
    {
        eval_rates<NS, NR>(m, T, mc, k);
    }
};

template <int NS, int NR, bool kReact, class Rt>
__global__ void __launch_bounds__(128) k_recover_react(const __grid_constant__ DevMech m, const DevGrid g,
                                                       const DevState st, const double *__restrict__ dt_dev,
                                                       int max_substeps)
{
    const long long ncell = (long long)g.ni * g.nj * g.nk;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncell)
        return;
    const int k = g.bc + int(t % g.nk);
    const int j = g.bc + int((t / g.nk) % g.nj);
    const int i = g.bc + int(t / ((long long)g.nk * g.nj));
    const long long n3 = g.n3;
    const long long c = cell_index(g, i, j, k);
    CellState<NS> cell;
#pragma unroll
    for (int q = 0; q < NS + 4; ++q) cell.cs[q] = st.cs[q * n3 + c];
    cell.T = st.T[c];
    cell.E = st.E[c];
    recover_state<NS>(m, cell);

    if (kReact) {
        const double dtm = *dt_dev;
        double mc[NS];
        scaled_concentrations<NS>(m, cell, mc);
        SpeciesRates<NS> rates;
        Rt::rates(m, cell.T, mc, rates);
        double dt = dtm;
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            if (cell.Y[s] >= 1e-6 && rates.W[s] != 0) {
                const double dt_temp = fabs(-(cell.cs[s] * 1e-3) / rates.W[s]);
                if (dt_temp < dt)
                    dt = dt_temp;
            }
        }
        const double ratio = ceil(dtm / dt);
        int nchem;
        if (!(ratio >= 1.0) || ratio > double(max_substeps)) {
            atomicAdd(&st.counters[kCntBadNchem], 1ULL);
            nchem = (ratio > double(max_substeps)) ? max_substeps : 0;
        } else {
            nchem = int(ratio);
        }
        st.nchem[c] = nchem;
        if (nchem > 0) {
            atomicMax(&st.counters[kCntMaxNchem], (unsigned long long)nchem);
            atomicAdd(&st.counters[kCntSumNchem], (unsigned long long)nchem);
        }
        const double dts = dtm / nchem;
        for (int step = 0; step < nchem; ++step) {
            if (step > 0) {
                scaled_concentrations<NS>(m, cell, mc);
                Rt::rates(m, cell.T, mc, rates);
            }
            if (st.cms) {
#pragma unroll
                for (int s = 0; s < NS; ++s) st.cms[s * n3 + c] = rates.W[s] * 1e3;
            }
            trapezoid_substep<NS>(m, rates, dts, mc, cell);
        }
    }
    store_cell<NS>(m, st, n3, c, cell);
}

// Derived output fields of Update_after_CS that the timestep does not keep
// (Wav, Rgas, Cp, C, Ma; src/Flowfield.cpp:1606-1616), from the stored state.
template <int NS>
__global__ void k_derived(const __grid_constant__ DevMech m, const DevGrid g, const DevState st, int which,
                          double *out)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.n3)
        return;
    const long long n3 = g.n3;
    double inv_w = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) inv_w += st.prim[(kY0 + s) * n3 + c] / m.mw[s];
    const double Wav = 1.0 / inv_w;
    double v;
    if (which == 0) {
        v = Wav;
    } else if (which == 1) {
        v = kRUniv * 1000 / Wav;
    } else if (which == 2) {
        const TPow p = make_tpow(st.T[c], false);
        double cp = 0;
#pragma unroll
        for (int s = 0; s < NS; ++s) cp += cp_species<NS>(m, p, m.ri[s], s) * st.prim[(kY0 + s) * n3 + c];
        v = cp * 1000;
    } else {
        const double C = sqrt(st.prim[kG * n3 + c] * st.prim[kP * n3 + c] / st.prim[kD * n3 + c]);
        if (which == 3) {
            v = C;
        } else {
            const double U = st.prim[kU * n3 + c], V = st.prim[kV * n3 + c], W = st.prim[kW * n3 + c];
            v = sqrt(U * U + V * V + W * W) / C;
        }
    }
    out[c] = v;
}

// Writes a scalar (the timestep) into device memory from a kernel argument, so
// the value is captured at launch and the caller's copy may go away.
__global__ void k_set_value(double *dst, double v) { *dst = v; }

} // namespace EU3D_NS
} // namespace eu3d
