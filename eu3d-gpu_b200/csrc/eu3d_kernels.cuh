// eu3d_kernels.cuh — the timestep kernels, templated on the species and
// reaction counts. Instantiated twice: eu3d_kernels_strict.cu (--fmad=false,
// EU_EXACT_CHEM/EU_EXACT_FLUX) and eu3d_kernels_fast.cu.
#pragma once

#include "eu3d_device.cuh"
#include "eu3d_mech_JA919.cuh"
#include "eu3d_tc.cuh"

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
// With g.bc_kind == 1 the x faces follow Flowfield::FieldBoundary_1dZND
// (src/Flowfield.cpp:317-411, commented out in the reference): x low a
// reflecting wall (mirror copy, U reflected), x high outflow (mirror copy of
// U, V, p, T, Y with rho/H/Gamma rebuilt as on the y-low face).
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
    double su = 1, sv = 1, sw = 1;
    bool rebuild = false;
    long long inflow = -1; // ODW x-low: index into the inflow tables
    if (t < nxf) {
        const int jk = fdiv(t, g.d_nk), q = fdiv(t, g.d_njnk); // q: 0 .. 2bc-1
        const int k = bc + int(t - (long long)jk * nk);
        const int j = bc + (jk - q * nj);
        if (q < bc ? g.exch_lo : g.exch_hi) // filled by the halo exchange
            return;
        const int i = q < bc ? q : ni + q;           // ghost index
        const int si = q < bc ? 2 * bc - 1 - i : 2 * (ni + bc) - 1 - i;
        dst = cell_index(g, i, j, k);
        src = cell_index(g, si, j, k);
        if (g.bc_kind == 1) {
            su = q < bc ? -1 : 1;
            rebuild = q >= bc;
        } else if (g.bc_kind == 2) { // ODW: freestream tables in, rebuilt outflow out
            if (q < bc)
                inflow = (long long)(j - bc) * nk + (k - bc);
            rebuild = q >= bc;
        }
    } else if (t < nxf + nyf) {
        t -= nxf;
        const int ik = fdiv(t, g.d_nk), q = fdiv(t, g.d_nink);
        const int k = bc + int(t - (long long)ik * nk);
        const int i = bc + (ik - q * ni);
        const int j = q < bc ? q : nj + q;
        const int sj = q < bc ? 2 * bc - 1 - j : 2 * (nj + bc) - 1 - j;
        dst = cell_index(g, i, j, k);
        src = cell_index(g, i, sj, k);
        if (q < bc) {
            if (g.bc_kind == 2 && i - bc < g.wall_i0) {
                inflow = k - bc; // ODW ahead of the wall: the freestream (first table row)
            } else {
                sv = -1;
                rebuild = true;
            }
        }
    } else {
        // the ghost index runs fastest: the 2 bc ghosts of one (i, j) row sit in
        // two contiguous pairs, so a warp touches 16 pairs instead of 32 rows
        t -= nxf + nyf;
        if (st.zm_fresh && *st.zm_fresh) // EU_GHOSTS_STORED: stored with the interior
            return;
        const int jq = fdiv(t, g.d_ghost), ii = fdiv(t, g.d_ghost_nj);
        const int q = int(t - (long long)jq * (2 * bc));
        const int j = bc + (jq - ii * nj);
        const int i = bc + ii;
        const int k = q < bc ? q : nk + q;
        const int sk = q < bc ? 2 * bc - 1 - k : 2 * (nk + bc) - 1 - k;
        dst = cell_index(g, i, j, k);
        src = cell_index(g, i, j, sk);
        sw = -1;
        rebuild = g.bc_kind == 2; // ODW rebuilds the thermo on the z faces
    }
    if (inflow >= 0) {
        const long long nt = (long long)nj * nk;
#pragma unroll
        for (int f = 0; f < 7 + NS; ++f) {
            const double v = st.inflow[f * nt + inflow];
            if (st.prim32)
                st.prim32[f * n3 + dst] = float(v);
            else
                st.prim[f * n3 + dst] = v;
        }
        st.T[dst] = st.inflow[(7 + NS) * nt + inflow];
        return;
    }
    // mixed precision keeps only the FP32 primitive planes current (the flux
    // kernel's input); the FP64 path its FP64 planes
    double v[7 + NS];
#pragma unroll
    for (int f = 0; f < 7 + NS; ++f) v[f] = st.prim32 ? double(st.prim32[f * n3 + src]) : st.prim[f * n3 + src];
    v[kU] = su * v[kU];
    v[kV] = sv * v[kV];
    v[kW] = sw * v[kW];
    const double T = st.T[src];
    if (rebuild) {
        const TPow p = make_tpow(T, true);
        double rg = 0, cp = 0, h = 0, e = 0;
        double Cpi[NS], Hi[NS];
        by_range(p.low, [&](auto range) {
            constexpr int kR = decltype(range)::value;
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                Cpi[s] = cp_species<NS, kR>(m, p, m.ri[s], s);
                Hi[s] = h_species<NS, kR>(m, p, m.ri[s], s);
            }
        });
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
        if (st.prim32)
            st.prim32[f * n3 + dst] = float(v[f]);
        else
            st.prim[f * n3 + dst] = v[f];
    }
}

// Halo messages between x blocks (Flowfield::Mpi_Boundary, src/Flowfield.cpp:809-911):
// plane p (0 .. bc-1) of field f of a message is node plane src_i(p) of the flux
// primitives. to_msg: planes -> message (pack), else message -> planes (unpack).
// Node planes: pack face 0 takes bc+1+p, pack face 1 takes ni+bc-2-p; unpack
// face 0 fills bc-1-p, unpack face 1 fills ni+bc+p.
template <typename R>
__global__ void k_halo_copy(R *planes, R *msg, int nf, int bc, long long n3, long long plane, int first, int step,
                            bool to_msg)
{
    const long long total = (long long)nf * bc * plane;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long fp = t / plane, e = t - fp * plane;
        const int f = int(fp / bc), p = int(fp - (long long)f * bc);
        R *node = planes + f * n3 + (long long)(first + step * p) * plane + e;
        if (to_msg)
            msg[t] = *node;
        else
            *node = msg[t];
    }
}

// ----------------------------------------------------------------- fluxes

// Face flux between cell c and c + stride along DIR, from the primitive planes
// (FP64 or FP32 copies): MUSCL_2 on every primitive, then AUSM+.
template <int NS, int DIR, typename R, bool kStrict>
__device__ __forceinline__ void face_flux(const R *__restrict__ prim, long long n3, long long c, long long stride,
                                          R (&F)[NS + 4])
{
    const R *a = prim + c - stride;
    face_ausm<NS, DIR, R, kStrict, R>([&](int f, int p) { return __ldg(a + f * n3 + p * stride); }, F);
}

// Flux divergence and the Euler-explicit update (TimeAdv::EE, src/TimeAdv.cpp:42-56,
// then CS += RHS, src/Flowfield.cpp:1350-1354) with every face flux formed once.
//
// A block owns a kFluxTJ x kFluxTK tile of (j, k) columns and marches along x
// over ci nodes (a launch parameter the autotuner picks). The x-face flux at
// i-1/2 stays in registers from the
// previous node; the y- and z-face fluxes of the current plane go through
// shared memory (row 0 / column 0 hold the faces below the tile, computed by
// warp 0 and by eight lanes of warp 1). RHS keeps the reference's order
// -dt/dx (F+ - F-) - dt/dy (G+ - G-) - dt/dz (Q+ - Q-), accumulated in FP64.
constexpr int kFluxTK = 32, kFluxTJ = 8;

template <int NS, typename R>
constexpr size_t flux_smem_bytes()
{
    return sizeof(R) * (NS + 4) * ((kFluxTJ + 1) * kFluxTK + kFluxTJ * (kFluxTK + 1));
}

template <int NS, typename R, bool kStrict>
__global__ void __launch_bounds__(kFluxTK *kFluxTJ, 1)
    k_flux_update(const DevGrid g, const DevState st, const R *__restrict__ prim, const double *__restrict__ dt_dev,
                  int ci)
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
    const int i_begin = g.bc + blockIdx.z * ci;
    const int i_end = min(i_begin + ci, g.bc + g.ni);
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

// Flux divergence and update for grids thin in z (nk below half a warp),
// where the (j, k) tiles of the kernels above and below would leave most lanes
// idle: one thread per (j, k) column (flattened, k fastest) marching ci nodes
// in x. The x face at i-1/2 is carried in registers from the previous node; the
// thread forms the y and z faces on both sides of its cell from the stencil in
// global memory (each interior y or z face twice, once by each of its cells).
// The RHS is formed in the same order as the other flux kernels (FP32
// differences and sum onto the FP64 conserved value for R = float, FP64 for
// R = double).
template <int NS, typename R, bool kStrict>
__global__ void __launch_bounds__(128) k_flux_update_cols(const DevGrid g, const DevState st,
                                                          const R *__restrict__ prim,
                                                          const double *__restrict__ dt_dev, int ci)
{
    constexpr int NV = NS + 4;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.nj * g.nk)
        return;
    const int jj = t / g.nk;
    const int j = g.bc + jj, k = g.bc + (t - jj * g.nk);
    const int i_begin = g.bc + blockIdx.y * ci;
    const int i_end = min(i_begin + ci, g.bc + g.ni);
    const long long n3 = g.n3, sx = (long long)g.ny * g.nz, sy = g.nz;
    const double dt = *dt_dev;
    const double cy = dt / (g.y[j] - g.y[j - 1]);
    const double cz = dt / (g.z[k] - g.z[k - 1]);
    R Fm[NV];
    face_flux<NS, 0, R, kStrict>(prim, n3, cell_index(g, i_begin - 1, j, k), sx, Fm);
    for (int i = i_begin; i < i_end; ++i) {
        const long long c = cell_index(g, i, j, k);
        const double cx = -dt / (g.x[i] - g.x[i - 1]);
        R Fp[NV], A[NV], B[NV];
        face_flux<NS, 0, R, kStrict>(prim, n3, c, sx, Fp);
        face_flux<NS, 1, R, kStrict>(prim, n3, c, sy, A);      // y face above
        face_flux<NS, 1, R, kStrict>(prim, n3, c - sy, sy, B); // y face below
        if (sizeof(R) == 4) {
            const float cx32 = float(cx), cy32 = float(cy), cz32 = float(cz);
            float rhs[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q) rhs[q] = cx32 * float(Fp[q] - Fm[q]) - cy32 * float(A[q] - B[q]);
            face_flux<NS, 2, R, kStrict>(prim, n3, c, 1, A);     // z face right
            face_flux<NS, 2, R, kStrict>(prim, n3, c - 1, 1, B); // z face left
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                const float r = rhs[q] - cz32 * float(A[q] - B[q]);
                st.cs[q * n3 + c] = st.cs[q * n3 + c] + double(r);
                Fm[q] = Fp[q];
            }
        } else {
            double rhs[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q)
                rhs[q] = cx * (double(Fp[q]) - double(Fm[q])) - cy * (double(A[q]) - double(B[q]));
            face_flux<NS, 2, R, kStrict>(prim, n3, c, 1, A);
            face_flux<NS, 2, R, kStrict>(prim, n3, c - 1, 1, B);
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                const double r = rhs[q] - cz * (double(A[q]) - double(B[q]));
                st.cs[q * n3 + c] = st.cs[q * n3 + c] + r;
                Fm[q] = Fp[q];
            }
        }
    }
}

// Plane-tiled flux divergence and update: the same faces, arithmetic and RHS
// order as k_flux_update (bitwise the same result), with every primitive read
// from HBM once per plane instead of once per stencil point, and the loads of
// the next plane overlapped with the current plane's arithmetic.
//
// A block owns a kTileJ x kTileK tile of (j, k) columns (TileShape) and
// marches along x with kTileJ + 1 warps. Warps 0 .. kTileJ-1 own a row of cells each: every
// thread keeps its column's x-stencil (planes i-1 .. i+2 of every primitive) in
// registers and loads plane i+3 one node ahead. Plane i of the tile plus a
// two-node halo in j and k is staged in shared memory, from which the y- and
// z-face fluxes are formed; two stages alternate, and while plane i is computed
// the halo of plane i+1 (cp.async) and the conserved values of plane i
// (cp.async, read by the update) are in flight. Face indices: sG[q][r] is the y
// face below tile row r (r = kTileJ: above the last row), sQ[q][r][c] the z
// face left of column c.
//
// Each cell warp forms three faces per plane (x, y, z). The edge warp (warp
// kTileJ) owns the first halo row above the tile, which it stages from its
// registers, and forms the two faces a full tile has beyond its cells: the y
// faces above the last row and the z faces right of the last column. No warp
// forms a fourth face, so no warp waits at the plane's barrier for another's
// extra face. Partial tiles: the faces of the valid rows/columns are formed,
// including the one past the last valid row/column.
//
// Tile height: 7 cell rows (8 warps) in FP32; 3 cell rows (4 warps) in FP64,
// whose x-stencil window takes twice the registers, so that two blocks still
// fit per SM (98 KB of shared memory each).
constexpr int kTileK = 32, kTileCols = kTileK + 4;
template <typename R>
struct TileShape {
    static constexpr int J = sizeof(R) == 4 ? 7 : 3; // cell rows
    static constexpr int Warps = J + 1, Rows = J + 4;
    // staged by cp.async: rows 0, 1 and J + 3 over the full width, and the
    // two columns each side of rows 2 .. J + 2 (the cell rows and the edge
    // warp's row)
    static constexpr int Halo = 3 * kTileCols + 4 * (J + 1);
};

template <int NS, typename R>
constexpr size_t tiled_flux_smem_bytes()
{
    constexpr int J = TileShape<R>::J, Rows = TileShape<R>::Rows;
    return sizeof(double) * (NS + 4) * J * kTileK + sizeof(R) * 2 * (7 + NS) * Rows * kTileCols +
           sizeof(R) * (NS + 4) * ((J + 1) * kTileK + J * (kTileK + 1));
}

// Face flux from four consecutive stencil points of the staged plane tile,
// starting at (r, c) and stepping (DR, DC). own: the values of stencil point 2
// when that point is the thread's own node (kept in registers), else null.
template <int NS, int DIR, int DR, int DC, typename R, bool kStrict, bool kOwn>
__device__ __forceinline__ void tile_face_flux(const R (*sP)[TileShape<R>::Rows][kTileCols], int r, int c,
                                               const R *own, R (&F)[NS + 4])
{
    face_ausm<NS, DIR, R, kStrict, R>(
        [&](int f, int p) { return (kOwn && p == 2) ? own[f] : sP[f][r + p * DR][c + p * DC]; }, F);
}

template <int NS, typename R, bool kStrict>
__device__ __forceinline__ void window_face_flux(const R (&w)[4][7 + NS], R (&F)[NS + 4])
{
    face_ausm<NS, 0, R, kStrict, R>([&](int f, int p) { return w[p][f]; }, F);
}

template <int NS, typename R, bool kStrict>
__global__ void __launch_bounds__(kTileK *TileShape<R>::Warps, 2)
    k_flux_update_tiled(const DevGrid g, const DevState st, const R *__restrict__ prim, const double *__restrict__ dt_dev,
                        int ci)
{
    constexpr int NP = 7 + NS, NV = NS + 4;
    constexpr int kTileJ = TileShape<R>::J, kTileWarps = TileShape<R>::Warps, kTileRows = TileShape<R>::Rows;
    constexpr int kTileHalo = TileShape<R>::Halo;
    using Plane = R[NP][kTileRows][kTileCols];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double(*sC)[kTileJ][kTileK] = reinterpret_cast<double(*)[kTileJ][kTileK]>(smem_raw);
    Plane *stage = reinterpret_cast<Plane *>(smem_raw + sizeof(double) * NV * kTileJ * kTileK);
    unsigned char *flux_raw = reinterpret_cast<unsigned char *>(stage + 2);
    R(*sG)[kTileJ + 1][kTileK] = reinterpret_cast<R(*)[kTileJ + 1][kTileK]>(flux_raw);
    R(*sQ)[kTileJ][kTileK + 1] =
        reinterpret_cast<R(*)[kTileJ][kTileK + 1]>(flux_raw + sizeof(R) * NV * (kTileJ + 1) * kTileK);

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTileK + tx;
    const int k0 = blockIdx.x * kTileK, j0 = blockIdx.y * kTileJ;
    const int k = g.bc + k0 + tx, j = g.bc + j0 + ty;
    const int rows = min(kTileJ, g.nj - j0), cols = min(kTileK, g.nk - k0); // valid rows / columns
    const bool valid = ty < rows && tx < cols;
    const bool resident = j < g.ny && k < g.nz; // inside the haloed arrays: staged for the neighbours
    // faces this thread forms (see above); the y face above a full tile's
    // last row is the edge warp's (ty == rows == kTileJ)
    const bool yface = tx < cols && ty <= rows;
    const bool zface = ty < rows && tx <= cols;
    const int zrow = tx; // lanes 0..kTileJ-1 of the edge warp: the z face right of the last column
    const bool zright = ty == kTileJ && zrow < rows && cols == kTileK;

    // the halo cell this thread stages, if any (counted from the last thread,
    // so the edge warp, which forms fewer faces, takes the first share)
    int hr = -1, hc = 0;
    {
        const int h = kTileWarps * kTileK - 1 - tid;
        if (h < 3 * kTileCols) {
            const int band = h / kTileCols;
            hr = band < 2 ? band : kTileJ + 3;
            hc = h % kTileCols;
        } else if (h < kTileHalo) {
            const int e = h - 3 * kTileCols, side = e % 4;
            hr = 2 + e / 4;
            hc = side < 2 ? side : kTileK + side;
        }
    }
    const int hj = g.bc + j0 - 2 + hr, hk = g.bc + k0 - 2 + hc;
    const bool halo = hr >= 0 && hj < g.ny && hk < g.nz;

    const long long n3 = g.n3, sx = (long long)g.ny * g.nz;
    const double dt = *dt_dev;
    const double cy = valid ? dt / (g.y[j] - g.y[j - 1]) : 0.0;
    const double cz = valid ? dt / (g.z[k] - g.z[k - 1]) : 0.0;
    const int i_begin = g.bc + blockIdx.z * ci;
    const int i_end = min(i_begin + ci, g.bc + g.ni);
    const long long col = resident ? cell_index(g, 0, j, k) : 0;
    const long long hcol = halo ? cell_index(g, 0, hj, hk) : 0;

    // plane p of the tile into stage s: the own node from registers, the halo
    // node by cp.async; one commit group per call (empty when nothing to copy)
    auto stage_plane = [&](int p, const R(&own)[NP], int s) {
        if (resident) {
#pragma unroll
            for (int f = 0; f < NP; ++f) stage[s][f][ty + 2][tx + 2] = own[f];
        }
        if (halo) {
#pragma unroll
            for (int f = 0; f < NP; ++f) {
                if constexpr (sizeof(R) == 4)
                    tc::cp_async4(&stage[s][f][hr][hc], prim + f * n3 + hcol + p * sx);
                else
                    tc::cp_async8(&stage[s][f][hr][hc], prim + f * n3 + hcol + p * sx);
            }
        }
        tc::cp_async_commit();
    };

    R w[4][NP];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int f = 0; f < NP; ++f) w[p][f] = resident ? __ldg(prim + f * n3 + col + (i_begin - 2 + p) * sx) : R(0);
    R Fm[NV];
    if (valid)
        window_face_flux<NS, R, kStrict>(w, Fm);
#pragma unroll
    for (int f = 0; f < NP; ++f) {
        w[0][f] = w[1][f];
        w[1][f] = w[2][f];
        w[2][f] = w[3][f];
        w[3][f] = resident ? __ldg(prim + f * n3 + col + (i_begin + 2) * sx) : R(0);
    }
    stage_plane(i_begin, w[1], 0);

    for (int i = i_begin; i < i_end; ++i) {
        // window: planes i-1, i, i+1, i+2. Stage s holds plane i (its halo may
        // still be in flight); the other stage was last read before the
        // previous iteration's second barrier.
        const int s = (i - i_begin) & 1;
        if (valid) {
#pragma unroll
            for (int q = 0; q < NV; ++q) tc::cp_async8(&sC[q][ty][tx], st.cs + q * n3 + col + i * sx);
        }
        tc::cp_async_commit();
        if (i + 1 < i_end)
            stage_plane(i + 1, w[2], s ^ 1);
        else
            tc::cp_async_commit();
        R next[NP];
        const bool more = resident && i + 1 < i_end;
#pragma unroll
        for (int f = 0; f < NP; ++f) next[f] = more ? __ldg(prim + f * n3 + col + (i + 3) * sx) : R(0);
        // groups in flight, oldest first: halo(i), conserved(i), halo(i+1)
        tc::cp_async_wait<2>();
        __syncthreads();
        R Fp[NV];
        if (valid)
            window_face_flux<NS, R, kStrict>(w, Fp);
        if (yface) {
            R G[NV];
            tile_face_flux<NS, 1, 1, 0, R, kStrict, true>(stage[s], ty, tx + 2, w[1], G);
#pragma unroll
            for (int q = 0; q < NV; ++q) sG[q][ty][tx] = G[q];
        }
        if (zface) {
            R Q[NV];
            tile_face_flux<NS, 2, 0, 1, R, kStrict, true>(stage[s], ty + 2, tx, w[1], Q);
#pragma unroll
            for (int q = 0; q < NV; ++q) sQ[q][ty][tx] = Q[q];
        }
        if (zright) {
            R Q[NV];
            tile_face_flux<NS, 2, 0, 1, R, kStrict, false>(stage[s], zrow + 2, kTileK, nullptr, Q);
#pragma unroll
            for (int q = 0; q < NV; ++q) sQ[q][zrow][kTileK] = Q[q];
        }
        __syncthreads();
        tc::cp_async_wait<1>(); // this thread's conserved values of plane i
        if (valid) {
            const long long c = col + i * sx;
            const double cx = -dt / (g.x[i] - g.x[i - 1]);
            if (sizeof(R) == 4) {
                // FP32 fluxes: the flux differences and their sum in FP32 (a
                // difference of two FP32 values within a factor of two is exact),
                // accumulated onto the FP64 conserved value
                const float cx32 = float(cx), cy32 = float(cy), cz32 = float(cz);
#pragma unroll
                for (int q = 0; q < NV; ++q) {
                    const float rhs = cx32 * float(Fp[q] - Fm[q]) - cy32 * float(sG[q][ty + 1][tx] - sG[q][ty][tx]) -
                                      cz32 * float(sQ[q][ty][tx + 1] - sQ[q][ty][tx]);
                    st.cs[q * n3 + c] = sC[q][ty][tx] + double(rhs);
                    Fm[q] = Fp[q];
                }
            } else {
#pragma unroll
                for (int q = 0; q < NV; ++q) {
                    const double rhs = cx * (double(Fp[q]) - double(Fm[q])) -
                                       cy * (double(sG[q][ty + 1][tx]) - double(sG[q][ty][tx])) -
                                       cz * (double(sQ[q][ty][tx + 1]) - double(sQ[q][ty][tx]));
                    st.cs[q * n3 + c] = sC[q][ty][tx] + rhs;
                    Fm[q] = Fp[q];
                }
            }
        }
#pragma unroll
        for (int f = 0; f < NP; ++f) {
            w[0][f] = w[1][f];
            w[1][f] = w[2][f];
            w[2][f] = w[3][f];
            w[3][f] = next[f];
        }
    }
    tc::cp_async_wait<0>();
}

// ------------------------------------------------- recovery + kinetics

// kWriteCs false: the conserved planes are unchanged (recovery alone reads
// them and changes nothing there), so they are not written back.
// tcache: the recovery's thermo sums for this state, or null.
template <int NS, bool kWriteCs = true>
__device__ __forceinline__ void store_cell(const DevMech &m, const DevState &st, long long n3, long long c,
                                           const CellState<NS> &cell, const ThermoCache<NS> *tcache = nullptr)
{
    double P, H, G;
    finish_primitives<NS>(m, cell, tcache, P, H, G);
    const double v[7] = {P, cell.D, cell.U, cell.V, cell.W, H, G};
    if (st.prim32) { // mixed precision: the FP64 planes are formed on demand (k_materialize)
#pragma unroll
        for (int f = 0; f < 7; ++f) st.prim32[f * n3 + c] = float(v[f]);
#pragma unroll
        for (int s = 0; s < NS; ++s) st.prim32[(kY0 + s) * n3 + c] = float(cell.Y[s]);
    } else {
#pragma unroll
        for (int f = 0; f < 7; ++f) st.prim[f * n3 + c] = v[f];
#pragma unroll
        for (int s = 0; s < NS; ++s) st.prim[(kY0 + s) * n3 + c] = cell.Y[s];
    }
    if (kWriteCs) {
#pragma unroll
        for (int q = 0; q < NS + 4; ++q) st.cs[q * n3 + c] = cell.cs[q];
    }
    st.T[c] = cell.T;
    st.E[c] = cell.E;
    if (!(isfinite(cell.D) && isfinite(cell.T)))
        atomicAdd(&st.counters[kCntNonfinite], 1ULL);
    if (st.zm_fresh) {
        // EU_GHOSTS_STORED: the z-face ghosts this node is the mirror source
        // of (k_boundary's z faces: ghost 2 bc - 1 - k below, 2 (nk + bc) - 1 -
        // k above, W reflected), the values the ghost fill would copy, in the
        // same 32-byte sectors as the node's own stores
        const long long row = fdiv(c, st.zm_dnz);
        const int k = int(c - row * st.zm_nz), bc = st.zm_bc, nk = st.zm_nk;
        auto mirror = [&](long long gc) {
            if (st.prim32) {
#pragma unroll
                for (int f = 0; f < 7; ++f) st.prim32[f * n3 + gc] = float(f == kW ? -v[f] : v[f]);
#pragma unroll
                for (int s = 0; s < NS; ++s) st.prim32[(kY0 + s) * n3 + gc] = float(cell.Y[s]);
            } else {
#pragma unroll
                for (int f = 0; f < 7; ++f) st.prim[f * n3 + gc] = f == kW ? -v[f] : v[f];
#pragma unroll
                for (int s = 0; s < NS; ++s) st.prim[(kY0 + s) * n3 + gc] = cell.Y[s];
            }
            st.T[gc] = cell.T;
        };
        if (k < 2 * bc)
            mirror(c + (2 * bc - 1 - 2 * k));
        if (k >= nk)
            mirror(c + (2 * (nk + bc) - 1 - 2 * k));
    }
}

// EU_GHOSTS_STORED: a recovery that stores every interior node has written
// every z-face ghost, so the next ghost fill (after it in stream order) may
// skip the z faces.
__device__ __forceinline__ void mark_z_fresh(const DevState &st)
{
    if (st.zm_fresh && blockIdx.x == 0 && threadIdx.x == 0)
        *st.zm_fresh = 1;
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

// Nchem prediction (Reaction::TrapezoidPrediction, src/Reaction.cpp:865-942)
// and the Nchem trapezoid substeps with state recovery after each
// (src/Euler.cpp:462-493, src/Reaction.cpp:562-805, src/Flowfield.cpp:1521-1536)
// on a recovered cell state. The prediction's rate evaluation is reused by
// the first substep: both evaluate the same expression on the same state.
// Returns Nchem; a prediction <= 0 or above max_substeps is counted as an error.
// Nchem = ceil(dtm / min_s |Di_s / Wi_s|) over species with Y_s >= 1e-6
// (src/Reaction.cpp:919-940); a prediction <= 0 or above max_substeps is
// counted as an error and gives 0 or max_substeps.
__device__ __forceinline__ int nchem_from_dt(double dtm, double dt, int max_substeps, unsigned long long *counters)
{
    const double ratio = ceil(dtm / dt);
    if (!(ratio >= 1.0) || ratio > double(max_substeps)) {
        atomicAdd(&counters[kCntBadNchem], 1ULL);
        return (ratio > double(max_substeps)) ? max_substeps : 0;
    }
    return int(ratio);
}

__device__ __forceinline__ void count_nchem(unsigned long long *counters, int nchem)
{
    if (nchem > 0) {
        atomicMax(&counters[kCntMaxNchem], (unsigned long long)nchem);
        atomicAdd(&counters[kCntSumNchem], (unsigned long long)nchem);
    }
}

// The prediction: start-of-step rates (kept in `rates` for the first substep)
// and Nchem.
template <int NS, class Rt>
__device__ __forceinline__ int predict_nchem(const DevMech &m, const CellState<NS> &cell, double dtm,
                                             int max_substeps, unsigned long long *counters, double (&mc)[NS],
                                             SpeciesRates<NS> &rates)
{
    scaled_concentrations<NS>(m, cell, mc);
    Rt::rates(m, cell.T, mc, rates);
    double dt = dtm;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        // formed for every species, then chosen: a select instead of a branch
        // that the cells diverge on
        const double dt_temp = fabs(-(cell.cs[s] * 1e-3) / rates.W[s]);
        dt = (cell.Y[s] >= 1e-6 && rates.W[s] != 0 && dt_temp < dt) ? dt_temp : dt;
    }
    return nchem_from_dt(dtm, dt, max_substeps, counters);
}

// The Nchem substeps, the first one on the prediction's rates.
template <int NS, class Rt>
__device__ __forceinline__ void run_substeps(const DevMech &m, CellState<NS> &cell, double dtm, int nchem,
                                             double (&mc)[NS], SpeciesRates<NS> &rates, double *cms,
                                             long long cms_stride)
{
    const double dts = dtm / nchem;
    for (int step = 0; step < nchem; ++step) {
        if (step > 0) {
            scaled_concentrations<NS>(m, cell, mc);
            Rt::rates(m, cell.T, mc, rates);
        }
        if (cms) {
#pragma unroll
            for (int s = 0; s < NS; ++s) cms[s * cms_stride] = rates.W[s] * 1e3;
        }
        trapezoid_substep<NS>(m, rates, dts, mc, cell);
    }
}

template <int NS, class Rt>
__device__ __forceinline__ int react_cell(const DevMech &m, CellState<NS> &cell, double dtm, int max_substeps,
                                          unsigned long long *counters, double *cms, long long cms_stride)
{
    double mc[NS];
    SpeciesRates<NS> rates;
    const int nchem = predict_nchem<NS, Rt>(m, cell, dtm, max_substeps, counters, mc, rates);
    count_nchem(counters, nchem);
    run_substeps<NS, Rt>(m, cell, dtm, nchem, mc, rates, cms, cms_stride);
    return nchem;
}

// Cells whose predicted Nchem exceeds kHeavyNchem are, in the mixed-precision
// flavour (EU_HEAVY_QUEUE), deferred to k_react_heavy: one warp per cell
// instead of one thread, so the long serial substep chains of igniting cells
// do not set the step's time. st.heavy = {count, next, cells...}. On the
// 48x32x32 igniting block the step takes 0.865 / 0.81 / 0.764 / 0.78 / 1.11 ms
// with the threshold at 16 / 8 / 4 / 2 / 0: below 4 a warp per cell costs more
// than the few substeps it shortens.
constexpr int kHeavyNchem = 4;

__device__ __forceinline__ void push_heavy(int *heavy, long long c)
{
    const int q = atomicAdd(&heavy[0], 1);
    heavy[2 + q] = int(c);
}

// React one recovered cell, or (mixed flavour, heavy queue present) defer it
// when its Nchem is large. Returns false when deferred.
template <int NS, class Rt>
__device__ __forceinline__ bool react_or_defer(const DevMech &m, const DevState &st, long long n3, long long c,
                                               CellState<NS> &cell, double dtm, int max_substeps)
{
    double mc[NS];
    SpeciesRates<NS> rates;
    const int nchem = predict_nchem<NS, Rt>(m, cell, dtm, max_substeps, st.counters, mc, rates);
#ifdef EU_HEAVY_QUEUE
    if (st.heavy && nchem > kHeavyNchem) {
        push_heavy(st.heavy, c);
        return false;
    }
#endif
    count_nchem(st.counters, nchem);
    run_substeps<NS, Rt>(m, cell, dtm, nchem, mc, rates, st.cms ? st.cms + c : nullptr, n3);
    st.nchem[c] = nchem;
    return true;
}

template <int NS>
__device__ __forceinline__ void load_cell(const DevState &st, long long n3, long long c, CellState<NS> &cell)
{
#pragma unroll
    for (int q = 0; q < NS + 4; ++q) cell.cs[q] = st.cs[q * n3 + c];
    cell.T = st.T[c];
    cell.E = st.E[c];
}

// The recovered state of a cell whose recovery already ran and was stored:
// D, Y, u, v, w are re-formed from CS with the expressions of recover_state
// (same values), T and E are the stored ones.
template <int NS>
__device__ __forceinline__ void load_recovered(const DevState &st, long long n3, long long c, CellState<NS> &cell)
{
    load_cell<NS>(st, n3, c, cell);
    double D = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) D += cell.cs[s];
    cell.D = D;
#ifdef EU_EXACT_CHEM
#pragma unroll
    for (int s = 0; s < NS; ++s) cell.Y[s] = cell.cs[s] / D;
    cell.U = cell.cs[NS + 0] / D;
    cell.V = cell.cs[NS + 1] / D;
    cell.W = cell.cs[NS + 2] / D;
#else
    const double invD = rcp_nr(D);
#pragma unroll
    for (int s = 0; s < NS; ++s) cell.Y[s] = cell.cs[s] * invD;
    cell.U = cell.cs[NS + 0] * invD;
    cell.V = cell.cs[NS + 1] * invD;
    cell.W = cell.cs[NS + 2] * invD;
#endif
}

// Mixed precision keeps the FP64 primitive planes out of the timestep (the
// FP32 planes feed the fluxes). This forms them on demand, for output: interior
// nodes from the stored conserved state, T and E (the values the FP64 store
// would have written), ghost nodes from the FP32 ghost planes.
template <int NS>
__global__ void __launch_bounds__(128) k_materialize(const __grid_constant__ DevMech m, const DevGrid g,
                                                     const DevState st)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.n3)
        return;
    const long long n3 = g.n3;
    const int jk = fdiv(c, g.d_nz), i = fdiv(c, g.d_nynz);
    const int k = int(c - (long long)jk * g.nz), j = jk - i * g.ny;
    const bool interior = i >= g.bc && i < g.bc + g.ni && j >= g.bc && j < g.bc + g.nj && k >= g.bc &&
                          k < g.bc + g.nk;
    if (!interior) {
#pragma unroll
        for (int f = 0; f < 7 + NS; ++f) st.prim[f * n3 + c] = double(st.prim32[f * n3 + c]);
        return;
    }
    CellState<NS> cell;
    load_recovered<NS>(st, n3, c, cell);
    double P, H, G;
    finish_primitives<NS>(m, cell, P, H, G);
    const double v[7] = {P, cell.D, cell.U, cell.V, cell.W, H, G};
#pragma unroll
    for (int f = 0; f < 7; ++f) st.prim[f * n3 + c] = v[f];
#pragma unroll
    for (int s = 0; s < NS; ++s) st.prim[(kY0 + s) * n3 + c] = cell.Y[s];
}

// FP32 copy of the FP64 primitive planes (state upload in mixed precision).
__global__ void k_to_f32(const double *__restrict__ src, float *__restrict__ dst, long long n)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        dst[t] = float(src[t]);
}

// Post-advection state recovery (Flowfield::Update_after_Adv ->
// Update_after_CS, src/Flowfield.cpp:1579-1617) followed, in the stiff modes,
// by the kinetics of react_cell. One thread per interior node.
// MINB: resident 128-thread blocks per SM the register allocation aims at
// (2: no spills, 8 warps; 3 and 4 trade spills for warps; the autotuner picks).
template <int NS, int NR, bool kReact, class Rt, int MINB = 2>
__global__ void __launch_bounds__(128, MINB) k_recover_react(const __grid_constant__ DevMech m, const DevGrid g,
                                                       const DevState st, const double *__restrict__ dt_dev,
                                                       int max_substeps)
{
    const long long ncell = (long long)g.ni * g.nj * g.nk;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    mark_z_fresh(st);
    if (t >= ncell)
        return;
    int i, j, k;
    interior_node(g, t, i, j, k);
    const long long n3 = g.n3;
    const long long c = cell_index(g, i, j, k);
    CellState<NS> cell;
    load_cell<NS>(st, n3, c, cell);
    if (!kReact) {
        ThermoCache<NS> tcache;
        recover_state<NS>(m, cell, tcache);
        store_cell<NS, false>(m, st, n3, c, cell, &tcache);
        return;
    }
    recover_state<NS>(m, cell);
    if (kReact) {
        if (!react_or_defer<NS, Rt>(m, st, n3, c, cell, *dt_dev, max_substeps)) {
            store_cell<NS, false>(m, st, n3, c, cell); // recovered state for k_react_heavy
            return;
        }
    }
    store_cell<NS, kReact>(m, st, n3, c, cell);
}

// ------------------------------------------------- learned chemistry

// Post-advection recovery of every cell; cells with chemistry to do are
// appended to the learned queue (warp-aggregated atomics), the others are
// final. Every cell's recovered state is stored.
// MINB: resident blocks per SM the register allocation aims at (the
// autotuner picks the instantiation; fewer registers, more warps, some spills).
template <int NS, int MINB = 4>
__global__ void __launch_bounds__(128, MINB) k_recover_classify(const __grid_constant__ DevMech m, const DevGrid g,
                                                          const DevState st, LearnedParams lp)
{
    const long long ncell = (long long)g.ni * g.nj * g.nk;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    mark_z_fresh(st);
    bool active = false;
    long long c = 0;
    if (t < ncell) {
        int i, j, k;
        interior_node(g, t, i, j, k);
        const long long n3 = g.n3;
        c = cell_index(g, i, j, k);
        CellState<NS> cell;
        load_cell<NS>(st, n3, c, cell);
        ThermoCache<NS> tcache;
        recover_state<NS>(m, cell, tcache);
        store_cell<NS, false>(m, st, n3, c, cell, &tcache);
        double reactive = 0, radical = 0;
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            if (!lp.inert[s])
                reactive += cell.Y[s];
            if (lp.radical[s])
                radical += cell.Y[s];
        }
        active = reactive >= lp.frozen_y && !(cell.T < lp.frozen_T && radical < lp.frozen_radical);
        st.nchem[c] = 0;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, active);
    if (mask) {
        const int lane = threadIdx.x & 31;
        int base = 0;
        if (lane == __ffs(mask) - 1)
            base = atomicAdd(&lp.counts[0], __popc(mask));
        base = __shfl_sync(0xffffffffu, base, __ffs(mask) - 1);
        if (active)
            lp.queue[base + __popc(mask & ((1u << lane) - 1))] = int(c);
    }
}

// Model inputs of the queued cells: T, log10 p, Y_0..Y_{NS-1}, log10 dt, with
// p = rho R T and R = 8314.34 / Wav (Update_after_CS, src/Flowfield.cpp:1606-1608).
template <int NS>
__global__ void k_learned_features(const __grid_constant__ DevMech m, const DevGrid g, const DevState st,
                                   LearnedParams lp, const double *__restrict__ dt_dev)
{
    // a fixed grid walks the queue (its length is read on the device)
    const int nq = lp.counts[0];
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        const long long n3 = g.n3, c = lp.queue[q];
        CellState<NS> cell;
        load_recovered<NS>(st, n3, c, cell);
        float *f = lp.feat + (long long)q * (NS + 3);
        double inv_w = 0;
#pragma unroll
        for (int s = 0; s < NS; ++s) inv_w += cell.Y[s] / m.mw[s];
        f[0] = float(cell.T);
        f[1] = float(log10(cell.T * cell.D * (kRUniv * 1000 * inv_w)));
#pragma unroll
        for (int s = 0; s < NS; ++s) f[2 + s] = float(cell.Y[s]);
        f[NS + 2] = float(log10(*dt_dev));
    }
}

// Apply the ensemble's prediction to each queued cell, or send it to the stiff
// fallback queue. Accepted when every input lies in the trained box and the
// members' spread (largest per-output standard deviation, in output-scale
// units) is below tau. The mean species change is projected onto element
// conservation (which implies sum Y = 1), clipped at zero and renormalised;
// density, momentum and internal energy are held (the reference's chemistry
// changes only the species densities); T is re-solved by the Newton inversion
// from the predicted T.
template <int NS>
__global__ void __launch_bounds__(128) k_learned_apply(const __grid_constant__ DevMech m, const DevGrid g,
                                                       const DevState st, LearnedParams lp)
{
    // a fixed grid walks the queue in whole warps (the fallback append is
    // warp-aggregated)
    const int nq = lp.counts[0];
    const int stride = gridDim.x * blockDim.x;
    const int span = (nq + 31) / 32 * 32;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < span; q += stride) {
        bool fallback = false;
        int c = 0;
        if (q < nq) {
            const long long n3 = g.n3;
            c = lp.queue[q];
            const float *f = lp.feat + (long long)q * (NS + 3);
            bool ok = true;
#pragma unroll
            for (int a = 0; a < NS + 3; ++a) ok = ok && f[a] >= float(lp.box_lo[a]) && f[a] <= float(lp.box_hi[a]);
            double mean[NS + 1], spread = 0;
#pragma unroll
            for (int o = 0; o < NS + 1; ++o) {
                double s1 = 0, s2 = 0;
                for (int e = 0; e < lp.members; ++e) {
                    const double v = lp.pred[(long long)q * lp.pred_row + (long long)e * lp.pred_mem + o];
                    s1 += v;
                    s2 += v * v;
                }
                const double mu = s1 / lp.members;
                const double var = fmax(s2 / lp.members - mu * mu, 0.0);
                // spread and mean in the model's output space, the change back in physical units
                spread = fmax(spread, sqrt(var) * lp.out_scale[o]);
                mean[o] = lp.out_eps[o] > 0 ? lp.out_eps[o] * sinh(mu) : mu;
                ok = ok && (lp.out_bound[o] <= 0 || fabs(mean[o]) <= lp.out_bound[o]);
            }
            ok = ok && spread <= lp.tau && isfinite(spread);
            if (ok) {
                CellState<NS> cell;
                load_recovered<NS>(st, n3, c, cell);
                double dY[NS], Y[NS], sum = 0;
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    double d = 0;
#pragma unroll
                    for (int r = 0; r < NS; ++r) d += lp.proj[s][r] * mean[r];
                    dY[s] = d;
                }
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    Y[s] = fmax(cell.Y[s] + dY[s], 0.0);
                    sum += Y[s];
                }
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    cell.Y[s] = Y[s] / sum;
                    cell.cs[s] = cell.D * cell.Y[s];
                }
                cell.T = newton_temperature<NS>(m, cell.T + mean[NS], cell.E, cell.Y);
                store_cell<NS>(m, st, n3, c, cell);
                atomicAdd(&st.counters[kCntLearned], 1ULL);
            } else {
                fallback = true;
            }
        }
        const unsigned mask = __ballot_sync(0xffffffffu, fallback);
        if (mask) {
            const int lane = threadIdx.x & 31;
            int base = 0;
            if (lane == __ffs(mask) - 1)
                base = atomicAdd(&lp.counts[1], __popc(mask));
            base = __shfl_sync(0xffffffffu, base, __ffs(mask) - 1);
            if (fallback)
                lp.fallback[base + __popc(mask & ((1u << lane) - 1))] = c;
        }
    }
}

// The stiff kinetics of one queued cell whose recovered state is stored.
template <int NS, class Rt>
__device__ __forceinline__ void react_queued(const DevMech &m, const DevState &st, long long n3, long long c,
                                             double dtm, int max_substeps, int counter)
{
    CellState<NS> cell;
    load_recovered<NS>(st, n3, c, cell);
    atomicAdd(&st.counters[counter], 1ULL);
    if (react_or_defer<NS, Rt>(m, st, n3, c, cell, dtm, max_substeps))
        store_cell<NS>(m, st, n3, c, cell);
}

// Position `pos` of the batch's queues taken end to end: the instance holding
// it and the position within that instance's queue (lengths from len(q)).
template <class Len>
__device__ __forceinline__ int batch_locate(int n, int pos, Len len, int &local)
{
    int q = 0, off = 0;
    for (; q < n; ++q) {
        const int l = len(q);
        if (pos < off + l)
            break;
        off += l;
    }
    local = pos - off;
    return q;
}

// The stiff-fallback queues of every instance of a batch drained by one fixed
// grid: warps take 32 positions at a time from one counter over the queues
// taken end to end (the shared reacting-cell work queue), so the cells of all
// instances are spread over the whole GPU. Per cell the same work as
// k_react_queue; every instance's statistics go to its own counters.
template <int NS, class Rt>
__global__ void __launch_bounds__(128) k_react_queue_batch(const __grid_constant__ DevMech m,
                                                           const BatchCell *__restrict__ tab, int n, int *next,
                                                           int max_substeps, int counter)
{
    auto len = [&](int q) { return tab[q].count ? *(volatile const int *)tab[q].count : 0; };
    int total = 0;
    for (int q = 0; q < n; ++q) total += len(q);
    if (total == 0)
        return;
    const int lane = threadIdx.x & 31;
    for (;;) {
        int base = 0;
        if (lane == 0)
            base = atomicAdd(next, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total)
            break;
        const int pos = base + lane;
        if (pos < total) {
            int local = 0;
            const int q = batch_locate(n, pos, len, local);
            if (q < n) {
                const BatchCell &b = tab[q];
                react_queued<NS, Rt>(m, b.st, b.n3, b.queue[local], *b.dt, max_substeps, counter);
            }
        }
    }
}

// The stiff kinetics on a queue of cells whose recovered state is stored.
template <int NS, class Rt>
__global__ void __launch_bounds__(128) k_react_queue(const __grid_constant__ DevMech m, const DevGrid g,
                                                     const DevState st, const int *__restrict__ queue, int *count,
                                                     const double *__restrict__ dt_dev, int max_substeps, int counter)
{
    // A fixed grid drains the queue (its length is read on the device): each
    // warp takes the next 32 cells from count[1] (reset before the launch).
    const int nq = *(volatile int *)count;
    if (nq == 0) // an empty queue: no warp touches the shared counter
        return;
    const int lane = threadIdx.x & 31;
    int *next = count + 1;
    for (;;) {
        int base = 0;
        if (lane == 0)
            base = atomicAdd(next, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= nq)
            break;
        const int q = base + lane;
        if (q < nq)
            react_queued<NS, Rt>(m, st, g.n3, queue[q], *dt_dev, max_substeps, counter);
    }
}

// Nchem routing of the learned mode: each active cell's Nchem is predicted
// (Reaction::TrapezoidPrediction, src/Reaction.cpp:865-942); a cell needing at
// most lp.min_nchem substeps takes the stiff kinetics here (its substeps cost
// less than the model's evaluation and carry no model error), the others are
// appended to the model's queue (lp.queue, length lp.counts[0]). With
// lp.min_nchem <= 0 every active cell goes to the model unpredicted. A fixed
// grid drains the active queue (length lp.counts[3], warp grabs on counts[4]).
template <int NS, class Rt>
__global__ void __launch_bounds__(128) k_learned_route(const __grid_constant__ DevMech m, const DevGrid g,
                                                       const DevState st, LearnedParams lp,
                                                       const double *__restrict__ dt_dev, int max_substeps)
{
    const int nq = *(volatile int *)(lp.counts + 3);
    if (nq == 0)
        return;
    const int lane = threadIdx.x & 31;
    const long long n3 = g.n3;
    for (;;) {
        int base = 0;
        if (lane == 0)
            base = atomicAdd(lp.counts + 4, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= nq)
            break;
        const int q = base + lane;
        bool to_model = false;
        long long c = 0;
        if (q < nq) {
            c = lp.active[q];
            to_model = true;
            if (lp.min_nchem > 0) {
                CellState<NS> cell;
                load_recovered<NS>(st, n3, c, cell);
                double mc[NS];
                SpeciesRates<NS> rates;
                const double dtm = *dt_dev;
                const int nchem = predict_nchem<NS, Rt>(m, cell, dtm, max_substeps, st.counters, mc, rates);
                if (nchem <= lp.min_nchem) {
                    to_model = false;
#ifdef EU_HEAVY_QUEUE
                    if (st.heavy && nchem > kHeavyNchem) {
                        push_heavy(st.heavy, c);
                    } else
#endif
                    {
                        count_nchem(st.counters, nchem);
                        run_substeps<NS, Rt>(m, cell, dtm, nchem, mc, rates, st.cms ? st.cms + c : nullptr, n3);
                        st.nchem[c] = nchem;
                        store_cell<NS>(m, st, n3, c, cell);
                    }
                }
            }
        }
        const unsigned routed = __ballot_sync(0xffffffffu, q < nq && !to_model);
        if (routed && lane == __ffs(routed) - 1)
            atomicAdd(&st.counters[kCntRouted], (unsigned long long)__popc(routed));
        const unsigned mask = __ballot_sync(0xffffffffu, to_model);
        if (mask) {
            int at = 0;
            if (lane == __ffs(mask) - 1)
                at = atomicAdd(&lp.counts[0], __popc(mask));
            at = __shfl_sync(0xffffffffu, at, __ffs(mask) - 1);
            if (to_model)
                lp.queue[at + __popc(mask & ((1u << lane) - 1))] = int(c);
        }
    }
}

// ------------------------------------------------- warp-per-cell kinetics
// The same kinetics as react_cell (prediction, Nchem trapezoid substeps,
// state rebuild after each) with one warp per cell: lane r evaluates reaction
// r, lane s owns species s's sums and trapezoid update, and every lane keeps
// the whole cell state (the rebuild runs redundantly on all lanes). The sums
// run in the same order as the one-thread form. Tables that lanes index by
// reaction or species are read from a shared-memory copy of the mechanism;
// the uniform reads of the state rebuild stay on the kernel parameter.

template <int NS>
__device__ __forceinline__ double lane_pick(const double (&v)[NS], int lane)
{
    double r = 0.0;
#pragma unroll
    for (int s = 0; s < NS; ++s) r = (lane == s) ? v[s] : r;
    return r;
}

// Per-lane constants of the warp-per-cell kinetics, read once per warp from
// the mechanism tables: lane r's reaction (r < NR; others repeat reaction 0)
// and lane s's species (s < NS; others repeat species 0).
template <int NS, int NR>
struct HeavyLane {
    double af, bf, eaf, xr, mw;
};

template <int NS, int NR>
__device__ __forceinline__ HeavyLane<NS, NR> heavy_lane(const DevMech &m, int lane)
{
    static_assert(NR <= 32 && NS <= 32, "one lane per reaction and per species");
    HeavyLane<NS, NR> h;
    const int r = lane < NR ? lane : 0, sl = lane < NS ? lane : 0;
    h.af = m.af[r];
    h.bf = m.bf[r];
    h.eaf = m.eaf[r];
    h.xr = m.xr[r];
    h.mw = m.mw[sl];
    return h;
}

// The mechanism's sparse structure for the warp-per-cell kinetics, built once
// per block, every array [entry][lane] so that a warp reads 32 consecutive
// elements. Lane r's reaction (lanes past NR repeat reaction 0) lists the
// species it involves, ascending: rent = s | nu' << 4 | nu'' << 6, then
// entries with nu' = nu'' = 0 (factors of exactly 1). Lane s's species (lanes
// past NS repeat species 0) lists the reactions it takes part in, ascending:
// sent = q with its coefficients as doubles in sbv, sfv, then entries of
// reaction slot 31, whose rates are zero (addends of exactly 0). So the
// loops run a fixed count without branches and the products and sums are
// the per-thread form's, whose other terms are factors of 1 and addends of
// 0. tb: third-body efficiencies [s][r]; imw: 1e-3 / W_s.
template <int NS, int NR>
struct HeavyTablesT {
    static_assert(NR < 32, "slot 31 holds zero rates");
    double tb[NS][32];
    double sbv[NR][32], sfv[NR][32];
    double imw[NS];
    unsigned char rent[NS][32], sent[NR][32];
};

// A warp's exchange buffers in shared memory: the species' exp(g) and
// exp(-g), the reactions' forward and backward rates and third-body sums.
struct HeavyScratch {
    double eg[32], ieg[32], fwd[32], bwd[32], rtb[32], mc[32];
};

// Fast-form rates (the mixed flavour's eval_rates) across a warp. On return
// lane s < NS holds P_s, Q_s and W_s (W with the molecular weight applied).
// The species' Gibbs exponentials and the reactions' rates change hands
// through the warp's shared buffers (one store each, broadcast loads); a
// reaction lane reads its coefficients from the transposed tables (tt), a
// species lane from the mechanism's (ms): the arithmetic and its order are
// the per-thread form's. inv, lnT: 1/T and log T (carried from the last
// rebuild's Newton).
template <int NS, int NR>
__device__ __forceinline__ void warp_rates(const DevMech &ms, const HeavyLane<NS, NR> &hl,
                                           const HeavyTablesT<NS, NR> &tt, HeavyScratch &x, double T, double inv,
                                           double lnT, const double (&mc)[NS], int lane, double &Pl, double &Ql,
                                           double &Wl)
{
    const TPow p = make_tpow_known(T, inv, lnT);
    const double invRT = inv * (1.0 / kRUniv);
    const int sl = lane < NS ? lane : 0;
    const double egl = exp((h_species<NS>(ms, p, kRUniv, sl) - s_species<NS>(ms, p, kRUniv, sl) * T) * invRT);
    x.eg[lane] = egl;
    x.ieg[lane] = rcp_nr(egl);
    x.mc[lane] = lane_pick<NS>(mc, sl);
    const double invRuT = inv * (1.0 / kRuCal);
    const double rt_p0 = (kRUniv * T) / (kP0 * 1e-6);
    const double p0_rt = rcp_nr(rt_p0);
    double rrf = 1.0, rrb = 1.0, kc_inv = 1.0, rtb = 0.0;
    const double b = hl.bf;
    // Every candidate is formed before it is chosen, so the choices are
    // selects: a conditional whose arms compute is a branch, and the lanes,
    // holding different reactions and species, diverge on it.
    const double kf_exp = hl.af * exp(b * p.lnT - hl.eaf * invRuT);
    double tpow = 1.0;
    tpow = b == 1.0 ? T : tpow;
    tpow = b == -1.0 ? p.inv : tpow;
    tpow = b == -2.0 ? p.inv2 : tpow;
    const double kf_pow = hl.af * tpow;
    const double kf = (hl.eaf == 0.0 && (b == 0.0 || b == 1.0 || b == -1.0 || b == -2.0)) ? kf_pow : kf_exp;
#pragma unroll
    for (int s = 0; s < NS; ++s) rtb += mc[s] * tt.tb[s][lane];
    __syncwarp();
    // a fixed count without branches: every entry's loads issue together
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        const unsigned e = tt.rent[i][lane];
        const int s = int(e & 15u), fi = int((e >> 4) & 3u), bi = int(e >> 6);
        const double m = x.mc[s], eg = x.eg[s], ieg = x.ieg[s];
        const double m2 = m * m, eg2 = eg * eg, ieg2 = ieg * ieg;
        double ff = fi == 1 ? m : 1.0, fb = bi == 1 ? m : 1.0;
        ff = fi == 2 ? m2 : ff;
        fb = bi == 2 ? m2 : fb;
        rrf *= ff;
        rrb *= fb;
        const int d = bi - fi;
        double fk = d == 1 ? eg : 1.0;
        fk = d == -1 ? ieg : fk;
        fk = d == 2 ? eg2 : fk;
        fk = d == -2 ? ieg2 : fk;
        kc_inv *= fk;
    }
    const double Xr = hl.xr;
    kc_inv *= (Xr == 0.0 ? 1.0 : Xr == 1.0 ? rt_p0 : p0_rt);
    if (rtb == 0.0)
        rtb = 1.0;
    const bool real = lane < NR; // slot 31 (and every slot past NR) holds zero rates
    x.fwd[lane] = real ? kf * rrf : 0.0;
    x.bwd[lane] = real ? kf * kc_inv * rrb : 0.0;
    x.rtb[lane] = real ? rtb : 0.0;
    __syncwarp();
    double P = 0.0, Q = 0.0, W = 0.0;
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        const int q = tt.sent[i][lane];
        const double bb = tt.sbv[i][lane], f = tt.sfv[i][lane];
        const double fr = x.fwd[q], br = x.bwd[q], tr = x.rtb[q];
        W += (bb - f) * tr * (fr - br);
        Q += (bb * fr + f * br) * tr;
        P += (bb * br + f * fr) * tr;
    }
    __syncwarp(); // the buffers are free for the next evaluation
    Pl = P;
    Ql = Q;
    Wl = hl.mw * W;
}

// The scaled concentrations of a deferred cell: one multiplication by
// 1e-3 / W_s per species instead of a division (within rounding of
// scaled_concentrations).
template <int NS, int NR>
__device__ __forceinline__ void heavy_concentrations(const DevMech &m, const HeavyTablesT<NS, NR> &tt,
                                                     const CellState<NS> &c, double (&mc)[NS])
{
#ifdef EU_EXACT_CHEM
    scaled_concentrations<NS>(m, c, mc);
#else
#pragma unroll
    for (int s = 0; s < NS; ++s) mc[s] = c.cs[s] * tt.imw[s];
#endif
}

// One deferred cell advanced by a whole warp: lane r evaluates reaction r,
// lane s owns species s's sums and trapezoid update, every lane rebuilds the
// state (ms: the mechanism tables in shared memory; hl, tt, x: see
// warp_rates).
template <int NS, int NR>
__device__ __forceinline__ void react_heavy_cell(const DevMech &m, const DevMech &ms, const HeavyLane<NS, NR> &hl,
                                                 const HeavyTablesT<NS, NR> &tt, HeavyScratch &x, const DevState &st,
                                                 long long n3, long long c, double dtm, int max_substeps, int lane)
{
    CellState<NS> cell;
    load_recovered<NS>(st, n3, c, cell);
    // 1/T and log T of the current temperature, carried through the substeps
    // by the rebuild's Newton
    double inv = rcp_nr(cell.T), lnT = log(cell.T);
    double mc[NS], P, Q, W;
    heavy_concentrations<NS, NR>(m, tt, cell, mc);
    warp_rates<NS, NR>(ms, hl, tt, x, cell.T, inv, lnT, mc, lane, P, Q, W);
    // prediction: min over the species lanes, then every lane has Nchem
    double dt = dtm;
    if (lane < NS && lane_pick<NS>(cell.Y, lane) >= 1e-6 && W != 0)
        dt = fmin(dt, fabs(-(lane_pick<NS + 4>(cell.cs, lane) * 1e-3) / W));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dt = fmin(dt, __shfl_xor_sync(0xffffffffu, dt, o));
    int nchem = 0;
    if (lane == 0) {
        nchem = nchem_from_dt(dtm, dt, max_substeps, st.counters);
        count_nchem(st.counters, nchem);
    }
    nchem = __shfl_sync(0xffffffffu, nchem, 0);
    const double dts = dtm / nchem, half = dts / 2.0;
    for (int step = 0; step < nchem; ++step) {
        if (step > 0) {
            heavy_concentrations<NS, NR>(m, tt, cell, mc);
            warp_rates<NS, NR>(ms, hl, tt, x, cell.T, inv, lnT, mc, lane, P, Q, W);
        }
        if (st.cms && lane < NS)
            st.cms[lane * n3 + c] = W * 1e3;
        double nd = 0.0;
        if (lane < NS) {
            const double di = lane_pick<NS + 4>(cell.cs, lane) * 1e-3;
            const double mcl = lane_pick<NS>(mc, lane);
            const double qv = hl.mw * Q;
#ifdef EU_EXACT_CHEM
            const double pv = (mcl == 0) ? 0.0 : P / mcl;
            nd = ((1.0 - half * pv) * di + dts * qv) / (1.0 + half * pv) * 1e3;
#else
            // refined reciprocals instead of IEEE divisions (1 + half pv >= 1);
            // the reciprocal formed before the choice (a select, not a branch)
            const double pq = P * rcp_nr(mcl);
            const double pv = (mcl == 0) ? 0.0 : pq;
            nd = ((1.0 - half * pv) * di + dts * qv) * rcp_nr(1.0 + half * pv) * 1e3;
#endif
        }
        double D = 0.0;
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            cell.cs[s] = __shfl_sync(0xffffffffu, nd, s);
            D += cell.cs[s];
        }
        cell.cs[NS + 0] = cell.U * D;
        cell.cs[NS + 1] = cell.V * D;
        cell.cs[NS + 2] = cell.W * D;
        cell.cs[NS + 3] = D * cell.E + 0.5 * (cell.U * cell.U + cell.V * cell.V + cell.W * cell.W) * D;
#ifdef EU_EXACT_CHEM
        recover_state<NS>(m, cell);
        inv = 1.0 / cell.T;
        lnT = log(cell.T);
#else
        recover_state_carry<NS>(m, cell, inv, lnT);
#endif
    }
    if (lane == 0) {
        st.nchem[c] = nchem;
        store_cell<NS>(m, st, n3, c, cell);
    }
    __syncwarp();
}

__device__ __forceinline__ void copy_mech_to_shared(const DevMech &m, DevMech &ms)
{
    const int *src = reinterpret_cast<const int *>(&m);
    int *dst = reinterpret_cast<int *>(&ms);
    for (int w = threadIdx.x; w < int(sizeof(DevMech) / sizeof(int)); w += blockDim.x) dst[w] = src[w];
}

// The block's tables of the warp-per-cell kinetics: the mechanism and its
// per-reaction tables transposed. Blocks are 128 threads: four warps, four
// exchange buffers.
template <int NS, int NR>
struct HeavyShared {
    DevMech ms;
    HeavyTablesT<NS, NR> tt;
    HeavyScratch x[4];
};

__device__ __forceinline__ unsigned coef2(double v) { return v <= 0.0 ? 0u : v <= 1.0 ? 1u : 2u; }

template <int NS, int NR>
__device__ __forceinline__ void heavy_shared_setup(const DevMech &m, HeavyShared<NS, NR> &sh)
{
    static_assert(NS <= 16 && NR <= 32, "4-bit species and 5-bit reaction indices");
    copy_mech_to_shared(m, sh.ms);
    HeavyTablesT<NS, NR> &t = sh.tt;
    for (int i = threadIdx.x; i < NS * 32; i += blockDim.x) {
        const int sp = i / 32, r = i % 32, rr = r < NR ? r : 0;
        t.tb[sp][r] = m.tb[rr][sp];
    }
    if (threadIdx.x < NS)
        t.imw[threadIdx.x] = 1e-3 / m.mw[threadIdx.x];
    if (threadIdx.x < 32) { // lane l's lists
        const int l = threadIdx.x, r = l < NR ? l : 0, sp = l < NS ? l : 0;
        int n = 0;
        for (int s = 0; s < NS; ++s) {
            const unsigned fi = coef2(m.sf[r][s]), bi = coef2(m.sb[r][s]);
            if (fi | bi)
                t.rent[n++][l] = (unsigned char)(s | fi << 4 | bi << 6);
        }
        for (; n < NS; ++n) t.rent[n][l] = 0;
        n = 0;
        for (int q = 0; q < NR; ++q) {
            const double bb = m.sb[q][sp], f = m.sf[q][sp];
            if (bb != 0.0 || f != 0.0) {
                t.sent[n][l] = (unsigned char)q;
                t.sbv[n][l] = bb;
                t.sfv[n][l] = f;
                ++n;
            }
        }
        for (; n < NR; ++n) {
            t.sent[n][l] = 31;
            t.sbv[n][l] = 0.0;
            t.sfv[n][l] = 0.0;
        }
    }
}

// The order in which the warps of a persistent grid take deferred cells:
// position p of n is entry p * s mod n, s near 0.618 n and coprime with n (a
// bijection of [0, n)). The queue holds the cells in about the order the
// recovery met them, so neighbouring cells, whose stiffness is alike, sit
// next to each other; the warps that start together belong to few blocks,
// and without the scatter the stiffest cells would share a few SMs.
__device__ __forceinline__ long long scatter_stride(long long n)
{
    long long s = static_cast<long long>(0.6180339887498949 * double(n)) | 1;
    for (;;) {
        long long a = s, b = n;
        while (b != 0) {
            const long long t = a % b;
            a = b;
            b = t;
        }
        if (a == 1)
            return s;
        s += 2;
    }
}

template <int NS, int NR>
__global__ void __launch_bounds__(128, 3) k_react_heavy(const __grid_constant__ DevMech m, const DevGrid g,
                                                     const DevState st, const double *__restrict__ dt_dev,
                                                     int max_substeps)
{
    __shared__ HeavyShared<NS, NR> sh;
    const int count = st.heavy[0];
    if (count == 0) // no deferred cell this step: skip the table copy
        return;
    heavy_shared_setup<NS, NR>(m, sh);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const HeavyLane<NS, NR> hl = heavy_lane<NS, NR>(sh.ms, lane);
    HeavyScratch &x = sh.x[threadIdx.x / 32];
    const double dtm = *dt_dev;
    const long long stride = scatter_stride(count);
    for (;;) {
        int q = 0;
        if (lane == 0)
            q = atomicAdd(&st.heavy[1], 1);
        q = __shfl_sync(0xffffffffu, q, 0);
        if (q >= count)
            break;
        const int e = int((q * stride) % count);
        react_heavy_cell<NS, NR>(m, sh.ms, hl, sh.tt, x, st, g.n3, st.heavy[2 + e], dtm, max_substeps, lane);
    }
}

// The deferred cells of every instance of a batch, their heavy queues taken
// end to end, drained by one persistent grid (one warp per cell, one counter).
template <int NS, int NR>
__global__ void __launch_bounds__(128, 3) k_react_heavy_batch(const __grid_constant__ DevMech m,
                                                           const BatchCell *__restrict__ tab, int n, int *next,
                                                           int max_substeps)
{
    __shared__ HeavyShared<NS, NR> sh;
    auto len = [&](int q) { return tab[q].st.heavy ? *(volatile const int *)tab[q].st.heavy : 0; };
    int total = 0;
    for (int q = 0; q < n; ++q) total += len(q);
    if (total == 0)
        return;
    heavy_shared_setup<NS, NR>(m, sh);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const HeavyLane<NS, NR> hl = heavy_lane<NS, NR>(sh.ms, lane);
    HeavyScratch &x = sh.x[threadIdx.x / 32];
    const long long stride = scatter_stride(total);
    for (;;) {
        int pos = 0;
        if (lane == 0)
            pos = atomicAdd(next, 1);
        pos = __shfl_sync(0xffffffffu, pos, 0);
        if (pos >= total)
            break;
        int local = 0;
        const int q = batch_locate(n, int((pos * stride) % total), len, local);
        if (q < n) {
            const BatchCell &b = tab[q];
            react_heavy_cell<NS, NR>(m, sh.ms, hl, sh.tt, x, b.st, b.n3, b.st.heavy[2 + local], *b.dt, max_substeps,
                                     lane);
        }
    }
}

// ------------------------------------------------- independent cell samples
// (training data for the learned model: the stiff chemistry on a batch of
// constant-volume, constant-energy cells, each with its own dt)

// Conserved state of cells at rest from (T, p, Y): FieldInitial's formulas
// (src/Flowfield.cpp:226-262). cs: NS + 4 planes of n; Y: NS planes of n.
template <int NS>
__global__ void k_state_from_tpy(const __grid_constant__ DevMech m, long long n, const double *__restrict__ T,
                                 const double *__restrict__ p, const double *__restrict__ Y, double *cs, double *E)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double y[NS], inv_w = 0, e = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) y[s] = Y[s * n + i];
#pragma unroll
    for (int s = 0; s < NS; ++s) inv_w += y[s] / m.mw[s];
    const double Tc = T[i];
    const double D = p[i] / (kRUniv * 1000 * inv_w * Tc);
    const TPow pw = make_tpow(Tc, true);
#pragma unroll
    for (int s = 0; s < NS; ++s) e += y[s] * (h_species<NS>(m, pw, m.ri[s], s) - m.ri[s] * Tc);
#pragma unroll
    for (int s = 0; s < NS; ++s) cs[s * n + i] = D * y[s];
    cs[(NS + 0) * n + i] = 0;
    cs[(NS + 1) * n + i] = 0;
    cs[(NS + 2) * n + i] = 0;
    cs[(NS + 3) * n + i] = D * e * 1000;
    E[i] = e * 1000;
}

// One chemistry step (react_cell) of each sample with its own dt, in place.
template <int NS, class Rt>
__global__ void __launch_bounds__(128) k_chem_samples(const __grid_constant__ DevMech m, long long n, double *cs,
                                                      double *T, double *E, const double *__restrict__ dt,
                                                      int *nchem, int max_substeps, unsigned long long *counters)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    CellState<NS> cell;
#pragma unroll
    for (int q = 0; q < NS + 4; ++q) cell.cs[q] = cs[q * n + i];
    cell.T = T[i];
    cell.E = E[i];
    double D = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) D += cell.cs[s];
#pragma unroll
    for (int s = 0; s < NS; ++s) cell.Y[s] = cell.cs[s] / D;
    cell.D = D;
    cell.U = cell.cs[NS] / D;
    cell.V = cell.cs[NS + 1] / D;
    cell.W = cell.cs[NS + 2] / D;
    const int nc = react_cell<NS, Rt>(m, cell, dt[i], max_substeps, counters, nullptr, 0);
    if (nchem)
        nchem[i] = nc;
#pragma unroll
    for (int q = 0; q < NS + 4; ++q) cs[q * n + i] = cell.cs[q];
    T[i] = cell.T;
    E[i] = cell.E;
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

// Stage combination of the three-stage TVD Runge-Kutta advection (Shu and
// Osher's SSP-RK3; the reference's TimeAdv::TVD_RK3, src/TimeAdv.cpp:210-221,
// is an empty stub): CS = a CS0 + b CS on the interior nodes, each product and
// the sum rounded separately (the same value in every arithmetic flavour).
__global__ void k_rk_combine(const DevGrid g, double *__restrict__ cs, const double *__restrict__ cs0, int planes,
                             double a, double b)
{
    const long long n = (long long)g.ni * g.nj * g.nk;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        interior_node(g, t, i, j, k);
        const long long c = cell_index(g, i, j, k);
        for (int q = 0; q < planes; ++q) {
            const long long o = q * g.n3 + c;
            cs[o] = __dadd_rn(__dmul_rn(a, cs0[o]), __dmul_rn(b, cs[o]));
        }
    }
}

// Writes a scalar (the timestep) into device memory from a kernel argument, so
// the value is captured at launch and the caller's copy may go away.
__global__ void k_set_value(double *dst, double v) { *dst = v; }

// Flowfield::CFLcondition (src/Flowfield.cpp:275-304): the smallest
// min(dx / (|u| + c), dy / (|v| + c)) over the interior nodes, c = sqrt(gamma p
// / rho), from the primitive planes the next flux step reads (FP32 in mixed
// precision). The spacings are the interior ones (the reference takes them
// from its first two ghost nodes, the same on a uniform grid with three or
// more nodes per axis). Positive doubles order as their bit patterns, so the
// block minima combine with an integer atomicMin into *slot (non-finite values
// map to the largest key and never win).
__global__ void __launch_bounds__(256) k_cfl_min(const DevGrid g, const DevState st, unsigned long long *slot)
{
    const long long ncell = (long long)g.ni * g.nj * g.nk;
    const double dx = g.x[g.bc + 1] - g.x[g.bc], dy = g.y[g.bc + 1] - g.y[g.bc];
    const long long n3 = g.n3;
    double m = __longlong_as_double(0x7ff0000000000000LL);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ncell;
         t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        interior_node(g, t, i, j, k);
        const long long c = cell_index(g, i, j, k);
        double P, D, U, V, G;
        if (st.prim32) {
            P = st.prim32[kP * n3 + c];
            D = st.prim32[kD * n3 + c];
            U = st.prim32[kU * n3 + c];
            V = st.prim32[kV * n3 + c];
            G = st.prim32[kG * n3 + c];
        } else {
            P = st.prim[kP * n3 + c];
            D = st.prim[kD * n3 + c];
            U = st.prim[kU * n3 + c];
            V = st.prim[kV * n3 + c];
            G = st.prim[kG * n3 + c];
        }
        const double C = sqrt(G * P / D);
        const double q = fmin(dx / (fabs(U) + C), dy / (fabs(V) + C));
        m = (q < m || !(q == q)) ? q : m; // a NaN sticks
    }
    unsigned long long b = (unsigned long long)__double_as_longlong(m);
    if (!(m >= 0.0)) // NaN (or a negative spacing): the largest key
        b = ~0ULL;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v = __shfl_xor_sync(0xffffffffu, b, o);
        b = v < b ? v : b;
    }
    __shared__ unsigned long long wmin[8];
    if ((threadIdx.x & 31) == 0)
        wmin[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) b = wmin[w] < b ? wmin[w] : b;
        atomicMin(slot, b);
    }
}

// dt = cfl * the minimum; the step's kernels read *dt_dev; *time accumulates
// the steps' dt; the slot is reset for the next step.
__global__ void k_cfl_finish(unsigned long long *slot, double cfl, double *dt_dev, double *time)
{
    const double dt = cfl * __longlong_as_double((long long)*slot);
    *dt_dev = dt;
    *time += dt;
    *slot = 0x7ff0000000000000ULL;
}

} // namespace EU3D_NS
} // namespace eu3d
