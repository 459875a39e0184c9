// eu3d_device.cuh — device-side types and per-cell / per-face arithmetic of the
// EU3D reacting-Euler timestep for sm_100a.
//
// Included by the kernel translation units. EU_STRICT selects the variants that
// round exactly as the reference's CPU build (no FMA: those units are compiled
// with --fmad=false; divisions and operand order as in the reference); without
// it, FMA contraction and algebraically equivalent fast forms are used.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "eu3d_types.h"

namespace eu3d {

__device__ __forceinline__ long long cell_index(const DevGrid &g, int i, int j, int k)
{
    return ((long long)i * g.ny + j) * g.nz + k;
}

// ------------------------------------------------------------------ thermo
// NASA 9-coefficient polynomials (src/Reaction.cpp:1165-1220). T powers are
// formed once per temperature.
struct TPow {
    double T, inv, inv2, t2, t3, t4, t5, lnT;
    bool low;
};

__device__ __forceinline__ TPow make_tpow(double T, bool need_log)
{
    TPow p;
    p.T = T;
    p.low = T < kThermoSwitch;
    p.inv = 1.0 / T;
    p.inv2 = p.inv * p.inv;
    p.t2 = T * T;
    p.t3 = p.t2 * T;
    p.t4 = p.t3 * T;
    p.t5 = p.t4 * T;
    p.lnT = need_log ? log(T) : 0.0;
    return p;
}

template <int NS>
__device__ __forceinline__ double coeff(const DevMech &m, const TPow &p, int k, int s)
{
    return p.low ? m.clo[k][s] : m.chi[k][s];
}

// Reaction::GetCpi: R*(a1 T^-2 + a2 T^-1 + a3 + a4 T + a5 T^2 + a6 T^3 + a7 T^4)
template <int NS>
__device__ __forceinline__ double cp_species(const DevMech &m, const TPow &p, double R, int s)
{
    const double a0 = coeff<NS>(m, p, 0, s), a1 = coeff<NS>(m, p, 1, s), a2 = coeff<NS>(m, p, 2, s),
                 a3 = coeff<NS>(m, p, 3, s), a4 = coeff<NS>(m, p, 4, s), a5 = coeff<NS>(m, p, 5, s),
                 a6 = coeff<NS>(m, p, 6, s);
    return R * (a0 * p.inv2 + a1 * p.inv + a2 + a3 * p.T + a4 * p.t2 + a5 * p.t3 + a6 * p.t4);
}

// Reaction::GetHi: R*(-a1/T + a2 lnT + a3 T + a4 T^2/2 + a5 T^3/3 + a6 T^4/4 + a7 T^5/5 + b1)
template <int NS>
__device__ __forceinline__ double h_species(const DevMech &m, const TPow &p, double R, int s)
{
    const double a0 = coeff<NS>(m, p, 0, s), a1 = coeff<NS>(m, p, 1, s), a2 = coeff<NS>(m, p, 2, s),
                 a3 = coeff<NS>(m, p, 3, s), a4 = coeff<NS>(m, p, 4, s), a5 = coeff<NS>(m, p, 5, s),
                 a6 = coeff<NS>(m, p, 6, s), a7 = coeff<NS>(m, p, 7, s);
#ifdef EU_STRICT
    return R * (-a0 * p.inv + a1 * p.lnT + a2 * p.T + a3 * p.t2 / 2 + a4 * p.t3 / 3 + a5 * p.t4 / 4 +
                a6 * p.t5 / 5 + a7);
#else
    return R * (-a0 * p.inv + a1 * p.lnT + a2 * p.T + a3 * p.t2 * 0.5 + a4 * p.t3 * (1.0 / 3.0) +
                a5 * p.t4 * 0.25 + a6 * p.t5 * 0.2 + a7);
#endif
}

// Reaction::GetSi: R*(-a1 T^-2/2 - a2/T + a3 lnT + a4 T + a5 T^2/2 + a6 T^3/3 + a7 T^4/4 + b2)
template <int NS>
__device__ __forceinline__ double s_species(const DevMech &m, const TPow &p, double R, int s)
{
    const double a0 = coeff<NS>(m, p, 0, s), a1 = coeff<NS>(m, p, 1, s), a2 = coeff<NS>(m, p, 2, s),
                 a3 = coeff<NS>(m, p, 3, s), a4 = coeff<NS>(m, p, 4, s), a5 = coeff<NS>(m, p, 5, s),
                 a6 = coeff<NS>(m, p, 6, s), a8 = coeff<NS>(m, p, 8, s);
#ifdef EU_STRICT
    return R * (-a0 * p.inv2 / 2 - a1 * p.inv + a2 * p.lnT + a3 * p.T + a4 * p.t2 / 2 + a5 * p.t3 / 3 +
                a6 * p.t4 / 4 + a8);
#else
    return R * (-a0 * p.inv2 * 0.5 - a1 * p.inv + a2 * p.lnT + a3 * p.T + a4 * p.t2 * 0.5 +
                a5 * p.t3 * (1.0 / 3.0) + a6 * p.t4 * 0.25 + a8);
#endif
}

// --------------------------------------------------------- state recovery

// Flowfield::Get_temp (src/Flowfield.cpp:2072-2131): Newton on
// sum_s Y_s h_s(T) - E*1e-3 - (sum_s Y_s R_s) T = 0, at most 10 iterations,
// stop when |dT| < 1e-6 K. E is the cell's previous internal energy.
template <int NS>
__device__ __forceinline__ double newton_temperature(const DevMech &m, double T, double E, const double (&Y)[NS])
{
    double rsum = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) rsum += Y[s] * m.ri[s];
    const double e_scaled = E * 1e-3;
    double T_temp = T;
    for (int count = 0; count < 10; ++count) {
        const double T0 = T_temp;
        const TPow p = make_tpow(T0, true);
        double hsum = 0, cpsum = 0;
#pragma unroll
        for (int s = 0; s < NS; ++s) hsum += Y[s] * h_species<NS>(m, p, m.ri[s], s);
#pragma unroll
        for (int s = 0; s < NS; ++s) cpsum += Y[s] * cp_species<NS>(m, p, m.ri[s], s);
        const double temp1 = (hsum - e_scaled) - rsum * T0;
        const double temp2 = cpsum - rsum;
        T_temp = T0 - temp1 / temp2;
        if (fabs(T_temp - T0) < 1e-6)
            break;
    }
    return T_temp;
}

// Per-cell flow state kept in registers by the recovery / kinetics kernel.
template <int NS>
struct CellState {
    double cs[NS + 4];
    double Y[NS];
    double D, T, E, U, V, W;
};

// Flowfield::Update_after_CS (src/Flowfield.cpp:1579-1617 / :1639-1673) for one
// cell, up to the point where P, H, Gamma are needed (those are formed by
// finish_primitives when the cell's primitives are written).
template <int NS>
__device__ __forceinline__ void recover_state(const DevMech &m, CellState<NS> &c)
{
    double D = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) D += c.cs[s];
#pragma unroll
    for (int s = 0; s < NS; ++s) c.Y[s] = c.cs[s] / D;
    c.D = D;
    c.T = newton_temperature<NS>(m, c.T, c.E, c.Y);
    c.U = c.cs[NS + 0] / D;
    c.V = c.cs[NS + 1] / D;
    c.W = c.cs[NS + 2] / D;
    c.E = (c.cs[NS + 3] - 0.5 * D * (c.U * c.U + c.V * c.V + c.W * c.W)) / D;
}

// P, H, Gamma of Update_after_CS (src/Flowfield.cpp:1606-1614).
template <int NS>
__device__ __forceinline__ void finish_primitives(const DevMech &m, const CellState<NS> &c, double &P, double &H,
                                                  double &G)
{
    double inv_w = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) inv_w += c.Y[s] / m.mw[s];
    const double Wav = 1.0 / inv_w;
    const double Rgas = kRUniv * 1000 / Wav;
    P = c.T * c.D * Rgas;
    H = P / c.D + c.E;
    const TPow p = make_tpow(c.T, false);
    double cp = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) cp += cp_species<NS>(m, p, m.ri[s], s) * c.Y[s];
    const double Cp = cp * 1000;
    G = Cp / (Cp - kRUniv * inv_w * 1000);
}

// ------------------------------------------------------------- kinetics

// pow(x, nu) for the reference's stoichiometric exponents (0, 1, 2 are exact).
__device__ __forceinline__ double pow_nu(double x, double nu, bool nu_int)
{
    if (nu_int)
        return nu == 0.0 ? 1.0 : (nu == 1.0 ? x : x * x);
    return pow(x, nu);
}

__device__ __forceinline__ double pow_int_or_real(double x, double e)
{
    if (e == 0.0)
        return 1.0;
    if (e == 1.0)
        return x;
    if (e == -1.0)
        return 1.0 / x;
    return pow(x, e);
}

// Net rates of one cell at temperature T and concentrations mc (scaled 1e-6):
// src/Reaction.cpp:597-623 (also :873-903 in TrapezoidPrediction). Outputs per
// reaction the forward and backward products kf*[X]^nu_f, kb*[X]^nu_b, the
// third-body factor and the species mass rates Wi (:720-727).
template <int NS, int NR>
struct Rates {
    double fwd[NR], bwd[NR], rtb[NR];
    double wi[NS];
};

template <int NS, int NR>
__device__ __forceinline__ void eval_rates(const DevMech &m, double T, const double (&mc)[NS], Rates<NS, NR> &k)
{
    double Gi[NS];
    {
        const TPow p = make_tpow(T, true);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const double hi = h_species<NS>(m, p, kRUniv, s);
            const double si = s_species<NS>(m, p, kRUniv, s);
            Gi[s] = hi - si * T;
        }
    }
    const bool nu_int = m.nu_int != 0;
    const double RT = kRUniv * T;
    const double RuT = kRuCal * T;
    const double p0 = kP0 * 1e-6;
#pragma unroll
    for (int s = 0; s < NS; ++s) k.wi[s] = 0.0;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        double delta_g = 0.0, rrf = 1.0, rrb = 1.0, rtb = 0.0;
        const double kf =
            m.af[r] * pow_int_or_real(T, m.bf[r]) * (m.eaf[r] == 0.0 ? 1.0 : exp(-m.eaf[r] / RuT));
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const double f = m.sf[r][s], b = m.sb[r][s];
            delta_g += (b - f) * Gi[s];
            rrf *= pow_nu(mc[s], f, nu_int);
            rrb *= pow_nu(mc[s], b, nu_int);
            rtb += mc[s] * m.tb[r][s];
        }
        const double Xr = m.xr[r];
        const double Kp = exp(-delta_g / RT) * pow_int_or_real(p0, Xr);
        const double Kc = Kp * pow_int_or_real(RT, -Xr);
        const double kb = kf / Kc;
        if (rtb == 0.0)
            rtb = 1.0;
        const double fwd = kf * rrf, bwd = kb * rrb;
        k.fwd[r] = fwd;
        k.bwd[r] = bwd;
        k.rtb[r] = rtb;
        const double rr = fwd - bwd;
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const double d = m.sb[r][s] - m.sf[r][s];
            if (d != 0.0)
                k.wi[s] += d * rtb * rr;
        }
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) k.wi[s] = m.mw[s] * k.wi[s];
}

// One linearised trapezoid substep (src/Reaction.cpp:786-805) followed by
// Flowfield::Explicit(step,i,j,k) (src/Flowfield.cpp:1521-1536) and the state
// recovery. mc/di hold the scaled concentrations/densities the rates used.
template <int NS, int NR>
__device__ __forceinline__ void trapezoid_substep(const DevMech &m, const Rates<NS, NR> &k, double dts,
                                                  const double (&mc)[NS], const double (&di)[NS],
                                                  CellState<NS> &c)
{
    double P[NS], Q[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        P[s] = 0.0;
        Q[s] = 0.0;
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const double fwd = k.fwd[r], bwd = k.bwd[r], rtb = k.rtb[r];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const double b = m.sb[r][s], f = m.sf[r][s];
            if (b != 0.0 || f != 0.0) {
                Q[s] += (b * fwd + f * bwd) * rtb;
                P[s] += (b * bwd + f * fwd) * rtb;
            }
        }
    }
    const double half = dts / 2.0;
    double D = 0.0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const double q = m.mw[s] * Q[s];
        const double p = (mc[s] == 0) ? 0.0 : P[s] / mc[s];
        const double nd = ((1.0 - half * p) * di[s] + dts * q) / (1.0 + half * p) * 1e3;
        c.cs[s] = nd;
        D += nd;
    }
    c.cs[NS + 0] = c.U * D;
    c.cs[NS + 1] = c.V * D;
    c.cs[NS + 2] = c.W * D;
    c.cs[NS + 3] = D * c.E + 0.5 * (c.U * c.U + c.V * c.V + c.W * c.W) * D;
    recover_state<NS>(m, c);
}

template <int NS>
__device__ __forceinline__ void scaled_species(const DevMech &m, const CellState<NS> &c, double (&mc)[NS],
                                               double (&di)[NS])
{
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        di[s] = c.cs[s] * 1e-3;
        mc[s] = (c.cs[s] / m.mw[s] * 1000) * 1e-6;
    }
}

// ----------------------------------------------------------------- fluxes

// Minmod (include/Differ.hpp:33-43) as selects.
template <typename R>
__device__ __forceinline__ R minmod(R r)
{
    return r > R(0) ? ((R(1) < r) ? R(1) : r) : R(0);
}

// MUSCL_2, kappa = 1/3, minmod (include/Differ.hpp:149-238) for the face
// between m and m+1: fm1, f0, f1, f2 are values at m-1, m, m+1, m+2.
template <typename R>
__device__ __forceinline__ void muscl(R fm1, R f0, R f1, R f2, R &left, R &right)
{
    const R kk = R(1.0) / R(3.0);
    const R A0 = f0 - fm1;
    const R A1 = f1 - f0;
    const R A2 = f2 - f1;
    const R L = A1 / (A0 + R(1e-12));
    const R Rr = A1 / (A2 + R(1e-12));
    const R L1 = minmod(L), L2 = minmod(R(1.0) / L), R1 = minmod(Rr), R2 = minmod(R(1.0) / Rr);
    left = f0 + R(0.25) * ((R(1.0) - kk) * L1 + (R(1) + kk) * L2 * L) * A0;
    right = f1 - R(0.25) * ((R(1.0) - kk) * R1 + (R(1) + kk) * R2 * Rr) * A2;
}

// AUSM+ flux of one face (src/Flowfield.cpp:1811-1930) for direction DIR
// (0: x, 1: y, 2: z). lr holds the reconstructed left/right primitives
// {P, D, U, V, W, H, Gamma} and species. Output F[NS+4] in FP64.
template <int NS, int DIR, typename R>
__device__ __forceinline__ void ausm(const R (&L)[7], const R (&Rt)[7], const R (&YL)[NS], const R (&YR)[NS],
                                     double (&F)[NS + 4])
{
    const R PL = L[kP], PR = Rt[kP], DL = L[kD], DR = Rt[kD];
    const R CL = sqrt(L[kG] * PL / DL);
    const R CR = sqrt(Rt[kG] * PR / DR);
    const R CI = R(0.5) * (CL + CR);
    const R MaL = L[kU + DIR] / CI;
    const R MaR = Rt[kU + DIR] / CI;
    R B1, G1, B2, G2;
    if (fabs(MaL) < R(1.0)) {
        const R a = MaL + R(1.0), t = MaL * MaL - R(1.0);
        B1 = R(0.25) * (a * a) + R(0.125) * (t * t);
        G1 = R(0.25) * (a * a) * (R(2.0) - MaL) + R(3.0) / R(16.0) * MaL * (t * t);
    } else {
        B1 = R(0.5) * (MaL + fabs(MaL));
        G1 = B1 / MaL;
    }
    if (fabs(MaR) < R(1.0)) {
        const R a = MaR - R(1.0), t = MaR * MaR - R(1.0);
        B2 = -R(0.25) * (a * a) - R(0.125) * (t * t);
        G2 = R(0.25) * (a * a) * (R(2.0) + MaR) - R(3.0) / R(16.0) * MaR * (t * t);
    } else {
        B2 = R(0.5) * (MaR - fabs(MaR));
        G2 = B2 / MaR;
    }
    const R MaI = B1 + B2;
    const R VI = MaI * CI;
    const bool up = VI >= R(0.0);
    const R Du = up ? DL : DR, Uu = up ? L[kU] : Rt[kU], Vu = up ? L[kV] : Rt[kV], Wu = up ? L[kW] : Rt[kW],
            Hu = up ? L[kH] : Rt[kH];
    const R m = VI * Du;
#pragma unroll
    for (int s = 0; s < NS; ++s) F[s] = double(m * (up ? YL[s] : YR[s]));
    R mom[3] = {m * Uu, m * Vu, m * Wu};
    mom[DIR] = mom[DIR] + G1 * PL + G2 * PR;
    F[NS + 0] = double(mom[0]);
    F[NS + 1] = double(mom[1]);
    F[NS + 2] = double(mom[2]);
    F[NS + 3] = double(VI * (Du * Hu + R(0.5) * Du * (Uu * Uu + Vu * Vu + Wu * Wu)));
}

} // namespace eu3d
