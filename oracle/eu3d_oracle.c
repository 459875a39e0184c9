/*
 * eu3d_oracle.c — CPU restatement of the EU3D reacting-Euler timestep.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; never part of the shipped library).
 * Compiled with -O3 -ffp-contract=off, the reference's own flags, so that every
 * expression rounds exactly as the reference's CPU build does. Expression
 * order (including the order of operands of + and *) follows the cited
 * reference lines; pow() calls are kept where the reference makes them so the
 * compiler treats them identically.
 */
#include "eu3d_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define EO_MAXS 16 /* include/ReactionCuda.cuh:4 limits */
#define EO_MAXR 24

static const double R_UNIV = 8.31434; /* include/Flowfield.hpp:57, include/Reaction.hpp:66 */
static const double RU_CAL = 1.987;   /* include/Reaction.hpp:67 */
static const double P0_ATM = 101325;  /* include/Reaction.hpp:68 */
static const double THERMO_SWITCH = 1000.0; /* include/ThermoConstants.hpp:3 */

struct eo_state {
    int ni, nj, nk, bc, nx, ny, nz;
    long n3;
    int ns, nr, nthreads;
    double *x, *y, *z;
    double mw[EO_MAXS], ri[EO_MAXS];
    double clo[9 * EO_MAXS], chi[9 * EO_MAXS];
    double af[EO_MAXR], bf[EO_MAXR], eaf[EO_MAXR];
    double sf[EO_MAXS * EO_MAXR], sb[EO_MAXS * EO_MAXR], tb[EO_MAXS * EO_MAXR];
    /* persistent fields */
    double *P, *D, *U, *V, *W, *H, *G, *T, *E;
    double *Y;  /* ns planes */
    double *CS; /* ns+4 planes */
    double *flux[3]; /* ns+4 planes each, face i+1/2 stored at the left cell */
    double *cms; /* ns planes */
    int *nchem;
    double dt;
    int bad_nchem;
    int bc_kind; /* 0: RSBI ghost fill, 1: ZND */
    int exch_lo, exch_hi; /* x faces filled by the halo exchange, not the ghost fill */
    int wall_i0;    /* ODW: first local x node of the y-low wall (0: the whole face) */
    double *inflow; /* ODW: x-low ghost values per interior (j, k), 9 + ns planes
                       (P D T U V W H Gamma E Y...), or NULL */
    int scheme;     /* 0: Euler explicit (TimeAdv::EE), 1: three-stage TVD Runge-Kutta */
    double *cs0;    /* RK: the conserved state at the start of the step */
    double rk_a, rk_b; /* RK stage combination CS = a CS0 + b CS (phase 4) */
};

#define IDX(st, i, j, k) (((long)(i) * (st)->ny + (j)) * (st)->nz + (k))

/* ---------------------------------------------------------------- thermo */

/* Reaction::GetCpi, src/Reaction.cpp:1165-1177 */
static double get_cpi(const eo_state *st, double T, double R, int sp)
{
    const double *c = (T < THERMO_SWITCH) ? st->clo : st->chi;
    const int ns = st->ns;
    return R * (c[0 * ns + sp] * pow(T, -2) + c[1 * ns + sp] * pow(T, -1) + c[2 * ns + sp] + c[3 * ns + sp] * T +
                c[4 * ns + sp] * pow(T, 2) + c[5 * ns + sp] * pow(T, 3) + c[6 * ns + sp] * pow(T, 4));
}

/* Reaction::GetHi, src/Reaction.cpp:1189-1199 */
static double get_hi(const eo_state *st, double T, double R, int sp)
{
    const double *c = (T < THERMO_SWITCH) ? st->clo : st->chi;
    const int ns = st->ns;
    return R * (-c[0 * ns + sp] * pow(T, -1) + c[1 * ns + sp] * log(T) + c[2 * ns + sp] * T +
                c[3 * ns + sp] * pow(T, 2) / 2 + c[4 * ns + sp] * pow(T, 3) / 3 + c[5 * ns + sp] * pow(T, 4) / 4 +
                c[6 * ns + sp] * pow(T, 5) / 5 + c[7 * ns + sp]);
}

/* Reaction::GetSi, src/Reaction.cpp:1211-1220 */
static double get_si(const eo_state *st, double T, double R, int sp)
{
    const double *c = (T < THERMO_SWITCH) ? st->clo : st->chi;
    const int ns = st->ns;
    return R * (-c[0 * ns + sp] * pow(T, -2) / 2 - c[1 * ns + sp] * pow(T, -1) + c[2 * ns + sp] * log(T) +
                c[3 * ns + sp] * T + c[4 * ns + sp] * pow(T, 2) / 2 + c[5 * ns + sp] * pow(T, 3) / 3 +
                c[6 * ns + sp] * pow(T, 4) / 4 + c[8 * ns + sp]);
}

/* ------------------------------------------------------- state recovery */

/* Flowfield::Get_temp, src/Flowfield.cpp:2072-2131 */
static double get_temp(const eo_state *st, double T, double E, const double *Y)
{
    const int ns = st->ns;
    double T0 = T, T_temp = T;
    int count = 0;
    while (count < 10) {
        double hsum = 0, cpsum = 0, rsum1 = 0, rsum2 = 0;
        T0 = T_temp;
        for (int s = 0; s < ns; s++) hsum += Y[s] * get_hi(st, T0, st->ri[s], s);
        for (int s = 0; s < ns; s++) rsum1 += Y[s] * st->ri[s];
        for (int s = 0; s < ns; s++) cpsum += Y[s] * get_cpi(st, T0, st->ri[s], s);
        rsum2 = rsum1;
        double temp1 = (hsum - E * 1e-3) - rsum1 * T0;
        double temp2 = cpsum - rsum2;
        T_temp = T0 - temp1 / temp2;
        if (fabs(T_temp - T0) < 1e-6)
            break;
        count = count + 1;
    }
    return T_temp;
}

/* Flowfield::Update_after_CS(step,i,j,k), src/Flowfield.cpp:1639-1673: every
 * field of cell c from its conserved variables, T from Newton with the cell's
 * current (old) E held. */
static void update_after_cs(eo_state *st, long c)
{
    const int ns = st->ns;
    const long n3 = st->n3;
    double Y[EO_MAXS];
    double D = 0;
    for (int s = 0; s < ns; s++) D += st->CS[s * n3 + c];
    for (int s = 0; s < ns; s++) {
        Y[s] = st->CS[s * n3 + c] / D;
        st->Y[s * n3 + c] = Y[s];
    }
    st->D[c] = D;
    const double T = get_temp(st, st->T[c], st->E[c], Y);
    st->T[c] = T;
    const double U = st->CS[(ns + 0) * n3 + c] / D;
    const double V = st->CS[(ns + 1) * n3 + c] / D;
    const double W = st->CS[(ns + 2) * n3 + c] / D;
    const double E = (st->CS[(ns + 3) * n3 + c] - 0.5 * D * (pow(U, 2) + pow(V, 2) + pow(W, 2))) / D;
    st->U[c] = U;
    st->V[c] = V;
    st->W[c] = W;
    st->E[c] = E;
    double inv_w = 0;
    for (int s = 0; s < ns; s++) inv_w += Y[s] / st->mw[s];
    const double Wav = 1.0 / inv_w;
    const double Rgas = R_UNIV * 1000 / Wav;
    const double P = T * D * Rgas;
    st->P[c] = P;
    st->H[c] = P / D + E;
    double cp = 0;
    for (int s = 0; s < ns; s++) cp += get_cpi(st, T, st->ri[s], s) * Y[s];
    const double Cp = cp * 1000;
    st->G[c] = Cp / (Cp - R_UNIV * inv_w * 1000);
}

/* --------------------------------------------------------------- kinetics */

typedef struct {
    double kf[EO_MAXR], kb[EO_MAXR], rrf[EO_MAXR], rrb[EO_MAXR], rtb[EO_MAXR], rr[EO_MAXR];
    double wi[EO_MAXS];
} eo_rates;

/* Rate evaluation shared by Reaction::TrapezoidPrediction (src/Reaction.cpp:873-917)
 * and the adaptive Reaction::Trapezoid (src/Reaction.cpp:597-623, :720-727).
 * mc holds concentrations already scaled by 1e-6. */
static void eval_rates(const eo_state *st, double T, const double *mc, eo_rates *k)
{
    const int ns = st->ns, nr = st->nr;
    double Gi[EO_MAXS];
    for (int s = 0; s < ns; s++) {
        double hi = get_hi(st, T, R_UNIV, s);
        double si = get_si(st, T, R_UNIV, s);
        Gi[s] = hi - si * T;
    }
    for (int r = 0; r < nr; r++) {
        k->rrf[r] = 1.0;
        k->rrb[r] = 1.0;
        k->rtb[r] = 0;
    }
    for (int r = 0; r < nr; r++) {
        double Xr = 0.0, delta_g = 0.0;
        k->kf[r] = st->af[r] * pow(T, st->bf[r]) * exp(-st->eaf[r] / (RU_CAL * T));
        for (int s = 0; s < ns; s++) {
            const double f = st->sf[s * nr + r], b = st->sb[s * nr + r];
            Xr += (b - f);
            delta_g += (b - f) * Gi[s];
            k->rrf[r] *= pow(mc[s], f);
            k->rrb[r] *= pow(mc[s], b);
            k->rtb[r] += mc[s] * st->tb[s * nr + r];
        }
        const double Kp = exp(-delta_g / (R_UNIV * T)) * pow((P0_ATM * 1e-6), Xr);
        const double Kc = Kp * pow(R_UNIV * T, -Xr);
        k->kb[r] = k->kf[r] / Kc;
        if (k->rtb[r] == 0.0)
            k->rtb[r] = 1.0;
        k->rr[r] = k->kf[r] * k->rrf[r] - k->kb[r] * k->rrb[r];
    }
    for (int s = 0; s < ns; s++) {
        double temp = 0.0;
        for (int r = 0; r < nr; r++) temp += (st->sb[s * nr + r] - st->sf[s * nr + r]) * k->rtb[r] * k->rr[r];
        k->wi[s] = st->mw[s] * temp;
    }
}

/* One cell's chemistry for the step: Nchem prediction (src/Reaction.cpp:919-940)
 * then Nchem trapezoid substeps (src/Reaction.cpp:720-805), each followed by
 * Flowfield::Explicit(step,i,j,k) (src/Flowfield.cpp:1521-1536). */
static void react_cell(eo_state *st, long c)
{
    const int ns = st->ns, nr = st->nr;
    const long n3 = st->n3;
    const double dtm = st->dt;
    double mc[EO_MAXS], di[EO_MAXS];
    eo_rates k;

    /* prediction */
    for (int s = 0; s < ns; s++) {
        di[s] = st->CS[s * n3 + c] * 1e-3;
        mc[s] = (st->CS[s * n3 + c] / st->mw[s] * 1000) * 1e-6;
    }
    eval_rates(st, st->T[c], mc, &k);
    double dt = dtm;
    for (int s = 0; s < ns; s++) {
        if (st->Y[s * n3 + c] >= 1e-6 && k.wi[s] != 0) {
            double dt_temp = fabs(-di[s] / k.wi[s]);
            if (dt_temp < dt)
                dt = dt_temp;
        }
    }
    const int nchem = (int)ceil(dtm / dt);
    st->nchem[c] = nchem;
    if (nchem <= 0) {
        st->bad_nchem = 1;
        return;
    }

    for (int step = 0; step < nchem; step++) {
        const double dts = dtm / nchem;
        if (step > 0) {
            for (int s = 0; s < ns; s++) {
                di[s] = st->CS[s * n3 + c] * 1e-3;
                mc[s] = (st->CS[s * n3 + c] / st->mw[s] * 1000) * 1e-6;
            }
            eval_rates(st, st->T[c], mc, &k);
        }
        double newdi[EO_MAXS];
        for (int s = 0; s < ns; s++) {
            st->cms[s * n3 + c] = k.wi[s] * 1e3;
            double P = 0, Q = 0;
            for (int r = 0; r < nr; r++) {
                const double f = st->sf[s * nr + r], b = st->sb[s * nr + r];
                Q += (b * k.kf[r] * k.rrf[r] + f * k.kb[r] * k.rrb[r]) * k.rtb[r];
                P += (b * k.kb[r] * k.rrb[r] + f * k.kf[r] * k.rrf[r]) * k.rtb[r];
            }
            Q = st->mw[s] * Q;
            if (mc[s] == 0)
                P = 0.0;
            else
                P = P / mc[s];
            newdi[s] = ((1.0 - dts / 2.0 * P) * di[s] + dts * Q) / (1.0 + dts / 2.0 * P) * 1e3;
        }
        /* Flowfield::Explicit(step,i,j,k) */
        double D = 0.0;
        for (int s = 0; s < ns; s++) {
            st->CS[s * n3 + c] = newdi[s];
            D += newdi[s];
        }
        const double U = st->U[c], V = st->V[c], W = st->W[c], E = st->E[c];
        st->CS[(ns + 0) * n3 + c] = U * D;
        st->CS[(ns + 1) * n3 + c] = V * D;
        st->CS[(ns + 2) * n3 + c] = W * D;
        st->CS[(ns + 3) * n3 + c] = D * E + 0.5 * (pow(U, 2) + pow(V, 2) + pow(W, 2)) * D;
        update_after_cs(st, c);
    }
}

/* ---------------------------------------------------------------- fluxes */

/* Minmod, include/Differ.hpp:33-43 */
static double minmod(double R)
{
    if (R > 0)
        return (1.0 < R) ? 1.0 : R;
    return 0.0;
}

/* MUSCL_2 with minmod (limit=0), include/Differ.hpp:149-238 for one face:
 * f[0..3] = values at m-1, m, m+1, m+2; the face lies between m and m+1. */
static void muscl_face(const double f[4], double *left, double *right)
{
    const double kk = 1.0 / 3.0;
    const double A0 = f[1] - f[0];
    const double A1 = f[2] - f[1];
    const double A2 = f[3] - f[2];
    const double L = A1 / (A0 + 1e-12);
    const double R = A1 / (A2 + 1e-12);
    const double L1 = minmod(L), L2 = minmod(1.0 / L), R1 = minmod(R), R2 = minmod(1.0 / R);
    *left = f[1] + 0.25 * ((1.0 - kk) * L1 + (1 + kk) * L2 * L) * A0;
    *right = f[2] - 0.25 * ((1.0 - kk) * R1 + (1 + kk) * R2 * R) * A2;
}

/* AUSM+ face flux, src/Flowfield.cpp:1811-1930 (one face, one direction). */
static void ausm_face(int ns, int dir, double PL, double PR, double DL, double DR, double UL, double UR, double VL,
                      double VR, double WL, double WR, double HL, double HR, double GL, double GR, const double *YL,
                      const double *YR, double *F, long stride)
{
    double MaL, MaR, B1, B2, G1, G2;
    const double CL = sqrt(GL * PL / DL);
    const double CR = sqrt(GR * PR / DR);
    const double CI = 0.5 * (CL + CR);
    if (dir == 1) {
        MaL = UL / CI;
        MaR = UR / CI;
    } else if (dir == 2) {
        MaL = VL / CI;
        MaR = VR / CI;
    } else {
        MaL = WL / CI;
        MaR = WR / CI;
    }
    if (fabs(MaL) < 1.0) {
        B1 = 0.25 * pow((MaL + 1.0), 2) + 0.125 * pow((pow(MaL, 2) - 1.0), 2);
        G1 = 0.25 * pow((MaL + 1.0), 2) * (2.0 - MaL) + 3.0 / 16.0 * MaL * pow((pow(MaL, 2) - 1.0), 2);
    } else {
        B1 = 0.5 * (MaL + fabs(MaL));
        G1 = B1 / MaL;
    }
    if (fabs(MaR) < 1.0) {
        B2 = -0.25 * pow((MaR - 1.0), 2) - 0.125 * pow((pow(MaR, 2) - 1.0), 2);
        G2 = 0.25 * pow((MaR - 1.0), 2) * (2.0 + MaR) - 3.0 / 16.0 * MaR * pow((pow(MaR, 2) - 1.0), 2);
    } else {
        B2 = 0.5 * (MaR - fabs(MaR));
        G2 = B2 / MaR;
    }
    const double MaI = B1 + B2;
    const double VI = MaI * CI;
    double m0, m1, m2;
    if (VI >= 0.0) {
        for (int s = 0; s < ns; s++) F[s * stride] = VI * DL * YL[s];
        m0 = VI * DL * UL;
        m1 = VI * DL * VL;
        m2 = VI * DL * WL;
        F[(ns + 3) * stride] = VI * (DL * HL + 0.5 * DL * (pow(UL, 2) + pow(VL, 2) + pow(WL, 2)));
    } else {
        for (int s = 0; s < ns; s++) F[s * stride] = VI * DR * YR[s];
        m0 = VI * DR * UR;
        m1 = VI * DR * VR;
        m2 = VI * DR * WR;
        F[(ns + 3) * stride] = VI * (DR * HR + 0.5 * DR * (pow(UR, 2) + pow(VR, 2) + pow(WR, 2)));
    }
    if (dir == 1)
        m0 = m0 + G1 * PL + G2 * PR;
    else if (dir == 2)
        m1 = m1 + G1 * PL + G2 * PR;
    else
        m2 = m2 + G1 * PL + G2 * PR;
    F[(ns + 0) * stride] = m0;
    F[(ns + 1) * stride] = m1;
    F[(ns + 2) * stride] = m2;
}

/* Face flux between c and its +1 neighbour along dir (stride s1 in the layout). */
static void face_flux(eo_state *st, int dir, long c, long s1)
{
    const int ns = st->ns;
    const long n3 = st->n3;
    double L[7], R[7], YL[EO_MAXS], YR[EO_MAXS];
    const double *fields[7] = {st->P, st->D, st->U, st->V, st->W, st->H, st->G};
    for (int q = 0; q < 7; q++) {
        const double *a = fields[q];
        const double f[4] = {a[c - s1], a[c], a[c + s1], a[c + 2 * s1]};
        muscl_face(f, &L[q], &R[q]);
    }
    for (int s = 0; s < ns; s++) {
        const double *a = st->Y + s * n3;
        const double f[4] = {a[c - s1], a[c], a[c + s1], a[c + 2 * s1]};
        muscl_face(f, &YL[s], &YR[s]);
    }
    ausm_face(ns, dir, L[0], R[0], L[1], R[1], L[2], R[2], L[3], R[3], L[4], R[4], L[5], R[5], L[6], R[6], YL, YR,
              st->flux[dir - 1] + c, n3);
}

/* ----------------------------------------------------------- boundaries */

/* Flowfield::FieldBoundary_3dRSBI, src/Flowfield.cpp:593-807, on the face
 * layers the stencils read (tangential ranges over interior nodes). */
static void copy_cell(eo_state *st, long dst, long src, double su, double sv, double sw)
{
    const long n3 = st->n3;
    st->U[dst] = su * st->U[src];
    st->V[dst] = sv * st->V[src];
    st->W[dst] = sw * st->W[src];
    st->P[dst] = st->P[src];
    st->D[dst] = st->D[src];
    st->T[dst] = st->T[src];
    st->H[dst] = st->H[src];
    st->G[dst] = st->G[src];
    st->E[dst] = st->E[src];
    for (int s = 0; s < st->ns; s++) st->Y[s * n3 + dst] = st->Y[s * n3 + src];
}

/* Ghost node d from node s0 with the thermo recomputed from the mirrored T,
 * p, Y (src/Flowfield.cpp:647-679; the same rebuild closes the ZND outflow,
 * :340-366, and the ODW faces, :436-461, :509-585); sv, sw flip the y and z
 * velocities. */
static void rebuild_cell_w(eo_state *st, long d, long s0, double sv, double sw)
{
    const int ns = st->ns;
    const long n3 = st->n3;
    st->U[d] = st->U[s0];
    st->V[d] = sv * st->V[s0];
    st->W[d] = sw * st->W[s0];
    st->P[d] = st->P[s0];
    st->T[d] = st->T[s0];
    const double T = st->T[d];
    double rg = 0, cp = 0, h = 0, e = 0;
    double Y[EO_MAXS], Cpi[EO_MAXS], Hi[EO_MAXS], Ei[EO_MAXS];
    for (int s = 0; s < ns; s++) {
        Y[s] = st->Y[s * n3 + s0];
        st->Y[s * n3 + d] = Y[s];
        Cpi[s] = get_cpi(st, T, st->ri[s], s);
        Hi[s] = get_hi(st, T, st->ri[s], s);
        Ei[s] = Hi[s] - st->ri[s] * T;
    }
    for (int s = 0; s < ns; s++) rg += Y[s] * st->ri[s];
    const double Rgas = rg * 1000;
    st->D[d] = st->P[d] / (T * Rgas);
    for (int s = 0; s < ns; s++) cp += Cpi[s] * Y[s];
    for (int s = 0; s < ns; s++) h += Y[s] * Hi[s];
    for (int s = 0; s < ns; s++) e += Y[s] * Ei[s];
    const double Cp = cp * 1000;
    st->H[d] = h * 1000;
    st->E[d] = e * 1000;
    st->G[d] = Cp / (Cp - Rgas);
}

static void rebuild_cell(eo_state *st, long d, long s0, double sv) { rebuild_cell_w(st, d, s0, sv, 1); }

static void boundary_fill(eo_state *st)
{
    const int ni = st->ni, nj = st->nj, nk = st->nk, bc = st->bc;
    /* x, RSBI: zero-gradient mirror copy (src/Flowfield.cpp:597-641);
     * ZND (Flowfield::FieldBoundary_1dZND, :317-366, commented out in the
     * reference): reflecting wall at x low (U reflected), outflow at x high
     * with the thermo rebuilt */
    for (int i = 0; i < bc; i++)
        for (int j = bc; j < nj + bc; j++)
            for (int k = bc; k < nk + bc; k++) {
                const long lo = IDX(st, i, j, k), hi = IDX(st, ni + bc + i, j, k);
                const long slo = IDX(st, 2 * bc - 1 - i, j, k), shi = IDX(st, 2 * (ni + bc) - 1 - (ni + bc + i), j, k);
                if (st->bc_kind == 2) {
                    /* ODW: freestream inflow tables at x low (:414-432), outflow
                     * with the thermo rebuilt at x high (:434-461) */
                    if (!st->exch_lo && st->inflow) {
                        const long nt = (long)nj * nk, t = (long)(j - bc) * nk + (k - bc);
                        const double *f = st->inflow;
                        st->P[lo] = f[0 * nt + t];
                        st->D[lo] = f[1 * nt + t];
                        st->T[lo] = f[2 * nt + t];
                        st->U[lo] = f[3 * nt + t];
                        st->V[lo] = f[4 * nt + t];
                        st->W[lo] = f[5 * nt + t];
                        st->H[lo] = f[6 * nt + t];
                        st->G[lo] = f[7 * nt + t];
                        st->E[lo] = f[8 * nt + t];
                        for (int s = 0; s < st->ns; s++) st->Y[s * st->n3 + lo] = f[(9 + s) * nt + t];
                    }
                    if (!st->exch_hi)
                        rebuild_cell(st, hi, shi, 1);
                } else if (st->bc_kind == 1) {
                    if (!st->exch_lo)
                        copy_cell(st, lo, slo, -1, 1, 1);
                    if (!st->exch_hi)
                        rebuild_cell(st, hi, shi, 1);
                } else {
                    if (!st->exch_lo)
                        copy_cell(st, lo, slo, 1, 1, 1);
                    if (!st->exch_hi)
                        copy_cell(st, hi, shi, 1, 1, 1);
                }
            }
    /* y front: symmetry with thermo recomputed from mirrored T, p, Y (:647-679);
     * ODW with a wall start (this build's addition): ahead of it the ghosts
     * take the freestream, the first row of the inflow tables */
    for (int i = bc; i < ni + bc; i++)
        for (int j = 0; j < bc; j++)
            for (int k = bc; k < nk + bc; k++) {
                const long d = IDX(st, i, j, k);
                if (st->bc_kind == 2 && i - bc < st->wall_i0 && st->inflow) {
                    const long nt = (long)nj * nk, t = (long)(k - bc);
                    const double *f = st->inflow;
                    st->P[d] = f[0 * nt + t];
                    st->D[d] = f[1 * nt + t];
                    st->T[d] = f[2 * nt + t];
                    st->U[d] = f[3 * nt + t];
                    st->V[d] = f[4 * nt + t];
                    st->W[d] = f[5 * nt + t];
                    st->H[d] = f[6 * nt + t];
                    st->G[d] = f[7 * nt + t];
                    st->E[d] = f[8 * nt + t];
                    for (int s = 0; s < st->ns; s++) st->Y[s * st->n3 + d] = f[(9 + s) * nt + t];
                } else {
                    rebuild_cell(st, d, IDX(st, i, 2 * bc - 1 - j, k), -1);
                }
            }
    /* y back: zero-gradient mirror copy (:684-705) */
    for (int i = bc; i < ni + bc; i++)
        for (int j = nj + bc; j < nj + 2 * bc; j++)
            for (int k = bc; k < nk + bc; k++)
                copy_cell(st, IDX(st, i, j, k), IDX(st, i, 2 * (nj + bc) - 1 - j, k), 1, 1, 1);
    /* z: mirror copy with W reflected (:710-802); ODW rebuilds the thermo
     * there as well (:524-585) */
    for (int i = bc; i < ni + bc; i++)
        for (int j = bc; j < nj + bc; j++)
            for (int k = 0; k < bc; k++) {
                const long lo = IDX(st, i, j, k), slo = IDX(st, i, j, 2 * bc - 1 - k);
                const long hi = IDX(st, i, j, nk + bc + k), shi = IDX(st, i, j, 2 * (nk + bc) - 1 - (nk + bc + k));
                if (st->bc_kind == 2) {
                    rebuild_cell_w(st, lo, slo, 1, -1);
                    rebuild_cell_w(st, hi, shi, 1, -1);
                } else {
                    copy_cell(st, lo, slo, 1, 1, -1);
                    copy_cell(st, hi, shi, 1, 1, -1);
                }
            }
}

/* ----------------------------------------------------- threaded phases */

typedef struct {
    eo_state *st;
    int phase, t0, t1;
} eo_job;

static void *run_job(void *arg)
{
    eo_job *jb = (eo_job *)arg;
    eo_state *st = jb->st;
    const int bc = st->bc, nj = st->nj, nk = st->nk, ns = st->ns;
    const long n3 = st->n3;
    for (int i = jb->t0; i < jb->t1; i++) {
        if (jb->phase == 0) {
            /* face fluxes at faces i+1/2 for this x index (faces bc-1 .. ni+bc-1) */
            for (int j = bc; j < nj + bc; j++)
                for (int k = bc; k < nk + bc; k++) {
                    const long c = IDX(st, i, j, k);
                    face_flux(st, 1, c, (long)st->ny * st->nz);
                    if (i >= bc) {
                        face_flux(st, 2, c, st->nz);
                        face_flux(st, 3, c, 1);
                        if (j == bc)
                            face_flux(st, 2, c - st->nz, st->nz);
                        if (k == bc)
                            face_flux(st, 3, c - 1, 1);
                    }
                }
        } else if (jb->phase == 1) {
            /* TimeAdv::EE (src/TimeAdv.cpp:42-56) + CS += RHS (src/Flowfield.cpp:1350-1354)
             * + Update_after_CS (src/Flowfield.cpp:1579-1617) */
            const double dt = st->dt;
            for (int j = bc; j < nj + bc; j++)
                for (int k = bc; k < nk + bc; k++) {
                    const long c = IDX(st, i, j, k);
                    const long cx = (long)st->ny * st->nz, cy = st->nz;
                    for (int s = 0; s < ns + 4; s++) {
                        const double *F = st->flux[0] + s * n3, *G = st->flux[1] + s * n3, *Q = st->flux[2] + s * n3;
                        const double rhs = -dt / (st->x[i] - st->x[i - 1]) * (F[c] - F[c - cx]) -
                                           dt / (st->y[j] - st->y[j - 1]) * (G[c] - G[c - cy]) -
                                           dt / (st->z[k] - st->z[k - 1]) * (Q[c] - Q[c - 1]);
                        st->CS[s * n3 + c] = st->CS[s * n3 + c] + rhs;
                    }
                    update_after_cs(st, c);
                }
        } else if (jb->phase == 3) {
            /* RK stage: CS += RHS alone (the recovery follows the combination) */
            const double dt = st->dt;
            for (int j = bc; j < nj + bc; j++)
                for (int k = bc; k < nk + bc; k++) {
                    const long c = IDX(st, i, j, k);
                    const long cx = (long)st->ny * st->nz, cy = st->nz;
                    for (int s = 0; s < ns + 4; s++) {
                        const double *F = st->flux[0] + s * n3, *G = st->flux[1] + s * n3, *Q = st->flux[2] + s * n3;
                        const double rhs = -dt / (st->x[i] - st->x[i - 1]) * (F[c] - F[c - cx]) -
                                           dt / (st->y[j] - st->y[j - 1]) * (G[c] - G[c - cy]) -
                                           dt / (st->z[k] - st->z[k - 1]) * (Q[c] - Q[c - 1]);
                        st->CS[s * n3 + c] = st->CS[s * n3 + c] + rhs;
                    }
                }
        } else if (jb->phase == 4) {
            /* RK stage combination CS = a CS0 + b CS (Shu-Osher form), then
             * Update_after_CS */
            for (int j = bc; j < nj + bc; j++)
                for (int k = bc; k < nk + bc; k++) {
                    const long c = IDX(st, i, j, k);
                    if (st->rk_a != 0)
                        for (int s = 0; s < ns + 4; s++)
                            st->CS[s * n3 + c] = st->rk_a * st->cs0[s * n3 + c] + st->rk_b * st->CS[s * n3 + c];
                    update_after_cs(st, c);
                }
        } else {
            for (int j = bc; j < nj + bc; j++)
                for (int k = bc; k < nk + bc; k++) react_cell(st, IDX(st, i, j, k));
        }
    }
    return NULL;
}

static void run_phase(eo_state *st, int phase, int i0, int i1)
{
    int nt = st->nthreads;
    if (nt > i1 - i0)
        nt = i1 - i0;
    if (nt <= 1) {
        eo_job jb = {st, phase, i0, i1};
        run_job(&jb);
        return;
    }
    pthread_t th[64];
    eo_job jobs[64];
    if (nt > 64)
        nt = 64;
    for (int t = 0; t < nt; t++) {
        jobs[t].st = st;
        jobs[t].phase = phase;
        jobs[t].t0 = i0 + (int)((long)(i1 - i0) * t / nt);
        jobs[t].t1 = i0 + (int)((long)(i1 - i0) * (t + 1) / nt);
        pthread_create(&th[t], NULL, run_job, &jobs[t]);
    }
    for (int t = 0; t < nt; t++) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------ API */

eo_state *eo_create(int ni, int nj, int nk, int bc, const double *x, const double *y, const double *z,
                    const eo_mechanism *m, int nthreads)
{
    if (m->ns > EO_MAXS || m->nr > EO_MAXR || bc < 2)
        return NULL;
    eo_state *st = (eo_state *)calloc(1, sizeof(eo_state));
    st->ni = ni;
    st->nj = nj;
    st->nk = nk;
    st->bc = bc;
    st->nx = ni + 2 * bc;
    st->ny = nj + 2 * bc;
    st->nz = nk + 2 * bc;
    st->n3 = (long)st->nx * st->ny * st->nz;
    st->ns = m->ns;
    st->nr = m->nr;
    st->nthreads = nthreads < 1 ? 1 : nthreads;
    st->x = (double *)malloc(sizeof(double) * st->nx);
    st->y = (double *)malloc(sizeof(double) * st->ny);
    st->z = (double *)malloc(sizeof(double) * st->nz);
    memcpy(st->x, x, sizeof(double) * st->nx);
    memcpy(st->y, y, sizeof(double) * st->ny);
    memcpy(st->z, z, sizeof(double) * st->nz);
    for (int s = 0; s < m->ns; s++) {
        st->mw[s] = m->mw[s];
        st->ri[s] = R_UNIV / m->mw[s]; /* src/Reaction.cpp:426-427 */
    }
    memcpy(st->clo, m->coeff_lo, sizeof(double) * 9 * m->ns);
    memcpy(st->chi, m->coeff_hi, sizeof(double) * 9 * m->ns);
    memcpy(st->af, m->af, sizeof(double) * m->nr);
    memcpy(st->bf, m->bf, sizeof(double) * m->nr);
    memcpy(st->eaf, m->eaf, sizeof(double) * m->nr);
    memcpy(st->sf, m->stoi_f, sizeof(double) * m->ns * m->nr);
    memcpy(st->sb, m->stoi_b, sizeof(double) * m->ns * m->nr);
    memcpy(st->tb, m->tb, sizeof(double) * m->ns * m->nr);
    const long n3 = st->n3;
    double **one[] = {&st->P, &st->D, &st->U, &st->V, &st->W, &st->H, &st->G, &st->T, &st->E};
    for (unsigned q = 0; q < sizeof(one) / sizeof(one[0]); q++) *one[q] = (double *)calloc(n3, sizeof(double));
    st->Y = (double *)calloc(n3 * st->ns, sizeof(double));
    st->CS = (double *)calloc(n3 * (st->ns + 4), sizeof(double));
    st->cms = (double *)calloc(n3 * st->ns, sizeof(double));
    for (int d = 0; d < 3; d++) st->flux[d] = (double *)calloc(n3 * (st->ns + 4), sizeof(double));
    st->nchem = (int *)calloc(n3, sizeof(int));
    return st;
}

void eo_destroy(eo_state *st)
{
    if (!st)
        return;
    double *bufs[] = {st->x, st->y, st->z, st->P, st->D, st->U, st->V, st->W, st->H, st->G, st->T, st->E,
                      st->Y, st->CS, st->cms, st->flux[0], st->flux[1], st->flux[2]};
    for (unsigned q = 0; q < sizeof(bufs) / sizeof(bufs[0]); q++) free(bufs[q]);
    free(st->nchem);
    free(st->inflow);
    free(st->cs0);
    free(st);
}

void eo_set_primitive(eo_state *st, const double *P, const double *T, const double *U, const double *V,
                      const double *W, const double *Y)
{
    const int ns = st->ns, bc = st->bc;
    const long n3 = st->n3;
    memcpy(st->P, P, n3 * sizeof(double));
    memcpy(st->T, T, n3 * sizeof(double));
    memcpy(st->U, U, n3 * sizeof(double));
    memcpy(st->V, V, n3 * sizeof(double));
    memcpy(st->W, W, n3 * sizeof(double));
    memcpy(st->Y, Y, n3 * ns * sizeof(double));
    /* Flowfield::FieldInitial derived quantities, src/Flowfield.cpp:226-262 */
    for (int i = bc; i < st->ni + bc; i++)
        for (int j = bc; j < st->nj + bc; j++)
            for (int k = bc; k < st->nk + bc; k++) {
                const long c = IDX(st, i, j, k);
                double inv_w = 0, cp = 0, h = 0, e = 0;
                double Yc[EO_MAXS], Cpi[EO_MAXS], Hi[EO_MAXS], Ei[EO_MAXS];
                for (int s = 0; s < ns; s++) Yc[s] = st->Y[s * n3 + c];
                for (int s = 0; s < ns; s++) inv_w += Yc[s] / st->mw[s];
                const double Wav = 1.0 / inv_w;
                const double Rgas = R_UNIV * 1000 / Wav;
                const double Tc = st->T[c];
                const double D = st->P[c] / (Rgas * Tc);
                st->D[c] = D;
                for (int s = 0; s < ns; s++) {
                    Cpi[s] = get_cpi(st, Tc, st->ri[s], s);
                    Hi[s] = get_hi(st, Tc, st->ri[s], s);
                    Ei[s] = Hi[s] - st->ri[s] * Tc;
                }
                for (int s = 0; s < ns; s++) cp += Cpi[s] * Yc[s];
                for (int s = 0; s < ns; s++) h += Yc[s] * Hi[s];
                for (int s = 0; s < ns; s++) e += Yc[s] * Ei[s];
                const double Cp = cp * 1000;
                st->H[c] = h * 1000;
                st->E[c] = e * 1000;
                st->G[c] = Cp / (Cp - R_UNIV * inv_w * 1000);
                for (int s = 0; s < ns; s++) st->CS[s * n3 + c] = D * Yc[s];
                st->CS[(ns + 0) * n3 + c] = D * st->U[c];
                st->CS[(ns + 1) * n3 + c] = D * st->V[c];
                st->CS[(ns + 2) * n3 + c] = D * st->W[c];
                st->CS[(ns + 3) * n3 + c] =
                    D * st->E[c] + 0.5 * (pow(st->U[c], 2) + pow(st->V[c], 2) + pow(st->W[c], 2)) * D;
            }
}

void eo_set_state(eo_state *st, const double *cs, const double *T, const double *E, const double *P,
                  const double *D, const double *U, const double *V, const double *W, const double *H,
                  const double *G, const double *Y)
{
    const long n3 = st->n3;
    const int ns = st->ns;
    memcpy(st->CS, cs, n3 * (ns + 4) * sizeof(double));
    memcpy(st->Y, Y, n3 * ns * sizeof(double));
    const double *src[] = {T, E, P, D, U, V, W, H, G};
    double *dst[] = {st->T, st->E, st->P, st->D, st->U, st->V, st->W, st->H, st->G};
    for (int q = 0; q < 9; q++) memcpy(dst[q], src[q], n3 * sizeof(double));
}

void eo_boundary(eo_state *st) { boundary_fill(st); }

void eo_set_boundary(eo_state *st, int kind) { st->bc_kind = kind; }

void eo_set_wall(eo_state *st, int first_wall_node) { st->wall_i0 = first_wall_node; }

void eo_set_inflow(eo_state *st, const double *P, const double *T, const double *U, const double *V,
                   const double *W, const double *Y)
{
    const int ns = st->ns, nj = st->nj, nk = st->nk;
    const long nt = (long)nj * nk;
    free(st->inflow);
    st->inflow = (double *)calloc((size_t)(9 + ns) * nt, sizeof(double));
    double *f = st->inflow;
    for (long t = 0; t < nt; t++) {
        /* Flowfield::FieldInitial's derived quantities (src/Flowfield.cpp:226-262) */
        double Yc[EO_MAXS], inv_w = 0, cp = 0, h = 0, e = 0;
        for (int s = 0; s < ns; s++) Yc[s] = Y[s * nt + t];
        for (int s = 0; s < ns; s++) inv_w += Yc[s] / st->mw[s];
        const double Wav = 1.0 / inv_w;
        const double Rgas = R_UNIV * 1000 / Wav;
        const double Tc = T[t];
        for (int s = 0; s < ns; s++) {
            const double Hs = get_hi(st, Tc, st->ri[s], s);
            cp += get_cpi(st, Tc, st->ri[s], s) * Yc[s];
            h += Yc[s] * Hs;
            e += Yc[s] * (Hs - st->ri[s] * Tc);
        }
        const double Cp = cp * 1000;
        f[0 * nt + t] = P[t];
        f[1 * nt + t] = P[t] / (Rgas * Tc);
        f[2 * nt + t] = Tc;
        f[3 * nt + t] = U[t];
        f[4 * nt + t] = V[t];
        f[5 * nt + t] = W[t];
        f[6 * nt + t] = h * 1000;
        f[7 * nt + t] = Cp / (Cp - R_UNIV * inv_w * 1000);
        f[8 * nt + t] = e * 1000;
        for (int s = 0; s < ns; s++) f[(9 + s) * nt + t] = Yc[s];
    }
}

void eo_set_exchange(eo_state *st, int x_low, int x_high)
{
    st->exch_lo = x_low != 0;
    st->exch_hi = x_high != 0;
}

/* Halo messages between x blocks (Flowfield::Mpi_Boundary, src/Flowfield.cpp:809-911):
 * [field][plane][j][k] over full haloed planes, fields P D U V W H Gamma Y_0..Y_ns-1.
 * Pack face 0 takes nodes bc+1+p (the reference's bc+1+i), face 1 nodes ni+bc-2-p
 * (its ni-i for bc = 2); unpack face 0 fills ghost nodes bc-1-p, face 1 ni+bc+p. */
static double *halo_field(eo_state *st, int f)
{
    double *one[7] = {st->P, st->D, st->U, st->V, st->W, st->H, st->G};
    return f < 7 ? one[f] : st->Y + (long)(f - 7) * st->n3;
}

static void halo_copy(eo_state *st, int face, int pack, double *msg)
{
    const long plane = (long)st->ny * st->nz;
    const int bc = st->bc, ni = st->ni;
    for (int f = 0; f < 7 + st->ns; f++)
        for (int p = 0; p < bc; p++) {
            int i;
            if (pack)
                i = face == 0 ? bc + 1 + p : ni + bc - 2 - p;
            else
                i = face == 0 ? bc - 1 - p : ni + bc + p;
            double *node = halo_field(st, f) + (long)i * plane;
            double *m = msg + ((long)f * bc + p) * plane;
            if (pack)
                memcpy(m, node, plane * sizeof(double));
            else
                memcpy(node, m, plane * sizeof(double));
        }
}

long eo_halo_count(const eo_state *st) { return (long)(7 + st->ns) * st->bc * st->ny * st->nz; }
void eo_halo_pack(eo_state *st, int face, double *msg) { halo_copy(st, face, 1, msg); }
void eo_halo_unpack(eo_state *st, int face, const double *msg) { halo_copy(st, face, 0, (double *)msg); }

/* The three-stage TVD Runge-Kutta advection of the timestep (Shu and Osher's
 * SSP-RK3; the reference's TimeAdv::TVD_RK3, src/TimeAdv.cpp:210-221, is an
 * empty stub): U1 = U0 + dt L(U0), U2 = 3/4 U0 + 1/4 (U1 + dt L(U1)),
 * U3 = 1/3 U0 + 2/3 (U2 + dt L(U2)), each stage with its own ghost fill and
 * state recovery; the chemistry then runs once on U3, as after the Euler
 * stage. */
static void rk3_advection(eo_state *st)
{
    const int bc = st->bc, ni = st->ni;
    memcpy(st->cs0, st->CS, (size_t)st->n3 * (st->ns + 4) * sizeof(double));
    static const double a[3] = {0.0, 0.75, 1.0 / 3.0}, b[3] = {1.0, 0.25, 2.0 / 3.0};
    for (int q = 0; q < 3; q++) {
        boundary_fill(st);
        run_phase(st, 0, bc - 1, ni + bc); /* faces */
        run_phase(st, 3, bc, ni + bc);     /* CS += RHS */
        st->rk_a = a[q];
        st->rk_b = b[q];
        run_phase(st, 4, bc, ni + bc);     /* combination + state recovery */
    }
}

void eo_set_scheme(eo_state *st, int scheme)
{
    st->scheme = scheme;
    if (scheme == 1 && !st->cs0)
        st->cs0 = (double *)calloc((size_t)st->n3 * (st->ns + 4), sizeof(double));
}

int eo_step(eo_state *st, int nsteps, double dt)
{
    const int bc = st->bc, ni = st->ni;
    for (int n = 0; n < nsteps; n++) {
        st->dt = dt;
        if (st->scheme == 1) {
            rk3_advection(st);
        } else {
            boundary_fill(st);
            run_phase(st, 0, bc - 1, ni + bc); /* faces */
            run_phase(st, 1, bc, ni + bc);     /* EE update + state recovery */
        }
        run_phase(st, 2, bc, ni + bc);     /* chemistry */
        if (st->bad_nchem)
            return -1;
    }
    return 0;
}

int eo_get(const eo_state *st, const char *name, double *out)
{
    const long n3 = st->n3;
    const int ns = st->ns;
    const double *one = NULL;
    if (!strcmp(name, "P")) one = st->P;
    else if (!strcmp(name, "D")) one = st->D;
    else if (!strcmp(name, "T")) one = st->T;
    else if (!strcmp(name, "U")) one = st->U;
    else if (!strcmp(name, "V")) one = st->V;
    else if (!strcmp(name, "W")) one = st->W;
    else if (!strcmp(name, "H")) one = st->H;
    else if (!strcmp(name, "E")) one = st->E;
    else if (!strcmp(name, "Gamma")) one = st->G;
    if (one) {
        memcpy(out, one, n3 * sizeof(double));
        return 1;
    }
    if (!strcmp(name, "Yi")) {
        memcpy(out, st->Y, n3 * ns * sizeof(double));
        return ns;
    }
    if (!strcmp(name, "Di")) {
        memcpy(out, st->CS, n3 * ns * sizeof(double));
        return ns;
    }
    if (!strcmp(name, "CS")) {
        memcpy(out, st->CS, n3 * (ns + 4) * sizeof(double));
        return ns + 4;
    }
    if (!strcmp(name, "CMS")) {
        memcpy(out, st->cms, n3 * ns * sizeof(double));
        return ns;
    }
    if (!strcmp(name, "Mc")) {
        for (int s = 0; s < ns; s++)
            for (long c = 0; c < n3; c++) out[s * n3 + c] = st->CS[s * n3 + c] / st->mw[s] * 1000;
        return ns;
    }
    if (!strcmp(name, "Nchem")) {
        for (long c = 0; c < n3; c++) out[c] = st->nchem[c];
        return 1;
    }
    /* Derived outputs of Update_after_CS (src/Flowfield.cpp:1606-1616) from the stored state. */
    if (!strcmp(name, "Wav") || !strcmp(name, "Rgas") || !strcmp(name, "Cp") || !strcmp(name, "C") ||
        !strcmp(name, "Ma")) {
        for (long c = 0; c < n3; c++) {
            double inv_w = 0, cp = 0;
            for (int s = 0; s < ns; s++) inv_w += st->Y[s * n3 + c] / st->mw[s];
            const double Wav = 1.0 / inv_w;
            double v = 0;
            if (!strcmp(name, "Wav")) v = Wav;
            else if (!strcmp(name, "Rgas")) v = R_UNIV * 1000 / Wav;
            else if (!strcmp(name, "Cp")) {
                for (int s = 0; s < ns; s++) cp += get_cpi(st, st->T[c], st->ri[s], s) * st->Y[s * n3 + c];
                v = cp * 1000;
            } else {
                const double C = sqrt(st->G[c] * st->P[c] / st->D[c]);
                v = !strcmp(name, "C") ? C
                                       : sqrt(pow(st->U[c], 2) + pow(st->V[c], 2) + pow(st->W[c], 2)) / C;
            }
            out[c] = v;
        }
        return 1;
    }
    return -1;
}

void eo_thermo(const eo_state *st, double T, double R, int s, double *cp_h_s)
{
    cp_h_s[0] = get_cpi(st, T, R, s);
    cp_h_s[1] = get_hi(st, T, R, s);
    cp_h_s[2] = get_si(st, T, R, s);
}

void eo_muscl(const double f[4], double *left, double *right) { muscl_face(f, left, right); }

void eo_ausm(const eo_state *st, const double lr[14], const double *yl, const double *yr, int dir, double *out)
{
    ausm_face(st->ns, dir, lr[0], lr[7], lr[1], lr[8], lr[2], lr[9], lr[3], lr[10], lr[4], lr[11], lr[5], lr[12],
              lr[6], lr[13], yl, yr, out, 1);
}

double eo_temperature(const eo_state *st, double T0, double E, const double *Y) { return get_temp(st, T0, E, Y); }
