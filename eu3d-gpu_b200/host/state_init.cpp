// state_init.cpp — Flowfield::FieldInitial's derived quantities on the host.
#include "state_init.hpp"

#include <cmath>
#include <cstring>

namespace eu3d {

namespace {
constexpr double kR = 8.31434;       // include/Flowfield.hpp:57
constexpr double kSwitch = 1000.0;   // include/ThermoConstants.hpp:3

// Reaction::GetCpi / GetHi (src/Reaction.cpp:1165-1199), same expression order.
double cpi(const MechanismTables &m, double T, double R, int sp)
{
    const double *c = T < kSwitch ? m.coeff_lo.data() : m.coeff_hi.data();
    const int ns = m.ns;
    return R * (c[0 * ns + sp] * std::pow(T, -2) + c[1 * ns + sp] * std::pow(T, -1) + c[2 * ns + sp] +
                c[3 * ns + sp] * T + c[4 * ns + sp] * std::pow(T, 2) + c[5 * ns + sp] * std::pow(T, 3) +
                c[6 * ns + sp] * std::pow(T, 4));
}

double hi(const MechanismTables &m, double T, double R, int sp)
{
    const double *c = T < kSwitch ? m.coeff_lo.data() : m.coeff_hi.data();
    const int ns = m.ns;
    return R * (-c[0 * ns + sp] * std::pow(T, -1) + c[1 * ns + sp] * std::log(T) + c[2 * ns + sp] * T +
                c[3 * ns + sp] * std::pow(T, 2) / 2 + c[4 * ns + sp] * std::pow(T, 3) / 3 +
                c[5 * ns + sp] * std::pow(T, 4) / 4 + c[6 * ns + sp] * std::pow(T, 5) / 5 + c[7 * ns + sp]);
}
} // namespace

void primitive_to_state(const MechanismTables &m, int ni, int nj, int nk, int bc, const double *P, const double *T,
                        const double *U, const double *V, const double *W, const double *Y, std::vector<double> &prim,
                        std::vector<double> &cs, std::vector<double> &Tout, std::vector<double> &Eout)
{
    const int ns = m.ns;
    const int nx = ni + 2 * bc, ny = nj + 2 * bc, nz = nk + 2 * bc;
    const long long n3 = (long long)nx * ny * nz;
    prim.assign((7 + ns) * n3, 0.0);
    cs.assign((ns + 4) * n3, 0.0);
    Tout.assign(T, T + n3);
    Eout.assign(n3, 0.0);
    std::memcpy(&prim[0 * n3], P, n3 * sizeof(double));
    std::memcpy(&prim[2 * n3], U, n3 * sizeof(double));
    std::memcpy(&prim[3 * n3], V, n3 * sizeof(double));
    std::memcpy(&prim[4 * n3], W, n3 * sizeof(double));
    std::memcpy(&prim[7 * n3], Y, ns * n3 * sizeof(double));
    std::vector<double> ri(ns), Yc(ns), Cpi(ns), Hi(ns), Ei(ns);
    for (int s = 0; s < ns; s++) ri[s] = kR / m.mw[s];
    for (int i = bc; i < ni + bc; i++)
        for (int j = bc; j < nj + bc; j++)
            for (int k = bc; k < nk + bc; k++) {
                const long long c = ((long long)i * ny + j) * nz + k;
                double inv_w = 0, cp = 0, h = 0, e = 0;
                for (int s = 0; s < ns; s++) Yc[s] = Y[s * n3 + c];
                for (int s = 0; s < ns; s++) inv_w += Yc[s] / m.mw[s];
                const double Wav = 1.0 / inv_w;
                const double Rgas = kR * 1000 / Wav;
                const double Tc = T[c];
                const double D = P[c] / (Rgas * Tc);
                for (int s = 0; s < ns; s++) {
                    Cpi[s] = cpi(m, Tc, ri[s], s);
                    Hi[s] = hi(m, Tc, ri[s], s);
                    Ei[s] = Hi[s] - ri[s] * Tc;
                }
                for (int s = 0; s < ns; s++) cp += Cpi[s] * Yc[s];
                for (int s = 0; s < ns; s++) h += Yc[s] * Hi[s];
                for (int s = 0; s < ns; s++) e += Yc[s] * Ei[s];
                const double Cp = cp * 1000;
                const double E = e * 1000;
                prim[1 * n3 + c] = D;
                prim[5 * n3 + c] = h * 1000;
                prim[6 * n3 + c] = Cp / (Cp - kR * inv_w * 1000);
                Eout[c] = E;
                for (int s = 0; s < ns; s++) cs[s * n3 + c] = D * Yc[s];
                cs[(ns + 0) * n3 + c] = D * U[c];
                cs[(ns + 1) * n3 + c] = D * V[c];
                cs[(ns + 2) * n3 + c] = D * W[c];
                cs[(ns + 3) * n3 + c] =
                    D * E + 0.5 * (std::pow(U[c], 2) + std::pow(V[c], 2) + std::pow(W[c], 2)) * D;
            }
}

} // namespace eu3d
