/*
 * Oracle harness around the reference's own CPU hot path (test infrastructure).
 *
 * The reference's Flowfield, Reaction and Mesh classes grant `friend class Euler`
 * (include/Flowfield.hpp:139, include/Reaction.hpp:140, include/Mesh.hpp:57).
 * This file supplies its own small `class Euler` so that it can
 *   - build the objects exactly as Euler::Euler does (src/Euler.cpp:59-97),
 *   - inject arbitrary initial primitive fields (the reference hard-codes RSBI),
 *   - run the per-timestep hot path of Euler::Computing (src/Euler.cpp:322-376)
 *     with the CPU branch of Euler::Trapezoid(1) (src/Euler.cpp:443-493),
 * and exposes that through a small C API that tests load with ctypes.
 * Every arithmetic line of the step is the reference's own code.
 */
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "Flowfield.hpp"
#include "Global.hpp"
#include "Mesh.hpp"
#include "Reaction.hpp"

namespace {
/* Discards the reference's per-step progress prints while the harness runs it. */
struct QuietCout {
    std::streambuf *saved;
    std::ostringstream sink;
    QuietCout() : saved(std::cout.rdbuf(sink.rdbuf())) {}
    ~QuietCout() { std::cout.rdbuf(saved); }
};

void single_rank_globals()
{
    /* What src/Main.cpp + Euler::Mpi_Initial (src/Euler.cpp:236-293) leave for 1 rank. */
    myid = 0;
    numprocs = 1;
    m_block_x = m_block_y = m_block_z = 1;
    myid_x = myid_y = myid_z = 0;
    m_left = m_right = m_front = m_back = m_down = m_up = -1;
    num_thread = 1;
}
} // namespace

class Euler {
public:
    Mesh mesh;
    Flowfield flow;
    Reaction react;
    int steps_done = 0;

    Euler(const char *grid, const char *input, const char *mech, const char *thermo)
    {
        QuietCout quiet;
        single_rank_globals();
        std::vector<char> g(grid, grid + std::strlen(grid) + 1), in(input, input + std::strlen(input) + 1),
            me(mech, mech + std::strlen(mech) + 1), th(thermo, thermo + std::strlen(thermo) + 1);
        /* src/Euler.cpp:71, :83, :87, :91 */
        mesh.MeshProcess(g.data());
        flow.InputRead(in.data(), mesh.xnode, mesh.ynode, mesh.znode, mesh.bc);
        react.ReactionRead(me.data(), th.data(), mesh.xnode, mesh.ynode, mesh.znode, mesh.bc);
        flow.FieldInitial(react.Ri, react.Mw, react.Mi, react.Yi, react.Coeff0, react.Coeff1);
        react.Nchem.Fill(0);
        react.CMS.Fill(0.0);
    }

    int nx() const { return mesh.ni + 2 * mesh.bc; }
    int ny() const { return mesh.nj + 2 * mesh.bc; }
    int nz() const { return mesh.nk + 2 * mesh.bc; }

    /*
     * Replace the initial condition with given primitive fields over the haloed
     * grid. Derived quantities are formed with the arithmetic of
     * Flowfield::FieldInitial (src/Flowfield.cpp:226-262) on interior nodes.
     */
    void set_primitive(const double *P, const double *T, const double *U, const double *V, const double *W,
                       const double *Y)
    {
        Flowfield &F = flow;
        const int NS = F.NS, bc = mesh.bc;
        const size_t n3 = size_t(nx()) * ny() * nz();
        for (size_t c = 0; c < n3; ++c) {
            F.P.Getbuf()[c] = P[c];
            F.T.Getbuf()[c] = T[c];
            F.U.Getbuf()[c] = U[c];
            F.V.Getbuf()[c] = V[c];
            F.W.Getbuf()[c] = W[c];
            for (int s = 0; s < NS; ++s) F.Yi.Getbuf()[c * NS + s] = Y[c * NS + s];
        }
        Function Fun;
        for (int i = bc; i < mesh.ni + bc; i++)
            for (int j = bc; j < mesh.nj + bc; j++)
                for (int k = bc; k < mesh.nk + bc; k++) {
                    Array<double, 1> Yt;
                    Yt.Initial(NS);
                    for (int s = 0; s < NS; s++) Yt(s) = F.Yi(i, j, k, s);
                    F.Wav(i, j, k) = 1.0 / Fun.sum(3, Yt, F.Mw);
                    F.Rgas(i, j, k) = F.R * 1000 / F.Wav(i, j, k);
                    F.D(i, j, k) = F.P(i, j, k) / (F.Rgas(i, j, k) * F.T(i, j, k));
                    for (int s = 0; s < NS; s++) {
                        F.Di(i, j, k, s) = F.Yi(i, j, k, s) * F.D(i, j, k);
                        F.Mc(i, j, k, s) = F.Di(i, j, k, s) / F.Mw(s) * 1000;
                        F.Cpi(s) = F.React.GetCpi(F.T(i, j, k), F.Ri(s), s, F.Coeff0, F.Coeff1);
                        F.Hi(s) = F.React.GetHi(F.T(i, j, k), F.Ri(s), s, F.Coeff0, F.Coeff1);
                        F.Ei(s) = F.Hi(s) - F.Ri(s) * F.T(i, j, k);
                    }
                    F.Cp(i, j, k) = Fun.sum(2, F.Cpi, Yt) * 1000;
                    F.H(i, j, k) = Fun.sum(2, Yt, F.Hi) * 1000;
                    F.E(i, j, k) = Fun.sum(2, Yt, F.Ei) * 1000;
                    F.Gamma(i, j, k) = F.Cp(i, j, k) / (F.Cp(i, j, k) - F.R * Fun.sum(3, Yt, F.Mw) * 1000);
                    F.C(i, j, k) = sqrt(F.Gamma(i, j, k) * F.P(i, j, k) / F.D(i, j, k));
                    for (int s = 0; s < NS; s++) F.CS(i, j, k, s) = F.D(i, j, k) * F.Yi(i, j, k, s);
                    F.CS(i, j, k, NS) = F.D(i, j, k) * F.U(i, j, k);
                    F.CS(i, j, k, NS + 1) = F.D(i, j, k) * F.V(i, j, k);
                    F.CS(i, j, k, NS + 2) = F.D(i, j, k) * F.W(i, j, k);
                    F.CS(i, j, k, NS + 3) =
                        F.D(i, j, k) * F.E(i, j, k) +
                        0.5 * (pow(F.U(i, j, k), 2) + pow(F.V(i, j, k), 2) + pow(F.W(i, j, k), 2)) * F.D(i, j, k);
                }
    }

    /* One reference timestep at fixed dt: src/Euler.cpp:327-376 with cfl==0,
     * then the CPU branch of Euler::Trapezoid(1), src/Euler.cpp:443-493. */
    void step(double dt)
    {
        QuietCout quiet;
        const int bc = mesh.bc;
        flow.dt = dt;
        fill_ghosts();
        flow.Mpi_Boundary();
        flow.Advection(0 /* EE */, 1 /* MUSCL_2 */);
        flow.Update_after_Adv();
        react.TrapezoidPrediction(flow.Mc, flow.Di, flow.Yi, flow.T, flow.dt);
        for (int i = bc; i < mesh.ni + bc; ++i)
            for (int j = bc; j < mesh.nj + bc; ++j)
                for (int k = bc; k < mesh.nk + bc; ++k)
                    for (int s = 0; s < react.Nchem(i, j, k); ++s) {
                        react.Trapezoid(flow.Mc, flow.Di, flow.Yi, flow.T, flow.dt, s, i, j, k);
                        flow.Explicit(s, i, j, k);
                    }
        react.PushNchemMax();
        ++steps_done;
    }

    /* The case's ghost fill: 0 FieldBoundary_3dRSBI (the one Euler::Computing
     * calls, src/Euler.cpp:348), 1 FieldBoundary_3dODW (src/Flowfield.cpp:412-592,
     * compiled but not called by the reference; its inflow tables come from
     * set_inflow). */
    int boundary_kind = 0;
    void fill_ghosts()
    {
        if (boundary_kind == 1)
            flow.FieldBoundary_3dODW();
        else
            flow.FieldBoundary_3dRSBI();
    }

    /* The boundary fill alone (used to check ghost handling in isolation). */
    void boundary() { QuietCout quiet; fill_ghosts(); }

    /* ODW inflow tables Uint .. Yint over the interior (j, k) nodes from
     * P, T, U, V, W and Y (planes of nj * nk, k fastest; Y: ns such planes),
     * the derived D, H, Gamma, E with FieldInitial's arithmetic
     * (src/Flowfield.cpp:226-262). The reference allocates these tables
     * (:138-147) but never fills them. */
    void set_inflow(const double *P, const double *T, const double *U, const double *V, const double *W,
                    const double *Y)
    {
        Flowfield &F = flow;
        const int NS = F.NS, nj = mesh.nj, nk = mesh.nk;
        Function Fun;
        for (int j = 0; j < nj; j++)
            for (int k = 0; k < nk; k++) {
                const size_t c = size_t(j) * nk + k;
                Array<double, 1> Yt;
                Yt.Initial(NS);
                for (int s = 0; s < NS; s++) Yt(s) = Y[s * size_t(nj) * nk + c];
                const double Wav = 1.0 / Fun.sum(3, Yt, F.Mw);
                const double Rgas = F.R * 1000 / Wav;
                const double D = P[c] / (Rgas * T[c]);
                for (int s = 0; s < NS; s++) {
                    F.Cpi(s) = F.React.GetCpi(T[c], F.Ri(s), s, F.Coeff0, F.Coeff1);
                    F.Hi(s) = F.React.GetHi(T[c], F.Ri(s), s, F.Coeff0, F.Coeff1);
                    F.Ei(s) = F.Hi(s) - F.Ri(s) * T[c];
                }
                const double Cp = Fun.sum(2, F.Cpi, Yt) * 1000;
                F.Uint(j, k) = U[c];
                F.Vint(j, k) = V[c];
                F.Wint(j, k) = W[c];
                F.Pint(j, k) = P[c];
                F.Dint(j, k) = D;
                F.Tint(j, k) = T[c];
                F.Hint(j, k) = Fun.sum(2, Yt, F.Hi) * 1000;
                F.Eint(j, k) = Fun.sum(2, Yt, F.Ei) * 1000;
                F.Gint(j, k) = Cp / (Cp - F.R * Fun.sum(3, Yt, F.Mw) * 1000);
                for (int s = 0; s < NS; s++) F.Yint(j, k, s) = Yt(s);
            }
    }

    Array<double, 3> *field3(const std::string &n)
    {
        Flowfield &F = flow;
        if (n == "P") return &F.P;
        if (n == "D") return &F.D;
        if (n == "T") return &F.T;
        if (n == "U") return &F.U;
        if (n == "V") return &F.V;
        if (n == "W") return &F.W;
        if (n == "H") return &F.H;
        if (n == "E") return &F.E;
        if (n == "Gamma") return &F.Gamma;
        if (n == "C") return &F.C;
        if (n == "Ma") return &F.Ma;
        if (n == "Wav") return &F.Wav;
        if (n == "Rgas") return &F.Rgas;
        if (n == "Cp") return &F.Cp;
        return nullptr;
    }
    Array<double, 4> *field4(const std::string &n)
    {
        Flowfield &F = flow;
        if (n == "Yi") return &F.Yi;
        if (n == "Di") return &F.Di;
        if (n == "Mc") return &F.Mc;
        if (n == "CS") return &F.CS;
        if (n == "CMS") return &react.CMS;
        return nullptr;
    }

    void dims(int *out7)
    {
        out7[0] = mesh.ni;
        out7[1] = mesh.nj;
        out7[2] = mesh.nk;
        out7[3] = mesh.bc;
        out7[4] = react.NS;
        out7[5] = react.NR;
        out7[6] = react.TB;
    }

    long get(const std::string &n, double *out)
    {
        if (auto *a = field3(n)) { std::memcpy(out, a->Getbuf(), a->GetLen() * sizeof(double)); return long(a->GetLen()); }
        if (auto *a = field4(n)) { std::memcpy(out, a->Getbuf(), a->GetLen() * sizeof(double)); return long(a->GetLen()); }
        if (n == "Nchem") {
            auto &a = react.Nchem;
            for (size_t c = 0; c < a.GetLen(); ++c) out[c] = a.Getbuf()[c];
            return long(a.GetLen());
        }
        Array<double, 1> *v1 = nullptr;
        if (n == "xnode") v1 = &mesh.xnode;
        if (n == "ynode") v1 = &mesh.ynode;
        if (n == "znode") v1 = &mesh.znode;
        if (n == "Mw") v1 = &react.Mw;
        if (n == "Ri") v1 = &react.Ri;
        if (n == "Af") v1 = &react.Af;
        if (n == "Bf") v1 = &react.Bf;
        if (n == "Eaf") v1 = &react.Eaf;
        if (v1) { std::memcpy(out, v1->Getbuf(), v1->GetLen() * sizeof(double)); return long(v1->GetLen()); }
        Array<double, 2> *v2 = nullptr;
        if (n == "Coeff0") v2 = &react.Coeff0;   /* (9, NS) row-major */
        if (n == "Coeff1") v2 = &react.Coeff1;
        if (n == "Stoi_F") v2 = &react.Stoi_F;   /* (NS, NR) row-major */
        if (n == "Stoi_B") v2 = &react.Stoi_B;
        if (n == "React_TB") v2 = &react.React_TB;
        if (v2) { std::memcpy(out, v2->Getbuf(), v2->GetLen() * sizeof(double)); return long(v2->GetLen()); }
        return -1;
    }

    long put(const std::string &n, const double *in)
    {
        if (auto *a = field3(n)) { std::memcpy(a->Getbuf(), in, a->GetLen() * sizeof(double)); return long(a->GetLen()); }
        if (auto *a = field4(n)) { std::memcpy(a->Getbuf(), in, a->GetLen() * sizeof(double)); return long(a->GetLen()); }
        return -1;
    }

    void thermo(double T, double R, int s, double *cp_h_s)
    {
        cp_h_s[0] = react.GetCpi(T, R, s, react.Coeff0, react.Coeff1);
        cp_h_s[1] = react.GetHi(T, R, s, react.Coeff0, react.Coeff1);
        cp_h_s[2] = react.GetSi(T, R, s, react.Coeff0, react.Coeff1);
    }
};

extern "C" {

void *ref_create(const char *grid, const char *input, const char *mech, const char *thermo)
{
    try {
        return new Euler(grid, input, mech, thermo);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_create: %s\n", e.what());
        return nullptr;
    }
}

void ref_destroy(void *h) { delete static_cast<Euler *>(h); }

/* ni, nj, nk (interior nodes), bc, NS, NR, TB */
void ref_dims(void *h, int *out7) { static_cast<Euler *>(h)->dims(out7); }

/* Copy a named field out, in the reference's layout: (i,j,k) row-major with k
 * fastest over the haloed grid; species fields (i,j,k,s) with s fastest.
 * Returns the element count copied, or -1 for an unknown name. */
long ref_get(void *h, const char *name, double *out) { return static_cast<Euler *>(h)->get(name, out); }

/* Overwrite a named 3-D/4-D field (same layout as ref_get). */
long ref_put(void *h, const char *name, const double *in) { return static_cast<Euler *>(h)->put(name, in); }

void ref_set_primitive(void *h, const double *P, const double *T, const double *U, const double *V,
                       const double *W, const double *Y)
{
    static_cast<Euler *>(h)->set_primitive(P, T, U, V, W, Y);
}

void ref_step(void *h, int nsteps, double dt)
{
    Euler *e = static_cast<Euler *>(h);
    for (int n = 0; n < nsteps; ++n) e->step(dt);
}

void ref_boundary(void *h) { static_cast<Euler *>(h)->boundary(); }

/* Ghost fill used by ref_step / ref_boundary: 0 RSBI (default), 1 ODW. */
void ref_set_boundary(void *h, int kind) { static_cast<Euler *>(h)->boundary_kind = kind; }

/* ODW inflow tables from interior (j, k) planes (k fastest). */
void ref_set_inflow(void *h, const double *P, const double *T, const double *U, const double *V, const double *W,
                    const double *Y)
{
    static_cast<Euler *>(h)->set_inflow(P, T, U, V, W, Y);
}

/* NASA thermo of one species at one temperature through the reference's own
 * Reaction::GetCpi/GetHi/GetSi (src/Reaction.cpp:1165-1220); R is the gas
 * constant the caller passes (Ri(s) in the flow solver, universal R in kinetics). */
void ref_thermo(void *h, double T, double R, int s, double *cp_h_s)
{
    static_cast<Euler *>(h)->thermo(T, R, s, cp_h_s);
}

} // extern "C"
