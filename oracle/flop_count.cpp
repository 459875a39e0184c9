// flop_count.cpp — TEST INFRASTRUCTURE ONLY (never linked into the library).
//
// The C restatement of the reference's timestep (eu3d_oracle.c) compiled as
// C++ with every `double` replaced by a counting scalar, to pin F_sub: the
// FP64 work of one adaptive-trapezoid kinetics substep of one cell. It
// counts what the restatement's react_cell executes, i.e. the reference's
// Reaction::TrapezoidPrediction + Reaction::Trapezoid (src/Reaction.cpp:562-942)
// followed per substep by Flowfield::Explicit + Update_after_CS with its
// temperature Newton (src/Flowfield.cpp:1521-1536, :1639-1673, :2072-2131),
// divided by the substeps run (sum of Nchem).
//
// Convention: add, subtract, multiply, divide, sqrt = 1 flop each (the code
// has no fused multiply-add: it is compiled -ffp-contract=off like the
// reference); exp, log and pow are counted separately and are not flops.
// pow with an exponent of 0, 1 or 2 (stoichiometric powers, pow(u, 2)) is
// counted apart from pow with other exponents. Comparisons, fabs and ceil are
// not counted.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <pthread.h>

namespace flopcount {
struct Counts {
    unsigned long long add, mul, div, sqrt, exp, log, pow_small, pow_other;
};
Counts counts;
bool counting = false;
} // namespace flopcount

struct Flop {
    double v;
    Flop() = default;
    Flop(double x) : v(x) {}
    explicit operator int() const { return int(v); }
    explicit operator long() const { return long(v); }
    explicit operator double() const { return v; }
};

#define FC_BINARY(op, field)                                                                       \
    inline Flop operator op(Flop a, Flop b)                                                        \
    {                                                                                              \
        if (flopcount::counting)                                                                   \
            ++flopcount::counts.field;                                                             \
        return Flop(a.v op b.v);                                                                   \
    }                                                                                              \
    inline Flop &operator op##=(Flop &a, Flop b)                                                   \
    {                                                                                              \
        a = a op b;                                                                                \
        return a;                                                                                  \
    }
FC_BINARY(+, add)
FC_BINARY(-, add)
FC_BINARY(*, mul)
FC_BINARY(/, div)
#undef FC_BINARY
inline Flop operator-(Flop a) { return Flop(-a.v); }
inline Flop operator+(Flop a) { return a; }
inline bool operator<(Flop a, Flop b) { return a.v < b.v; }
inline bool operator>(Flop a, Flop b) { return a.v > b.v; }
inline bool operator<=(Flop a, Flop b) { return a.v <= b.v; }
inline bool operator>=(Flop a, Flop b) { return a.v >= b.v; }
inline bool operator==(Flop a, Flop b) { return a.v == b.v; }
inline bool operator!=(Flop a, Flop b) { return a.v != b.v; }
inline Flop fabs(Flop a) { return Flop(std::fabs(a.v)); }
inline Flop ceil(Flop a) { return Flop(std::ceil(a.v)); }
inline Flop sqrt(Flop a)
{
    if (flopcount::counting)
        ++flopcount::counts.sqrt;
    return Flop(std::sqrt(a.v));
}
inline Flop exp(Flop a)
{
    if (flopcount::counting)
        ++flopcount::counts.exp;
    return Flop(std::exp(a.v));
}
inline Flop log(Flop a)
{
    if (flopcount::counting)
        ++flopcount::counts.log;
    return Flop(std::log(a.v));
}
inline Flop pow(Flop a, Flop b)
{
    if (flopcount::counting) {
        if (b.v == 0.0 || b.v == 1.0 || b.v == 2.0)
            ++flopcount::counts.pow_small;
        else
            ++flopcount::counts.pow_other;
    }
    return Flop(std::pow(a.v, b.v));
}

#define double Flop
#include "eu3d_oracle.c"
#undef double

// One timestep like eo_step, with counting switched on for the kinetics phase
// only. out[8] accumulates add/sub, mul, div, sqrt, exp, log, pow (exponent
// 0/1/2), pow (other); *substeps accumulates the interior cells' Nchem.
extern "C" int fc_step(eo_state *st, double dt, unsigned long long *out, long long *substeps)
{
    const int bc = st->bc, ni = st->ni;
    st->dt = Flop(dt);
    boundary_fill(st);
    run_phase(st, 0, bc - 1, ni + bc);
    run_phase(st, 1, bc, ni + bc);
    flopcount::counts = flopcount::Counts{};
    flopcount::counting = true;
    for (int i = bc; i < ni + bc; i++)
        for (int j = bc; j < st->nj + bc; j++)
            for (int k = bc; k < st->nk + bc; k++) react_cell(st, IDX(st, i, j, k));
    flopcount::counting = false;
    const flopcount::Counts &c = flopcount::counts;
    const unsigned long long v[8] = {c.add, c.mul, c.div, c.sqrt, c.exp, c.log, c.pow_small, c.pow_other};
    for (int q = 0; q < 8; ++q) out[q] += v[q];
    long long n = 0;
    for (int i = bc; i < ni + bc; i++)
        for (int j = bc; j < st->nj + bc; j++)
            for (int k = bc; k < st->nk + bc; k++) n += st->nchem[IDX(st, i, j, k)];
    *substeps += n;
    return st->bad_nchem ? -1 : 0;
}
