// gen_mech.cpp — build-time generator of mechanism-specialised rate code.
//
// Reads a mechanism file and thermo.dat with the library's own parser (the
// reference's semantics, readers.cpp) and writes two headers:
//   <out>.cuh : a device function computing the per-species production/loss
//               sums P, Q and mass rates W of one cell as straight-line code,
//               with the stoichiometry, Arrhenius constants and third-body
//               efficiencies as literals. Two bodies: the strict one evaluates
//               exactly the expressions of the reference (src/Reaction.cpp:
//               597-623, 720-727, 786-797) minus terms that are exact zeros
//               there; the fast one uses exp-of-sums for the equilibrium
//               constants.
//   <out>_tables.h : the parsed tables as hexadecimal literals and a host
//               function telling whether a loaded mechanism is this one
//               (bitwise), so the library picks the specialised kernels only
//               for identical tables.
//
//   gen_mech <mech> <thermo> <Name> <out_dir>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>

#include "readers.hpp"

using eu3d::MechanismTables;

namespace {

std::string hex(double v)
{
    char b[64];
    std::snprintf(b, sizeof b, "%a", v);
    return b;
}

// pow(x, e) of an integer-valued exponent as the reference evaluates it
// (glibc pow is correctly rounded for these): 0 -> 1, 1 -> x, -1 -> 1/x.
std::string pow_expr(const std::string &x, double e)
{
    if (e == 0.0) return "1.0";
    if (e == 1.0) return x;
    if (e == -1.0) return "(1.0 / " + x + ")";
    return "pow(" + x + ", " + hex(e) + ")";
}

void emit_strict(std::ostream &o, const MechanismTables &m)
{
    const int ns = m.ns, nr = m.nr;
    o << "    double Gi[" << ns << "];\n"
      << "    {\n"
      << "        const TPow p = make_tpow(T, true);\n"
      << "        gibbs_all<" << ns << ">(m, p, T, Gi);\n"
      << "    }\n"
      << "    const double RT = kRUniv * T;\n"
      << "    const double RuT = kRuCal * T;\n"
      << "    const double p0 = kP0 * 1e-6;\n"
      << "#pragma unroll\n"
      << "    for (int s = 0; s < " << ns << "; ++s) { k.P[s] = 0.0; k.Q[s] = 0.0; k.W[s] = 0.0; }\n";
    for (int r = 0; r < nr; ++r) {
        o << "    { // reaction " << r + 1 << "\n";
        // delta_g = sum_s (b - f) G_s over nonzero coefficients, in s order
        o << "        double delta_g = 0.0;\n";
        double xr = 0;
        for (int s = 0; s < ns; ++s) {
            const double d = m.stoi_b[s * nr + r] - m.stoi_f[s * nr + r];
            xr += d;
            if (d != 0.0) o << "        delta_g += " << hex(d) << " * Gi[" << s << "];\n";
        }
        std::string rrf = "1.0", rrb = "1.0";
        for (int s = 0; s < ns; ++s) {
            const double f = m.stoi_f[s * nr + r], b = m.stoi_b[s * nr + r];
            auto term = [&](double e) -> std::string {
                const std::string x = "mc[" + std::to_string(s) + "]";
                if (e == 1.0) return x;
                if (e == 2.0) return "(" + x + " * " + x + ")";
                return "pow(" + x + ", " + hex(e) + ")";
            };
            if (f != 0.0) rrf = (rrf == "1.0") ? term(f) : "(" + rrf + " * " + term(f) + ")";
            if (b != 0.0) rrb = (rrb == "1.0") ? term(b) : "(" + rrb + " * " + term(b) + ")";
        }
        o << "        const double rrf = " << rrf << ";\n";
        o << "        const double rrb = " << rrb << ";\n";
        bool has_tb = false;
        for (int s = 0; s < ns; ++s) has_tb |= m.tb[s * nr + r] != 0.0;
        if (has_tb) {
            o << "        double rtb = 0.0;\n";
            for (int s = 0; s < ns; ++s) {
                const double e = m.tb[s * nr + r];
                if (e != 0.0) o << "        rtb += mc[" << s << "] * " << hex(e) << ";\n";
            }
            o << "        if (rtb == 0.0) rtb = 1.0;\n";
        } else {
            o << "        const double rtb = 1.0;\n";
        }
        const double A = m.af[r], b = m.bf[r], E = m.eaf[r];
        std::string tp = pow_expr("T", b);
        std::string kf = "(" + hex(A) + " * " + tp + ")";
        if (E != 0.0) kf = "(" + kf + " * exp(" + hex(-E) + " / RuT))";
        o << "        const double kf = " << kf << ";\n";
        o << "        const double Kp = exp(-delta_g / RT) * " << pow_expr("p0", xr) << ";\n";
        o << "        const double Kc = Kp * " << pow_expr("RT", -xr) << ";\n";
        o << "        const double kb = kf / Kc;\n";
        o << "        const double fwd = kf * rrf, bwd = kb * rrb;\n";
        o << "        const double rr = fwd - bwd;\n";
        for (int s = 0; s < ns; ++s) {
            const double f = m.stoi_f[s * nr + r], bb = m.stoi_b[s * nr + r];
            if (f == 0.0 && bb == 0.0) continue;
            o << "        k.W[" << s << "] += " << hex(bb - f) << " * rtb * rr;\n";
            o << "        k.Q[" << s << "] += (" << hex(bb) << " * fwd + " << hex(f) << " * bwd) * rtb;\n";
            o << "        k.P[" << s << "] += (" << hex(bb) << " * bwd + " << hex(f) << " * fwd) * rtb;\n";
        }
        o << "    }\n";
    }
    o << "#pragma unroll\n    for (int s = 0; s < " << ns << "; ++s) k.W[s] = m.mw[s] * k.W[s];\n";
}

void emit_fast(std::ostream &o, const MechanismTables &m)
{
    const int ns = m.ns, nr = m.nr;
    o << "    double eg[" << ns << "], ieg[" << ns << "], Gs[" << ns << "];\n"
      << "    const TPow p = make_tpow(T, true);\n"
      << "    const double invRT = 1.0 / (kRUniv * T);\n"
      << "    gibbs_all<" << ns << ">(m, p, T, Gs);\n"
      << "#pragma unroll\n"
      << "    for (int s = 0; s < " << ns << "; ++s) {\n"
      << "        const double g = Gs[s] * invRT;\n"
      << "        eg[s] = exp(g);\n"
      << "        ieg[s] = exp(-g);\n"
      << "    }\n"
      << "    const double invRuT = 1.0 / (kRuCal * T);\n"
      << "    const double rt_p0 = (kRUniv * T) * " << hex(1.0 / (101325.0 * 1e-6)) << ";\n"
      << "#pragma unroll\n"
      << "    for (int s = 0; s < " << ns << "; ++s) { k.P[s] = 0.0; k.Q[s] = 0.0; k.W[s] = 0.0; }\n";
    for (int r = 0; r < nr; ++r) {
        o << "    { // reaction " << r + 1 << "\n";
        std::string rrf = "1.0", rrb = "1.0", kc = "1.0";
        double xr = 0;
        for (int s = 0; s < ns; ++s) {
            const double f = m.stoi_f[s * nr + r], b = m.stoi_b[s * nr + r];
            const std::string x = "mc[" + std::to_string(s) + "]";
            auto term = [&](double e) { return e == 1.0 ? x : "(" + x + " * " + x + ")"; };
            if (f != 0.0) rrf = (rrf == "1.0") ? term(f) : rrf + " * " + term(f);
            if (b != 0.0) rrb = (rrb == "1.0") ? term(b) : rrb + " * " + term(b);
            const double d = b - f;
            xr += d;
            std::string fac;
            const std::string e = "eg[" + std::to_string(s) + "]", ie = "ieg[" + std::to_string(s) + "]";
            if (d == 1.0) fac = e;
            else if (d == -1.0) fac = ie;
            else if (d == 2.0) fac = e + " * " + e;
            else if (d == -2.0) fac = ie + " * " + ie;
            if (!fac.empty()) kc = (kc == "1.0") ? fac : kc + " * " + fac;
        }
        if (xr == 1.0) kc += " * rt_p0";
        else if (xr == -1.0) kc += " / rt_p0";
        else if (xr != 0.0) kc += " * pow(rt_p0, " + hex(xr) + ")";
        o << "        const double rrf = " << rrf << ";\n";
        o << "        const double rrb = " << rrb << ";\n";
        bool has_tb = false;
        for (int s = 0; s < ns; ++s) has_tb |= m.tb[s * nr + r] != 0.0;
        if (has_tb) {
            o << "        double rtb = 0.0;\n";
            for (int s = 0; s < ns; ++s) {
                const double e = m.tb[s * nr + r];
                if (e != 0.0) o << "        rtb = fma(mc[" << s << "], " << hex(e) << ", rtb);\n";
            }
            o << "        if (rtb == 0.0) rtb = 1.0;\n";
        } else {
            o << "        const double rtb = 1.0;\n";
        }
        const double A = m.af[r], b = m.bf[r], E = m.eaf[r];
        std::string kf;
        if (E == 0.0 && (b == 0.0 || b == 1.0 || b == -1.0 || b == -2.0)) {
            const char *tp = b == 0.0 ? "1.0" : b == 1.0 ? "T" : b == -1.0 ? "p.inv" : "p.inv2";
            kf = hex(A) + " * " + tp;
        } else {
            kf = hex(A) + " * exp(" + hex(b) + " * p.lnT - " + hex(E) + " * invRuT)";
        }
        o << "        const double kf = " << kf << ";\n";
        o << "        const double kb = kf * (" << kc << ");\n";
        o << "        const double fwd = kf * rrf, bwd = kb * rrb;\n";
        o << "        const double rrt = (fwd - bwd) * rtb;\n";
        o << "        const double fr = fwd * rtb, br = bwd * rtb;\n";
        for (int s = 0; s < ns; ++s) {
            const double f = m.stoi_f[s * nr + r], bb = m.stoi_b[s * nr + r];
            if (f == 0.0 && bb == 0.0) continue;
            auto scaled = [&](double c, const char *v) -> std::string {
                if (c == 1.0) return v;
                return hex(c) + " * " + v;
            };
            const double d = bb - f;
            if (d != 0.0) o << "        k.W[" << s << "] = fma(" << hex(d) << ", rrt, k.W[" << s << "]);\n";
            std::string q, pl;
            if (bb != 0.0) q = scaled(bb, "fr");
            if (f != 0.0) q = q.empty() ? scaled(f, "br") : q + " + " + scaled(f, "br");
            if (bb != 0.0) pl = scaled(bb, "br");
            if (f != 0.0) pl = pl.empty() ? scaled(f, "fr") : pl + " + " + scaled(f, "fr");
            o << "        k.Q[" << s << "] += " << q << ";\n";
            o << "        k.P[" << s << "] += " << pl << ";\n";
        }
        o << "    }\n";
    }
    o << "#pragma unroll\n    for (int s = 0; s < " << ns << "; ++s) k.W[s] = m.mw[s] * k.W[s];\n";
}

void emit_tables(std::ostream &o, const MechanismTables &m, const std::string &name)
{
    auto arr = [&](const char *nm, const std::vector<double> &v) {
        o << "static const double k" << name << "_" << nm << "[" << v.size() << "] = {";
        for (size_t i = 0; i < v.size(); ++i) o << (i ? ", " : "") << hex(v[i]);
        o << "};\n";
    };
    arr("mw", m.mw);
    arr("coeff_lo", m.coeff_lo);
    arr("coeff_hi", m.coeff_hi);
    arr("af", m.af);
    arr("bf", m.bf);
    arr("eaf", m.eaf);
    arr("stoi_f", m.stoi_f);
    arr("stoi_b", m.stoi_b);
    arr("tb", m.tb);
    o << "\n// True when tables m are bitwise the ones this code was generated from.\n"
      << "inline bool matches_" << name << "(int ns, int nr, const double *mw, const double *clo, const double *chi,\n"
      << "                            const double *af, const double *bf, const double *eaf, const double *sf,\n"
      << "                            const double *sb, const double *tb)\n{\n"
      << "    if (ns != " << m.ns << " || nr != " << m.nr << ") return false;\n"
      << "    auto same = [](const double *a, const double *b, int n) {\n"
      << "        for (int i = 0; i < n; ++i)\n"
      << "            if (std::memcmp(&a[i], &b[i], sizeof(double)) != 0) return false;\n"
      << "        return true;\n    };\n"
      << "    return same(mw, k" << name << "_mw, " << m.ns << ") && same(clo, k" << name << "_coeff_lo, "
      << 9 * m.ns << ") &&\n"
      << "           same(chi, k" << name << "_coeff_hi, " << 9 * m.ns << ") && same(af, k" << name << "_af, " << m.nr
      << ") &&\n"
      << "           same(bf, k" << name << "_bf, " << m.nr << ") && same(eaf, k" << name << "_eaf, " << m.nr
      << ") &&\n"
      << "           same(sf, k" << name << "_stoi_f, " << m.ns * m.nr << ") && same(sb, k" << name << "_stoi_b, "
      << m.ns * m.nr << ") &&\n"
      << "           same(tb, k" << name << "_tb, " << m.ns * m.nr << ");\n}\n";
}

} // namespace

int main(int argc, char **argv)
{
    if (argc != 5) {
        std::fprintf(stderr, "usage: gen_mech <mech> <thermo> <Name> <out_dir>\n");
        return 2;
    }
    MechanismTables m;
    std::string err;
    if (!eu3d::read_mechanism(argv[1], argv[2], m, err)) {
        std::fprintf(stderr, "gen_mech: %s\n", err.c_str());
        return 1;
    }
    for (double v : m.stoi_f)
        if (!(v == 0 || v == 1 || v == 2)) { std::fprintf(stderr, "gen_mech: coefficient %g unsupported\n", v); return 1; }
    for (double v : m.stoi_b)
        if (!(v == 0 || v == 1 || v == 2)) { std::fprintf(stderr, "gen_mech: coefficient %g unsupported\n", v); return 1; }
    const std::string name = argv[3], dir = argv[4];
    {
        std::ofstream o(dir + "/eu3d_mech_" + name + ".cuh");
        auto base = [](const std::string &path) { return path.substr(path.find_last_of('/') + 1); };
        o << "// Generated by eu3d-gpu_b200/host/gen_mech.cpp from " << base(argv[1]) << " and " << base(argv[2])
          << ". Do not edit.\n#pragma once\n#include \"eu3d_device.cuh\"\n\nnamespace eu3d {\n\n"
          << "// Rates of mechanism " << name << " (" << m.ns << " species, " << m.nr << " reactions).\n"
          << "struct Mech_" << name << " {\n    static constexpr int NS = " << m.ns << ", NR = " << m.nr << ";\n"
          << "    __device__ __forceinline__ static void rates(const DevMech &m, double T, const double (&mc)[" << m.ns
          << "], SpeciesRates<" << m.ns << "> &k)\n    {\n#ifdef EU_EXACT_CHEM\n";
        emit_strict(o, m);
        o << "#else\n";
        emit_fast(o, m);
        o << "#endif\n    }\n};\n\n} // namespace eu3d\n";
    }
    {
        std::ofstream o(dir + "/eu3d_mech_" + name + "_tables.h");
        o << "// Generated by eu3d-gpu_b200/host/gen_mech.cpp. Do not edit.\n#pragma once\n#include <cstring>\n\n"
          << "namespace eu3d {\n";
        emit_tables(o, m, name);
        o << "} // namespace eu3d\n";
    }
    return 0;
}
