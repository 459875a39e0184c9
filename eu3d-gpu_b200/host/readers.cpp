// readers.cpp — the reference's input formats, parsed with its semantics.
#include "readers.hpp"

#include <cstdio>
#include <fstream>
#include <sstream>

namespace eu3d {

namespace {

// FileReader stores a parsed number as `ss << value` (default precision 6,
// src/FileReader.cpp:33-41) and every getter re-parses that text.
std::string as_stream_text(double v)
{
    std::stringstream ss;
    ss << v;
    return ss.str();
}

// seek_to_line (src/Reaction.cpp:128-143): rewind, then discard `line` lines
// of at most 1023 characters each.
void seek_to_line(std::ifstream &in, int line)
{
    in.clear();
    in.seekg(0, std::ios::beg);
    char buf[1024];
    for (int i = 0; i < line; i++) {
        in.getline(buf, sizeof(buf));
        if (in.fail() && !in.eof()) {
            in.clear(); // an over-long line: getline stops mid-line as the reference's does
        }
    }
}

} // namespace

bool KeyValueFile::read(const std::string &path)
{
    std::ifstream f(path);
    if (!f.is_open())
        return false;
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream ss(line);
        std::string k, v;
        ss >> k >> v;
        if (k.empty() || v.empty() || k[0] == '#' || v[0] == '#')
            continue;
        try {
            size_t used = 0;
            double d = std::stod(v, &used);
            (void)used;
            values_[k] = as_stream_text(d);
        } catch (...) {
            values_[k] = v;
        }
    }
    return true;
}

double KeyValueFile::get_double(const std::string &key, double fallback) const
{
    auto it = values_.find(key);
    if (it == values_.end())
        return fallback;
    try {
        return std::stod(it->second);
    } catch (...) {
        return 0; // include/FileReader.hpp:87-99
    }
}

int KeyValueFile::get_int(const std::string &key, int fallback) const
{
    auto it = values_.find(key);
    if (it == values_.end())
        return fallback;
    try {
        return std::stoi(it->second);
    } catch (...) {
        return 0; // include/FileReader.hpp:74-86
    }
}

std::string KeyValueFile::get_string(const std::string &key, const std::string &fallback) const
{
    auto it = values_.find(key);
    return it == values_.end() ? fallback : it->second;
}

bool read_grid(const std::string &path, GridSpec &g, std::string &err)
{
    KeyValueFile f;
    if (!f.read(path)) {
        err = "cannot open grid file " + path;
        return false;
    }
    const char *need[] = {"total_ni", "xa", "xb", "total_nj", "ya", "yb", "total_nk", "za", "zb", "bc"};
    for (const char *k : need)
        if (!f.has(k)) {
            err = std::string("grid file lacks ") + k;
            return false;
        }
    g.total_ni = f.get_int("total_ni");
    g.xa = f.get_double("xa");
    g.xb = f.get_double("xb");
    g.total_nj = f.get_int("total_nj");
    g.ya = f.get_double("ya");
    g.yb = f.get_double("yb");
    g.total_nk = f.get_int("total_nk");
    g.za = f.get_double("za");
    g.zb = f.get_double("zb");
    g.bc = f.get_int("bc");
    if (g.total_ni < 2 || g.total_nj < 2 || g.total_nk < 2) { // src/Mesh.cpp:55-62
        err = "each grid dimension must be >= 2";
        return false;
    }
    return true;
}

std::vector<double> node_coordinates(int total_n, double a, double b, int bc, int blocks, int block)
{
    const int n = (total_n - 1) / blocks + 1;
    std::vector<double> x(n + 2 * bc, 0.0);
    const double d = (b - a) / (total_n - 1);
    for (int i = bc; i < n + bc; i++) x[i] = a + (block * (n - 1) + i - bc) * d;
    for (int i = 0; i < bc; i++) {
        x[i] = 2 * x[bc] - x[2 * bc - i];
        x[n + bc + i] = 2 * x[n + bc - 1] - x[n + bc - 1 - i - 1];
    }
    return x;
}

bool read_mechanism(const std::string &mech_path, const std::string &thermo_path, MechanismTables &m,
                    std::string &err)
{
    std::ifstream fin(mech_path);
    if (!fin.is_open()) {
        err = "cannot open mechanism file " + mech_path;
        return false;
    }
    std::string s, item;
    int line = 2;
    try {
        // NS NR TB, tab-separated (src/Reaction.cpp:167-189)
        seek_to_line(fin, line);
        std::getline(fin, s, '\n');
        {
            std::stringstream ts(s);
            std::vector<int> a;
            while (std::getline(ts, item, '\t')) a.push_back(std::stoi(item));
            if (a.size() < 3) {
                err = "mechanism: cannot read NS NR TB";
                return false;
            }
            m.ns = a[0];
            m.nr = a[1];
            m.tb_count = a[2];
        }
        if (m.ns <= 0 || m.nr <= 0 || m.ns > 16 || m.nr > 24 || m.tb_count < 0 || m.tb_count > m.nr) {
            err = "mechanism sizes outside NS<=16, NR<=24";
            return false;
        }
        const int ns = m.ns, nr = m.nr;
        // species names: the line before the stoichiometry block
        seek_to_line(fin, line + 5);
        std::getline(fin, s, '\n');
        {
            std::stringstream ts(s);
            std::string nm;
            while (ts >> nm) m.species.push_back(nm);
        }
        m.stoi_f.assign(ns * nr, 0.0);
        m.stoi_b.assign(ns * nr, 0.0);
        // stoichiometry: forward row then backward row per reaction (:191-219)
        line = line + 6;
        seek_to_line(fin, line);
        for (int j = 0; j < nr; j++) {
            for (int pass = 0; pass < 2; ++pass) {
                std::getline(fin, s, '\n');
                std::stringstream rs(s);
                int i = 0;
                while (std::getline(rs, item, '\t')) {
                    if (i >= ns) {
                        err = "mechanism: stoichiometry row longer than NS";
                        return false;
                    }
                    (pass == 0 ? m.stoi_f : m.stoi_b)[i * nr + j] = std::stoi(item);
                    i++;
                }
            }
        }
        // Arrhenius: index A b E per reaction (:222-241)
        m.af.assign(nr, 0.0);
        m.bf.assign(nr, 0.0);
        m.eaf.assign(nr, 0.0);
        line = line + 2 * nr + 2;
        seek_to_line(fin, line);
        for (int j = 0; j < nr; j++) {
            int i = 0;
            double b[4] = {0, 0, 0, 0};
            while (fin >> s) {
                std::stringstream geek(s);
                geek >> b[i];
                i++;
                if (i == 4)
                    break;
            }
            m.af[j] = b[1];
            m.bf[j] = b[2];
            m.eaf[j] = b[3];
        }
        // third-body efficiencies: reaction index then NS integers (:244-263)
        m.tb.assign(ns * nr, 0.0);
        line = line + nr + 3;
        seek_to_line(fin, line);
        for (int j = 0; j < m.tb_count; j++) {
            int a[100] = {0};
            int i = 0;
            while (fin >> s) {
                std::stringstream geek(s);
                geek >> a[i];
                i++;
                if (i == ns + 1)
                    break;
            }
            if (a[0] < 1 || a[0] > nr) {
                err = "mechanism: third-body reaction index out of range";
                return false;
            }
            for (int k = 0; k < ns; k++) m.tb[k * nr + (a[0] - 1)] = a[k + 1];
        }
        // mole ratio line (:266-283)
        line = line + m.tb_count + 2;
        seek_to_line(fin, line);
        {
            double c[100] = {0};
            int i = 0;
            while (fin >> s) {
                std::stringstream geek(s);
                geek >> c[i];
                i++;
                if (i == ns)
                    break;
            }
            m.mole_ratio.assign(c, c + ns);
        }
    } catch (const std::exception &e) {
        err = std::string("mechanism parse error: ") + e.what();
        return false;
    }

    // thermo.dat: from line 16, per species 19 numbers (9 low, 9 high, Mw),
    // blocks of 6 lines, taken positionally (:291-326)
    std::ifstream in(thermo_path);
    if (!in.is_open()) {
        err = "cannot open thermo file " + thermo_path;
        return false;
    }
    m.coeff_lo.assign(9 * m.ns, 0.0);
    m.coeff_hi.assign(9 * m.ns, 0.0);
    m.mw.assign(m.ns, 0.0);
    int tline = 15;
    for (int j = 0; j < m.ns; j++) {
        seek_to_line(in, tline);
        double aa[100] = {0};
        int i = 0;
        while (in >> s) {
            std::stringstream geek(s);
            geek >> aa[i];
            i++;
            if (i == 19)
                break;
        }
        if (i < 19) {
            err = "thermo file ends before species " + std::to_string(j);
            return false;
        }
        for (int k = 0; k < 9; k++) m.coeff_lo[k * m.ns + j] = aa[k];
        for (int k = 0; k < 9; k++) m.coeff_hi[k * m.ns + j] = aa[k + 9];
        m.mw[j] = aa[18];
        if (!(m.mw[j] > 0)) {
            err = "thermo: non-positive molecular weight for species " + std::to_string(j);
            return false;
        }
        tline = tline + 6;
    }
    return true;
}

} // namespace eu3d
