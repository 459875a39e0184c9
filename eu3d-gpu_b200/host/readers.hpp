// readers.hpp — parsers for the reference's input formats (host side of the
// drop-in boundary). They reproduce the reference's parsing semantics so that
// the same files give the same doubles:
//   key/value files (ctrl.txt, grid-*.txt, input-*.txt): FileReader
//     (src/FileReader.cpp:53-84, include/FileReader.hpp:74-103)
//   mechanism file (H2_JA919.txt) and thermo.dat: Reaction::ReactionRead
//     (src/Reaction.cpp:156-327)
#pragma once

#include <map>
#include <string>
#include <vector>

namespace eu3d {

// `key value` lines; '#' starts a comment. A numeric value is stored the way
// the reference's FileReader stores it: parsed, then printed with the default
// stream precision (6 significant digits) and parsed again on each read.
class KeyValueFile {
public:
    bool read(const std::string &path);
    bool has(const std::string &key) const { return values_.count(key) != 0; }
    double get_double(const std::string &key, double fallback = 0.0) const;
    int get_int(const std::string &key, int fallback = 0) const;
    std::string get_string(const std::string &key, const std::string &fallback = "") const;

private:
    std::map<std::string, std::string> values_;
};

struct GridSpec {
    int total_ni = 0, total_nj = 0, total_nk = 0, bc = 0;
    double xa = 0, xb = 0, ya = 0, yb = 0, za = 0, zb = 0;
};

bool read_grid(const std::string &path, GridSpec &out, std::string &err);

// Node coordinates with ghosts of block `block` of `blocks` along one axis
// (Mesh::Initial, src/Mesh.cpp:96-119: (total_n - 1) / blocks + 1 nodes from
// the global spacing; Mesh::Boundary, :131-142: ghosts extrapolated linearly).
std::vector<double> node_coordinates(int total_n, double a, double b, int bc, int blocks = 1, int block = 0);

struct MechanismTables {
    int ns = 0, nr = 0, tb_count = 0;
    std::vector<double> mw;           // [ns]
    std::vector<double> coeff_lo;     // [9*ns] (k, s)
    std::vector<double> coeff_hi;     // [9*ns]
    std::vector<double> af, bf, eaf;  // [nr]
    std::vector<double> stoi_f, stoi_b, tb; // [ns*nr] (s, r)
    std::vector<double> mole_ratio;   // [ns] the file's mole-ratio line
    std::vector<std::string> species; // names from the species header line
};

bool read_mechanism(const std::string &mech_path, const std::string &thermo_path, MechanismTables &out,
                    std::string &err);

} // namespace eu3d
