// state_init.hpp — host-side initial-state construction (FP64, compiled with
// -ffp-contract=off so it rounds as the reference's CPU build).
#pragma once

#include <vector>

#include "readers.hpp"

namespace eu3d {

// Flowfield::FieldInitial's derived fields (src/Flowfield.cpp:226-262) from
// primitive P, T, U, V, W, Y over a haloed grid. Outputs are full haloed planes;
// derived values are formed on interior nodes (ghost D, H, Gamma, E stay 0
// until the first ghost fill, as the reference leaves them unset).
//   prim: (7 + ns) planes P D U V W H Gamma Y...;  cs: ns + 4 planes;  T, E: planes
void primitive_to_state(const MechanismTables &m, int ni, int nj, int nk, int bc, const double *P, const double *T,
                        const double *U, const double *V, const double *W, const double *Y, std::vector<double> &prim,
                        std::vector<double> &cs, std::vector<double> &Tout, std::vector<double> &Eout);

} // namespace eu3d
