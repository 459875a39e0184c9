// eu3d_types.h — plain structs shared by host code and kernels: mechanism
// tables as the kernels see them, grid geometry and device state pointers.
#pragma once

#include <cstdint>

namespace eu3d {

constexpr int kMaxS = 16; // include/ReactionCuda.cuh:4
constexpr int kMaxR = 24; // include/ReactionCuda.cuh:5

constexpr double kRUniv = 8.31434;      // include/Flowfield.hpp:57
constexpr double kRuCal = 1.987;        // include/Reaction.hpp:67
constexpr double kP0 = 101325.0;        // include/Reaction.hpp:68
constexpr double kThermoSwitch = 1000.0; // include/ThermoConstants.hpp:3

// Mechanism + thermo tables, passed to kernels by value (__grid_constant__) so
// that uniform reads come from the constant bank and handles stay independent.
struct DevMech {
    int ns, nr;
    int nu_int;             // 1 when every stoichiometric coefficient is 0, 1 or 2
    int pad;
    double mw[kMaxS];
    double ri[kMaxS];       // R / Mw (src/Reaction.cpp:426-427)
    double clo[9][kMaxS];   // Coeff0(k, s)
    double chi[9][kMaxS];   // Coeff1(k, s)
    double af[kMaxR], bf[kMaxR], eaf[kMaxR];
    double xr[kMaxR];       // sum_s (nu_b - nu_f)
    double sf[kMaxR][kMaxS], sb[kMaxR][kMaxS], tb[kMaxR][kMaxS];
    int has_tb[kMaxR];
};

// Division of an index n < 2^31 by a fixed divisor d >= 1 without a divide
// instruction: q = (n m) >> (32 + s) with s = ceil(log2 d), m = 2^(32+s) / d + 1.
// For n < 2^32 <= 2^(32+s)/d the rounding error n (m - 2^(32+s)/d) / 2^(32+s) stays
// below 1/d, so q = floor(n / d); n m < 2^31 2^33 fits 64 bits.
struct FastDiv {
    unsigned long long m;
    unsigned d;
    int s;
};
inline FastDiv make_fastdiv(unsigned d)
{
    int s = 0;
    while ((1ull << s) < d) ++s;
    return FastDiv{(1ull << (32 + s)) / d + 1, d, s};
}

// Grid and field pointers of one handle (all device memory).
struct DevGrid {
    int ni, nj, nk, bc, nx, ny, nz;
    long long n3;
    const double *x, *y, *z; // node coordinates with ghosts
    // index decompositions of the kernels' flat thread indices
    FastDiv d_nk, d_njnk, d_nink, d_ghost, d_ghost_nj, d_nz, d_nynz;
    int bc_kind; // eu_boundary
    // x faces whose ghost nodes come from a neighbouring block (halo exchange)
    // instead of the boundary condition
    int exch_lo, exch_hi;
    // EU_BC_ODW: y-low ghosts of local x nodes below wall_i0 take the freestream
    // (the wedge surface starts there); 0: the wall runs along the whole face
    int wall_i0;
};

// Primitive planes the stencils read, in this order (haloed, FP64).
enum PrimIdx { kP = 0, kD = 1, kU = 2, kV = 3, kW = 4, kH = 5, kG = 6, kY0 = 7 };

struct DevState {
    double *prim;     // (7 + ns) planes
    float *prim32;    // (7 + ns) planes, FP32 copy for EU_PREC_MIXED (or null)
    double *cs;       // ns + 4 planes
    double *T, *E;    // planes
    int *nchem;       // plane
    double *cms;      // ns planes (or null)
    unsigned long long *counters; // see CounterIdx
    int *heavy;       // mixed precision: {count, next, cells...} of cells left to the warp-per-cell kinetics
    const double *inflow; // ODW x-low ghost values per interior (j, k): 7 + ns primitive planes, then T
    // EU_GHOSTS_STORED: store_cell also writes the z-face ghosts a node is the
    // mirror source of (W reflected), and the ghost fill skips the z faces while
    // *zm_fresh is set (by each full recovery; cleared by host uploads). Null:
    // the ghost fill forms every face, as the reference does.
    int *zm_fresh;
    FastDiv zm_dnz; // nz, the node row length along z
    int zm_nz, zm_nk, zm_bc;
};

// Device counters. The first kCntPerStep are statistics of the latest step
// (cleared before each step); the rest accumulate over one eu_step call so an
// error in any step of the call is reported.
enum CounterIdx {
    kCntMaxNchem = 0,
    kCntSumNchem = 1,
    kCntReacting = 2,
    kCntLearned = 3,
    kCntFallback = 4,
    kCntRouted = 5, // learned mode: active cells the Nchem routing gave to the stiff kinetics
    kCntPerStep = 6,
    kCntNonfinite = 6,
    kCntBadNchem = 7,
    kCntCount = 8
};

// One instance of a batch in the batch's shared kinetics stage: its state, its
// dt, and its stiff-fallback queue (learned mode; null otherwise). The
// deferred cells are st.heavy's (null: none).
struct BatchCell {
    DevState st;
    long long n3;
    const double *dt;
    const int *queue; // cell indices
    const int *count; // queue length (count[0])
};

// Parameters and buffers of the learned-chemistry step (set by eu_set_learned).
struct LearnedParams {
    float *feat;           // [queue capacity x (3 + NS)] fp32 model inputs
    float *pred;           // [members x queue length x (NS + 1)] fp32 physical outputs
    int *queue, *fallback; // cell indices: the model's queue, the gate's rejections
    int *active;           // cells with chemistry to do (recovery's output, before the Nchem routing)
    int *counts;           // [0] model queue length, [1] fallback queue length, [2] fallback cells taken,
                           // [3] active cells, [4] active cells taken by the routing
    int min_nchem;         // predicted Nchem <= this: stiff kinetics right away (0: all to the model)
    long long pred_row, pred_mem; // ensemble output o of member e for queue row q: pred[q pred_row + e pred_mem + o]
    int members;
    double frozen_y;       // a cell whose non-inert mass fraction is below this is frozen
    double frozen_T;       // a cell colder than this whose radical pool is below frozen_radical is frozen
    double frozen_radical;
    double tau;            // largest accepted ensemble spread, in output-scale units
    double box_lo[kMaxS + 3], box_hi[kMaxS + 3]; // accepted input ranges
    double out_scale[kMaxS + 1];
    double out_eps[kMaxS + 1]; // model output o is asinh(change / eps) when eps > 0
    double out_bound[kMaxS + 1]; // |mean change| above it (> 0) sends the cell to the stiff kinetics
    double proj[kMaxS][kMaxS]; // element-conservation projector
    int inert[kMaxS];
    int radical[kMaxS];
};

} // namespace eu3d
