/*
 * eu3d_oracle — CPU restatement of the EU3D reacting-Euler timestep.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the GPU library is compared
 * against; the shipped library never links, loads or calls it. It restates, in
 * plain C with the same floating-point expression order, the reference's CPU
 * path for one timestep (src/Euler.cpp:322-376 with the adaptive-trapezoid CPU
 * branch :443-493): RSBI ghost fill, MUSCL_2/minmod + AUSM+ fluxes in x, y, z,
 * Euler-explicit update, state recovery with Newton temperature inversion, Nchem
 * prediction and the linearised trapezoid substeps. Each function cites the
 * reference lines it follows. It is pinned bit-for-bit against the reference's
 * own code built from source (oracle/_ref) and against the golden fixtures in
 * tests/golden/.
 *
 * Layout: haloed grid nx = ni+2bc, ny = nj+2bc, nz = nk+2bc, cell
 * c = (i*ny + j)*nz + k (k fastest, as the reference's Array<double,3>).
 * Fields are structure-of-arrays: species and conserved components are planes
 * of n3 = nx*ny*nz doubles, plane s at offset s*n3.
 */
#ifndef EU3D_ORACLE_H
#define EU3D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct eo_state eo_state;

/* Mechanism tables in the reference's own layouts (src/Reaction.cpp:156-327):
 * coeff_lo/coeff_hi are Coeff0/Coeff1 as (9, ns) row-major; stoi_f/stoi_b/tb are
 * Stoi_F/Stoi_B/React_TB as (ns, nr) row-major. */
typedef struct {
    int ns, nr;
    const double *mw, *coeff_lo, *coeff_hi;
    const double *af, *bf, *eaf;
    const double *stoi_f, *stoi_b, *tb;
} eo_mechanism;

/* x, y, z: node coordinates including ghosts (length ni+2bc etc.). */
eo_state *eo_create(int ni, int nj, int nk, int bc, const double *x, const double *y, const double *z,
                    const eo_mechanism *mech, int nthreads);
void eo_destroy(eo_state *st);

/* Initial primitive fields over the haloed grid (Y: ns planes); derived
 * quantities follow Flowfield::FieldInitial (src/Flowfield.cpp:226-262). */
void eo_set_primitive(eo_state *st, const double *P, const double *T, const double *U, const double *V,
                      const double *W, const double *Y);

/* Exact state injection: every persistent field of the reference's timestep.
 * cs: ns+4 planes; y: ns planes; the 3-D fields are single planes. */
void eo_set_state(eo_state *st, const double *cs, const double *T, const double *E, const double *P,
                  const double *D, const double *U, const double *V, const double *W, const double *H,
                  const double *G, const double *Y);

/* nsteps reference timesteps at fixed dt. Returns 0, or -1 if a prediction gave
 * Nchem <= 0 (the reference aborts there, src/Reaction.cpp:936-940). */
int eo_step(eo_state *st, int nsteps, double dt);
/* Time scheme of eo_step's advection: 0 Euler explicit (the reference's
 * TimeAdv::EE), 1 the three-stage TVD Runge-Kutta (Shu-Osher SSP-RK3, this
 * build's; the reference's TimeAdv::TVD_RK3 is an empty stub). */
void eo_set_scheme(eo_state *st, int scheme);

/* The RSBI ghost fill alone (src/Flowfield.cpp:593-807, face layers). */
void eo_boundary(eo_state *st);
/* Ghost fill kind: 0 RSBI (default), 1 ZND (reflecting wall at x low, outflow
 * with the thermo rebuilt at x high; Flowfield::FieldBoundary_1dZND,
 * src/Flowfield.cpp:317-411, commented out in the reference), 2 ODW (inflow
 * tables at x low, rebuilt outflow at x high, y as RSBI, z mirrored with W
 * reflected and the thermo rebuilt; Flowfield::FieldBoundary_3dODW). */
void eo_set_boundary(eo_state *st, int kind);

/* Domain decomposition along x (the reference's MPI layout with m_block_x > 1):
 * x faces whose ghost nodes come from a neighbouring block are skipped by the
 * ghost fill and filled by eo_halo_unpack (Flowfield::Mpi_Boundary,
 * src/Flowfield.cpp:809-911). Messages hold eo_halo_count doubles. */
void eo_set_exchange(eo_state *st, int x_low, int x_high);

/* ODW ghost fill (kind 2, Flowfield::FieldBoundary_3dODW, src/Flowfield.cpp:412-592):
 * the x-low ghosts take these inflow tables (planes of nj * nk interior (j, k)
 * nodes, k fastest; Y: ns planes), with D, H, Gamma, E formed as FieldInitial
 * forms them (src/Flowfield.cpp:226-262). */
/* ODW: the y-low ghosts of local x nodes below first_wall_node take the
 * freestream (the first row of the inflow tables) instead of the symmetry
 * fill; 0 (the default) is the reference's fill. */
void eo_set_wall(eo_state *st, int first_wall_node);
void eo_set_inflow(eo_state *st, const double *P, const double *T, const double *U, const double *V,
                   const double *W, const double *Y);
long eo_halo_count(const eo_state *st);
void eo_halo_pack(eo_state *st, int face, double *msg);
void eo_halo_unpack(eo_state *st, int face, const double *msg);

/* Copy a named field out (SoA, haloed). Names: P D T U V W H E Gamma C Ma Wav
 * Rgas Cp (1 plane); Yi Di Mc CMS (ns planes); CS (ns+4 planes); Nchem (1 plane,
 * as doubles). Returns planes copied, or -1 for an unknown name. */
int eo_get(const eo_state *st, const char *name, double *out);

/* Single-point kernels for golden unit vectors. */
void eo_thermo(const eo_state *st, double T, double R, int s, double *cp_h_s);
/* Face L/R states of one scalar from its four stencil values (include/Differ.hpp:149-238). */
void eo_muscl(const double f[4], double *left, double *right);
/* AUSM+ flux at one face (src/Flowfield.cpp:1794-1931); lr = {P,D,U,V,W,H,Gamma} left
 * then right, yl/yr species, dir 1..3, out ns+4 values. */
void eo_ausm(const eo_state *st, const double lr[14], const double *yl, const double *yr, int dir, double *out);
/* Newton temperature inversion (src/Flowfield.cpp:2072-2131). */
double eo_temperature(const eo_state *st, double T0, double E, const double *Y);

#ifdef __cplusplus
}
#endif
#endif
