/*
 * eu3d.h — C ABI of the B200 EU3D reacting-Euler timestep library (libeu3d.so).
 *
 * One handle owns one solution (a haloed node grid, a mechanism and every device
 * buffer) on one GPU and one CUDA stream. Several handles may coexist in one
 * process; a handle is not thread-safe, distinct handles are.
 *
 * Host arrays are structure-of-arrays over the reference's haloed node grid:
 * nx = total_ni + 2*bc, ny = total_nj + 2*bc, nz = total_nk + 2*bc, node
 * (i,j,k) at c = (i*ny + j)*nz + k (k fastest, the reference's Array<double,3>
 * order); species and conserved components are consecutive planes of nx*ny*nz
 * doubles. Every call returns an eu_status; nothing exits the process.
 *
 * The entry points replace the reference's C++-linkage GPU glue:
 *   eu_step            Euler::Computing loop body (src/Euler.cpp:322-376) with
 *                      FieldBoundary_3dRSBI, Flowfield::Advection -> muscl_ausm_host
 *                      (include/FlowfieldCuda.cuh:53-67) + TimeAdv::EE_GPU/launch_ee_cuda
 *                      (include/TimeAdvCuda.cuh:4-15), Update_after_Adv ->
 *                      post_advection_state_host / post_advection_from_ee_host
 *                      (include/ReactionCuda.cuh:266, :282) and Euler::Trapezoid(1) ->
 *                      reaction_cells_host (include/ReactionCuda.cuh:230-248)
 *   eu_load_mechanism  Reaction::ReactionRead (src/Reaction.cpp:156-327)
 *   eu_read_grid       Mesh::MeshProcess (src/Mesh.cpp:36-84)
 *   eu_set_primitive   Flowfield::FieldInitial (src/Flowfield.cpp:193-264)
 *   eu_get_field       reaction_packed_output / download_resident_output
 *                      (include/ReactionCuda.cuh:274, :287) and the host scatter of
 *                      Flowfield::Update_after_Adv (src/Flowfield.cpp:1432-1450)
 */
#ifndef EU3D_H
#define EU3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EU3D_ABI_VERSION 1
#define EU3D_MAX_SPECIES 16   /* include/ReactionCuda.cuh:4 */
#define EU3D_MAX_REACTIONS 24 /* include/ReactionCuda.cuh:5 */

typedef struct eu_handle eu_handle;

typedef enum {
    EU_OK = 0,
    EU_ERR_INVALID_ARGUMENT = 1, /* bad pointer, size, name or option */
    EU_ERR_CUDA = 2,             /* a CUDA runtime call failed; see eu_last_error */
    EU_ERR_OUT_OF_MEMORY = 3,
    EU_ERR_IO = 4,               /* an input file is missing or does not parse */
    EU_ERR_NONFINITE = 5,        /* a density or temperature became non-finite */
    EU_ERR_NCHEM = 6,            /* a cell predicted Nchem <= 0 (the reference aborts,
                                    src/Reaction.cpp:936-940) or above max_substeps */
    EU_ERR_NOT_READY = 7,        /* call order: no mechanism or no state yet */
    EU_ERR_UNSUPPORTED = 8,      /* configuration outside what this build implements */
    EU_ERR_TIMEOUT = 9           /* a bounded device wait gave up */
} eu_status;

typedef enum {
    EU_PREC_FP64 = 0,  /* every flux, update, recovery and kinetics operation in FP64 */
    EU_PREC_MIXED = 1  /* MUSCL/AUSM in FP32; conserved update, recovery and kinetics FP64 */
} eu_precision;

typedef enum {
    EU_CHEM_STIFF = 0,   /* the reference's adaptive trapezoid kinetics on every cell */
    EU_CHEM_FROZEN = 1,  /* no kinetics (advection and state recovery only) */
    EU_CHEM_LEARNED = 2  /* learned-chemistry MLP with trust gate, stiff fallback */
} eu_chemistry;

typedef enum {
    EU_ARITH_STRICT = 0, /* no FMA contraction: rounds as the reference's CPU build */
    EU_ARITH_FAST = 1    /* FMA contraction allowed */
} eu_arith;

/* Ghost fill of the case (the reference wires one per case). */
typedef enum {
    EU_BC_RSBI = 0, /* Flowfield::FieldBoundary_3dRSBI (src/Flowfield.cpp:593-807) */
    EU_BC_ZND = 1,  /* Flowfield::FieldBoundary_1dZND (src/Flowfield.cpp:317-411, commented out in the
                       reference): reflecting wall at x low, outflow with the thermo rebuilt at x high;
                       y and z faces as RSBI */
    EU_BC_ODW = 2   /* Flowfield::FieldBoundary_3dODW (src/Flowfield.cpp:412-592, compiled in the
                       reference but not called): freestream inflow tables at x low (eu_set_inflow),
                       outflow with the thermo rebuilt at x high, y as RSBI (symmetry with the thermo
                       rebuilt at y low, zero gradient at y high), z mirrored with W reflected and
                       the thermo rebuilt */
} eu_boundary;

typedef struct {
    int total_ni, total_nj, total_nk; /* nodes per axis (grid file total_ni, ...) */
    double xa, xb, ya, yb, za, zb;    /* domain extents (grid file xa, xb, ...) */
    int bc;                           /* ghost layers per side; must be 2 (MUSCL_2 stencil) */
    int device;                       /* CUDA device ordinal */
    int precision;                    /* eu_precision */
    int chemistry;                    /* eu_chemistry */
    int arith;                        /* eu_arith */
    int max_substeps;                 /* Nchem cap; 0 selects 1 << 20 */
    int record_sources;               /* nonzero: keep per-cell mass sources (CMS) */
    int profile;                      /* nonzero: time each kernel phase with CUDA events */
    int eager;                        /* nonzero: launch each step's kernels one by one instead of
                                         replaying the step's captured CUDA graph */
    int boundary;                     /* eu_boundary: which case's ghost fill */
    int blocks_x;                     /* domain decomposition along x (the reference's m_block_x): the
                                         handle holds (total_ni - 1) / blocks_x + 1 nodes of the global
                                         grid, neighbouring blocks sharing one node (Mesh::Initial,
                                         src/Mesh.cpp:96-119); 0 or 1: the whole grid */
    int block_x;                      /* this handle's block, 0 .. blocks_x - 1 (the reference's myid_x);
                                         x faces between blocks take their ghost nodes from
                                         eu_halo_unpack instead of the boundary condition */
} eu_config;

/* Mechanism and thermo tables in the reference's layouts (src/Reaction.cpp:156-327). */
typedef struct {
    int ns, nr;
    const double *mw;       /* [ns] molecular weights, g/mol */
    const double *coeff_lo; /* [9*ns] Coeff0 (T < 1000 K), (k, s) row-major: a1..a7, b1, b2 */
    const double *coeff_hi; /* [9*ns] Coeff1 */
    const double *af;       /* [nr] pre-exponential factors */
    const double *bf;       /* [nr] temperature exponents */
    const double *eaf;      /* [nr] activation energies, cal/mol */
    const double *stoi_f;   /* [ns*nr] reactant coefficients, (s, r) row-major */
    const double *stoi_b;   /* [ns*nr] product coefficients */
    const double *tb;       /* [ns*nr] third-body efficiencies (all 0 for ordinary reactions) */
} eu_mechanism;

/* Per-call step statistics (device counters read back after the last step). */
typedef struct {
    int steps;
    int max_nchem;          /* largest Nchem of the last step */
    long long sum_nchem;    /* substeps over all cells, last step */
    long long reacting;     /* cells given to the kinetics in the last step */
    long long learned;      /* cells advanced by the learned model (EU_CHEM_LEARNED) */
    long long fallback;     /* cells the trust gate sent back to the stiff path */
    long long nonfinite;    /* cells with non-finite density or temperature */
    double device_ms;       /* device time of the call (CUDA events) */
    double phase_ms[4];     /* with cfg.profile: ghost fill, flux + update, recovery + kinetics, other */
    int launches;           /* kernels launched by the call */
    long long routed;       /* EU_CHEM_LEARNED: active cells whose predicted Nchem sent them to the
                               stiff kinetics (eu_learned_config.min_nchem), last step */
} eu_step_stats;

/* Library version / ABI check. */
int eu_abi_version(void);

/* Parse a grid file in the reference's format (input/grid-*.txt) into cfg's
 * grid members; other members are left as they are. */
eu_status eu_read_grid(const char *grid_path, eu_config *cfg);

/* One numeric value of a key/value file in the reference's format (ctrl.txt,
 * input-*.txt), read as FileReader::getdoubleParameter reads it
 * (src/FileReader.cpp:53-84); EU_ERR_INVALID_ARGUMENT when the key is absent.
 * The case initialisers take their parameters (P_bound, T_bound, P, T, ...)
 * from these files. */
eu_status eu_read_value(const char *path, const char *key, double *value);

/* Parse a mechanism file and thermo.dat (reference formats) without a device.
 * Replaces Reaction::ReactionRead (src/Reaction.cpp:156-327). Pass NULL arrays
 * to query ns/nr first; arrays sized as in eu_mechanism. */
eu_status eu_parse_mechanism(const char *mech_path, const char *thermo_path, int *ns, int *nr, double *mw,
                             double *coeff_lo, double *coeff_hi, double *af, double *bf, double *eaf,
                             double *stoi_f, double *stoi_b, double *tb);

/* Host-only initial state (no device): Flowfield::FieldInitial's derived fields
 * (src/Flowfield.cpp:226-262) from primitives over the haloed grid of
 * total_ni x total_nj x total_nk nodes with bc ghosts. Outputs: prim (7+ns planes:
 * P D U V W H Gamma Y...), cs (ns+4 planes), T, E (1 plane each). */
eu_status eu_initial_state(const eu_mechanism *m, int total_ni, int total_nj, int total_nk, int bc,
                           const double *P, const double *T, const double *U, const double *V, const double *W,
                           const double *Y, double *prim, double *cs, double *T_out, double *E_out);

/* Create a handle: allocates every device buffer for cfg's grid on cfg->device. */
eu_status eu_create(const eu_config *cfg, eu_handle **out);
eu_status eu_destroy(eu_handle *h);

/* Text of the last error on this handle (never NULL). */
const char *eu_last_error(const eu_handle *h);

/* Read a mechanism file and thermo.dat in the reference's formats
 * (input/H2_JA919.txt, input/thermo.dat). */
eu_status eu_load_mechanism(eu_handle *h, const char *mech_path, const char *thermo_path);
/* Install mechanism tables directly (copied). */
eu_status eu_set_mechanism(eu_handle *h, const eu_mechanism *m);
/* Copy the installed tables out; each pointer of m must have room for the sizes
 * above (ns, nr are filled first; pass NULL arrays to query sizes only). */
eu_status eu_get_mechanism(const eu_handle *h, int *ns, int *nr, double *mw, double *coeff_lo,
                           double *coeff_hi, double *af, double *bf, double *eaf, double *stoi_f,
                           double *stoi_b, double *tb);

/* Node coordinates with mirrored ghosts (src/Mesh.cpp:96-142), lengths nx, ny, nz. */
eu_status eu_node_coordinates(const eu_handle *h, double *x, double *y, double *z);

/* Initial condition from primitive fields over the haloed grid (host arrays;
 * Y has ns planes). Derived fields follow Flowfield::FieldInitial. */
eu_status eu_set_primitive(eu_handle *h, const double *P, const double *T, const double *U, const double *V,
                           const double *W, const double *Y);

/* Exact state injection: conserved CS (ns+4 planes), T, E, and the primitives the
 * stencils read (P, D, U, V, W, H, Gamma, Y) over the haloed grid. */
eu_status eu_set_state(eu_handle *h, const double *cs, const double *T, const double *E, const double *P,
                       const double *D, const double *U, const double *V, const double *W, const double *H,
                       const double *G, const double *Y);

/* Upload the conserved state alone (CS: ns + 4 haloed planes; T, E: haloed planes)
 * and form the primitives on the device as the step's recovery does
 * (Flowfield::Update_after_CS, src/Flowfield.cpp:1579-1617: T by the Newton
 * inversion from the given T with the given E as its energy, then u, v, w, e, p,
 * H, Gamma). Ghost primitives are formed by the next step's ghost fill. The
 * reference's post_advection_state_host (include/ReactionCuda.cuh:266) takes the
 * same inputs. Half the bytes of eu_set_state for a full state. */
eu_status eu_set_conserved(eu_handle *h, const double *cs, const double *T, const double *E);

/* EU_BC_ODW inflow tables: the x-low ghost nodes take these values each step
 * (Flowfield::FieldBoundary_3dODW, src/Flowfield.cpp:414-432, which copies the
 * tables Uint .. Yint; the reference allocates them, :138-147, but never fills
 * them). P, T, U, V, W: host planes over the interior (j, k) nodes, nj * nk values
 * with k fastest; Y: ns such planes. D, H, Gamma are formed from P, T, Y as
 * Flowfield::FieldInitial forms them (src/Flowfield.cpp:226-262). */
eu_status eu_set_inflow(eu_handle *h, const double *P, const double *T, const double *U, const double *V,
                        const double *W, const double *Y);
/* Time scheme of the advection part of eu_step. EU_TIME_EE (default): the
 * reference's Euler-explicit stage (TimeAdv::EE, src/TimeAdv.cpp:42-56).
 * EU_TIME_RK3: the three-stage TVD Runge-Kutta of Shu and Osher, U1 = U0 +
 * dt L(U0), U2 = 3/4 U0 + 1/4 (U1 + dt L(U1)), U3 = 1/3 U0 + 2/3 (U2 + dt
 * L(U2)), each stage with its own ghost fill and state recovery, then the
 * chemistry once on U3 (the reference declares TimeAdv::TVD_RK3,
 * src/TimeAdv.cpp:210-221, with an empty body). Each combination rounds its
 * two products and their sum separately. The start-of-step copy of the
 * conserved planes is allocated at the first switch to RK3. */
#define EU_TIME_EE 0
#define EU_TIME_RK3 1
eu_status eu_set_time_scheme(eu_handle *h, int scheme);

/* Where the z-face ghost nodes are formed (no counterpart in the reference).
 * EU_GHOSTS_REFERENCE (default): by the ghost fill at the start of each step,
 * as FieldBoundary_3dRSBI does (src/Flowfield.cpp:710-802), so after a step
 * every ghost node mirrors the interior as it was when the step began, which
 * is what the reference's outputs show. EU_GHOSTS_STORED: each stored
 * interior node also writes the z ghosts it is the mirror source of, and the
 * next ghost fill skips the z faces (whose mirror copies touch two 32-byte
 * sectors per row for 16 useful bytes); the interior state is bitwise the
 * same, but after a step the z-face ghost nodes mirror the interior as it is
 * at the step's end, so outputs that include ghost nodes (eu_get_field,
 * eu_write_state, eu_write_tecplot) differ from the reference's there. Needs
 * the RSBI or ZND fill and at least bc interior z nodes; set it before
 * creating a batch that holds the handle. */
#define EU_GHOSTS_REFERENCE 0
#define EU_GHOSTS_STORED 1
eu_status eu_set_ghost_mode(eu_handle *h, int mode);

/* EU_BC_ODW: where the wall begins on the y-low face. The ghost nodes of the
 * y-low face below global x node first_wall_node take the freestream (the
 * first row of the eu_set_inflow tables, per k) instead of the reflecting
 * wall, so the wedge surface starts at that node with free flow ahead of it
 * (a wedge tip inside the domain). 0, the default, is the reference's fill
 * (FieldBoundary_3dODW, src/Flowfield.cpp:464-493: symmetry along the whole
 * face). Needs the inflow tables when the freestream part is not empty. No
 * counterpart in the reference. */
eu_status eu_set_odw_wall(eu_handle *h, int first_wall_node);

/* Advance nsteps timesteps of fixed dt. Asynchronous on the handle's stream
 * unless stats is non-NULL (then it synchronises and fills stats). */
eu_status eu_step(eu_handle *h, int nsteps, double dt, eu_step_stats *stats);

/* Advance nsteps timesteps, each of dt = cfl x min over the interior nodes of
 * min(dx / (|u| + c), dy / (|v| + c)) on its own starting state, the reduction
 * done on the device (Flowfield::CFLcondition, src/Flowfield.cpp:275-304, with
 * the interior node spacings; the reference takes its spacings from the first
 * two ghost nodes, which is the same for three or more nodes per axis).
 * time_advanced (or NULL) receives the sum of the steps' dt (the call then
 * synchronises). */
eu_status eu_step_cfl(eu_handle *h, int nsteps, double cfl, eu_step_stats *stats, double *time_advanced);

/* Copy a named field to host (haloed SoA planes). Names: P D T U V W H E Gamma
 * C Ma Wav Rgas Cp (1 plane); Yi Di Mc CMS (ns planes); CS (ns+4 planes); Nchem
 * (1 plane, as doubles). Synchronises the handle's stream. */
eu_status eu_get_field(eu_handle *h, const char *name, double *host_out);

/* Write the solution in the reference's EU3D_STATE_V1_LE dump format
 * (Euler::Output with EU3D_DUMP_STATE=1, src/Euler.cpp:1540-1598): header line,
 * sizes/times line, column names, then 22 + 5 ns little-endian doubles per
 * interior node, (i, j, k) order with k fastest, as rank 0 of a 1 x 1 x 1
 * decomposition. CMS columns are zeros unless cfg.record_sources. */
eu_status eu_write_state(eu_handle *h, const char *path, int iteration, int num, double final_time, double dt);
/* Restart from such a dump (one rank's file whose local sizes and ns match the
 * handle): the conserved, thermodynamic and primitive fields are injected as by
 * eu_set_state; the header's iteration, output number, time and dt are returned
 * (NULL to skip). */
eu_status eu_read_state(eu_handle *h, const char *path, int *iteration, int *num, double *final_time, double *dt);

/* Output without stalling the time loop (the reference's Euler::Output,
 * src/Euler.cpp:1540-1790, writes synchronously from host arrays). The fields
 * the file needs are copied, in the handle's stream order, into a device
 * snapshot buffer of the handle, so eu_step may be called again at once; a
 * second stream moves the snapshot to pinned host memory and a host thread
 * writes the file. kind:
 *   EU_OUTPUT_STATE    the EU3D_STATE_V1_LE dump of eu_write_state (same bytes;
 *                      iteration, num, final_time and dt go to its header);
 *   EU_OUTPUT_TECPLOT  the reference's Tecplot file (Euler::Output,
 *                      src/Euler.cpp:1600-1790): "Variables = X,Y,Z,T,D,P,U,V,
 *                      Ma,Y1,...,Y7", one zone over every haloed node, block
 *                      packing with i fastest and k slowest, each value as a
 *                      C++ stream writes it by default (six significant digits);
 *                      the caller names the file (the reference's is
 *                      output_<ranks>/results/Series<name><num>_<rank>.dat).
 * One output is in flight per handle: a call waits for the previous one.
 * eu_output_wait waits for the file and returns the writer's status. The
 * snapshot buffers (device and pinned host, the size of the fields written)
 * are allocated at the first call and kept by the handle. */
#define EU_OUTPUT_STATE 0
#define EU_OUTPUT_TECPLOT 1
eu_status eu_output_async(eu_handle *h, int kind, const char *path, int iteration, int num, double final_time,
                          double dt);
eu_status eu_output_wait(eu_handle *h);
/* The Tecplot file of EU_OUTPUT_TECPLOT, written before the call returns. */
eu_status eu_write_tecplot(eu_handle *h, const char *path);

/* Wait for all work queued on the handle. */
eu_status eu_sync(eu_handle *h);

/* The stiff chemistry of the timestep on independent cells at rest (no
 * counterpart call in the reference; it runs the same kinetics as
 * Euler::Trapezoid(1), src/Euler.cpp:462-493, cell by cell). All pointers are
 * device memory; fields are planes of n values (cs: ns + 4 planes, Y: ns).
 * eu_chem_states forms cs and E from (T, p, Y) as FieldInitial does;
 * eu_chem_advance advances every cell by its own dt in place. With nchem
 * (optional) each sample's substep count is returned and a prediction above
 * max_substeps is not an error: that sample runs max_substeps substeps and
 * reports nchem == max_substeps (0 marks an invalid prediction).
 * Used to generate the learned model's training data. */
eu_status eu_chem_states(eu_handle *h, long long n, const double *T, const double *p, const double *Y, double *cs,
                         double *E);
eu_status eu_chem_advance(eu_handle *h, long long n, double *cs, double *T, double *E, const double *dt, int *nchem);

/* Device pointers and the stream of a handle, for callers that keep inputs
 * resident and time kernels themselves. */
eu_status eu_device_info(const eu_handle *h, void **stream, size_t *device_bytes);

/* ---------------------------------------------------------------------------
 * Halo exchange between x blocks (Flowfield::Mpi_Boundary, src/Flowfield.cpp:809-911,
 * the m_block_x > 1 part). A message holds the bc node planes one neighbour needs of
 * the primitive planes the flux reads (P, D, U, V, W, H, Gamma, Y_0 .. Y_ns-1; FP32 in
 * EU_PREC_MIXED, FP64 otherwise), laid out [field][plane][j][k] with full haloed planes.
 * The caller moves messages between ranks (NCCL, MPI) and unpacks them before each step:
 *   face 0 (x low):  pack = nodes bc+1 .. 2bc (the reference's bc+1+i), sent to block_x-1;
 *                    unpack fills ghost nodes bc-1-i from the x-low neighbour's face-1 message
 *   face 1 (x high): pack = nodes ni, ni-1 (the reference's ni-i, bc = 2), sent to block_x+1;
 *                    unpack fills ghost nodes ni+bc+i from the x-high neighbour's face-0 message
 * device_buf is device memory of eu_halo_bytes bytes. Both are asynchronous on the
 * handle's stream (eu_device_info). */
eu_status eu_halo_bytes(const eu_handle *h, size_t *bytes);
eu_status eu_halo_pack(eu_handle *h, int face, void *device_buf);
eu_status eu_halo_unpack(eu_handle *h, int face, const void *device_buf);

/* The CFL timestep of this block's current state, written to device memory on the
 * handle's stream (the local part of Flowfield::CFLcondition, src/Flowfield.cpp:275-304,
 * before its MPI_Allreduce(MPI_MIN)); the caller reduces it across blocks and steps with
 * eu_step_dt_device. */
eu_status eu_cfl_dt(eu_handle *h, double cfl, double *device_dt);

/* eu_step with dt read from device memory (each step uses the value at *device_dt when
 * the call is queued; asynchronous unless stats is non-NULL). */
eu_status eu_step_dt_device(eu_handle *h, int nsteps, const double *device_dt, eu_step_stats *stats);

/* ---------------------------------------------------------------------------
 * Learned chemistry (no counterpart in the reference, which has no learned
 * model): a small MLP evaluated and trained with BF16 tensor-core kernels.
 * ------------------------------------------------------------------------- */
typedef struct eu_mlp eu_mlp;

eu_status eu_mlp_create(int device, eu_mlp **out);
eu_status eu_mlp_destroy(eu_mlp *m);
const char *eu_mlp_last_error(const eu_mlp *m);

/* Tensor-core building block on device pointers: C = act(A * B^T + bias) with
 * A (M x K) and B (N x K) row-major bf16, fp32 accumulation; K % 16 == 0,
 * lda and ldb multiples of 8, 16-byte aligned operands. act: 0 none, 1 SiLU.
 * Outputs (each optional, ldc): Cf fp32, Cb bf16, Cpre fp32 pre-activation.
 * Runs on `stream` (a cudaStream_t, NULL: the model's stream) and waits for it. */
eu_status eu_mlp_gemm(eu_mlp *m, const void *A, int lda, const void *B, int ldb, int M, int N, int K,
                      const float *bias, int act, float *Cf, void *Cb, float *Cpre, int ldc, void *stream);

/* Build an ensemble of `members` MLPs n_in -> width (x hidden_layers, SiLU) ->
 * n_out with He-uniform weights from `seed`; max_batch (multiple of 16) sizes
 * the device scratch. BF16 weights/activations, fp32 master weights. */
eu_status eu_mlp_init(eu_mlp *m, int n_in, int width, int hidden_layers, int n_out, int members, int max_batch,
                      unsigned seed);
/* Affine normalisation: network input = (x - in_shift) * in_scale, physical
 * output = y / out_scale + out_shift (host arrays of n_in / n_out floats). */
eu_status eu_mlp_set_scaling(eu_mlp *m, const float *in_shift, const float *in_scale, const float *out_shift,
                             const float *out_scale);
/* Parameters flattened per member, per layer: W (out x in, row-major) then b. */
long long eu_mlp_num_params(const eu_mlp *m);
eu_status eu_mlp_get_params(eu_mlp *m, float *out);
eu_status eu_mlp_set_params(eu_mlp *m, const float *in);
/* Mean-squared-error loss (normalised outputs) and its gradient for one member
 * on n rows (device fp32 X [n x n_in], T [n x n_out]; n % 16 == 0); gradients
 * to host in the parameter order above (NULL to skip). */
eu_status eu_mlp_loss_grad(eu_mlp *m, int member, const float *X, const float *T, int n, float *loss,
                           float *grads);
/* `steps` Adam steps per member on random batches drawn on the device from
 * n training rows (device fp32 X, T); mean_loss receives each member's last
 * batch loss. */
eu_status eu_mlp_train(eu_mlp *m, const float *X, const float *T, long long n, int batch, int steps, float lr,
                       unsigned seed, float *mean_loss);
/* Physical outputs of every member: out[member][row][n_out] (device fp32). */
eu_status eu_mlp_predict(eu_mlp *m, const float *X, long long n, float *out);
/* The same outputs from one persistent tensor-core kernel that runs every
 * member's whole network per 128-row tile with the activations in shared
 * memory and the accumulators in tensor memory (the form the learned timestep
 * uses). Needs width <= 256 (multiple of 16), n_in <= 64, n_out <= width;
 * other shapes return EU_ERR_UNSUPPORTED. No counterpart in the reference
 * (its DNN scheme runs no model, src/Euler.cpp:1473-1480). */
eu_status eu_mlp_predict_fused(eu_mlp *m, const float *X, long long n, float *out);

/* eu_mlp_predict_fused without waiting: the kernel is queued on the model's
 * stream (eu_mlp_stream) and the call returns. X and out must stay valid until
 * that stream has run it. eu_mlp_sync waits for the stream and reports a
 * tensor-core pipeline wait that gave up (EU_ERR_TIMEOUT) in any work queued
 * since the last check. For callers that overlap inference with other work
 * and for timing the kernel with events on that stream. No counterpart in the
 * reference. */
eu_status eu_mlp_predict_fused_async(eu_mlp *m, const float *X, long long n, float *out);
eu_status eu_mlp_sync(eu_mlp *m);
eu_status eu_mlp_stream(eu_mlp *m, void **stream);

/* eu_mlp_predict without any device allocation, for callers that cannot call
 * cudaMalloc while they run: a solver that gives all free device memory to its
 * own pool after start-up (where a library's allocation fails or fragments
 * it), or a time loop that cannot take the device-wide synchronisation of
 * cudaMalloc/cudaFree. It has no counterpart in the reference.
 * Same inputs, outputs and results as eu_mlp_predict. The scratch (packed
 * inputs, hidden activations, outputs before unscaling, an error flag) is one
 * fixed array of EU_MLP_NOALLOC_SCRATCH_BYTES in the library's device memory.
 * eu_mlp_init loads it on the model's device and looks up its device address
 * there (CUDA loads the library's modules lazily, so this is when the device
 * memory is taken); from then on that GPU holds it until the process exits.
 * Create the model before handing free device memory to a pool of your own,
 * and before any stream capture. After a cudaDeviceReset the model is gone
 * with the rest of the device's memory: eu_mlp_init of a new one looks the
 * address up again. n may be
 * at most (EU_MLP_NOALLOC_SCRATCH_BYTES - 1024) / (2 in_pad + 4 width + 4
 * out_pad) rows (in_pad, out_pad: n_in, n_out rounded up to 16), 14978 for
 * the 12 -> 256 x 3 -> 10 chemistry model; more is EU_ERR_INVALID_ARGUMENT.
 * All calls share
 * the one array: calls that overlap on the GPU (other threads, other streams
 * of the same device) race and corrupt each other's results. Returns after
 * the model's stream has finished the work. */
#define EU_MLP_NOALLOC_SCRATCH_BYTES (16u << 20)
eu_status eu_mlp_predict_noalloc(eu_mlp *m, const float *X, long long n, float *out);

/* Learned chemistry in the timestep (cfg.chemistry == EU_CHEM_LEARNED). The
 * model maps (T, log10 p, Y_0..Y_{ns-1}, log10 dt) to (dY_0..dY_{ns-1}, dT) and
 * must have ns + 3 inputs and ns + 1 outputs. A cell is advanced by the
 * ensemble mean when every input lies in [box_lo, box_hi] and the members'
 * largest per-output standard deviation times out_scale is at most tau;
 * otherwise the stiff kinetics advances it. Cells whose non-inert mass
 * fraction is below frozen_y, or that are colder than frozen_T with a radical
 * pool (H, O, OH, HO2, H2O2 by species name) below frozen_radical, skip
 * chemistry. When out_eps[o] > 0 the model's output o is asinh(change/out_eps[o]).
 * When out_bound[o] > 0, a mean change of magnitude above it (outside the
 * range the model was trained on) also sends the cell to the stiff kinetics. */
typedef struct {
    double tau;
    double frozen_y;
    double frozen_T;
    double frozen_radical;
    const double *box_lo;    /* [ns + 3] */
    const double *box_hi;    /* [ns + 3] */
    const double *out_scale; /* [ns + 1] */
    const double *out_eps;   /* [ns + 1], NULL: linear outputs */
    const double *out_bound; /* [ns + 1], NULL: no output range check */
    int min_nchem;           /* active cells whose predicted Nchem (Reaction::TrapezoidPrediction,
                                src/Reaction.cpp:865-942) is at most this take the stiff kinetics
                                directly; the model sees the rest. 0: every active cell goes to the
                                model. A substep costs ~6 kflop in FP64, the model 0.82 MFLOP in
                                BF16, so the model pays only on cells that need several substeps */
} eu_learned_config;

eu_status eu_set_learned(eu_handle *h, eu_mlp *model, const eu_learned_config *cfg);

/* Autotuner: times the launch shapes that change no arithmetic (every
 * candidate gives bitwise the same state) on the handle's current state, which
 * it restores: the x-march length of the flux kernels, the block size of the
 * recovery kernels and, in learned mode, the recovery's register target. The choice applies to this handle and to handles
 * created later in the process with the same grid and mode. reps: timed
 * launches per candidate. report (or NULL) receives the candidates' times.
 * Allocates a temporary copy of the state. No counterpart in the reference. */
typedef struct {
    int flux_candidates;
    int flux_ci[16];
    float flux_ms[16];
    int recover_candidates;
    int recover_block[16];      /* threads per block */
    int recover_minblocks[16];  /* register target: resident blocks per SM (learned mode) */
    float recover_ms[16];
    int chosen_flux_ci;
    int chosen_recover_block;
    int chosen_recover_minblocks;
} eu_tune_report;
eu_status eu_autotune(eu_handle *h, int reps, eu_tune_report *report);

/* Batches of independent instances (any grid sizes, any modes) on one device,
 * advanced together: each step is one launch of a CUDA graph whose branches
 * are the instances' captured timesteps, so small and uneven instances share
 * the GPU instead of running one after another. No counterpart in the
 * reference (one grid per run; its multi-block runs are MPI ranks).
 * eu_batch_step: dt[count] per instance; stats[count] (or NULL) per instance;
 * device_ms (or NULL) the device time of the whole call. The handles stay
 * usable on their own between batch calls (the batch orders itself after
 * their earlier work and their later work after it). Learned instances need a
 * model with the fused inference kernel. Destroy the batch before its handles. */
typedef struct eu_batch eu_batch;
eu_status eu_batch_create(eu_handle *const *handles, int count, eu_batch **out);
eu_status eu_batch_step(eu_batch *b, int nsteps, const double *dt, eu_step_stats *stats, double *device_ms);
const char *eu_batch_last_error(const eu_batch *b);
eu_status eu_batch_destroy(eu_batch *b);
/* The kinetics the instances leave to the stiff integrator after their own
 * recovery (the learned mode's fallback queue, the cells deferred to the
 * warp-per-cell kinetics) run by default as one shared stage after every
 * instance's branch: one launch drains the fallback queues of all instances
 * of one flavour and mechanism taken end to end, one persistent launch their
 * deferred cells. on = 0 keeps those launches inside each instance's branch
 * instead. Results are the same either way (every cell's kinetics is
 * independent of the others). */
eu_status eu_batch_set_shared_kinetics(eu_batch *b, int on);
/* Kernel launches per batch step (after the first eu_batch_step): all of
 * them, and those of the shared kinetics stage. */
eu_status eu_batch_launches(const eu_batch *b, int *per_step, int *shared_stage);

#ifdef __cplusplus
}
#endif
#endif /* EU3D_H */
