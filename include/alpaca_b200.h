/*
 * alpaca_b200 — C ABI of the B200 block right-hand side / SSP-RK3 engine.
 *
 * Drop-in for the hot path of tumaer/ALPACA (paths below are relative to the
 * reference's src/): the convective term of SpaceSolver::UpdateFluxes, the
 * prime-state conversion, the same-level halo update, ComputeTimestepSize and
 * the RungeKutta3TVD stage update. Every buffer uses the reference's block
 * layout (block_definitions/field_buffer.h:37-40): per block and field a
 * C-ordered double[TCX][TCY][TCZ], TC = 24 in active dimensions and 1 in
 * inactive ones, conservatives ordered Mass, Energy, MomentumX[, Y[, Z]]
 * (block_definitions/field_setup.h:101-112), blocks one after the other.
 *
 * Conventions: pointers named d_* are device pointers, h_* host pointers.
 * Every call is asynchronous on the given stream (0 = legacy default stream)
 * and returns ALP_OK or an error code; no C++ exception crosses the ABI. The
 * stateless calls allocate nothing; the engine allocates its device pool when
 * it is created and never while stepping.
 */
#ifndef ALPACA_B200_H
#define ALPACA_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *alp_stream_t; /* == cudaStream_t */

/* ---- status codes -------------------------------------------------------- */
enum {
  ALP_OK = 0,
  ALP_ERR_INVALID = 1,       /* bad argument or unsupported selection */
  ALP_ERR_CUDA = 2,          /* a CUDA call failed (see alp_last_error) */
  ALP_ERR_CAPACITY = 3,      /* engine pool / case table full */
  ALP_ERR_NOT_FOUND = 4,     /* unknown case id */
  ALP_ERR_NUMERIC = 5,       /* non-finite or non-positive state detected */
  ALP_ABORTED = 6            /* alp_serve stopped by its abort file */
};

/* ---- scheme selection ---------------------------------------------------
 * The values mirror the reference's compile-time enums so that a shadow of
 * user_specifications/ selects the same combination:
 *   convective_term_solver   riemann_solver_settings.h:28  (FluxSplitting=0, FiniteVolume=1)
 *   state_reconstruction     state_reconstruction_settings.h:25 (Conservative=0, Primitive=1, Characteristic=2)
 *   reconstruction_stencil   stencil_setup.h:26-43 (FirstOrder=0, WENO3=1, WENO5=4, WENO5Z=7, TENO5=11,
 *                                                  WENO7=13)
 *   riemann_solver           riemann_solver_settings.h:47 (Hllc=0, Hllc_LM=1, Hll=2)
 *   signal_speed             enums/signal_speed.h:31 (Einfeldt=0, Davis=1, Toro=2, Arithmetic=3)
 *   flux_splitting           enums/flux_splitting.h:31 (Roe=0, LLF=1, GLF=2, Roe_M=3, LLF_M=4)
 *   time_integrator          numerical_setup.h:26 (RK2=0, RK3=1)
 * Supported: FiniteVolume + {Primitive, Characteristic} reconstruction with
 * the stencils FirstOrder, WENO3, WENO5, WENO5Z, TENO5 or WENO7 (8-cell
 * stencils; not in multi-level cases), the Riemann solvers
 * Hllc, Hllc_LM or Hll and the signal speeds Einfeldt, Davis, Toro or
 * Arithmetic; FluxSplitting with Roe, LocalLaxFriedrichs, GlobalLaxFriedrichs,
 * Roe_M or LocalLaxFriedrichs_M and the same stencils; RK3, or RK2 (TVD, two
 * stages) in the engine and serving forms (alp_rk3_stage and multi-level
 * cases: RK3). WENO5 + Hllc +
 * Einfeldt and WENO5 + Roe are the compiled fast path (FP64 and FP32_FLUX,
 * pencil sweeps); the other choices run through one FP64 face kernel that
 * selects them at run time. GlobalLaxFriedrichs takes the largest |u - c|,
 * |u|, |u + c| of the x velocity over all interior cells before every flux
 * evaluation and uses them in every direction, as the reference does
 * (modular_algorithm_assembler.cpp:957-985, eigendecomposition.h:457-460):
 * over the case in the engine, over the blocks of the call in the stateless
 * calls (which then share one library slot per device, so GLF calls that may
 * overlap must be ordered); multi-level cases reject it.
 * precision: ALP_FP64 (all arithmetic in double) or ALP_FP32_FLUX
 * (reconstruction, smoothness indicators and Riemann fluxes in float; state,
 * RK accumulation, pressure recovery and dt in double). */
enum { ALP_FLUX_SPLITTING = 0, ALP_FINITE_VOLUME = 1 };
enum { ALP_RECON_CONSERVATIVE = 0, ALP_RECON_PRIMITIVE = 1, ALP_RECON_CHARACTERISTIC = 2 };
enum {
  ALP_STENCIL_FIRST_ORDER = 0,
  ALP_STENCIL_WENO3 = 1,
  ALP_STENCIL_WENO5 = 4,
  ALP_STENCIL_WENO5Z = 7,
  ALP_STENCIL_TENO5 = 11,
  ALP_STENCIL_WENO7 = 13
};
enum { ALP_RIEMANN_HLLC = 0, ALP_RIEMANN_HLLC_LM = 1, ALP_RIEMANN_HLL = 2 };
enum {
  ALP_SIGNAL_SPEED_EINFELDT = 0,
  ALP_SIGNAL_SPEED_DAVIS = 1,
  ALP_SIGNAL_SPEED_TORO = 2,
  ALP_SIGNAL_SPEED_ARITHMETIC = 3
};
enum {
  ALP_FLUX_SPLITTING_ROE = 0,
  ALP_FLUX_SPLITTING_LLF = 1,
  ALP_FLUX_SPLITTING_GLF = 2,
  ALP_FLUX_SPLITTING_ROE_M = 3,
  ALP_FLUX_SPLITTING_LLF_M = 4
};
enum { ALP_RK2 = 0, ALP_RK3 = 1 };
enum { ALP_FP64 = 0, ALP_FP32_FLUX = 1 };

typedef struct {
  int convective_term_solver;
  int state_reconstruction;
  int reconstruction_stencil;
  int riemann_solver;
  int signal_speed;
  int flux_splitting;
  int time_integrator;
  int precision;
} alp_scheme;

/* Stiffened-gas material (materials/equations_of_state/stiffened_gas.cpp;
 * ideal gas = B 0). Values are non-dimensional, as the reference holds them
 * after UnitHandler (unit_handler.cpp:33-56). safe selects StiffenedGasSafe. */
typedef struct {
  double gamma;
  double background_pressure;
  int safe;
} alp_material;

/* Library version string and the message of the last failing call (per thread). */
const char *alp_version(void);
const char *alp_last_error(void);

/* Fills *s with the reference's default-like selection: FiniteVolume,
 * Characteristic, WENO5, HLLC, Einfeldt, Roe, RK3, FP64. */
void alp_scheme_default(alp_scheme *s);

/* ---- stateless drop-in calls --------------------------------------------- */

/* Replaces ConvectiveTermSolver<D>::UpdateConvectiveFluxes
 * (solvers/convective_term_contributions/convective_term_solver.h:67-81) for nb
 * blocks at once: fluxes of the average buffer d_blocks (halos filled) are
 * ADDED to the caller-zeroed reference arrays d_fx/d_fy/d_fz, each
 * [nb][NE][ICX+1][ICY+1][ICZ+1]; d_fy / d_fz are ignored below 2 / 3 dims.
 * cell_size as in the reference call. */
int alp_convective_fluxes(int dim, const alp_scheme *scheme, const alp_material *mat,
                          const double *d_blocks, int nb, double cell_size,
                          double *d_fx, double *d_fy, double *d_fz, alp_stream_t stream);

/* Bytes of scratch alp_space_rhs needs for nb blocks. */
size_t alp_space_rhs_workspace_size(int dim, int nb);

/* Replaces SpaceSolver::UpdateFluxes (solvers/space_solver.cpp:50-184) for
 * single-phase blocks without source terms: d_rhs (reference layout) is zeroed
 * and its interior set to the consistency-managed flux divergence / cell_size
 * (space_solver.cpp:131-153). d_workspace: alp_space_rhs_workspace_size bytes. */
int alp_space_rhs(int dim, const alp_scheme *scheme, const alp_material *mat,
                  const double *d_blocks, int nb, double cell_size, double *d_rhs,
                  void *d_workspace, size_t workspace_bytes, alp_stream_t stream);

/* alp_space_rhs for callers that may not allocate device memory; it has no
 * counterpart in the reference. The face-flux scratch is a 16 MiB array of
 * this library in device memory instead of a caller workspace, so at most 28
 * blocks in 3D, 453 in 2D and 10,280 in 1D per call; a larger nb returns
 * ALP_ERR_CAPACITY and launches nothing (after the dim, scheme and material
 * checks of alp_space_rhs, which come first). Nothing is allocated by the
 * call. Every call looks up the array's address in the current context; the
 * first call in a context (the first on a device, or the first after
 * cudaDeviceReset) may load the library's module: make that call before any
 * stream capture. All calls on a device share the one array and it keeps
 * the last call's contents (no call relies on them): calls that may overlap
 * (different streams or threads without ordering) race on it, so order them.
 * Results are those of alp_space_rhs on the same inputs. */
int alp_space_rhs_static(int dim, const alp_scheme *scheme, const alp_material *mat,
                         const double *d_blocks, int nb, double cell_size, double *d_rhs,
                         alp_stream_t stream);

/* Replaces PrimeStateHandler::ConvertConservativesToPrimeStates over every
 * cell (prime_states/prime_state_handler.h:141-152): d_primes [nb][NE][cells]
 * in the order Density, Pressure, VelocityX[, Y[, Z]]. */
int alp_prime_states(int dim, const alp_material *mat, const double *d_blocks, int nb,
                     double *d_primes, alp_stream_t stream);

/* Replaces the same-level part of HaloManager::MaterialHaloUpdate
 * (halo_manager.cpp:59-124, internal_halo_manager.cpp:439-459): d_nbr26
 * [nb][26] holds the neighbour block of each of the 26 directions (offsets
 * (ox,oy,oz) in {-1,0,1}^3 without the centre, x slowest), -1 for a
 * zero-gradient domain face or, in a face slot, -2 for a symmetry wall
 * (SymmetryBoundaryCondition: mirror image with field 2 + d, the momentum or
 * velocity normal to the wall, negated). mode ALP_HALO_ALL: all 26 regions
 * then the reference's full zero-gradient / symmetry slabs; ALP_HALO_FACES:
 * only the 2*dim face regions over the interior extent (all a
 * dimension-split scheme reads). */
enum { ALP_HALO_ALL = 0, ALP_HALO_FACES = 1 };
int alp_halo_update(int dim, double *d_blocks, int nb, int nfields, const int *d_nbr26,
                    int mode, alp_stream_t stream);

/* Replaces ModularAlgorithmAssembler::ComputeTimestepSize
 * (modular_algorithm_assembler.cpp:1777-1997) for one material on one level:
 * *h_dt = min(CFL / (max_cells sum_d(|u_d| + c) / cell_size), t_end - t).
 * d_workspace: 8 bytes of device scratch for the reduction. Synchronises
 * the stream. */
int alp_timestep_size(int dim, const alp_material *mat, const double *d_blocks, int nb,
                      double cell_size, double cfl, double t, double t_end, double *h_dt,
                      void *d_workspace, alp_stream_t stream);

/* One RungeKutta3TVD stage on the interiors (time_integrator.h:98-113,
 * 369-457; runge_kutta_3_TVD.h:41-59): stage 0 saves d_blocks to d_initial,
 * then d_blocks = a0*d_blocks + a1*d_initial + c*dt*d_rhs. */
int alp_rk3_stage(int dim, double *d_blocks, double *d_initial, const double *d_rhs, int nb,
                  int stage, double dt, alp_stream_t stream);

/* ---- engine: device-resident cases, fused step, CUDA graphs ------------- */

typedef struct alp_engine alp_engine;

/* Creates an engine for one dimension and scheme with room for
 * capacity_blocks blocks and max_cases cases. All device memory is
 * allocated here. */
int alp_engine_create(int dim, const alp_scheme *scheme, int capacity_blocks, int max_cases,
                      alp_engine **out);
int alp_engine_destroy(alp_engine *e);

/* Device bytes an engine of this size allocates. */
size_t alp_engine_bytes(int dim, int capacity_blocks, int max_cases);

/* Adds a case: nb blocks of one cell size and material. h_nbr26 [nb][26]
 * gives neighbours as case-local block indices (-1 = zero-gradient domain
 * face, -2 in a face slot = symmetry wall). h_blocks [nb][NE][cells]: only the interiors are read; halos are
 * filled on the device. The case runs until t_end or max_steps (<= 0: no
 * limit). Returns the case id in *case_id. Copies from host memory on the
 * engine stream; h_blocks may be reused once the call returns. */
int alp_engine_add_case(alp_engine *e, const alp_material *mat, double cell_size, double cfl,
                        double t0, double t_end, int max_steps, int nb, const int *h_nbr26,
                        const double *h_blocks, int *case_id);

/* Boundary types of a regular grid, per dimension (periodic[d] below). */
enum { ALP_BOUNDARY_ZERO_GRADIENT = 0, ALP_BOUNDARY_PERIODIC = 1, ALP_BOUNDARY_SYMMETRY = 2 };

/* Adds a case whose initial condition is evaluated on the device, on a
 * regular grid of nblocks[0] x nblocks[1] x nblocks[2] blocks (entries past
 * the engine's dimension ignored); periodic[d] is the boundary type of both
 * domain faces of dimension d: ALP_BOUNDARY_PERIODIC wraps, ALP_BOUNDARY_SYMMETRY
 * puts symmetry walls (SymmetryBoundaryCondition: mirror image, momentum normal
 * to the wall negated), ALP_BOUNDARY_ZERO_GRADIENT (0) zero-gradient faces. Block (bx, by, bz) has index
 * (bx * ny + by) * nz + bz; cell centres are ((16 b + i + 1/2) cell_size).
 * Initial conditions (prime states converted with PrimeStatesToConservatives,
 * prime_states/prime_state_handler.h:195-275):
 *   ALP_IC_QUADRANTS (2D): params x0, y0, then rho, u, v, p of the quadrants
 *     (x<x0, y<y0), (x>=x0, y<y0), (x<x0, y>=y0), (x>=x0, y>=y0)   (18 values)
 *   ALP_IC_BLAST: params centre x, y, z, radius, rho and p inside, rho and p
 *     outside, at rest                                               (8 values)
 * Nothing is copied from the host but the parameters (at most 24). */
enum { ALP_IC_QUADRANTS = 1, ALP_IC_BLAST = 2 };
int alp_engine_add_case_ic(alp_engine *e, const alp_material *mat, double cell_size, double cfl,
                           double t0, double t_end, int max_steps, const int *nblocks,
                           const int *periodic, int ic_type, const double *ic_params,
                           int n_params, int *case_id);

/* ---- initial conditions as expressions -------------------------------------
 * Replaces PrimeStateInitializer (initial_condition/prime_state_initializer.h,
 * GetInitialPrimeStates at prime_state_initializer.cpp:34-85) and the exprtk
 * UserExpression it evaluates (user_expression.h): a material's initial
 * condition as the statements of the reference's input files, e.g.
 *     if (x < 0.5) { density := 1.0; velocityX := 0.0; pressure := 1.0; }
 *     else { density := 0.125; velocityX := 0.0; pressure := 0.1; }
 * compiled once on the host and evaluated per cell on the device. The program
 * reads x, y, z (the cell centre in the units of the expression) and assigns
 * density, velocityX, velocityY, velocityZ, pressure (0 when not assigned).
 * The language is the exprtk subset the reference's inputs use: statements
 * ":=" (also written ": ="), "+=" ... "%=", "var", "if (c) S else S", blocks;
 * expressions with ?:, if(c, a, b), and/or/not (& | !), comparisons, + - * / %
 * ^, implicit multiplication after a number or ')', the usual one- and
 * two-argument functions, variadic min/max, pi; comments // # and block. */
typedef struct alp_ic_program alp_ic_program;

/* UnitHandler references (unit_handler.cpp:33-56): values are divided by
 * density, velocity and density * velocity^2 (pressure); cell centres are in
 * units of length. A null pointer means 1, 1, 1. */
typedef struct {
  double density, velocity, length;
} alp_units;

/* Compiles an initial-condition program (host only). ALP_ERR_INVALID, with
 * the position and the cause in alp_last_error, for a syntax error, an unknown
 * symbol or function, an assignment to a name that is neither a prime state
 * nor declared with var, or nesting deeper than 32 values; the reference's
 * UserExpression throws in those cases. */
int alp_ic_program_create(const char *text, alp_ic_program **out);
void alp_ic_program_destroy(alp_ic_program *p);
/* Instructions, largest stack depth and variable slots of a compiled program. */
int alp_ic_program_info(const alp_ic_program *p, int *n_instructions, int *max_stack,
                        int *n_variables);
/* The compiled program as text, one instruction per line ("CONST 0.5",
 * "LOAD x", "JZ 12", ...), NUL-terminated; *written = its length. */
int alp_ic_program_listing(const alp_ic_program *p, char *buf, int size, int *written);

/* GetInitialPrimeStates for nb nodes of 16^dim cells: node b's cell (i, j, k)
 * has centre d_origins[3b + d] + (index_d + 1/2) cell_size * units->length;
 * the non-dimensional prime states go to d_prims[b][dim + 2][16^dim] in the
 * reference's prime-state order Density, Pressure, VelocityX[, Y[, Z]]
 * (block_definitions/field_details.h:201-212), cells in C order, as
 * GetInitialPrimeStates fills its prime_state_buffer. Device pointers, stream
 * order; the program is copied to the device on its first use. */
int alp_ic_evaluate(const alp_ic_program *p, int dim, int nb, const double *d_origins,
                    double cell_size, const alp_units *units, double *d_prims, void *stream);

/* alp_engine_add_case_ic with the initial condition given by a program on the
 * regular grid of nblocks blocks whose first cell has its corner at origin
 * (units of length; null: 0), cell_size non-dimensional. */
int alp_engine_add_case_expr(alp_engine *e, const alp_material *mat, double cell_size,
                             double cfl, double t0, double t_end, int max_steps,
                             const int *nblocks, const int *periodic, const double *origin,
                             const alp_units *units, const alp_ic_program *prog, int *case_id);

/* Removes a case and frees its blocks. */
int alp_engine_remove_case(alp_engine *e, int case_id);

/* Advances every active case by n steps (each: dt reduction, the RK3 (or RK2)
 * stages of flux / divergence+stage update / halo). Cases whose time reached
 * t_end or whose step budget is spent do no work. Asynchronous. */
int alp_engine_step(alp_engine *e, int n);

/* An engine whose block pools grow and shrink in place: the pools and their
 * scratch are reserved (virtual address range) for max_blocks blocks, and
 * device memory is mapped into them only by alp_engine_reserve, in chunks of
 * 32 MiB per array. Pointers into the pools stay valid as they change, so
 * the step's CUDA graph and a caller's stream order need no update. Such an
 * engine steps on the face-flux path (no fused tile path). Cases are added
 * as to any engine, within the slots reserved. */
int alp_engine_create_elastic(int dim, const alp_scheme *scheme, int max_blocks, int max_cases,
                              alp_engine **out);
/* Backs exactly capacity_blocks block slots of an elastic engine with device
 * memory (mapping or unmapping chunks at the pools' end); when the resident
 * cases reach beyond that, they are moved together first (their order and
 * results are unchanged). Synchronises the engine's streams. ALP_ERR_CAPACITY
 * when the cases need more slots, or the device has no memory left (the
 * engine then keeps the smaller of the two capacities). */
int alp_engine_reserve(alp_engine *e, int capacity_blocks);
/* Block slots backed by memory, blocks in use by cases, and the device bytes
 * of the pools and scratch (what alp_engine_reserve maps, for an elastic
 * engine); any output may be null. */
int alp_engine_capacity(alp_engine *e, int *capacity_blocks, int *used_blocks,
                        size_t *pool_bytes);

/* Copies a case's state (reference layout, halos included) to h_blocks and
 * its time / step count. Synchronises the engine stream. Any of the outputs
 * may be null. */
int alp_engine_get_case(alp_engine *e, int case_id, double *h_blocks, double *t, int *steps);

/* alp_engine_add_case / alp_engine_get_case with the blocks' interiors only:
 * h_interior [nb][NE][16][16][16] (16^dim cells per field, C order), which is
 * all the engine keeps of a case (its pools' halos are never read while
 * stepping), so a transfer moves 16^3 instead of 24^3 cells per field in 3D.
 * The copy is staged in the engine's own device scratch and placed into (or
 * taken from) the pool by a kernel on the engine stream; both calls
 * synchronise that stream. */
int alp_engine_add_case_interior(alp_engine *e, const alp_material *mat, double cell_size,
                                 double cfl, double t0, double t_end, int max_steps, int nb,
                                 const int *h_nbr26, const double *h_interior, int *case_id);
int alp_engine_get_case_interior(alp_engine *e, int case_id, double *h_interior, double *t,
                                 int *steps);

/* Checkpoint and resume of one case: what the reference's restart file keeps
 * of a simulation (RestartManager::WriteRestartFile / RestoreSimulation,
 * input_output/restart_manager.h:66-68: the time, and every node's
 * conservatives in the block layout), plus the case's own settings. A case
 * restored from its checkpoint continues exactly as the uninterrupted case:
 * state, time and step count are the same, and nothing else carries over
 * between steps. The checkpoint records the engine's scheme selection
 * (precision and time integrator included); restoring into an engine with
 * another selection returns ALP_ERR_INVALID, since the case would continue
 * with other numerics. */
typedef struct {
  int dim, nb;
  int steps, max_steps;  /* steps taken; the step budget (<= 0: none) */
  double t, t_end, cfl, cell_size;
  alp_material material;
  alp_scheme scheme;     /* the selection the case was stepped with */
} alp_case_checkpoint;

/* Fills *info, and (when not null) h_nbr26 [nb][26] with the case-local
 * neighbour table and h_blocks [nb][NE][cells] with the state (halos filled).
 * Synchronises the engine stream. */
int alp_engine_checkpoint_case(alp_engine *e, int case_id, alp_case_checkpoint *info,
                               int *h_nbr26, double *h_blocks);
/* Adds a case from a checkpoint (interiors of h_blocks read); its step count
 * continues from info->steps. */
int alp_engine_restore_case(alp_engine *e, const alp_case_checkpoint *info, const int *h_nbr26,
                            const double *h_blocks, int *case_id);

/* True (1) when every case is done; synchronises. */
int alp_engine_all_done(alp_engine *e, int *done);

/* Engine stream, for callers that order their own work after the engine. */
alp_stream_t alp_engine_stream(alp_engine *e);

/* Enables (1) or disables (0) CUDA-graph replay of the step (default on). */
int alp_engine_set_graph(alp_engine *e, int enabled);

/* Number of stepping candidates of alp_engine_autotune / alp_engine_set_path. */
#define ALP_STEP_CANDIDATES 6

/* Times the stepping candidates on the engine's resident cases and keeps the
 * fastest: 0 = face fluxes (128-thread blocks, all directions in one launch)
 * + divergence/stage update, 1 = the same with 64-thread blocks, 2 = pencil
 * sweeps (one thread per line of cells, 17 faces with a sliding stencil
 * window, flux differences summed in the kernels and the RK stage applied by
 * the last direction; not available in the strict build; default schemes
 * only), 3 = candidate 0 in batches of about 64 blocks, the stage update of
 * one batch on a second stream overlapping the face fluxes of the next (same
 * arithmetic), 4 = fused tile stages with 16 warps per CTA, 5 = the same with
 * 12 warps. The fused tile stages (3D engines with WENO5 + HLLC/Einfeldt or
 * Roe splitting, RK3 or RK2) advance all steps of one alp_engine_step call in
 * one persistent launch: per (step, stage, block) work item, the block's cell
 * planes and the neighbours' cells beyond its faces are staged into shared
 * memory by TMA, every face flux is computed once into shared memory and the
 * divergence and RK stage are applied there, so no face flux reaches HBM. Its
 * arithmetic is that of candidate 0, so results are bit-identical; it is the
 * default where it applies. Each candidate runs trial_steps steps whose last
 * stage writes scratch memory and that are not committed, so the cases' state
 * and time are unchanged. *chosen receives the candidate (-1 when no case is
 * resident), ms_per_step[ALP_STEP_CANDIDATES] (may be null) the measured time
 * per step of each candidate (-1 when not run). Synchronises. */
int alp_engine_autotune(alp_engine *e, int trial_steps, int *chosen, float *ms_per_step);

/* Selects a stepping candidate (as numbered for alp_engine_autotune);
 * ALP_ERR_INVALID for a candidate that cannot step this engine. */
int alp_engine_set_path(alp_engine *e, int candidate);

/* The engine's current stepping candidate (-1 for a null engine). */
int alp_engine_path(alp_engine *e);

/* Number of kernel launches one engine step issues (the fused tile stages:
 * per alp_engine_step call, whatever its step count). */
int alp_engine_launches_per_step(alp_engine *e);

/* Number of kernel launches alp_engine_step(e, n) issues. */
int alp_engine_launches(alp_engine *e, int n);

/* ---- multi-level cases: leaves of a block tree, local time stepping ----- */

/* A case whose blocks are the leaves of a block tree (the reference's
 * multiresolution levels, topology/node.cpp) over a box of n0[0] x n0[1] x
 * n0[2] level-0 nodes with zero-gradient domain faces. Leaf b has level
 * h_level[b] (0..6) and integer node coordinates h_coord[3b..3b+2] in units of
 * its own node size; its cell size is h0 / 2^level. Face neighbours may differ
 * by one level at most. Time stepping as ModularAlgorithmAssembler::Advance
 * (modular_algorithm_assembler.cpp:575-874): a macro step is 2^lmax micro
 * steps, micro step t integrates the levels of GetLevels(t) (:2564-2573), each
 * with the sum of its last 2^(lmax-level) micro time steps (Integrate,
 * :1068-1098); the micro time step is ComputeTimestepSize over all leaves with
 * the finest cell size (:1925-1982). Halo cells across a level jump are the
 * average of the finer leaves (Multiresolution::Average,
 * multiresolution/multiresolution.h:94-166) or, on the finer side, the
 * fifth-order prediction from the coarser level (Multiresolution::Prediction,
 * multiresolution.cpp:146-283), as the reference's jump halos hold them; node
 * positions the prediction reads that are not leaves are averaged or predicted
 * in turn. Conservation at jumps as JumpFluxAdjustment
 * (modular_algorithm_assembler.cpp:1347-1636): jump-face fluxes integrated
 * with the integrator's jump multipliers (SSP-RK3 1/6, 1/6, 2/3; TVD-RK2 1/2, 1/2),
 * fine sums averaged onto the parent faces
 * after each fine step, coarse cells corrected after each coarse step.
 * h_blocks: [nleaf][NE][cells], interiors read. All levels run in the same
 * batched launches; one CUDA graph per macro step. */
typedef struct alp_levels alp_levels;
int alp_levels_create(int dim, const alp_scheme *scheme, const alp_material *mat, const int *n0,
                      double h0, int nleaf, const int *h_level, const int *h_coord, double cfl,
                      double t0, double t_end, int max_macro_steps, const double *h_blocks,
                      alp_levels **out);
int alp_levels_destroy(alp_levels *m);
/* Advances n macro steps (asynchronous). */
int alp_levels_step(alp_levels *m, int n_macro);
/* Copies the leaves (interiors valid) and the time / macro steps reached;
 * synchronises. ALP_ERR_NUMERIC once a non-finite state stopped the case. */
int alp_levels_get(alp_levels *m, double *h_blocks, double *t, int *macro_steps);
/* Ghost blocks at level jumps, finest level, interior cells x time steps per
 * macro step summed over the leaves, kernel launches per macro step. */
int alp_levels_info(alp_levels *m, int *n_ghosts, int *max_level,
                    long long *cell_updates_per_macro_step, int *launches_per_macro_step);
alp_stream_t alp_levels_stream(alp_levels *m);
/* Test of the ghost kernel's bounded waits (no ALPACA counterpart): the next
 * macro step's first ghost launch skips its first group, so the launch's waits
 * for that group run out (about a second) and set the engine's error word;
 * the next alp_levels_get returns ALP_ERR_CUDA and clears it. The leaves are
 * not valid after that step. ALP_ERR_INVALID before the first alp_levels_step
 * (nothing recorded yet) and when that launch has one group. */
int alp_levels_test_stall_ghosts(alp_levels *m);

/* ---- serving: continuous batching of independent cases ------------------ */

/* One request: a case on a regular block grid with a device-evaluated initial
 * condition (see alp_engine_add_case_ic; ic_type ALP_IC_PROGRAM: the program,
 * origin and units of alp_engine_add_case_expr, ic_params unused, units all 0
 * meaning 1), arriving arrival_s seconds after alp_serve starts. h_result,
 * when not null, receives the final state (reference layout, halos filled)
 * before the case leaves the pool. */
enum { ALP_IC_PROGRAM = 3 };
typedef struct {
  int dim;
  int nblocks[3];
  int periodic[3];
  double cell_size;
  alp_material material;
  double cfl;
  double t_end;
  int max_steps;
  int ic_type;
  double ic_params[24];
  int n_params;
  double arrival_s;
  double *h_result;
  const alp_ic_program *program;
  double origin[3];
  alp_units units;
} alp_request;

/* Wall-clock times are seconds after the start of alp_serve. */
typedef struct {
  double arrival_s;
  double admitted_s;
  double finished_s;
  double t;       /* simulated time reached */
  int steps;      /* SSP-RK3 steps taken */
  int status;     /* ALP_OK, ALP_ERR_NUMERIC, ALP_ERR_CAPACITY or ALP_ABORTED */
} alp_result;

typedef struct {
  size_t hbm_budget_bytes;  /* device memory for case state, shared by the 2D and 3D
                               pools: alp_engine_bytes(dim, 1, 0) per backed block slot
                               (the pools map it in 32 MiB chunks, so the device bytes
                               exceed it by less than 5 chunks per dimension) */
  alp_scheme scheme;
  int max_cases;            /* resident cases per dimension */
  int steps_per_poll;       /* steps between completion checks */
  int one_at_a_time;        /* 1: admit a case only into an idle GPU (baseline) */
  int shortest_first;       /* 1: step only the resident cases with the least remaining
                               work (cells x steps left) up to step_set_cells cells, holding
                               the others; 0: every resident case steps */
  double step_set_cells;    /* cells stepped together under shortest_first (>= one case) */
  const char *abort_file;   /* null, or a path checked after every poll, as the reference
                               checks its ABORTFILE after each micro step
                               (modular_algorithm_assembler.cpp:903-907), and while no case
                               is resident (the loop waits for arrivals): once the file
                               exists, every request ends with status ALP_ABORTED (resident
                               cases with their state, time and steps so far, written to
                               h_result; the others with none) and alp_serve returns
                               ALP_ABORTED */
} alp_server_config;

/* Serves n requests: admits arrived requests whose blocks fit (FIFO with
 * backfill), advances all resident cases in the engines' batched steps (2D and
 * 3D on separate streams), retires finished cases. Blocks until every request
 * has finished; results[i] belongs to reqs[i]. *makespan_s (may be null)
 * receives the wall time from start to the last completion. Returns ALP_OK, or
 * ALP_ERR_CAPACITY when a request could not fit into an empty pool (its result
 * carries that status; the others are served). */
int alp_serve(const alp_server_config *cfg, const alp_request *reqs, int n, alp_result *results,
              double *makespan_s);

#ifdef __cplusplus
}
#endif
#endif
