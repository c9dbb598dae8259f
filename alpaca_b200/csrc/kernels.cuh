// Launch interface of the block kernels (implemented in kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "layout.cuh"

namespace alp {

// Scheme ids of the compiled instantiations. They correspond to the
// reference's compile-time selections (user_specifications):
//   FV_CHAR : ConvectiveTermSolvers::FiniteVolume + StateReconstructionType::Characteristic
//   FV_PRIM : ConvectiveTermSolvers::FiniteVolume + StateReconstructionType::Primitive
//   FS_ROE  : ConvectiveTermSolvers::FluxSplitting + FluxSplitting::Roe
// all with ReconstructionStencils::WENO5, RiemannSolvers::Hllc, SignalSpeed::Einfeldt.
enum Scheme { FV_CHAR = 0, FV_PRIM = 1, FS_ROE = 2 };
enum Precision { FP64 = 0, FP32_FLUX = 1 };

// Further selections of the reference's plugin surface, dispatched at run time
// in FP64 (schemes_ext.cuh); the values are those of the reference's enums
// (stencil_setup.h:26-43, riemann_solver_settings.h:47, enums/signal_speed.h:31,
// enums/flux_splitting.h:31).
enum StencilId {
  ST_FIRST_ORDER = 0,
  ST_WENO3 = 1,
  ST_WENO5 = 4,
  ST_WENO5Z = 7,
  ST_TENO5 = 11,
  ST_WENO7 = 13
};
enum RiemannId { RS_HLLC = 0, RS_HLLC_LM = 1, RS_HLL = 2 };
enum SignalSpeedId { SS_EINFELDT = 0, SS_DAVIS = 1, SS_TORO = 2, SS_ARITHMETIC = 3 };
enum SplittingId { FSP_ROE = 0, FSP_LLF = 1, FSP_GLF = 2, FSP_ROE_M = 3, FSP_LLF_M = 4 };

struct SchemeOptions {
  int stencil = ST_WENO5, riemann = RS_HLLC, signal = SS_EINFELDT, splitting = FSP_ROE;
  __host__ __device__ bool is_default() const {
    return stencil == ST_WENO5 && riemann == RS_HLLC && signal == SS_EINFELDT &&
           splitting == FSP_ROE;
  }
};

// Work description shared by the launchers. A null `work` means the identity
// worklist (item i is slot i); a null `meta` means every block uses `def`.
struct Launch {
  int dim;
  int scheme;
  int precision;
  double *U;               // [slots][NE][cells]
  int const *work;         // [nwork] slot ids, or null
  int nwork;
  BlockMeta const *meta;   // [slots], or null
  BlockMeta def;
  cudaStream_t stream;
  SchemeOptions opt = SchemeOptions();  // non-default: FP64 run-time dispatch, face kernels only
  // GlobalLaxFriedrichs wave speeds |u-c|, |u|, |u+c| per case, as the bit
  // patterns of non-negative doubles, 4 words per case (launch_glf_maxima)
  unsigned long long const *glf = nullptr;
  // launch_face_flux_all only: the work-list positions the launch covers, in
  // order (nwork of them; null: positions 0 .. nwork-1). Fluxes still go to
  // the F slot of the work-list position.
  int const *items = nullptr;
};

// GlobalLaxFriedrichs: zeroes glf[0 .. 4 ncases) and sets, per case, the
// largest |u - c|, |u|, |u + c| of the x velocity over the interior cells of
// the launch's blocks with positive density (ComputeMaxEigenvaluesOnBlock,
// eigendecomposition.cpp:46-110, maxima over blocks as
// modular_algorithm_assembler.cpp:957-985).
cudaError_t launch_glf_maxima(Launch const &L, unsigned long long *glf, int ncases);
// The library's slot for the stateless calls (one case, id 0).
unsigned long long *glf_stateless_slot();

// Face fluxes of direction `dir` for every work item into
// F[item * flux_item_stride + field * FACES + face] (reference flux-array
// layout). accumulate: += (drop-in contract), else = (zero for skipped faces).
cudaError_t launch_face_flux(Launch const &L, int dir, double *F, long long flux_item_stride,
                             bool accumulate, int block_threads = 0);

// SpaceSolver right-hand side: rhs (reference layout, all cells) = 0, interior
// = consistency-managed flux divergence / cell size. F as written by
// launch_face_flux for each direction at F + dir * dir_stride.
cudaError_t launch_divergence(Launch const &L, double const *F, long long flux_item_stride,
                              long long dir_stride, double *rhs);

// Face fluxes of every direction of every work item in one launch (engine):
// stencils gathered from neighbour interiors through nbr26 (zero gradient at
// domain faces), so block halos are never read; items of inactive cases
// (dt == 0) skipped. Direction d goes to F + d * dir_stride.
cudaError_t launch_face_flux_all(Launch const &L, int const *nbr26, CaseState const *cases,
                                 double *F, long long flux_item_stride, long long dir_stride,
                                 int threads = 128);

// One SSP-RK3 stage of every work item by pencil sweeps (engine fast path):
// the faces of each line of cells along x, then y, then z, with the
// per-cell flux differences accumulated in R ([slot][NE][interior cells]) and
// the last direction applying Uout = (stage ? a0 Uin + a1 U0 : Uin) + c dt
// ((dFx + dFy) + dFz) / h, Uin = L.U. Uout may alias U0, not Uin.
cudaError_t launch_pencil_stage(Launch const &L, double const *U0, double *Uout, double *R,
                                int const *nbr26, CaseState const *cases, int stage);

// Runge-Kutta stage on the interior: Uout = (first stage ? Uin : a0*Uin +
// a1*U0) + c*dt*div(F) with Uin = L.U; stage 0-2 the SSP-RK3 stages, 3-4 the
// TVD-RK2 stages; dt per case from cases[meta.case_id].dt (skip when dt == 0),
// or `dt` for every block when cases is null. Uout may alias U0, not Uin.
cudaError_t launch_stage_update(Launch const &L, double const *U0, double *Uout, double const *F,
                                long long flux_item_stride, long long dir_stride, int stage,
                                CaseState const *cases, double dt);

// RK3 stage from a reference-layout RHS buffer, blocks 0..nb-1.
cudaError_t launch_rk_stage_rhs(int dim, double *U, double *U0, double const *rhs, int nb,
                                int stage, double dt, cudaStream_t stream);

// Halo update of the work items' blocks. nbr26: [slots][26] neighbour slot ids
// (-1 = domain face with zero gradient). faces_only copies the 2*dim face
// slabs over the interior extent (all the dimension-split scheme reads);
// otherwise all 26 regions followed by the reference's full zero-gradient slabs.
// nfields: number of fields per block (NE for conservative buffers).
// When cases != null, blocks of cases with dt == 0 are skipped.
cudaError_t launch_halo(Launch const &L, int const *nbr26, bool faces_only, int nfields,
                        CaseState const *cases);

// Prime states of every cell (reference layout) into P.
cudaError_t launch_prime_states(Launch const &L, double *P);

// Max signal speed per case over the work items' interior cells, folded into
// cases[case_id].smax_bits; with cases == null into *smax_bits_out.
cudaError_t launch_signal_speed(Launch const &L, CaseState *cases,
                                unsigned long long *smax_bits_out);

// Device-evaluated initial conditions (parameters by value).
enum IcType { IC_QUADRANTS = 1, IC_BLAST = 2 };
struct IcParams {
  double v[24];
};
// Fills the nblocks[0] x nblocks[1] x nblocks[2] blocks stored from slot
// `first` (C order) with the initial condition `type` (stiffened gas gamma, B).
cudaError_t launch_initial_condition(int dim, double *U, int first, int const nblocks[3],
                                     double cell_size, double gamma, double B, int type,
                                     IcParams const &params, cudaStream_t stream);

// dt for every case from its smax (ComputeTimestepSize), then resets smax;
// with dtflag, also sets dtflag[c] = 1 (dt of the first step of a tile-stage
// launch is ready).
cudaError_t launch_dt_finalize(CaseState *cases, int ncases, cudaStream_t stream,
                               int *dtflag = nullptr);
// Interiors of the nb pool blocks from slot `first` to (to_pool false) or from
// (to_pool true) packed [nb][NE][ICX][ICY][ICZ]; halos untouched.
cudaError_t launch_interior_copy(int dim, double *U, int first, int nb, double *packed,
                                 bool to_pool, cudaStream_t stream);
// t += dt, steps += (dt > 0) for every case.
cudaError_t launch_step_commit(CaseState *cases, int ncases, cudaStream_t stream);

}  // namespace alp
