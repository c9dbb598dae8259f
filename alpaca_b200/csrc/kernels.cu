// Block kernels of the ALPACA right-hand side and SSP-RK3 stage update on sm_100a.
//
// Data stays in the reference's block layout (layout.cuh). One launch per sweep
// direction computes the face fluxes of all work items (thread per face, the
// 6-cell stencil read through L1), one launch applies the flux divergence and
// the RK3 stage, one launch refreshes the face halos from neighbour interiors.
#include <cfloat>
#include <cstdio>


#include "kernels.cuh"
#include "face.cuh"
#include "rotate.cuh"
#include "step_common.cuh"

namespace alp {

namespace {

__device__ __forceinline__ int slot_of(int const *work, int item) {
  return work ? work[item] : item;
}

// ---------------------------------------------------------------------------
// face flux
// ---------------------------------------------------------------------------

template <int DIM, int DIR> struct FaceMap {
  static constexpr int O1 = DIR == 0 ? 1 : 0;
  static constexpr int O2 = DIR == 2 ? 1 : 2;
  static constexpr int E1 = Geo<DIM>::ic(O1);
  static constexpr int E2 = Geo<DIM>::ic(O2);
  static constexpr int COUNT = (IC + 1) * E1 * E2;
  // Thread t -> face (a along DIR, p1, p2 across). Consecutive threads walk the
  // fastest-varying stored dimension so that stencil loads coalesce.
  __device__ static void decode(int t, int &a, int &p1, int &p2) {
    if constexpr (DIR == DIM - 1) {
      a = t % (IC + 1);
      int const r = t / (IC + 1);
      p1 = r / E2;
      p2 = r % E2;
    } else {
      a = t / (E1 * E2);
      p1 = (t / E2) % E1;
      p2 = t % E2;
    }
  }
};

// Minimum resident 128-thread CTAs per SM of the face kernels, which caps
// their registers (168 / 128 / 102 at 3 / 4 / 5); compile-time tunable.
// Measured on the FP64 128^3 step: FV char 4 CTAs 1.60 ms vs 3: 1.71, 5: 1.66;
// FV prim 5: 1.37 vs 4: 1.46, 6: 1.37; flux splitting 3: 1.91 vs 1-2: 2.23
// (at 4 it spills ~0.7 KB per thread).
#ifndef ALP_FS_ROE_CTAS
#define ALP_FS_ROE_CTAS 3
#endif
#ifndef ALP_FV_CHAR_CTAS
#define ALP_FV_CHAR_CTAS 4
#endif
#ifndef ALP_FV_PRIM_CTAS
#define ALP_FV_PRIM_CTAS 5
#endif
// FP32-flux instantiations (fewer live doubles) have their own limits
// (measured on the 128^3 step: FS 4 CTAs 2.05 ms vs 3: 2.23, 2: 2.86; FV
// char 5 CTAs 1.56 ms vs 4: 1.64, 6: 1.59; FV prim 5: 1.455 vs 6: 1.48).
#ifndef ALP_FS_ROE_CTAS_F32
#define ALP_FS_ROE_CTAS_F32 4
#endif
#ifndef ALP_FV_CHAR_CTAS_F32
#define ALP_FV_CHAR_CTAS_F32 5
#endif
#ifndef ALP_FV_PRIM_CTAS_F32
#define ALP_FV_PRIM_CTAS_F32 ALP_FV_PRIM_CTAS
#endif
template <int SCHEME, typename T = double> struct FaceOccupancy {
  static constexpr bool f32 = sizeof(T) == 4;
  static constexpr int min_ctas =
      SCHEME == FV_CHAR ? (f32 ? ALP_FV_CHAR_CTAS_F32 : ALP_FV_CHAR_CTAS)
      : SCHEME == FV_PRIM ? (f32 ? ALP_FV_PRIM_CTAS_F32 : ALP_FV_PRIM_CTAS)
                          : (f32 ? ALP_FS_ROE_CTAS_F32 : ALP_FS_ROE_CTAS);
};

// Stores one face's fluxes in the reference flux-array layout: = (zero for a
// skipped face) or, for the drop-in contract, += (skipped faces untouched).
template <int DIM, int DIR, bool ACCUM>
__device__ __forceinline__ void write_flux(double *__restrict__ F, int item, long long stride,
                                           int a, int p1, int p2, bool valid,
                                           double const (&flux)[DIM + 2]) {
  using G = Geo<DIM>;
  using M = FaceMap<DIM, DIR>;
  int fi[3];
  fi[DIR] = a;
  fi[M::O1] = p1 + 1;
  fi[M::O2] = p2 + 1;
  double *fo = F + (long long)item * stride + G::face(fi[0], fi[1], fi[2]);
#pragma unroll
  for (int f = 0; f < DIM + 2; ++f) {
    double const v = valid ? flux[f] : 0.0;
    if (ACCUM) {
      if (valid) fo[f * G::FACES] += v;
    } else {
      fo[f * G::FACES] = v;
    }
  }
}

// Stencil of the face a (between cells a-1 and a along DIR) at transverse
// position (p1, p2): cells a-3 .. a+2 in interior numbering, all fields.
// GATHER: cells outside the interior along DIR come from the neighbour blocks'
// interiors (nbr26; zero gradient at domain faces) instead of the block's own
// halo cells, so no halo copy is needed between stages.
template <int DIM, int DIR, bool GATHER>
__device__ __forceinline__ double const *stencil_cell(double const *__restrict__ U,
                                                      double const *blk, int c, int cell0,
                                                      int nlo, int nhi) {
  using G = Geo<DIM>;
  constexpr int step = DIR == 0 ? G::TCY * G::TCZ : (DIR == 1 ? G::TCZ : 1);
  // cell0: offset of (transverse position, DIR index 0) in the block
  if (GATHER && c < HS)
    return nlo >= 0 ? U + (size_t)nlo * G::BLOCK_DOUBLES + cell0 + (c + IC) * step
                    : blk + cell0 + HS * step;
  if (GATHER && c >= HS + IC)
    return nhi >= 0 ? U + (size_t)nhi * G::BLOCK_DOUBLES + cell0 + (c - IC) * step
                    : blk + cell0 + (HS + IC - 1) * step;
  return blk + cell0 + c * step;
}

template <int DIM, int DIR>
__device__ __forceinline__ int line_origin(int p1, int p2) {
  using G = Geo<DIM>;
  using M = FaceMap<DIM, DIR>;
  int c[3];
  c[DIR] = 0;
  c[M::O1] = G::fic(M::O1) + p1;
  c[M::O2] = G::fic(M::O2) + p2;
  return G::cell(c[0], c[1], c[2]);
}

template <int DIM, int DIR>
__device__ __forceinline__ void load_cell(double const *src, double (&dst)[DIM + 2]) {
#pragma unroll
  for (int f = 0; f < DIM + 2; ++f) dst[f] = __ldg(src + f * Geo<DIM>::CELLS);
}

// Cell c of a stencil line (stencil_cell), with symmetry walls: a neighbour
// entry of -2 across the block face mirrors the line about the wall and negates
// the momentum normal to it (symmetry_boundary_condition.h:60-113, 148-217;
// boundary_constants.h:35-46, 167-209); -1 is zero gradient.
template <int DIM, int DIR, bool GATHER>
__device__ __forceinline__ void stencil_load(double const *__restrict__ U, double const *blk,
                                             int c, int cell0, int nlo, int nhi,
                                             double (&dst)[DIM + 2]) {
  constexpr int step = DIR == 0 ? Geo<DIM>::TCY * Geo<DIM>::TCZ : (DIR == 1 ? Geo<DIM>::TCZ : 1);
  if (GATHER && ((c < HS && nlo == -2) || (c >= HS + IC && nhi == -2))) {
    int const m = c < HS ? 2 * HS - 1 - c : 2 * (HS + IC) - 1 - c;
    load_cell<DIM, DIR>(blk + cell0 + m * step, dst);
    dst[MOMX + DIR] = -1.0 * dst[MOMX + DIR];
    return;
  }
  load_cell<DIM, DIR>(stencil_cell<DIM, DIR, GATHER>(U, blk, c, cell0, nlo, nhi), dst);
}

// Flux of the face with thread index t of direction DIR of the block in `slot`.
template <int DIM, int DIR, int SCHEME, typename T, bool ACCUM, bool GATHER,
          typename P = DefaultPolicy, int W = 6>
__device__ __forceinline__ void face_flux(double const *__restrict__ U,
                                          int const *__restrict__ nbr26, int slot, int item,
                                          int t, BlockMeta const &bm, double *__restrict__ F,
                                          long long stride, P const &pol = P()) {
  using G = Geo<DIM>;
  using M = FaceMap<DIM, DIR>;
  constexpr int NE = G::NE;
  Eos const eos{bm.gamma, bm.B, bm.safe};
  int a, p1, p2;
  M::decode(t, a, p1, p2);
  double const *blk = U + (size_t)slot * G::BLOCK_DOUBLES;
  int const cell0 = line_origin<DIM, DIR>(p1, p2);
  // low / high neighbour along DIR (26-table slots of W,E / S,N / B,T)
  constexpr int lo_slot = DIR == 0 ? 4 : (DIR == 1 ? 10 : 12);
  constexpr int hi_slot = DIR == 0 ? 21 : (DIR == 1 ? 15 : 13);
  int const nlo = GATHER && a < W / 2 ? __ldg(nbr26 + (size_t)slot * 26 + lo_slot) : 0;
  int const nhi = GATHER && a > IC - W / 2 ? __ldg(nbr26 + (size_t)slot * 26 + hi_slot) : 0;
  double cons[W][NE];
#pragma unroll
  for (int m = 0; m < W; ++m)
    stencil_load<DIM, DIR, GATHER>(U, blk, HS + a - W / 2 + m, cell0, nlo, nhi, cons[m]);
  double fd[NE];
  bool valid;
  if constexpr (DIM == 3 && DIR != 0) {
    // 3D y and z faces: the x-face computation of the rotated stencil
    // (canon_field), the same code as the fused tile kernel
    double rc[W][NE];
#pragma unroll
    for (int m = 0; m < W; ++m)
#pragma unroll
      for (int c = 0; c < NE; ++c) rc[m][c] = cons[m][canon_field(DIR, c)];
    double rf[NE];
    valid = face_compute<3, 0, SCHEME, T, P, W>(eos, bm.B, rc, rf, pol);
#pragma unroll
    for (int c = 0; c < NE; ++c) fd[canon_field(DIR, c)] = rf[c];
  } else {
    valid = face_compute<DIM, DIR, SCHEME, T, P, W>(eos, bm.B, cons, fd, pol);
  }
  write_flux<DIM, DIR, ACCUM>(F, item, stride, a, p1, p2, valid, fd);
}

// One direction over all work items (drop-in calls: halos from the buffer).
template <int DIM, int DIR, int SCHEME, typename T, bool ACCUM>
__global__ void __launch_bounds__(128, FaceOccupancy<SCHEME, T>::min_ctas)
face_flux_kernel(double const *__restrict__ U, int const *__restrict__ work,
                 BlockMeta const *__restrict__ meta, BlockMeta def, double *__restrict__ F,
                 long long stride) {
  int const t = blockIdx.y * blockDim.x + threadIdx.x;
  if (t >= FaceMap<DIM, DIR>::COUNT) return;
  int const item = blockIdx.x;
  int const slot = slot_of(work, item);
  BlockMeta const bm = meta ? meta[slot] : def;
  face_flux<DIM, DIR, SCHEME, T, ACCUM, false>(U, nullptr, slot, item, t, bm, F, stride);
}

// Every direction of every work item in one launch (engine): blockIdx.z is the
// direction, stencils gathered from neighbours, direction d written to
// F + d * dstride. Items whose case is inactive (dt == 0) are skipped.
template <int DIM, int SCHEME, typename T>
__global__ void __launch_bounds__(128, FaceOccupancy<SCHEME, T>::min_ctas)
face_flux_all_kernel(double const *__restrict__ U, int const *__restrict__ work,
                     BlockMeta const *__restrict__ meta, int const *__restrict__ nbr26,
                     CaseState const *__restrict__ cases, double *__restrict__ F,
                     long long stride, long long dstride, int chunks,
                     int const *__restrict__ items) {
  // grid (items x chunks, 1, dir): an item's chunks are consecutive, so the
  // CTAs resident at any time share few blocks' stencils (a few MB of L2
  // instead of one stencil plane of every item in the launch). items (when
  // given): the work-list position of each launch position
  int const chunk = (int)(blockIdx.x % chunks);
  int const pos = (int)(blockIdx.x / chunks);
  int const item = items ? items[pos] : pos;
  int const t = chunk * blockDim.x + threadIdx.x;
  int const slot = work[item];
  BlockMeta const bm = meta[slot];
  if (!(cases[bm.case_id].dt > 0.0)) return;
  int const dir = blockIdx.z;
  if (dir == 0) {
    if (t < FaceMap<DIM, 0>::COUNT)
      face_flux<DIM, 0, SCHEME, T, false, true>(U, nbr26, slot, item, t, bm, F, stride);
  } else if (DIM > 1 && dir == 1) {
    if (t < FaceMap<DIM, 1>::COUNT)
      face_flux<DIM, (DIM > 1 ? 1 : 0), SCHEME, T, false, true>(U, nbr26, slot, item, t, bm,
                                                                 F + dstride, stride);
  } else if (DIM > 2) {
    if (t < FaceMap<DIM, 2>::COUNT)
      face_flux<DIM, (DIM > 2 ? 2 : 0), SCHEME, T, false, true>(U, nbr26, slot, item, t, bm,
                                                                 F + 2 * dstride, stride);
  }
}

// The run-time selected schemes read 6-cell stencils (i-2 .. i+3), or 8-cell
// stencils (i-3 .. i+4) when the stencil is WENO7; the narrower stencils use
// the middle cells. The 8-wide instantiation holds 33 % more stencil state, so
// the launchers pick it only for WENO7.
inline bool ext_wide(SchemeOptions const &o) { return o.stencil == ST_WENO7; }

// The policy of one block: the GlobalLaxFriedrichs wave speeds of its case.
__device__ __forceinline__ ExtPolicy block_policy(ExtPolicy pol, BlockMeta const &bm,
                                                  unsigned long long const *glf) {
  if (glf && pol.o.splitting == FSP_GLF)
    for (int k = 0; k < 3; ++k) pol.glf[k] = __longlong_as_double(glf[4 * bm.case_id + k]);
  return pol;
}

// The same two kernels for the run-time selected schemes (ExtPolicy, FP64).
template <int DIM, int DIR, int SCHEME, bool ACCUM, int W>
__global__ void __launch_bounds__(128)
face_flux_ext_kernel(double const *__restrict__ U, int const *__restrict__ work,
                     BlockMeta const *__restrict__ meta, BlockMeta def, double *__restrict__ F,
                     long long stride, ExtPolicy pol, unsigned long long const *__restrict__ glf) {
  int const t = blockIdx.y * blockDim.x + threadIdx.x;
  if (t >= FaceMap<DIM, DIR>::COUNT) return;
  int const item = blockIdx.x;
  int const slot = slot_of(work, item);
  BlockMeta const bm = meta ? meta[slot] : def;
  face_flux<DIM, DIR, SCHEME, double, ACCUM, false, ExtPolicy, W>(U, nullptr, slot, item, t, bm, F,
                                                               stride, block_policy(pol, bm, glf));
}

template <int DIM, int SCHEME, int W>
__global__ void __launch_bounds__(128)
face_flux_all_ext_kernel(double const *__restrict__ U, int const *__restrict__ work,
                         BlockMeta const *__restrict__ meta, int const *__restrict__ nbr26,
                         CaseState const *__restrict__ cases, double *__restrict__ F,
                         long long stride, long long dstride, ExtPolicy pol0,
                         unsigned long long const *__restrict__ glf,
                         int const *__restrict__ items) {
  int const t = blockIdx.y * blockDim.x + threadIdx.x;
  int const item = items ? items[blockIdx.x] : (int)blockIdx.x;
  int const slot = work[item];
  BlockMeta const bm = meta[slot];
  if (!(cases[bm.case_id].dt > 0.0)) return;
  ExtPolicy const pol = block_policy(pol0, bm, glf);
  int const dir = blockIdx.z;
  if (dir == 0) {
    if (t < FaceMap<DIM, 0>::COUNT)
      face_flux<DIM, 0, SCHEME, double, false, true, ExtPolicy, W>(U, nbr26, slot, item, t, bm, F,
                                                                stride, pol);
  } else if (DIM > 1 && dir == 1) {
    if (t < FaceMap<DIM, 1>::COUNT)
      face_flux<DIM, (DIM > 1 ? 1 : 0), SCHEME, double, false, true, ExtPolicy, W>(
          U, nbr26, slot, item, t, bm, F + dstride, stride, pol);
  } else if (DIM > 2) {
    if (t < FaceMap<DIM, 2>::COUNT)
      face_flux<DIM, (DIM > 2 ? 2 : 0), SCHEME, double, false, true, ExtPolicy, W>(
          U, nbr26, slot, item, t, bm, F + 2 * dstride, stride, pol);
  }
}

// ---------------------------------------------------------------------------
// pencil sweeps (engine fast path)
// ---------------------------------------------------------------------------

// Interior linear index of the cell with index c along DIR at transverse (p1, p2).
template <int DIM, int DIR>
__device__ __forceinline__ int interior_index(int c, int p1, int p2) {
  using M = FaceMap<DIM, DIR>;
  int ci[3] = {0, 0, 0};
  ci[DIR] = c;
  ci[M::O1] = p1;
  ci[M::O2] = p2;
  if constexpr (DIM == 3) return (ci[0] * IC + ci[1]) * IC + ci[2];
  else if constexpr (DIM == 2) return ci[0] * IC + ci[1];
  else return ci[0];
}

// One thread walks a line of 16 cells along DIR: it computes the 17 face
// fluxes in order with a sliding 6-cell stencil window (each cell is loaded
// once per line instead of six times) and forms each cell's flux difference
// F(a-1/2) - F(a+1/2) as soon as both faces are known. The directions run one
// after the other: MODE 0 stores the difference in R, MODE 1 adds to R, MODE 2
// (the last direction) adds, scales by 1/cell size and applies the SSP-RK3
// stage: Uout = (stage ? a0 Uin + a1 U0 : Uin) + c dt rhs. The summation order
// is therefore (dx + dy) + dz instead of the reference's three-order symmetric
// sum (the strict build keeps that one). Stencils are gathered from neighbour
// interiors; cases with dt == 0 are skipped.
template <int DIM, int DIR, int SCHEME, typename T, int MODE>
__global__ void __launch_bounds__(128, FaceOccupancy<SCHEME>::min_ctas)
pencil_kernel(double const *Uin, double const *U0, double *Uout, double *R,
              int const *__restrict__ work, int nwork, BlockMeta const *__restrict__ meta,
              int const *__restrict__ nbr26, CaseState const *__restrict__ cases, int stage) {
  using G = Geo<DIM>;
  using M = FaceMap<DIM, DIR>;
  constexpr int NE = G::NE;
  constexpr int P = M::E1 * M::E2;  // lines per block
  constexpr int step = DIR == 0 ? G::TCY * G::TCZ : (DIR == 1 ? G::TCZ : 1);
  constexpr int lo_slot = DIR == 0 ? 4 : (DIR == 1 ? 10 : 12);
  constexpr int hi_slot = DIR == 0 ? 21 : (DIR == 1 ? 15 : 13);
  int const g = blockIdx.x * blockDim.x + threadIdx.x;
  int const item = g / P;
  if (item >= nwork) return;
  int const p = g - item * P;
  int const p1 = p / M::E2, p2 = p - (p / M::E2) * M::E2;
  int const slot = work[item];
  BlockMeta const bm = meta[slot];
  double const dt = cases[bm.case_id].dt;
  if (!(dt > 0.0)) return;
  Eos const eos{bm.gamma, bm.B, bm.safe};
  double const *blk = Uin + (size_t)slot * G::BLOCK_DOUBLES;
  int const cell0 = line_origin<DIM, DIR>(p1, p2);
  int const nlo = __ldg(nbr26 + (size_t)slot * 26 + lo_slot);
  int const nhi = __ldg(nbr26 + (size_t)slot * 26 + hi_slot);
  double *Rb = R ? R + (size_t)slot * NE * G::INTERIOR : nullptr;

  double w[6][NE];
#pragma unroll
  for (int m = 0; m < 6; ++m)
    stencil_load<DIM, DIR, true>(Uin, blk, HS - 3 + m, cell0, nlo, nhi, w[m]);
  double const ocs = inv(bm.cell_size);
  RkStage const rk = rk_stage(stage, dt);
  double fprev[NE];
#pragma unroll 1
  for (int a = 0; a <= IC; ++a) {
    double f[NE];
    bool const valid = face_compute<DIM, DIR, SCHEME, T>(eos, bm.B, w, f);
#pragma unroll
    for (int n = 0; n < NE; ++n)
      if (!valid) f[n] = 0.0;
    if (a > 0) {
      int const ix = interior_index<DIM, DIR>(a - 1, p1, p2);
      size_t const x = (size_t)slot * G::BLOCK_DOUBLES + cell0 + (HS + a - 1) * step;
#pragma unroll
      for (int n = 0; n < NE; ++n) {
        double const d = fprev[n] - f[n];
        if constexpr (MODE == 0) {
          Rb[n * G::INTERIOR + ix] = d;
        } else if constexpr (MODE == 1) {
          Rb[n * G::INTERIOR + ix] += d;
        } else {
          double const sum = DIM > 1 ? Rb[n * G::INTERIOR + ix] + d : d;
          double const rhs = 0.0 + sum * ocs;
          size_t const xf = x + (size_t)n * G::CELLS;
          Uout[xf] = rk_apply(rk, Uin[xf], rk.first ? 0.0 : U0[xf], rhs);
        }
      }
    }
#pragma unroll
    for (int n = 0; n < NE; ++n) fprev[n] = f[n];
    if (a < IC) {
#pragma unroll
      for (int m = 0; m < 5; ++m)
#pragma unroll
        for (int n = 0; n < NE; ++n) w[m][n] = w[m + 1][n];
      stencil_load<DIM, DIR, true>(Uin, blk, HS + a + 3, cell0, nlo, nhi, w[5]);
    }
  }
}

// ---------------------------------------------------------------------------
// divergence, stage update
// ---------------------------------------------------------------------------

template <int DIM>
__global__ void __launch_bounds__(256)
divergence_kernel(int const *__restrict__ work, BlockMeta const *__restrict__ meta, BlockMeta def,
                  double const *__restrict__ F, long long stride, long long dstride,
                  double *__restrict__ rhs) {
  using G = Geo<DIM>;
  int const item = blockIdx.x;
  int const slot = slot_of(work, item);
  double *rb = rhs + (size_t)slot * G::BLOCK_DOUBLES;
  // zero every cell (space_solver.cpp:58-70), then write the interior
  for (int x = threadIdx.x; x < G::BLOCK_DOUBLES; x += blockDim.x) rb[x] = 0.0;
  __syncthreads();
  BlockMeta const bm = meta ? meta[slot] : def;
  double const ocs = inv(bm.cell_size);
  double const *Fb = F + (long long)item * stride;
  for (int t = threadIdx.x; t < G::INTERIOR; t += blockDim.x) {
    int i, j, k;
    interior_coords<DIM>(t, i, j, k);
    int const c = G::cell(i + G::fic(0), j + G::fic(1), k + G::fic(2));
#pragma unroll
    for (int f = 0; f < G::NE; ++f) {
      double const *fx = Fb + f * G::FACES;
      rb[f * G::CELLS + c] =
          0.0 + divergence<DIM>(fx, fx + dstride, fx + 2 * dstride, i, j, k, ocs);
    }
  }
}


// Uin: stage input, U0: state at the start of the step, Uout: stage output.
// Uout may alias U0 (each cell is read and written by the same thread) but
// not Uin, whose cells other blocks' stencils read during the stage.
template <int DIM>
__global__ void __launch_bounds__(256)
stage_update_kernel(double const *Uin, double const *U0, double *Uout,
                    int const *__restrict__ work, BlockMeta const *__restrict__ meta, BlockMeta def,
                    double const *__restrict__ F, long long stride, long long dstride, int stage,
                    CaseState const *__restrict__ cases, double dt_all) {
  using G = Geo<DIM>;
  int const item = blockIdx.x;
  int const slot = slot_of(work, item);
  BlockMeta const bm = meta ? meta[slot] : def;
  double const dt = cases ? cases[bm.case_id].dt : dt_all;
  if (!(dt > 0.0)) return;
  int const t = blockIdx.y * blockDim.x + threadIdx.x;
  if (t >= G::INTERIOR) return;
  stage_update_cell<DIM>(Uin, U0, Uout, F + (long long)item * stride, dstride, slot, t,
                         inv(bm.cell_size), rk_stage(stage, dt));
}

// Stage update from a reference-layout right-hand-side buffer.
template <int DIM>
__global__ void __launch_bounds__(256)
rk_stage_rhs_kernel(double *__restrict__ U, double *__restrict__ U0,
                    double const *__restrict__ rhs, int stage, double dt) {
  using G = Geo<DIM>;
  int const slot = blockIdx.x;
  int const t = blockIdx.y * blockDim.x + threadIdx.x;
  if (t >= G::INTERIOR) return;
  int i, j, k;
  interior_coords<DIM>(t, i, j, k);
  int const c = G::cell(i + G::fic(0), j + G::fic(1), k + G::fic(2));
  RkStage const rk = rk_stage(stage, dt);
#pragma unroll
  for (int f = 0; f < G::NE; ++f) {
    size_t const x = (size_t)slot * G::BLOCK_DOUBLES + (size_t)f * G::CELLS + c;
    double const u = U[x];
    if (stage == 0) U0[x] = u;
    U[x] = rk_apply(rk, u, rk.first ? 0.0 : U0[x], rhs[x]);
  }
}

// ---------------------------------------------------------------------------
// halos
// ---------------------------------------------------------------------------

// Same-level halo regions (communication_types.h:45-132): for direction offset
// o = +1 the halo [HS+IC, TC) takes the neighbour's [HS, 2HS); o = -1 the halo
// [0, HS) takes the neighbour's [IC, IC+HS); o = 0 spans the interior.
template <int DIM>
__global__ void __launch_bounds__(256)
halo_region_kernel(double *__restrict__ U, int const *__restrict__ work,
                   int const *__restrict__ nbr26, BlockMeta const *__restrict__ meta,
                   CaseState const *__restrict__ cases, int faces_only, int nfields) {
  using G = Geo<DIM>;
  int const item = blockIdx.x;
  int const slot = slot_of(work, item);
  if (cases && meta && !(cases[meta[slot].case_id].dt > 0.0)) return;
  // blockIdx.y enumerates the 26 (or 2*DIM) regions
  int o;
  if (faces_only) {
    int const face = blockIdx.y;  // W,E,S,N,B,T
    int off[3] = {0, 0, 0};
    off[face / 2] = (face & 1) ? 1 : -1;
    o = (off[0] + 1) * 9 + (off[1] + 1) * 3 + (off[2] + 1);
  } else {
    o = blockIdx.y < 13 ? blockIdx.y : blockIdx.y + 1;
  }
  int const off[3] = {o / 9 - 1, (o / 3) % 3 - 1, o % 3 - 1};
  for (int d = DIM; d < 3; ++d)
    if (off[d] != 0) return;
  int const n = nbr26[(size_t)slot * 26 + (o < 13 ? o : o - 1)];
  if (n < 0) return;  // domain face: zero gradient below
  int lo[3], ext[3], src[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d >= DIM) {
      lo[d] = 0; ext[d] = 1; src[d] = 0;
    } else if (off[d] == 0) {
      lo[d] = HS; ext[d] = IC; src[d] = HS;
    } else if (off[d] > 0) {
      lo[d] = HS + IC; ext[d] = HS; src[d] = HS;
    } else {
      lo[d] = 0; ext[d] = HS; src[d] = IC;
    }
  }
  int const cells = ext[0] * ext[1] * ext[2];
  double *dst = U + (size_t)slot * nfields * G::CELLS;
  double const *sb = U + (size_t)n * nfields * G::CELLS;
  for (int x = threadIdx.x; x < cells * nfields; x += blockDim.x) {
    int const f = x / cells;
    int const r = x - f * cells;
    int const kk = r % ext[2];
    int const jj = (r / ext[2]) % ext[1];
    int const ii = r / (ext[2] * ext[1]);
    dst[f * G::CELLS + G::cell(lo[0] + ii, lo[1] + jj, lo[2] + kk)] =
        sb[f * G::CELLS + G::cell(src[0] + ii, src[1] + jj, src[2] + kk)];
  }
}

// Zero-gradient halos of domain faces (boundary_constants.h:103-160, 211-252):
// the halo takes the value of the first / last interior plane. With
// faces_only the copy covers the interior extent of the face, otherwise the
// reference's full TC x TC slab. The faces of one block are applied one after
// the other in x, y, z order (CommunicationManager::NeighborsOfNode lists
// domain sides East, West, North, South, Top, Bottom), which fixes the values
// the overlapping slabs leave in edge and corner halos.
template <int DIM>
__global__ void __launch_bounds__(256)
zero_gradient_kernel(double *__restrict__ U, int const *__restrict__ work,
                     int const *__restrict__ nbr26, BlockMeta const *__restrict__ meta,
                     CaseState const *__restrict__ cases, int faces_only, int nfields) {
  using G = Geo<DIM>;
  int const item = blockIdx.x;
  int const slot = slot_of(work, item);
  if (cases && meta && !(cases[meta[slot].case_id].dt > 0.0)) return;
  double *b = U + (size_t)slot * nfields * G::CELLS;
  for (int face = 0; face < 2 * DIM; ++face) {
    int const dir = face / 2, high = face & 1;
    int off[3] = {0, 0, 0};
    off[dir] = high ? 1 : -1;
    int const o = (off[0] + 1) * 9 + (off[1] + 1) * 3 + (off[2] + 1);
    int const nface = nbr26[(size_t)slot * 26 + (o < 13 ? o : o - 1)];
    if (nface >= 0) continue;
    bool const sym = nface == -2;  // symmetry wall: mirror, normal momentum negated
    int lo[3], ext[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      lo[d] = faces_only ? G::fic(d) : 0;
      ext[d] = faces_only ? G::ic(d) : G::tc(d);
    }
    lo[dir] = high ? HS + IC : 0;
    ext[dir] = HS;
    int const plane = high ? HS + IC - 1 : HS;
    int const mirror = high ? 2 * (HS + IC) - 1 : 2 * HS - 1;
    int const cells = ext[0] * ext[1] * ext[2];
    for (int x = threadIdx.x; x < cells * nfields; x += blockDim.x) {
      int const f = x / cells;
      int const r = x - f * cells;
      int c[3];
      c[2] = lo[2] + r % ext[2];
      c[1] = lo[1] + (r / ext[2]) % ext[1];
      c[0] = lo[0] + r / (ext[2] * ext[1]);
      int s[3] = {c[0], c[1], c[2]};
      s[dir] = sym ? mirror - c[dir] : plane;
      double const v = b[f * G::CELLS + G::cell(s[0], s[1], s[2])];
      // the momentum (or, for prime states, the velocity) normal to the wall is field 2 + dir
      b[f * G::CELLS + G::cell(c[0], c[1], c[2])] = (sym && f == 2 + dir) ? -1.0 * v : v;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// prime states, signal speed, dt
// ---------------------------------------------------------------------------

template <int DIM>
__global__ void __launch_bounds__(256)
prime_states_kernel(double const *__restrict__ U, int const *__restrict__ work,
                    BlockMeta const *__restrict__ meta, BlockMeta def, double *__restrict__ P) {
  using G = Geo<DIM>;
  int const item = blockIdx.x;
  int const slot = slot_of(work, item);
  BlockMeta const bm = meta ? meta[slot] : def;
  Eos const eos{bm.gamma, bm.B, bm.safe};
  double const *ub = U + (size_t)slot * G::BLOCK_DOUBLES;
  double *pb = P + (size_t)slot * G::BLOCK_DOUBLES;
  for (int x = blockIdx.y * blockDim.x + threadIdx.x; x < G::CELLS; x += gridDim.y * blockDim.x) {
    double c[G::NE];
#pragma unroll
    for (int f = 0; f < G::NE; ++f) c[f] = ub[f * G::CELLS + x];
    double const one_density = inv(c[MASS]);
    pb[RHO * G::CELLS + x] = c[MASS];
#pragma unroll
    for (int d = 0; d < DIM; ++d) pb[(VELX + d) * G::CELLS + x] = c[MOMX + d] * one_density;
    pb[PRES * G::CELLS + x] = eos_pressure<DIM>(eos, c[MASS], c[MOMX],
                                                DIM > 1 ? c[MOMX + (DIM > 1)] : 0.0,
                                                DIM > 2 ? c[MOMX + 2 * (DIM > 2)] : 0.0, c[ENERGY],
                                                one_density);
  }
}

// Signal speed of ComputeTimestepSize (modular_algorithm_assembler.cpp:1840-1870):
// max over interior cells of ConsistencyManagedSum(|u_d| + c).
template <int DIM>
__global__ void __launch_bounds__(256)
signal_speed_kernel(double const *__restrict__ U, int const *__restrict__ work,
                    BlockMeta const *__restrict__ meta, BlockMeta def, CaseState *cases,
                    unsigned long long *out) {
  using G = Geo<DIM>;
  int const item = blockIdx.x;
  int const slot = slot_of(work, item);
  BlockMeta const bm = meta ? meta[slot] : def;
  Eos const eos{bm.gamma, bm.B, bm.safe};
  double const *ub = U + (size_t)slot * G::BLOCK_DOUBLES;
  double smax = 0.0;
  int bad = 0;
  for (int t = threadIdx.x; t < G::INTERIOR; t += blockDim.x) {
    int i, j, k;
    interior_coords<DIM>(t, i, j, k);
    int const x = G::cell(i + G::fic(0), j + G::fic(1), k + G::fic(2));
    double c[G::NE];
#pragma unroll
    for (int f = 0; f < G::NE; ++f) c[f] = ub[f * G::CELLS + x];
    double const s = cell_signal_speed<DIM>(eos, c, bad);
    smax = dmax(smax, s);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0 && cases) atomicOr(&cases[bm.case_id].status, 1);
  // warp then CTA max (non-negative doubles order like their bit patterns)
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) smax = dmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = smax;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = dmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) {
      unsigned long long *dst = cases ? &cases[bm.case_id].smax_bits : out;
      atomicMax(dst, (unsigned long long)__double_as_longlong(v));
    }
  }
}

// dt = CFL / (smax / dx_finest), clipped to the end time
// (modular_algorithm_assembler.cpp:1932, 1961-1982); 0 once t >= t_end or the
// step budget is spent, which makes every kernel skip the case.
// dt of every case from its smax (case_dt_finalize); dtflag, when given,
// marks each case's dt as ready for a tile-stage launch (its step 0).
__global__ void dt_finalize_kernel(CaseState *cases, int n, int *dtflag) {
  int const c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  case_dt_finalize(cases[c]);
  if (dtflag) dtflag[c] = 1;
}

__global__ void step_commit_kernel(CaseState *cases, int n) {
  int const c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  case_commit(cases[c]);
}

}  // namespace

// Initial conditions evaluated on the device for a regular block grid whose
// blocks occupy consecutive slots from `first` in C order (x slowest). Cell
// centres are ((block index * 16 + i + 0.5) * cell_size, ...). Prime states
// are converted with PrimeStatesToConservatives (prime_state_handler.h:195-275).
// Every cell of the block (halos too) is written; halos are refreshed before
// they are read.
template <int DIM>
__global__ void __launch_bounds__(256)
initial_condition_kernel(double *__restrict__ U, int first, int nbx, int nby, int nbz,
                         double cell_size, double gamma, double B, int type,
                         IcParams params) {
  using G = Geo<DIM>;
  int const b = blockIdx.x;
  int const bx = b / (nby * nbz), by = (b / nbz) % nby, bz = b % nbz;
  double *ub = U + (size_t)(first + b) * G::BLOCK_DOUBLES;
  Eos const eos{gamma, B, 0};
  for (int x = threadIdx.x; x < G::CELLS; x += blockDim.x) {
    int const k = x % G::TCZ, j = (x / G::TCZ) % G::TCY, i = x / (G::TCZ * G::TCY);
    double pos[3] = {0.0, 0.0, 0.0};
    pos[0] = (bx * IC + i - HS + 0.5) * cell_size;
    if (DIM > 1) pos[1] = (by * IC + j - HS + 0.5) * cell_size;
    if (DIM > 2) pos[2] = (bz * IC + k - HS + 0.5) * cell_size;
    double const *q = params.v;
    double rho, p, vel[3] = {0.0, 0.0, 0.0};
    if (type == IC_QUADRANTS) {
      // q: x0, y0, then (rho, u, v, p) for quadrants (x<x0,y<y0), (x>=x0,y<y0),
      // (x<x0,y>=y0), (x>=x0,y>=y0)
      int const quad = (pos[0] >= q[0] ? 1 : 0) + (pos[1] >= q[1] ? 2 : 0);
      double const *s = q + 2 + 4 * quad;
      rho = s[0];
      vel[0] = s[1];
      vel[1] = s[2];
      p = s[3];
    } else {
      // IC_BLAST: q: centre (3), radius, (rho, p) inside, (rho, p) outside
      double r2 = 0.0;
      for (int d = 0; d < DIM; ++d) r2 += (pos[d] - q[d]) * (pos[d] - q[d]);
      bool const in = r2 < q[3] * q[3];
      rho = in ? q[4] : q[6];
      p = in ? q[5] : q[7];
    }
    double c[G::NE];
    c[MASS] = rho;
#pragma unroll
    for (int d = 0; d < DIM; ++d) c[MOMX + d] = vel[d] * rho;
    c[ENERGY] = eos_energy<DIM, double>(eos, rho, vel[0], vel[1], vel[2], p);
#pragma unroll
    for (int f = 0; f < G::NE; ++f) ub[f * G::CELLS + x] = c[f];
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

namespace {

template <int DIM, int DIR, bool ACC, int W>
cudaError_t face_flux_ext_dir(Launch const &L, dim3 grid, double *F, long long stride,
                              int threads) {
  ExtPolicy const pol{L.opt};
  switch (L.scheme) {
    case FV_CHAR:
      face_flux_ext_kernel<DIM, DIR, FV_CHAR, ACC, W>
          <<<grid, threads, 0, L.stream>>>(L.U, L.work, L.meta, L.def, F, stride, pol, L.glf);
      break;
    case FV_PRIM:
      face_flux_ext_kernel<DIM, DIR, FV_PRIM, ACC, W>
          <<<grid, threads, 0, L.stream>>>(L.U, L.work, L.meta, L.def, F, stride, pol, L.glf);
      break;
    case FS_ROE:
      face_flux_ext_kernel<DIM, DIR, FS_ROE, ACC, W>
          <<<grid, threads, 0, L.stream>>>(L.U, L.work, L.meta, L.def, F, stride, pol, L.glf);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int DIM, int DIR, typename T, bool ACC>
cudaError_t face_flux_dir(Launch const &L, double *F, long long stride, int threads) {
  using M = FaceMap<DIM, DIR>;
  dim3 grid(L.nwork, (M::COUNT + threads - 1) / threads);
  if (!L.opt.is_default())
    return ext_wide(L.opt) ? face_flux_ext_dir<DIM, DIR, ACC, 8>(L, grid, F, stride, threads)
                           : face_flux_ext_dir<DIM, DIR, ACC, 6>(L, grid, F, stride, threads);
  switch (L.scheme) {
    case FV_CHAR:
      face_flux_kernel<DIM, DIR, FV_CHAR, T, ACC>
          <<<grid, threads, 0, L.stream>>>(L.U, L.work, L.meta, L.def, F, stride);
      break;
    case FV_PRIM:
      face_flux_kernel<DIM, DIR, FV_PRIM, T, ACC>
          <<<grid, threads, 0, L.stream>>>(L.U, L.work, L.meta, L.def, F, stride);
      break;
    case FS_ROE:
      face_flux_kernel<DIM, DIR, FS_ROE, T, ACC>
          <<<grid, threads, 0, L.stream>>>(L.U, L.work, L.meta, L.def, F, stride);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int DIM, typename T, bool ACC>
cudaError_t face_flux_dim(Launch const &L, int dir, double *F, long long stride, int threads) {
  if (dir == 0) return face_flux_dir<DIM, 0, T, ACC>(L, F, stride, threads);
  if constexpr (DIM > 1)
    if (dir == 1) return face_flux_dir<DIM, 1, T, ACC>(L, F, stride, threads);
  if constexpr (DIM > 2)
    if (dir == 2) return face_flux_dir<DIM, 2, T, ACC>(L, F, stride, threads);
  return cudaErrorInvalidValue;
}

template <typename T, bool ACC>
cudaError_t face_flux_t(Launch const &L, int dir, double *F, long long stride, int threads) {
  switch (L.dim) {
    case 1: return face_flux_dim<1, T, ACC>(L, dir, F, stride, threads);
    case 2: return face_flux_dim<2, T, ACC>(L, dir, F, stride, threads);
    case 3: return face_flux_dim<3, T, ACC>(L, dir, F, stride, threads);
  }
  return cudaErrorInvalidValue;
}

int interior_of(int dim) { return dim == 3 ? 4096 : (dim == 2 ? 256 : 16); }

}  // namespace

cudaError_t launch_face_flux(Launch const &L, int dir, double *F, long long stride, bool accumulate,
                             int block_threads) {
  if (L.nwork <= 0) return cudaSuccess;
  int const threads = block_threads > 0 ? block_threads : 128;
  if (threads > 128 || (threads & 31)) return cudaErrorInvalidValue;
  if (!L.opt.is_default() && L.precision != FP64) return cudaErrorInvalidValue;
  if (L.precision == FP32_FLUX)
    return accumulate ? face_flux_t<float, true>(L, dir, F, stride, threads)
                      : face_flux_t<float, false>(L, dir, F, stride, threads);
  return accumulate ? face_flux_t<double, true>(L, dir, F, stride, threads)
                    : face_flux_t<double, false>(L, dir, F, stride, threads);
}

cudaError_t launch_divergence(Launch const &L, double const *F, long long stride,
                              long long dstride, double *rhs) {
  if (L.nwork <= 0) return cudaSuccess;
  dim3 grid(L.nwork);
  switch (L.dim) {
    case 1: divergence_kernel<1><<<grid, 256, 0, L.stream>>>(L.work, L.meta, L.def, F, stride, dstride, rhs); break;
    case 2: divergence_kernel<2><<<grid, 256, 0, L.stream>>>(L.work, L.meta, L.def, F, stride, dstride, rhs); break;
    case 3: divergence_kernel<3><<<grid, 256, 0, L.stream>>>(L.work, L.meta, L.def, F, stride, dstride, rhs); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_stage_update(Launch const &L, double const *U0, double *Uout, double const *F,
                                long long stride, long long dstride, int stage,
                                CaseState const *cases, double dt) {
  if (L.nwork <= 0) return cudaSuccess;
  if (stage < 0 || stage > 4) return cudaErrorInvalidValue;
  int const threads = 256;
  dim3 grid(L.nwork, (interior_of(L.dim) + threads - 1) / threads);
  switch (L.dim) {
    case 1: stage_update_kernel<1><<<grid, threads, 0, L.stream>>>(L.U, U0, Uout, L.work, L.meta, L.def, F, stride, dstride, stage, cases, dt); break;
    case 2: stage_update_kernel<2><<<grid, threads, 0, L.stream>>>(L.U, U0, Uout, L.work, L.meta, L.def, F, stride, dstride, stage, cases, dt); break;
    case 3: stage_update_kernel<3><<<grid, threads, 0, L.stream>>>(L.U, U0, Uout, L.work, L.meta, L.def, F, stride, dstride, stage, cases, dt); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

namespace {
template <int DIM, int W>
cudaError_t face_flux_all_ext(Launch const &L, dim3 grid, int const *nbr26, CaseState const *cases,
                              double *F, long long stride, long long dstride, int threads) {
  ExtPolicy const pol{L.opt};
  switch (L.scheme) {
    case FV_CHAR:
      face_flux_all_ext_kernel<DIM, FV_CHAR, W><<<grid, threads, 0, L.stream>>>(L.U, L.work, L.meta, nbr26, cases, F, stride, dstride, pol, L.glf, L.items);
      break;
    case FV_PRIM:
      face_flux_all_ext_kernel<DIM, FV_PRIM, W><<<grid, threads, 0, L.stream>>>(L.U, L.work, L.meta, nbr26, cases, F, stride, dstride, pol, L.glf, L.items);
      break;
    case FS_ROE:
      face_flux_all_ext_kernel<DIM, FS_ROE, W><<<grid, threads, 0, L.stream>>>(L.U, L.work, L.meta, nbr26, cases, F, stride, dstride, pol, L.glf, L.items);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int DIM, typename T>
cudaError_t face_flux_all_t(Launch const &L, int const *nbr26, CaseState const *cases, double *F,
                            long long stride, long long dstride, int threads) {
  int const count = (IC + 1) * (DIM > 1 ? IC : 1) * (DIM > 2 ? IC : 1);
  dim3 grid(L.nwork, (count + threads - 1) / threads, DIM);
  if (!L.opt.is_default())
    return ext_wide(L.opt)
               ? face_flux_all_ext<DIM, 8>(L, grid, nbr26, cases, F, stride, dstride, threads)
               : face_flux_all_ext<DIM, 6>(L, grid, nbr26, cases, F, stride, dstride, threads);
  // items x chunks < 2^31 for up to 2^31 / 68 items (64-thread chunks)
  int const chunks = (count + threads - 1) / threads;
  if ((long long)L.nwork * chunks > 0x7fffffffLL) return cudaErrorInvalidValue;
  dim3 const g2((unsigned)(L.nwork * chunks), 1, DIM);
  switch (L.scheme) {
    case FV_CHAR:
      face_flux_all_kernel<DIM, FV_CHAR, T><<<g2, threads, 0, L.stream>>>(L.U, L.work, L.meta, nbr26, cases, F, stride, dstride, chunks, L.items);
      break;
    case FV_PRIM:
      face_flux_all_kernel<DIM, FV_PRIM, T><<<g2, threads, 0, L.stream>>>(L.U, L.work, L.meta, nbr26, cases, F, stride, dstride, chunks, L.items);
      break;
    case FS_ROE:
      face_flux_all_kernel<DIM, FS_ROE, T><<<g2, threads, 0, L.stream>>>(L.U, L.work, L.meta, nbr26, cases, F, stride, dstride, chunks, L.items);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}
}  // namespace

namespace {
template <int DIM, int DIR, typename T, int MODE>
cudaError_t pencil_t(Launch const &L, double const *U0, double *Uout, double *R, int const *nbr26,
                     CaseState const *cases, int stage) {
  constexpr int P = FaceMap<DIM, DIR>::E1 * FaceMap<DIM, DIR>::E2;
  long long const threads = (long long)L.nwork * P;
  dim3 grid((unsigned)((threads + 127) / 128));
  switch (L.scheme) {
    case FV_CHAR:
      pencil_kernel<DIM, DIR, FV_CHAR, T, MODE><<<grid, 128, 0, L.stream>>>(L.U, U0, Uout, R, L.work, L.nwork, L.meta, nbr26, cases, stage);
      break;
    case FV_PRIM:
      pencil_kernel<DIM, DIR, FV_PRIM, T, MODE><<<grid, 128, 0, L.stream>>>(L.U, U0, Uout, R, L.work, L.nwork, L.meta, nbr26, cases, stage);
      break;
    case FS_ROE:
      pencil_kernel<DIM, DIR, FS_ROE, T, MODE><<<grid, 128, 0, L.stream>>>(L.U, U0, Uout, R, L.work, L.nwork, L.meta, nbr26, cases, stage);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int DIM, typename T>
cudaError_t pencil_dim(Launch const &L, double const *U0, double *Uout, double *R, int const *nbr26,
                       CaseState const *cases, int stage) {
  if (cudaError_t e = pencil_t<DIM, 0, T, DIM == 1 ? 2 : 0>(L, U0, Uout, R, nbr26, cases, stage))
    return e;
  if constexpr (DIM > 1)
    if (cudaError_t e = pencil_t<DIM, (DIM > 1 ? 1 : 0), T, DIM == 2 ? 2 : 1>(L, U0, Uout, R, nbr26, cases, stage))
      return e;
  if constexpr (DIM > 2)
    if (cudaError_t e = pencil_t<DIM, (DIM > 2 ? 2 : 0), T, 2>(L, U0, Uout, R, nbr26, cases, stage))
      return e;
  return cudaSuccess;
}
}  // namespace

cudaError_t launch_pencil_stage(Launch const &L, double const *U0, double *Uout, double *R,
                                int const *nbr26, CaseState const *cases, int stage) {
  if (L.nwork <= 0) return cudaSuccess;
  if (!L.work || !L.meta || !nbr26 || !cases || stage < 0 || stage > 2) return cudaErrorInvalidValue;
  if (L.dim > 1 && !R) return cudaErrorInvalidValue;
  if (!L.opt.is_default()) return cudaErrorInvalidValue;  // pencils: default schemes only
  bool const f32 = L.precision == FP32_FLUX;
  switch (L.dim) {
    case 1: return f32 ? pencil_dim<1, float>(L, U0, Uout, R, nbr26, cases, stage)
                       : pencil_dim<1, double>(L, U0, Uout, R, nbr26, cases, stage);
    case 2: return f32 ? pencil_dim<2, float>(L, U0, Uout, R, nbr26, cases, stage)
                       : pencil_dim<2, double>(L, U0, Uout, R, nbr26, cases, stage);
    case 3: return f32 ? pencil_dim<3, float>(L, U0, Uout, R, nbr26, cases, stage)
                       : pencil_dim<3, double>(L, U0, Uout, R, nbr26, cases, stage);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_face_flux_all(Launch const &L, int const *nbr26, CaseState const *cases,
                                 double *F, long long stride, long long dstride, int threads) {
  if (L.nwork <= 0) return cudaSuccess;
  if (!L.work || !L.meta || !nbr26 || !cases) return cudaErrorInvalidValue;
  if (threads <= 0) threads = 128;
  if (threads > 128 || (threads & 31)) return cudaErrorInvalidValue;
  if (!L.opt.is_default() && L.precision != FP64) return cudaErrorInvalidValue;
  bool const f32 = L.precision == FP32_FLUX;
  switch (L.dim) {
    case 1: return f32 ? face_flux_all_t<1, float>(L, nbr26, cases, F, stride, dstride, threads)
                       : face_flux_all_t<1, double>(L, nbr26, cases, F, stride, dstride, threads);
    case 2: return f32 ? face_flux_all_t<2, float>(L, nbr26, cases, F, stride, dstride, threads)
                       : face_flux_all_t<2, double>(L, nbr26, cases, F, stride, dstride, threads);
    case 3: return f32 ? face_flux_all_t<3, float>(L, nbr26, cases, F, stride, dstride, threads)
                       : face_flux_all_t<3, double>(L, nbr26, cases, F, stride, dstride, threads);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_rk_stage_rhs(int dim, double *U, double *U0, double const *rhs, int nb,
                                int stage, double dt, cudaStream_t stream) {
  if (nb <= 0) return cudaSuccess;
  if (stage < 0 || stage > 2) return cudaErrorInvalidValue;
  dim3 grid(nb, (interior_of(dim) + 255) / 256);
  switch (dim) {
    case 1: rk_stage_rhs_kernel<1><<<grid, 256, 0, stream>>>(U, U0, rhs, stage, dt); break;
    case 2: rk_stage_rhs_kernel<2><<<grid, 256, 0, stream>>>(U, U0, rhs, stage, dt); break;
    case 3: rk_stage_rhs_kernel<3><<<grid, 256, 0, stream>>>(U, U0, rhs, stage, dt); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_halo(Launch const &L, int const *nbr26, bool faces_only, int nfields,
                        CaseState const *cases) {
  if (L.nwork <= 0) return cudaSuccess;
  int const regions = faces_only ? 2 * L.dim : 26;
  dim3 g1(L.nwork, regions), g2(L.nwork);
  int const fo = faces_only ? 1 : 0;
  switch (L.dim) {
    case 1:
      halo_region_kernel<1><<<g1, 256, 0, L.stream>>>(L.U, L.work, nbr26, L.meta, cases, fo, nfields);
      zero_gradient_kernel<1><<<g2, 256, 0, L.stream>>>(L.U, L.work, nbr26, L.meta, cases, fo, nfields);
      break;
    case 2:
      halo_region_kernel<2><<<g1, 256, 0, L.stream>>>(L.U, L.work, nbr26, L.meta, cases, fo, nfields);
      zero_gradient_kernel<2><<<g2, 256, 0, L.stream>>>(L.U, L.work, nbr26, L.meta, cases, fo, nfields);
      break;
    case 3:
      halo_region_kernel<3><<<g1, 256, 0, L.stream>>>(L.U, L.work, nbr26, L.meta, cases, fo, nfields);
      zero_gradient_kernel<3><<<g2, 256, 0, L.stream>>>(L.U, L.work, nbr26, L.meta, cases, fo, nfields);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_prime_states(Launch const &L, double *P) {
  if (L.nwork <= 0) return cudaSuccess;
  dim3 grid(L.nwork, 8);
  switch (L.dim) {
    case 1: prime_states_kernel<1><<<grid, 256, 0, L.stream>>>(L.U, L.work, L.meta, L.def, P); break;
    case 2: prime_states_kernel<2><<<grid, 256, 0, L.stream>>>(L.U, L.work, L.meta, L.def, P); break;
    case 3: prime_states_kernel<3><<<grid, 256, 0, L.stream>>>(L.U, L.work, L.meta, L.def, P); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_signal_speed(Launch const &L, CaseState *cases, unsigned long long *out) {
  if (L.nwork <= 0) return cudaSuccess;
  dim3 grid(L.nwork);
  switch (L.dim) {
    case 1: signal_speed_kernel<1><<<grid, 256, 0, L.stream>>>(L.U, L.work, L.meta, L.def, cases, out); break;
    case 2: signal_speed_kernel<2><<<grid, 256, 0, L.stream>>>(L.U, L.work, L.meta, L.def, cases, out); break;
    case 3: signal_speed_kernel<3><<<grid, 256, 0, L.stream>>>(L.U, L.work, L.meta, L.def, cases, out); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_initial_condition(int dim, double *U, int first, int const nblocks[3],
                                     double cell_size, double gamma, double B, int type,
                                     IcParams const &params, cudaStream_t stream) {
  int const nb = nblocks[0] * nblocks[1] * nblocks[2];
  if (nb <= 0) return cudaSuccess;
  if (type != IC_QUADRANTS && type != IC_BLAST) return cudaErrorInvalidValue;
  switch (dim) {
    case 1: initial_condition_kernel<1><<<nb, 256, 0, stream>>>(U, first, nblocks[0], nblocks[1], nblocks[2], cell_size, gamma, B, type, params); break;
    case 2: initial_condition_kernel<2><<<nb, 256, 0, stream>>>(U, first, nblocks[0], nblocks[1], nblocks[2], cell_size, gamma, B, type, params); break;
    case 3: initial_condition_kernel<3><<<nb, 256, 0, stream>>>(U, first, nblocks[0], nblocks[1], nblocks[2], cell_size, gamma, B, type, params); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_dt_finalize(CaseState *cases, int n, cudaStream_t stream, int *dtflag) {
  if (n <= 0) return cudaSuccess;
  dt_finalize_kernel<<<(n + 127) / 128, 128, 0, stream>>>(cases, n, dtflag);
  return cudaGetLastError();
}

cudaError_t launch_step_commit(CaseState *cases, int n, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  step_commit_kernel<<<(n + 127) / 128, 128, 0, stream>>>(cases, n);
  return cudaGetLastError();
}

namespace {
__device__ unsigned long long g_glf_stateless[4];

__device__ __forceinline__ double max_keep(double m, double v) { return (m < v) ? v : m; }

// One CTA per block: the block's maxima of |u - c|, |u|, |u + c| (x velocity,
// interior cells with positive density; std::max keeps the running maximum
// against a NaN as the reference's does), then one atomicMax per value on
// its case's slot (bit patterns of non-negative doubles order like the values).
template <int DIM>
__global__ void __launch_bounds__(256)
glf_maxima_kernel(double const *__restrict__ U, int const *__restrict__ work,
                  BlockMeta const *__restrict__ meta, BlockMeta def,
                  unsigned long long *__restrict__ glf) {
  using G = Geo<DIM>;
  int const item = blockIdx.x;
  int const slot = slot_of(work, item);
  BlockMeta const bm = meta ? meta[slot] : def;
  Eos const eos{bm.gamma, bm.B, bm.safe};
  double const *ub = U + (size_t)slot * G::BLOCK_DOUBLES;
  double m[3] = {0.0, 0.0, 0.0};
  for (int c = threadIdx.x; c < G::INTERIOR; c += blockDim.x) {
    int const k = c % G::ICZ, j = (c / G::ICZ) % G::ICY, i = c / (G::ICZ * G::ICY);
    int const x = ((i + HS) * G::TCY + (j + (DIM > 1 ? HS : 0))) * G::TCZ + (k + (DIM > 2 ? HS : 0));
    double cons[G::NE];
#pragma unroll
    for (int f = 0; f < G::NE; ++f) cons[f] = ub[f * G::CELLS + x];
    auto const pr = cell_prims<DIM, 0>(eos, cons);
    if (!(pr.rho > 0.0)) continue;
    double const cs = eos_speed_of_sound<double>(eos, pr.rho, pr.p, pr.one_rho);
    m[0] = max_keep(m[0], fabs(pr.up - cs));
    m[1] = max_keep(m[1], fabs(pr.up));
    m[2] = max_keep(m[2], fabs(pr.up + cs));
  }
  __shared__ double red[3][8];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double v = m[q];
    for (int o = 16; o > 0; o >>= 1) v = max_keep(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = max_keep(v, red[threadIdx.x][w]);
    atomicMax(&glf[4 * bm.case_id + threadIdx.x], (unsigned long long)__double_as_longlong(v));
  }
}
}  // namespace

cudaError_t launch_glf_maxima(Launch const &L, unsigned long long *glf, int ncases) {
  if (ncases <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(glf, 0, sizeof(unsigned long long) * 4 * ncases, L.stream);
  if (e != cudaSuccess || L.nwork <= 0) return e;
  switch (L.dim) {
    case 1: glf_maxima_kernel<1><<<L.nwork, 256, 0, L.stream>>>(L.U, L.work, L.meta, L.def, glf); break;
    case 2: glf_maxima_kernel<2><<<L.nwork, 256, 0, L.stream>>>(L.U, L.work, L.meta, L.def, glf); break;
    default: glf_maxima_kernel<3><<<L.nwork, 256, 0, L.stream>>>(L.U, L.work, L.meta, L.def, glf); break;
  }
  return cudaGetLastError();
}

// The address is looked up on every call (a symbol lookup in the loaded
// module): after cudaDeviceReset the module loads again, possibly at another
// address, so an address kept from an earlier call could be stale.
unsigned long long *glf_stateless_slot() {
  void *addr = nullptr;
  if (cudaGetSymbolAddress(&addr, g_glf_stateless) != cudaSuccess) return nullptr;
  return static_cast<unsigned long long *>(addr);
}

namespace {
// packed [b][field][ICX][ICY][ICZ] <-> the interiors of pool blocks first + b
// (one thread per cell; consecutive threads take consecutive z cells).
template <int DIM>
__global__ void interior_copy_kernel(double *U, int first, int nb, double *P, bool to_pool) {
  using G = Geo<DIM>;
  long long const n = (long long)nb * G::NE * G::INTERIOR;
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n;
       x += (long long)gridDim.x * blockDim.x) {
    int const c = int(x % G::INTERIOR);
    long long const bf = x / G::INTERIOR;  // b * NE + field
    int const k = c % G::ICZ, j = (c / G::ICZ) % G::ICY, i = c / (G::ICZ * G::ICY);
    long long const u = ((long long)first * G::NE + bf) * G::CELLS +
                        G::cell(i + G::fic(0), j + G::fic(1), k + G::fic(2));
    if (to_pool) U[u] = P[x];
    else P[x] = U[u];
  }
}
}  // namespace

cudaError_t launch_interior_copy(int dim, double *U, int first, int nb, double *packed,
                                 bool to_pool, cudaStream_t stream) {
  if (nb <= 0) return cudaSuccess;
  int const grid = 148 * 8, threads = 256;
  switch (dim) {
    case 1: interior_copy_kernel<1><<<grid, threads, 0, stream>>>(U, first, nb, packed, to_pool); break;
    case 2: interior_copy_kernel<2><<<grid, threads, 0, stream>>>(U, first, nb, packed, to_pool); break;
    default: interior_copy_kernel<3><<<grid, threads, 0, stream>>>(U, first, nb, packed, to_pool); break;
  }
  return cudaGetLastError();
}

}  // namespace alp
