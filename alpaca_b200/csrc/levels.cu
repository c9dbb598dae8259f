// Multi-level cases: the leaves of a block tree (levels of the reference's
// multiresolution hierarchy) advanced with its local time stepping, all levels
// batched into the engine's face-flux and stage-update launches.
//
// Time stepping (ModularAlgorithmAssembler::Advance,
// modular_algorithm_assembler.cpp:575-874): a macro step is 2^lmax micro steps;
// micro step t integrates the levels GetLevels(t) returns (:2564-2573), level l
// with the sum of its last 2^(lmax-l) micro time steps (Integrate :1068-1098,
// time_integrator.h:312-340); a level's stage-0 right-hand side is evaluated at
// the start of its interval, i.e. during micro step t for the levels of
// GetLevels(t-1) (all levels at t = 0), and kept in the face-flux scratch until
// the level integrates. The micro time step is ComputeTimestepSize over all
// leaves with the finest cell size, clipped to the end time with the micro
// steps already taken (:1925-1982).
//
// Leaves are ordered finest level first in the work list, so the levels of
// GetLevels(t) (always the finest `height` levels) are a prefix of it and every
// launch covers exactly the leaves that work.
//
// Jumps: the face kernels gather stencil cells from a neighbour block's
// interior. Where the face neighbour of a leaf is one level coarser or finer,
// the neighbour slot is a ghost block: a virtual node of the leaf's level whose
// cell layers next to the shared face that the stencils reach (three, four for
// WENO7) are filled before each stage. On
// the coarse side they average the finer leaves (Multiresolution::Average,
// multiresolution.h:94-166); on the fine side they are the fifth-order
// prediction from the coarser level (Multiresolution::Prediction,
// multiresolution.cpp:146-283), which is what the reference's jump halos hold
// (InternalHaloManager::UpdateMaterialJumpNoMpi, internal_halo_manager.cpp:
// 230-290, predicting from the parent's buffer: its interior the average of
// its children, its halos its neighbours' cells). The prediction reads two
// parent-level cells around each parent cell, so the parent position's
// neighbours that are not leaves become ghosts filled whole: averages of their
// children, or predictions from one level coarser still. Averaged ghosts are
// filled finest level first, predicted ones coarsest first. Face neighbours may
// differ by one level at most.
//
// Conservation at jumps as in the reference: after each stage update the
// leaves integrate their jump-face fluxes with the RK3 jump multipliers times
// their level step (space_solver.cpp:155-182, time_integrator.h:64-80); at the
// end of each fine step these sums are averaged onto the parent's face
// (Multiresolution::AverageJumpBuffer, multiresolution.cpp:47-128); at the end
// of a coarse step the cells next to a refined neighbour get
// - CMS(coarse sums) + CMS(fine sums) per unit cell size (JumpFluxAdjustment,
// modular_algorithm_assembler.cpp:1347-1636).
#include <cuda_runtime.h>
#include <nvtx3/nvtx3.hpp>

#include <algorithm>
#include <cfloat>
#include <map>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/alpaca_b200.h"
#include "engine.hpp"
#include "numerics.cuh"
#include "step_common.cuh"

namespace {

using alp::cms3;
using alp::Geo;
using alp::HS;
using alp::IC;
using alp::interior_coords;
using alp::inv;
using alp::rk_stage;
using alp::stage_update_cell;
using alp::wait_count;

constexpr int kMaxLevels = 7;            // lmax <= 6: 64 micro steps per macro step
constexpr int kMaxMicro = 1 << (kMaxLevels - 1);

struct LevelState {
  double t, t_end, cfl, h_fine;
  double hist[kMaxMicro];  // micro time steps of the macro step in flight
  int macro, max_macro, micro, active, status, pad;
};

// A ghost block: a node position of a leaf's level that is not a leaf, filled
// before every stage in which a block reading it computes. Type 1 (a refined
// node): the average of its children src[o] (child o has x in bit 0, y in bit
// 1, z in bit 2; Multiresolution::Average). Type 0 (inside a coarser leaf): the
// fifth-order prediction from the parent level (Multiresolution::Prediction),
// which reads the 3^dim nodes nb[] around the parent position q (nb index
// (dx+1)*9 + (dy+1)*3 + (dz+1); cells beyond the domain take the value of the
// nearest domain cell, zero gradient); oct is the ghost's octant in its parent.
// A ghost the face kernels read fills the `layers` cell layers next to each face
// in `faces` (bits W, E, S, N, B, T); a ghost other ghosts read (`full`: its
// sources are all resolved) also fills the box of cells those reads reach,
// lo[e] <= cell < hi[e]. Slots below nleaf are leaves, read from the pool of
// their level. gate: the finest level whose computing needs the ghost.
struct GhostRec {
  int slot, type, level, gate, faces, full, oct;
  int layers;        // cell layers next to a served face: the stencil's reach (3, WENO7 4)
  int lo[3], hi[3];  // the box other ghosts read (empty: lo >= hi)
  int q[3], ext[3];  // parent position (nodes) and level extent (cells) of the parent level
  int src[8];
  int nb[27];
};

__device__ __forceinline__ double ghost_average3(double a0, double a1, double a2, double a3,
                                                 double a4, double a5, double a6, double a7) {
  // children (x,y,z) = bits of the index; pairs of Multiresolution::Average
  double const a = a0 + a7;  // (0,0,0) + (1,1,1)
  double const b = a4 + a3;  // (0,0,1) + (1,1,0)
  double const c = a2 + a5;  // (0,1,0) + (1,0,1)
  double const d = a6 + a1;  // (0,1,1) + (1,0,0)
  double const s1 = (a + b) + (c + d);
  double const s2 = (a + c) + (b + d);
  double const s3 = (a + d) + (b + c);
  // min / max as std::min / std::max order them (first argument on ties)
  double const i1 = s3 < s2 ? s3 : s2, mn = i1 < s1 ? i1 : s1;
  double const i2 = s2 < s3 ? s3 : s2, mx = s1 < i2 ? i2 : s1;
  return 0.125 * (0.5 * (mn + mx));
}

// The pool a slot's cells are read from in this stage.
__device__ __forceinline__ double const *ghost_source(int slot, int nleaf, int leaf_level,
                                                      double const *Ug, double const *UA,
                                                      CaseState const *cu, int stage) {
  if (slot >= nleaf) return Ug;
  return (stage > 0 && cu[leaf_level].dt > 0.0) ? Ug : UA;
}

// The cells a part of the fill covers: part < 2 DIM, the three layers next to
// face part (if served); part == 2 DIM, the box other ghosts read (if any).
template <int DIM>
__device__ __forceinline__ bool ghost_part(GhostRec const &g, int part, int lo[3], int hi[3]) {
  if (part == 2 * DIM) {
    bool any = true;
    for (int e = 0; e < 3; ++e) {
      lo[e] = e < DIM ? g.lo[e] : 0;
      hi[e] = e < DIM ? g.hi[e] : 1;
      any = any && lo[e] < hi[e];
    }
    return any;
  }
  if (!((g.faces >> part) & 1)) return false;
  for (int e = 0; e < 3; ++e) {
    lo[e] = 0;
    hi[e] = e < DIM ? IC : 1;
  }
  int const d = part / 2;
  lo[d] = (part & 1) ? IC - g.layers : 0;
  hi[d] = lo[d] + g.layers;
  return true;
}

// Fields whose children one thread holds at once in the averages (two fit the
// ghost kernel's 64 registers; one was 1 % slower on the three-level step).
constexpr int kAverageFields = 2;

// Part `part` of a type 1 ghost, by one CTA: averages of the children.
template <int DIM>
__device__ __forceinline__ void ghost_average_unit(GhostRec const &g, int part, double *Ug,
                                                   double const *UA, int nleaf,
                                                   CaseState const *__restrict__ gate,
                                                   CaseState const *__restrict__ cu, int stage) {
  using G = Geo<DIM>;
  int lo[3], hi[3];
  if (!ghost_part<DIM>(g, part, lo, hi)) return;
  if (!(gate[g.gate].dt > 0.0)) return;  // no block reading this ghost computes now
  int const n1 = hi[1] - lo[1], n2 = hi[2] - lo[2];
  int const count = (hi[0] - lo[0]) * n1 * n2;
  double *dst = Ug + (size_t)g.slot * G::BLOCK_DOUBLES;
  for (int t = threadIdx.x; t < count; t += blockDim.x) {
    int const a[3] = {lo[0] + t / (n1 * n2), lo[1] + (t / n2) % n1, lo[2] + t % n2};
    int const x = G::cell(a[0] + G::fic(0), a[1] + G::fic(1), a[2] + G::fic(2));
    int o = 0, c[3] = {0, 0, 0};
    for (int e = 0; e < DIM; ++e) {
      o |= (a[e] / (IC / 2)) << e;
      c[e] = 2 * (a[e] % (IC / 2)) + G::fic(e);
    }
    int const child = g.src[o];
    if (child < 0) continue;  // never read: the host checks face children are leaves
    double const *sb =
        ghost_source(child, nleaf, g.level + 1, Ug, UA, cu, stage) + (size_t)child * G::BLOCK_DOUBLES;
    // kAverageFields fields' children are loaded before any of their averages
    // is stored: the stores may alias the sources, so the compiler would not
    // move later loads above them, and these loads in flight are what keeps
    // the averages near the memory rate
#pragma unroll
    for (int e0 = 0; e0 < G::NE; e0 += kAverageFields) {
      constexpr int K = 1 << DIM;
      double w[kAverageFields][K];
#pragma unroll
      for (int f = 0; f < kAverageFields; ++f)
        if (e0 + f < G::NE) {
          double const *s = sb + (e0 + f) * G::CELLS;
#pragma unroll
          for (int k = 0; k < K; ++k)
            w[f][k] = s[G::cell(c[0] + (k & 1), c[1] + (DIM > 1 ? (k >> 1) & 1 : 0),
                                c[2] + (DIM > 2 ? (k >> 2) & 1 : 0))];
        }
#pragma unroll
      for (int f = 0; f < kAverageFields; ++f)
        if (e0 + f < G::NE) {
          double v;
          if constexpr (DIM == 1) {
            v = (w[f][0] + w[f][1]) * 0.5;
          } else if constexpr (DIM == 2) {
            v = ((w[f][0] + w[f][3]) + (w[f][1] + w[f][2])) * 0.25;
          } else {
            v = ghost_average3(w[f][0], w[f][1], w[f][2], w[f][3], w[f][4], w[f][5], w[f][6],
                               w[f][7]);
          }
          dst[(e0 + f) * G::CELLS + x] = v;
        }
    }
  }
}

// Fifth-order prediction of the children of one parent cell
// (Multiresolution::Prediction, multiresolution.cpp:146-283): V(a, b, c) is the
// parent value at offsets (a, b, c) in -2..2 along x, y, z. The terms and their
// order are the reference's: one-axis differences, pairs of axes, and the
// consistency-managed triple term, combined per child with its signs.
constexpr double kPc0 = -22.0 / 128.0, kPc1 = 3.0 / 128.0;
constexpr double kPc00 = kPc0 * kPc0, kPc01 = kPc0 * kPc1, kPc11 = kPc1 * kPc1;
constexpr double kPc000 = kPc00 * kPc0, kPc001 = kPc00 * kPc1, kPc011 = kPc0 * kPc11,
                 kPc111 = kPc1 * kPc11;

__device__ __forceinline__ double cms4(double a, double b, double c, double d) {
  double const s1 = (a + b) + (c + d);
  double const s2 = (a + c) + (b + d);
  double const s3 = (a + d) + (b + c);
  double const i1 = s2 < s1 ? s2 : s1, mn = s3 < i1 ? s3 : i1;
  double const i2 = s1 < s2 ? s2 : s1, mx = i2 < s3 ? s3 : i2;
  return 0.5 * (mn + mx);
}

template <int DIM, typename V>
__device__ __forceinline__ void predict_children(V const &val, double (&out)[1 << DIM]) {
  auto at1 = [&](int d, int s) { return val(d == 0 ? s : 0, d == 1 ? s : 0, d == 2 ? s : 0); };
  auto at2 = [&](int d, int sd, int e, int se) {
    int o[3] = {0, 0, 0};
    o[d] = sd;
    o[e] = se;
    return val(o[0], o[1], o[2]);
  };
  auto q1 = [&](int d) {
    return kPc0 * (at1(d, 1) - at1(d, -1)) + kPc1 * (at1(d, 2) - at1(d, -2));
  };
  auto x2 = [&](int d, int e, int a, int b) {
    return (at2(d, a, e, b) + at2(d, -a, e, -b)) - (at2(d, -a, e, b) + at2(d, a, e, -b));
  };
  auto q2 = [&](int d, int e) {
    return (kPc00 * x2(d, e, 1, 1) + kPc11 * x2(d, e, 2, 2)) +
           (kPc01 * x2(d, e, 1, 2) + kPc01 * x2(d, e, 2, 1));
  };
  auto x3 = [&](int a, int b, int c) {
    return cms4(val(a, b, c) - val(-a, -b, -c), val(-a, -b, c) - val(a, b, -c),
                val(a, -b, -c) - val(-a, b, c), val(-a, b, -c) - val(a, -b, c));
  };
  double qx = 0.0, qy = 0.0, qz = 0.0, qxy = 0.0, qxz = 0.0, qyz = 0.0, qxyz = 0.0;
  qx = q1(0);
  if constexpr (DIM > 1) {
    qy = q1(1);
    qxy = q2(0, 1);
  }
  if constexpr (DIM > 2) {
    qz = q1(2);
    qxz = q2(0, 2);
    qyz = q2(1, 2);
    qxyz = cms4(kPc000 * x3(1, 1, 1) + kPc111 * x3(2, 2, 2),
                kPc001 * x3(1, 1, 2) + kPc011 * x3(2, 2, 1),
                kPc011 * x3(1, 2, 2) + kPc001 * x3(2, 1, 1),
                kPc001 * x3(1, 2, 1) + kPc011 * x3(2, 1, 2));
  }
  double const p = val(0, 0, 0);
#pragma unroll
  for (int o = 0; o < (1 << DIM); ++o) {
    double const sx = (o & 1) ? -1.0 : 1.0, sy = (o & 2) ? -1.0 : 1.0, sz = (o & 4) ? -1.0 : 1.0;
    double s1, s2;
    if constexpr (DIM == 1) {
      s1 = sx * qx;
      s2 = sx * sy * qxy;
    } else if constexpr (DIM == 2) {
      s1 = sx * qx + sy * qy;
      s2 = sx * sy * qxy + sx * sz * qxz;
    } else {
      s1 = cms3(sx * qx, sy * qy, sz * qz);
      s2 = cms3(sx * sy * qxy, sx * sz * qxz, sy * sz * qyz);
    }
    out[o] = ((p + s1) + s2) + sx * sy * sz * qxyz;
  }
}

// Part `part` of a type 0 ghost, by one CTA: predicted from the parent level.
// The parent cells under the part plus two on every side are staged in the
// shared memory `box`, kFieldsPerPass fields at a time; then one thread per
// (field, parent cell) writes the children. The CTA's threads take the same
// early returns.
constexpr int kBox = IC / 2 + 4;  // parent cells of a whole octant plus the stencil reach
// Two fields per pass keep the box at 28 KB in 3D, within the 56 KB a CTA
// has at the ghost kernel's 4 CTAs per SM (64 registers a thread). On the
// three-level step one field per pass was 1.3 % slower and three 1.4 %.
constexpr int kFieldsPerPass = 2;

template <int DIM>
__host__ __device__ constexpr int predict_box_doubles() {
  return kBox * (DIM > 1 ? kBox : 1) * (DIM > 2 ? kBox : 1);
}
template <int DIM>
constexpr size_t predict_smem_bytes() {
  return sizeof(double) * kFieldsPerPass * predict_box_doubles<DIM>();
}

template <int DIM>
__device__ __forceinline__ void ghost_predict_unit(GhostRec const &g, int part, double *Ug,
                                                   double const *UA, int nleaf,
                                                   CaseState const *__restrict__ gate,
                                                   CaseState const *__restrict__ cu, int stage,
                                                   double *box) {
  using G = Geo<DIM>;
  constexpr int B1 = DIM > 1 ? kBox : 1, B2 = DIM > 2 ? kBox : 1;
  constexpr int BOX = predict_box_doubles<DIM>();
  int lo[3], hi[3];
  if (!ghost_part<DIM>(g, part, lo, hi)) return;
  if (!(gate[g.gate].dt > 0.0)) return;
  // parent cells (relative to the parent node's origin) under the part
  int plo[3] = {0, 0, 0}, pn[3] = {1, 1, 1}, bn[3] = {1, 1, 1};
  for (int e = 0; e < DIM; ++e) {
    int const base = (IC / 2) * ((g.oct >> e) & 1);
    plo[e] = base + lo[e] / 2;
    pn[e] = (hi[e] + 1) / 2 - lo[e] / 2;
    bn[e] = pn[e] + 4;
  }
  int const nbox = bn[0] * bn[1] * bn[2], npar = pn[0] * pn[1] * pn[2];
  double *dst = Ug + (size_t)g.slot * G::BLOCK_DOUBLES;
  for (int e0 = 0; e0 < G::NE; e0 += kFieldsPerPass) {
    int const ne = G::NE - e0 < kFieldsPerPass ? G::NE - e0 : kFieldsPerPass;
    if (e0 > 0) __syncthreads();  // the previous pass has read the box
    for (int t = threadIdx.x; t < nbox; t += blockDim.x) {
      int const r[3] = {t / (bn[1] * bn[2]), (t / bn[2]) % bn[1], t % bn[2]};
      int y[3] = {0, 0, 0}, k = 0;
      for (int d = 0; d < 3; ++d) {
        int dn = 0;
        if (d < DIM) {
          int gc = g.q[d] * IC + plo[d] - 2 + r[d];  // parent-level cell
          gc = gc < 0 ? 0 : (gc >= g.ext[d] ? g.ext[d] - 1 : gc);
          dn = gc / IC - g.q[d];
          y[d] = gc - (g.q[d] + dn) * IC + G::fic(d);
        }
        k = 3 * k + dn + 1;
      }
      int const slot = g.nb[k];
      double const *sb = ghost_source(slot, nleaf, g.level - 1, Ug, UA, cu, stage) +
                         (size_t)slot * G::BLOCK_DOUBLES;
      int const c = G::cell(y[0], y[1], y[2]);
      int const b = (r[0] * B1 + r[1]) * B2 + r[2];
#pragma unroll
      for (int e = 0; e < kFieldsPerPass; ++e)
        if (e < ne) box[e * BOX + b] = sb[(e0 + e) * G::CELLS + c];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < npar * ne; t += blockDim.x) {
      int const e = t / npar, tp = t - e * npar;
      int const r[3] = {tp / (pn[1] * pn[2]) + 2, (tp / pn[2]) % pn[1] + (DIM > 1 ? 2 : 0),
                        tp % pn[2] + (DIM > 2 ? 2 : 0)};
      double const *bx = box + e * BOX;
      auto val = [&](int a, int b, int c) {
        return bx[((r[0] + a) * B1 + (DIM > 1 ? r[1] + b : 0)) * B2 + (DIM > 2 ? r[2] + c : 0)];
      };
      double out[1 << DIM];
      predict_children<DIM>(val, out);
#pragma unroll
      for (int o = 0; o < (1 << DIM); ++o) {
        int a[3] = {0, 0, 0};
        for (int d = 0; d < DIM; ++d)
          a[d] = 2 * (plo[d] + r[d] - 2 - (IC / 2) * ((g.oct >> d) & 1)) + ((o >> d) & 1);
        dst[(e0 + e) * G::CELLS + G::cell(a[0] + G::fic(0), a[1] + G::fic(1), a[2] + G::fic(2))] =
            out[o];
      }
    }
  }
}

// The ghost groups of a stage in launch order (averages finest level first,
// then predictions coarsest first): a group's records read only records of
// earlier groups.
constexpr int kMaxGhostGroups = 16;
struct GhostPlan {
  int n;
  int type[kMaxGhostGroups], first[kMaxGhostGroups];
  int start[kMaxGhostGroups + 1];  // the groups' first (record, part) units, then the total
};

// The ghost groups of one stage in one launch. The CTAs pull the (record,
// part) units of all groups in order from one counter, so that cheap units
// (parts a record does not serve, ghosts whose readers are idle) and
// expensive ones (prediction boxes) even out. A unit that fills cells first
// waits until every ghost record it reads (children of an average, the
// parent's neighbourhood of a prediction; rank: ghost slot - nleaf -> record)
// has all its parts done. Those records belong to earlier groups (checked on
// the host), so they were handed out earlier and are held by running CTAs:
// every wait ends. Each is bounded all the same (wait_count) and sets *err on
// running out. A record whose reader does not compute reads nothing new and
// waits for nothing; a record whose reader computes reads only records whose
// readers compute as well (the host gives a ghost the finest gate of its
// readers), which are in the plan.
// words: [0] the next unit, [1] the CTAs done, [2 + r] the parts of record r
// done; the last CTA done zeroes them for the next launch.
template <int DIM>
__global__ void __launch_bounds__(256, 4)
ghost_kernel(GhostRec const *__restrict__ ghosts, GhostPlan plan, double *Ug, double const *UA,
             int nleaf, CaseState const *__restrict__ gate, CaseState const *__restrict__ cu,
             int stage, unsigned *words, int const *__restrict__ rank, int *err) {
  extern __shared__ double box[];
  __shared__ unsigned unit;
  __shared__ int ok;
  constexpr int PARTS = 2 * DIM + 1;
  unsigned *const next = words, *const finished = words + 1, *const done = words + 2;
  unsigned const total = (unsigned)plan.start[plan.n];
  for (;;) {
    if (threadIdx.x == 0) unit = atomicAdd(next, 1u);
    __syncthreads();
    unsigned const u = unit;
    if (u >= total) break;
    int k = 0;
    while (u >= (unsigned)plan.start[k + 1]) ++k;
    unsigned const v = u - (unsigned)plan.start[k];
    int const rec = plan.first[k] + (int)(v / PARTS), part = (int)(v % PARTS);
    GhostRec const &g = ghosts[rec];
    int lo[3], hi[3];
    if (gate[g.gate].dt > 0.0 && ghost_part<DIM>(g, part, lo, hi)) {
      if (threadIdx.x == 0) {
        ok = 1;
        int const *src = plan.type[k] == 1 ? g.src : g.nb;
        int const n = plan.type[k] == 1 ? (1 << DIM) : 27;
        for (int o = 0; o < n && ok; ++o)
          if (src[o] >= nleaf) ok = wait_count(done + rank[src[o] - nleaf], PARTS, err);
      }
      __syncthreads();
      if (!ok) return;
      if (plan.type[k] == 1)
        ghost_average_unit<DIM>(g, part, Ug, UA, nleaf, gate, cu, stage);
      else
        ghost_predict_unit<DIM>(g, part, Ug, UA, nleaf, gate, cu, stage, box);
    }
    __syncthreads();  // the unit's stores are issued; the box and `unit` are free again
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(done + rec, 1u);
    }
  }
  if (threadIdx.x == 0) {
    __threadfence();
    ok = atomicAdd(finished, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (ok) {
    for (int k = 0; k < plan.n; ++k)
      for (int r = threadIdx.x; r < (plan.start[k + 1] - plan.start[k]) / PARTS; r += blockDim.x)
        done[plan.first[k] + r] = 0u;
    if (threadIdx.x == 0) {
      *next = 0u;
      *finished = 0u;
    }
  }
}

// The ghost kernel's device words: the next unit, the CTAs done, the parts
// done of each ghost record.
inline size_t ghost_words(int nghost) { return 2 + (size_t)nghost; }

// The GlobalLaxFriedrichs maxima of all levels into every level's words (bit
// patterns of non-negative doubles order as the values).
__global__ void glf_fold_kernel(unsigned long long *glf, int nlev) {
  int const k = threadIdx.x;
  if (k >= 3) return;
  unsigned long long m = 0ull;
  for (int l = 0; l < nlev; ++l) m = glf[4 * l + k] > m ? glf[4 * l + k] : m;
  for (int l = 0; l < nlev; ++l) glf[4 * l + k] = m;
}

// A jump face of a leaf: kind 2 (coarse side: the neighbour is refined) or 3
// (fine side: the neighbour lies in a coarser leaf). Face loc: East 0, West 1,
// North 2, South 3, Top 4, Bottom 5 (boundary_specifications.h:56-63). acc:
// the parent-face accumulator the coarse side reads and the fine side fills;
// o1, o2: offsets of the fine face on the parent face (transverse cells).
struct JumpRec {
  int item, slot, loc, level, kind, acc, o1, o2;
};
// A coarse leaf with jump faces: its record per face location (-1: none).
struct CorrectRec {
  int slot, level, rec[6];
};

// jump multipliers per stage: SSP-RK3 (runge_kutta_3_TVD.h:42-46), then
// TVD-RK2 (runge_kutta_2_TVD.h:40-44), as the stage tables of the update kernel
__constant__ double kRkJump[5] = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0, 0.5, 0.5};

template <int DIM> struct FaceCells {
  __host__ __device__ static int t1(int d) { return d == 0 ? 1 : 0; }
  __host__ __device__ static int t2(int d) { return d == 2 ? 1 : 2; }
  __host__ __device__ static int n(int t) { return t < DIM ? IC : 1; }
};

// A stage's update and jump sums in one launch: CTAs (x < nupd, y) run the
// stage update of work item x (stage_update_cell, the arithmetic of every
// stage update); CTAs (nupd + r, 0) add jump record r's face fluxes to its
// sums, J += (w_stage * dt_level) * F (IntegrateJumpConservatives,
// time_integrator.h:64-80). The sums read the stage's fluxes, not its output,
// so the two parts are independent.
template <int DIM>
__global__ void __launch_bounds__(256)
level_update_kernel(double const *Uin, double const *U0, double *Uout, int const *__restrict__ work,
                    BlockMeta const *__restrict__ meta, double const *__restrict__ F,
                    long long stride, long long dstride, int stage,
                    CaseState const *__restrict__ cu, int nupd, JumpRec const *__restrict__ recs,
                    double *__restrict__ jbuf) {
  using G = Geo<DIM>;
  // 1D grid: the update CTAs of each leaf consecutively (parts of its cells),
  // then one CTA per jump record
  constexpr int PARTS = (G::INTERIOR + 255) / 256;
  int const x = blockIdx.x / PARTS;
  if (x < nupd) {
    int const slot = work[x];
    BlockMeta const bm = meta[slot];
    double const dt = cu[bm.case_id].dt;
    if (!(dt > 0.0)) return;
    int const t = (blockIdx.x - x * PARTS) * blockDim.x + threadIdx.x;
    if (t >= G::INTERIOR) return;
    stage_update_cell<DIM>(Uin, U0, Uout, F + (long long)x * stride, dstride, slot, t,
                           inv(bm.cell_size), rk_stage(stage, dt));
    return;
  }
  using FC = FaceCells<DIM>;
  int const ri = (int)blockIdx.x - nupd * PARTS;
  JumpRec const r = recs[ri];
  double const dtl = cu[r.level].dt;
  if (!(dtl > 0.0)) return;
  double const jstep = kRkJump[stage] * dtl;
  int const d = r.loc / 2, a = (r.loc % 2) ? 0 : IC;
  int const t1 = FC::t1(d), t2 = FC::t2(d), n1 = FC::n(t1), n2 = FC::n(t2);
  double const *Fd = F + (long long)r.item * stride + d * dstride;
  double *J = jbuf + (size_t)ri * G::NE * IC * IC;
  for (int y = threadIdx.x; y < G::NE * n1 * n2; y += blockDim.x) {
    int const e = y / (n1 * n2), q = y % (n1 * n2), p1 = q / n2, p2 = q % n2;
    int fi[3];
    fi[d] = a;
    fi[t1] = p1 + 1;
    fi[t2] = p2 + 1;
    J[e * IC * IC + p1 * IC + p2] += jstep * Fd[e * G::FACES + G::face(fi[0], fi[1], fi[2])];
  }
}

// AverageJumpBuffer of the fine faces of leaves that finished a step onto the
// parent faces, then their reset.
template <int DIM>
__global__ void __launch_bounds__(256)
jump_average_kernel(int const *__restrict__ fine, JumpRec const *__restrict__ recs,
                    double *__restrict__ jbuf, double *__restrict__ acc,
                    CaseState const *__restrict__ cu) {
  using G = Geo<DIM>;
  using FC = FaceCells<DIM>;
  int const ri = fine[blockIdx.x];
  JumpRec const r = recs[ri];
  if (!(cu[r.level].dt > 0.0)) return;
  int const d = r.loc / 2, t1 = FC::t1(d), t2 = FC::t2(d);
  int const h1 = t1 < DIM ? IC / 2 : 1, h2 = t2 < DIM ? IC / 2 : 1;
  double *J = jbuf + (size_t)ri * G::NE * IC * IC;
  double *A = acc + (size_t)r.acc * G::NE * IC * IC;
  for (int x = threadIdx.x; x < G::NE * h1 * h2; x += blockDim.x) {
    int const e = x / (h1 * h2), q = x % (h1 * h2), i = q / h2, j = q % h2;
    double const *c = J + e * IC * IC;
    double v;
    if constexpr (DIM == 1) v = c[0];
    else if constexpr (DIM == 2) v = (c[(2 * i) * IC] + c[(2 * i + 1) * IC]) * 0.5;
    else
      v = ((c[(2 * i) * IC + 2 * j] + c[(2 * i + 1) * IC + 2 * j + 1]) +
           (c[(2 * i + 1) * IC + 2 * j] + c[(2 * i) * IC + 2 * j + 1])) * 0.25;
    A[e * IC * IC + (r.o1 + i) * IC + (r.o2 + j)] += v;
  }
  __syncthreads();
  for (int x = threadIdx.x; x < G::NE * IC * IC; x += blockDim.x) J[x] = 0.0;
}

// JumpFluxAdjustment of the coarse leaves that finished a step: cells next to
// a refined neighbour get - CMS(coarse) + CMS(fine) of their face sums divided
// by the cell size (signs: +1 on West / South / Bottom faces, -1 on East /
// North / Top), then the sums are reset.
template <int DIM>
__global__ void __launch_bounds__(256)
jump_correct_kernel(CorrectRec const *__restrict__ corr, JumpRec const *__restrict__ recs,
                    double *__restrict__ jbuf, double *__restrict__ acc, double *U,
                    BlockMeta const *__restrict__ meta, CaseState const *__restrict__ cu) {
  using G = Geo<DIM>;
  using FC = FaceCells<DIM>;
  CorrectRec const cr = corr[blockIdx.x];
  if (!(cu[cr.level].dt > 0.0)) return;
  double const ocs = 1.0 / meta[cr.slot].cell_size;
  double *ub = U + (size_t)cr.slot * G::BLOCK_DOUBLES;
  for (int t = threadIdx.x; t < G::INTERIOR; t += blockDim.x) {
    int a[3];
    interior_coords<DIM>(t, a[0], a[1], a[2]);
    bool touched = false;
#pragma unroll
    for (int loc = 0; loc < 2 * DIM; ++loc) {
      int const d = loc / 2;
      touched |= cr.rec[loc] >= 0 && a[d] == ((loc % 2) ? 0 : IC - 1);
    }
    if (!touched) continue;
    int const cell = G::cell(a[0] + G::fic(0), a[1] + G::fic(1), a[2] + G::fic(2));
    for (int e = 0; e < G::NE; ++e) {
      double cf[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, ff[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int loc = 0; loc < 2 * DIM; ++loc) {
        int const d = loc / 2, high = (loc % 2) == 0;
        int const ri = cr.rec[loc];
        if (ri < 0 || a[d] != (high ? IC - 1 : 0)) continue;
        int const t1 = FC::t1(d), t2 = FC::t2(d);
        int const x = e * IC * IC + a[t1] * IC + a[t2];
        double const dir = high ? -1.0 : 1.0;
        cf[loc] = jbuf[(size_t)ri * G::NE * IC * IC + x] * ocs * dir;
        ff[loc] = acc[(size_t)recs[ri].acc * G::NE * IC * IC + x] * ocs * dir;
      }
      double &u = ub[e * G::CELLS + cell];
      u -= cms3(cf[0] + cf[1], cf[2] + cf[3], cf[4] + cf[5]);
      u += cms3(ff[0] + ff[1], ff[2] + ff[3], ff[4] + ff[5]);
    }
  }
  __syncthreads();
  for (int loc = 0; loc < 2 * DIM; ++loc) {
    int const ri = cr.rec[loc];
    if (ri < 0) continue;
    double *J = jbuf + (size_t)ri * G::NE * IC * IC;
    double *A = acc + (size_t)recs[ri].acc * G::NE * IC * IC;
    for (int x = threadIdx.x; x < G::NE * IC * IC; x += blockDim.x) {
      J[x] = 0.0;
      A[x] = 0.0;
    }
  }
}

__device__ __forceinline__ int levels_height(int t) { return __popc((t + 1) ^ t); }

// Micro time step from the per-level signal speeds, the per-level step sizes
// (cu: integrating levels, dt = sum of their micro steps) and the stage-0 flux
// gate (cf: levels whose interval starts now, dt = 1).
__global__ void levels_dt_kernel(LevelState *ls, CaseState *cu, CaseState *cf, int lmax, int tm) {
  LevelState &S = *ls;
  if (tm == 0)
    S.active = S.t < S.t_end && (S.max_macro <= 0 || S.macro < S.max_macro) && !S.status;
  double smax = 0.0;
  int st = 0;
  for (int l = 0; l <= lmax; ++l) {
    smax = fmax(smax, __longlong_as_double((long long)cu[l].smax_bits));
    cu[l].smax_bits = 0ull;
    st |= cu[l].status;
  }
  S.status |= st;
  bool const run = S.active && !S.status;
  double dt = 0.0;
  if (run) {
    double cur = S.t;
    for (int k = 0; k < tm; ++k) cur = cur + S.hist[k];
    double const rate = smax / S.h_fine;
    double local = rate == 0.0 ? DBL_MAX : S.cfl / rate;
    if (cur + local > S.t_end) local = fmax(S.t_end - cur, 0.0);
    dt = local;
  }
  S.hist[tm] = dt;
  int const lu = lmax - levels_height(tm) + 1;
  int const lf = tm == 0 ? 0 : lmax - levels_height(tm - 1) + 1;
  for (int l = 0; l <= lmax; ++l) {
    double dtl = 0.0;
    if (l >= lu)
      for (int k = tm; k > tm - (1 << (lmax - l)); --k) dtl += S.hist[k];
    cu[l].dt = run ? dtl : 0.0;
    cf[l].dt = (run && l >= lf) ? 1.0 : 0.0;
  }
}

__global__ void levels_commit_kernel(LevelState *ls, int tm, int nmicro) {
  LevelState &S = *ls;
  if (!S.active) return;
  S.micro += 1;
  if (tm == nmicro - 1) {
    double sum = 0.0;
    for (int k = 0; k < nmicro; ++k) sum = sum + S.hist[k];
    S.t = S.t + sum;
    S.macro += 1;
  }
}

struct NodeKey {
  int l, c[3];
  bool operator<(NodeKey const &o) const {
    return std::tie(l, c[0], c[1], c[2]) < std::tie(o.l, o.c[0], o.c[1], o.c[2]);
  }
};

// A leaf face at a level jump, as the tree builder finds it: kind 2 (coarse
// side) or 3 (fine side); the parent face (node, face location) whose
// accumulator the two sides share; the fine face's offsets on it.
struct JumpFace {
  int leaf, loc, kind;
  NodeKey node;
  int node_loc, o1, o2;
};

}  // namespace

// A run of ghost records of one type and level, filled by one launch.
struct GhostGroup {
  int type, level, first, count;
  int max_gate;  // the finest level that reads a ghost of the group
};

struct alp_levels {
  int dim = 3, scheme = 0, precision = 0, lmax = 0, nlev = 1, nmicro = 1;
  bool rk2 = false;  // TVD-RK2: two stages (stage tables from entry 3)
  alp::SchemeOptions opt;
  int nleaf = 0, nghost = 0, nslots = 0, ne = 5, cells = 0, faces = 0;
  long long cell_updates_per_macro = 0;
  double *U = nullptr, *UB = nullptr, *UC = nullptr, *F = nullptr;
  BlockMeta *meta = nullptr;
  int *nbr26 = nullptr, *work = nullptr;
  GhostRec *ghosts = nullptr;
  std::vector<GhostGroup> ghost_groups;  // launch order of the ghost records
  int ghost_grid = 0;                     // CTAs of the ghost kernel: one per SM
  unsigned *gwords = nullptr;  // its unit counters (ghost_words)
  int *grank = nullptr;        // [nghost] launch-order record of each ghost slot
  int *gerr = nullptr;                    // set when a wait for a ghost group ran out
  unsigned stall_next = 0;                // the second group's first unit in the macro step's first ghost launch
  // jump-flux conservation: records, per-record sums, parent-face sums,
  // fine-side record list, coarse leaves to correct
  int nrec = 0, nfine = 0, ncorr = 0, nacc = 0;
  JumpRec *jrecs = nullptr;
  double *jbuf = nullptr, *jacc = nullptr;
  int *jfine = nullptr;
  CorrectRec *jcorr = nullptr;
  CaseState *cu = nullptr, *cf = nullptr;
  LevelState *ls = nullptr;
  // GlobalLaxFriedrichs: wave-speed maxima, 4 words per level (all levels hold
  // the maxima over the leaves computing in the stage); null unless selected
  unsigned long long *glf = nullptr;
  std::vector<int> nwork_ge;  // work items of level >= l
  // The face launches of a stage with ghosts, split: work-list positions of
  // the leaves whose face neighbours are all leaves (`plain`, fluxes computed
  // while the ghost kernel runs on stream2), then of the others (`near`,
  // after it); each list finest first, with its prefix counts per level.
  int *fitems = nullptr;  // [nplain_total] plain positions, then the near ones
  std::vector<int> nplain_ge, nnear_ge;
  int nplain_total = 0;
  int ghost_prio = 0;  // the ghost kernel's launch priority (the greatest)
  cudaStream_t stream = nullptr;
  cudaStream_t stream2 = nullptr;  // the ghost kernel's, inside the macro-step graph
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaGraphExec_t graph = nullptr;

  long long dstride() const { return (long long)ne * faces; }
  long long stride() const { return dstride() * dim; }
  int cells_interior() const { return dim == 3 ? 4096 : (dim == 2 ? 256 : 16); }

  // The ghost kernel on stream st, at the greatest launch priority, so that
  // its CTAs take SM room as the concurrent face launch's CTAs finish.
  cudaError_t launch_ghosts(GhostPlan const &plan, double *Ug, CaseState const *gate, int s,
                            cudaStream_t st) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)ghost_grid);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = ghost_prio;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    GhostRec const *g = ghosts;
    double const *UA = U;
    int const *rk = grank;
    switch (dim) {
      case 1:
        cfg.dynamicSmemBytes = predict_smem_bytes<1>();
        return cudaLaunchKernelEx(&cfg, ghost_kernel<1>, g, plan, Ug, UA, nleaf, gate, cu, s, gwords, rk, gerr);
      case 2:
        cfg.dynamicSmemBytes = predict_smem_bytes<2>();
        return cudaLaunchKernelEx(&cfg, ghost_kernel<2>, g, plan, Ug, UA, nleaf, gate, cu, s, gwords, rk, gerr);
      default:
        cfg.dynamicSmemBytes = predict_smem_bytes<3>();
        return cudaLaunchKernelEx(&cfg, ghost_kernel<3>, g, plan, Ug, UA, nleaf, gate, cu, s, gwords, rk, gerr);
    }
  }

  // Reads and clears the ghost kernel's error word (a wait for a group that
  // ran out: the results of those steps are not valid).
  int ghost_check() {
    if (!gerr) return ALP_OK;
    int e = 0;
    ALP_CUDA(cudaMemcpyAsync(&e, gerr, sizeof(int), cudaMemcpyDeviceToHost, stream));
    ALP_CUDA(cudaStreamSynchronize(stream));
    if (!e) return ALP_OK;
    ALP_CUDA(cudaMemsetAsync(gwords, 0, ghost_words(nghost) * sizeof(unsigned), stream));
    ALP_CUDA(cudaMemsetAsync(gerr, 0, sizeof(int), stream));
    ALP_CUDA(cudaStreamSynchronize(stream));
    return alp::fail(ALP_ERR_CUDA, "level ghosts: a wait for a ghost group ran out; the step "
                                   "results are not valid");
  }

  int record_macro() {
    Launch L{dim, scheme, precision, U, work, nleaf, meta, BlockMeta{}, stream};
    L.opt = opt;
    L.glf = glf;
    double *in[3] = {U, UB, UC};
    double *out[3] = {UB, UC, U};
    int const nst = rk2 ? 2 : 3, s0 = rk2 ? 3 : 0;
    if (rk2) out[1] = U;
    bool first_ghost = true;
    stall_next = 0;
    for (int tm = 0; tm < nmicro; ++tm) {
      Launch La = L;
      ALP_CUDA(launch_signal_speed(La, cu, nullptr));
      levels_dt_kernel<<<1, 1, 0, stream>>>(ls, cu, cf, lmax, tm);
      ALP_CUDA(cudaGetLastError());
      auto height = [](int t) { return __builtin_popcount((unsigned)((t + 1) ^ t)); };
      int const lu = lmax - height(tm) + 1;
      int const lf = tm == 0 ? 0 : lmax - height(tm - 1) + 1;
      for (int s = 0; s < nst; ++s) {
        CaseState const *gate = s == 0 ? cf : cu;
        // the stage's ghosts in one launch: averaged ghosts finest level
        // first, then predicted ones coarsest first, each group after the one
        // before. A group fires only when a level reading it computes in this
        // stage (level >= lf for the first stage's fluxes, >= lu after), so
        // the others are left out of the plan.
        GhostPlan plan{};
        int const thr = s == 0 ? lf : lu;
        for (GhostGroup const &gg : ghost_groups)
          if (gg.max_gate >= thr) {
            plan.type[plan.n] = gg.type;
            plan.first[plan.n] = gg.first;
            plan.start[plan.n + 1] = plan.start[plan.n] + gg.count * (2 * dim + 1);
            ++plan.n;
          }
        bool const split = plan.n > 0;
        if (plan.n > 0) {
          if (first_ghost) stall_next = plan.n >= 2 ? (unsigned)plan.start[1] : 0u;
          first_ghost = false;
          if (split) {
            // the ghosts on stream2 beside the faces of the leaves that read none
            ALP_CUDA(cudaEventRecord(ev_fork, stream));
            ALP_CUDA(cudaStreamWaitEvent(stream2, ev_fork, 0));
            ALP_CUDA(launch_ghosts(plan, in[s], gate, s, stream2));
            ALP_CUDA(cudaEventRecord(ev_join, stream2));
          } else {
            ALP_CUDA(launch_ghosts(plan, in[s], gate, s, stream));
          }
        }
        Launch Ls = L;
        Ls.U = in[s];
        Ls.nwork = nwork_ge[s == 0 ? lf : lu];
        if (glf && Ls.nwork > 0) {
          // maxima over the leaves computing now (ComputeRightHandSide over its
          // levels, modular_algorithm_assembler.cpp:957-988): per level, then
          // the largest into every level's words
          ALP_CUDA(launch_glf_maxima(Ls, glf, nlev));
          glf_fold_kernel<<<1, 32, 0, stream>>>(glf, nlev);
          ALP_CUDA(cudaGetLastError());
        }
        if (split) {
          int const lv = s == 0 ? lf : lu;
          Launch Lp = Ls;
          Lp.items = fitems;
          Lp.nwork = nplain_ge[lv];
          if (Lp.nwork > 0)
            ALP_CUDA(launch_face_flux_all(Lp, nbr26, gate, F, stride(), dstride(), 128));
          ALP_CUDA(cudaStreamWaitEvent(stream, ev_join, 0));
          Launch Ln = Ls;
          Ln.items = fitems + nplain_total;
          Ln.nwork = nnear_ge[lv];
          if (Ln.nwork > 0)
            ALP_CUDA(launch_face_flux_all(Ln, nbr26, gate, F, stride(), dstride(), 128));
        } else if (Ls.nwork > 0) {
          ALP_CUDA(launch_face_flux_all(Ls, nbr26, gate, F, stride(), dstride(), 128));
        }
        // stage update of the integrating leaves and their jump sums, one launch
        int const nupd = nwork_ge[lu];
        if (nupd + nrec > 0) {
          dim3 const grid((unsigned)(nupd * ((cells_interior() + 255) / 256) + nrec));
          switch (dim) {
            case 1: level_update_kernel<1><<<grid, 256, 0, stream>>>(in[s], U, out[s], work, meta, F, stride(), dstride(), s0 + s, cu, nupd, jrecs, jbuf); break;
            case 2: level_update_kernel<2><<<grid, 256, 0, stream>>>(in[s], U, out[s], work, meta, F, stride(), dstride(), s0 + s, cu, nupd, jrecs, jbuf); break;
            default: level_update_kernel<3><<<grid, 256, 0, stream>>>(in[s], U, out[s], work, meta, F, stride(), dstride(), s0 + s, cu, nupd, jrecs, jbuf); break;
          }
          ALP_CUDA(cudaGetLastError());
        }
      }
      // the levels that integrated have finished a step: fine sums onto the
      // parent faces, then the coarse corrections
      if (nfine > 0) {
        switch (dim) {
          case 1: jump_average_kernel<1><<<nfine, 256, 0, stream>>>(jfine, jrecs, jbuf, jacc, cu); break;
          case 2: jump_average_kernel<2><<<nfine, 256, 0, stream>>>(jfine, jrecs, jbuf, jacc, cu); break;
          default: jump_average_kernel<3><<<nfine, 256, 0, stream>>>(jfine, jrecs, jbuf, jacc, cu); break;
        }
        ALP_CUDA(cudaGetLastError());
      }
      if (ncorr > 0) {
        switch (dim) {
          case 1: jump_correct_kernel<1><<<ncorr, 256, 0, stream>>>(jcorr, jrecs, jbuf, jacc, U, meta, cu); break;
          case 2: jump_correct_kernel<2><<<ncorr, 256, 0, stream>>>(jcorr, jrecs, jbuf, jacc, U, meta, cu); break;
          default: jump_correct_kernel<3><<<ncorr, 256, 0, stream>>>(jcorr, jrecs, jbuf, jacc, U, meta, cu); break;
        }
        ALP_CUDA(cudaGetLastError());
      }
      levels_commit_kernel<<<1, 1, 0, stream>>>(ls, tm, nmicro);
      ALP_CUDA(cudaGetLastError());
    }
    return ALP_OK;
  }

  void release() {
    if (graph) cudaGraphExecDestroy(graph);
    cudaFree(gwords);
    cudaFree(grank);
    cudaFree(fitems);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (stream2) cudaStreamDestroy(stream2);
    cudaFree(gerr);
    cudaFree(U);
    cudaFree(UB);
    cudaFree(UC);
    cudaFree(F);
    cudaFree(meta);
    cudaFree(nbr26);
    cudaFree(work);
    cudaFree(ghosts);
    cudaFree(jrecs);
    cudaFree(jbuf);
    cudaFree(jacc);
    cudaFree(jfine);
    cudaFree(jcorr);
    cudaFree(cu);
    cudaFree(cf);
    cudaFree(ls);
    cudaFree(glf);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

// Validates the tree and builds the per-slot neighbour table and the ghosts.
int build_tree(int dim, int layers, int const n0[3], int nleaf, int const *level, int const *coord,
               std::vector<int> &nbr26, std::vector<GhostRec> &ghosts,
               std::vector<JumpFace> &jumps, int *lmax_out) {
  using alp::fail;
  int lmax = 0;
  for (int b = 0; b < nleaf; ++b) {
    if (level[b] < 0 || level[b] >= kMaxLevels)
      return fail(ALP_ERR_INVALID, "leaf level outside 0.." + std::to_string(kMaxLevels - 1));
    lmax = std::max(lmax, level[b]);
  }
  std::map<NodeKey, int> leaf, refined;  // refined: value unused
  auto key = [&](int l, int const *c) {
    NodeKey k{l, {0, 0, 0}};
    for (int d = 0; d < dim; ++d) k.c[d] = c[d];
    return k;
  };
  auto extent = [&](int l, int d) { return d < dim ? n0[d] << l : 1; };
  for (int b = 0; b < nleaf; ++b) {
    int const *c = coord + 3 * b;
    for (int d = 0; d < dim; ++d)
      if (c[d] < 0 || c[d] >= extent(level[b], d))
        return fail(ALP_ERR_INVALID, "leaf " + std::to_string(b) + " lies outside the box");
    if (!leaf.emplace(key(level[b], c), b).second)
      return fail(ALP_ERR_INVALID, "two leaves share node " + std::to_string(b));
  }
  for (int b = 0; b < nleaf; ++b)
    for (int a = level[b] - 1; a >= 0; --a) {
      int c[3] = {0, 0, 0};
      for (int d = 0; d < dim; ++d) c[d] = coord[3 * b + d] >> (level[b] - a);
      NodeKey const k = key(a, c);
      if (leaf.count(k)) return fail(ALP_ERR_INVALID, "a leaf overlaps leaf " + std::to_string(b));
      refined.emplace(k, 0);
    }
  // tiling: level-0 nodes all present; refined nodes have all children
  long long n0tot = 1;
  for (int d = 0; d < dim; ++d) n0tot *= n0[d];
  long long covered = 0;
  for (auto const &kv : leaf)
    if (kv.first.l == 0) ++covered;
  for (auto const &kv : refined)
    if (kv.first.l == 0) ++covered;
  if (covered != n0tot) return fail(ALP_ERR_INVALID, "leaves do not cover every level-0 node");
  for (auto const &kv : refined)
    for (int o = 0; o < (1 << dim); ++o) {
      int c[3] = {0, 0, 0};
      for (int d = 0; d < dim; ++d) c[d] = 2 * kv.first.c[d] + ((o >> d) & 1);
      NodeKey const k = key(kv.first.l + 1, c);
      if (!leaf.count(k) && !refined.count(k))
        return fail(ALP_ERR_INVALID, "a refined node misses a child");
    }
  // face neighbours: same-level leaf, ghost of a refined node (finer leaves),
  // ghost inside a coarser leaf, or -1 (domain face)
  static int const face_slot[6] = {4, 21, 10, 15, 12, 13};
  nbr26.assign((size_t)nleaf * 26, -1);
  std::map<NodeKey, int> ghost_of;
  std::vector<NodeKey> ghost_key;
  std::vector<int> pending;  // ghosts to be filled whole whose sources are not resolved yet
  // the ghost of node position k (created on first use: refined -> type 1,
  // otherwise inside a coarser leaf -> type 0)
  auto ghost_for = [&](NodeKey const &k) {
    auto gi = ghost_of.find(k);
    if (gi != ghost_of.end()) return gi->second;
    GhostRec gr{};
    gr.slot = nleaf + (int)ghosts.size();
    gr.level = k.l;
    gr.layers = layers;
    gr.gate = -1;
    for (int o = 0; o < 8; ++o) gr.src[o] = -1;
    for (int o = 0; o < 27; ++o) gr.nb[o] = -1;
    if (refined.count(k)) {
      gr.type = 1;
    } else {
      gr.type = 0;
      for (int e = 0; e < dim; ++e) {
        gr.q[e] = k.c[e] >> 1;
        gr.oct |= (k.c[e] & 1) << e;
        gr.ext[e] = extent(k.l - 1, e) * IC;
      }
    }
    ghosts.push_back(gr);
    ghost_key.push_back(k);
    ghost_of.emplace(k, (int)ghosts.size() - 1);
    return (int)ghosts.size() - 1;
  };
  // the slot holding node position k whole: a leaf, or a ghost filled whole
  auto whole = [&](NodeKey const &k) {
    auto it = leaf.find(k);
    if (it != leaf.end()) return it->second;
    int const idx = ghost_for(k);
    if (!ghosts[idx].full) {
      ghosts[idx].full = 1;
      pending.push_back(idx);
    }
    return nleaf + idx;
  };
  for (int b = 0; b < nleaf; ++b) {
    int const l = level[b];
    for (int f = 0; f < 2 * dim; ++f) {
      int const d = f / 2, s = (f % 2) ? 1 : -1;
      int p[3] = {0, 0, 0};
      for (int e = 0; e < dim; ++e) p[e] = coord[3 * b + e];
      p[d] += s;
      if (p[d] < 0 || p[d] >= extent(l, d)) continue;
      NodeKey const k = key(l, p);
      auto it = leaf.find(k);
      if (it != leaf.end()) {
        nbr26[(size_t)b * 26 + face_slot[f]] = it->second;
        continue;
      }
      int const loc = f ^ 1;  // East 0, West 1, North 2, South 3, Top 4, Bottom 5
      if (refined.count(k)) {
        // coarse side: the neighbour's opposite face collects the fine sums
        jumps.push_back({b, loc, 2, k, loc ^ 1, 0, 0});
        for (int o = 0; o < (1 << dim); ++o) {
          int c[3] = {0, 0, 0};
          for (int e = 0; e < dim; ++e) c[e] = 2 * p[e] + ((o >> e) & 1);
          bool const face_child = ((o >> d) & 1) == (s > 0 ? 0 : 1);
          if (face_child && !leaf.count(key(l + 1, c)))
            return fail(ALP_ERR_INVALID, "face neighbours more than one level apart at leaf " +
                                             std::to_string(b));
        }
      } else {
        int q[3] = {0, 0, 0};
        for (int e = 0; e < dim; ++e) q[e] = p[e] >> 1;
        if (l == 0 || !leaf.count(key(l - 1, q)))
          return fail(ALP_ERR_INVALID, "face neighbours more than one level apart at leaf " +
                                           std::to_string(b));
        // fine side: this leaf's face lies on its parent's face of the same location
        NodeKey parent{l - 1, {0, 0, 0}};
        int oc[3] = {0, 0, 0};
        for (int e = 0; e < dim; ++e) {
          parent.c[e] = coord[3 * b + e] >> 1;
          oc[e] = coord[3 * b + e] & 1;
        }
        int const t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
        jumps.push_back({b, loc, 3, parent, loc, t1 < dim ? oc[t1] * (IC / 2) : 0,
                         t2 < dim ? oc[t2] * (IC / 2) : 0});
      }
      int const idx = ghost_for(k);
      GhostRec &gr = ghosts[idx];
      if (gr.type == 1)
        for (int o = 0; o < (1 << dim); ++o) {
          int c[3] = {0, 0, 0};
          for (int e = 0; e < dim; ++e) c[e] = 2 * p[e] + ((o >> e) & 1);
          auto ci = leaf.find(key(l + 1, c));
          if (ci != leaf.end()) gr.src[o] = ci->second;
        }
      else if (gr.full == 0 && gr.nb[13] < 0)
        pending.push_back(idx);
      // the leaf sits on the (s < 0 ? high : low) side of the ghost
      gr.faces |= 1 << (2 * d + (s < 0 ? 1 : 0));
      gr.gate = l;
      nbr26[(size_t)b * 26 + face_slot[f]] = gr.slot;
    }
  }
  // sources of the ghosts: a predicted ghost reads its parent position's 3^dim
  // neighbours whole, an averaged ghost filled whole reads all its children
  // whole; both may add further ghosts
  while (!pending.empty()) {
    int const idx = pending.back();
    pending.pop_back();
    GhostRec const g = ghosts[idx];
    if (g.type == 0) {
      if (g.nb[13] >= 0) continue;  // resolved already
      int nb[27];
      for (int o = 0; o < 27; ++o) {
        int const off[3] = {o / 9 - 1, (o / 3) % 3 - 1, o % 3 - 1};
        bool ok = true;
        int c[3] = {0, 0, 0};
        for (int e = 0; e < 3; ++e) {
          if (e >= dim) {
            ok = ok && off[e] == 0;
            continue;
          }
          c[e] = g.q[e] + off[e];
          ok = ok && c[e] >= 0 && c[e] < extent(g.level - 1, e);
        }
        nb[o] = ok ? whole(key(g.level - 1, c)) : -1;
      }
      for (int o = 0; o < 27; ++o) ghosts[idx].nb[o] = nb[o];
    } else {
      NodeKey const k = ghost_key[idx];
      int src[8];
      for (int o = 0; o < (1 << dim); ++o) {
        int c[3] = {0, 0, 0};
        for (int e = 0; e < dim; ++e) c[e] = 2 * k.c[e] + ((o >> e) & 1);
        src[o] = whole(key(g.level + 1, c));
      }
      for (int o = 0; o < (1 << dim); ++o) ghosts[idx].src[o] = src[o];
    }
  }
  // a ghost is needed whenever a ghost reading it is: its gate is the finest
  // gate of its readers (a level computes whenever a coarser one does)
  for (bool changed = true; changed;) {
    changed = false;
    for (GhostRec const &g : ghosts) {
      if (g.gate < 0) continue;
      int const *deps = g.type == 0 ? g.nb : g.src;
      int const n = g.type == 0 ? 27 : 8;
      for (int o = 0; o < n; ++o)
        if (deps[o] >= nleaf && ghosts[deps[o] - nleaf].gate < g.gate) {
          ghosts[deps[o] - nleaf].gate = g.gate;
          changed = true;
        }
    }
  }
  for (GhostRec const &g : ghosts)
    if (g.gate < 0 || g.gate > lmax) return fail(ALP_ERR_INVALID, "a ghost block has no reader");
  // the box of each ghost other ghosts read: grown from the cells its readers
  // hold (face layers and their own boxes) until nothing changes
  for (GhostRec &g : ghosts)
    for (int e = 0; e < 3; ++e) {
      g.lo[e] = e < dim ? IC : 0;
      g.hi[e] = e < dim ? 0 : 1;
    }
  auto grow = [&](int slot, int const lo[3], int const hi[3]) {
    GhostRec &t = ghosts[slot - nleaf];
    bool changed = false;
    for (int e = 0; e < dim; ++e) {
      if (lo[e] < t.lo[e]) t.lo[e] = lo[e], changed = true;
      if (hi[e] > t.hi[e]) t.hi[e] = hi[e], changed = true;
    }
    return changed;
  };
  for (bool changed = true; changed;) {
    changed = false;
    for (size_t gi = 0; gi < ghosts.size(); ++gi) {
      GhostRec const g = ghosts[gi];
      if (g.type == 1 && !g.full) continue;  // an averaged face ghost reads leaves only
      // bounding box of the cells g holds
      int lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
      bool any = false;
      for (int e = 0; e < dim; ++e) lo[e] = IC, hi[e] = 0;
      auto add = [&](int const *a, int const *b) {
        bool ok = true;
        for (int e = 0; e < dim; ++e) ok = ok && a[e] < b[e];
        if (!ok) return;
        any = true;
        for (int e = 0; e < dim; ++e) lo[e] = std::min(lo[e], a[e]), hi[e] = std::max(hi[e], b[e]);
      };
      add(g.lo, g.hi);
      for (int f = 0; f < 2 * dim; ++f)
        if ((g.faces >> f) & 1) {
          int a[3] = {0, 0, 0}, b[3] = {1, 1, 1};
          for (int e = 0; e < dim; ++e) b[e] = IC;
          a[f / 2] = (f & 1) ? IC - layers : 0;
          b[f / 2] = a[f / 2] + layers;
          add(a, b);
        }
      if (!any) continue;
      if (g.type == 0) {
        // parent-level cells read: the parent cells under the box, two more on
        // each side, clamped to the domain (global cells of the parent level)
        int plo[3] = {0, 0, 0}, phi[3] = {1, 1, 1};
        for (int e = 0; e < dim; ++e) {
          int const base = g.q[e] * IC + (IC / 2) * ((g.oct >> e) & 1);
          plo[e] = std::max(0, base + lo[e] / 2 - 2);
          phi[e] = std::min(g.ext[e], base + (hi[e] + 1) / 2 + 2);
        }
        for (int o = 0; o < 27; ++o) {
          int const src = g.nb[o];
          if (src < nleaf) continue;
          int const off[3] = {o / 9 - 1, (o / 3) % 3 - 1, o % 3 - 1};
          int a[3] = {0, 0, 0}, b[3] = {1, 1, 1};
          bool ok = true;
          for (int e = 0; e < dim; ++e) {
            int const n0c = (g.q[e] + off[e]) * IC;
            a[e] = std::max(plo[e], n0c) - n0c;
            b[e] = std::min(phi[e], n0c + IC) - n0c;
            ok = ok && a[e] < b[e];
          }
          if (ok && grow(src, a, b)) changed = true;
        }
      } else {
        for (int o = 0; o < (1 << dim); ++o) {
          int const src = g.src[o];
          if (src < nleaf) continue;
          int a[3] = {0, 0, 0}, b[3] = {1, 1, 1};
          bool ok = true;
          for (int e = 0; e < dim; ++e) {
            int const base = (IC / 2) * ((o >> e) & 1);
            a[e] = 2 * (std::max(lo[e], base) - base);
            b[e] = 2 * (std::min(hi[e], base + IC / 2) - base);
            ok = ok && a[e] < b[e];
          }
          if (ok && grow(src, a, b)) changed = true;
        }
      }
    }
  }
  *lmax_out = lmax;
  return ALP_OK;
}

}  // namespace

extern "C" {

int alp_levels_create(int dim, const alp_scheme *scheme, const alp_material *mat, const int *n0,
                      double h0, int nleaf, const int *h_level, const int *h_coord, double cfl,
                      double t0, double t_end, int max_macro_steps, const double *h_blocks,
                      alp_levels **out) {
  using namespace alp;
  if (!out) return fail(ALP_ERR_INVALID, "out is null");
  *out = nullptr;
  if (dim < 1 || dim > 3) return fail(ALP_ERR_INVALID, "dim must be 1, 2 or 3");
  int sid, prec;
  if (int rc = scheme_id(scheme, &sid, &prec)) return rc;
  if (int rc = check_material(mat)) return rc;
  if (!n0 || !h_level || !h_coord || !h_blocks || nleaf <= 0)
    return fail(ALP_ERR_INVALID, "empty or null tree description");
  for (int d = 0; d < dim; ++d)
    if (n0[d] <= 0) return fail(ALP_ERR_INVALID, "n0 must be positive");
  if (!(h0 > 0.0) || !(cfl > 0.0)) return fail(ALP_ERR_INVALID, "h0 and cfl must be positive");
  int n0v[3] = {1, 1, 1};
  for (int d = 0; d < dim; ++d) n0v[d] = n0[d];
  std::vector<int> nbr;
  std::vector<GhostRec> gh;
  std::vector<JumpFace> jf;
  int lmax = 0;
  int const layers = scheme->reconstruction_stencil == ST_WENO7 ? 4 : 3;
  if (int rc = build_tree(dim, layers, n0v, nleaf, h_level, h_coord, nbr, gh, jf, &lmax)) return rc;

  alp_levels *m = new (std::nothrow) alp_levels;
  if (!m) return fail(ALP_ERR_CUDA, "host allocation failed");
  m->dim = dim;
  m->scheme = sid;
  m->precision = prec;
  m->opt = scheme_options(scheme);
  m->rk2 = scheme->time_integrator == ALP_RK2;
  m->lmax = lmax;
  m->nlev = lmax + 1;
  m->nmicro = 1 << lmax;
  m->nleaf = nleaf;
  m->nghost = (int)gh.size();
  m->nslots = nleaf + m->nghost;
  m->ne = dim + 2;
  m->cells = 24 * (dim > 1 ? 24 : 1) * (dim > 2 ? 24 : 1);
  m->faces = 17 * (dim > 1 ? 17 : 2) * (dim > 2 ? 17 : 2);
  int const icells = 16 * (dim > 1 ? 16 : 1) * (dim > 2 ? 16 : 1);
  for (int b = 0; b < nleaf; ++b) m->cell_updates_per_macro += (long long)icells << h_level[b];

  // work list: finest level first (stable), prefix counts per level
  std::vector<int> work(nleaf);
  for (int b = 0; b < nleaf; ++b) work[b] = b;
  std::stable_sort(work.begin(), work.end(),
                   [&](int a, int b) { return h_level[a] > h_level[b]; });
  m->nwork_ge.assign(m->nlev + 1, 0);
  for (int l = 0; l <= lmax; ++l)
    for (int b = 0; b < nleaf; ++b)
      if (h_level[b] >= l) ++m->nwork_ge[l];

  // jump records: one per jump face, an accumulator per parent face
  std::vector<int> item_of(nleaf);
  for (int i = 0; i < nleaf; ++i) item_of[work[i]] = i;
  std::vector<JumpRec> recs;
  std::vector<int> fine;
  std::vector<CorrectRec> corr;
  std::map<std::pair<NodeKey, int>, int> acc_of;
  std::map<int, int> corr_of;  // leaf -> CorrectRec index
  for (JumpFace const &j : jf) {
    auto key = std::make_pair(j.node, j.node_loc);
    auto it = acc_of.find(key);
    int const acc = it == acc_of.end() ? (int)acc_of.size() : it->second;
    if (it == acc_of.end()) acc_of.emplace(key, acc);
    int const ri = (int)recs.size();
    recs.push_back({item_of[j.leaf], j.leaf, j.loc, h_level[j.leaf], j.kind, acc, j.o1, j.o2});
    if (j.kind == 3) {
      fine.push_back(ri);
    } else {
      auto ci = corr_of.find(j.leaf);
      if (ci == corr_of.end()) {
        CorrectRec c{j.leaf, h_level[j.leaf], {-1, -1, -1, -1, -1, -1}};
        ci = corr_of.emplace(j.leaf, (int)corr.size()).first;
        corr.push_back(c);
      }
      corr[ci->second].rec[j.loc] = ri;
    }
  }
  m->nrec = (int)recs.size();
  m->nfine = (int)fine.size();
  m->ncorr = (int)corr.size();
  m->nacc = (int)acc_of.size();

  std::vector<BlockMeta> meta(m->nslots);
  for (int b = 0; b < nleaf; ++b)
    meta[b] = meta_of(mat, h0 / (double)(1 << h_level[b]), h_level[b]);
  for (int g = 0; g < m->nghost; ++g)
    meta[nleaf + g] = meta_of(mat, h0 / (double)(1 << gh[g].level), gh[g].level);
  nbr.resize((size_t)m->nslots * 26, -1);

  size_t const blk = (size_t)m->ne * m->cells * sizeof(double);
  size_t const pool = blk * m->nslots;
  auto cleanup = [&](int rc) {
    m->release();
    delete m;
    return rc;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaStreamCreate"));
  {
    int least = 0, greatest = 0;
    e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    m->ghost_prio = greatest;
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&m->stream2, cudaStreamNonBlocking, greatest);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "ghost stream"));
  }
  // the ghost kernel's grid: the CTAs the device holds at once (one wave,
  // each pulling units until none is left), and its counters
  {
    void const *fn = dim == 1 ? (void const *)ghost_kernel<1>
                     : dim == 2 ? (void const *)ghost_kernel<2> : (void const *)ghost_kernel<3>;
    size_t const smem = dim == 1 ? predict_smem_bytes<1>()
                        : dim == 2 ? predict_smem_bytes<2>() : predict_smem_bytes<3>();
    int per_sm = 0, sms = 0, dev = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, smem);
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "ghost kernel setup"));
    if (per_sm < 1) return cleanup(alp::fail(ALP_ERR_CUDA, "the ghost kernel does not fit an SM"));
    // one CTA per SM: the ghost kernel runs beside the face launch of the
    // leaves that read no ghost, which keeps three of its four CTAs per SM
    // (three-level step: 19.4 ms per macro step against 20.3 without the
    // overlap, and 20.3 with four ghost CTAs per SM, which leave the faces no room)
    m->ghost_grid = sms;
    size_t const gw = ghost_words(m->nghost) * sizeof(unsigned);
    if ((e = cudaMalloc(&m->gwords, gw)) != cudaSuccess ||
        (e = cudaMalloc(&m->grank, sizeof(int) * std::max(m->nghost, 1))) != cudaSuccess ||
        (e = cudaMalloc(&m->gerr, sizeof(int))) != cudaSuccess ||
        (e = cudaMemsetAsync(m->gwords, 0, gw, m->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(m->gerr, 0, sizeof(int), m->stream)) != cudaSuccess)
      return cleanup(cuda_fail(e, "ghost counters"));
  }
  void **bufs[] = {(void **)&m->U, (void **)&m->UB, (void **)&m->UC};
  for (void **b : bufs) {
    e = cudaMalloc(b, pool);
    if (e == cudaSuccess) e = cudaMemsetAsync(*b, 0, pool, m->stream);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(level pools)"));
  }
  size_t const fbytes = (size_t)m->stride() * nleaf * sizeof(double);
  if ((e = cudaMalloc(&m->F, fbytes)) != cudaSuccess ||
      (e = cudaMalloc(&m->meta, sizeof(BlockMeta) * m->nslots)) != cudaSuccess ||
      (e = cudaMalloc(&m->nbr26, sizeof(int) * nbr.size())) != cudaSuccess ||
      (e = cudaMalloc(&m->work, sizeof(int) * nleaf)) != cudaSuccess ||
      (e = cudaMalloc(&m->ghosts, sizeof(GhostRec) * std::max(m->nghost, 1))) != cudaSuccess ||
      (e = cudaMalloc(&m->cu, sizeof(CaseState) * m->nlev)) != cudaSuccess ||
      (e = cudaMalloc(&m->cf, sizeof(CaseState) * m->nlev)) != cudaSuccess ||
      (e = cudaMalloc(&m->ls, sizeof(LevelState))) != cudaSuccess ||
      (sid == FS_ROE && scheme->flux_splitting == FSP_GLF &&
       (e = cudaMalloc(&m->glf, sizeof(unsigned long long) * 4 * m->nlev)) != cudaSuccess))
    return cleanup(cuda_fail(e, "cudaMalloc(level tables)"));
  size_t const jface = (size_t)m->ne * IC * IC * sizeof(double);
  if (m->nrec > 0) {
    if ((e = cudaMalloc(&m->jrecs, sizeof(JumpRec) * m->nrec)) != cudaSuccess ||
        (e = cudaMalloc(&m->jbuf, jface * m->nrec)) != cudaSuccess ||
        (e = cudaMalloc(&m->jacc, jface * std::max(m->nacc, 1))) != cudaSuccess ||
        (e = cudaMalloc(&m->jfine, sizeof(int) * std::max(m->nfine, 1))) != cudaSuccess ||
        (e = cudaMalloc(&m->jcorr, sizeof(CorrectRec) * std::max(m->ncorr, 1))) != cudaSuccess ||
        (e = cudaMemsetAsync(m->jbuf, 0, jface * m->nrec, m->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(m->jacc, 0, jface * std::max(m->nacc, 1), m->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(m->jrecs, recs.data(), sizeof(JumpRec) * m->nrec,
                             cudaMemcpyHostToDevice, m->stream)) != cudaSuccess ||
        (m->nfine > 0 && (e = cudaMemcpyAsync(m->jfine, fine.data(), sizeof(int) * m->nfine,
                                              cudaMemcpyHostToDevice, m->stream)) != cudaSuccess) ||
        (m->ncorr > 0 && (e = cudaMemcpyAsync(m->jcorr, corr.data(), sizeof(CorrectRec) * m->ncorr,
                                              cudaMemcpyHostToDevice, m->stream)) != cudaSuccess))
      return cleanup(cuda_fail(e, "jump-flux tables"));
  }
  std::vector<CaseState> cs(m->nlev);
  for (auto &c : cs) {
    c = CaseState{};
    c.t = t0;
    c.t_end = t_end;
    c.cfl = cfl;
    c.h_min = h0 / (double)m->nmicro;
  }
  LevelState st{};
  st.t = t0;
  st.t_end = t_end;
  st.cfl = cfl;
  st.h_fine = h0 / (double)m->nmicro;
  st.max_macro = max_macro_steps;
  for (int b = 0; b < nleaf; ++b) {
    e = cudaMemcpyAsync(m->U + (size_t)b * m->ne * m->cells, h_blocks + (size_t)b * m->ne * m->cells,
                        blk, cudaMemcpyHostToDevice, m->stream);
    if (e != cudaSuccess) break;
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(m->meta, meta.data(), sizeof(BlockMeta) * m->nslots,
                        cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(m->nbr26, nbr.data(), sizeof(int) * nbr.size(), cudaMemcpyHostToDevice,
                        m->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(m->work, work.data(), sizeof(int) * nleaf, cudaMemcpyHostToDevice,
                        m->stream);
  // the face launches beside the ghost kernel: positions of the leaves whose
  // face neighbours (the only blocks the face kernels read) are all leaves,
  // then of the others, each in work-list order (so finest first)
  std::vector<int> fit;
  {
    int const face_nb[6] = {4, 21, 10, 15, 12, 13};  // -x, +x, -y, +y, -z, +z in the 26 table
    std::vector<char> near(nleaf, 0);
    for (int p = 0; p < nleaf; ++p)
      for (int k = 0; k < 2 * dim; ++k)
        if (nbr[(size_t)work[p] * 26 + face_nb[k]] >= nleaf) near[p] = 1;
    for (int p = 0; p < nleaf; ++p)
      if (!near[p]) fit.push_back(p);
    m->nplain_total = (int)fit.size();
    for (int p = 0; p < nleaf; ++p)
      if (near[p]) fit.push_back(p);
    m->nplain_ge.assign(m->nlev + 1, 0);
    m->nnear_ge.assign(m->nlev + 1, 0);
    for (int l = 0; l <= lmax; ++l)
      for (int p = 0; p < nleaf; ++p)
        if (h_level[work[p]] >= l) ++(near[p] ? m->nnear_ge[l] : m->nplain_ge[l]);
  }
  if (e == cudaSuccess && (e = cudaMalloc(&m->fitems, sizeof(int) * std::max(nleaf, 1))) == cudaSuccess)
    e = cudaMemcpyAsync(m->fitems, fit.data(), sizeof(int) * nleaf, cudaMemcpyHostToDevice,
                        m->stream);
  // launch order: averaged ghosts finest level first (their children may be
  // averaged ghosts one level finer), then predicted ghosts coarsest level
  // first (their sources may be predicted ghosts one level coarser)
  std::vector<GhostRec> order;
  auto group = [&](int type, int lev) {
    int const first = (int)order.size();
    int max_gate = -1;
    for (GhostRec const &g : gh)
      if (g.type == type && g.level == lev) {
        order.push_back(g);
        max_gate = std::max(max_gate, g.gate);
      }
    if ((int)order.size() > first)
      m->ghost_groups.push_back({type, lev, first, (int)order.size() - first, max_gate});
  };
  for (int l = lmax; l >= 0; --l) group(1, l);
  for (int l = 0; l <= lmax; ++l) group(0, l);
  if ((int)m->ghost_groups.size() > kMaxGhostGroups)
    return cleanup(alp::fail(ALP_ERR_INVALID, "too many ghost groups for the ghost kernel"));
  // the launch-order record of each ghost slot; every ghost a record reads
  // must come from an earlier group (the ghost kernel's waits rely on it)
  std::vector<int> rank(m->nghost);
  for (int r = 0; r < m->nghost; ++r) rank[order[r].slot - nleaf] = r;
  for (GhostGroup const &gg : m->ghost_groups)
    for (int r = gg.first; r < gg.first + gg.count; ++r) {
      GhostRec const &g = order[r];
      int const *src = g.type == 1 ? g.src : g.nb;
      int const n = g.type == 1 ? (1 << dim) : 27;
      for (int o = 0; o < n; ++o)
        if (src[o] >= nleaf && rank[src[o] - nleaf] >= gg.first)
          return cleanup(alp::fail(ALP_ERR_INVALID,
                                   "a ghost block reads a ghost of its own or a later group"));
    }
  if (e == cudaSuccess && m->nghost)
    e = cudaMemcpyAsync(m->grank, rank.data(), sizeof(int) * m->nghost, cudaMemcpyHostToDevice,
                        m->stream);
  if (e == cudaSuccess && m->nghost)
    e = cudaMemcpyAsync(m->ghosts, order.data(), sizeof(GhostRec) * m->nghost,
                        cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(m->cu, cs.data(), sizeof(CaseState) * m->nlev, cudaMemcpyHostToDevice,
                        m->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(m->cf, cs.data(), sizeof(CaseState) * m->nlev, cudaMemcpyHostToDevice,
                        m->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(m->ls, &st, sizeof(st), cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  if (e != cudaSuccess) return cleanup(cuda_fail(e, "level case upload"));
  *out = m;
  return ALP_OK;
}

int alp_levels_destroy(alp_levels *m) {
  if (!m) return alp::fail(ALP_ERR_INVALID, "null level case");
  cudaStreamSynchronize(m->stream);
  m->release();
  delete m;
  return ALP_OK;
}

int alp_levels_step(alp_levels *m, int n_macro) {
  if (!m) return alp::fail(ALP_ERR_INVALID, "null level case");
  if (n_macro <= 0) return ALP_OK;
  nvtx3::scoped_range range{"alp_levels_step"};
  if (!m->graph) {
    cudaGraph_t g;
    ALP_CUDA(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
    int const rc = m->record_macro();
    cudaError_t const e = cudaStreamEndCapture(m->stream, &g);
    if (rc) {
      if (e == cudaSuccess) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return alp::cuda_fail(e, "cudaStreamEndCapture");
    cudaError_t const ei = cudaGraphInstantiate(&m->graph, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return alp::cuda_fail(ei, "cudaGraphInstantiate");
  }
  for (int i = 0; i < n_macro; ++i) ALP_CUDA(cudaGraphLaunch(m->graph, m->stream));
  return ALP_OK;
}

int alp_levels_get(alp_levels *m, double *h_blocks, double *t, int *macro_steps) {
  if (!m) return alp::fail(ALP_ERR_INVALID, "null level case");
  if (h_blocks)
    ALP_CUDA(cudaMemcpyAsync(h_blocks, m->U, sizeof(double) * m->ne * m->cells * m->nleaf,
                             cudaMemcpyDeviceToHost, m->stream));
  LevelState st;
  ALP_CUDA(cudaMemcpyAsync(&st, m->ls, sizeof(st), cudaMemcpyDeviceToHost, m->stream));
  ALP_CUDA(cudaStreamSynchronize(m->stream));
  if (int rc = m->ghost_check()) return rc;
  if (t) *t = st.t;
  if (macro_steps) *macro_steps = st.macro;
  if (st.status) return alp::fail(ALP_ERR_NUMERIC, "non-finite or non-positive state; case stopped");
  return ALP_OK;
}

int alp_levels_info(alp_levels *m, int *n_ghosts, int *max_level,
                    long long *cell_updates_per_macro_step, int *launches_per_macro_step) {
  if (!m) return alp::fail(ALP_ERR_INVALID, "null level case");
  if (n_ghosts) *n_ghosts = m->nghost;
  if (max_level) *max_level = m->lmax;
  if (cell_updates_per_macro_step) *cell_updates_per_macro_step = m->cell_updates_per_macro;
  if (launches_per_macro_step) {
    int per_micro = 2 + 1;  // signal speed, micro dt, commit
    auto height = [](int t) { return __builtin_popcount((unsigned)((t + 1) ^ t)); };
    int n = 0;
    for (int tm = 0; tm < m->nmicro; ++tm) {
      int const lu = m->lmax - height(tm) + 1;
      int const lf = tm == 0 ? 0 : m->lmax - height(tm - 1) + 1;
      n += per_micro;
      for (int s = 0; s < (m->rk2 ? 2 : 3); ++s) {
        int const thr = s == 0 ? lf : lu;
        bool any = false;
        for (auto const &gg : m->ghost_groups) any |= gg.max_gate >= thr;
        n += any ? 1 : 0;  // the ghost kernel
        int const lv = s == 0 ? lf : lu;
        int const faces = any ? (m->nplain_ge[lv] > 0 ? 1 : 0) + (m->nnear_ge[lv] > 0 ? 1 : 0)
                              : (m->nwork_ge[lv] > 0 ? 1 : 0);  // beside / after the ghosts
        n += faces + (m->glf && m->nwork_ge[lv] > 0 ? 2 : 0);  // GLF: maxima, fold
        n += m->nwork_ge[lu] + m->nrec > 0 ? 1 : 0;  // stage update with the jump sums
      }
      n += (m->nfine > 0 ? 1 : 0) + (m->ncorr > 0 ? 1 : 0);
    }
    *launches_per_macro_step = n;
  }
  return ALP_OK;
}

alp_stream_t alp_levels_stream(alp_levels *m) { return m ? (alp_stream_t)m->stream : nullptr; }

// The next ghost launch starts handing out units at its second group, so the
// first group never finishes and the waits for it run out.
int alp_levels_test_stall_ghosts(alp_levels *m) {
  if (!m) return alp::fail(ALP_ERR_INVALID, "null level case");
  if (!m->graph)
    return alp::fail(ALP_ERR_INVALID, "no macro step recorded yet: step the case first");
  if (m->stall_next == 0)
    return alp::fail(ALP_ERR_INVALID, "the macro step's first ghost launch has one group");
  ALP_CUDA(cudaStreamSynchronize(m->stream));
  ALP_CUDA(cudaMemcpy(m->gwords, &m->stall_next, sizeof(unsigned), cudaMemcpyHostToDevice));
  return ALP_OK;
}

}  // extern "C"
