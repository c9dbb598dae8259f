// Index plan of the fused tile-stage kernel (tile_step.cuh), as host and
// device functions so that tests can replay it on the CPU.
//
// One work item is one SSP-RK3 (or TVD-RK2) stage of one 3D block. The block's
// cells are walked in x-planes. Stencils are read from shared memory:
//   * a ring of RING x-planes (16 x 16 cells, all five conserved fields) of the
//     stage input: planes -3 .. 18 in interior numbering, the six outside the
//     block taken from the x neighbours, none at walls (the readers map those
//     cells onto the block, stencil_src);
//   * per plane, the three rows beyond each y face and the (aligned, four wide)
//     columns beyond each z face, from the y / z neighbours.
// The item is a stream of warp tasks, taken by the CTA's warps in order:
//   X0              x face 0 (8 tasks of 32 faces)
//   for g = 0 .. 15:
//     U(g - LAG)    flux divergence and stage update of plane g - LAG (8 tasks
//                   of 32 cells), for g >= LAG
//     FX(g)         x face g + 1 (8 tasks)
//     FY(g), FZ(g)  the 17 x 16 y faces and 16 x 17 z faces of plane g (9 tasks
//                   each, the last one half full)
//   U(16 - LAG) .. U(15)
// A plane's update trails its faces by LAG planes, so that the fluxes it reads
// were computed a whole plane of tasks earlier, and the flux buffers it frees
// are next written a plane of tasks later. Every task waits only for tasks
// earlier in the stream (arrivals on shared-memory mbarriers) and for the
// loads those tasks released, so the warps never wait in a cycle. Faces are
// numbered as in the reference's flux arrays: face a of a direction lies
// between cells a - 1 and a (convective_term_solver.h:67-81).
#pragma once

#include "layout.cuh"
#include "rotate.cuh"

namespace alp {
namespace tile {

constexpr int NE = 5;           // conserved fields in 3D
constexpr int PLANE = IC * IC;  // cells of one x-plane
constexpr int YROW = 3 * IC;    // cells of one y halo (3 rows of 16)
constexpr int ZCOL = IC * 4;    // cells of one z halo (16 rows, 4 columns loaded)
constexpr int FACE_ROW = IC + 1;
constexpr int NPLANES = IC + 6;  // planes -3 .. 18

// shared-memory buffers
constexpr int RING = 8;  // x-planes of the stage input
constexpr int RFX = 4;   // x-face flux planes (face a in slot a % RFX)
constexpr int BYZ = 3;   // y / z face flux buffers (plane g in buffer g % BYZ)
constexpr int BH = 2;    // y / z halo buffers (plane g in buffer g % BH)
constexpr int BU = 2;    // U0 planes (plane g in buffer g % BU)

// Neighbour entries of the six faces in the 26-direction table (x slowest):
// W, E, S, N, B, T = (-1,0,0), (+1,0,0), (0,-1,0), (0,+1,0), (0,0,-1), (0,0,+1).
__host__ __device__ constexpr int face_slot(int d) {
  return d == 0 ? 4 : d == 1 ? 21 : d == 2 ? 10 : d == 3 ? 15 : d == 4 ? 12 : 13;
}

__host__ __device__ constexpr int ring_slot(int q) { return (q + 3) % RING; }

// Source of a stencil cell beyond the block along one direction: the index in
// the neighbour's buffer, or, at a domain face, the block's own cell (zero
// gradient: the first / last interior cell; symmetry: the mirror image, whose
// momentum normal to the wall is negated; symmetry_boundary_condition.h:60-217,
// boundary_constants.h:35-46, 103-160).
struct Src {
  int index;    // -3 .. 18: cell index along the direction
  bool own;     // true: the block's own cell `index` (0 .. 15)
  bool negate;  // mirror cell of a symmetry wall
};
// Written with selects only: the lanes of a warp hold faces at different
// positions, and a branch here would split the warp for the whole face
// computation that follows.
__host__ __device__ inline Src stencil_src(int c, int nlo, int nhi) {
  bool const lo = c < 0, out = lo || c >= IC;
  int const n = lo ? nlo : nhi;
  bool const wall = out && n < 0;
  bool const sym = wall && n == -2;
  int const mirror = lo ? -1 - c : 2 * IC - 1 - c;
  int const clamp = lo ? 0 : IC - 1;
  int const index = !wall ? c : (sym ? mirror : clamp);
  return Src{index, !out || wall, sym};
}

// ---- the task stream ------------------------------------------------------
enum TaskType { T_FX = 0, T_FY = 1, T_FZ = 2, T_U = 3, T_NONE = 4 };
constexpr int XT = PLANE / 32;                  // warp tasks of one x-face plane (8)
// The 17 x 16 y (or z) faces of a plane split into interior faces (a = 3 ..
// 13, whose six stencil cells all lie in the block's own plane: one warp
// reads them with constant offsets) and edge faces (a = 0, 1, 2, 14, 15, 16,
// whose stencils reach the halo rows / columns or a wall).
constexpr int NIF = (IC - 5) * IC;             // interior faces (176)
constexpr int NEF = 6 * IC;                    // edge faces (96)
constexpr int IFT = (NIF + 31) / 32;           // tasks of interior faces (6)
constexpr int EFT = NEF / 32;                  // tasks of edge faces (3)
constexpr int YT = IFT + EFT;                  // of the y faces of one plane (9)
static_assert(NEF % 32 == 0, "edge-face tasks are full");
constexpr int UT = PLANE / 32;                  // of one plane's stage update (8)
constexpr int FT = XT + 2 * YT;                  // face tasks of one plane (26)
constexpr int ITER = FT + UT;                     // tasks of one plane g >= LAG (34)
constexpr int LAG = 2;                            // planes between faces and update
constexpr int STREAM = XT + LAG * FT + (IC - LAG) * ITER + LAG * UT;  // 552

struct Task {
  int type;  // TaskType
  int g;     // FX: face g (0 .. 16); FY, FZ, U: plane g
  int w;     // task index within its kind (selects the 32 faces or cells)
};
// Face task r (0 .. FT - 1) of plane g.
__host__ __device__ inline Task face_task(int g, int r) {
  if (r < XT) return Task{T_FX, g + 1, r};
  if (r < XT + YT) return Task{T_FY, g, r - XT};
  return Task{T_FZ, g, r - XT - YT};
}
__host__ __device__ inline Task decode(int pos) {
  if (pos < XT) return Task{T_FX, 0, pos};
  pos -= XT;
  if (pos < LAG * FT) return face_task(pos / FT, pos % FT);
  pos -= LAG * FT;
  if (pos < (IC - LAG) * ITER) {
    int const g = LAG + pos / ITER, r = pos % ITER;
    return r < UT ? Task{T_U, g - LAG, r} : face_task(g, r - UT);
  }
  pos -= (IC - LAG) * ITER;
  if (pos < LAG * UT) return Task{T_U, IC - LAG + pos / UT, pos % UT};
  return Task{T_NONE, 0, 0};
}

// Reads of each x-plane (index q + 3) by the item's warp tasks, given the x
// neighbours (walls map cells onto the block): 8 tasks per x face per stencil
// cell, and for the block's own planes 9 + 9 (y, z faces) + 8 (stage update).
// A plane with no reads is not loaded; when a plane's count drops to zero its
// ring slot takes the next loaded plane of that slot.
__host__ __device__ inline void plane_reads(int nlo, int nhi, int (&reads)[NPLANES]) {
  for (int q = 0; q < NPLANES; ++q) reads[q] = 0;
  for (int a = 0; a <= IC; ++a)
    for (int m = 0; m < 6; ++m) reads[stencil_src(a - 3 + m, nlo, nhi).index + 3] += XT;
  for (int g = 0; g < IC; ++g) reads[g + 3] += 2 * YT + UT;
}
// First loaded plane of ring slot s (or 99 when none).
__host__ __device__ inline int first_plane_of_slot(int s, int const (&reads)[NPLANES]) {
  for (int q = s - 3; q <= IC + 2; q += RING)
    if (reads[q + 3] > 0) return q;
  return 99;
}
// The loaded plane after q in q's ring slot (or 99 when none).
__host__ __device__ inline int next_plane_of_slot(int q, int const (&reads0)[NPLANES]) {
  for (int n = q + RING; n <= IC + 2; n += RING)
    if (reads0[n + 3] > 0) return n;
  return 99;
}


// ---- TMA boxes ------------------------------------------------------------------
// Start of a box in the reference-layout pool [block][field][24][24][24]
// (coordinates z, y, x, field 0, block; z fastest). The z start must be a
// multiple of two doubles (16 bytes), which HS and HS + 12 are.
struct Box {
  int k, j, i, blk;
};
// Plane q (-3..18) of block `slot`: box 16 (z) x 16 (y) x 1 (x) x 5 fields.
__host__ __device__ inline Box plane_box(int q, int slot, int const (&nbr)[6]) {
  if (q < 0) return Box{HS, HS, HS + q + IC, nbr[0]};
  if (q >= IC) return Box{HS, HS, HS + q - IC, nbr[1]};
  return Box{HS, HS, HS + q, slot};
}
// y halo rows of plane g: rows 13..15 of the low neighbour (side 0), 0..2 of
// the high one (side 1); box 16 x 3 x 1 x 5.
__host__ __device__ inline Box yhalo_box(int g, int side, int const (&nbr)[6]) {
  return Box{HS, side ? HS : HS + IC - 3, HS + g, nbr[2 + side]};
}
// z halo columns of plane g: columns 12..15 of the low neighbour, 0..3 of the
// high one; box 4 x 16 x 1 x 5.
__host__ __device__ inline Box zhalo_box(int g, int side, int const (&nbr)[6]) {
  return Box{side ? HS : HS + IC - 4, HS, HS + g, nbr[4 + side]};
}

// ---- shared memory of one CTA ------------------------------------------------
struct Smem {
  double ring[RING][NE][PLANE];
  double fx[RFX][NE][PLANE];
  double fy[BYZ][NE][FACE_ROW * IC];  // [a][k]
  double fz[BYZ][NE][IC * FACE_ROW];  // [j][a]
  double yh[BH][2][NE][YROW];         // [buffer][low / high side]
  double zh[BH][2][NE][ZCOL];
  double u0[BU][NE][PLANE];
  // mbarriers, one phase per item: the loads (TMA transaction bytes) and the
  // finished tasks of each x face (XT arrivals), of each plane's y and z faces
  // (2 YT) and of each plane's stage update (UT)
  unsigned long long bar_plane[NPLANES];
  unsigned long long bar_halo[IC];
  unsigned long long bar_u0[IC];
  unsigned long long bar_x[IC + 1];
  unsigned long long bar_yz[IC];
  unsigned long long bar_u[IC];
  int reads[NPLANES];   // outstanding reads of each x-plane
  int reads0[NPLANES];  // reads at the item's start
  int reads_h[IC];      // outstanding reads of each plane's y / z halos
  int reads_u[IC];      // outstanding reads of each U0 plane
  int next_task;
  int item, skip, bad, dt_ready;
  int nbr[6];
  double dt;
  double red[32];
};


// One face of a warp task: direction dir; x faces: face a at jk = j * 16 + k
// (q = jk); y faces of plane g: face a of column k = t; z faces of plane g:
// face a of row j = t. Lanes q < 32 IFT take the interior faces (y: t fastest,
// z: a fastest, so that a warp's stencil reads are consecutive cells), the
// others the edge faces; `valid` is false for the idle lanes of the last
// interior task (their a, t name a real face, which they neither compute nor
// store).
struct FaceAt {
  int a, t;
  bool valid;
};
__host__ __device__ inline FaceAt face_at(int dir, int q) {
  if (dir == 0) return FaceAt{0, q, true};
  if (q < 32 * IFT) {
    bool const valid = q < NIF;
    int const i = valid ? q : NIF - 1;
    return dir == 1 ? FaceAt{3 + i / IC, i % IC, valid} : FaceAt{3 + i % (IC - 5), i / (IC - 5), valid};
  }
  int const r = q - 32 * IFT;
  int const e = dir == 1 ? r / IC : r % 6;  // which edge face: a = 0, 1, 2, 14, 15, 16
  return FaceAt{e < 3 ? e : e + IC - 5, dir == 1 ? r % IC : r / 6, true};
}
// True for the tasks of interior y / z faces (uniform over the warp).
__host__ __device__ inline bool interior_task(int dir, int w) { return dir != 0 && w < IFT; }

// Stencil of an interior face from consecutive cells of the block's own plane
// with constant offsets: cell m at p[m * STEP], field f at f * PLANE; the
// momenta in canonical order for direction DIR.
template <int DIR, int STEP>
__host__ __device__ inline void gather_interior(double const *p, double (&cons)[6][NE]) {
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    double const *c = p + m * STEP;
    cons[m][MASS] = c[MASS * PLANE];
    cons[m][ENERGY] = c[ENERGY * PLANE];
    cons[m][MOMX] = c[canon_field(DIR, MOMX) * PLANE];
    cons[m][MOMX + 1] = c[canon_field(DIR, MOMX + 1) * PLANE];
    cons[m][MOMX + 2] = c[canon_field(DIR, MOMX + 2) * PLANE];
  }
}

// The 6-cell stencil (cells a - 3 .. a + 2 along dir, the five fields in
// canonical order) of face q of x face plane g (dir 0) or of plane g (dir 1,
// 2), from the ring and the halo buffers; symmetry walls negate the principal
// momentum of mirrored cells.
__host__ __device__ inline void gather_face(Smem const &S, int dir, int g, int w, int q,
                                            double (&cons)[6][NE]) {
  FaceAt const f = face_at(dir, q);
  double const *plane = &S.ring[ring_slot(g)][0][0];
  if (interior_task(dir, w)) {
    if (dir == 1) gather_interior<1, IC>(plane + (f.a - 3) * IC + f.t, cons);
    else gather_interior<2, 1>(plane + f.t * IC + f.a - 3, cons);
    return;
  }
  int const a = dir == 0 ? g : f.a;
  int const nlo = S.nbr[2 * dir], nhi = S.nbr[2 * dir + 1];
  int const o2 = canon_field(dir, MOMX), o3 = canon_field(dir, MOMX + 1),
            o4 = canon_field(dir, MOMX + 2);
  int const hb = g % BH;
  // base and field stride of the halo buffers of the face's direction; the
  // cell offsets below are chosen with selects (the lanes' faces differ, a
  // branch would split the warp)
  double const *lo_buf = dir == 1 ? &S.yh[hb][0][0][0] : &S.zh[hb][0][0][0];
  double const *hi_buf = dir == 1 ? &S.yh[hb][1][0][0] : &S.zh[hb][1][0][0];
  int const hfs = dir == 1 ? YROW : ZCOL;
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    Src const s = stencil_src(a - 3 + m, nlo, nhi);
    double const *src;
    int fs;
    if (dir == 0) {  // uniform over the warp
      src = &S.ring[ring_slot(s.index)][0][f.t];
      fs = PLANE;
    } else {
      int const own_off = dir == 1 ? s.index * IC + f.t : f.t * IC + s.index;
      int const lo_off = dir == 1 ? (s.index + 3) * IC + f.t : f.t * 4 + s.index + 4;
      int const hi_off = dir == 1 ? (s.index - IC) * IC + f.t : f.t * 4 + s.index - IC;
      src = s.own ? plane + own_off : (s.index < 0 ? lo_buf + lo_off : hi_buf + hi_off);
      fs = s.own ? PLANE : hfs;
    }
    cons[m][MASS] = src[MASS * fs];
    cons[m][ENERGY] = src[ENERGY * fs];
    cons[m][MOMX] = src[o2 * fs];
    cons[m][MOMX + 1] = src[o3 * fs];
    cons[m][MOMX + 2] = src[o4 * fs];
    if (s.negate) cons[m][MOMX] = -1.0 * cons[m][MOMX];
  }
}

// Where the flux of that face goes (field f of the reference's order at
// base + f * stride).
struct FluxAt {
  double *base;
  int stride;
};
__host__ __device__ inline FluxAt flux_at(Smem &S, int dir, int g, int q) {
  FaceAt const f = face_at(dir, q);
  if (dir == 0) return FluxAt{&S.fx[g % RFX][0][f.t], PLANE};
  if (dir == 1) return FluxAt{&S.fy[g % BYZ][0][f.a * IC + f.t], FACE_ROW * IC};
  return FluxAt{&S.fz[g % BYZ][0][f.t * FACE_ROW + f.a], IC * FACE_ROW};
}

}  // namespace tile
}  // namespace alp
