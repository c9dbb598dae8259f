// Block layout shared by every kernel: the reference's Block buffers
// (block_definitions/field_buffer.h:37-40, compile_time_constants.h:39-45).
// A block is 16^d interior cells with a 4-cell halo, stored per field as a
// C-ordered double[TCX][TCY][TCZ] (z fastest); inactive dimensions have extent 1.
// Fields of one block are contiguous, blocks follow each other:
//   U[slot][field][TCX][TCY][TCZ]
// Face fluxes use the reference's per-direction arrays
//   F[slot][field][ICX+1][ICY+1][ICZ+1]        (convective_term_solver.h:67-81)
// where the face between interior cells a-1 and a along the sweep direction has
// index a, and the other two indices are the interior index + 1.
#pragma once

#include <cstddef>
#include <cstdint>

namespace alp {

constexpr int IC = 16;
constexpr int HS = 4;
constexpr int TC = IC + 2 * HS;

// conservative order Mass, Energy, MomentumX.. (field_setup.h:101-112)
constexpr int MASS = 0, ENERGY = 1, MOMX = 2;
// prime-state order Density, Pressure, VelocityX.. (field_setup.h:114-130)
constexpr int RHO = 0, PRES = 1, VELX = 2;

template <int DIM> struct Geo {
  static constexpr int NE = DIM + 2;
  static constexpr int TCX = TC;
  static constexpr int TCY = DIM > 1 ? TC : 1;
  static constexpr int TCZ = DIM > 2 ? TC : 1;
  static constexpr int ICX = IC;
  static constexpr int ICY = DIM > 1 ? IC : 1;
  static constexpr int ICZ = DIM > 2 ? IC : 1;
  static constexpr int CELLS = TCX * TCY * TCZ;
  static constexpr int INTERIOR = ICX * ICY * ICZ;
  static constexpr int FX = ICX + 1, FY = ICY + 1, FZ = ICZ + 1;
  static constexpr int FACES = FX * FY * FZ;  // one field of one direction
  // faces computed per direction: 17 along the sweep, interior across
  static constexpr int SWEEP_FACES = (IC + 1) * (DIM > 1 ? IC : 1) * (DIM > 2 ? IC : 1);
  static constexpr int BLOCK_DOUBLES = NE * CELLS;
  static constexpr int BLOCK_FLUX_DOUBLES = NE * FACES;

  __host__ __device__ static constexpr int fic(int d) { return d < DIM ? HS : 0; }
  __host__ __device__ static constexpr int tc(int d) { return d < DIM ? TC : 1; }
  __host__ __device__ static constexpr int ic(int d) { return d < DIM ? IC : 1; }
  __host__ __device__ static constexpr int cell(int i, int j, int k) {
    return (i * TCY + j) * TCZ + k;
  }
  __host__ __device__ static constexpr int face(int i, int j, int k) {
    return (i * FY + j) * FZ + k;
  }
};

// Per-block parameters: cell size and material (stiffened gas gamma, B,
// safe variant), plus the index of the block's case for per-case dt.
struct BlockMeta {
  double cell_size;
  double gamma;
  double B;
  int safe;
  int case_id;
};

// Per-case time-step state, device resident.
struct CaseState {
  double t;        // time reached
  double t_end;    // end time (LimitEndTime clip)
  double cfl;
  double dt;       // dt of the step in flight (0: case inactive)
  double h_min;    // finest cell size of the case
  unsigned long long smax_bits;  // max signal speed (non-negative double bits)
  int steps;       // steps taken
  int max_steps;   // <= 0: unbounded
  int status;      // bit 0: non-finite or non-positive state seen (case stopped)
  int hold;        // 1: the case takes no steps until released (request scheduling)
};

}  // namespace alp
