// CPU replay of the fused tile kernel's plan (alpaca_b200/csrc/tile_plan.cuh)
// for one work item: the TMA boxes are emulated as copies out of a reference-
// layout pool, the warp-task stream runs in order with the kernel's
// bookkeeping (reads counted down, buffers handed to the next plane by their
// last reader), and every stencil the kernel would read from shared memory is
// compared with the stencil indexed directly in the pool (neighbour interiors,
// zero gradient or symmetry walls). Buffer contents are tagged so that a stage
// update reading a flux plane, a ring plane or a U0 plane that was overwritten
// too early is caught, as is a task whose wait would not be satisfied in
// stream order (a wait cycle).
//
// Usage: tile_plan_emu W E S N B T   (neighbour kinds: 0 periodic neighbour,
//        1 zero gradient, 2 symmetry); prints "ok <faces> <cells>" or fails.
#define __host__
#define __device__
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../alpaca_b200/csrc/tile_plan.cuh"

using namespace alp;
using namespace alp::tile;

namespace {

constexpr int NB = 27;  // a 3 x 3 x 3 block grid; the item is block 13 (the centre)
constexpr int CELLS = TC * TC * TC;
std::vector<double> pool;

double &P(int b, int f, int i, int j, int k) {
  return pool[(((size_t)b * NE + f) * TC + i) * TC * TC + (size_t)j * TC + k];
}

int fail_count = 0;
void check(bool ok, char const *what, int a, int b, int c) {
  if (!ok && fail_count++ < 20) std::printf("FAIL %s %d %d %d\n", what, a, b, c);
}

// TMA box copy: extents ek (z) x ej (y) x 1 (x) x 5 fields, dense in smem
void copy_box(double *dst, Box const &x, int ek, int ej) {
  check(x.k % 2 == 0, "box z start not 16-byte aligned", x.k, x.j, x.i);
  check(x.blk >= 0 && x.blk < NB, "box block", x.blk, x.i, 0);
  for (int f = 0; f < NE; ++f)
    for (int j = 0; j < ej; ++j)
      for (int k = 0; k < ek; ++k) {
        check(x.k + k < TC && x.j + j < TC && x.i < TC, "box outside pool", x.k + k, x.j + j, x.i);
        dst[(f * ej + j) * ek + k] = P(x.blk, f, x.i, x.j + j, x.k + k);
      }
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 7) return 2;
  int kind[6];
  for (int d = 0; d < 6; ++d) kind[d] = std::atoi(argv[1 + d]);
  // pool: interiors with distinct values, halos NaN (never read)
  pool.assign((size_t)NB * NE * CELLS, std::nan(""));
  for (int b = 0; b < NB; ++b)
    for (int f = 0; f < NE; ++f)
      for (int i = 0; i < IC; ++i)
        for (int j = 0; j < IC; ++j)
          for (int k = 0; k < IC; ++k)
            P(b, f, HS + i, HS + j, HS + k) = 1e6 * b + 1e5 * f + 1e4 * i + 1e2 * j + k + 0.5;
  int const self = 13;  // (1, 1, 1)
  int nbr[6];
  int const nslot[6] = {13 - 9, 13 + 9, 13 - 3, 13 + 3, 13 - 1, 13 + 1};
  for (int d = 0; d < 6; ++d) nbr[d] = kind[d] == 0 ? nslot[d] : -kind[d];

  // the expected value of cell c along direction dir (other two interior)
  auto expect = [&](int dir, int c, int p1, int p2, int f) {
    int const lo = nbr[2 * dir], hi = nbr[2 * dir + 1];
    int blk = self, idx = c;
    bool neg = false;
    if (c < 0) {
      if (lo >= 0) { blk = lo; idx = c + IC; }
      else if (lo == -1) idx = 0;
      else { idx = -1 - c; neg = true; }
    } else if (c >= IC) {
      if (hi >= 0) { blk = hi; idx = c - IC; }
      else if (hi == -1) idx = IC - 1;
      else { idx = 2 * IC - 1 - c; neg = true; }
    }
    int ii[3];
    ii[dir] = idx;
    ii[dir == 0 ? 1 : 0] = p1;
    ii[dir == 2 ? 1 : 2] = p2;
    double v = P(blk, f, HS + ii[0], HS + ii[1], HS + ii[2]);
    if (neg && f == MOMX + dir) v = -1.0 * v;
    return v;
  };

  static Smem S;
  // finished tasks of each x face / plane (the kernel counts them on mbarriers)
  int cnt_x[IC + 1] = {}, cnt_yz[IC] = {}, cnt_u[IC] = {};
  std::memset(&S, 0, sizeof(S));
  for (int d = 0; d < 6; ++d) S.nbr[d] = nbr[d];
  // buffer tags: which plane / face each buffer holds (-100: none)
  int ring_tag[RING], fx_tag[RFX], fyz_tag[BYZ], h_tag[BH], u_tag[BU];
  for (int &t : ring_tag) t = -100;
  for (int &t : fx_tag) t = -100;
  for (int &t : fyz_tag) t = -100;
  for (int &t : h_tag) t = -100;
  for (int &t : u_tag) t = -100;
  bool plane_loaded[NPLANES] = {}, halo_loaded[IC] = {}, u0_loaded[IC] = {};

  int reads[NPLANES];
  plane_reads(nbr[0], nbr[1], reads);
  for (int q = 0; q < NPLANES; ++q) S.reads[q] = S.reads0[q] = reads[q];
  for (int g = 0; g < IC; ++g) {
    S.reads_h[g] = 2 * YT;
    S.reads_u[g] = UT;
  }
  int actual_reads[NPLANES] = {};

  auto issue_plane = [&](int q) {
    int const s = ring_slot(q);
    check(ring_tag[s] == -100 || S.reads[ring_tag[s] + 3] == 0, "ring slot reused early", q,
          ring_tag[s], 0);
    copy_box(&S.ring[s][0][0], plane_box(q, self, nbr), IC, IC);
    ring_tag[s] = q;
    check(!plane_loaded[q + 3], "plane loaded twice", q, 0, 0);
    plane_loaded[q + 3] = true;
  };
  auto issue_halos = [&](int g) {
    int const hb = g % BH;
    check(h_tag[hb] == -100 || S.reads_h[h_tag[hb]] == 0, "halo buffer reused early", g, 0, 0);
    for (int side = 0; side < 2; ++side) {
      Box const y = yhalo_box(g, side, nbr), z = zhalo_box(g, side, nbr);
      if (y.blk >= 0) copy_box(&S.yh[hb][side][0][0], y, IC, 3);
      if (z.blk >= 0) copy_box(&S.zh[hb][side][0][0], z, 4, IC);
    }
    h_tag[hb] = g;
    halo_loaded[g] = true;
  };
  auto issue_u0 = [&](int g) {
    int const ub = g % BU;
    check(u_tag[ub] == -100 || S.reads_u[u_tag[ub]] == 0, "U0 buffer reused early", g, 0, 0);
    copy_box(&S.u0[ub][0][0], plane_box(g, self, nbr), IC, IC);
    u_tag[ub] = g;
    u0_loaded[g] = true;
  };
  auto release_plane = [&](int q) {
    actual_reads[q + 3]++;
    if (--S.reads[q + 3] == 0) {
      int const n = next_plane_of_slot(q, S.reads0);
      if (n != 99) issue_plane(n);
    }
  };

  for (int r = 0; r < RING; ++r) {
    int const q = first_plane_of_slot(r, reads);
    if (q != 99) issue_plane(q);
  }
  for (int g = 0; g < BH; ++g) issue_halos(g);
  for (int g = 0; g < BU; ++g) issue_u0(g);

  long faces = 0, cells = 0;
  int covered_x[IC + 1][PLANE] = {}, covered_y[IC][FACE_ROW * IC] = {},
      covered_z[IC][FACE_ROW * IC] = {}, covered_u[IC][PLANE] = {};
  for (int pos = 0; pos < STREAM; ++pos) {
    Task const t = decode(pos);
    if (t.type == T_FX) {
      int const a = t.g;
      // waits: flux slot free, source planes loaded
      if (a > RFX) check(cnt_u[a - RFX - 1] >= UT, "fx wait (a-5) unsatisfied", a, pos, 0);
      if (a >= RFX) check(cnt_u[a - RFX] >= UT, "fx wait (a-4) unsatisfied", a, pos, 0);
      for (int m = 0; m < 6; ++m) {
        int const q = stencil_src(a - 3 + m, nbr[0], nbr[1]).index;
        check(plane_loaded[q + 3], "fx source plane not loaded", a, q, pos);
        check(ring_tag[ring_slot(q)] == q, "fx source slot holds another plane", a, q,
              ring_tag[ring_slot(q)]);
      }
      for (int l = 0; l < 32; ++l) {
        int const jk = t.w * 32 + l;
        double cons[6][NE];
        gather_face(S, 0, a, t.w, jk, cons);
        for (int m = 0; m < 6; ++m)
          for (int c = 0; c < NE; ++c)
            check(cons[m][c] == expect(0, a - 3 + m, jk / IC, jk % IC, canon_field(0, c)),
                  "x stencil", a, jk, m);
        FluxAt const o = flux_at(S, 0, a, jk);
        check(o.base == &S.fx[a % RFX][0][jk] && o.stride == PLANE, "x flux slot", a, jk, 0);
        covered_x[a][jk]++;
        faces++;
      }
      fx_tag[a % RFX] = a;
      cnt_x[a]++;
      for (int m = 0; m < 6; ++m) release_plane(stencil_src(a - 3 + m, nbr[0], nbr[1]).index);
    } else if (t.type == T_FY || t.type == T_FZ) {
      int const g = t.g, dir = t.type == T_FY ? 1 : 2;
      if (g >= BYZ) check(cnt_u[g - BYZ] >= UT, "yz buffer wait unsatisfied", g, pos, 0);
      check(plane_loaded[g + 3] && ring_tag[ring_slot(g)] == g, "yz plane", g, pos, 0);
      check(halo_loaded[g] && h_tag[g % BH] == g, "yz halos", g, pos, 0);
      for (int l = 0; l < 32; ++l) {
        int const q = t.w * 32 + l;
        FaceAt const fa = face_at(dir, q);
        if (!fa.valid) continue;
        int const a = fa.a, tt = fa.t;
        double cons[6][NE];
        gather_face(S, dir, g, t.w, q, cons);
        for (int m = 0; m < 6; ++m)
          for (int c = 0; c < NE; ++c) {
            // transverse indices: y faces (x = g, z = tt); z faces (x = g, y = tt);
            // canonical slot c holds the rotated field
            double const e = expect(dir, a - 3 + m, g, tt, canon_field(dir, c));
            check(cons[m][c] == e, dir == 1 ? "y stencil" : "z stencil", a, tt, m);
          }
        FluxAt const o = flux_at(S, dir, g, q);
        check(dir == 1 ? (o.base == &S.fy[g % BYZ][0][a * IC + tt] && o.stride == FACE_ROW * IC)
                       : (o.base == &S.fz[g % BYZ][0][tt * FACE_ROW + a] && o.stride == IC * FACE_ROW),
              "yz flux slot", dir, q, g);
        if (dir == 1) covered_y[g][a * IC + tt]++;
        else covered_z[g][tt * FACE_ROW + a]++;
        faces++;
      }
      fyz_tag[g % BYZ] = g;
      cnt_yz[g]++;
      release_plane(g);
      if (--S.reads_h[g] == 0 && g + BH < IC) issue_halos(g + BH);
    } else if (t.type == T_U) {
      int const g = t.g;
      check(cnt_x[g] >= XT && cnt_x[g + 1] >= XT && cnt_yz[g] >= 2 * YT,
            "update wait unsatisfied", g, pos, 0);
      check(u0_loaded[g] && u_tag[g % BU] == g, "U0 plane", g, pos, 0);
      check(fx_tag[g % RFX] == g && fx_tag[(g + 1) % RFX] == g + 1, "update reads fx", g,
            fx_tag[g % RFX], fx_tag[(g + 1) % RFX]);
      check(fyz_tag[g % BYZ] == g, "update reads fy/fz", g, fyz_tag[g % BYZ], 0);
      check(ring_tag[ring_slot(g)] == g, "update reads Uin", g, ring_tag[ring_slot(g)], 0);
      for (int l = 0; l < 32; ++l) {
        int const jk = t.w * 32 + l;
        for (int f = 0; f < NE; ++f) {
          check(S.ring[ring_slot(g)][f][jk] == P(self, f, HS + g, HS + jk / IC, HS + jk % IC),
                "Uin value", g, jk, f);
          check(S.u0[g % BU][f][jk] == P(self, f, HS + g, HS + jk / IC, HS + jk % IC),
                "U0 value", g, jk, f);
        }
        covered_u[g][jk]++;
        cells++;
      }
      cnt_u[g]++;
      release_plane(g);
      if (--S.reads_u[g] == 0 && g + BU < IC) issue_u0(g + BU);
    } else {
      check(false, "task past the stream", pos, 0, 0);
    }
  }
  for (int a = 0; a <= IC; ++a)
    for (int x = 0; x < PLANE; ++x) check(covered_x[a][x] == 1, "x face coverage", a, x, 0);
  for (int g = 0; g < IC; ++g) {
    for (int x = 0; x < FACE_ROW * IC; ++x) {
      check(covered_y[g][x] == 1, "y face coverage", g, x, 0);
      check(covered_z[g][x] == 1, "z face coverage", g, x, 0);
    }
    for (int x = 0; x < PLANE; ++x) check(covered_u[g][x] == 1, "cell coverage", g, x, 0);
  }
  for (int q = 0; q < NPLANES; ++q) {
    check(actual_reads[q] == S.reads0[q], "plane read count", q - 3, actual_reads[q], S.reads0[q]);
    check(S.reads[q] == 0, "plane reads left", q - 3, S.reads[q], 0);
    check(plane_loaded[q] == (S.reads0[q] > 0), "plane loaded iff read", q - 3, 0, 0);
  }
  for (int g = 0; g < IC; ++g)
    check(halo_loaded[g] && u0_loaded[g], "halo / U0 load", g, 0, 0);
  if (fail_count) {
    std::printf("%d failures\n", fail_count);
    return 1;
  }
  std::printf("ok %ld %ld\n", faces, cells);
  return 0;
}
