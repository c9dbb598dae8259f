// Fused 3D stepping kernel: one persistent launch advances every resident case
// of an engine n SSP-RK3 (or TVD-RK2) steps.
//
// Work items are (step, stage, block) in a fixed order; each CTA takes the next
// item from a device counter. An item
//   1. waits (thread 0, bounded) until its block and its six face neighbours
//      have finished the previous stage (per-block flags, release / acquire);
//   2. streams the stage input into shared memory with TMA
//      (cp.async.bulk.tensor, no multicast): the block's x-planes through a ring
//      (tile_plan.cuh), the neighbours' planes beyond the x faces, and per plane
//      the rows / columns beyond the y and z faces; for stages after the first
//      also the step's initial state U0 per plane;
//   3. runs the item's task stream (tile_plan.cuh): the warps take face tasks
//      (32 faces through face_compute, the per-face arithmetic of the face-flux
//      kernels, into shared-memory flux planes) and stage-update tasks (32 cells:
//      flux_divergence and rk_apply, the arithmetic of stage_update_kernel,
//      written to the stage output) in order; shared-memory mbarriers order a
//      task after the tasks it reads from, and a plane's last reader issues the
//      load that reuses its buffer. The last stage also reduces the cells' signal
//      speed for the next step's dt;
//   4. publishes its block's flag. The last block of a case in a step commits
//      the step and computes the case's next dt (case_commit, case_dt_finalize).
// Results are therefore bit-identical to the face-flux + stage-update path, and
// the face fluxes never reach HBM: per stage the kernel reads the input state
// (and U0) and writes the output state.
//
// Items only wait on items taken earlier from the counter, and every taken item
// belongs to a running CTA, so the waits end; within an item a task only waits
// on earlier tasks. Every wait is bounded all the same: one that runs out sets
// an error bit in ctrl[1] (reported by the host) instead of hanging.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "face.cuh"
#include "step_common.cuh"
#include "tile_api.cuh"
#include "tile_plan.cuh"

namespace alp {

namespace tile {

// ---- PTX wrappers --------------------------------------------------------
__device__ __forceinline__ unsigned smem_addr(void const *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned count = 1) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
// One arrival (release at CTA scope: the arriving thread's earlier writes, and
// those its warp barrier ordered before them, are visible to the waiters).
__device__ __forceinline__ void mbar_arrive(unsigned long long *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}
__device__ __forceinline__ void mbar_inval(unsigned long long *b) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned long long *b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned long long *b) {
  unsigned ok;
  asm volatile(
      "{ .reg .pred P; mbarrier.try_wait.parity.shared::cta.b64 P, [%1], 0; selp.u32 %0, 1, 0, P; "
      "}"
      : "=r"(ok)
      : "r"(smem_addr(b))
      : "memory");
  return ok != 0;
}
// Every wait below is executed by all lanes of a warp and decided with
// __all_sync / __any_sync, so that a warp never splits around a wait: a split
// warp would run the face arithmetic that follows in two partial passes.
constexpr unsigned kFull = 0xffffffffu;

// Set once any wait of the launch ran out: every other wait then returns at
// once, so a failed launch ends within about one wait's bound.
__device__ __forceinline__ bool failed(int const *err) {
  return __any_sync(kFull, *reinterpret_cast<int const volatile *>(err) != 0);
}
// TMA tile load of a 5D box into shared memory, completion on mbarrier b.
__device__ __forceinline__ void tma_load(void *dst, CUtensorMap const *map, int k, int j, int i,
                                         int f, int blk, unsigned long long *b) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, "
      "{%3, %4, %5, %6, %7}], [%2];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(smem_addr(b)), "r"(k), "r"(j), "r"(i),
      "r"(f), "r"(blk)
      : "memory");
}
__device__ __forceinline__ int ld_acquire(int const *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Bounded spin of a warp until *p >= v (global, another CTA's release); on
// running out sets err bit `code` and returns.
__device__ __forceinline__ void spin_ge(int const *p, int v, int *err, int code) {
  unsigned ns = 32;
  for (int i = 0; i < (1 << 22); ++i) {
    if (__all_sync(kFull, ld_acquire(p) >= v)) return;
    if (failed(err)) return;
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
  }
  if ((threadIdx.x & 31) == 0) atomicOr(err, code);
}
// ---- loads ---------------------------------------------------------------
constexpr unsigned kPlaneBytes = NE * PLANE * sizeof(double);
constexpr unsigned kYBytes = NE * YROW * sizeof(double);
constexpr unsigned kZBytes = NE * ZCOL * sizeof(double);

// Plane q (-3..18) of the stage input into its ring slot: the block's own plane
// or the x neighbour's plane beyond the face.
__device__ __forceinline__ void issue_plane(Smem &S, CUtensorMap const *map, int slot, int q) {
  unsigned long long *b = &S.bar_plane[q + 3];
  Box const x = plane_box(q, slot, S.nbr);
  mbar_expect(b, kPlaneBytes);
  tma_load(&S.ring[ring_slot(q)][0][0], map, x.k, x.j, x.i, 0, x.blk, b);
}

// The y and z halos of plane g into halo buffer g % BH: rows 13..15 of the low
// y neighbour and 0..2 of the high one; columns 12..15 of the low z neighbour
// and 0..3 of the high one (the box's innermost start must be 16-byte aligned,
// so four columns are loaded). Walls load nothing.
__device__ __forceinline__ void issue_halos(Smem &S, CUtensorMap const *ymap,
                                            CUtensorMap const *zmap, int g) {
  int const hb = g % BH;
  unsigned long long *b = &S.bar_halo[g];
  int const ns = S.nbr[2], nn = S.nbr[3], nb = S.nbr[4], nt = S.nbr[5];
  unsigned const bytes = (ns >= 0 ? kYBytes : 0) + (nn >= 0 ? kYBytes : 0) +
                         (nb >= 0 ? kZBytes : 0) + (nt >= 0 ? kZBytes : 0);
  mbar_expect(b, bytes);
  for (int side = 0; side < 2; ++side) {
    Box const y = yhalo_box(g, side, S.nbr), z = zhalo_box(g, side, S.nbr);
    if (y.blk >= 0) tma_load(&S.yh[hb][side][0][0], ymap, y.k, y.j, y.i, 0, y.blk, b);
    if (z.blk >= 0) tma_load(&S.zh[hb][side][0][0], zmap, z.k, z.j, z.i, 0, z.blk, b);
  }
}

__device__ __forceinline__ void issue_u0(Smem &S, CUtensorMap const *map, int slot, int g) {
  mbar_expect(&S.bar_u0[g], kPlaneBytes);
  tma_load(&S.u0[g % BU][0][0], map, HS, HS, HS + g, 0, slot, &S.bar_u0[g]);
}

// ---- tasks -----------------------------------------------------------------
struct ItemCtx {
  CUtensorMap const *pmap, *ymap, *zmap, *u0map;
  double *out;  // the block in the stage output pool
  int slot, stage, step;
  bool first, reduce;
  Eos eos;
  double B, ocs;
  int *err;
  int const *dtflag_case;
  double const *dt_case;
};

// Warp wait until ready() holds on every lane (each lane tests its own
// condition: a counter, a load barrier, or nothing); on success the lane that
// saw a condition acquires it (fence) and the warp barrier passes that on to
// every lane. Bounded: on running out sets err bit `code` and returns.
template <class Ready>
__device__ __forceinline__ void wait_until(Ready ready, int *err, int code) {
  for (int i = 0; i < (1 << 22); ++i) {
    if (__all_sync(kFull, ready())) {
      __threadfence_block();
      __syncwarp();
      return;
    }
    if ((i & 255) == 255 && failed(err)) return;
    __nanosleep(20);
  }
  if ((threadIdx.x & 31) == 0) atomicOr(err, code);
}
__device__ __forceinline__ int vol(int const &x) { return *reinterpret_cast<int const volatile *>(&x); }

// A face task: 32 faces of x face plane g (FX) or of plane g's y / z faces
// (FY, FZ). The warp waits until the buffers the task writes are free and the
// planes it reads have arrived, and afterwards counts the task done and
// releases its reads; the waits and the bookkeeping atomics run on separate
// lanes side by side. Every direction goes through the one face_compute<3, 0>
// of the rotated stencil (gather_face), so the SM runs one copy of the face
// arithmetic.
template <int SCHEME, typename T>
__device__ __forceinline__ void task_face(Smem &S, ItemCtx const &C, Task const &t, bool compute) {
  int const lane = threadIdx.x & 31;
  int const dir = t.type;  // T_FX, T_FY, T_FZ are 0, 1, 2
  int const g = t.g;
  if (dir == 0) {
    // the flux slot of face g held face g - RFX, read by the updates of
    // planes g - RFX - 1 and g - RFX; lanes 2..7 wait for the six stencil
    // planes
    int const nlo = S.nbr[0], nhi = S.nbr[1];
    wait_until(
        [&] {
          if (lane == 0) return g <= RFX || mbar_try(&S.bar_u[g - RFX - 1]);
          if (lane == 1) return g < RFX || mbar_try(&S.bar_u[g - RFX]);
          if (lane < 8) return mbar_try(&S.bar_plane[stencil_src(g - 5 + lane, nlo, nhi).index + 3]);
          return true;
        },
        C.err, 2);
  } else {
    // the flux buffer held plane g - BYZ, read by its stage update; interior
    // faces read no halo
    bool const edge = !interior_task(dir, t.w);
    wait_until(
        [&] {
          if (lane == 0) return g < BYZ || mbar_try(&S.bar_u[g - BYZ]);
          if (lane == 1) return mbar_try(&S.bar_plane[g + 3]);
          if (lane == 2) return !edge || mbar_try(&S.bar_halo[g]);
          return true;
        },
        C.err, 2);
  }
  int const q = t.w * 32 + lane;
  if (compute && face_at(dir, q).valid) {
    double cons[6][NE];
    gather_face(S, dir, g, t.w, q, cons);
    double fd[NE];
    bool const valid = face_compute<3, 0, SCHEME, T>(C.eos, C.B, cons, fd);
    FluxAt const o = flux_at(S, dir, g, q);
#pragma unroll
    for (int c = 0; c < NE; ++c) o.base[canon_field(dir, c) * o.stride] = valid ? fd[c] : 0.0;
  }
  __syncwarp();
  __threadfence_block();
  if (dir == 0) {
    // lane 0 counts the task, lanes 1..6 release the six stencil planes
    if (lane == 0) {
      mbar_arrive(&S.bar_x[g]);
    } else if (lane < 7) {
      int const pq = stencil_src(g - 4 + lane, S.nbr[0], S.nbr[1]).index;
      if (atomicSub(&S.reads[pq + 3], 1) == 1) {
        int const n = next_plane_of_slot(pq, S.reads0);
        if (n != 99) issue_plane(S, C.pmap, C.slot, n);
      }
    }
  } else {
    if (lane == 0) {
      mbar_arrive(&S.bar_yz[g]);
    } else if (lane == 1) {
      if (atomicSub(&S.reads[g + 3], 1) == 1) {
        int const n = next_plane_of_slot(g, S.reads0);
        if (n != 99) issue_plane(S, C.pmap, C.slot, n);
      }
    } else if (lane == 2) {
      if (atomicSub(&S.reads_h[g], 1) == 1 && g + BH < IC) issue_halos(S, C.ymap, C.zmap, g + BH);
    }
  }
  __syncwarp();
}

// Stage update of 32 cells of plane g: flux divergence and RK stage into the
// output; the last stage also takes the cells' signal speed.
__device__ __forceinline__ void task_u(Smem &S, ItemCtx const &C, int g, int w, double &smax,
                                       int &bad) {
  int const lane = threadIdx.x & 31;
  bool const first = C.first;
  wait_until(
      [&] {
        if (lane == 0) return mbar_try(&S.bar_x[g]);
        if (lane == 1) return mbar_try(&S.bar_x[g + 1]);
        if (lane == 2) return mbar_try(&S.bar_yz[g]);
        if (lane == 3) return first || mbar_try(&S.bar_u0[g]);
        return true;
      },
      C.err, 8);
  if (!__all_sync(kFull, vol(S.dt_ready) != 0)) {
    // a first stage computes its fluxes ahead of the step's dt; every lane
    // reads and stores the same values
    spin_ge(C.dtflag_case, C.step + 1, C.err, 4);
    double const dt = *reinterpret_cast<double const volatile *>(C.dt_case);
    *reinterpret_cast<double volatile *>(&S.dt) = dt;
    *reinterpret_cast<int volatile *>(&S.skip) = dt == 0.0;
    __threadfence_block();
    *reinterpret_cast<int volatile *>(&S.dt_ready) = 1;
  }
  if (!__any_sync(kFull, vol(S.skip) != 0)) {
    RkStage const rk = rk_stage(C.stage, *reinterpret_cast<double volatile *>(&S.dt));
    int const jk = w * 32 + lane, j = jk / IC, k = jk % IC;
    double const *uin = &S.ring[ring_slot(g)][0][jk];
    double *out = C.out + Geo<3>::cell(HS + g, HS + j, HS + k);
    int const by = g % BYZ;
    double c[NE];
#pragma unroll
    for (int f = 0; f < NE; ++f) {
      double const rhs =
          0.0 + flux_divergence<3>(S.fx[g % RFX][f][jk], S.fx[(g + 1) % RFX][f][jk],
                                   S.fy[by][f][j * IC + k], S.fy[by][f][(j + 1) * IC + k],
                                   S.fz[by][f][j * FACE_ROW + k], S.fz[by][f][j * FACE_ROW + k + 1],
                                   C.ocs);
      double const v = rk_apply(rk, uin[f * PLANE], first ? 0.0 : S.u0[g % BU][f][jk], rhs);
      out[(size_t)f * Geo<3>::CELLS] = v;
      c[f] = v;
    }
    if (C.reduce) smax = dmax(smax, cell_signal_speed<3>(C.eos, c, bad));
  }
  __syncwarp();
  __threadfence_block();
  // lane 0 counts the task, lane 1 releases the plane, lane 2 the U0 plane
  if (lane == 0) {
    mbar_arrive(&S.bar_u[g]);
  } else if (lane == 1) {
    if (atomicSub(&S.reads[g + 3], 1) == 1) {
      int const n = next_plane_of_slot(g, S.reads0);
      if (n != 99) issue_plane(S, C.pmap, C.slot, n);
    }
  } else if (lane == 2 && !first) {
    if (atomicSub(&S.reads_u[g], 1) == 1 && g + BU < IC) issue_u0(S, C.u0map, C.slot, g + BU);
  }
  __syncwarp();
}

}  // namespace tile

// The persistent kernel: NW warps, one CTA per SM (shared memory).
template <int SCHEME, typename T, int NW>
__global__ void __launch_bounds__(NW * 32, 1) tile_step_kernel(__grid_constant__ const TileArgs A) {
  using namespace tile;
  // no static shared memory: the dynamic block starts the CTA's shared window,
  // so it is aligned as declared (TMA destinations need 128 bytes); the cast
  // keeps the shared state space, so the stencil reads are shared loads
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem &S = *reinterpret_cast<Smem *>(smem_raw);
  int const tid = threadIdx.x, lane = tid & 31;
  int const per_step = A.nstages * A.nwork;
  int const total = per_step * A.nsteps;
  int *err = A.ctrl + 1;
  if (smem_addr(smem_raw) & 127) {
    if (tid == 0) atomicOr(err, 16);  // never issue a TMA to a misaligned buffer
    return;
  }
  bool bars_live = false;  // thread 0: the barriers hold an earlier item's phases

#pragma unroll 1
  for (;;) {
    if (tid < 32) {
      bool const f = failed(err);
      if (tid == 0) S.item = f ? total : atomicAdd(A.ctrl, 1);
    }
    __syncthreads();
    int const item = S.item;
    if (item >= total) break;
    int const step = item / per_step;
    int const s = (item / A.nwork) % A.nstages;
    int const slot = A.order[s * A.nwork + item % A.nwork];
    int const stage = A.stage0 + s;
    bool const last = s == A.nstages - 1;
    int const need = A.nstages * step + s;
    // stage input / output pools: RK3 A -> B, (B, A) -> C, (C, A) -> A;
    // RK2 A -> B, (B, A) -> A; a trial's last stage writes B (RK3) or C (RK2)
    int const pin = s;
    int pout = A.nstages == 3 ? (s == 0 ? 1 : (s == 1 ? 2 : 0)) : (s == 0 ? 1 : 0);
    if (last && A.trial) pout = A.nstages == 3 ? 1 : 2;
    BlockMeta const bm = A.meta[slot];
    int const cid = bm.case_id;
    bool const first = rk_first_stage(stage);

    if (tid < 32) {
      // the inputs of this stage are final once the block and its face
      // neighbours finished the previous one (warp 0 waits)
      int const *nb = A.nbr26 + (size_t)slot * 26;
      spin_ge(A.done + slot, need, err, 1);
#pragma unroll 1
      for (int d = 0; d < 6; ++d) {
        int const n = nb[face_slot(d)];
        if (n >= 0) spin_ge(A.done + n, need, err, 1);
      }
    }
    if (tid == 0) {
      int const *nb = A.nbr26 + (size_t)slot * 26;
      for (int d = 0; d < 6; ++d) S.nbr[d] = nb[face_slot(d)];
      // dt of this step: final for later stages; for a first stage only once
      // the previous step's last blocks of the case committed
      int const ready = s > 0 || ld_acquire(A.dtflag + cid) >= step + 1;
      double const dt = ready ? *reinterpret_cast<double const volatile *>(&A.cases[cid].dt) : -1.0;
      S.dt = dt;
      S.dt_ready = ready;
      S.skip = ready && dt == 0.0;
      S.bad = 0;
      S.next_task = 0;
      int reads[NPLANES];
      plane_reads(S.nbr[0], S.nbr[1], reads);
      for (int q = 0; q < NPLANES; ++q) S.reads[q] = S.reads0[q] = reads[q];
      for (int g = 0; g < IC; ++g) {
        S.reads_h[g] = 2 * YT;
        S.reads_u[g] = UT;
      }
      // every barrier of the previous item has no operation pending (its
      // phase completed and was waited for, or, in a skipped item, nothing was
      // issued), so the barriers restart at phase 0 for this item
      for (int q = 0; q < NPLANES; ++q) {
        if (bars_live) mbar_inval(&S.bar_plane[q]);
        mbar_init(&S.bar_plane[q]);
      }
      for (int g = 0; g <= IC; ++g) {
        if (bars_live) mbar_inval(&S.bar_x[g]);
        mbar_init(&S.bar_x[g], XT);
      }
      for (int g = 0; g < IC; ++g) {
        if (bars_live) {
          mbar_inval(&S.bar_halo[g]);
          mbar_inval(&S.bar_u0[g]);
          mbar_inval(&S.bar_yz[g]);
          mbar_inval(&S.bar_u[g]);
        }
        mbar_init(&S.bar_halo[g]);
        mbar_init(&S.bar_u0[g]);
        mbar_init(&S.bar_yz[g], 2 * YT);
        mbar_init(&S.bar_u[g], UT);
      }
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      bars_live = true;
      if (!S.skip) {
        // the TMA (async proxy) reads what other CTAs wrote and released
        asm volatile("fence.proxy.async;" ::: "memory");
        CUtensorMap const *pmap = &A.plane[pin];
        for (int r = 0; r < RING; ++r) {
          int const q = first_plane_of_slot(r, reads);
          if (q != 99) issue_plane(S, pmap, slot, q);
        }
        for (int g = 0; g < BH; ++g) issue_halos(S, &A.yhalo[pin], &A.zhalo[pin], g);
        if (!first)
          for (int g = 0; g < BU; ++g) issue_u0(S, &A.plane[0], slot, g);
      }
    }
    __syncthreads();
    __syncwarp();

    if (!S.skip) {
      ItemCtx C;
      C.pmap = &A.plane[pin];
      C.ymap = &A.yhalo[pin];
      C.zmap = &A.zhalo[pin];
      C.u0map = &A.plane[0];
      C.out = A.pool[pout] + (size_t)slot * Geo<3>::BLOCK_DOUBLES;
      C.slot = slot;
      C.stage = stage;
      C.step = step;
      C.first = first;
      C.reduce = last && !A.trial;
      C.eos = Eos{bm.gamma, bm.B, bm.safe};
      C.B = bm.B;
      C.ocs = inv(bm.cell_size);
      C.err = err;
      C.dtflag_case = A.dtflag + cid;
      C.dt_case = &A.cases[cid].dt;
      double smax = 0.0;
      int bad = 0;
      // a warp claims its next task when it starts one (the claim's latency
      // hides behind the task); tasks still only wait on earlier positions, and
      // the earliest unfinished one is always some warp's current task
      int pos = 0;
      if (lane == 0) pos = atomicAdd(&S.next_task, 1);
      pos = __shfl_sync(kFull, pos, 0);
#pragma unroll 1
      while (pos < STREAM) {
        int claim = 0;
        if (lane == 0) claim = atomicAdd(&S.next_task, 1);
        Task const t = decode(pos);
        // a first stage whose dt turned out 0 keeps the bookkeeping, skips the work
        bool const compute = !*reinterpret_cast<int volatile *>(&S.skip);
        if (t.type == T_U) task_u(S, C, t.g, t.w, smax, bad);
        else if (t.type != T_NONE) task_face<SCHEME, T>(S, C, t, compute);
        pos = __shfl_sync(kFull, claim, 0);
      }
      __syncthreads();
      if (C.reduce && !S.skip) {
        // block maximum of the signal speed (non-negative doubles order like
        // their bit patterns) and the bad-cell flag
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) smax = dmax(smax, __shfl_xor_sync(kFull, smax, o));
        if (lane == 0) S.red[tid >> 5] = smax;
        if (__syncthreads_or(bad) && tid == 0) S.bad = 1;
        if (tid == 0) {
          double v = 0.0;
          for (int w = 0; w < NW; ++w) v = dmax(v, S.red[w]);
          if (S.bad) atomicOr(&A.cases[cid].status, 1);
          atomicMax(&A.cases[cid].smax_bits, (unsigned long long)__double_as_longlong(v));
        }
      }
    }
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      st_release(A.done + slot, need + 1);
      if (last) {
        // the case's last block of this step commits it and computes the next dt
        int const old = atomicAdd(A.cnt + cid, 1);
        if (old == (step + 1) * A.case_nb[cid] - 1) {
          __threadfence();
          if (!A.trial) {
            CaseState volatile *vs = A.cases + cid;
            CaseState cs;
            cs.t = vs->t;
            cs.t_end = vs->t_end;
            cs.cfl = vs->cfl;
            cs.dt = vs->dt;
            cs.h_min = vs->h_min;
            cs.smax_bits = vs->smax_bits;
            cs.steps = vs->steps;
            cs.max_steps = vs->max_steps;
            cs.status = vs->status;
            cs.hold = vs->hold;
            case_commit(cs);
            case_dt_finalize(cs);
            vs->t = cs.t;
            vs->steps = cs.steps;
            vs->smax_bits = cs.smax_bits;
            vs->dt = cs.dt;
          }
          __threadfence();
          st_release(A.dtflag + cid, step + 2);
        }
      }
    }
  }
}

namespace tile {
template <int SCHEME, typename T, int NW>
cudaError_t info_one(TileKernelInfo *out) {
  void const *fn = reinterpret_cast<void const *>(&tile_step_kernel<SCHEME, T, NW>);
  size_t const smem = sizeof(Smem);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, NW * 32, smem);
  if (e != cudaSuccess) return e;
  *out = TileKernelInfo{fn, NW * 32, smem, per_sm};
  return cudaSuccess;
}
template <int SCHEME, typename T>
cudaError_t info_t(int variant, TileKernelInfo *out) {
  switch (variant) {
    case 0: return info_one<SCHEME, T, 16>(out);
    case 1: return info_one<SCHEME, T, 12>(out);
  }
  return cudaErrorInvalidValue;
}
}  // namespace tile

// Sets the kernel's shared-memory limit and reports its launch shape.
template <int SCHEME>
cudaError_t tile_kernel_info(int variant, int precision, TileKernelInfo *out) {
  return precision == FP32_FLUX ? tile::info_t<SCHEME, float>(variant, out)
                                : tile::info_t<SCHEME, double>(variant, out);
}

}  // namespace alp
