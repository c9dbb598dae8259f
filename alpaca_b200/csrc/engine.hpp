// Engine internals shared by the C ABI (capi.cu) and the request loop (server.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "../../include/alpaca_b200.h"
#include "kernels.cuh"
#include "tile_api.cuh"

namespace alp {
int fail(int code, std::string const &msg);
int cuda_fail(cudaError_t e, char const *where);

// A device array that grows and shrinks in place (elastic.cu): its virtual
// range is reserved for the largest size, physical memory is mapped into it
// in chunks of elastic_chunk_bytes() from the start.
struct ElasticArray {
  unsigned long long base = 0;  // reserved virtual address
  size_t reserved = 0;          // bytes of virtual range
  size_t mapped = 0;            // bytes backed from base
  int device = 0;
  std::vector<unsigned long long> chunks;  // physical allocation handles, in order
};
size_t elastic_chunk_bytes();
int elastic_reserve(ElasticArray &a, size_t bytes);
// Maps or unmaps whole chunks at the end so that the array holds at least
// `bytes` with the fewest chunks; the caller makes sure nothing in flight
// touches a range it unmaps.
int elastic_resize(ElasticArray &a, size_t bytes);
void elastic_release(ElasticArray &a);
}  // namespace alp

#define ALP_CUDA(call)                                        \
  do {                                                        \
    cudaError_t const e_ = (call);                            \
    if (e_ != cudaSuccess) return alp::cuda_fail(e_, #call);  \
  } while (0)

using alp::BlockMeta;
using alp::CaseState;
using alp::Launch;
using alp::FP64;
using alp::FV_CHAR;
using alp::fail;
using alp::launch_face_flux_all;
using alp::launch_stage_update;
using alp::launch_signal_speed;
using alp::launch_dt_finalize;
using alp::launch_step_commit;

// The engine keeps every case in three block pools: A holds the state at the
// start of a step (and at its end), B and C the first and second RK3 stages.
// Stencils read neighbour blocks directly, so pool halos are only filled when
// a case is exported.
struct alp_engine {
  int dim = 3, scheme = FV_CHAR, precision = FP64;
  alp_scheme selection{};  // the selection the engine was created with
  alp::SchemeOptions opt;  // run-time selected schemes (face-flux path only)
  int rk2 = 0;             // 1: TVD-RK2 (2 stages, face-flux paths), 0: SSP-RK3
  int capacity = 0, max_cases = 0;
  int slots_max = 0;  // slots of the per-block tables (= capacity unless elastic)
  int ne = 5, cells = 0, faces = 0;
  double *U = nullptr, *UB = nullptr, *UC = nullptr;
  double *F = nullptr;  // face fluxes [slot][dim][NE][faces] (face-flux path)
  double *R = nullptr;  // per-cell flux differences [slot][NE][interior] (pencil path)
  int path = 1;         // 0: pencil sweeps, 1: face fluxes + stage update, 2: the same in
                        // overlapped batches, 3: fused tile stages (one persistent launch
                        // for all steps of a call; 3D, default schemes)
  cudaStream_t stream2 = nullptr;  // stage updates of the overlapped path
  static constexpr int kMaxBatches = 16;
  cudaEvent_t ev_batch[kMaxBatches] = {};
  cudaEvent_t ev_join = nullptr;
  int face_threads = 128;
  BlockMeta *meta = nullptr;
  int *nbr26 = nullptr;
  int *work = nullptr;
  CaseState *cases = nullptr;
  unsigned long long *glf = nullptr;  // GlobalLaxFriedrichs wave speeds [case][4]
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  bool use_graph = true;
  bool graph_dirty = true;

  // fused tile stages (path 3)
  bool tile_ok = false;       // 3D, default schemes, descriptors encoded
  int tile_variant = 0;       // index into alp::kTileWarps
  alp::TileArgs targs{};      // TMA descriptors and device pointers (nsteps set per launch)
  alp::TileKernelInfo tinfo[alp::kTileVariants] = {};
  int tgrid[alp::kTileVariants] = {};
  int *tsync = nullptr;       // [2 + capacity + 2 max_cases]: next item, error, block flags,
                              // dt flags, last-stage counts
  int *torder = nullptr;      // [3][capacity] block slots per stage, in readiness order
  int *tcase_nb = nullptr;    // [max_cases] blocks of each case in the work list
  cudaGraph_t tile_graph_src = nullptr;  // the graph `graph` was instantiated from (kept:
                                         // its node handle addresses the launch to update)
  cudaGraphNode_t tile_node = nullptr;    // the persistent launch in it
  int tile_graph_n = 0;                   // its step count

  // host mirrors
  std::vector<BlockMeta> h_meta;
  std::vector<int> h_nbr26;
  std::map<int, int> free_ranges;  // start -> length
  struct CaseRec {
    bool live = false;
    int first = 0, nb = 0;
    alp_material mat{};     // as given, for checkpoints
    double cell_size = 0.0;
  };
  std::vector<CaseRec> case_rec;
  std::vector<int> h_work;
  std::vector<int> h_torder, h_case_nb;  // staging of the tile path's orders and case sizes
  std::vector<CaseState> h_case_state;  // staging for case records sent to the device
  int nwork = 0;
  int compactions = 0;  // times the live cases were moved together (compact)

  long long dstride() const { return (long long)ne * faces; }
  long long stride() const { return dstride() * dim; }

  // dt, then per stage the fluxes and the stage update: A -> B, (B, A) -> C,
  // (C, A) -> A. trial: the last stage writes B instead of A and the step is
  // not committed, so the case state is left as it was (autotuning).
  int record_step(bool trial = false) {
    Launch L{dim, scheme, precision, U, work, nwork, meta, BlockMeta{}, stream};
    L.opt = opt;
    ALP_CUDA(launch_signal_speed(L, cases, nullptr));
    ALP_CUDA(launch_dt_finalize(cases, max_cases, stream));
    // RK3: A -> B, (B, A) -> C, (C, A) -> A; RK2: A -> B, (B, A) -> A (trial: C)
    double *in[3] = {U, UB, UC};
    double *out[3] = {UB, UC, trial ? UB : U};
    if (rk2) out[1] = trial ? UC : U;
    int const nst = rk2 ? 2 : 3, s0 = rk2 ? 3 : 0;
    bool const glf_due = scheme == alp::FS_ROE && opt.splitting == alp::FSP_GLF;
    for (int s = 0; s < nst; ++s) {
      Launch Ls = L;
      Ls.U = in[s];
      if (glf_due) {
        // the case's maxima over its blocks before this stage's fluxes
        ALP_CUDA(launch_glf_maxima(Ls, glf, max_cases));
        Ls.glf = glf;
      }
      if (path == 0) {
        ALP_CUDA(alp::launch_pencil_stage(Ls, U, out[s], R, nbr26, cases, s));
      } else if (path == 2) {
        if (int rc = record_overlapped_stage(Ls, out[s], s0 + s)) return rc;
      } else {
        ALP_CUDA(launch_face_flux_all(Ls, nbr26, cases, F, stride(), dstride(), face_threads));
        ALP_CUDA(launch_stage_update(Ls, U, out[s], F, stride(), dstride(), s0 + s, cases, 0.0));
      }
    }
    if (!trial) ALP_CUDA(launch_step_commit(cases, max_cases, stream));
    return ALP_OK;
  }

  // Path 3: the dt of the first step (signal speed, dt_finalize, which marks
  // it ready), then one persistent launch for n steps (tile_step.cuh); the
  // flags and counters of the launch start at zero, the error word is kept.
  int record_tiles(int n, bool trial) {
    if (nwork == 0 || n <= 0) return ALP_OK;
    int *dtflag = tsync + 2 + slots_max;
    ALP_CUDA(cudaMemsetAsync(tsync, 0, sizeof(int), stream));
    ALP_CUDA(cudaMemsetAsync(tsync + 2, 0, sizeof(int) * ((size_t)slots_max + 2 * max_cases), stream));
    Launch L{dim, scheme, precision, U, work, nwork, meta, BlockMeta{}, stream};
    ALP_CUDA(launch_signal_speed(L, cases, nullptr));
    ALP_CUDA(launch_dt_finalize(cases, max_cases, stream, dtflag));
    alp::TileArgs a = targs;
    a.nwork = nwork;
    a.nsteps = n;
    a.trial = trial ? 1 : 0;
    // one CTA per SM and kernel variant; CTAs that find no item left return
    ALP_CUDA(alp::tile_launch(a, tinfo[tile_variant], tgrid[tile_variant], stream));
    return ALP_OK;
  }

  // Path 3 through a CUDA graph: captured once per work list; a call with a
  // different step count updates the persistent launch's parameters in place.
  int run_tiles(int n) {
    if (!use_graph) return record_tiles(n, false);
    if (graph_dirty || !graph) {
      if (graph) {
        cudaGraphExecDestroy(graph);
        graph = nullptr;
      }
      if (tile_graph_src) {
        cudaGraphDestroy(tile_graph_src);
        tile_graph_src = nullptr;
      }
      cudaGraph_t g;
      ALP_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      int const rc = record_tiles(n, false);
      cudaError_t const ce = cudaStreamEndCapture(stream, &g);
      if (rc) {
        if (ce == cudaSuccess) cudaGraphDestroy(g);
        return rc;
      }
      if (ce != cudaSuccess) return alp::cuda_fail(ce, "cudaStreamEndCapture");
      tile_node = nullptr;
      size_t nn = 0;
      cudaGraphGetNodes(g, nullptr, &nn);
      std::vector<cudaGraphNode_t> nodes(nn);
      if (nn) cudaGraphGetNodes(g, nodes.data(), &nn);
      for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType ty;
        cudaKernelNodeParams kp;
        if (cudaGraphNodeGetType(nd, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel &&
            cudaGraphKernelNodeGetParams(nd, &kp) == cudaSuccess &&
            kp.func == tinfo[tile_variant].fn)
          tile_node = nd;
      }
      cudaError_t const ie = cudaGraphInstantiate(&graph, g, 0);
      if (ie != cudaSuccess) {
        cudaGraphDestroy(g);
        return alp::cuda_fail(ie, "cudaGraphInstantiate");
      }
      tile_graph_src = g;
      if (!tile_node) return fail(ALP_ERR_CUDA, "tile launch not found in the step graph");
      graph_dirty = false;
      tile_graph_n = n;
    } else if (n != tile_graph_n) {
      alp::TileArgs a = targs;
      a.nwork = nwork;
      a.nsteps = n;
      a.trial = 0;
      void *args[] = {&a};
      cudaKernelNodeParams kp{};
      kp.func = const_cast<void *>(tinfo[tile_variant].fn);
      kp.gridDim = dim3(tgrid[tile_variant]);
      kp.blockDim = dim3(tinfo[tile_variant].threads);
      kp.sharedMemBytes = (unsigned)tinfo[tile_variant].smem;
      kp.kernelParams = args;
      kp.extra = nullptr;
      ALP_CUDA(cudaGraphExecKernelNodeSetParams(graph, tile_node, &kp));
      tile_graph_n = n;
    }
    ALP_CUDA(cudaGraphLaunch(graph, stream));
    return ALP_OK;
  }

  // Per-stage orders of the work list for the tile path: a block is taken as
  // soon after the blocks its stage reads (itself and its face neighbours, in
  // the previous stage's order) as the order allows, so that a CTA seldom waits.
  // The cycle of stage orders is relaxed a few times so that the first stage of
  // the next step also follows the last stage of this one.
  void tile_orders(int nst, std::vector<int> &ord) const {
    static int const faces6[6] = {4, 21, 10, 15, 12, 13};
    std::vector<int> pos((size_t)capacity, 0);
    std::vector<std::vector<int>> o(nst, h_work);
    auto relax = [&](std::vector<int> const &prev, std::vector<int> &next) {
      for (size_t i = 0; i < prev.size(); ++i) pos[prev[i]] = (int)i;
      std::vector<std::pair<int, int>> key;
      key.reserve(prev.size());
      for (int b : h_work) {
        int k = pos[b];
        for (int f : faces6) {
          int const n = h_nbr26[(size_t)b * 26 + f];
          if (n >= 0) k = std::max(k, pos[n]);
        }
        key.push_back({k, pos[b]});
      }
      std::vector<int> idx(h_work.size());
      for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int)i;
      std::stable_sort(idx.begin(), idx.end(),
                       [&](int x, int y) { return key[x] < key[y]; });
      next.resize(h_work.size());
      for (size_t i = 0; i < idx.size(); ++i) next[i] = h_work[idx[i]];
    };
    for (int it = 0; it < 3; ++it)
      for (int s = 0; s < nst; ++s) relax(o[(s + nst - 1) % nst], o[s]);
    ord.clear();
    for (int s = 0; s < nst; ++s) ord.insert(ord.end(), o[s].begin(), o[s].end());
  }

  // One stage in batches of work items: the faces of batch k+1 run on `stream`
  // while the stage update of batch k runs on stream2 (the update is bound by
  // HBM, the faces by the FP64 pipe). Faces read only the stage input and the
  // updates write the stage output, so batches do not interfere; the next
  // stage waits for every update. Same kernels and arithmetic as path 1.
  int record_overlapped_stage(Launch const &Ls, double *Uout, int s) {
    int const nb = std::min(kMaxBatches, std::max(1, nwork / 64));
    int const per = (nwork + nb - 1) / nb;
    for (int k = 0, off = 0; off < nwork; ++k, off += per) {
      Launch Lk = Ls;
      Lk.work = work + off;
      Lk.nwork = std::min(per, nwork - off);
      double *Fk = F + (size_t)off * stride();
      ALP_CUDA(launch_face_flux_all(Lk, nbr26, cases, Fk, stride(), dstride(), face_threads));
      ALP_CUDA(cudaEventRecord(ev_batch[k], stream));
      ALP_CUDA(cudaStreamWaitEvent(stream2, ev_batch[k], 0));
      Lk.stream = stream2;
      ALP_CUDA(launch_stage_update(Lk, U, Uout, Fk, stride(), dstride(), s, cases, 0.0));
    }
    ALP_CUDA(cudaEventRecord(ev_join, stream2));
    ALP_CUDA(cudaStreamWaitEvent(stream, ev_join, 0));
    return ALP_OK;
  }

  // work-list offset of a case's blocks (cases are listed in id order)
  int work_offset(int cid) const {
    int off = 0;
    for (int c = 0; c < cid; ++c)
      if (case_rec[c].live) off += case_rec[c].nb;
    return off;
  }

  int rebuild_work() {
    h_work.clear();
    for (auto const &c : case_rec)
      if (c.live)
        for (int b = 0; b < c.nb; ++b) h_work.push_back(c.first + b);
    nwork = (int)h_work.size();
    if (nwork)
      ALP_CUDA(cudaMemcpyAsync(work, h_work.data(), sizeof(int) * nwork, cudaMemcpyHostToDevice,
                               stream));
    if (tile_ok && nwork) {
      tile_orders(rk2 ? 2 : 3, h_torder);
      h_case_nb.assign(max_cases, 0);
      for (int c = 0; c < max_cases; ++c)
        if (case_rec[c].live) h_case_nb[c] = case_rec[c].nb;
      ALP_CUDA(cudaMemcpyAsync(torder, h_torder.data(), sizeof(int) * h_torder.size(),
                               cudaMemcpyHostToDevice, stream));
      ALP_CUDA(cudaMemcpyAsync(tcase_nb, h_case_nb.data(), sizeof(int) * max_cases,
                               cudaMemcpyHostToDevice, stream));
      // the staging vectors must outlive the copies
      ALP_CUDA(cudaStreamSynchronize(stream));
    }
    graph_dirty = true;
    return ALP_OK;
  }

  // Reads and clears the tile path's error word: a bounded device wait that
  // ran out (the results of that launch are not trusted).
  int tile_check() {
    if (!tsync) return ALP_OK;
    int e = 0;
    ALP_CUDA(cudaMemcpyAsync(&e, tsync + 1, sizeof(int), cudaMemcpyDeviceToHost, stream));
    ALP_CUDA(cudaStreamSynchronize(stream));
    if (!e) return ALP_OK;
    ALP_CUDA(cudaMemsetAsync(tsync + 1, 0, sizeof(int), stream));
    return fail(ALP_ERR_CUDA, "tile path: a bounded device wait ran out (code " +
                                  std::to_string(e) + "); the step results are not valid");
  }

  // A range of n slots: the first free range that holds it; when the free
  // slots suffice only in total, the live cases are compacted first.
  int alloc_range(int n, int *first) {
    for (int pass = 0; pass < 2; ++pass) {
      for (auto it = free_ranges.begin(); it != free_ranges.end(); ++it) {
        if (it->second >= n) {
          *first = it->first;
          int const rest = it->second - n, start = it->first + n;
          free_ranges.erase(it);
          if (rest > 0) free_ranges[start] = rest;
          return ALP_OK;
        }
      }
      int total = 0;
      for (auto const &r : free_ranges) total += r.second;
      if (pass > 0 || total < n) break;
      if (int rc = compact()) return rc;
    }
    return fail(ALP_ERR_CAPACITY, "not enough free block slots for the case");
  }

  // Moves the live cases down, in slot order, so that they occupy slots
  // [0, used) and the free slots form one range at the end. Between steps a
  // case's state lives in U alone (B and C hold stage values within a step),
  // so U moves on the stream (in pieces no longer than the shift, so that no
  // copy overlaps itself); the block metadata and the neighbour rows move on
  // the host mirrors (neighbours are blocks of the same case, so their slots
  // shift by the same amount) and are uploaded again.
  int compact() {
    std::vector<int> order;
    for (int c = 0; c < max_cases; ++c)
      if (case_rec[c].live) order.push_back(c);
    std::sort(order.begin(), order.end(),
              [&](int a, int b) { return case_rec[a].first < case_rec[b].first; });
    size_t const blk = (size_t)ne * cells;
    int next = 0;
    for (int c : order) {
      CaseRec &r = case_rec[c];
      int const shift = r.first - next;
      if (shift > 0) {
        for (int b = 0; b < r.nb; b += shift) {
          int const n = std::min(shift, r.nb - b);
          ALP_CUDA(cudaMemcpyAsync(U + blk * (next + b), U + blk * (r.first + b),
                                   blk * n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        }
        for (int b = 0; b < r.nb; ++b) {
          h_meta[next + b] = h_meta[r.first + b];
          for (int s = 0; s < 26; ++s) {
            int const nb = h_nbr26[(size_t)(r.first + b) * 26 + s];
            h_nbr26[(size_t)(next + b) * 26 + s] = nb < 0 ? nb : nb - shift;
          }
        }
        r.first = next;
      }
      next += r.nb;
    }
    if (next > 0) {
      ALP_CUDA(cudaMemcpyAsync(meta, h_meta.data(), sizeof(BlockMeta) * next,
                               cudaMemcpyHostToDevice, stream));
      ALP_CUDA(cudaMemcpyAsync(nbr26, h_nbr26.data(), sizeof(int) * 26 * (size_t)next,
                               cudaMemcpyHostToDevice, stream));
      // the host mirrors are changed again by later calls: the copies finish first
      ALP_CUDA(cudaStreamSynchronize(stream));
    }
    free_ranges.clear();
    if (next < capacity) free_ranges[next] = capacity - next;
    ++compactions;
    return rebuild_work();
  }

  void free_range(int first, int n) {
    auto it = free_ranges.emplace(first, n).first;
    auto nx = std::next(it);
    if (nx != free_ranges.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_ranges.erase(nx);
    }
    if (it != free_ranges.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_ranges.erase(it);
      }
    }
  }

  // ---- elastic engines (alp_engine_create_elastic): the block pools U, UB,
  // UC and the scratch F, R are elastic arrays; `capacity` is the number of
  // slots backed by memory, slots_max the reservation.
  bool elastic = false;
  alp::ElasticArray ea[5];  // U, UB, UC, F, R

  size_t slot_bytes(int k) const {
    size_t const blk = (size_t)ne * cells * sizeof(double);
    if (k < 3) return blk;
    if (k == 3) return (size_t)stride() * sizeof(double);
    return (size_t)ne * (dim == 3 ? 4096 : (dim == 2 ? 256 : 16)) * sizeof(double);
  }
  // device bytes the elastic arrays take when n slots are backed
  size_t elastic_bytes(int n) const {
    size_t const q = alp::elastic_chunk_bytes();
    size_t b = 0;
    for (int k = 0; k < 5; ++k) b += ((size_t)n * slot_bytes(k) + q - 1) / q * q;
    return b;
  }
  size_t mapped_bytes() const {
    size_t b = 0;
    for (auto const &a : ea) b += a.mapped;
    return b;
  }
  // one past the highest slot a live case holds
  int used_slots() const {
    int top = 0;
    for (auto const &c : case_rec)
      if (c.live) top = std::max(top, c.first + c.nb);
    return top;
  }
  // Backs exactly n slots (compacting the cases first when they reach beyond
  // n); refused when the cases need more than n slots.
  int set_capacity(int n) {
    if (!elastic) return fail(ALP_ERR_INVALID, "the engine's pools are not elastic");
    if (n < 0 || n > slots_max) return fail(ALP_ERR_CAPACITY, "beyond the engine's reservation");
    if (used_slots() > n) {
      if (int rc = compact()) return rc;
      if (used_slots() > n) return fail(ALP_ERR_CAPACITY, "the resident cases need more slots");
    }
    // nothing in flight may touch a range that is unmapped
    ALP_CUDA(cudaStreamSynchronize(stream));
    ALP_CUDA(cudaStreamSynchronize(stream2));
    int const old = capacity;
    for (int k = 0; k < 5; ++k) {
      if (int rc = alp::elastic_resize(ea[k], (size_t)n * slot_bytes(k))) {
        // keep every array at the smaller of the two sizes, as `capacity` says
        int const keep = std::min(old, n);
        for (int j = 0; j < 5; ++j) alp::elastic_resize(ea[j], (size_t)keep * slot_bytes(j));
        set_free_tail(keep);
        return rc;
      }
    }
    set_free_tail(n);
    return ALP_OK;
  }
  // capacity becomes n: free ranges end at n, slots from the old capacity up
  // to n are free
  void set_free_tail(int n) {
    if (n < capacity) {
      for (auto it = free_ranges.begin(); it != free_ranges.end();) {
        if (it->first >= n) {
          it = free_ranges.erase(it);
        } else {
          if (it->first + it->second > n) it->second = n - it->first;
          ++it;
        }
      }
      capacity = n;
    } else if (n > capacity) {
      int const old = capacity;
      capacity = n;
      free_range(old, n - old);
    }
  }

  void release() {
    if (graph) cudaGraphExecDestroy(graph);
    if (tile_graph_src) cudaGraphDestroy(tile_graph_src);
    if (elastic) {
      if (stream) cudaStreamSynchronize(stream);
      for (auto &a : ea) alp::elastic_release(a);
    } else {
      cudaFree(U);
      cudaFree(UB);
      cudaFree(UC);
      cudaFree(F);
      cudaFree(R);
    }
    cudaFree(meta);
    cudaFree(nbr26);
    cudaFree(work);
    cudaFree(cases);
    cudaFree(glf);
    cudaFree(tsync);
    cudaFree(torder);
    cudaFree(tcase_nb);
    for (cudaEvent_t &ev : ev_batch)
      if (ev) cudaEventDestroy(ev);
    if (ev_join) cudaEventDestroy(ev_join);
    if (stream2) cudaStreamDestroy(stream2);
    if (stream) cudaStreamDestroy(stream);
  }
};


namespace alp {
// Neighbour table (26 directions, x slowest; -1 = domain face) of a regular
// nx x ny x nz block grid in C order, periodic per dimension.
std::vector<int> regular_grid_neighbours(int dim, int const n[3], int const periodic[3]);
// Adds a case's blocks, metadata and state record; returns its id and first slot.
int engine_add_case_core(alp_engine *e, alp_material const *mat, double cell_size, double cfl,
                         double t0, double t_end, int max_steps, int nb, int const *nbr26,
                         int *case_id, int *first);
// Copies the device case table to host.
int engine_case_states(alp_engine *e, std::vector<CaseState> &out);
// Holds (1) or releases (0) a case: a held case takes no steps (dt 0).
int engine_set_hold(alp_engine *e, int case_id, int hold);
// Compiled scheme id and precision of a selection (ALP_ERR_INVALID otherwise).
int scheme_id(alp_scheme const *s, int *id, int *precision);
// Stencil / Riemann / signal-speed / splitting choices of a validated selection
// (the fields the selected convective term solver does not use are default).
SchemeOptions scheme_options(alp_scheme const *s);
// Rejects gamma <= 1 and negative background pressure.
int check_material(alp_material const *m);
// Block metadata of one material and cell size.
BlockMeta meta_of(alp_material const *m, double cell_size, int case_id);
}  // namespace alp
