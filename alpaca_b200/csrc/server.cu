// Request loop of the serving form (alp_serve, include/alpaca_b200.h).
//
// Continuous batching over the engines: cases arrive on a wall-clock
// schedule, are admitted as soon as their blocks fit into the engine pool of
// their dimension (FIFO order with backfill: a later request that fits is
// admitted while an earlier one waits for room), advance together in the
// engine's batched step (one launch per kernel for all resident blocks of all
// cases, each case with its own dt), and leave the pool when their end time or
// step budget is reached. The 2D and 3D engines step on their own streams, so
// their work overlaps on the device. Their pools share one HBM budget: each
// engine is elastic (alp_engine_create_elastic), its address range reserved
// for the whole budget, and a request that does not fit grows its engine's
// backed slots while the budget allows, after the other engines have given
// back the slots their cases no longer hold (moving their cases together).
// Memory is mapped and unmapped only then, never between the polls of a
// steady batch. With shortest_first, only the
// resident cases with the least remaining work (cells x steps left) step, up to
// step_set_cells cells together, and the others are held (they keep their
// state and take no steps): the GPU stays busy while short cases finish first.
// Holding changes no arithmetic, so every case gets the same bits either way.
#include <algorithm>
#include <chrono>
#include <deque>
#include <memory>
#include <thread>
#include <vector>

#include <nvtx3/nvtx3.hpp>
#include <unistd.h>

#include "engine.hpp"

namespace {

using Clock = std::chrono::steady_clock;

struct Active {
  int req;
};

struct DimPool {
  alp_engine *eng = nullptr;
  std::vector<int> req_of_case;  // case id -> request index (-1 free)
  std::vector<int> held;         // case id -> hold flag on the device
  std::vector<CaseState> states; // last case records read back
  int active = 0;
};

}  // namespace

extern "C" int alp_serve(const alp_server_config *cfg, const alp_request *reqs, int n,
                         alp_result *results, double *makespan_s) {
  using namespace alp;
  if (!cfg || (n > 0 && (!reqs || !results))) return fail(ALP_ERR_INVALID, "null argument");
  if (cfg->steps_per_poll <= 0 || cfg->max_cases <= 0)
    return fail(ALP_ERR_INVALID, "steps_per_poll and max_cases must be positive");
  if (cfg->shortest_first && !(cfg->step_set_cells > 0.0))
    return fail(ALP_ERR_INVALID, "step_set_cells must be positive");
  bool need[4] = {false, false, false, false};
  for (int i = 0; i < n; ++i) {
    if (reqs[i].dim < 1 || reqs[i].dim > 3) return fail(ALP_ERR_INVALID, "request dim");
    need[reqs[i].dim] = true;
  }
  nvtx3::scoped_range range{"alp_serve"};  // its engine steps show as alp_engine_step
  // one budget for the pools of every dimension: each engine may grow to all
  // of it, and holds memory only for the block slots it backs
  DimPool pool[4];
  size_t per_block[4] = {0, 0, 0, 0};
  auto cleanup = [&]() {
    for (auto &p : pool)
      if (p.eng) alp_engine_destroy(p.eng);
  };
  for (int d = 1; d <= 3; ++d) {
    if (!need[d]) continue;
    per_block[d] = alp_engine_bytes(d, 1, 0);
    size_t const cap = cfg->hbm_budget_bytes / per_block[d];
    if (cap < 1) {
      cleanup();
      return fail(ALP_ERR_CAPACITY, "HBM budget below one block");
    }
    if (int rc = alp_engine_create_elastic(d, &cfg->scheme, (int)std::min<size_t>(cap, 1 << 30),
                                           cfg->max_cases, &pool[d].eng)) {
      cleanup();
      return rc;
    }
    pool[d].req_of_case.assign(cfg->max_cases, -1);
    pool[d].held.assign(cfg->max_cases, 0);
    pool[d].states.assign(cfg->max_cases, CaseState{});
  }
  auto blocks_used = [&](int d) {
    int u = 0;
    alp_engine_capacity(pool[d].eng, nullptr, &u, nullptr);
    return u;
  };
  auto budget_used = [&]() {
    size_t b = 0;
    for (int d = 1; d <= 3; ++d)
      if (pool[d].eng) b += (size_t)pool[d].eng->capacity * per_block[d];
    return b;
  };
  // Backs enough slots in dimension d's engine for nb more blocks, within the
  // budget; first the other engines give back what their cases do not hold.
  // ALP_ERR_CAPACITY when the budget cannot hold it now.
  auto make_room = [&](int d, int nb) -> int {
    alp_engine *e = pool[d].eng;
    int const want = blocks_used(d) + nb;
    if (want <= e->capacity) return e->set_capacity(e->capacity);  // compacts if needed
    size_t const extra = (size_t)(want - e->capacity) * per_block[d];
    if (budget_used() + extra > cfg->hbm_budget_bytes)
      for (int o = 1; o <= 3; ++o)
        if (o != d && pool[o].eng && pool[o].eng->capacity > blocks_used(o))
          if (int rc = pool[o].eng->set_capacity(blocks_used(o))) return rc;
    if (budget_used() + extra > cfg->hbm_budget_bytes)
      return fail(ALP_ERR_CAPACITY, "the HBM budget is held by resident cases");
    return e->set_capacity(want);
  };


  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return reqs[a].arrival_s < reqs[b].arrival_s; });
  std::deque<int> queue;
  int next = 0, done = 0;
  std::vector<char> ended(n, 0);  // requests with a final result
  Clock::time_point const t0 = Clock::now();
  auto elapsed = [&]() { return std::chrono::duration<double>(Clock::now() - t0).count(); };
  int rc_all = ALP_OK;

  // A clean stop on request: once the abort file exists, every unfinished
  // request ends with ALP_ABORTED (resident cases with their state so far).
  auto abort_requested = [&]() {
    return done < n && cfg->abort_file && access(cfg->abort_file, F_OK) == 0;
  };
  auto abort_now = [&]() -> int {
    double const t_now = elapsed();
    for (auto &p : pool) {
      if (p.active == 0) continue;
      for (int c = 0; c < cfg->max_cases; ++c) {
        int const ri = p.req_of_case[c];
        if (ri < 0) continue;
        ended[ri] = 1;
        double t = 0.0;
        int st = 0;
        int const grc = alp_engine_get_case(p.eng, c, reqs[ri].h_result, &t, &st);
        if (grc != ALP_OK && grc != ALP_ERR_NUMERIC) {
          cleanup();
          return grc;
        }
        alp_result &out = results[ri];
        out.finished_s = t_now;
        out.t = t;
        out.steps = st;
        out.status = ALP_ABORTED;
      }
    }
    for (int i = 0; i < n; ++i)
      if (!ended[i]) results[i] = alp_result{reqs[i].arrival_s, -1.0, t_now, 0.0, 0, ALP_ABORTED};
    if (makespan_s) *makespan_s = t_now;
    cleanup();
    return fail(ALP_ABORTED, "stopped: the abort file exists");
  };

  while (done < n) {
    double const now = elapsed();
    while (next < n && reqs[order[next]].arrival_s <= now) queue.push_back(order[next++]);

    // admission: FIFO with backfill; one-at-a-time admits only into an idle GPU
    int total_active = 0;
    for (auto &p : pool) total_active += p.active;
    for (auto it = queue.begin(); it != queue.end();) {
      if (cfg->one_at_a_time && total_active > 0) break;
      alp_request const &r = reqs[*it];
      DimPool &p = pool[r.dim];
      int cid = -1;
      bool const unit = r.units.density == 0.0 && r.units.velocity == 0.0 && r.units.length == 0.0;
      auto add = [&]() {
        return r.ic_type == ALP_IC_PROGRAM
                   ? alp_engine_add_case_expr(p.eng, &r.material, r.cell_size, r.cfl, 0.0,
                                              r.t_end, r.max_steps, r.nblocks, r.periodic,
                                              r.origin, unit ? nullptr : &r.units, r.program,
                                              &cid)
                   : alp_engine_add_case_ic(p.eng, &r.material, r.cell_size, r.cfl, 0.0, r.t_end,
                                            r.max_steps, r.nblocks, r.periodic, r.ic_type,
                                            r.ic_params, r.n_params, &cid);
      };
      int rc = add();
      if (rc == ALP_ERR_CAPACITY && p.active < cfg->max_cases) {
        // the blocks of the request against the budget shared by all engines
        long long const nb = (long long)r.nblocks[0] * (r.dim > 1 ? r.nblocks[1] : 1) *
                             (r.dim > 2 ? r.nblocks[2] : 1);
        int const room = nb * (long long)per_block[r.dim] <= (long long)cfg->hbm_budget_bytes
                             ? make_room(r.dim, (int)nb)
                             : ALP_ERR_CAPACITY;
        if (room == ALP_OK) rc = add();
        else if (room != ALP_ERR_CAPACITY) rc = room;
      }
      if (rc == ALP_OK) {
        p.req_of_case[cid] = *it;
        p.held[cid] = 0;
        p.states[cid] = CaseState{};
        ++p.active;
        ++total_active;
        results[*it].arrival_s = r.arrival_s;
        results[*it].admitted_s = elapsed();
        it = queue.erase(it);
      } else if (rc == ALP_ERR_CAPACITY) {
        if (total_active == 0 && it == queue.begin()) {
          // does not fit even into an empty pool: fail the request
          results[*it] = alp_result{r.arrival_s, now, now, 0.0, 0, ALP_ERR_CAPACITY};
          ended[*it] = 1;
          ++done;
          it = queue.erase(it);
          rc_all = ALP_ERR_CAPACITY;
        } else {
          ++it;
        }
      } else {
        cleanup();
        return rc;
      }
    }

    if (total_active == 0) {
      // nothing resident: the file is checked while the loop waits for arrivals
      if (abort_requested()) return abort_now();
      if (next < n && queue.empty()) {
        double const wait = reqs[order[next]].arrival_s - elapsed();
        if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 1e-3)));
      }
      continue;
    }

    // shortest remaining work first: release the shortest cases up to the
    // step-set size, hold the rest
    if (cfg->shortest_first && !cfg->one_at_a_time) {
      struct Cand {
        double work, cells;
        int dim, cid, req;
      };
      std::vector<Cand> cands;
      for (int d = 1; d <= 3; ++d) {
        DimPool &p = pool[d];
        if (!p.eng) continue;
        for (int c = 0; c < cfg->max_cases; ++c) {
          int const ri = p.req_of_case[c];
          if (ri < 0) continue;
          alp_request const &r = reqs[ri];
          double cells = 1.0;
          for (int k = 0; k < d; ++k) cells *= 16.0 * r.nblocks[k];
          double const left = r.max_steps > 0 ? double(r.max_steps - p.states[c].steps) : 1e30;
          cands.push_back({cells * left, cells, d, c, ri});
        }
      }
      std::stable_sort(cands.begin(), cands.end(), [](Cand const &a, Cand const &b) {
        return a.work < b.work || (a.work == b.work && a.req < b.req);
      });
      double acc = 0.0;
      for (Cand const &c : cands) {
        int const hold = acc >= cfg->step_set_cells ? 1 : 0;
        if (!hold) acc += c.cells;
        DimPool &p = pool[c.dim];
        if (p.held[c.cid] != hold) {
          if (int rc = engine_set_hold(p.eng, c.cid, hold)) {
            cleanup();
            return rc;
          }
          p.held[c.cid] = hold;
        }
      }
    }

    // advance every pool with resident cases (asynchronous, one stream each)
    for (auto &p : pool)
      if (p.active > 0) {
        if (int rc = alp_engine_step(p.eng, cfg->steps_per_poll)) {
          cleanup();
          return rc;
        }
      }
    // retire finished cases
    for (auto &p : pool) {
      if (p.active == 0) continue;
      if (int rc = engine_case_states(p.eng, p.states)) {
        cleanup();
        return rc;
      }
      std::vector<CaseState> const &states = p.states;
      double const t_now = elapsed();
      for (int c = 0; c < cfg->max_cases; ++c) {
        int const ri = p.req_of_case[c];
        if (ri < 0) continue;
        CaseState const &s = states[c];
        bool const finished = !(s.t < s.t_end) || (s.max_steps > 0 && s.steps >= s.max_steps) ||
                              s.status != 0;
        if (!finished) continue;
        alp_request const &r = reqs[ri];
        alp_result &out = results[ri];
        out.finished_s = t_now;
        out.t = s.t;
        out.steps = s.steps;
        out.status = s.status ? ALP_ERR_NUMERIC : ALP_OK;
        if (r.h_result) {
          double t;
          int st;
          int const grc = alp_engine_get_case(p.eng, c, r.h_result, &t, &st);
          if (grc != ALP_OK && grc != ALP_ERR_NUMERIC) {
            cleanup();
            return grc;
          }
        }
        if (int rc = alp_engine_remove_case(p.eng, c)) {
          cleanup();
          return rc;
        }
        p.req_of_case[c] = -1;
        ended[ri] = 1;
        --p.active;
        ++done;
      }
    }
    // after every poll, as the reference checks its ABORTFILE after every step
    if (abort_requested()) return abort_now();
  }
  if (makespan_s) *makespan_s = elapsed();
  cleanup();
  return rc_all;
}
