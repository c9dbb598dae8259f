// C ABI (include/alpaca_b200.h): stateless drop-in calls and the engine that
// keeps cases device-resident and replays its step as a CUDA graph.
#include <cuda_runtime.h>
#include <nvtx3/nvtx3.hpp>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "../../include/alpaca_b200.h"
#include "kernels.cuh"

namespace alp {
thread_local std::string g_last_error;

int fail(int code, std::string const &msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, char const *where) {
  return fail(ALP_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
}  // namespace alp

using namespace alp;

#include "engine.hpp"

namespace {

int faces_of(int dim) {
  return 17 * (dim > 1 ? 17 : 2) * (dim > 2 ? 17 : 2);
}
int cells_of(int dim) { return 24 * (dim > 1 ? 24 : 1) * (dim > 2 ? 24 : 1); }
int interior_of(int dim) { return 16 * (dim > 1 ? 16 : 1) * (dim > 2 ? 16 : 1); }

}  // namespace

namespace alp {

int scheme_id(alp_scheme const *s, int *id, int *precision) {
  if (!s) return fail(ALP_ERR_INVALID, "scheme is null");
  int const st = s->reconstruction_stencil;
  if (st != ST_WENO5 && st != ST_WENO5Z && st != ST_TENO5 && st != ST_WENO3 &&
      st != ST_FIRST_ORDER && st != ST_WENO7)
    return fail(ALP_ERR_INVALID,
                "compiled ReconstructionStencils: FirstOrder, WENO3, WENO5, WENO5Z, TENO5, WENO7");
  if (s->time_integrator != ALP_RK3 && s->time_integrator != ALP_RK2)
    return fail(ALP_ERR_INVALID, "TimeIntegrators must be RK2 or RK3");
  if (s->precision != ALP_FP64 && s->precision != ALP_FP32_FLUX)
    return fail(ALP_ERR_INVALID, "precision must be ALP_FP64 or ALP_FP32_FLUX");
  *precision = s->precision;
  if (s->convective_term_solver == ALP_FINITE_VOLUME) {
    if (s->riemann_solver < RS_HLLC || s->riemann_solver > RS_HLL)
      return fail(ALP_ERR_INVALID, "RiemannSolvers must be Hllc, Hllc_LM or Hll");
    if (s->signal_speed < SS_EINFELDT || s->signal_speed > SS_ARITHMETIC)
      return fail(ALP_ERR_INVALID, "SignalSpeed must be Einfeldt, Davis, Toro or Arithmetic");
    if (s->state_reconstruction == ALP_RECON_CHARACTERISTIC) *id = FV_CHAR;
    else if (s->state_reconstruction == ALP_RECON_PRIMITIVE) *id = FV_PRIM;
    else return fail(ALP_ERR_INVALID, "FiniteVolume needs Primitive or Characteristic reconstruction");
  } else if (s->convective_term_solver == ALP_FLUX_SPLITTING) {
    int const fs = s->flux_splitting;
    if (fs != FSP_ROE && fs != FSP_LLF && fs != FSP_GLF && fs != FSP_ROE_M && fs != FSP_LLF_M)
      return fail(ALP_ERR_INVALID,
                  "FluxSplitting must be Roe, LocalLaxFriedrichs, GlobalLaxFriedrichs, Roe_M or "
                  "LocalLaxFriedrichs_M");
    *id = FS_ROE;
  } else {
    return fail(ALP_ERR_INVALID, "unknown convective_term_solver");
  }
  if (*precision == ALP_FP32_FLUX && !scheme_options(s).is_default())
    return fail(ALP_ERR_INVALID,
                "ALP_FP32_FLUX is compiled for WENO5 + HLLC/Einfeldt and Roe splitting only");
  return ALP_OK;
}

SchemeOptions scheme_options(alp_scheme const *s) {
  SchemeOptions o;
  o.stencil = s->reconstruction_stencil;
  if (s->convective_term_solver == ALP_FINITE_VOLUME) {
    o.riemann = s->riemann_solver;
    o.signal = s->signal_speed;
  } else {
    o.splitting = s->flux_splitting;
  }
  return o;
}

int check_material(alp_material const *m) {
  if (!m) return fail(ALP_ERR_INVALID, "material is null");
  if (!(m->gamma > 1.0)) return fail(ALP_ERR_INVALID, "gamma must exceed 1");
  if (!(m->background_pressure >= 0.0)) return fail(ALP_ERR_INVALID, "background pressure < 0");
  return ALP_OK;
}

BlockMeta meta_of(alp_material const *m, double cell_size, int case_id) {
  BlockMeta b;
  b.cell_size = cell_size;
  b.gamma = m->gamma;
  b.B = m->background_pressure;
  b.safe = m->safe ? 1 : 0;
  b.case_id = case_id;
  return b;
}

}  // namespace alp

namespace {
// GlobalLaxFriedrichs in the stateless calls: the maxima over the call's blocks
// (all leaves handed to one call, as ComputeRightHandSide takes them over all
// leaves) in the library's slot, before the fluxes.
int stateless_glf(Launch &L) {
  if (L.scheme != FS_ROE || L.opt.splitting != FSP_GLF || L.nwork <= 0) return ALP_OK;
  unsigned long long *slot = glf_stateless_slot();
  if (!slot) return fail(ALP_ERR_CUDA, "GlobalLaxFriedrichs: no device slot");
  ALP_CUDA(launch_glf_maxima(L, slot, 1));
  L.glf = slot;
  return ALP_OK;
}
}  // namespace

extern "C" {

const char *alp_version(void) { return "alpaca_b200 0.1 (sm_100a)"; }
const char *alp_last_error(void) { return g_last_error.c_str(); }

void alp_scheme_default(alp_scheme *s) {
  s->convective_term_solver = ALP_FINITE_VOLUME;
  s->state_reconstruction = ALP_RECON_CHARACTERISTIC;
  s->reconstruction_stencil = ALP_STENCIL_WENO5;
  s->riemann_solver = ALP_RIEMANN_HLLC;
  s->signal_speed = ALP_SIGNAL_SPEED_EINFELDT;
  s->flux_splitting = ALP_FLUX_SPLITTING_ROE;
  s->time_integrator = ALP_RK3;
  s->precision = ALP_FP64;
}

int alp_convective_fluxes(int dim, const alp_scheme *scheme, const alp_material *mat,
                          const double *d_blocks, int nb, double cell_size, double *d_fx,
                          double *d_fy, double *d_fz, alp_stream_t stream) {
  if (dim < 1 || dim > 3) return fail(ALP_ERR_INVALID, "dim must be 1, 2 or 3");
  int sid, prec;
  if (int rc = scheme_id(scheme, &sid, &prec)) return rc;
  if (int rc = check_material(mat)) return rc;
  if (nb < 0 || (nb > 0 && !d_blocks)) return fail(ALP_ERR_INVALID, "bad block buffer");
  double *F[3] = {d_fx, d_fy, d_fz};
  for (int d = 0; d < dim; ++d)
    if (!F[d] && nb > 0) return fail(ALP_ERR_INVALID, "flux buffer is null");
  Launch L{dim, sid, prec, const_cast<double *>(d_blocks), nullptr, nb, nullptr,
           meta_of(mat, cell_size, 0), (cudaStream_t)stream};
  L.opt = scheme_options(scheme);
  if (int rc = stateless_glf(L)) return rc;
  long long const stride = (long long)(dim + 2) * faces_of(dim);
  for (int d = 0; d < dim; ++d) ALP_CUDA(launch_face_flux(L, d, F[d], stride, true));
  return ALP_OK;
}

size_t alp_space_rhs_workspace_size(int dim, int nb) {
  if (dim < 1 || dim > 3 || nb < 0) return 0;
  return (size_t)nb * dim * (dim + 2) * faces_of(dim) * sizeof(double);
}

int alp_space_rhs(int dim, const alp_scheme *scheme, const alp_material *mat,
                  const double *d_blocks, int nb, double cell_size, double *d_rhs,
                  void *d_workspace, size_t workspace_bytes, alp_stream_t stream) {
  if (dim < 1 || dim > 3) return fail(ALP_ERR_INVALID, "dim must be 1, 2 or 3");
  int sid, prec;
  if (int rc = scheme_id(scheme, &sid, &prec)) return rc;
  if (int rc = check_material(mat)) return rc;
  if (nb <= 0) return ALP_OK;
  if (!d_blocks || !d_rhs) return fail(ALP_ERR_INVALID, "null buffer");
  if (!d_workspace || workspace_bytes < alp_space_rhs_workspace_size(dim, nb))
    return fail(ALP_ERR_INVALID, "workspace too small");
  double *F = static_cast<double *>(d_workspace);
  Launch L{dim, sid, prec, const_cast<double *>(d_blocks), nullptr, nb, nullptr,
           meta_of(mat, cell_size, 0), (cudaStream_t)stream};
  L.opt = scheme_options(scheme);
  if (int rc = stateless_glf(L)) return rc;
  long long const dstride = (long long)(dim + 2) * faces_of(dim);
  long long const stride = dstride * dim;
  for (int d = 0; d < dim; ++d) ALP_CUDA(launch_face_flux(L, d, F + d * dstride, stride, false));
  ALP_CUDA(launch_divergence(L, F, stride, dstride, d_rhs));
  return ALP_OK;
}

int alp_prime_states(int dim, const alp_material *mat, const double *d_blocks, int nb,
                     double *d_primes, alp_stream_t stream) {
  if (dim < 1 || dim > 3) return fail(ALP_ERR_INVALID, "dim must be 1, 2 or 3");
  if (int rc = check_material(mat)) return rc;
  if (nb <= 0) return ALP_OK;
  if (!d_blocks || !d_primes) return fail(ALP_ERR_INVALID, "null buffer");
  Launch L{dim, 0, 0, const_cast<double *>(d_blocks), nullptr, nb, nullptr,
           meta_of(mat, 1.0, 0), (cudaStream_t)stream};
  ALP_CUDA(launch_prime_states(L, d_primes));
  return ALP_OK;
}

int alp_halo_update(int dim, double *d_blocks, int nb, int nfields, const int *d_nbr26, int mode,
                    alp_stream_t stream) {
  if (dim < 1 || dim > 3) return fail(ALP_ERR_INVALID, "dim must be 1, 2 or 3");
  if (mode != ALP_HALO_ALL && mode != ALP_HALO_FACES) return fail(ALP_ERR_INVALID, "bad mode");
  if (nfields < 1) return fail(ALP_ERR_INVALID, "nfields < 1");
  if (nb <= 0) return ALP_OK;
  if (!d_blocks || !d_nbr26) return fail(ALP_ERR_INVALID, "null buffer");
  BlockMeta def{};
  Launch L{dim, 0, 0, d_blocks, nullptr, nb, nullptr, def, (cudaStream_t)stream};
  ALP_CUDA(launch_halo(L, d_nbr26, mode == ALP_HALO_FACES, nfields, nullptr));
  return ALP_OK;
}

int alp_timestep_size(int dim, const alp_material *mat, const double *d_blocks, int nb,
                      double cell_size, double cfl, double t, double t_end, double *h_dt,
                      void *d_workspace, alp_stream_t stream) {
  if (dim < 1 || dim > 3) return fail(ALP_ERR_INVALID, "dim must be 1, 2 or 3");
  if (int rc = check_material(mat)) return rc;
  if (!h_dt) return fail(ALP_ERR_INVALID, "h_dt is null");
  unsigned long long bits = 0ull;
  if (nb > 0) {
    if (!d_workspace) return fail(ALP_ERR_INVALID, "workspace is null");
    auto *d_bits = static_cast<unsigned long long *>(d_workspace);
    ALP_CUDA(cudaMemsetAsync(d_bits, 0, sizeof(unsigned long long), (cudaStream_t)stream));
    Launch L{dim, 0, 0, const_cast<double *>(d_blocks), nullptr, nb, nullptr,
             meta_of(mat, cell_size, 0), (cudaStream_t)stream};
    ALP_CUDA(launch_signal_speed(L, nullptr, d_bits));
    ALP_CUDA(cudaMemcpyAsync(&bits, d_bits, sizeof(bits), cudaMemcpyDeviceToHost,
                             (cudaStream_t)stream));
    ALP_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  }
  double smax;
  std::memcpy(&smax, &bits, sizeof(smax));
  // modular_algorithm_assembler.cpp:1932, 1961-1982
  double const dt = smax / cell_size;
  double local = dt == 0.0 ? 1.7976931348623157e308 : cfl / dt;
  if (t + local > t_end) local = std::max(t_end - t, 0.0);
  *h_dt = local;
  return ALP_OK;
}

int alp_rk3_stage(int dim, double *d_blocks, double *d_initial, const double *d_rhs, int nb,
                  int stage, double dt, alp_stream_t stream) {
  if (dim < 1 || dim > 3) return fail(ALP_ERR_INVALID, "dim must be 1, 2 or 3");
  if (stage < 0 || stage > 2) return fail(ALP_ERR_INVALID, "stage must be 0, 1 or 2");
  if (nb <= 0) return ALP_OK;
  if (!d_blocks || !d_initial || !d_rhs) return fail(ALP_ERR_INVALID, "null buffer");
  ALP_CUDA(launch_rk_stage_rhs(dim, d_blocks, d_initial, d_rhs, nb, stage, dt,
                               (cudaStream_t)stream));
  return ALP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// engine
// ---------------------------------------------------------------------------

namespace alp {

std::vector<int> regular_grid_neighbours(int dim, int const n[3], int const periodic[3]) {
  int const nb = n[0] * n[1] * n[2];
  std::vector<int> nbr((size_t)nb * 26, -1);
  for (int b = 0; b < nb; ++b) {
    int const c[3] = {b / (n[1] * n[2]), (b / n[2]) % n[1], b % n[2]};
    int slot = 0;
    for (int o = 0; o < 27; ++o) {
      if (o == 13) continue;
      int const off[3] = {o / 9 - 1, (o / 3) % 3 - 1, o % 3 - 1};
      int q[3] = {c[0], c[1], c[2]};
      bool ok = true, wall = false;
      int const nonzero = (off[0] != 0) + (off[1] != 0) + (off[2] != 0);
      for (int d = 0; d < 3 && ok; ++d) {
        if (off[d] == 0) continue;
        if (d >= dim) {
          ok = false;
          break;
        }
        q[d] += off[d];
        if (q[d] < 0 || q[d] >= n[d]) {
          if (periodic[d] == ALP_BOUNDARY_SYMMETRY) {
            wall = nonzero == 1;  // face slots only (edges and corners stay -1)
            ok = false;
          } else if (periodic[d]) {
            q[d] = (q[d] + n[d]) % n[d];
          } else {
            ok = false;
          }
        }
      }
      if (ok) nbr[(size_t)b * 26 + slot] = (q[0] * n[1] + q[1]) * n[2] + q[2];
      else if (wall) nbr[(size_t)b * 26 + slot] = -2;
      ++slot;
    }
  }
  return nbr;
}

int engine_add_case_core(alp_engine *e, alp_material const *mat, double cell_size, double cfl,
                         double t0, double t_end, int max_steps, int nb, int const *h_nbr26,
                         int *case_id, int *first_out) {
  if (int rc = check_material(mat)) return rc;
  if (!(cell_size > 0.0) || !(cfl > 0.0)) return fail(ALP_ERR_INVALID, "bad cell size / cfl");
  for (size_t i = 0; i < (size_t)nb * 26; ++i) {
    // -2 (symmetry wall) only in the six face slots 4, 10, 12, 13, 15, 21
    int const s = (int)(i % 26);
    bool const face = s == 4 || s == 10 || s == 12 || s == 13 || s == 15 || s == 21;
    if (h_nbr26[i] < (face ? -2 : -1) || h_nbr26[i] >= nb)
      return fail(ALP_ERR_INVALID, "neighbour out of range");
  }
  int cid = -1;
  for (int c = 0; c < e->max_cases; ++c)
    if (!e->case_rec[c].live) {
      cid = c;
      break;
    }
  if (cid < 0) return fail(ALP_ERR_CAPACITY, "case table full");
  int first;
  if (int rc = e->alloc_range(nb, &first)) return rc;
  e->case_rec[cid] = {true, first, nb, *mat, cell_size};
  for (int b = 0; b < nb; ++b) {
    e->h_meta[first + b] = meta_of(mat, cell_size, cid);
    for (int s = 0; s < 26; ++s) {
      int const n = h_nbr26[(size_t)b * 26 + s];
      e->h_nbr26[(size_t)(first + b) * 26 + s] = n < 0 ? n : first + n;  // -1 / -2 kept
    }
  }
  ALP_CUDA(cudaMemcpyAsync(e->meta + first, e->h_meta.data() + first, sizeof(BlockMeta) * nb,
                           cudaMemcpyHostToDevice, e->stream));
  ALP_CUDA(cudaMemcpyAsync(e->nbr26 + (size_t)first * 26, e->h_nbr26.data() + (size_t)first * 26,
                           sizeof(int) * 26 * nb, cudaMemcpyHostToDevice, e->stream));
  CaseState cs{};
  cs.t = t0;
  cs.t_end = t_end;
  cs.cfl = cfl;
  cs.dt = 0.0;
  cs.h_min = cell_size;
  cs.smax_bits = 0ull;
  cs.steps = 0;
  cs.max_steps = max_steps;
  cs.status = 0;
  e->h_case_state[cid] = cs;
  ALP_CUDA(cudaMemcpyAsync(e->cases + cid, &e->h_case_state[cid], sizeof(cs),
                           cudaMemcpyHostToDevice, e->stream));
  if (int rc = e->rebuild_work()) return rc;
  *case_id = cid;
  *first_out = first;
  return ALP_OK;
}

int engine_case_states(alp_engine *e, std::vector<CaseState> &out) {
  out.resize(e->max_cases);
  ALP_CUDA(cudaMemcpyAsync(out.data(), e->cases, sizeof(CaseState) * e->max_cases,
                           cudaMemcpyDeviceToHost, e->stream));
  ALP_CUDA(cudaStreamSynchronize(e->stream));
  return e->tile_check();
}

int engine_set_hold(alp_engine *e, int case_id, int hold) {
  // the staging record keeps the source alive until the copy has run
  e->h_case_state[case_id].hold = hold;
  ALP_CUDA(cudaMemcpyAsync(&e->cases[case_id].hold, &e->h_case_state[case_id].hold, sizeof(int),
                           cudaMemcpyHostToDevice, e->stream));
  return ALP_OK;
}

}  // namespace alp

namespace {

// Engine with block tables for capacity_blocks slots. Fixed: the pools and
// scratch are allocated for all of them. Elastic: they are reserved for all of
// them and backed by nothing until alp_engine_reserve (no fused tile path).
int engine_create(int dim, const alp_scheme *scheme, int capacity_blocks, int max_cases,
                  bool elastic, alp_engine **out) {
  if (!out) return fail(ALP_ERR_INVALID, "out is null");
  *out = nullptr;
  if (dim < 1 || dim > 3) return fail(ALP_ERR_INVALID, "dim must be 1, 2 or 3");
  if (capacity_blocks <= 0 || max_cases <= 0) return fail(ALP_ERR_INVALID, "empty engine");
  int sid, prec;
  if (int rc = scheme_id(scheme, &sid, &prec)) return rc;
  alp_engine *e = new (std::nothrow) alp_engine;
  if (!e) return fail(ALP_ERR_CAPACITY, "host allocation failed");
  e->dim = dim;
  e->scheme = sid;
  e->precision = prec;
  e->selection = *scheme;
  e->opt = scheme_options(scheme);
  e->rk2 = scheme->time_integrator == ALP_RK2;
  e->elastic = elastic;
  e->slots_max = capacity_blocks;
  e->capacity = elastic ? 0 : capacity_blocks;
  e->max_cases = max_cases;
  e->ne = dim + 2;
  e->cells = cells_of(dim);
  e->faces = faces_of(dim);
  cudaError_t err = cudaSuccess;
  int erc = ALP_OK;
  auto grab = [&](void **p, size_t bytes) {
    if (err == cudaSuccess) err = cudaMalloc(p, bytes);
  };
  // The strict build reproduces the reference's three-order symmetric flux
  // sum, so it keeps the face-flux arrays; the fast build sweeps pencils.
  // Both stepping paths keep their scratch so the autotuner can switch; the
  // strict build always uses the face-flux path, whose three-order symmetric
  // flux sum matches the reference bit for bit.
  // R also stages interior-only case transfers (alp_engine_*_case_interior).
  e->path = 1;
  double **big[5] = {&e->U, &e->UB, &e->UC, &e->F, &e->R};
  for (int k = 0; k < 5; ++k) {
    size_t const bytes = e->slot_bytes(k) * (size_t)capacity_blocks;
    if (!elastic) {
      grab((void **)big[k], bytes);
    } else if (erc == ALP_OK && err == cudaSuccess) {
      erc = alp::elastic_reserve(e->ea[k], bytes);
      *big[k] = reinterpret_cast<double *>(e->ea[k].base);
    }
  }
  if (erc != ALP_OK) {
    e->release();
    delete e;
    return erc;
  }
  grab((void **)&e->meta, sizeof(BlockMeta) * capacity_blocks);
  grab((void **)&e->nbr26, sizeof(int) * 26 * capacity_blocks);
  grab((void **)&e->work, sizeof(int) * capacity_blocks);
  grab((void **)&e->cases, sizeof(CaseState) * max_cases);
  grab((void **)&e->glf, sizeof(unsigned long long) * 4 * max_cases);
  // fused tile stages: 3D, the compiled default schemes (WENO5, HLLC/Einfeldt, Roe)
  bool const tiles = dim == 3 && e->opt.is_default() && !elastic;
  if (tiles) {
    grab((void **)&e->tsync, sizeof(int) * (2 + (size_t)capacity_blocks + 2 * (size_t)max_cases));
    grab((void **)&e->torder, sizeof(int) * 3 * (size_t)capacity_blocks);
    grab((void **)&e->tcase_nb, sizeof(int) * (size_t)max_cases);
    if (err == cudaSuccess) err = cudaMemset(e->tsync, 0, sizeof(int) * 2);
  }
  if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
  if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&e->stream2, cudaStreamNonBlocking);
  for (cudaEvent_t &ev : e->ev_batch)
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming);
  if (err == cudaSuccess)
    err = cudaMemsetAsync(e->cases, 0, sizeof(CaseState) * max_cases, e->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
  if (err != cudaSuccess) {
    e->release();
    delete e;
    return cuda_fail(err, "alp_engine_create");
  }
  if (tiles) {
    // TMA descriptors of the pools and the launch shapes; engines whose
    // descriptors or kernels are unavailable keep the face-flux path
    double *const pools[3] = {e->U, e->UB, e->UC};
    std::string why;
    bool ok = alp::tile_encode(e->targs, pools, capacity_blocks, why);
    int sms = 0, dev = 0;
    if (ok && (cudaGetDevice(&dev) != cudaSuccess ||
               cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess))
      ok = false;
    for (int v = 0; ok && v < alp::kTileVariants; ++v) {
      if (alp::tile_info(sid, v, prec, &e->tinfo[v]) != cudaSuccess || e->tinfo[v].ctas_per_sm < 1)
        ok = false;
      else
        e->tgrid[v] = e->tinfo[v].ctas_per_sm * sms;
    }
    cudaGetLastError();  // a refused attribute or query leaves the face-flux path
    if (ok) {
      alp::TileArgs &a = e->targs;
      a.order = e->torder;
      a.nstages = e->rk2 ? 2 : 3;
      a.stage0 = e->rk2 ? 3 : 0;
      a.meta = e->meta;
      a.nbr26 = e->nbr26;
      a.cases = e->cases;
      a.ctrl = e->tsync;
      a.done = e->tsync + 2;
      a.dtflag = e->tsync + 2 + capacity_blocks;
      a.cnt = e->tsync + 2 + capacity_blocks + max_cases;
      a.case_nb = e->tcase_nb;
      e->tile_ok = true;
      e->path = 3;
    }
  }
  e->h_meta.assign(capacity_blocks, BlockMeta{});
  e->h_nbr26.assign((size_t)capacity_blocks * 26, -1);
  if (e->capacity > 0) e->free_ranges[0] = e->capacity;
  e->case_rec.assign(max_cases, {});
  e->h_case_state.assign(max_cases, CaseState{});
  *out = e;
  return ALP_OK;
}

}  // namespace

extern "C" {

size_t alp_engine_bytes(int dim, int capacity_blocks, int max_cases) {
  if (dim < 1 || dim > 3) return 0;
  size_t const ne = dim + 2;
  size_t const blk = ne * cells_of(dim) * sizeof(double);
  size_t const flux = (size_t)dim * ne * faces_of(dim) * sizeof(double) +
                      ne * (dim == 3 ? 4096 : (dim == 2 ? 256 : 16)) * sizeof(double);
  // the fused tile path's flags, orders and case sizes (3D)
  size_t const tiles = dim == 3 ? sizeof(int) * (2 + 4 * (size_t)capacity_blocks + 3 * (size_t)max_cases) : 0;
  return (size_t)capacity_blocks *
             (3 * blk + flux + sizeof(BlockMeta) + 26 * sizeof(int) + sizeof(int)) +
         (size_t)max_cases * sizeof(CaseState) + tiles;
}

int alp_engine_create(int dim, const alp_scheme *scheme, int capacity_blocks, int max_cases,
                      alp_engine **out) {
  return engine_create(dim, scheme, capacity_blocks, max_cases, false, out);
}

int alp_engine_create_elastic(int dim, const alp_scheme *scheme, int max_blocks, int max_cases,
                              alp_engine **out) {
  return engine_create(dim, scheme, max_blocks, max_cases, true, out);
}

int alp_engine_reserve(alp_engine *e, int capacity_blocks) {
  if (!e) return fail(ALP_ERR_INVALID, "null engine");
  return e->set_capacity(capacity_blocks);
}

int alp_engine_capacity(alp_engine *e, int *capacity_blocks, int *used_blocks,
                        size_t *pool_bytes) {
  if (!e) return fail(ALP_ERR_INVALID, "null engine");
  if (capacity_blocks) *capacity_blocks = e->capacity;
  if (used_blocks) {
    int u = 0;
    for (auto const &c : e->case_rec)
      if (c.live) u += c.nb;
    *used_blocks = u;
  }
  if (pool_bytes) {
    size_t b = 0;
    for (int k = 0; k < 5; ++k) b += e->slot_bytes(k) * (size_t)e->capacity;
    *pool_bytes = e->elastic ? e->mapped_bytes() : b;
  }
  return ALP_OK;
}

int alp_engine_destroy(alp_engine *e) {
  if (!e) return ALP_OK;
  cudaStreamSynchronize(e->stream);
  e->release();
  delete e;
  return ALP_OK;
}

int alp_engine_add_case(alp_engine *e, const alp_material *mat, double cell_size, double cfl,
                        double t0, double t_end, int max_steps, int nb, const int *h_nbr26,
                        const double *h_blocks, int *case_id) {
  if (!e || !case_id) return fail(ALP_ERR_INVALID, "null argument");
  if (nb <= 0 || !h_nbr26 || !h_blocks) return fail(ALP_ERR_INVALID, "bad case blocks");
  int cid, first;
  if (int rc = engine_add_case_core(e, mat, cell_size, cfl, t0, t_end, max_steps, nb, h_nbr26,
                                    &cid, &first))
    return rc;
  size_t const blk = (size_t)e->ne * e->cells;
  ALP_CUDA(cudaMemcpyAsync(e->U + blk * first, h_blocks, blk * nb * sizeof(double),
                           cudaMemcpyHostToDevice, e->stream));
  // the source may be pageable or reused by the caller right after the call
  ALP_CUDA(cudaStreamSynchronize(e->stream));
  *case_id = cid;
  return ALP_OK;
}

int alp_engine_add_case_interior(alp_engine *e, const alp_material *mat, double cell_size,
                                 double cfl, double t0, double t_end, int max_steps, int nb,
                                 const int *h_nbr26, const double *h_interior, int *case_id) {
  if (!e || !case_id) return fail(ALP_ERR_INVALID, "null argument");
  if (nb <= 0 || !h_nbr26 || !h_interior) return fail(ALP_ERR_INVALID, "bad case blocks");
  int cid, first;
  if (int rc = engine_add_case_core(e, mat, cell_size, cfl, t0, t_end, max_steps, nb, h_nbr26,
                                    &cid, &first))
    return rc;
  // staged in the pencil path's per-cell scratch R, sized [capacity][NE][interior]
  size_t const bytes = (size_t)nb * e->ne * interior_of(e->dim) * sizeof(double);
  ALP_CUDA(cudaMemcpyAsync(e->R, h_interior, bytes, cudaMemcpyHostToDevice, e->stream));
  ALP_CUDA(launch_interior_copy(e->dim, e->U, first, nb, e->R, true, e->stream));
  ALP_CUDA(cudaStreamSynchronize(e->stream));
  *case_id = cid;
  return ALP_OK;
}

int alp_engine_add_case_ic(alp_engine *e, const alp_material *mat, double cell_size, double cfl,
                           double t0, double t_end, int max_steps, const int *nblocks,
                           const int *periodic, int ic_type, const double *ic_params,
                           int n_params, int *case_id) {
  if (!e || !case_id || !nblocks || !periodic || (n_params > 0 && !ic_params))
    return fail(ALP_ERR_INVALID, "null argument");
  if (ic_type != ALP_IC_QUADRANTS && ic_type != ALP_IC_BLAST)
    return fail(ALP_ERR_INVALID, "unknown initial-condition type");
  if (n_params < 0 || n_params > 24) return fail(ALP_ERR_INVALID, "at most 24 parameters");
  if (ic_type == ALP_IC_QUADRANTS && e->dim != 2)
    return fail(ALP_ERR_INVALID, "the four-quadrant problem is two-dimensional");
  int n[3] = {1, 1, 1};
  for (int d = 0; d < e->dim; ++d) {
    if (nblocks[d] <= 0) return fail(ALP_ERR_INVALID, "block counts must be positive");
    n[d] = nblocks[d];
  }
  std::vector<int> nbr = regular_grid_neighbours(e->dim, n, periodic);
  int const nb = n[0] * n[1] * n[2];
  int cid, first;
  if (int rc = engine_add_case_core(e, mat, cell_size, cfl, t0, t_end, max_steps, nb, nbr.data(),
                                    &cid, &first))
    return rc;
  IcParams p{};
  for (int i = 0; i < n_params; ++i) p.v[i] = ic_params[i];
  ALP_CUDA(launch_initial_condition(e->dim, e->U, first, n, cell_size, mat->gamma,
                                    mat->background_pressure, ic_type, p, e->stream));
  *case_id = cid;
  return ALP_OK;
}

int alp_engine_remove_case(alp_engine *e, int case_id) {
  if (!e) return fail(ALP_ERR_INVALID, "null engine");
  if (case_id < 0 || case_id >= e->max_cases || !e->case_rec[case_id].live)
    return fail(ALP_ERR_NOT_FOUND, "unknown case");
  ALP_CUDA(cudaStreamSynchronize(e->stream));
  auto &c = e->case_rec[case_id];
  e->free_range(c.first, c.nb);
  c = {};
  e->h_case_state[case_id] = CaseState{};
  ALP_CUDA(cudaMemcpyAsync(e->cases + case_id, &e->h_case_state[case_id], sizeof(CaseState),
                           cudaMemcpyHostToDevice, e->stream));
  return e->rebuild_work();
}

int alp_engine_step(alp_engine *e, int n) {
  if (!e) return fail(ALP_ERR_INVALID, "null engine");
  if (n <= 0 || e->nwork == 0) return ALP_OK;
  // profiler ranges (no cost unless a tool is attached): one per call, one per capture
  nvtx3::scoped_range range{"alp_engine_step"};
  if (e->path == 3) return e->run_tiles(n);
  if (!e->use_graph) {
    for (int i = 0; i < n; ++i)
      if (int rc = e->record_step()) return rc;
    return ALP_OK;
  }
  if (e->graph_dirty || !e->graph) {
    if (e->graph) {
      cudaGraphExecDestroy(e->graph);
      e->graph = nullptr;
    }
    cudaGraph_t g;
    nvtx3::scoped_range capture{"alp_engine_step: capture the step graph"};
    ALP_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    int const rc = e->record_step();
    cudaError_t const ce = cudaStreamEndCapture(e->stream, &g);
    if (rc) {
      if (ce == cudaSuccess) cudaGraphDestroy(g);
      return rc;
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
    cudaError_t const ie = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate");
    e->graph_dirty = false;
  }
  for (int i = 0; i < n; ++i) ALP_CUDA(cudaGraphLaunch(e->graph, e->stream));
  return ALP_OK;
}

int alp_engine_get_case_interior(alp_engine *e, int case_id, double *h_interior, double *t,
                                 int *steps) {
  if (!e) return fail(ALP_ERR_INVALID, "null engine");
  if (case_id < 0 || case_id >= e->max_cases || !e->case_rec[case_id].live)
    return fail(ALP_ERR_NOT_FOUND, "unknown case");
  auto const &c = e->case_rec[case_id];
  if (h_interior) {
    size_t const bytes = (size_t)c.nb * e->ne * interior_of(e->dim) * sizeof(double);
    ALP_CUDA(launch_interior_copy(e->dim, e->U, c.first, c.nb, e->R, false, e->stream));
    ALP_CUDA(cudaMemcpyAsync(h_interior, e->R, bytes, cudaMemcpyDeviceToHost, e->stream));
  }
  return alp_engine_get_case(e, case_id, nullptr, t, steps);
}

int alp_engine_get_case(alp_engine *e, int case_id, double *h_blocks, double *t, int *steps) {
  if (!e) return fail(ALP_ERR_INVALID, "null engine");
  if (case_id < 0 || case_id >= e->max_cases || !e->case_rec[case_id].live)
    return fail(ALP_ERR_NOT_FOUND, "unknown case");
  auto const &c = e->case_rec[case_id];
  size_t const blk = (size_t)e->ne * e->cells;
  CaseState cs;
  if (h_blocks) {
    // the pool's halos are not maintained while stepping: fill them (all 26
    // regions + zero gradient, as the reference's halo update) before export
    BlockMeta def{};
    Launch L{e->dim, e->scheme, e->precision, e->U, e->work + e->work_offset(case_id), c.nb,
             nullptr, def, e->stream};
    ALP_CUDA(launch_halo(L, e->nbr26, false, e->ne, nullptr));
    ALP_CUDA(cudaMemcpyAsync(h_blocks, e->U + blk * c.first, blk * c.nb * sizeof(double),
                             cudaMemcpyDeviceToHost, e->stream));
  }
  ALP_CUDA(cudaMemcpyAsync(&cs, e->cases + case_id, sizeof(cs), cudaMemcpyDeviceToHost, e->stream));
  ALP_CUDA(cudaStreamSynchronize(e->stream));
  if (int rc = e->tile_check()) return rc;
  if (t) *t = cs.t;
  if (steps) *steps = cs.steps;
  if (cs.status) return fail(ALP_ERR_NUMERIC, "non-finite or non-positive state; case stopped");
  return ALP_OK;
}

int alp_engine_checkpoint_case(alp_engine *e, int case_id, alp_case_checkpoint *info,
                               int *h_nbr26, double *h_blocks) {
  if (!e || !info) return fail(ALP_ERR_INVALID, "null argument");
  if (case_id < 0 || case_id >= e->max_cases || !e->case_rec[case_id].live)
    return fail(ALP_ERR_NOT_FOUND, "unknown case");
  if (int rc = alp_engine_get_case(e, case_id, h_blocks, nullptr, nullptr)) return rc;
  auto const &c = e->case_rec[case_id];
  CaseState cs;
  ALP_CUDA(cudaMemcpyAsync(&cs, e->cases + case_id, sizeof(cs), cudaMemcpyDeviceToHost, e->stream));
  ALP_CUDA(cudaStreamSynchronize(e->stream));
  info->dim = e->dim;
  info->nb = c.nb;
  info->steps = cs.steps;
  info->max_steps = cs.max_steps;
  info->t = cs.t;
  info->t_end = cs.t_end;
  info->cfl = cs.cfl;
  info->cell_size = c.cell_size;
  info->material = c.mat;
  info->scheme = e->selection;
  if (h_nbr26)
    for (size_t i = 0; i < (size_t)c.nb * 26; ++i) {
      int const n = e->h_nbr26[(size_t)c.first * 26 + i];
      h_nbr26[i] = n < 0 ? n : n - c.first;
    }
  return ALP_OK;
}

int alp_engine_restore_case(alp_engine *e, const alp_case_checkpoint *info, const int *h_nbr26,
                            const double *h_blocks, int *case_id) {
  if (!e || !info || !case_id) return fail(ALP_ERR_INVALID, "null argument");
  if (info->dim != e->dim) return fail(ALP_ERR_INVALID, "checkpoint of another dimension");
  if (info->steps < 0) return fail(ALP_ERR_INVALID, "negative step count");
  {
    alp_scheme const &a = info->scheme, &b = e->selection;
    if (a.convective_term_solver != b.convective_term_solver ||
        a.state_reconstruction != b.state_reconstruction ||
        a.reconstruction_stencil != b.reconstruction_stencil ||
        a.riemann_solver != b.riemann_solver || a.signal_speed != b.signal_speed ||
        a.flux_splitting != b.flux_splitting || a.time_integrator != b.time_integrator ||
        a.precision != b.precision)
      return fail(ALP_ERR_INVALID,
                  "checkpoint of another scheme selection (solver, reconstruction, stencil, "
                  "Riemann solver, signal speed, splitting, time integrator or precision "
                  "differs from the engine's)");
  }
  int cid;
  if (int rc = alp_engine_add_case(e, &info->material, info->cell_size, info->cfl, info->t,
                                   info->t_end, info->max_steps, info->nb, h_nbr26, h_blocks,
                                   &cid))
    return rc;
  // the step count carries on from the checkpoint (max_steps counts from the start)
  e->h_case_state[cid].steps = info->steps;
  ALP_CUDA(cudaMemcpyAsync(e->cases + cid, &e->h_case_state[cid], sizeof(CaseState),
                           cudaMemcpyHostToDevice, e->stream));
  ALP_CUDA(cudaStreamSynchronize(e->stream));
  *case_id = cid;
  return ALP_OK;
}

int alp_engine_all_done(alp_engine *e, int *done) {
  if (!e || !done) return fail(ALP_ERR_INVALID, "null argument");
  std::vector<CaseState> cs(e->max_cases);
  ALP_CUDA(cudaMemcpyAsync(cs.data(), e->cases, sizeof(CaseState) * e->max_cases,
                           cudaMemcpyDeviceToHost, e->stream));
  ALP_CUDA(cudaStreamSynchronize(e->stream));
  if (int rc = e->tile_check()) return rc;
  int d = 1;
  for (int c = 0; c < e->max_cases; ++c) {
    if (!e->case_rec[c].live) continue;
    bool const finished = !(cs[c].t < cs[c].t_end) ||
                          (cs[c].max_steps > 0 && cs[c].steps >= cs[c].max_steps) ||
                          cs[c].status != 0;
    if (!finished) d = 0;
  }
  *done = d;
  return ALP_OK;
}

alp_stream_t alp_engine_stream(alp_engine *e) { return e ? (alp_stream_t)e->stream : nullptr; }

namespace {
// Stepping candidates of alp_engine_autotune / alp_engine_set_path: path,
// face-kernel threads (paths 0-2) or tile variant (path 3).
struct Cand {
  int path, param;
};
Cand const kCands[ALP_STEP_CANDIDATES] = {{1, 128}, {1, 64}, {0, 128}, {2, 128}, {3, 0}, {3, 1}};

// Why candidate i cannot step engine e (null: it can).
char const *cand_refusal(alp_engine const *e, int i) {
  if (kCands[i].path == 0) {
#ifdef ALP_STRICT
    return "the strict build steps the face-flux path";
#endif
    if (!e->opt.is_default() || e->rk2)
      return "pencil sweeps are compiled for WENO5 + HLLC/Einfeldt and Roe with RK3 only";
  }
  if (kCands[i].path == 3 && !e->tile_ok)
    return "fused tile stages are compiled for 3D blocks with WENO5 + HLLC/Einfeldt and Roe";
  return nullptr;
}

void select_cand(alp_engine *e, int i) {
  e->path = kCands[i].path;
  if (e->path == 3) e->tile_variant = kCands[i].param;
  else e->face_threads = kCands[i].param;
  e->graph_dirty = true;
}
}  // namespace

int alp_engine_autotune(alp_engine *e, int trial_steps, int *chosen, float *ms_per_step) {
  if (!e) return fail(ALP_ERR_INVALID, "null engine");
  if (trial_steps <= 0) return fail(ALP_ERR_INVALID, "trial_steps must be positive");
  int const saved_path = e->path, saved_threads = e->face_threads, saved_var = e->tile_variant;
  float best = 0.f;
  int best_i = 0;
  cudaEvent_t t0, t1;
  ALP_CUDA(cudaEventCreate(&t0));
  ALP_CUDA(cudaEventCreate(&t1));
  for (int i = 0; i < ALP_STEP_CANDIDATES; ++i) {
    float ms = -1.f;
    if (!cand_refusal(e, i) && e->nwork > 0) {
      select_cand(e, i);
      auto trial = [&](int n) {
        if (e->path == 3) return e->record_tiles(n, true);
        for (int k = 0; k < n; ++k)
          if (int rc = e->record_step(true)) return rc;
        return (int)ALP_OK;
      };
      if (int rc = trial(1)) return rc;  // warm-up
      ALP_CUDA(cudaEventRecord(t0, e->stream));
      if (int rc = trial(trial_steps)) return rc;
      ALP_CUDA(cudaEventRecord(t1, e->stream));
      ALP_CUDA(cudaEventSynchronize(t1));
      ALP_CUDA(cudaEventElapsedTime(&ms, t0, t1));
      if (int rc = e->tile_check()) return rc;
      ms /= trial_steps;
      if (best == 0.f || ms < best) {
        best = ms;
        best_i = i;
      }
    }
    if (ms_per_step) ms_per_step[i] = ms;
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (e->nwork > 0) {
    select_cand(e, best_i);
  } else {
    e->path = saved_path;
    e->face_threads = saved_threads;
    e->tile_variant = saved_var;
  }
  e->graph_dirty = true;
  if (chosen) *chosen = e->nwork > 0 ? best_i : -1;
  return ALP_OK;
}

int alp_engine_set_path(alp_engine *e, int candidate) {
  if (!e) return fail(ALP_ERR_INVALID, "null engine");
  if (candidate < 0 || candidate >= ALP_STEP_CANDIDATES)
    return fail(ALP_ERR_INVALID, "candidate must be 0 .. ALP_STEP_CANDIDATES - 1");
  if (char const *why = cand_refusal(e, candidate)) return fail(ALP_ERR_INVALID, why);
  select_cand(e, candidate);
  return ALP_OK;
}

int alp_engine_path(alp_engine *e) {
  if (!e) return -1;
  for (int i = 0; i < ALP_STEP_CANDIDATES; ++i)
    if (kCands[i].path == e->path &&
        (e->path == 3 ? kCands[i].param == e->tile_variant : kCands[i].param == e->face_threads))
      return i;
  return -1;
}

int alp_engine_set_graph(alp_engine *e, int enabled) {
  if (!e) return fail(ALP_ERR_INVALID, "null engine");
  e->use_graph = enabled != 0;
  return ALP_OK;
}

int alp_engine_launches_per_step(alp_engine *e) {
  if (!e) return 0;
  // signal speed, dt, 3 stages x (one pencil sweep per direction, or face
  // fluxes + stage update, per batch on the overlapped path), commit; the tile
  // path launches signal speed, dt and one persistent kernel per call
  if (e->path == 3) return 3;
  int const batches = e->path == 2 ? std::min(alp_engine::kMaxBatches, std::max(1, e->nwork / 64)) : 1;
  return 2 + (e->rk2 ? 2 : 3) * (e->path == 0 ? e->dim : 2 * batches) + 1;
}

int alp_engine_launches(alp_engine *e, int n) {
  if (!e || n <= 0 || e->nwork == 0) return 0;
  return e->path == 3 ? 3 : n * alp_engine_launches_per_step(e);
}

}  // extern "C"
