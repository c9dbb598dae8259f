// TEST INFRASTRUCTURE ONLY — never part of the product path.
//
// A C-ABI wrapper around ALPACA's own hot-path classes. oracle/Makefile compiles
// this file together with the reference's sources (read in place, never copied)
// into oracle/_ref/libalpref_d<DIM>_<variant>.so. The variant is selected the way
// ALPACA selects it: by the constexpr enums in user_specifications/*.h, which the
// Makefile regenerates per variant into oracle/_ref/shadow_<variant>/.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU arm load these libraries.
//
// What runs here is the reference's code:
//   * ConvectiveTermSolverSetup::Concretize<convective_term_solver>::type, i.e.
//     FiniteVolumeScheme (finite_volume_scheme.cpp:45) or FluxSplittingScheme
//     (flux_splitting_scheme.cpp:97) with the reference's EigenDecomposition,
//     state reconstruction, WENO5 and HLLC/Einfeldt classes,
//   * StiffenedGas / StiffenedGasSafe (materials/equations_of_state/),
//   * PrimeStateHandler::ConvertConservativesToPrimeStates (prime_state_handler.h:141),
//   * RungeKutta3TVD or RungeKutta2TVD (TimeIntegratorSetup::Concretize of the
//     shadow numerical_setup.h) + TimeIntegrator on Node objects
//     (integrator/time_integrator.h).
// What is restated (the reference's versions need mpi.h, which is absent):
//   * the divergence of SpaceSolver::UpdateFluxes (space_solver.cpp:58-70, 131-153),
//   * the same-level halo copy (internal_halo_manager.cpp:439-459 with the plane
//     index tables of communication/communication_types.h:45-132) and the
//     zero-gradient slabs (boundary_constants.h:103-160, 211-252),
//   * ComputeTimestepSize (modular_algorithm_assembler.cpp:1777-1997),
//   * the single-level stage sequence of Advance (modular_algorithm_assembler.cpp:575-874).
#include "boundary_condition/boundary_constants.h"
#include "integrator/runge_kutta_2_TVD.h"
#include "integrator/runge_kutta_3_TVD.h"
#include "integrator/time_integrator_setup.h"
#include "materials/equations_of_state/stiffened_gas.h"
#include "materials/equations_of_state/stiffened_gas_safe.h"
#include "materials/material_manager.h"
#include "multiresolution/multiresolution.h"
#include "prime_states/prime_state_handler.h"
#include "solvers/convective_term_contributions/convective_term_solver_setup.h"
#include "solvers/eigendecomposition.h"
#include "stencils/spatial_reconstruction_stencils/weno5.h"
#include "stencils/stencil_utilities.h"
#include "topology/id_information.h"
#include "topology/node.h"
#include "unit_handler.h"
#include "utilities/mathematical_functions.h"

#include <pthread.h>

#include <algorithm>
#include <cstring>
#include <functional>
#include <memory>
#include <vector>

namespace {

constexpr unsigned TCX = CC::TCX(), TCY = CC::TCY(), TCZ = CC::TCZ();
constexpr unsigned ICX = CC::ICX(), ICY = CC::ICY(), ICZ = CC::ICZ();
constexpr unsigned NE = MF::ANOE(), NP = MF::ANOP();
constexpr std::size_t CELLS = std::size_t(TCX) * TCY * TCZ;
constexpr std::size_t FACES = std::size_t(ICX + 1) * (ICY + 1) * (ICZ + 1);

using Solver = ConvectiveTermSolverSetup::Concretize<convective_term_solver>::type;
using Field = double[TCX][TCY][TCZ];
using FluxArray = double[NE][ICX + 1][ICY + 1][ICZ + 1];
using ForceArray = double[NE][ICX][ICY][ICZ];

constexpr MaterialName kMat = MaterialName::MaterialOne;

struct Context {
  UnitHandler unit_handler{1.0, 1.0, 1.0, 1.0};
  std::unique_ptr<MaterialManager> materials;
  std::unique_ptr<EigenDecomposition> eigen;
  std::unique_ptr<Solver> solver;
  std::unique_ptr<PrimeStateHandler> primes;

  Context(double gamma, double B, int safe) {
    std::unordered_map<std::string, double> eos_data = {
        {"gamma", gamma}, {"backgroundPressure", B}};
    std::unique_ptr<EquationOfState const> eos;
    if (safe)
      eos = std::make_unique<StiffenedGasSafe const>(eos_data, unit_handler);
    else
      eos = std::make_unique<StiffenedGas const>(eos_data, unit_handler);
    std::vector<std::tuple<MaterialType, Material>> mats;
    mats.emplace_back(MaterialType::Fluid,
                      Material(std::move(eos), 0.0, 0.0, 0.0, 0.0, nullptr,
                               nullptr, unit_handler));
    materials = std::make_unique<MaterialManager>(std::move(mats),
                                                  std::vector<MaterialPairing>{});
    eigen = std::make_unique<EigenDecomposition>(*materials);
    solver = std::make_unique<Solver>(*materials, *eigen);
    primes = std::make_unique<PrimeStateHandler>(*materials);
  }
};

// Runs fn(t) on n threads with large stacks: the reference keeps 2-3.5 MB of
// scratch on the stack per RHS call.
void ParallelFor(int nthreads, std::function<void(int)> const &fn) {
  if (nthreads <= 1) {
    fn(0);
    return;
  }
  struct Arg {
    std::function<void(int)> const *fn;
    int t;
  };
  std::vector<pthread_t> th(nthreads);
  std::vector<Arg> args(nthreads);
  pthread_attr_t attr;
  pthread_attr_init(&attr);
  pthread_attr_setstacksize(&attr, std::size_t(64) << 20);
  for (int t = 0; t < nthreads; ++t) {
    args[t] = {&fn, t};
    pthread_create(
        &th[t], &attr,
        [](void *p) -> void * {
          Arg *a = static_cast<Arg *>(p);
          (*a->fn)(a->t);
          return nullptr;
        },
        &args[t]);
  }
  for (auto &t : th)
    pthread_join(t, nullptr);
  pthread_attr_destroy(&attr);
}

void LoadAverages(Block &b, double const *u) {
  for (unsigned e = 0; e < NE; ++e)
    std::memcpy(&b.GetAverageBuffer(MF::ASOE()[e])[0][0][0], u + e * CELLS,
                CELLS * sizeof(double));
}

void StoreBuffer(double const (&f)[TCX][TCY][TCZ], double *out) {
  std::memcpy(out, &f[0][0][0], CELLS * sizeof(double));
}

// Zero + convective fluxes + divergence: SpaceSolver::UpdateFluxes
// (space_solver.cpp:58-70, 89-116, 131-153) for one single-phase block,
// restated because SpaceSolver links the MPI interface solver.
void SpaceRhs(Context const &ctx, std::pair<MaterialName const, Block> &mb,
              double cell_size, FluxArray &fx, FluxArray &fy, FluxArray &fz,
              ForceArray &vf) {
  Block &b = mb.second;
  for (unsigned e = 0; e < NE; ++e) {
    Field &r = b.GetRightHandSideBuffer(MF::ASOE()[e]);
    for (unsigned i = 0; i < TCX; ++i)
      for (unsigned j = 0; j < TCY; ++j)
        for (unsigned k = 0; k < TCZ; ++k)
          r[i][j][k] = 0.0;
  }
  double const one_cell_size = 1.0 / cell_size;
  std::memset(&fx[0][0][0][0], 0, sizeof(FluxArray));
  std::memset(&fy[0][0][0][0], 0, sizeof(FluxArray));
  std::memset(&fz[0][0][0][0], 0, sizeof(FluxArray));
  std::memset(&vf[0][0][0][0], 0, sizeof(ForceArray));
  ctx.solver->UpdateConvectiveFluxes(mb, cell_size, fx, fy, fz, vf);
  for (Equation const eq : MF::ASOE()) {
    auto const e = ETI(eq);
    Field &cells = b.GetRightHandSideBuffer(eq);
    for (unsigned i = 0; i < ICX; ++i)
      for (unsigned j = 0; j < ICY; ++j)
        for (unsigned k = 0; k < ICZ; ++k)
          cells[i + CC::FICX()][j + CC::FICY()][k + CC::FICZ()] +=
              vf[e][i][j][k] +
              DimensionAwareConsistencyManagedSum(
                  fx[e][i][j + 1][k + 1] - fx[e][i + 1][j + 1][k + 1],
                  fy[e][i + 1][j][k + 1] - fy[e][i + 1][j + 1][k + 1],
                  fz[e][i + 1][j + 1][k] - fz[e][i + 1][j + 1][k + 1]) *
                  one_cell_size;
  }
}

// Global Lax-Friedrichs: ComputeRightHandSide (modular_algorithm_assembler.cpp:
// 957-985) takes the maxima of EigenDecomposition::ComputeMaxEigenvaluesOnBlock
// over all blocks (then over MPI ranks, one rank here) and hands them to
// SetGlobalEigenvalues before the fluxes of each stage. block(b) returns the
// (material, block) pair of block b with its prime states up to date.
template <class BlockOf>
void SetGlobalLaxFriedrichs(Context const &ctx, int nb, BlockOf block) {
  if constexpr (convective_term_solver == ConvectiveTermSolvers::FluxSplitting &&
                FluxSplittingSettings::flux_splitting_scheme ==
                    FluxSplitting::GlobalLaxFriedrichs) {
    double max_eigenvalues[DTI(CC::DIM())][MF::ANOE()];
    for (unsigned d = 0; d < DTI(CC::DIM()); ++d)
      for (unsigned e = 0; e < MF::ANOE(); ++e)
        max_eigenvalues[d][e] = 0.0;
    double current[DTI(CC::DIM())][MF::ANOE()];
    for (int b = 0; b < nb; ++b) {
      ctx.eigen->ComputeMaxEigenvaluesOnBlock(block(b), current);
      for (unsigned d = 0; d < DTI(CC::DIM()); ++d)
        for (unsigned e = 0; e < MF::ANOE(); ++e)
          max_eigenvalues[d][e] = std::max(max_eigenvalues[d][e], current[d][e]);
    }
    ctx.eigen->SetGlobalEigenvalues(max_eigenvalues);
  } else {
    (void)ctx;
    (void)nb;
    (void)block;
  }
}

struct ScratchBuffers {
  FluxArray fx, fy, fz;
  ForceArray vf;
};
struct Scratch {
  std::unique_ptr<ScratchBuffers> buf{new ScratchBuffers};
  FluxArray *fx = &buf->fx, *fy = &buf->fy, *fz = &buf->fz;
  ForceArray *vf = &buf->vf;
};

// Same-level face-halo copy (the six "planes" of communication_types.h:45-132,
// copied as in internal_halo_manager.cpp:439-459) followed by zero-gradient
// slabs for domain faces (boundary_constants.h:103-160, 211-252). nbr holds six
// entries per block ordered W,E,S,N,B,T; -1 marks a zero-gradient domain face.
// Reads the interiors and writes the halos of the buffer selected by get().
// Symmetry wall at location LOC: the reference's mirror indices and halo
// slab (BoundaryConstants<LOC>::SymmetryInternalValue / HaloStart/EndIndices,
// boundary_constants.h:35-46, 167-209) with the sign of
// SymmetryBoundaryCondition<LOC>::SymmetrySign (-1.0 for the momentum normal
// to the wall, symmetry_boundary_condition.h:148-217).
template <BoundaryLocation LOC>
void SymmetrySlab(Field &f, double const sign) {
  constexpr auto lo = BoundaryConstants<LOC>::HaloStartIndices();
  constexpr auto hi = BoundaryConstants<LOC>::HaloEndIndices();
  for (unsigned i = lo[0]; i < hi[0]; ++i)
    for (unsigned j = lo[1]; j < hi[1]; ++j)
      for (unsigned k = lo[2]; k < hi[2]; ++k)
        f[i][j][k] = sign * BoundaryConstants<LOC>::SymmetryInternalValue(f, i, j, k);
}

void SymmetryFace(Field &f, int dir, int high, Equation eq) {
  Equation const normal = dir == 0 ? Equation::MomentumX
                                   : (dir == 1 ? Equation::MomentumY : Equation::MomentumZ);
  double const sign = eq == normal ? -1.0 : 1.0;
  if (dir == 0) {
    if (high) SymmetrySlab<BoundaryLocation::East>(f, sign);
    else SymmetrySlab<BoundaryLocation::West>(f, sign);
  } else if (dir == 1) {
    if (high) SymmetrySlab<BoundaryLocation::North>(f, sign);
    else SymmetrySlab<BoundaryLocation::South>(f, sign);
  } else {
    if (high) SymmetrySlab<BoundaryLocation::Top>(f, sign);
    else SymmetrySlab<BoundaryLocation::Bottom>(f, sign);
  }
}

// Same-level halos from the six face neighbours nbr[6 b + face] (W, E, S, N,
// B, T): >= 0 a neighbour, -1 a zero-gradient domain face, -2 a symmetry wall.
void HaloUpdate(std::vector<std::unique_ptr<Node>> &nodes, int const *nbr,
                std::function<Field &(Block &, Equation)> const &get) {
  int const nb = int(nodes.size());
  unsigned const HS = CC::HS();
  int const ndim = int(DTI(CC::DIM()));
  for (int b = 0; b < nb; ++b) {
    Block &me = nodes[b]->GetSinglePhase();
    for (int face = 0; face < 2 * ndim; ++face) {
      int const n = nbr[6 * b + face];
      if (n < 0)
        continue;
      Block &other = nodes[n]->GetSinglePhase();
      int const dir = face / 2, high = face % 2;
      for (Equation const eq : MF::ASOE()) {
        Field &dst = get(me, eq);
        Field &src = get(other, eq);
        unsigned lo[3] = {CC::FICX(), CC::FICY(), CC::FICZ()};
        unsigned ext[3] = {ICX, ICY, ICZ};
        unsigned srclo[3] = {CC::FICX(), CC::FICY(), CC::FICZ()};
        ext[dir] = HS;
        // high face: halo [FHH, TC) <- neighbour's first HS interior cells;
        // low face: halo [0, HS) <- neighbour's last HS interior cells.
        unsigned const icd = dir == 0 ? ICX : (dir == 1 ? ICY : ICZ);
        lo[dir] = high ? HS + icd : 0;
        srclo[dir] = high ? HS : icd;
        for (unsigned i = 0; i < ext[0]; ++i)
          for (unsigned j = 0; j < ext[1]; ++j)
            for (unsigned k = 0; k < ext[2]; ++k)
              dst[lo[0] + i][lo[1] + j][lo[2] + k] =
                  src[srclo[0] + i][srclo[1] + j][srclo[2] + k];
      }
    }
  }
  // External (zero-gradient, symmetry) boundaries after all internal halos, as in
  // HaloManager::MaterialHaloUpdateOnLevel (halo_manager.cpp:87-124).
  for (int b = 0; b < nb; ++b) {
    Block &me = nodes[b]->GetSinglePhase();
    for (int face = 0; face < 2 * ndim; ++face) {
      if (nbr[6 * b + face] >= 0)
        continue;
      int const dir = face / 2, high = face % 2;
      for (Equation const eq : MF::ASOE()) {
        Field &f = get(me, eq);
        if (nbr[6 * b + face] == -2) {
          SymmetryFace(f, dir, high, eq);
          continue;
        }
        if (dir == 0) {
          unsigned const s = high ? CC::FHHX() - 1 : CC::HSSX();
          unsigned const i0 = high ? CC::FHHX() : 0, i1 = high ? TCX : CC::HSSX();
          for (unsigned i = i0; i < i1; ++i)
            for (unsigned j = 0; j < TCY; ++j)
              for (unsigned k = 0; k < TCZ; ++k)
                f[i][j][k] = f[s][j][k];
        } else if (dir == 1) {
          unsigned const s = high ? CC::FHHY() - 1 : CC::HSSY();
          unsigned const j0 = high ? CC::FHHY() : 0, j1 = high ? TCY : CC::HSSY();
          for (unsigned i = 0; i < TCX; ++i)
            for (unsigned j = j0; j < j1; ++j)
              for (unsigned k = 0; k < TCZ; ++k)
                f[i][j][k] = f[i][s][k];
        } else {
          unsigned const s = high ? CC::FHHZ() - 1 : CC::HSSZ();
          unsigned const k0 = high ? CC::FHHZ() : 0, k1 = high ? TCZ : CC::HSSZ();
          for (unsigned i = 0; i < TCX; ++i)
            for (unsigned j = 0; j < TCY; ++j)
              for (unsigned k = k0; k < k1; ++k)
                f[i][j][k] = f[i][j][s];
        }
      }
    }
  }
}

// ComputeTimestepSize (modular_algorithm_assembler.cpp:1840-1870, 1932,
// 1961-1982) for a single material without viscosity, heat conduction,
// capillarity or gravity coefficients (their max() terms leave dt unchanged).
double TimestepSize(Context const &ctx, std::vector<std::unique_ptr<Node>> &nodes,
                    double cell_size, double cfl, double current_time,
                    double end_time) {
  std::array<double, DTI(CC::DIM())> velocity_plus_sound;
  double sum_of_signalspeeds = 0.0;
  EquationOfState const &eos =
      ctx.materials->GetMaterial(kMat).GetEquationOfState();
  for (auto &node : nodes) {
    PrimeStates const &ps = node->GetSinglePhase().GetPrimeStateBuffer();
    for (unsigned i = CC::FICX(); i <= CC::LICX(); ++i)
      for (unsigned j = CC::FICY(); j <= CC::LICY(); ++j)
        for (unsigned k = CC::FICZ(); k <= CC::LICZ(); ++k) {
          double const c = eos.SpeedOfSound(ps[PrimeState::Density][i][j][k],
                                            ps[PrimeState::Pressure][i][j][k]);
          for (unsigned d = 0; d < DTI(CC::DIM()); ++d)
            velocity_plus_sound[d] = std::abs(ps[MF::AV()[d]][i][j][k]) + c;
          sum_of_signalspeeds = std::max(
              sum_of_signalspeeds, ConsistencyManagedSum(velocity_plus_sound));
        }
  }
  double dt = sum_of_signalspeeds / cell_size;
  double local_dt;
  if (dt == 0.0)
    local_dt = std::numeric_limits<double>::max();
  else
    local_dt = cfl / dt;
  if (current_time + local_dt > end_time)
    local_dt = std::max(end_time - current_time, 0.0);
  return local_dt;
}

} // namespace

extern "C" {

int ref_config(int *dim, int *neq, int *nprime, int *solver, int *recon) {
  *dim = int(DTI(CC::DIM()));
  *neq = int(NE);
  *nprime = int(NP);
  *solver = convective_term_solver == ConvectiveTermSolvers::FiniteVolume ? 1 : 0;
  *recon = int(state_reconstruction_type);
  return 0;
}

// WENO5 (weno5.h:88-158) through SU::Reconstruction with UpwindLeft / UpwindRight.
int ref_weno5(double const *v, double *left, double *right) {
  std::array<double, 6> a;
  for (int i = 0; i < 6; ++i)
    a[i] = v[i];
  *left = SU::Reconstruction<WENO5, SP::UpwindLeft>(a, 1.0);
  *right = SU::Reconstruction<WENO5, SP::UpwindRight>(a, 1.0);
  return 0;
}

// Multiresolution::Prediction (multiresolution.cpp:146-283) of one field:
// parent and child are full [TCX][TCY][TCZ] buffers; octant is the child's
// position among its siblings (bit 0 x, bit 1 y, bit 2 z); start and count
// give the child cells to fill, as the reference's halo managers pass them.
int ref_prediction(double const *parent, int octant, int const *start, int const *count,
                   double *child) {
  using Buf = double[CC::TCX()][CC::TCY()][CC::TCZ()];
  nid_t child_id = 0;
  bool found = false;
  for (nid_t const id : IdsOfChildren(IdSeed()))
    if (int(PositionOfNodeAmongSiblings(id)) == octant) {
      child_id = id;
      found = true;
    }
  if (!found) return 1;
  Multiresolution::Prediction(*reinterpret_cast<Buf const *>(parent),
                              *reinterpret_cast<Buf *>(child), child_id,
                              unsigned(start[0]), unsigned(count[0]), unsigned(start[1]),
                              unsigned(count[1]), unsigned(start[2]), unsigned(count[2]));
  return 0;
}

// EOS queries through the reference's virtual EquationOfState interface.
// cons = (mass, energy, mx, my, mz); prim = (rho, p, u, v, w).
// out = pressure, enthalpy, energy, speed of sound, psi, gruneisen.
int ref_eos(double gamma, double B, int safe, double const *cons,
            double const *prim, double *out) {
  Context ctx(gamma, B, safe);
  EquationOfState const &eos =
      ctx.materials->GetMaterial(kMat).GetEquationOfState();
  out[0] = eos.Pressure(cons[0], cons[2], cons[3], cons[4], cons[1]);
  out[1] = eos.Enthalpy(cons[0], cons[2], cons[3], cons[4], cons[1]);
  out[2] = eos.Energy(prim[0], prim[2], prim[3], prim[4], prim[1]);
  out[3] = eos.SpeedOfSound(prim[0], prim[1]);
  out[4] = eos.Psi(prim[1], 1.0 / prim[0]);
  out[5] = eos.Gruneisen();
  return 0;
}

// Prime states of every cell (prime_state_handler.h:141-152).
// u: [nb][NE][cells] in, p: [nb][NP][cells] out.
int ref_prime_states(double const *u, int nb, double gamma, double B, int safe,
                     double *p) {
  Context ctx(gamma, B, safe);
  auto mb = std::make_unique<std::pair<MaterialName const, Block>>(
      std::piecewise_construct, std::forward_as_tuple(kMat),
      std::forward_as_tuple());
  for (int b = 0; b < nb; ++b) {
    LoadAverages(mb->second, u + std::size_t(b) * NE * CELLS);
    ctx.primes->ConvertConservativesToPrimeStates(
        kMat, mb->second.GetAverageBuffer(), mb->second.GetPrimeStateBuffer());
    for (unsigned q = 0; q < NP; ++q)
      StoreBuffer(mb->second.GetPrimeStateBuffer(MF::ASOP()[q]),
                  p + (std::size_t(b) * NP + q) * CELLS);
  }
  return 0;
}

// ConvectiveTermSolver::UpdateConvectiveFluxes (convective_term_solver.h:67-81)
// on nb blocks whose halos are already filled. Fluxes are returned in the
// reference's [NE][ICX+1][ICY+1][ICZ+1] layout per block and direction, starting
// from zero (SpaceSolver zeroes them before the call, space_solver.cpp:89-98).
// With rhs != nullptr also returns the SpaceSolver right-hand side [NE][cells].
int ref_space_rhs(double const *u, int nb, double gamma, double B, int safe,
                  double cell_size, double *fx, double *fy, double *fz,
                  double *rhs, int nthreads) {
  Context ctx(gamma, B, safe);
  if (nthreads < 1)
    nthreads = 1;
  {
    // prime states of every block first (global Lax-Friedrichs maxima)
    auto mb = std::make_unique<std::pair<MaterialName const, Block>>(
        std::piecewise_construct, std::forward_as_tuple(kMat),
        std::forward_as_tuple());
    SetGlobalLaxFriedrichs(ctx, nb, [&](int b) -> std::pair<MaterialName const, Block> const & {
      Block &blk = mb->second;
      LoadAverages(blk, u + std::size_t(b) * NE * CELLS);
      ctx.primes->ConvertConservativesToPrimeStates(kMat, blk.GetAverageBuffer(),
                                                    blk.GetPrimeStateBuffer());
      return *mb;
    });
  }
  ParallelFor(nthreads, [&](int t) {
    auto mb = std::make_unique<std::pair<MaterialName const, Block>>(
        std::piecewise_construct, std::forward_as_tuple(kMat),
        std::forward_as_tuple());
    Scratch s;
    for (int b = t; b < nb; b += nthreads) {
      Block &blk = mb->second;
      LoadAverages(blk, u + std::size_t(b) * NE * CELLS);
      ctx.primes->ConvertConservativesToPrimeStates(
          kMat, blk.GetAverageBuffer(), blk.GetPrimeStateBuffer());
      SpaceRhs(ctx, *mb, cell_size, *s.fx, *s.fy, *s.fz, *s.vf);
      std::size_t const fo = std::size_t(b) * NE * FACES;
      if (fx)
        std::memcpy(fx + fo, &(*s.fx)[0][0][0][0], sizeof(FluxArray));
      if (fy)
        std::memcpy(fy + fo, &(*s.fy)[0][0][0][0], sizeof(FluxArray));
      if (fz)
        std::memcpy(fz + fo, &(*s.fz)[0][0][0][0], sizeof(FluxArray));
      if (rhs)
        for (unsigned e = 0; e < NE; ++e)
          StoreBuffer(blk.GetRightHandSideBuffer(MF::ASOE()[e]),
                      rhs + (std::size_t(b) * NE + e) * CELLS);
    }
  });
  return 0;
}

// Single-level time loop (Advance, modular_algorithm_assembler.cpp:575-874,
// single phase, no multiresolution): nb blocks of cell size cell_size with the
// six-face neighbour table nbr (W,E,S,N,B,T; -1 = zero gradient). u holds the
// conservatives [nb][NE][cells]; on entry only the interiors are used (halos
// are filled first), on exit it holds the final state with halos.
// Runs until t_end or max_steps (max_steps <= 0: no step limit). Writes the
// time reached to *t_io (which holds the start time on entry), the number of
// steps to *steps_done and, if dt_log != nullptr, each step's dt.
int ref_run(double *u, int nb, int const *nbr, double gamma, double B, int safe,
            double cell_size, double cfl, double t_end, int max_steps,
            int nthreads, double *t_io, int *steps_done, double *dt_log) {
  Context ctx(gamma, B, safe);
  if (nthreads < 1)
    nthreads = 1;
  TimeIntegratorSetup::Concretize<time_integrator>::type rk(*t_io);
  std::vector<std::unique_ptr<Node>> nodes(nb);
  double const node_size = cell_size * ICX;
  for (int b = 0; b < nb; ++b) {
    nodes[b] = std::make_unique<Node>(IdSeed(), node_size,
                                      std::vector<MaterialName>{kMat});
    LoadAverages(nodes[b]->GetSinglePhase(), u + std::size_t(b) * NE * CELLS);
  }
  auto average = [](Block &b, Equation e) -> Field & {
    return b.GetAverageBuffer(e);
  };
  auto rhs_buffer = [](Block &b, Equation e) -> Field & {
    return b.GetRightHandSideBuffer(e);
  };
  auto obtain_primes = [&]() {
    ParallelFor(nthreads, [&](int t) {
      for (int b = t; b < nb; b += nthreads) {
        Block &blk = nodes[b]->GetSinglePhase();
        ctx.primes->ConvertConservativesToPrimeStates(
            kMat, blk.GetAverageBuffer(), blk.GetPrimeStateBuffer());
      }
    });
  };
  HaloUpdate(nodes, nbr, average);
  obtain_primes();

  double t = *t_io;
  int steps = 0;
  while (t < t_end && (max_steps <= 0 || steps < max_steps)) {
    double const dt = TimestepSize(ctx, nodes, cell_size, cfl, t, t_end);
    if (dt_log)
      dt_log[steps] = dt;
    rk.AppendMicroTimestep(dt);
    for (unsigned stage = 0; stage < rk.NumberOfStages(); ++stage) {
      // ComputeRightHandSide (:954-1008): global Lax-Friedrichs maxima,
      // FillInitialBuffer, UpdateFluxes, PrepareBufferForIntegration.
      SetGlobalLaxFriedrichs(ctx, nb, [&](int b) -> std::pair<MaterialName const, Block> const & {
        return *nodes[b]->GetPhases().begin();
      });
      ParallelFor(nthreads, [&](int th) {
        Scratch s;
        for (int b = th; b < nb; b += nthreads) {
          Node &node = *nodes[b];
          rk.FillInitialBuffer(node, stage);
          for (auto &phase : node.GetPhases())
            SpaceRhs(ctx, phase, cell_size, *s.fx, *s.fy, *s.fz, *s.vf);
          rk.PrepareBufferForIntegration(node, stage);
        }
      });
      // Integrate (:1068-1098) on the interior, then the halo update of the
      // integrated buffer (:726) and the swap (:830) + prime states (:839).
      ParallelFor(nthreads, [&](int th) {
        for (int b = th; b < nb; b += nthreads)
          rk.IntegrateNode(*nodes[b], stage, 1);
      });
      HaloUpdate(nodes, nbr, rhs_buffer);
      for (auto &node : nodes)
        rk.SwapBuffersForNextStage(*node);
      obtain_primes();
    }
    rk.FinishMacroTimestep();
    t = rk.CurrentRunTime();
    ++steps;
  }
  for (int b = 0; b < nb; ++b)
    for (unsigned e = 0; e < NE; ++e)
      StoreBuffer(nodes[b]->GetSinglePhase().GetAverageBuffer(MF::ASOE()[e]),
                  u + (std::size_t(b) * NE + e) * CELLS);
  *t_io = t;
  *steps_done = steps;
  return 0;
}

} // extern "C"
