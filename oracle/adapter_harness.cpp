// TEST INFRASTRUCTURE ONLY — never part of the product path.
//
// Runs the drop-in adapter B200ConvectiveTermSolver (b200_convective_term_solver.h)
// inside the reference's own object model: the reference's MaterialManager,
// EigenDecomposition and Block, with UpdateConvectiveFluxes called through the
// reference's CRTP base (convective_term_solver.h:67-81) exactly as
// SpaceSolver::UpdateFluxes calls it (space_solver.cpp:89-116, arrays zeroed
// first). oracle/Makefile compiles this file against the reference's headers
// (read in place) with the same shadow user_specifications as
// libalpref_d<DIM>_<variant>.so, and links it with the reference's sources and
// with libalpaca_b200.so (or the strict build): tests compare its fluxes with
// the reference's FiniteVolumeScheme / FluxSplittingScheme on the same blocks.
#include "b200_convective_term_solver.h"
#include "materials/equations_of_state/stiffened_gas.h"
#include "materials/equations_of_state/stiffened_gas_safe.h"
#include "materials/material_manager.h"
#include "solvers/eigendecomposition.h"
#include "unit_handler.h"

#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace {

constexpr std::size_t CELLS = std::size_t(CC::TCX()) * CC::TCY() * CC::TCZ();
constexpr std::size_t FACES = std::size_t(CC::ICX() + 1) * (CC::ICY() + 1) * (CC::ICZ() + 1);
constexpr unsigned NE = MF::ANOE();
using FluxArray = double[NE][CC::ICX() + 1][CC::ICY() + 1][CC::ICZ() + 1];
using ForceArray = double[NE][CC::ICX()][CC::ICY()][CC::ICZ()];

std::string g_error;

}  // namespace

extern "C" {

char const *adapter_last_error() { return g_error.c_str(); }

// Fluxes of nb blocks u [nb][NE][cells] (halos filled) through the adapter:
// fx, fy, fz [nb][NE][ICX+1][ICY+1][ICZ+1], each block's arrays zeroed before
// the call as SpaceSolver does. precision: ALP_FP64 or ALP_FP32_FLUX.
// Returns 0, or -1 with adapter_last_error() set when the adapter threw.
int adapter_fluxes(double const *u, int nb, double gamma, double B, int safe, double cell_size,
                   double *fx, double *fy, double *fz, int precision) {
  try {
    UnitHandler const unit_handler{1.0, 1.0, 1.0, 1.0};
    std::unordered_map<std::string, double> eos_data = {{"gamma", gamma},
                                                        {"backgroundPressure", B}};
    std::unique_ptr<EquationOfState const> eos;
    if (safe)
      eos = std::make_unique<StiffenedGasSafe const>(eos_data, unit_handler);
    else
      eos = std::make_unique<StiffenedGas const>(eos_data, unit_handler);
    std::vector<std::tuple<MaterialType, Material>> mats;
    mats.emplace_back(MaterialType::Fluid, Material(std::move(eos), 0.0, 0.0, 0.0, 0.0, nullptr,
                                                    nullptr, unit_handler));
    MaterialManager const materials(std::move(mats), std::vector<MaterialPairing>{});
    EigenDecomposition const eigen(materials);
    B200ConvectiveTermSolver const solver(materials, eigen, precision);
    auto mb = std::make_unique<std::pair<MaterialName const, Block>>(
        std::piecewise_construct, std::forward_as_tuple(MaterialName::MaterialOne),
        std::forward_as_tuple());
    auto f = std::make_unique<FluxArray[]>(3);
    auto vf = std::make_unique<ForceArray[]>(1);
    for (int b = 0; b < nb; ++b) {
      Block &blk = mb->second;
      for (unsigned e = 0; e < NE; ++e)
        std::memcpy(&blk.GetAverageBuffer(MF::ASOE()[e])[0][0][0],
                    u + (std::size_t(b) * NE + e) * CELLS, CELLS * sizeof(double));
      std::memset(f.get(), 0, 3 * sizeof(FluxArray));
      std::memset(vf.get(), 0, sizeof(ForceArray));
      solver.UpdateConvectiveFluxes(*mb, cell_size, f[0], f[1], f[2], vf[0]);
      std::size_t const o = std::size_t(b) * NE * FACES;
      std::memcpy(fx + o, &f[0][0][0][0][0], sizeof(FluxArray));
      std::memcpy(fy + o, &f[1][0][0][0][0], sizeof(FluxArray));
      std::memcpy(fz + o, &f[2][0][0][0][0], sizeof(FluxArray));
    }
  } catch (std::exception const &e) {
    g_error = e.what();
    return -1;
  }
  return 0;
}

}  // extern "C"
