// TEST INFRASTRUCTURE ONLY — the drop-in adapter of the integration guide,
// compiled against the reference's own headers to show that the library's C
// ABI fits ALPACA's convective-term plugin surface.
//
// B200ConvectiveTermSolver is a concretization of the reference's CRTP base
// ConvectiveTermSolver<Derived> (solvers/convective_term_contributions/
// convective_term_solver.h:67-81), beside FiniteVolumeScheme and
// FluxSplittingScheme: UpdateImplementation stages the block's average buffer
// (halos filled, reference layout) on the device, calls alp_convective_fluxes
// and copies the three flux arrays back into the reference's arrays. The
// scheme is taken from the reference's compile-time settings
// (user_specifications/*.h), whose enum values alp_scheme carries unchanged.
#ifndef B200_CONVECTIVE_TERM_SOLVER_H
#define B200_CONVECTIVE_TERM_SOLVER_H

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "alpaca_b200.h"
#include "materials/equations_of_state/stiffened_gas_safe.h"
#include "solvers/convective_term_contributions/convective_term_solver.h"
#include "user_specifications/numerical_setup.h"
#include "user_specifications/riemann_solver_settings.h"
#include "user_specifications/state_reconstruction_settings.h"
#include "user_specifications/stencil_setup.h"

// The library's selection equal to the reference's compile-time one.
inline alp_scheme AlpSchemeFromSettings(int precision = ALP_FP64) {
  alp_scheme s;
  alp_scheme_default(&s);
  s.convective_term_solver = static_cast<int>(convective_term_solver);
  s.state_reconstruction = static_cast<int>(state_reconstruction_type);
  s.reconstruction_stencil = static_cast<int>(reconstruction_stencil);
  s.riemann_solver = static_cast<int>(FiniteVolumeSettings::riemann_solver);
  s.signal_speed = static_cast<int>(FiniteVolumeSettings::signal_speed_selection);
  s.flux_splitting = static_cast<int>(FluxSplittingSettings::flux_splitting_scheme);
  s.time_integrator = static_cast<int>(time_integrator);
  s.precision = precision;
  return s;
}

class B200ConvectiveTermSolver : public ConvectiveTermSolver<B200ConvectiveTermSolver> {
  friend ConvectiveTermSolver;

  static constexpr std::size_t kCells = std::size_t(CC::TCX()) * CC::TCY() * CC::TCZ();
  static constexpr std::size_t kFlux =
      std::size_t(MF::ANOE()) * (CC::ICX() + 1) * (CC::ICY() + 1) * (CC::ICZ() + 1);
  static constexpr int kDim =
      CC::DIM() == Dimension::One ? 1 : (CC::DIM() == Dimension::Two ? 2 : 3);

  alp_scheme const scheme_;
  double *d_block_ = nullptr;  // one block's average buffer [NE][TCX][TCY][TCZ]
  double *d_flux_ = nullptr;   // fx, fy, fz, each [NE][ICX+1][ICY+1][ICZ+1]
  cudaStream_t stream_ = nullptr;

  static void Check(cudaError_t e, char const *what) {
    if (e != cudaSuccess)
      throw std::runtime_error(std::string("B200ConvectiveTermSolver: ") + what + ": " +
                               cudaGetErrorString(e));
  }

  void UpdateImplementation(
      std::pair<MaterialName const, Block> const &mat_block, double const cell_size,
      double (&fluxes_x)[MF::ANOE()][CC::ICX() + 1][CC::ICY() + 1][CC::ICZ() + 1],
      double (&fluxes_y)[MF::ANOE()][CC::ICX() + 1][CC::ICY() + 1][CC::ICZ() + 1],
      double (&fluxes_z)[MF::ANOE()][CC::ICX() + 1][CC::ICY() + 1][CC::ICZ() + 1],
      double (&)[MF::ANOE()][CC::ICX()][CC::ICY()][CC::ICZ()]) const {
    EquationOfState const &eos =
        material_manager_.GetMaterial(mat_block.first).GetEquationOfState();
    alp_material const m{eos.Gamma(), eos.B(),
                         dynamic_cast<StiffenedGasSafe const *>(&eos) != nullptr ? 1 : 0};
    Block const &b = mat_block.second;
    for (unsigned e = 0; e < MF::ANOE(); ++e)
      Check(cudaMemcpyAsync(d_block_ + e * kCells, &b.GetAverageBuffer(MF::ASOE()[e])[0][0][0],
                            kCells * sizeof(double), cudaMemcpyHostToDevice, stream_),
            "copy of the average buffer");
    // the reference's schemes add their fluxes to the caller's arrays (zeroed
    // by SpaceSolver::UpdateFluxes), and so does alp_convective_fluxes: the
    // arrays of the active directions go to the device and come back
    double *const out[3] = {&fluxes_x[0][0][0][0], &fluxes_y[0][0][0][0], &fluxes_z[0][0][0][0]};
    for (int d = 0; d < kDim; ++d)
      Check(cudaMemcpyAsync(d_flux_ + d * kFlux, out[d], kFlux * sizeof(double),
                            cudaMemcpyHostToDevice, stream_),
            "copy of the flux arrays");
    if (alp_convective_fluxes(kDim, &scheme_, &m, d_block_, 1, cell_size, d_flux_,
                              d_flux_ + kFlux, d_flux_ + 2 * kFlux, stream_) != ALP_OK)
      throw std::runtime_error(alp_last_error());
    for (int d = 0; d < kDim; ++d)
      Check(cudaMemcpyAsync(out[d], d_flux_ + d * kFlux, kFlux * sizeof(double),
                            cudaMemcpyDeviceToHost, stream_),
            "copy of the fluxes");
    Check(cudaStreamSynchronize(stream_), "stream synchronisation");
  }

public:
  B200ConvectiveTermSolver(MaterialManager const &material_manager,
                           EigenDecomposition const &eigendecomposition_calculator,
                           int precision = ALP_FP64)
      : ConvectiveTermSolver(material_manager, eigendecomposition_calculator),
        scheme_(AlpSchemeFromSettings(precision)) {
    Check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
    Check(cudaMalloc(&d_block_, MF::ANOE() * kCells * sizeof(double)), "block buffer");
    Check(cudaMalloc(&d_flux_, 3 * kFlux * sizeof(double)), "flux buffers");
  }
  ~B200ConvectiveTermSolver() {
    cudaFree(d_flux_);
    cudaFree(d_block_);
    if (stream_)
      cudaStreamDestroy(stream_);
  }
  B200ConvectiveTermSolver(B200ConvectiveTermSolver const &) = delete;
  B200ConvectiveTermSolver &operator=(B200ConvectiveTermSolver const &) = delete;
};

#endif  // B200_CONVECTIVE_TERM_SOLVER_H
