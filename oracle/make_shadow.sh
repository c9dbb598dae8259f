#!/bin/sh
# Generates ALPACA's compile-time selection headers for one oracle variant:
# copies of the reference's user_specifications/{equation,riemann_solver,
# state_reconstruction}_settings.h and stencil_setup.h with the selection enums
# edited, written to $OUT/user_specifications/ (under oracle/_ref/, never
# committed).
#   make_shadow.sh REF_SRC OUT SOLVER RECON [STENCIL RIEMANN SIGNAL SPLITTING]
#   SOLVER: FiniteVolume | FluxSplitting    RECON: Characteristic | Primitive
#   STENCIL: WENO5 (default) | WENO5Z | TENO5 | WENO3 | FirstOrder
#   RIEMANN: Hllc (default) | Hllc_LM | Hll
#   SIGNAL: Einfeldt (default) | Davis | Toro | Arithmetic
#   SPLITTING: Roe (default) | LocalLaxFriedrichs | GlobalLaxFriedrichs | Roe_M |
#              LocalLaxFriedrichs_M
#   INTEGRATOR: RK3 (default) | RK2   (numerical_setup.h)
set -e
SRC="$1"; OUT="$2"; SOLVER="$3"; RECON="$4"
STENCIL="${5:-WENO5}"; RIEMANN="${6:-Hllc}"; SIGNAL="${7:-Einfeldt}"; SPLITTING="${8:-Roe}"
INTEGRATOR="${9:-RK3}"
mkdir -p "$OUT/user_specifications"
U="$SRC/user_specifications"
D="$OUT/user_specifications"
sed -e 's/active_equations = EquationSet::[A-Za-z]*;/active_equations = EquationSet::Euler;/' \
  "$U/equation_settings.h" > "$D/equation_settings.h"
# the selections may be split over two lines in the reference headers
sed -e ':a' -e 'N' -e '$!ba' \
  -e "s/convective_term_solver =[[:space:]]*ConvectiveTermSolvers::[A-Za-z]*;/convective_term_solver = ConvectiveTermSolvers::$SOLVER;/" \
  -e "s/flux_splitting_scheme =[[:space:]]*FluxSplitting::[A-Za-z_]*;/flux_splitting_scheme = FluxSplitting::$SPLITTING;/" \
  -e "s/riemann_solver =[[:space:]]*RiemannSolvers::[A-Za-z_]*;/riemann_solver = RiemannSolvers::$RIEMANN;/" \
  -e "s/signal_speed_selection =[[:space:]]*SignalSpeed::[A-Za-z_]*;/signal_speed_selection = SignalSpeed::$SIGNAL;/" \
  "$U/riemann_solver_settings.h" > "$D/riemann_solver_settings.h"
sed -e ':a' -e 'N' -e '$!ba' \
  -e "s/state_reconstruction_type =[[:space:]]*StateReconstructionType::[A-Za-z]*;/state_reconstruction_type = StateReconstructionType::$RECON;/" \
  "$U/state_reconstruction_settings.h" > "$D/state_reconstruction_settings.h"
sed -e ':a' -e 'N' -e '$!ba' \
  -e "s/ReconstructionStencils reconstruction_stencil =[[:space:]]*ReconstructionStencils::[A-Za-z0-9]*;/ReconstructionStencils reconstruction_stencil = ReconstructionStencils::$STENCIL;/" \
  "$U/stencil_setup.h" > "$D/stencil_setup.h"
sed -e "s/time_integrator = TimeIntegrators::RK[0-9];/time_integrator = TimeIntegrators::$INTEGRATOR;/" \
  "$U/numerical_setup.h" > "$D/numerical_setup.h"
grep -q "time_integrator = TimeIntegrators::$INTEGRATOR;" "$D/numerical_setup.h"
grep -q "EquationSet::Euler;" "$D/equation_settings.h"
grep -q "convective_term_solver = ConvectiveTermSolvers::$SOLVER;" "$D/riemann_solver_settings.h"
grep -q "flux_splitting_scheme = FluxSplitting::$SPLITTING;" "$D/riemann_solver_settings.h"
grep -q "riemann_solver = RiemannSolvers::$RIEMANN;" "$D/riemann_solver_settings.h"
grep -q "signal_speed_selection = SignalSpeed::$SIGNAL;" "$D/riemann_solver_settings.h"
grep -q "state_reconstruction_type = StateReconstructionType::$RECON;" "$D/state_reconstruction_settings.h"
grep -q "reconstruction_stencil = ReconstructionStencils::$STENCIL;" "$D/stencil_setup.h"
