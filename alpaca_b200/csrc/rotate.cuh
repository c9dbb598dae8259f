// The rotation that makes every 3D face an x face.
#pragma once

#include "layout.cuh"

namespace alp {

// Conserved field held in canonical slot c for a face of direction dir: mass
// and energy stay; the momenta rotate so that the principal one comes first
// and the two minor ones follow in the order in which the reference's
// characteristic projection sums them for dir (state_reconstruction.h:35-58:
// Y, Z | Z, X | X, Y). Every 3D face is then the x-face computation
// (face_compute<3, 0>) of its rotated stencil, with the flux rotated back: one
// code path for all three directions. The reference's projection order is
// kept for every direction; for y faces the two minor momenta are also
// numbered the other way round than Minor<1>, which negates and exchanges the
// two minor characteristic variables (WENO5 is odd, the back-projection adds
// their terms in an order-free way) and leaves every other operation as it
// is, so the strict build still reproduces the reference bit for bit.
__host__ __device__ constexpr int canon_field(int dir, int c) {
  return c < MOMX ? c : MOMX + (dir + c - MOMX) % 3;
}

}  // namespace alp
