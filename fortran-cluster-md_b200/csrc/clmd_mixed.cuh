// Device helpers shared by the mixed-precision kernels (k_cycle, k_force,
// k_ens): the FP32 reciprocal of the pair terms and the closed-form
// Nose-Hoover velocity solve.
#pragma once

#include <math.h>

// 1/x by the hardware's approximate reciprocal (PTX rcp.approx.ftz.f32, at
// most 1 ulp from the exact quotient): x = r^2 of a pair inside the cut-off,
// a normal number.  The pair terms are FP32 anyway; the IEEE-rounded
// division costs several instructions more per pair.
__device__ __forceinline__ float clmd_rcp_f32(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// The implicit Nose-Hoover velocity step of int-verlet-nh-mav.f:105-147 in
// closed form (mixed precision).  The reference's Newton sweeps stop at the
// fixed point v (1 + dth p) = V + dth a =: W, p = psi1 + (m sum v^2 - 3NkT)
// dth / Q.  With S = m sum W^2 the new PSI is therefore the root of
//   f(p) = p - psi1 - (S / (1 + dth p)^2 - 3NkT) dth / Q,
// which is increasing and concave for 1 + dth p > 0 (one root), and every
// velocity is W / (1 + dth p): one reduction instead of a reduction per
// sweep.  Newton's method from psi1, two or three steps in practice; the
// step limit is 1e-13 of the terms' scale (|p| + |psi1| + (S + 3NkT) dth/Q;
// rounding noise in f is a few 1e-16 of it, so a tighter limit can stall).
// False (no convergence) if the root is not finite or the iteration does not
// settle, as the reference's STOP.
__device__ __forceinline__ bool clmd_nh_root(double S, double psi1, double nkt3, double dth,
                                             double Q, double& p) {
  const double k0 = dth / Q;
  const double scale = fabs(psi1) + k0 * (S + fabs(nkt3));
  p = psi1;
  for (int it = 0; it < 64; it++) {
    const double c = 1.0 / (1.0 + dth * p);
    const double f = p - psi1 - (S * c * c - nkt3) * k0;
    const double fp = 1.0 + 2.0 * S * dth * k0 * c * c * c;
    const double d = f / fp;
    p = p - d;
    if (!(fabs(d) > 1e-13 * (scale + fabs(p)))) return isfinite(p) && 1.0 + dth * p > 0.0;
  }
  return false;
}
