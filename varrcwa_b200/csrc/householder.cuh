// Complex Householder reflectors shared by the Hessenberg reduction and the
// QR iteration (published construction, Golub & Van Loan 5.1.13, complex form).
#pragma once

#include "common.cuh"

namespace vrc {

// Reflector H = I - tau v v^H with v = (1, x*scale) mapping (alpha, x) to
// (beta, 0), beta real; xnorm2 = ||x||^2.
__device__ __forceinline__ void householder(cplx alpha, double xnorm2, double* beta, cplx* tau, cplx* scale) {
  if (xnorm2 == 0.0 && alpha.y == 0.0) {
    *beta = alpha.x;
    *tau = mk(0.0, 0.0);
    *scale = mk(0.0, 0.0);
    return;
  }
  const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2);
  const double b = alpha.x >= 0.0 ? -nrm : nrm;
  // alpha - beta = (alpha.x + sign(alpha.x) nrm, alpha.y): |real part| >= nrm > 0,
  // so both reciprocals are safe; they are independent and overlap.
  const double ux = alpha.x - b;
  const double rb = 1.0 / b, rd = 1.0 / (ux * ux + alpha.y * alpha.y);
  *beta = b;
  *tau = mk(-ux * rb, -alpha.y * rb);
  *scale = mk(ux * rd, -alpha.y * rd);
}

// Two-element reflector for (a, b): returns the new leading entry, tau and
// v2 (v = (1, v2)).
__device__ __forceinline__ void refl2(cplx a, cplx b, cplx* beta, cplx* tau, cplx* v2) {
  double b0;
  cplx t, sc;
  householder(a, cabs2(b), &b0, &t, &sc);
  if (t.x == 0.0 && t.y == 0.0) {
    *beta = a;
    *tau = t;
    *v2 = mk(0.0, 0.0);
    return;
  }
  *beta = mk(b0, 0.0);
  *tau = t;
  *v2 = cmul(b, sc);
}

constexpr double EIG_ULP = 2.220446049250313e-16;  // 2^-52
constexpr double EIG_SAFMIN = 2.2250738585072014e-308;

}  // namespace vrc
