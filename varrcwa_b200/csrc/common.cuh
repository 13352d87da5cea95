// Common device/host helpers for the varRCWA B200 engine.
//
// Matrices are complex128, column-major, leading dimension n (the layout of
// Eigen::MatrixXcs and of the reference GPU path, src/gpu/types.cuh:18).
#pragma once

#include <string>
#include <utility>

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

namespace vrc {

typedef double2 cplx;  // (re, im)

__host__ __device__ __forceinline__ cplx mk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ cplx cadd(cplx a, cplx b) { return mk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cplx csub(cplx a, cplx b) { return mk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ cplx cmulc(cplx a, cplx b) {  // conj(a) * b
  return mk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ cplx cconj(cplx a) { return mk(a.x, -a.y); }
__host__ __device__ __forceinline__ cplx cscale(cplx a, double s) { return mk(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ cplx cneg(cplx a) { return mk(-a.x, -a.y); }
__host__ __device__ __forceinline__ double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ __forceinline__ double cabs1(cplx a) { return fabs(a.x) + fabs(a.y); }
__device__ __forceinline__ double cabs(cplx a) { return hypot(a.x, a.y); }
// a * b + c
__host__ __device__ __forceinline__ cplx cfma(cplx a, cplx b, cplx c) {
  return mk(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
// Smith's algorithm for a / b.
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, d = b.x + b.y * r;
    return mk((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  } else {
    double r = b.x / b.y, d = b.y + b.x * r;
    return mk((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
}
__device__ __forceinline__ cplx cinv(cplx b) { return cdiv(mk(1.0, 0.0), b); }
// 1 / b as conj(b) / |b|^2 with one real reciprocal, for |b| well inside the
// double range (no intermediate over- or underflow); Smith's form otherwise.
__device__ __forceinline__ cplx cinv_fast(cplx b) {
  const double m = fmax(fabs(b.x), fabs(b.y));
  if (m > 1e-150 && m < 1e150) {
    const double r = 1.0 / (b.x * b.x + b.y * b.y);
    return mk(b.x * r, -b.y * r);
  }
  return cinv(b);
}
__device__ __forceinline__ cplx cexp_i(cplx g, double t) {
  // exp(i * g * t)
  double re = -g.y * t, im = g.x * t;
  double e = exp(re), s, c;
  sincos(im, &s, &c);
  return mk(e * c, e * s);
}
// Principal square root.
__device__ __forceinline__ cplx csqrt(cplx a) {
  double r = hypot(a.x, a.y);
  if (r == 0.0) return mk(0.0, 0.0);
  double t = sqrt(0.5 * (r + fabs(a.x)));
  if (a.x >= 0.0) return mk(t, 0.5 * a.y / t);
  return mk(0.5 * fabs(a.y) / t, copysign(t, a.y));
}

__device__ __forceinline__ cplx ld(const cplx* p) { return __ldg(p); }

// Status codes shared with the C-ABI (include/vrc.h).
enum {
  ST_OK = 0,
  ST_EINVAL = 1,
  ST_ECUDA = 2,
  ST_ENOMEM = 3,
  ST_ESINGULAR = 4,
  ST_ENOCONV = 5,
  ST_ENONFINITE = 6,
  ST_ETIMEOUT = 7,
  ST_EDEPTH = 8,
  ST_ENODEV = 9,
};

}  // namespace vrc

#define VRC_CUDA_CHECK(x)                                                            \
  do {                                                                               \
    cudaError_t _e = (x);                                                            \
    if (_e != cudaSuccess) {                                                         \
      fprintf(stderr, "[vrc] CUDA error %s at %s:%d\n", cudaGetErrorString(_e), __FILE__, \
              __LINE__);                                                             \
      throw vrc::CudaError(_e);                                                      \
    }                                                                                \
  } while (0)

namespace vrc {
struct CudaError {
  cudaError_t err;
  explicit CudaError(cudaError_t e) : err(e) {}
};
struct StatusError {
  int status;
  std::string what;
  StatusError(int s, std::string w) : status(s), what(std::move(w)) {}
};
}  // namespace vrc
