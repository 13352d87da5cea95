// Elementwise kernels of the integrators: propagation-constant branch,
// Simpson-rule perturbative segment with its fused max-abs error, the
// A/B combinations of basis projections, diagonal phase scalings and the
// per-order diffraction powers.
#include "common.cuh"
#include "kernels.h"

namespace vrc {
namespace {

inline dim3 grid_for(long long total, int batch, int threads = 256) {
  long long bx = (total + threads - 1) / threads;
  if (bx > 1024) bx = 1024;
  if (bx < 1) bx = 1;
  return dim3((unsigned)bx, batch);
}

// gamma = sqrt(lambda) on the branch Im >= 0, flipped when |Im| < |Re| and
// Re < 0 (GammaSqrtOp, src/rcwa/WaveEquationSolver.cpp:8-22); also 1/gamma.
__global__ void gamma_kernel(const cplx* const* __restrict__ lams, cplx* const* __restrict__ gams,
                             cplx* const* __restrict__ invgams, int n) {
  const cplx* l = lams[blockIdx.y];
  cplx* g = gams[blockIdx.y];
  cplx* ig = invgams[blockIdx.y];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    cplx v = csqrt(l[i]);
    if (v.y < 0.0) v = cneg(v);
    if (fabs(v.y) < fabs(v.x) && v.x < 0.0) v = cneg(v);
    g[i] = v;
    ig[i] = cinv(v);
  }
}

// C = A - B
__global__ void sub_kernel(const cplx* const* __restrict__ As, const cplx* const* __restrict__ Bs,
                           cplx* const* __restrict__ Cs, long long total) {
  const cplx* a = As[blockIdx.y];
  const cplx* b = Bs[blockIdx.y];
  cplx* c = Cs[blockIdx.y];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    c[i] = csub(a[i], b[i]);
}

// A = 0.5 (F + G), B = 0.5 (F - G)   (in place: F -> A, G -> B)
__global__ void ab_kernel(cplx* const* __restrict__ Fs, cplx* const* __restrict__ Gs, long long total) {
  cplx* f = Fs[blockIdx.y];
  cplx* g = Gs[blockIdx.y];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    cplx a = f[i], b = g[i];
    f[i] = cscale(cadd(a, b), 0.5);
    g[i] = cscale(csub(a, b), 0.5);
  }
}

// Simpson-rule segment (src/core/RedhefferIntegrator.cpp:317-399).  The
// reference sample of a segment is its midpoint sample, so the middle
// perturbation term (Pm - Pr) vanishes identically; the end terms are
//   dA_k = X_k + Y_k,  dB_k = X_k - Y_k,  X_k = W^-1 (P_k-Pr) V,  Y_k = V^-1 (Q_k-Qr) W.
__global__ void simpson_kernel(const SegDesc* __restrict__ segs, int n) {
  const SegDesc s = segs[blockIdx.y];
  const double k0 = s.k0;
  const double dz = s.z1 - s.z0;
  const cplx c = mk(0.0, dz / (12.0 * k0));
  const long long total = (long long)n * n;
  double errmax = 0.0;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    int j = (int)(idx / n), i = (int)(idx - (long long)j * n);
    cplx x0 = s.X0[idx], y0 = s.Y0[idx], x2 = s.X2[idx], y2 = s.Y2[idx];
    cplx dA0 = cadd(x0, y0), dB0 = csub(x0, y0), dA2 = cadd(x2, y2), dB2 = csub(x2, y2);
    cplx pfi = cexp_i(s.gam[i], dz / k0), pfj = cexp_i(s.gam[j], dz / k0);
    cplx tuu = cmul(c, cadd(cmul(pfi, dA0), cmul(dA2, pfj)));
    cplx rud = cneg(cmul(c, cadd(cmul(cmul(pfi, dB0), pfj), dB2)));
    cplx rdu = cneg(cmul(c, cadd(dB0, cmul(cmul(pfi, dB2), pfj))));
    cplx tdd = cmul(c, cadd(cmul(dA0, pfj), cmul(pfi, dA2)));
    errmax = fmax(errmax, fmax(fmax(cabs(tuu), cabs(rud)), fmax(cabs(rdu), cabs(tdd))));
    if (i == j) {
      tuu = cadd(tuu, pfi);
      tdd = cadd(tdd, pfi);
    }
    s.tuu[idx] = tuu;
    s.rud[idx] = rud;
    s.rdu[idx] = rdu;
    s.tdd[idx] = tdd;
  }
  // block max -> atomic max on the segment's error (non-negative doubles
  // order like their bit patterns)
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) errmax = fmax(errmax, __shfl_xor_sync(0xffffffffu, errmax, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = errmax;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) {
      if (!isfinite(v)) v = __longlong_as_double(0x7ff0000000000000LL);  // +inf
      atomicMax(reinterpret_cast<unsigned long long*>(s.err), (unsigned long long)__double_as_longlong(v));
    }
  }
}

// out = diag(x) * A   (row scaling), x = exp(i gamma t) when t != 0 else x
__global__ void phase_rows_kernel(const cplx* const* __restrict__ As, const cplx* const* __restrict__ gams,
                                  const double* __restrict__ ts, cplx* const* __restrict__ outs, int n) {
  const cplx* a = As[blockIdx.y];
  const cplx* g = gams[blockIdx.y];
  const double t = ts[blockIdx.y];
  cplx* o = outs[blockIdx.y];
  const long long total = (long long)n * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    int i = (int)(idx % n);
    o[idx] = cmul(cexp_i(g[i], t), a[idx]);
  }
}

__global__ void set_identity_kernel(cplx* const* __restrict__ As, int n, double diag) {
  cplx* a = As[blockIdx.y];
  const long long total = (long long)n * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    int j = (int)(idx / n), i = (int)(idx - (long long)j * n);
    a[idx] = mk(i == j ? diag : 0.0, 0.0);
  }
}

// C = alpha*A + beta*B + delta*I; a null A or B stands for zero
__global__ void axpby_kernel(const cplx* const* __restrict__ As, const cplx* const* __restrict__ Bs,
                             cplx* const* __restrict__ Cs, cplx alpha, cplx beta, double delta, int n) {
  const cplx* a = As[blockIdx.y];
  const cplx* b = Bs[blockIdx.y];
  cplx* c = Cs[blockIdx.y];
  const long long total = (long long)n * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    int j = (int)(idx / n), i = (int)(idx - (long long)j * n);
    cplx v = a ? cmul(alpha, a[idx]) : mk(0.0, 0.0);
    if (b) v = cfma(beta, b[idx], v);
    if (i == j) v.x += delta;
    c[idx] = v;
  }
}

// Per-order power for one incidence (RCWASolver::scatterPlaneWave,
// src/rcwa/RCWASolver.cpp:1636-1733): given field harmonics r = [rx; ry]
// and t = [tx; ty], the z components follow from div E = 0.
__global__ void order_power_kernel(const PowerDesc* __restrict__ pds, int m) {
  const PowerDesc d = pds[blockIdx.x];
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    double a = d.alpha[i], b = d.beta[i];
    cplx kr2 = mk(d.k0 * d.k0 * d.eps_in.x - a * a - b * b, d.k0 * d.k0 * d.eps_in.y);
    cplx kt2 = mk(d.k0 * d.k0 * d.eps_out.x - a * a - b * b, d.k0 * d.k0 * d.eps_out.y);
    cplx kzr = cneg(csqrt(kr2));
    cplx kzt = csqrt(kt2);
    cplx rx = d.r[i], ry = d.r[i + m], tx = d.t[i], ty = d.t[i + m];
    double R = 0.0, T = 0.0;
    if (kzr.x != 0.0 || kzr.y != 0.0) {
      cplx rz = cdiv(mk(a * rx.x + b * ry.x, a * rx.y + b * ry.y), kzr);
      R = fabs(kzr.x) * (cabs2(rx) + cabs2(ry) + cabs2(rz)) / (sqrt(d.eps_in.x) * d.k0);
    }
    if (kzt.x != 0.0 || kzt.y != 0.0) {
      cplx tz = cdiv(mk(a * tx.x + b * ty.x, a * tx.y + b * ty.y), kzt);
      T = fabs(kzt.x) * (cabs2(tx) + cabs2(ty) + cabs2(tz)) / (d.tnorm * d.k0);
    }
    d.R[i] = R;
    d.T[i] = T;
  }
}

// y = A x (n x n complex, one CTA per product, warp per 32 rows)
__global__ void matvec_kernel(const MatVecDesc* __restrict__ ds, int n) {
  const MatVecDesc d = ds[blockIdx.x];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    cplx acc = mk(0.0, 0.0);
    for (int k = 0; k < n; ++k) acc = cfma(d.A[(size_t)k * n + i], d.x[k], acc);
    d.y[i] = acc;
  }
}

}  // namespace

void gamma_batched(const cplx* const* lams, cplx* const* gams, cplx* const* invgams, int batch, int n,
                   cudaStream_t st) {
  if (batch <= 0) return;
  gamma_kernel<<<grid_for(n, batch), 256, 0, st>>>(lams, gams, invgams, n);
  VRC_CUDA_CHECK(cudaGetLastError());
}
void sub_batched(const cplx* const* A, const cplx* const* B, cplx* const* C, int batch, long long total,
                 cudaStream_t st) {
  if (batch <= 0) return;
  sub_kernel<<<grid_for(total, batch), 256, 0, st>>>(A, B, C, total);
  VRC_CUDA_CHECK(cudaGetLastError());
}
void ab_batched(cplx* const* F, cplx* const* G, int batch, long long total, cudaStream_t st) {
  if (batch <= 0) return;
  ab_kernel<<<grid_for(total, batch), 256, 0, st>>>(F, G, total);
  VRC_CUDA_CHECK(cudaGetLastError());
}
void simpson_batched(const SegDesc* d_segs, int batch, int n, cudaStream_t st) {
  if (batch <= 0) return;
  long long total = (long long)n * n;
  long long bx = (total + 255) / 256;
  if (bx > 256) bx = 256;
  simpson_kernel<<<dim3((unsigned)bx, batch), 256, 0, st>>>(d_segs, n);
  VRC_CUDA_CHECK(cudaGetLastError());
}
void phase_rows_batched(const cplx* const* A, const cplx* const* gam, const double* t, cplx* const* out, int batch,
                        int n, cudaStream_t st) {
  if (batch <= 0) return;
  phase_rows_kernel<<<grid_for((long long)n * n, batch), 256, 0, st>>>(A, gam, t, out, n);
  VRC_CUDA_CHECK(cudaGetLastError());
}
void set_identity_batched(cplx* const* A, int batch, int n, double diag, cudaStream_t st) {
  if (batch <= 0) return;
  set_identity_kernel<<<grid_for((long long)n * n, batch), 256, 0, st>>>(A, n, diag);
  VRC_CUDA_CHECK(cudaGetLastError());
}
void axpby_batched(const cplx* const* A, const cplx* const* B, cplx* const* C, cplx alpha, cplx beta, double delta,
                   int batch, int n, cudaStream_t st) {
  if (batch <= 0) return;
  axpby_kernel<<<grid_for((long long)n * n, batch), 256, 0, st>>>(A, B, C, alpha, beta, delta, n);
  VRC_CUDA_CHECK(cudaGetLastError());
}
void order_power_batched(const PowerDesc* d, int batch, int m, cudaStream_t st) {
  if (batch <= 0) return;
  order_power_kernel<<<batch, 128, 0, st>>>(d, m);
  VRC_CUDA_CHECK(cudaGetLastError());
}
void matvec_batched(const MatVecDesc* d, int batch, int n, cudaStream_t st) {
  if (batch <= 0) return;
  matvec_kernel<<<batch, 256, 0, st>>>(d, n);
  VRC_CUDA_CHECK(cudaGetLastError());
}

}  // namespace vrc
