// Kernels of the layer-stack forward solve and its adjoint (gradients of
// per-order power with respect to permittivity pixels).
//
// Complex gradients follow dL = Re(sum(conj(G) * dZ)).  With every eigen
// basis held fixed, a perturbation (dP, dQ) of a z-uniform layer changes only
// the layer's own-basis blocks, by the first-order term of the perturbative
// segment (src/core/RedhefferIntegrator.cpp:317-399) with the z-integrals
// done exactly:
//   dtuu = dtdd =  K_E o (W^-1 dP V + V^-1 dQ W),
//   drud = drdu = -K_D o (W^-1 dP V - V^-1 dQ W),
//   K_E[i,j] = i/(2k0) int_0^d exp(i(g_i(d-z) + g_j z)/k0) dz,
//   K_D[i,j] = i/(2k0) int_0^d exp(i(g_i + g_j) z/k0) dz.
// These are divided differences of exponentials; nearly equal eigenvalues take
// the series form, so degenerate modes need no separate treatment.
#include "common.cuh"
#include "kernels.h"

namespace vrc {

namespace {

constexpr double PI_D = 3.1415926535897932;  // src/rcwa/defns.h:25

inline dim3 grid_for(long long total, int batch, int threads = 256) {
  long long bx = (total + threads - 1) / threads;
  if (bx > 1024) bx = 1024;
  if (bx < 1) bx = 1;
  return dim3((unsigned)bx, (unsigned)batch);
}

__device__ __forceinline__ cplx cexp(cplx x) {
  double s, c;
  sincos(x.y, &s, &c);
  const double e = exp(x.x);
  return mk(e * c, e * s);
}

// (exp(x) - 1) / x for |x| < 0.1 by its Taylor series (terms to x^10).
__device__ __forceinline__ cplx phi_series(cplx x) {
  cplx s = mk(1.0, 0.0), term = mk(1.0, 0.0);
#pragma unroll
  for (int k = 2; k < 12; ++k) {
    term = cscale(cmul(term, x), 1.0 / k);
    s = cadd(s, term);
  }
  return s;
}

// int_0^d exp(i (a (d - z) + b z) / k0) dz
__device__ cplx int_exp2(cplx a, cplx b, double d, double k0) {
  const double t = d / k0;
  const cplx ea = cexp_i(a, t);
  const cplx x = mk(-(b.y - a.y) * t, (b.x - a.x) * t);  // i (b - a) d / k0
  if (fabs(x.x) + fabs(x.y) < 0.1) return cscale(cmul(ea, phi_series(x)), d);
  const cplx eb = cexp_i(b, t);
  return cscale(cdiv(csub(eb, ea), x), d);
}

// int_0^d exp(i s z / k0) dz
__device__ cplx int_exp1(cplx s, double d, double k0) {
  const double t = d / k0;
  const cplx x = mk(-s.y * t, s.x * t);  // i s d / k0
  if (fabs(x.x) + fabs(x.y) < 0.1) return cscale(phi_series(x), d);
  return cscale(cdiv(csub(cexp(x), mk(1.0, 0.0)), x), d);
}

__global__ void scale_kernel(const cplx* const* __restrict__ As, const cplx* const* __restrict__ rss,
                             const cplx* const* __restrict__ css, cplx* const* __restrict__ outs, int n) {
  const cplx* a = As[blockIdx.y];
  const cplx* rs = rss ? rss[blockIdx.y] : nullptr;
  const cplx* cs = css ? css[blockIdx.y] : nullptr;
  cplx* o = outs[blockIdx.y];
  const long long total = (long long)n * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    cplx v = a[idx];
    if (rs) v = cmul(rs[i], v);
    if (cs) v = cmul(v, cs[j]);
    o[idx] = v;
  }
}

__global__ void phase_vec_kernel(const cplx* const* __restrict__ gams, const double* __restrict__ ts,
                                 cplx* const* __restrict__ outs, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) outs[blockIdx.y][i] = cexp_i(gams[blockIdx.y][i], ts[blockIdx.y]);
}

__global__ void layer_adjoint_kernel(const LayerAdjDesc* __restrict__ ds, int n) {
  const LayerAdjDesc d = ds[blockIdx.y];
  const long long total = (long long)n * n;
  const cplx c = mk(0.0, 0.5 / d.k0);  // i / (2 k0)
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    const cplx gi = d.gam[i], gj = d.gam[j];
    const cplx KE = cmul(c, int_exp2(gi, gj, d.d, d.k0));
    const cplx KD = cmul(c, int_exp1(cadd(gi, gj), d.d, d.k0));
    const cplx gA = cmulc(KE, cadd(d.gtdd[idx], d.gtuu[idx]));
    const cplx gB = cneg(cmulc(KD, cadd(d.grud[idx], d.grdu[idx])));
    d.gS[idx] = cadd(gA, gB);
    d.gD[idx] = csub(gA, gB);
  }
}

// The thickness enters a layer's own-basis blocks only through
// X = diag(exp(i gam d / k0)); dX/dd = (i gam / k0) X.
__global__ void thick_adjoint_kernel(const ThickAdjDesc* __restrict__ ds, int n) {
  const ThickAdjDesc d = ds[blockIdx.x];
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const size_t ii = (size_t)i * n + i;
    const cplx g = cadd(d.gtdd[ii], d.gtuu[ii]);
    const cplx dx = cmul(mk(-d.gam[i].y / d.k0, d.gam[i].x / d.k0), d.x[i]);  // (i gam / k0) x
    s += g.x * dx.x + g.y * dx.y;                                              // Re(conj(g) dx)
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    *d.out = t;
  }
}

__global__ void interface_e_kernel(const IfFieldDesc* __restrict__ ds, int n) {
  const IfFieldDesc d = ds[blockIdx.x];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    cplx s = mk(0.0, 0.0);
    for (int k = 0; k < n; ++k) s = cfma(d.W[(size_t)k * n + i], cadd(d.ap[k], d.am[k]), s);
    d.e[i] = s;
  }
}

// Ex, Ey at pixel (p, q) = sum over harmonics of e_k exp(i (alpha_k x_p + beta_k y_q))
__global__ void field_image_kernel(const IfFieldDesc* __restrict__ ds, int m, int ngx, int ngy) {
  const IfFieldDesc d = ds[blockIdx.y];
  if (!d.img) return;
  const int npix = ngx * ngy;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < npix; idx += gridDim.x * blockDim.x) {
    const int q = idx / ngx, p = idx - q * ngx;
    const double x = d.Lx * p / ngx, y = d.Ly * q / ngy;
    cplx ex = mk(0.0, 0.0), ey = mk(0.0, 0.0);
    for (int k = 0; k < m; ++k) {
      double sn, cs;
      sincos(d.alpha[k] * x + d.beta[k] * y, &sn, &cs);
      const cplx ph = mk(cs, sn);
      ex = cfma(d.e[k], ph, ex);
      ey = cfma(d.e[m + k], ph, ey);
    }
    d.img[idx] = ex;
    d.img[npix + idx] = ey;
  }
}

__global__ void vec_axpy_kernel(const cplx* const* __restrict__ as, const cplx* const* __restrict__ bs, cplx s,
                                cplx* const* __restrict__ ys, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ys[blockIdx.y][i] = cfma(s, bs[blockIdx.y][i], as[blockIdx.y][i]);
}

// dL/dP, dL/dQ of Layer::waveEqnCoeff (src/rcwa/Layer.cpp:36-171, periodic)
// -> dL/dfe11, dL/dfe22 and Z = dL/dF1 Kx + dL/dF2 Ky (F = fe33^-1 [Kx Ky]).
__global__ void pq_adjoint_kernel(const PQAdjDesc* __restrict__ ds, int m) {
  const PQAdjDesc d = ds[blockIdx.y];
  const int n = 2 * m;
  const double k2 = d.k0 * d.k0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < m * m; idx += gridDim.x * blockDim.x) {
    const int i = idx % m, j = idx / m;
    auto at = [&](const cplx* M, int r, int col) { return M[(size_t)col * n + r]; };
    d.g11[idx] = cscale(at(d.gQ, m + i, j), k2);
    d.g22[idx] = cscale(at(d.gQ, i, m + j), -k2);
    const double ai = d.alpha[i], bi = d.beta[i], aj = d.alpha[j], bj = d.beta[j];
    const cplx gF2 = cadd(cscale(at(d.gP, i, j), ai), cscale(at(d.gP, m + i, j), bi));
    const cplx gF1 = cneg(cadd(cscale(at(d.gP, i, m + j), ai), cscale(at(d.gP, m + i, m + j), bi)));
    d.Z[idx] = cadd(cscale(gF1, aj), cscale(gF2, bj));
  }
}

// Twiddle factor of FourierSolver1D (src/rcwa/FourierSolver1D.cpp:11-41) for
// harmonic p - half and cell [x0, x1] of a period D.
__device__ cplx twiddle(int p, int half, double x0, double x1, double D) {
  const int mm = p - half;
  const double w = x1 - x0;
  if (mm == 0) return mk(w / D, 0.0);
  double sn, cs;
  sincos(-(mm * PI_D * (x1 + x0) / D), &sn, &cs);
  const double amp = sin(PI_D * mm * w / D) / (PI_D * mm);
  return mk(amp * cs, amp * sn);
}

// In-place inverse of a t x t column-major matrix by one warp (Gauss-Jordan,
// partial pivoting).  Returns false on a zero pivot.
__device__ bool warp_inverse(cplx* a, cplx* fcol, int* piv, int t, int lane) {
  bool ok = true;
  for (int k = 0; k < t; ++k) {
    double best = -1.0;
    int p = t;
    for (int i = k + lane; i < t; i += 32) {
      double v = cabs1(a[k * t + i]);
      if (v > best) { best = v; p = i; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double ob = __shfl_xor_sync(0xffffffffu, best, o);
      int op = __shfl_xor_sync(0xffffffffu, p, o);
      if (ob > best || (ob == best && op < p)) { best = ob; p = op; }
    }
    if (!(best > 0.0)) { ok = false; p = k; }
    if (lane == 0) piv[k] = p;
    if (p != k)
      for (int j = lane; j < t; j += 32) {
        cplx tmp = a[j * t + k];
        a[j * t + k] = a[j * t + p];
        a[j * t + p] = tmp;
      }
    __syncwarp();
    const cplx ip = (best > 0.0) ? cinv(a[k * t + k]) : mk(1.0, 0.0);
    for (int i = lane; i < t; i += 32) fcol[i] = a[k * t + i];
    __syncwarp();
    for (int j = lane; j < t; j += 32) {
      cplx v = (j == k) ? mk(1.0, 0.0) : a[j * t + k];
      a[j * t + k] = cmul(v, ip);
    }
    __syncwarp();
    for (int j = lane; j < t; j += 32) {
      const cplx prow = a[j * t + k];
      for (int i = 0; i < t; ++i) {
        if (i == k) continue;
        cplx v = (j == k) ? mk(0.0, 0.0) : a[j * t + i];
        a[j * t + i] = csub(v, cmul(fcol[i], prow));
      }
    }
    __syncwarp();
  }
  for (int k = t - 1; k >= 0; --k) {
    const int p = piv[k];
    if (p != k)
      for (int i = lane; i < t; i += 32) {
        cplx tmp = a[k * t + i];
        a[k * t + i] = a[p * t + i];
        a[p * t + i] = tmp;
      }
    __syncwarp();
  }
  return ok;
}

constexpr int PX_THREADS = 256, PX_WARPS = PX_THREADS / 32;

// Per-warp scratch (complex elements) of pixel_adjoint_kernel.
__host__ __device__ inline int px_warp_scratch(int t) { return 3 * t * t + 2 * (2 * t - 1) + t; }

// One CTA per (stack, layer): dL/d(pixel) from dL/dfe11, dL/dfe22, dL/dfe33 on a
// uniform npy x npx grid (FourierSolver2D::solve, src/rcwa/FourierSolver2D.cpp:
// 43-349: Laurent rule for fe33, Li's inverse rule for fe11 (y strips) and
// fe22 (x columns)).  The per-strip Toeplitz inverses are recomputed here.
// The Toeplitz-diagonal sums of dL/dfe11 and dL/dfe22 (K11, K22: read by every
// strip) go to a global scratch of the layer (L2 resident), so that 15 x 15
// orders fit; the CTA has as many warps as its shared memory allows.
__global__ void __launch_bounds__(PX_THREADS)
    pixel_adjoint_kernel(const PixAdjDesc* __restrict__ ds, int nx, int ny, int npx, int npy) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const PixAdjDesc d = ds[blockIdx.x];
  const int P = 2 * nx - 1, Q = 2 * ny - 1, m = nx * ny, t = nx > ny ? nx : ny;
  const int NW = blockDim.x >> 5;
  cplx* Ex = reinterpret_cast<cplx*>(smem_raw);  // [npx][P]
  cplx* Ey = Ex + (size_t)P * npx;               // [npy][Q]
  cplx* gf = Ey + (size_t)Q * npy;               // [Q][P]
  cplx* H1 = gf + (size_t)P * Q;                 // [Q][npx]
  cplx* wsc = H1 + (size_t)Q * npx;              // per-warp scratch
  double* acc = reinterpret_cast<double*>(wsc + (size_t)NW * px_warp_scratch(t));  // [npy][npx]
  int* pivs = reinterpret_cast<int*>(acc + (size_t)npy * npx);
  cplx* K11 = d.kscr;                            // [Q][nx][nx]
  cplx* K22 = d.kscr + (size_t)Q * nx * nx;      // [P][ny][ny]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int NT = blockDim.x;

  for (int idx = tid; idx < P * npx; idx += NT) {
    const int c = idx / P, p = idx - c * P;
    Ex[idx] = twiddle(p, nx - 1, d.Lx * c / npx, d.Lx * (c + 1) / npx, d.Lx);
  }
  for (int idx = tid; idx < Q * npy; idx += NT) {
    const int r = idx / Q, q = idx - r * Q;
    Ey[idx] = twiddle(q, ny - 1, d.Ly * r / npy, d.Ly * (r + 1) / npy, d.Ly);
  }
  auto G = [&](const cplx* M, int a, int c, int b, int dd) { return M[(size_t)(b * ny + dd) * m + a * ny + c]; };
  // Toeplitz-diagonal sums of the three Fourier-block adjoints
  for (int idx = tid; idx < Q * nx * nx; idx += NT) {
    const int q = idx / (nx * nx), rem = idx - q * nx * nx, b = rem / nx, a = rem - b * nx;
    const int qq = q - (ny - 1);
    cplx s = mk(0.0, 0.0);
    for (int c = 0; c < ny; ++c) {
      const int dd = c - qq;
      if (dd >= 0 && dd < ny) s = cadd(s, G(d.g11, a, c, b, dd));
    }
    K11[idx] = s;
  }
  for (int idx = tid; idx < P * ny * ny; idx += NT) {
    const int p = idx / (ny * ny), rem = idx - p * ny * ny, dd = rem / ny, c = rem - dd * ny;
    const int pp = p - (nx - 1);
    cplx s = mk(0.0, 0.0);
    for (int a = 0; a < nx; ++a) {
      const int b = a - pp;
      if (b >= 0 && b < nx) s = cadd(s, G(d.g22, a, c, b, dd));
    }
    K22[idx] = s;
  }
  for (int idx = tid; idx < P * Q; idx += NT) {
    const int q = idx / P, p = idx - q * P;
    const int pp = p - (nx - 1), qq = q - (ny - 1);
    cplx s = mk(0.0, 0.0);
    for (int a = 0; a < nx; ++a) {
      const int b = a - pp;
      if (b < 0 || b >= nx) continue;
      for (int c = 0; c < ny; ++c) {
        const int dd = c - qq;
        if (dd >= 0 && dd < ny) s = cadd(s, G(d.g33, a, c, b, dd));
      }
    }
    gf[idx] = s;
  }
  __syncthreads();
  // fe33 (Laurent rule): four = Ex f^T Ey^T  ->  df = Ey^H-weighted sums
  for (int idx = tid; idx < Q * npx; idx += NT) {
    const int q = idx / npx, c = idx - q * npx;
    cplx s = mk(0.0, 0.0);
    for (int p = 0; p < P; ++p) s = cadd(s, cmulc(Ex[c * P + p], gf[q * P + p]));
    H1[idx] = s;
  }
  __syncthreads();
  for (int idx = tid; idx < npy * npx; idx += NT) {
    const int r = idx / npx, c = idx - r * npx;
    double s = 0.0;
    for (int q = 0; q < Q; ++q) {
      const cplx h = H1[q * npx + c], e = Ey[r * Q + q];  // h * conj(e)
      s += h.x * e.x + h.y * e.y;
    }
    acc[idx] = s;
  }
  __syncthreads();
  cplx* T = wsc + (size_t)warp * px_warp_scratch(t);
  cplx* gT = T + t * t;
  cplx* tmp = gT + t * t;
  cplx* gvec = tmp + t * t;        // 2t-1: Fourier coefficients of 1/eps
  cplx* gv = gvec + (2 * t - 1);   // 2t-1: Toeplitz-diagonal adjoint
  cplx* fcol = gv + (2 * t - 1);   // t
  int* piv = pivs + warp * 32;
  // fe11: one y strip r per warp pass; T_r = inv(Toep(Ex (1/eps[r, :])))
  for (int r = warp; r < npy; r += NW) {
    const cplx* er = d.eps + (size_t)r * npx;
    for (int p = lane; p < P; p += 32) {
      cplx s = mk(0.0, 0.0);
      for (int c = 0; c < npx; ++c) s = cadd(s, cmul(Ex[c * P + p], cinv(er[c])));
      gvec[p] = s;
    }
    __syncwarp();
    for (int idx = lane; idx < nx * nx; idx += 32) {
      const int k = idx / nx, i = idx - k * nx;
      T[k * nx + i] = gvec[nx - 1 + i - k];
    }
    __syncwarp();
    warp_inverse(T, fcol, piv, nx, lane);
    // gT[a,b] = sum_q conj(Ey[q, r]) K11[q, b, a]
    for (int idx = lane; idx < nx * nx; idx += 32) {
      const int b = idx / nx, a = idx - b * nx;
      cplx s = mk(0.0, 0.0);
      for (int q = 0; q < Q; ++q) s = cadd(s, cmulc(Ey[r * Q + q], K11[(q * nx + b) * nx + a]));
      gT[b * nx + a] = s;
    }
    __syncwarp();
    // tmp = T^H gT ; gT <- -tmp T^H
    for (int idx = lane; idx < nx * nx; idx += 32) {
      const int b = idx / nx, a = idx - b * nx;
      cplx s = mk(0.0, 0.0);
      for (int k = 0; k < nx; ++k) s = cadd(s, cmulc(T[a * nx + k], gT[b * nx + k]));
      tmp[b * nx + a] = s;
    }
    __syncwarp();
    for (int idx = lane; idx < nx * nx; idx += 32) {
      const int b = idx / nx, a = idx - b * nx;
      cplx s = mk(0.0, 0.0);
      for (int k = 0; k < nx; ++k) s = cadd(s, cmul(tmp[k * nx + a], cconj(T[k * nx + b])));
      gT[b * nx + a] = cneg(s);
    }
    __syncwarp();
    for (int k = lane; k < P; k += 32) {
      const int off = k - (nx - 1);  // a - b
      cplx s = mk(0.0, 0.0);
      for (int b = 0; b < nx; ++b) {
        const int a = b + off;
        if (a >= 0 && a < nx) s = cadd(s, gT[b * nx + a]);
      }
      gv[k] = s;
    }
    __syncwarp();
    for (int c = lane; c < npx; c += 32) {
      cplx s = mk(0.0, 0.0);
      for (int k = 0; k < P; ++k) s = cadd(s, cmulc(Ex[c * P + k], gv[k]));
      const cplx w = cinv(er[c]);
      const cplx w2 = cmul(w, w);
      // conj(-w^2) * s, real part
      acc[r * npx + c] += -(w2.x * s.x + w2.y * s.y);
    }
    __syncwarp();
  }
  __syncthreads();
  // fe22: one x column i per warp pass; T_i = inv(Toep(Ey (1/eps[:, i])))
  for (int i = warp; i < npx; i += NW) {
    for (int q = lane; q < Q; q += 32) {
      cplx s = mk(0.0, 0.0);
      for (int r = 0; r < npy; ++r) s = cadd(s, cmul(Ey[r * Q + q], cinv(d.eps[(size_t)r * npx + i])));
      gvec[q] = s;
    }
    __syncwarp();
    for (int idx = lane; idx < ny * ny; idx += 32) {
      const int k = idx / ny, ii = idx - k * ny;
      T[k * ny + ii] = gvec[ny - 1 + ii - k];
    }
    __syncwarp();
    warp_inverse(T, fcol, piv, ny, lane);
    for (int idx = lane; idx < ny * ny; idx += 32) {
      const int dd = idx / ny, c = idx - dd * ny;
      cplx s = mk(0.0, 0.0);
      for (int p = 0; p < P; ++p) s = cadd(s, cmulc(Ex[i * P + p], K22[(p * ny + dd) * ny + c]));
      gT[dd * ny + c] = s;
    }
    __syncwarp();
    for (int idx = lane; idx < ny * ny; idx += 32) {
      const int b = idx / ny, a = idx - b * ny;
      cplx s = mk(0.0, 0.0);
      for (int k = 0; k < ny; ++k) s = cadd(s, cmulc(T[a * ny + k], gT[b * ny + k]));
      tmp[b * ny + a] = s;
    }
    __syncwarp();
    for (int idx = lane; idx < ny * ny; idx += 32) {
      const int b = idx / ny, a = idx - b * ny;
      cplx s = mk(0.0, 0.0);
      for (int k = 0; k < ny; ++k) s = cadd(s, cmul(tmp[k * ny + a], cconj(T[k * ny + b])));
      gT[b * ny + a] = cneg(s);
    }
    __syncwarp();
    for (int k = lane; k < Q; k += 32) {
      const int off = k - (ny - 1);
      cplx s = mk(0.0, 0.0);
      for (int b = 0; b < ny; ++b) {
        const int a = b + off;
        if (a >= 0 && a < ny) s = cadd(s, gT[b * ny + a]);
      }
      gv[k] = s;
    }
    __syncwarp();
    for (int r = lane; r < npy; r += 32) {
      cplx s = mk(0.0, 0.0);
      for (int k = 0; k < Q; ++k) s = cadd(s, cmulc(Ey[r * Q + k], gv[k]));
      const cplx w = cinv(d.eps[(size_t)r * npx + i]);
      const cplx w2 = cmul(w, w);
      acc[r * npx + i] += -(w2.x * s.x + w2.y * s.y);
    }
    __syncwarp();
  }
  __syncthreads();
  for (int idx = tid; idx < npy * npx; idx += NT) d.grad[idx] = acc[idx];
}

// Per-order powers of a stack (RCWASolver::scatterPlaneWave,
// src/rcwa/RCWASolver.cpp:1636-1733, incidence from the z0 medium, flux
// normalised) and, with adj != 0, dL/dRdu and dL/dTuu for
// L = sum_k wR[k] REF[k] + wT[k] TRN[k] (rank-one: (W^H g) c^H).
__global__ void stack_power_kernel(const StackPowerDesc* __restrict__ ds, int m, int adj) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const StackPowerDesc d = ds[blockIdx.x];
  const int n = 2 * m;
  cplx* c = reinterpret_cast<cplx*>(smem_raw);
  cplx* u = c + n;
  cplx* v = u + n;
  cplx* r = v + n;
  cplx* tt = r + n;
  cplx* gr = tt + n;
  cplx* gt = gr + n;
  const int tid = threadIdx.x;
  const int ctr = (d.ny * (d.nx - 1)) / 2 + (d.ny - 1) / 2;
  for (int i = tid; i < n; i += blockDim.x)
    c[i] = cadd(cscale(d.W0inv[(size_t)ctr * n + i], d.px), cscale(d.W0inv[(size_t)(m + ctr) * n + i], d.py));
  __syncthreads();
  for (int i = tid; i < n; i += blockDim.x) {
    cplx a = mk(0.0, 0.0), b = mk(0.0, 0.0);
    for (int k = 0; k < n; ++k) {
      a = cfma(d.Tuu[(size_t)k * n + i], c[k], a);
      b = cfma(d.Rdu[(size_t)k * n + i], c[k], b);
    }
    u[i] = a;
    v[i] = b;
  }
  __syncthreads();
  for (int i = tid; i < n; i += blockDim.x) {
    cplx a = mk(0.0, 0.0), b = mk(0.0, 0.0);
    for (int k = 0; k < n; ++k) {
      a = cfma(d.W1[(size_t)k * n + i], u[k], a);
      b = cfma(d.W0[(size_t)k * n + i], v[k], b);
    }
    tt[i] = a;
    r[i] = b;
  }
  __syncthreads();
  const double norm = sqrt(d.eps_in.x) * d.k0;
  for (int i = tid; i < m; i += blockDim.x) {
    const double a = d.alpha[i], b = d.beta[i];
    const cplx kzr = cneg(csqrt(mk(d.k0 * d.k0 * d.eps_in.x - a * a - b * b, d.k0 * d.k0 * d.eps_in.y)));
    const cplx kzt = csqrt(mk(d.k0 * d.k0 * d.eps_out.x - a * a - b * b, d.k0 * d.k0 * d.eps_out.y));
    for (int side = 0; side < 2; ++side) {
      const cplx kz = side ? kzt : kzr;
      cplx* f = side ? tt : r;
      const cplx fx = f[i], fy = f[i + m];
      double Pw = 0.0;
      cplx ux = mk(0.0, 0.0), uy = mk(0.0, 0.0), fz = mk(0.0, 0.0);
      if (kz.x != 0.0 || kz.y != 0.0) {
        ux = cdiv(mk(a, 0.0), kz);
        uy = cdiv(mk(b, 0.0), kz);
        fz = cadd(cmul(ux, fx), cmul(uy, fy));
        Pw = fabs(kz.x) * (cabs2(fx) + cabs2(fy) + cabs2(fz)) / norm;
      }
      if (side) d.TRN[i] = Pw; else d.REF[i] = Pw;
      if (adj) {
        const double w = side ? d.wT[i] : d.wR[i];
        const double aw = 2.0 * w * fabs(kz.x) / norm;
        cplx* g = side ? gt : gr;
        g[i] = cscale(cadd(fx, cmulc(ux, fz)), aw);
        g[i + m] = cscale(cadd(fy, cmulc(uy, fz)), aw);
      }
    }
  }
  if (!adj) return;
  __syncthreads();
  // u <- W1^H gt, v <- W0^H gr
  for (int i = tid; i < n; i += blockDim.x) {
    cplx a = mk(0.0, 0.0), b = mk(0.0, 0.0);
    for (int k = 0; k < n; ++k) {
      a = cadd(a, cmulc(d.W1[(size_t)i * n + k], gt[k]));
      b = cadd(b, cmulc(d.W0[(size_t)i * n + k], gr[k]));
    }
    u[i] = a;
    v[i] = b;
  }
  __syncthreads();
  for (long long idx = tid; idx < (long long)n * n; idx += blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    const cplx cj = cconj(c[j]);
    d.gTuu[idx] = cmul(u[i], cj);
    d.gRdu[idx] = cmul(v[i], cj);
  }
}

}  // namespace

void scale_batched(const cplx* const* A, const cplx* const* rs, const cplx* const* cs, cplx* const* out, int batch,
                   int n, cudaStream_t st) {
  if (batch <= 0) return;
  scale_kernel<<<grid_for((long long)n * n, batch), 256, 0, st>>>(A, rs, cs, out, n);
  VRC_CUDA_CHECK(cudaGetLastError());
}

void phase_vec_batched(const cplx* const* gam, const double* t, cplx* const* out, int batch, int n, cudaStream_t st) {
  if (batch <= 0) return;
  dim3 grid((n + 127) / 128, batch);
  phase_vec_kernel<<<grid, 128, 0, st>>>(gam, t, out, n);
  VRC_CUDA_CHECK(cudaGetLastError());
}

void layer_adjoint_batched(const LayerAdjDesc* d, int batch, int n, cudaStream_t st) {
  if (batch <= 0) return;
  layer_adjoint_kernel<<<grid_for((long long)n * n, batch), 256, 0, st>>>(d, n);
  VRC_CUDA_CHECK(cudaGetLastError());
}

void pq_adjoint_batched(const PQAdjDesc* d, int batch, int m, cudaStream_t st) {
  if (batch <= 0) return;
  pq_adjoint_kernel<<<grid_for((long long)m * m, batch), 256, 0, st>>>(d, m);
  VRC_CUDA_CHECK(cudaGetLastError());
}

void interface_fields_batched(const IfFieldDesc* d, int batch, int n, int ngx, int ngy, cudaStream_t st) {
  if (batch <= 0) return;
  interface_e_kernel<<<batch, 256, 0, st>>>(d, n);
  VRC_CUDA_CHECK(cudaGetLastError());
  if (ngx > 0 && ngy > 0) {
    field_image_kernel<<<grid_for((long long)ngx * ngy, batch), 256, 0, st>>>(d, n / 2, ngx, ngy);
    VRC_CUDA_CHECK(cudaGetLastError());
  }
}

void vec_axpy_batched(const cplx* const* a, const cplx* const* b, cplx s, cplx* const* y, int batch, int n,
                      cudaStream_t st) {
  if (batch <= 0) return;
  dim3 grid((n + 127) / 128, batch);
  vec_axpy_kernel<<<grid, 128, 0, st>>>(a, b, s, y, n);
  VRC_CUDA_CHECK(cudaGetLastError());
}

void thick_adjoint_batched(const ThickAdjDesc* d, int batch, int n, cudaStream_t st) {
  if (batch <= 0) return;
  thick_adjoint_kernel<<<batch, 256, 0, st>>>(d, n);
  VRC_CUDA_CHECK(cudaGetLastError());
}

size_t pixel_adjoint_smem(int nx, int ny, int npx, int npy, int nw) {
  const int P = 2 * nx - 1, Q = 2 * ny - 1, t = nx > ny ? nx : ny;
  size_t c = (size_t)P * npx + (size_t)Q * npy + (size_t)P * Q + (size_t)Q * npx + (size_t)nw * px_warp_scratch(t);
  return c * 16 + (size_t)npy * npx * 8 + (size_t)nw * 32 * sizeof(int);
}

// warps per CTA: the most (up to eight) whose shared memory fits; 0 if none
int pixel_adjoint_warps(int nx, int ny, int npx, int npy) {
  if (nx > 32 || ny > 32) return 0;
  for (int nw = PX_WARPS; nw >= 1; nw /= 2)
    if (pixel_adjoint_smem(nx, ny, npx, npy, nw) <= 227 * 1024) return nw;
  return 0;
}

bool pixel_adjoint_fits(int nx, int ny, int npx, int npy) { return pixel_adjoint_warps(nx, ny, npx, npy) > 0; }

size_t pixel_adjoint_scratch(int nx, int ny) {
  return ((size_t)(2 * ny - 1) * nx * nx + (size_t)(2 * nx - 1) * ny * ny) * 16;
}

void pixel_adjoint_batched(const PixAdjDesc* d, int batch, int nx, int ny, int npx, int npy, cudaStream_t st) {
  if (batch <= 0) return;
  const int nw = pixel_adjoint_warps(nx, ny, npx, npy);
  if (!nw) throw StatusError(ST_EINVAL, "pixel adjoint: raster and harmonics exceed the shared-memory tile");
  const size_t smem = pixel_adjoint_smem(nx, ny, npx, npy, nw);
  ensure_smem((const void*)pixel_adjoint_kernel, smem);
  pixel_adjoint_kernel<<<batch, nw * 32, smem, st>>>(d, nx, ny, npx, npy);
  VRC_CUDA_CHECK(cudaGetLastError());
}

void stack_power_batched(const StackPowerDesc* d, int batch, int m, int adj, cudaStream_t st) {
  if (batch <= 0) return;
  const size_t smem = (size_t)7 * 2 * m * 16;
  if (smem > 227 * 1024) throw StatusError(ST_EINVAL, "stack powers: n too large");
  ensure_smem((const void*)stack_power_kernel, smem);
  stack_power_kernel<<<batch, 256, smem, st>>>(d, m, adj);
  VRC_CUDA_CHECK(cudaGetLastError());
}

}  // namespace vrc
