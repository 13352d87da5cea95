// Batched FP64 complex non-Hermitian eigensolver (right eigenvectors), one
// CTA per matrix, replacing LAPACKE_zgeev / magma_zgeev of the reference
// (src/rcwa/MKLEigenSolver.hpp:45-55, src/gpu/RedhefferIntegratorGPU.cpp:220-223).
//
//   1. hess_kernel   Householder reduction to upper Hessenberg form
//                    (H = Q^H A Q) with the left and right reflector
//                    applications fused into one rank-2 update per column,
//                    then backward accumulation of Q.
//   2. hqr_kernel    complex Schur form T = Z^H A Z by implicitly shifted
//                    single-shift QR (Wilkinson shifts, exceptional shifts at
//                    iterations 10/20, deflation on small subdiagonals).  The
//                    bulge chase runs in chunks of B steps: one warp chases
//                    the bulge through a (B+3)^2 diagonal window held in
//                    shared memory; the chunk's B rotations are then applied
//                    by the whole CTA to the rows/columns outside the window
//                    and to Z, each thread streaming one row or column.
//   3. trevc_kernel  eigenvectors of T by back substitution (one warp per
//                    eigenvalue, near-singular diagonals perturbed to smin).
//   4. vecnorm_kernel  X = Z Y is formed by the GEMM; each column is scaled to
//                    unit 2-norm with its largest component real (the zgeev
//                    convention).
// Every loop is bounded: QR gives up after 30*max(10,n) iterations per
// eigenvalue and reports ST_ENOCONV through the status array.
#include "common.cuh"
#include "kernels.h"

namespace vrc {
namespace {

constexpr int HESS_THREADS = 256;
constexpr int HESS_WARPS = HESS_THREADS / 32;

__device__ __forceinline__ cplx warp_sum(cplx v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}
__device__ __forceinline__ double warp_sumd(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Elementary reflector for a vector (alpha, x): returns beta (real), tau and
// the scale applied to x so that v = (1, x*scale).  Published Householder
// construction (Golub & Van Loan 5.1.13, complex form).
__device__ __forceinline__ void householder(cplx alpha, double xnorm2, double* beta, cplx* tau,
                                            cplx* scale) {
  if (xnorm2 == 0.0 && alpha.y == 0.0) {
    *beta = alpha.x;
    *tau = mk(0.0, 0.0);
    *scale = mk(0.0, 0.0);
    return;
  }
  double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2);
  double b = alpha.x >= 0.0 ? -nrm : nrm;
  *beta = b;
  *tau = mk((b - alpha.x) / b, -alpha.y / b);
  *scale = cinv(mk(alpha.x - b, alpha.y));
}

// ---------------------------------------------------------------------------
// 1. Hessenberg reduction + Q accumulation
// ---------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(HESS_THREADS)
    hess_kernel(cplx* const* __restrict__ Hs, cplx* const* __restrict__ Zs, int n) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* v = reinterpret_cast<cplx*>(smem_raw);  // [n]
  cplx* y = v + n;                              // [n]
  cplx* u = y + n;                              // [n]
  cplx* taus = u + n;                           // [n]
  cplx* yp = taus + n;                          // [HESS_WARPS][n]
  __shared__ double red[HESS_WARPS];
  __shared__ cplx s_tau, s_scale, s_s;

  cplx* H = Hs[blockIdx.x];
  cplx* Z = Zs[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  for (int k = 0; k + 2 < n; ++k) {
    const int j0 = k + 1;  // J = [j0, n)
    // --- reflector from x = H[j0:n, k]
    double part = 0.0;
    for (int i = j0 + 1 + tid; i < n; i += HESS_THREADS) part += cabs2(H[(size_t)k * n + i]);
    part = warp_sumd(part);
    if (lane == 0) red[warp] = part;
    __syncthreads();
    if (tid == 0) {
      double xn = 0.0;
      for (int w = 0; w < HESS_WARPS; ++w) xn += red[w];
      cplx alpha = H[(size_t)k * n + j0];
      double beta;
      cplx tau, scale;
      householder(alpha, xn, &beta, &tau, &scale);
      s_tau = tau;
      s_scale = scale;
      taus[k] = tau;
      H[(size_t)k * n + j0] = mk(beta, 0.0);
    }
    __syncthreads();
    const cplx tau = s_tau;
    for (int i = tid; i < n; i += HESS_THREADS) {
      cplx vi;
      if (i < j0) vi = mk(0.0, 0.0);
      else if (i == j0) vi = mk(1.0, 0.0);
      else {
        vi = cmul(H[(size_t)k * n + i], s_scale);
        H[(size_t)k * n + i] = vi;  // keep v below the subdiagonal for Q
      }
      v[i] = vi;
    }
    __syncthreads();
    if (tau.x == 0.0 && tau.y == 0.0) continue;
    // --- fused products: y = H[:, J] v (all rows), u_j = v^H H[J, j]
    cplx ypart[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) ypart[t] = mk(0.0, 0.0);
    for (int j = j0 + warp; j < n; j += HESS_WARPS) {
      const cplx vj = v[j];
      const cplx* col = H + (size_t)j * n;
      cplx up = mk(0.0, 0.0);
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        int i = lane + 32 * t;
        if (i < n) {
          cplx h = col[i];
          ypart[t] = cfma(h, vj, ypart[t]);
          if (i >= j0) up = cadd(up, cmulc(v[i], h));
        }
      }
      up = warp_sum(up);
      if (lane == 0) u[j] = up;
    }
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      int i = lane + 32 * t;
      if (i < n) yp[warp * n + i] = ypart[t];
    }
    __syncthreads();
    for (int i = tid; i < n; i += HESS_THREADS) {
      cplx s = mk(0.0, 0.0);
      for (int w = 0; w < HESS_WARPS; ++w) s = cadd(s, yp[w * n + i]);
      y[i] = s;
    }
    __syncthreads();
    // s = v^H y_J
    {
      cplx sp = mk(0.0, 0.0);
      for (int i = j0 + tid; i < n; i += HESS_THREADS) sp = cadd(sp, cmulc(v[i], y[i]));
      sp = warp_sum(sp);
      if (lane == 0) yp[warp] = sp;  // reuse
      __syncthreads();
      if (tid == 0) {
        cplx s = mk(0.0, 0.0);
        for (int w = 0; w < HESS_WARPS; ++w) s = cadd(s, yp[w]);
        s_s = s;
      }
      __syncthreads();
    }
    // z_j = u_j - tau * s * conj(v_j)
    const cplx ts = cmul(tau, s_s);
    for (int j = j0 + tid; j < n; j += HESS_THREADS) u[j] = csub(u[j], cmul(ts, cconj(v[j])));
    __syncthreads();
    // --- rank-2 update of H[:, J]
    const cplx tauc = cconj(tau);
    for (int j = j0 + warp; j < n; j += HESS_WARPS) {
      const cplx vjc = cconj(v[j]);
      const cplx zj = u[j];
      cplx* col = H + (size_t)j * n;
      const cplx tv = cmul(tau, vjc);
      const cplx tz = cmul(tauc, zj);
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        int i = lane + 32 * t;
        if (i < n) {
          cplx h = col[i];
          h = csub(h, cmul(y[i], tv));
          if (i >= j0) h = csub(h, cmul(v[i], tz));
          col[i] = h;
        }
      }
    }
    __syncthreads();
  }
  // --- Q = H_0 H_1 ... H_{n-3}, accumulated backward into Z.
  for (int idx = tid; idx < n * n; idx += HESS_THREADS) {
    int c = idx / n, r = idx - c * n;
    Z[idx] = mk(r == c ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  for (int k = n - 3; k >= 0; --k) {
    const int j0 = k + 1;
    const cplx tau = taus[k];
    for (int i = tid; i < n; i += HESS_THREADS) {
      v[i] = (i < j0) ? mk(0.0, 0.0) : (i == j0 ? mk(1.0, 0.0) : H[(size_t)k * n + i]);
    }
    __syncthreads();
    if (!(tau.x == 0.0 && tau.y == 0.0)) {
      for (int j = j0 + warp; j < n; j += HESS_WARPS) {
        cplx* col = Z + (size_t)j * n;
        cplx wp = mk(0.0, 0.0);
        for (int i = j0 + lane; i < n; i += 32) wp = cadd(wp, cmulc(v[i], col[i]));
        wp = warp_sum(wp);
        const cplx tw = cmul(tau, wp);
        for (int i = j0 + lane; i < n; i += 32) col[i] = csub(col[i], cmul(v[i], tw));
      }
    }
    __syncthreads();
  }
  // Clear everything below the subdiagonal (the stored reflectors).
  for (int idx = tid; idx < n * n; idx += HESS_THREADS) {
    int c = idx / n, r = idx - c * n;
    if (r > c + 1) H[idx] = mk(0.0, 0.0);
  }
}

// ---------------------------------------------------------------------------
// 2. Shifted QR to complex Schur form
// ---------------------------------------------------------------------------
constexpr int QR_THREADS = 256;
constexpr int QB = 32;          // bulge-chase steps per chunk
constexpr int QD = QB + 3;      // diagonal window size
constexpr double ULP = 2.220446049250313e-16;  // 2^-52 (unit roundoff * base)
constexpr double SMLNUM_BASE = 2.2250738585072014e-308;

__device__ __forceinline__ void refl2(cplx a, cplx b, cplx* beta, cplx* tau, cplx* v2) {
  double bx2 = cabs2(b);
  double b0;
  cplx t, sc;
  householder(a, bx2, &b0, &t, &sc);
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

__global__ void __launch_bounds__(QR_THREADS)
    hqr_kernel(cplx* const* __restrict__ Hs, cplx* const* __restrict__ Zs, cplx* const* __restrict__ Ws,
               int n, int* __restrict__ status) {
  __shared__ cplx D[QD * QD];
  __shared__ cplx s_tau[QB], s_v2[QB];
  __shared__ int s_red[QR_THREADS / 32];
  __shared__ int s_l;
  __shared__ cplx s_shift;

  cplx* H = Hs[blockIdx.x];
  cplx* Z = Zs[blockIdx.x];
  cplx* W = Ws[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double smlnum = SMLNUM_BASE * ((double)n / ULP);
  const int itmax = 30 * max(10, n);       // per eigenvalue
  const long long totmax = 30LL * n + 300;  // whole matrix (typical total is ~3n)
  long long tot = 0;
  auto h = [&](int r, int c) -> cplx& { return H[(size_t)c * n + r]; };

  int i = n - 1;
  int failed = 0;
  while (i >= 0) {
    int l = 0;
    int its;
    for (its = 0; its <= itmax && tot <= totmax; ++its, ++tot) {
      // Deflation search: largest k in (l, i] with a negligible H[k][k-1].
      int best = l;
      for (int k = l + 1 + tid; k <= i; k += QR_THREADS) {
        cplx sub = h(k, k - 1);
        bool small = false;
        double cs = cabs1(sub);
        if (cs <= smlnum) {
          small = true;
        } else {
          cplx dkm = h(k - 1, k - 1), dk = h(k, k);
          double tst = cabs1(dkm) + cabs1(dk);
          if (tst == 0.0) {
            if (k - 2 >= 0) tst += fabs(h(k - 1, k - 2).x);
            if (k + 1 <= n - 1) tst += fabs(h(k + 1, k).x);
          }
          if (cs <= ULP * tst) {
            double a1 = cs, a2 = cabs1(h(k - 1, k));
            double ab = fmax(a1, a2), ba = fmin(a1, a2);
            double b1 = cabs1(dk), b2 = cabs1(csub(dkm, dk));
            double aa = fmax(b1, b2), bb = fmin(b1, b2);
            double s = aa + ab;
            if (ba * (ab / s) <= fmax(smlnum, ULP * (bb * (aa / s)))) small = true;
          }
        }
        if (small && k > best) best = k;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
      if (lane == 0) s_red[warp] = best;
      __syncthreads();
      if (tid == 0) {
        int b = l;
        for (int w = 0; w < QR_THREADS / 32; ++w) b = max(b, s_red[w]);
        s_l = b;
        if (b > l) h(b, b - 1) = mk(0.0, 0.0);
      }
      __syncthreads();
      l = s_l;
      if (l >= i) break;  // H[i][i] isolated
      // Shift.
      if (tid == 0) {
        cplx t;
        if (its == 10) {
          double s = 0.75 * fabs(h(l + 1, l).x);
          t = cadd(mk(s, 0.0), h(l, l));
        } else if (its == 20) {
          double s = 0.75 * fabs(h(i, i - 1).x);
          t = cadd(mk(s, 0.0), h(i, i));
        } else {
          t = h(i, i);
          cplx uu = cmul(csqrt(h(i - 1, i)), csqrt(h(i, i - 1)));
          double s = cabs1(uu);
          if (s != 0.0) {
            cplx x = cscale(csub(h(i - 1, i - 1), t), 0.5);
            double sx = cabs1(x);
            s = fmax(s, sx);
            cplx xs = cscale(x, 1.0 / s), us = cscale(uu, 1.0 / s);
            cplx yv = cscale(csqrt(cadd(cmul(xs, xs), cmul(us, us))), s);
            if (sx > 0.0) {
              cplx xn = cscale(x, 1.0 / sx);
              if (xn.x * yv.x + xn.y * yv.y < 0.0) yv = cneg(yv);
            }
            t = csub(t, cmul(uu, cdiv(uu, cadd(x, yv))));
          }
        }
        s_shift = t;
      }
      __syncthreads();
      const cplx shift = s_shift;
      const int m = l;
      // Single-shift sweep over steps k = m .. i-1, in chunks.
      for (int k0 = m; k0 < i; k0 += QB) {
        const int k1 = min(k0 + QB, i);  // steps k0..k1-1
        const int ds = (k0 > m) ? k0 - 1 : m;
        const int de = min(k1 + 1, i);
        const int dn = de - ds + 1;
        for (int idx = tid; idx < dn * dn; idx += QR_THREADS) {
          int c = idx / dn, r = idx - c * dn;
          D[c * QD + r] = h(ds + r, ds + c);
        }
        __syncthreads();
        if (warp == 0) {
          for (int k = k0; k < k1; ++k) {
            if (lane == 0) {
              cplx a, b;
              if (k == m) {
                a = csub(D[(k - ds) * QD + (k - ds)], shift);
                b = D[(k - ds) * QD + (k + 1 - ds)];
              } else {
                a = D[(k - 1 - ds) * QD + (k - ds)];
                b = D[(k - 1 - ds) * QD + (k + 1 - ds)];
              }
              cplx beta, tau, v2;
              refl2(a, b, &beta, &tau, &v2);
              if (k > m) {
                D[(k - 1 - ds) * QD + (k - ds)] = beta;
                D[(k - 1 - ds) * QD + (k + 1 - ds)] = mk(0.0, 0.0);
              }
              s_tau[k - k0] = tau;
              s_v2[k - k0] = v2;
            }
            __syncwarp();
            const cplx tau = s_tau[k - k0], v2 = s_v2[k - k0];
            const cplx tauc = cconj(tau), v2c = cconj(v2);
            // Row transform (rows k, k+1), columns k..de.
            for (int j = k + lane; j <= de; j += 32) {
              cplx x = D[(j - ds) * QD + (k - ds)], y = D[(j - ds) * QD + (k + 1 - ds)];
              cplx sum = cmul(tauc, cadd(x, cmul(v2c, y)));
              D[(j - ds) * QD + (k - ds)] = csub(x, sum);
              D[(j - ds) * QD + (k + 1 - ds)] = csub(y, cmul(sum, v2));
            }
            __syncwarp();
            // Column transform (cols k, k+1), rows ds..min(k+2, i).
            const int re = min(k + 2, i);
            for (int r = ds + lane; r <= re; r += 32) {
              cplx p = D[(k - ds) * QD + (r - ds)], q = D[(k + 1 - ds) * QD + (r - ds)];
              cplx sum = cmul(tau, cadd(p, cmul(v2, q)));
              D[(k - ds) * QD + (r - ds)] = csub(p, sum);
              D[(k + 1 - ds) * QD + (r - ds)] = csub(q, cmul(sum, v2c));
            }
            __syncwarp();
          }
        }
        __syncthreads();
        for (int idx = tid; idx < dn * dn; idx += QR_THREADS) {
          int c = idx / dn, r = idx - c * dn;
          h(ds + r, ds + c) = D[c * QD + r];
        }
        // Deferred updates outside the window.
        const int nsteps = k1 - k0;
        const int nright = n - 1 - de;      // columns de+1 .. n-1, rows k0..k1
        const int nabove = ds;              // rows 0 .. ds-1, cols k0..k1
        const int ntask = nright + nabove + n;
        for (int task = tid; task < ntask; task += QR_THREADS) {
          cplx e[QB + 1];
          if (task < nright) {
            const int j = de + 1 + task;
            cplx* col = H + (size_t)j * n + k0;
#pragma unroll
            for (int s = 0; s <= QB; ++s)
              if (s <= nsteps) e[s] = col[s];
#pragma unroll
            for (int s = 0; s < QB; ++s) {
              if (s < nsteps) {
                const cplx tauc = cconj(s_tau[s]), v2 = s_v2[s];
                cplx sum = cmul(tauc, cadd(e[s], cmul(cconj(v2), e[s + 1])));
                e[s] = csub(e[s], sum);
                e[s + 1] = csub(e[s + 1], cmul(sum, v2));
              }
            }
#pragma unroll
            for (int s = 0; s <= QB; ++s)
              if (s <= nsteps) col[s] = e[s];
          } else {
            int r;
            cplx* base;
            if (task < nright + nabove) {
              r = task - nright;
              base = H;
            } else {
              r = task - nright - nabove;
              base = Z;
            }
#pragma unroll
            for (int s = 0; s <= QB; ++s)
              if (s <= nsteps) e[s] = base[(size_t)(k0 + s) * n + r];
#pragma unroll
            for (int s = 0; s < QB; ++s) {
              if (s < nsteps) {
                const cplx tau = s_tau[s], v2 = s_v2[s];
                cplx sum = cmul(tau, cadd(e[s], cmul(v2, e[s + 1])));
                e[s] = csub(e[s], sum);
                e[s + 1] = csub(e[s + 1], cmul(sum, cconj(v2)));
              }
            }
#pragma unroll
            for (int s = 0; s <= QB; ++s)
              if (s <= nsteps) base[(size_t)(k0 + s) * n + r] = e[s];
          }
        }
        __syncthreads();
      }
    }
    if (its > itmax || tot > totmax) {
      failed = 1;
      break;
    }
    i = l - 1;
  }
  __syncthreads();
  for (int k = tid; k < n; k += QR_THREADS) W[k] = h(k, k);
  if (tid == 0 && failed && status) status[blockIdx.x] = ST_ENOCONV;
}

// ---------------------------------------------------------------------------
// 3. Eigenvectors of the triangular Schur factor
// ---------------------------------------------------------------------------
constexpr int TV_WARPS = 8;

__global__ void __launch_bounds__(TV_WARPS * 32)
    trevc_kernel(cplx* const* __restrict__ Ts, cplx* const* __restrict__ Ys, int n) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* work = reinterpret_cast<cplx*>(smem_raw) + (threadIdx.x >> 5) * n;
  const int lane = threadIdx.x & 31;
  const int mat = blockIdx.y;
  const cplx* T = Ts[mat];
  cplx* Y = Ys[mat];
  const int ki = blockIdx.x * TV_WARPS + (threadIdx.x >> 5);
  if (ki >= n) return;
  const cplx lam = T[(size_t)ki * n + ki];
  const double smin = fmax(ULP * cabs1(lam), SMLNUM_BASE * ((double)n / ULP));
  for (int r = lane; r < n; r += 32) work[r] = (r < ki) ? cneg(T[(size_t)ki * n + r]) : mk(0.0, 0.0);
  __syncwarp();
  for (int j = ki - 1; j >= 0; --j) {
    // x_j = work_j / (T_jj - lam)
    cplx dj = csub(T[(size_t)j * n + j], lam);
    if (cabs1(dj) < smin) dj = mk(smin, 0.0);
    cplx xj = cdiv(work[j], dj);
    __syncwarp();
    if (lane == 0) work[j] = xj;
    const cplx* colj = T + (size_t)j * n;
    for (int r = lane; r < j; r += 32) work[r] = csub(work[r], cmul(xj, colj[r]));
    __syncwarp();
  }
  cplx* y = Y + (size_t)ki * n;
  for (int r = lane; r < n; r += 32) y[r] = (r < ki) ? work[r] : (r == ki ? mk(1.0, 0.0) : mk(0.0, 0.0));
}

// ---------------------------------------------------------------------------
// 4. Column normalisation: unit 2-norm, largest-modulus component real.
// ---------------------------------------------------------------------------
__global__ void vecnorm_kernel(cplx* const* __restrict__ Xs, int n) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int col = blockIdx.x * (blockDim.x >> 5) + warp;
  if (col >= n) return;
  cplx* x = Xs[blockIdx.y] + (size_t)col * n;
  double s2 = 0.0, best = -1.0;
  int bi = 0;
  for (int r = lane; r < n; r += 32) {
    double a = cabs2(x[r]);
    s2 += a;
    if (a > best) { best = a; bi = r; }
  }
  s2 = warp_sumd(s2);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double ob = __shfl_xor_sync(0xffffffffu, best, o);
    int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
  }
  cplx xm = x[bi];
  double am = sqrt(cabs2(xm));
  double nrm = sqrt(s2);
  cplx f = (am > 0.0 && nrm > 0.0) ? mk(xm.x / (am * nrm), -xm.y / (am * nrm)) : mk(1.0, 0.0);
  for (int r = lane; r < n; r += 32) x[r] = cmul(x[r], f);
  __syncwarp();
  if (lane == 0) x[bi] = mk(x[bi].x, 0.0);
}

template <int NT>
void launch_hess(cplx* const* H, cplx* const* Z, int batch, int n, cudaStream_t st) {
  size_t smem = (size_t)(4 + HESS_WARPS) * n * 16;
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    VRC_CUDA_CHECK(cudaFuncSetAttribute(hess_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
    configured = smem;
  }
  for (int b0 = 0; b0 < batch; b0 += 65535) {
    int nb = min(65535, batch - b0);
    hess_kernel<NT><<<nb, HESS_THREADS, smem, st>>>(H + b0, Z + b0, n);
  }
}

}  // namespace

void hessenberg_batched(cplx* const* d_H, cplx* const* d_Z, int batch, int n, cudaStream_t st) {
  if (batch <= 0) return;
  if (n <= 256) launch_hess<8>(d_H, d_Z, batch, n, st);
  else if (n <= 512) launch_hess<16>(d_H, d_Z, batch, n, st);
  else if (n <= 1024) launch_hess<32>(d_H, d_Z, batch, n, st);
  else throw StatusError(ST_EINVAL, "eigensolver supports n <= 1024");
  VRC_CUDA_CHECK(cudaGetLastError());
}

void schur_batched(cplx* const* d_H, cplx* const* d_Z, cplx* const* d_W, int batch, int n, int* d_status,
                   cudaStream_t st) {
  if (batch <= 0) return;
  for (int b0 = 0; b0 < batch; b0 += 65535) {
    int nb = min(65535, batch - b0);
    hqr_kernel<<<nb, QR_THREADS, 0, st>>>(d_H + b0, d_Z + b0, d_W + b0, n, d_status ? d_status + b0 : nullptr);
  }
  VRC_CUDA_CHECK(cudaGetLastError());
}

void trevc_batched(cplx* const* d_T, cplx* const* d_Y, int batch, int n, cudaStream_t st) {
  if (batch <= 0) return;
  size_t smem = (size_t)TV_WARPS * n * 16;
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    VRC_CUDA_CHECK(cudaFuncSetAttribute(trevc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured = smem;
  }
  for (int b0 = 0; b0 < batch; b0 += 65535) {
    int nb = min(65535, batch - b0);
    dim3 grid((n + TV_WARPS - 1) / TV_WARPS, nb);
    trevc_kernel<<<grid, TV_WARPS * 32, smem, st>>>(d_T + b0, d_Y + b0, n);
  }
  VRC_CUDA_CHECK(cudaGetLastError());
}

void vecnorm_batched(cplx* const* d_X, int batch, int n, cudaStream_t st) {
  if (batch <= 0) return;
  for (int b0 = 0; b0 < batch; b0 += 65535) {
    int nb = min(65535, batch - b0);
    dim3 grid((n + 7) / 8, nb);
    vecnorm_kernel<<<grid, 256, 0, st>>>(d_X + b0, n);
  }
  VRC_CUDA_CHECK(cudaGetLastError());
}

}  // namespace vrc
