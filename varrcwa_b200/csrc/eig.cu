// Batched FP64 complex non-Hermitian eigensolver (right eigenvectors), one
// CTA per matrix, replacing LAPACKE_zgeev / magma_zgeev of the reference
// (src/rcwa/MKLEigenSolver.hpp:45-55, src/gpu/RedhefferIntegratorGPU.cpp:220-223).
//
//   1. hess_kernel   Householder reduction to upper Hessenberg form
//                    (H = Q^H A Q) with the left and right reflector
//                    applications fused into one rank-2 update per column,
//                    then backward accumulation of Q.
//   2. hqr_kernel    complex Schur form T = Z^H A Z (qr.cu: multi-bulge
//                    shifted QR with a rotation log replayed onto Z).
//   3. trevc_kernel  eigenvectors of T by back substitution (one warp per
//                    eigenvalue, near-singular diagonals perturbed to smin).
//   4. vecnorm_kernel  X = Z Y is formed by the GEMM; each column is scaled to
//                    unit 2-norm with its largest component real (the zgeev
//                    convention).
#include <cstdlib>

#include "common.cuh"
#include "householder.cuh"
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

constexpr double ULP = EIG_ULP;
constexpr double SMLNUM_BASE = EIG_SAFMIN;

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
  ensure_smem((const void*)hess_kernel<NT>, smem);
  for (int b0 = 0; b0 < batch; b0 += 65535) {
    int nb = min(65535, batch - b0);
    hess_kernel<NT><<<nb, HESS_THREADS, smem, st>>>(H + b0, Z + b0, n);
  }
}

}  // namespace

void hessenberg_batched(cplx* const* d_H, cplx* const* d_Z, int batch, int n, cudaStream_t st) {
  if (batch <= 0) return;
  // Cluster or single-CTA reduction, by measured crossovers on B200 (ms per
  // batch, both variants): the single-CTA kernel wins for n <= 128 at every
  // batch (4-9x at n = 50..98 once the batch fills the SMs, because eight
  // CTAs of a few columns each spend the reduction in cluster barriers); for
  // 128 < n <= 192 and 256 < n < 400 it wins only once the batch gives every
  // SM two matrices; the cluster kernel wins for 192 < n <= 256 at every batch
  // (matrix in shared memory) and for n >= 400, where the single-CTA
  // reduction's per-matrix latency dominates.
  static const int sms = [] {
    int dev = 0, v = 0;
    VRC_CUDA_CHECK(cudaGetDevice(&dev));
    VRC_CUDA_CHECK(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
    return v;
  }();
  const bool full = batch >= 2 * sms;
  const bool cluster = hessenberg_cluster_fits(n) && n > 128 &&
                       ((n > 192 && n <= 256) || n >= 400 || !full);
  if (cluster && !std::getenv("VRC_HESS_SINGLE_CTA")) {
    hessenberg_cluster_batched(d_H, d_Z, batch, n, st);
    return;
  }
  if (n <= 256) launch_hess<8>(d_H, d_Z, batch, n, st);
  else if (n <= 512) launch_hess<16>(d_H, d_Z, batch, n, st);
  else if (n <= 1024) launch_hess<32>(d_H, d_Z, batch, n, st);
  else throw StatusError(ST_EINVAL, "eigensolver supports n <= 1024");
  VRC_CUDA_CHECK(cudaGetLastError());
}

void trevc_batched(cplx* const* d_T, cplx* const* d_Y, int batch, int n, cudaStream_t st) {
  if (batch <= 0) return;
  size_t smem = (size_t)TV_WARPS * n * 16;
  ensure_smem((const void*)trevc_kernel, smem);
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
