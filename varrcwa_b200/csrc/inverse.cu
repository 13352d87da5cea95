// Batched in-place matrix inversion: blocked Gauss-Jordan with partial
// (row) pivoting, one CTA per matrix.
//
// The reference inverts through Eigen PartialPivLU (explicit inverse of
// I - rdu*Rud, src/core/RedhefferIntegrator.cpp:267-270) and uses LU solves
// elsewhere; here every W^{-1}X / M^{-1}X of the hot path is an explicit
// inverse followed by a tensor-core GEMM (same 8n^3 flops as getrf+getrs).
//
// Blocking: a panel of nb columns is reduced in shared memory (pivot search
// by warp-shuffle max reduction); the nb accumulated row operations are then
// applied to every other column as one rank-nb update
//     a[:, j] <- P a[:, j];  a[:, j] += (Tp - E) a[k:k+nb, j]
// so the matrix is streamed once per panel instead of once per pivot.
#include "common.cuh"
#include "kernels.h"

namespace vrc {
namespace {

constexpr int INV_THREADS = 512;

struct PivotCand {
  double v;
  int i;
};

__device__ __forceinline__ PivotCand warp_argmax(PivotCand c) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double ov = __shfl_xor_sync(0xffffffffu, c.v, o);
    int oi = __shfl_xor_sync(0xffffffffu, c.i, o);
    if (ov > c.v || (ov == c.v && oi < c.i)) {
      c.v = ov;
      c.i = oi;
    }
  }
  return c;
}

__global__ void __launch_bounds__(INV_THREADS)
    zinv_kernel(cplx* const* __restrict__ mats, int n, int nb, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* panel = reinterpret_cast<cplx*>(smem_raw);  // [nb][n] column-major panel
  cplx* fcol = panel + (size_t)nb * n;                       // [n] multipliers
  int* piv = reinterpret_cast<int*>(fcol + n);                // [n]
  __shared__ PivotCand red[INV_THREADS / 32];
  __shared__ cplx s_inv;
  __shared__ int s_p;
  __shared__ int s_bad;

  cplx* a = mats[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = INV_THREADS / 32;
  if (tid == 0) s_bad = 0;

  for (int k = 0; k < n; k += nb) {
    const int w = min(nb, n - k);
    // Load panel columns k..k+w-1.
    for (int idx = tid; idx < w * n; idx += INV_THREADS) {
      int c = idx / n, r = idx - c * n;
      panel[c * n + r] = a[(size_t)(k + c) * n + r];
    }
    __syncthreads();
    for (int s = 0; s < w; ++s) {
      const int r0 = k + s;
      cplx* col = panel + s * n;
      // Pivot search over rows >= r0 (|re|+|im|, as izamax).
      PivotCand c{-1.0, n};
      for (int i = r0 + tid; i < n; i += INV_THREADS) {
        double v = cabs1(col[i]);
        if (v > c.v) { c.v = v; c.i = i; }
      }
      c = warp_argmax(c);
      if (lane == 0) red[warp] = c;
      __syncthreads();
      if (warp == 0) {
        PivotCand cc = lane < nwarps ? red[lane] : PivotCand{-1.0, n};
        cc = warp_argmax(cc);
        if (lane == 0) {
          int p = cc.i;
          cplx pv = col[p];
          if (!(cc.v > 0.0) || !isfinite(cc.v)) {
            s_bad = 1;
            pv = mk(1.0, 0.0);
            p = r0;
          }
          s_p = p;
          s_inv = cinv(pv);
          piv[r0] = p;
        }
      }
      __syncthreads();
      const int p = s_p;
      const cplx ip = s_inv;
      // Swap rows r0 and p inside the panel.
      if (p != r0) {
        for (int c2 = tid; c2 < w; c2 += INV_THREADS) {
          cplx t = panel[c2 * n + r0];
          panel[c2 * n + r0] = panel[c2 * n + p];
          panel[c2 * n + p] = t;
        }
      }
      __syncthreads();
      // Save the multipliers (column s), then scale the pivot row:
      // a[r0][s] := 1, row *= 1/piv.
      for (int i = tid; i < n; i += INV_THREADS) fcol[i] = col[i];
      __syncthreads();
      for (int c2 = tid; c2 < w; c2 += INV_THREADS) {
        cplx v = (c2 == s) ? mk(1.0, 0.0) : panel[c2 * n + r0];
        panel[c2 * n + r0] = cmul(v, ip);
      }
      __syncthreads();
      // Eliminate column s from the other rows (panel columns only).
      for (int idx = tid; idx < n * w; idx += INV_THREADS) {
        int c2 = idx / n, i = idx - c2 * n;
        if (i == r0) continue;
        cplx prow = panel[c2 * n + r0];
        cplx v = (c2 == s) ? mk(0.0, 0.0) : panel[c2 * n + i];
        panel[c2 * n + i] = csub(v, cmul(fcol[i], prow));
      }
      __syncthreads();
    }
    // Write the panel back.
    for (int idx = tid; idx < w * n; idx += INV_THREADS) {
      int c = idx / n, r = idx - c * n;
      a[(size_t)(k + c) * n + r] = panel[c * n + r];
    }
    // Rank-w update of all other columns: one warp per column.
    for (int j = warp; j < n; j += nwarps) {
      if (j >= k && j < k + w) continue;
      cplx* colj = a + (size_t)j * n;
      // Row swaps in order.
      if (lane == 0) {
        for (int s = 0; s < w; ++s) {
          int p = piv[k + s];
          if (p != k + s) {
            cplx t = colj[k + s];
            colj[k + s] = colj[p];
            colj[p] = t;
          }
        }
      }
      __syncwarp();
      cplx x[16];
#pragma unroll
      for (int s = 0; s < 16; ++s) x[s] = (s < w) ? colj[k + s] : mk(0.0, 0.0);
      __syncwarp();
      for (int i = lane; i < n; i += 32) {
        cplx v = colj[i];
        cplx acc = mk(0.0, 0.0);
#pragma unroll
        for (int s = 0; s < 16; ++s) {
          if (s < w) {
            cplx t = panel[s * n + i];
            if (i == k + s) t.x -= 1.0;
            acc = cfma(t, x[s], acc);
          }
        }
        colj[i] = cadd(v, acc);
      }
    }
    __syncthreads();
  }
  // Undo the row interchanges as column interchanges, in reverse order.
  for (int k = n - 1; k >= 0; --k) {
    int p = piv[k];
    if (p != k) {
      for (int i = tid; i < n; i += INV_THREADS) {
        cplx t = a[(size_t)k * n + i];
        a[(size_t)k * n + i] = a[(size_t)p * n + i];
        a[(size_t)p * n + i] = t;
      }
    }
    __syncthreads();
  }
  if (tid == 0 && status && s_bad) status[blockIdx.x] = ST_ESINGULAR;
}

// ---------------------------------------------------------------------------
// Blocked form with the rank-w updates on the tensor cores.  Per panel of w
// columns: zinv_panel_kernel reduces the panel in shared memory (as above),
// writes it back, stores the update factor M = Tp - E (n x w) and, for every
// other column, applies the panel's row interchanges and extracts
// X = a[k:k+w, :] (w x n, zero in the panel's columns); the batched GEMM then
// performs a += M X for all columns at once (the panel's columns get + 0).
// zinv_colswap_kernel finally undoes the row interchanges as column
// interchanges.  Scratch per matrix: M, X and the pivots.
constexpr int PANEL_THREADS = 256;

__global__ void __launch_bounds__(PANEL_THREADS)
    zinv_panel_kernel(cplx* const* __restrict__ mats, cplx* __restrict__ scratch, size_t per, int n, int k, int w,
                      int W, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* panel = reinterpret_cast<cplx*>(smem_raw);  // [w][n]
  cplx* fcol = panel + (size_t)w * n;                // [n]
  int* src = reinterpret_cast<int*>(fcol + n);       // [n]: row r of P a is row src[r] of a
  int* rows = src + n;                               // [2 W]: rows that move
  __shared__ PivotCand red[PANEL_THREADS / 32];
  __shared__ cplx s_inv;
  __shared__ int s_p, s_bad, s_nrows;

  cplx* a = mats[blockIdx.x];
  cplx* M = scratch + (size_t)blockIdx.x * per;  // [w][n] (room for W)
  cplx* X = M + (size_t)n * W;                   // [n][w]: X(s, j) at X[j * w + s]
  int* piv = reinterpret_cast<int*>(M + 2 * (size_t)n * W);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int nwarps = PANEL_THREADS / 32;
  if (tid == 0) {
    s_bad = 0;
    s_nrows = 0;
  }
  for (int c2 = 0; c2 < w; ++c2)
    for (int i = tid; i < n; i += PANEL_THREADS) panel[c2 * n + i] = a[(size_t)(k + c2) * n + i];
  for (int i = tid; i < n; i += PANEL_THREADS) src[i] = i;
  __syncthreads();
  for (int s = 0; s < w; ++s) {
    const int r0 = k + s;
    cplx* col = panel + (size_t)s * n;
    PivotCand c{-1.0, n};
    for (int i = r0 + tid; i < n; i += PANEL_THREADS) {
      const double v = cabs1(col[i]);
      if (v > c.v) {
        c.v = v;
        c.i = i;
      }
    }
    c = warp_argmax(c);
    if (lane == 0) red[warp] = c;
    __syncthreads();
    if (warp == 0) {
      PivotCand cc = lane < nwarps ? red[lane] : PivotCand{-1.0, n};
      cc = warp_argmax(cc);
      if (lane == 0) {
        int p = cc.i;
        cplx pv = col[p < n ? p : r0];
        if (!(cc.v > 0.0) || !isfinite(cc.v)) {
          s_bad = 1;
          pv = mk(1.0, 0.0);
          p = r0;
        }
        s_p = p;
        s_inv = cinv(pv);
        piv[r0] = p;
        const int t = src[r0];
        src[r0] = src[p];
        src[p] = t;
      }
    }
    __syncthreads();
    const int p = s_p;
    const cplx ip = s_inv;
    if (p != r0 && tid < w) {
      const cplx t = panel[tid * n + r0];
      panel[tid * n + r0] = panel[tid * n + p];
      panel[tid * n + p] = t;
    }
    __syncthreads();
    // multipliers, then the scaled pivot row (fcol[r0] is never used)
    for (int i = tid; i < n; i += PANEL_THREADS) fcol[i] = col[i];
    if (tid < w) panel[tid * n + r0] = cmul(tid == s ? mk(1.0, 0.0) : panel[tid * n + r0], ip);
    __syncthreads();
    for (int c2 = 0; c2 < w; ++c2) {
      const cplx prow = panel[c2 * n + r0];
      cplx* pc = panel + (size_t)c2 * n;
      for (int i = tid; i < n; i += PANEL_THREADS) {
        if (i == r0) continue;
        const cplx v = (c2 == s) ? mk(0.0, 0.0) : pc[i];
        pc[i] = csub(v, cmul(fcol[i], prow));
      }
    }
    __syncthreads();
  }
  for (int c2 = 0; c2 < w; ++c2)
    for (int i = tid; i < n; i += PANEL_THREADS) {
      const cplx v = panel[c2 * n + i];
      a[(size_t)(k + c2) * n + i] = v;
      M[(size_t)c2 * n + i] = (i == k + c2) ? mk(v.x - 1.0, v.y) : v;
    }
  // rows moved by the panel's interchanges (at most 2w)
  for (int i = tid; i < n; i += PANEL_THREADS)
    if (src[i] != i) rows[atomicAdd(&s_nrows, 1)] = i;
  __syncthreads();
  const int nrows = s_nrows;
  // other columns: permute the moved rows, staged through the panel's shared
  // memory (all reads of a group of columns before any write; a warp per
  // column, a lane per moved row), then x_s = (P a)[k+s]
  const int cw = max(1, (int)((size_t)w * n / max(nrows, 1)));  // columns per group
  for (int g0 = 0; g0 < n && nrows > 0; g0 += cw) {
    const int g1 = min(n, g0 + cw);
    for (int j = g0 + warp; j < g1; j += nwarps) {
      if (j >= k && j < k + w) continue;
      for (int q = lane; q < nrows; q += 32) panel[(size_t)(j - g0) * nrows + q] = a[(size_t)j * n + src[rows[q]]];
    }
    __syncthreads();
    for (int j = g0 + warp; j < g1; j += nwarps) {
      if (j >= k && j < k + w) continue;
      for (int q = lane; q < nrows; q += 32) a[(size_t)j * n + rows[q]] = panel[(size_t)(j - g0) * nrows + q];
    }
    __syncthreads();
  }
  for (int j = warp; j < n; j += nwarps) {
    const bool pc = j >= k && j < k + w;
    for (int s2 = lane; s2 < w; s2 += 32) X[(size_t)j * w + s2] = pc ? mk(0.0, 0.0) : a[(size_t)j * n + k + s2];
  }
  if (tid == 0 && status && s_bad) status[blockIdx.x] = ST_ESINGULAR;
}

__global__ void __launch_bounds__(256)
    zinv_colswap_kernel(cplx* const* __restrict__ mats, const cplx* __restrict__ scratch, size_t per, int n, int w) {
  cplx* a = mats[blockIdx.x];
  const int* piv = reinterpret_cast<const int*>(scratch + (size_t)blockIdx.x * per + 2 * (size_t)n * w);
  for (int k = n - 1; k >= 0; --k) {
    const int p = piv[k];
    if (p != k)
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const cplx t = a[(size_t)k * n + i];
        a[(size_t)k * n + i] = a[(size_t)p * n + i];
        a[(size_t)p * n + i] = t;
      }
    __syncthreads();
  }
}

}  // namespace

int zinv_panel_width(int n) {
  // panel (nb x n complex) + pivots must fit comfortably in shared memory.
  int nb = 16;
  while (nb > 1 && (size_t)(nb + 1) * n * 16 + (size_t)n * 4 > 200 * 1024) nb >>= 1;
  return nb;
}

int zinv_blocked_width(int n) {
  int w = 32;
  while (w > 4 && ((size_t)(w + 1) * n * 16 + (size_t)n * 4 + 2 * w * 4 > 200 * 1024)) w >>= 1;
  return w;
}

size_t zinv_blocked_scratch(int n) {
  const int w = zinv_blocked_width(n);
  return (2 * (size_t)n * w + ((size_t)n * 4 + 15) / 16) * 16;  // M, X, pivots
}

void zinv_blocked_batched(cplx* const* d_mats, int batch, int n, int* d_status, void* scratch,
                          const GemmDesc* d_descs, cudaStream_t stream) {
  if (batch <= 0) return;
  const int W = zinv_blocked_width(n);
  const size_t per = zinv_blocked_scratch(n) / 16;
  const size_t smem = (size_t)(W + 1) * n * 16 + (size_t)n * 4 + 2 * W * 4;
  static size_t configured = 0;
  if (smem > configured && smem > 48 * 1024) {
    VRC_CUDA_CHECK(cudaFuncSetAttribute(zinv_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured = smem;
  }
  cplx* scr = static_cast<cplx*>(scratch);
  for (int b0 = 0; b0 < batch; b0 += 65535) {
    const int nb = min(65535, batch - b0);
    for (int k = 0; k < n; k += W) {
      const int w = min(W, n - k);
      zinv_panel_kernel<<<nb, PANEL_THREADS, smem, stream>>>(d_mats + b0, scr + (size_t)b0 * per, per, n, k, w, W,
                                                             d_status ? d_status + b0 : nullptr);
      VRC_CUDA_CHECK(cudaGetLastError());
      // descriptor b: A = M (n x w, leading dimension n), B = X (w x n,
      // leading dimension w) at M + n W, C = Cin = the matrix
      zgemm_batched(d_descs + b0, nb, n, mk(1.0, 0.0), mk(1.0, 0.0), 0.0, stream, w);
    }
    zinv_colswap_kernel<<<nb, 256, 0, stream>>>(d_mats + b0, scr + (size_t)b0 * per, per, n, W);
  }
  VRC_CUDA_CHECK(cudaGetLastError());
}

void zinv_batched(cplx* const* d_mats, int batch, int n, int* d_status, cudaStream_t stream) {
  if (batch <= 0) return;
  int nb = zinv_panel_width(n);
  size_t smem = (size_t)(nb + 1) * n * 16 + (size_t)n * 4;
  static int configured_smem = 0;
  if ((int)smem > configured_smem && smem > 48 * 1024) {
    VRC_CUDA_CHECK(cudaFuncSetAttribute(zinv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
    configured_smem = (int)smem;
  }
  for (int b0 = 0; b0 < batch; b0 += 65535) {
    int nbat = batch - b0 < 65535 ? batch - b0 : 65535;
    zinv_kernel<<<nbat, INV_THREADS, smem, stream>>>(d_mats + b0, n, nb,
                                                      d_status ? d_status + b0 : nullptr);
  }
  VRC_CUDA_CHECK(cudaGetLastError());
}

}  // namespace vrc
