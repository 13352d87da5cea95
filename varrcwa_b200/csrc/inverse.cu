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
#include <cstdlib>

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

// The same panel step with the panel held in registers (n <= 256): thread
// (h, i) of 512 keeps row i of panel columns [16h, 16h+16); per pivot only
// the pivot candidates, the exchanged rows, the multipliers and the scaled
// pivot row pass through shared memory.
constexpr int RPN_THREADS = 512;
constexpr int RPN_STAGE = 32 * 1024;  // bytes for the row moves of the other columns

__global__ void __launch_bounds__(RPN_THREADS, 1)
    zinv_panel_reg_kernel(cplx* const* __restrict__ mats, cplx* __restrict__ scratch, size_t per, int n, int k,
                          int w, int W, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* stage = reinterpret_cast<cplx*>(smem_raw);                 // [RPN_STAGE bytes]
  int* src = reinterpret_cast<int*>(smem_raw + RPN_STAGE);         // [256]
  int* rows = src + 256;                                           // [64]
  __shared__ PivotCand red[8];
  __shared__ cplx prow[32];
  __shared__ cplx fcol[256];
  __shared__ int s_bad, s_nrows;

  cplx* a = mats[blockIdx.x];
  cplx* M = scratch + (size_t)blockIdx.x * per;
  cplx* X = M + (size_t)n * W;
  int* piv = reinterpret_cast<int*>(M + 2 * (size_t)n * W);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int h = tid >> 8, i = tid & 255;
  const bool row = i < n;

#ifdef ZP_TIMING
  long long zt0 = clock64(), zt1 = 0, zt2 = 0, zt3 = 0, zt4 = 0, zs[4] = {0, 0, 0, 0};
#endif
  cplx r[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const int gc = 16 * h + c;
    r[c] = (row && gc < w) ? a[(size_t)(k + gc) * n + i] : mk(0.0, 0.0);
  }
  for (int q = tid; q < n; q += RPN_THREADS) src[q] = q;
  if (tid == 0) {
    s_bad = 0;
    s_nrows = 0;
  }
  // Rows stay in their threads; the interchanges only relabel them: lpos is
  // the row index this thread's row has after the interchanges so far.
  int lpos = i;
  __syncthreads();
#ifdef ZP_TIMING
  zt1 = clock64();
#endif
  // the step loop is not unrolled (its body is large); a thread's entry of
  // column s is picked from the register row by an unrolled select
  auto pick = [&](int cs) {
    cplx v = r[0];
#pragma unroll
    for (int c = 1; c < 16; ++c)
      if (c == cs) v = r[c];
    return v;
  };
#pragma unroll 1
  for (int s = 0; s < 32; ++s) {
    if (s < w) {
      const int r0 = k + s;
      const int hs = s >> 4, cs = s & 15;
      if (h == hs) {
        PivotCand c{-1.0, n};
        if (row && lpos >= r0) {
          c.v = cabs1(pick(cs));
          c.i = lpos;
        }
        c = warp_argmax(c);
        if (lane == 0) red[warp & 7] = c;
      }
#ifdef ZP_TIMING
      long long ta = clock64();
#endif
      __syncthreads();
#ifdef ZP_TIMING
      long long tb = clock64();
      zs[0] += tb - ta;
#endif
      // every thread reduces the eight candidates itself (same order, same result)
      PivotCand cc = red[0];
#pragma unroll
      for (int q = 1; q < 8; ++q) {
        const PivotCand o = red[q];
        if (o.v > cc.v || (o.v == cc.v && o.i < cc.i)) cc = o;
      }
      const bool bad = !(cc.v > 0.0) || !isfinite(cc.v) || cc.i >= n;
      const int p = bad ? r0 : cc.i;
      if (tid == 0) {
        if (bad) s_bad = 1;
        piv[r0] = p;
        const int t = src[r0];
        src[r0] = src[p];
        src[p] = t;
      }
      if (lpos == p) lpos = r0;
      else if (lpos == r0) lpos = p;
      // the pivot row (now labelled r0) and the multipliers of column s
      const bool prow_thread = row && lpos == r0;
      if (prow_thread) {
#pragma unroll
        for (int c = 0; c < 16; ++c) prow[16 * h + c] = r[c];
      }
      if (h == hs && row) fcol[i] = pick(cs);
#ifdef ZP_TIMING
      long long tc = clock64();
      zs[1] += tc - tb;
#endif
      __syncthreads();
#ifdef ZP_TIMING
      long long td = clock64();
      zs[2] += td - tc;
#endif
      const cplx ip = bad ? mk(1.0, 0.0) : cinv_fast(prow[s]);
      if (prow_thread) {
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          const int gc = 16 * h + c;
          r[c] = cmul(gc == s ? mk(1.0, 0.0) : r[c], ip);
        }
      } else if (row) {
        const cplx f = cmul(fcol[i], ip);
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          const int gc = 16 * h + c;
          // column s: -a(i, s) / pivot; others: a(i, c) - a(i, s) / pivot * a(r0, c)
          if (gc < w) r[c] = (gc == s) ? cneg(f) : csub(r[c], cmul(f, prow[gc]));
        }
      }
#ifdef ZP_TIMING
      zs[3] += clock64() - td;
#endif
    }
  }
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const int gc = 16 * h + c;
    if (row && gc < w) {
      const cplx v = r[c];
      a[(size_t)(k + gc) * n + lpos] = v;
      M[(size_t)gc * n + lpos] = (lpos == k + gc) ? mk(v.x - 1.0, v.y) : v;
    }
  }
#ifdef ZP_TIMING
  zt2 = clock64();
#endif
  for (int q = tid; q < n; q += RPN_THREADS)
    if (src[q] != q) rows[atomicAdd(&s_nrows, 1)] = q;
  __syncthreads();
  const int nrows = s_nrows;
  constexpr int nwarps = RPN_THREADS / 32;
  const int cw = max(1, (int)(RPN_STAGE / 16 / max(nrows, 1)));
  for (int g0 = 0; g0 < n && nrows > 0; g0 += cw) {
    const int g1 = min(n, g0 + cw);
    for (int j = g0 + warp; j < g1; j += nwarps) {
      if (j >= k && j < k + w) continue;
      for (int q = lane; q < nrows; q += 32) stage[(size_t)(j - g0) * nrows + q] = a[(size_t)j * n + src[rows[q]]];
    }
    __syncthreads();
    for (int j = g0 + warp; j < g1; j += nwarps) {
      if (j >= k && j < k + w) continue;
      for (int q = lane; q < nrows; q += 32) a[(size_t)j * n + rows[q]] = stage[(size_t)(j - g0) * nrows + q];
    }
    __syncthreads();
  }
#ifdef ZP_TIMING
  zt3 = clock64();
#endif
  for (int j = warp; j < n; j += nwarps) {
    const bool pc = j >= k && j < k + w;
    for (int s2 = lane; s2 < w; s2 += 32) X[(size_t)j * w + s2] = pc ? mk(0.0, 0.0) : a[(size_t)j * n + k + s2];
  }
  if (tid == 0 && status && s_bad) status[blockIdx.x] = ST_ESINGULAR;
#ifdef ZP_TIMING
  __syncthreads();
  zt4 = clock64();
  if (tid == 0 && blockIdx.x == 0)
    printf("zp k=%d load %lld pivots %lld [sync1 %lld reduce %lld sync2 %lld elim %lld] permute %lld extract %lld\n", k,
           zt1 - zt0, zt2 - zt1, zs[0], zs[1], zs[2], zs[3], zt3 - zt2, zt4 - zt3);
#endif
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
  ensure_smem((const void*)zinv_panel_kernel, smem);
  // registers hold the panel when every row has a thread of each half
  const bool use_reg = n <= 256 && W == 32 && !std::getenv("VRC_ZINV_SMEM_PANEL");
  const size_t reg_smem = RPN_STAGE + (256 + 64) * sizeof(int);
  if (use_reg) ensure_smem((const void*)zinv_panel_reg_kernel, reg_smem);
  cplx* scr = static_cast<cplx*>(scratch);
  for (int b0 = 0; b0 < batch; b0 += 65535) {
    const int nb = min(65535, batch - b0);
    for (int k = 0; k < n; k += W) {
      const int w = min(W, n - k);
      if (use_reg)
        zinv_panel_reg_kernel<<<nb, RPN_THREADS, reg_smem, stream>>>(
            d_mats + b0, scr + (size_t)b0 * per, per, n, k, w, W, d_status ? d_status + b0 : nullptr);
      else
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
  ensure_smem((const void*)zinv_kernel, smem);
  for (int b0 = 0; b0 < batch; b0 += 65535) {
    int nbat = batch - b0 < 65535 ? batch - b0 : 65535;
    zinv_kernel<<<nbat, INV_THREADS, smem, stream>>>(d_mats + b0, n, nb,
                                                      d_status ? d_status + b0 : nullptr);
  }
  VRC_CUDA_CHECK(cudaGetLastError());
}

}  // namespace vrc
