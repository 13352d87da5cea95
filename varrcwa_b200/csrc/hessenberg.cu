// Hessenberg reduction H = Q^H A Q with Q accumulated, one thread-block
// cluster of HC_CS CTAs per matrix and the matrix held on chip.
//
// The single-CTA reduction streams the trailing matrix through L2/HBM twice
// per column (BLAS-2), which makes it memory bound.  Here CTA c of the
// cluster keeps columns c, c + HC_CS, c + 2 HC_CS, ... in its shared memory,
// so every pass runs out of shared memory; the only cross-CTA data are the
// reflector v (written by the owner of column k into every CTA) and the
// partial products y = A[:, J] v (each CTA writes its part into every CTA,
// which sums them), exchanged through distributed shared memory between two
// cluster barriers per column.  Buffers alternate by the parity of k, so a
// CTA one step ahead never overwrites data a slower CTA still reads.
//
// Per column k (J = [k+1, n), v = (1, v_2, ...) on J, tau):
//   y = A[:, J] v,  u_j = v^H A[J, j],  s = v^H y_J,  z_j = u_j - tau s conj(v_j)
//   A[:, J] -= y (tau v^H);  A[J, j] -= v (conj(tau) z_j)
// (the two-sided application of I - tau v v^H fused into one rank-2 update,
// the published Householder reduction of Golub & Van Loan 7.4.3 in complex
// form).  Afterwards every CTA forms its own columns of
// Q = H_0 H_1 ... H_{n-3} by backward accumulation, reading the reflectors
// stored below the subdiagonal of the written-back matrix.
#include <cooperative_groups.h>

#include <algorithm>

#include "common.cuh"
#include "householder.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace vrc {
namespace {

constexpr int HC_CS = 8;         // CTAs per cluster (portable maximum)
constexpr int HC_THREADS = 256;  // one thread per matrix row: n <= HC_THREADS
constexpr int HC_WARPS = HC_THREADS / 32;

__device__ __forceinline__ cplx warp_sum_c(cplx v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

struct HcLayout {
  int w;                                  // columns per CTA
  size_t a, vb, yp, tau, u, total;  // byte offsets
};

__host__ __device__ inline HcLayout hc_layout(int n) {
  HcLayout L;
  L.w = (n + HC_CS - 1) / HC_CS;
  size_t o = 0;
  L.a = o;
  o += (size_t)L.w * n * sizeof(cplx);  // own columns, column-major, leading dimension n
  L.vb = o;
  o += 2 * (size_t)HC_THREADS * sizeof(cplx);  // reflector, two parities
  L.yp = o;
  o += 2 * (size_t)HC_CS * HC_THREADS * sizeof(cplx);  // partial y from every CTA, two parities
  L.tau = o;
  o += (size_t)HC_THREADS * sizeof(cplx);  // tau of every column
  L.u = o;
  o += 2 * (size_t)L.w * sizeof(cplx);  // u (then b) and a per own column
  L.total = o;
  return L;
}

// Block-wide sum of one complex value per thread (all threads get the sum).
__device__ __forceinline__ cplx block_sum(cplx v, cplx* scratch) {
  v = warp_sum_c(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();  // scratch free
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  cplx s = mk(0.0, 0.0);
#pragma unroll
  for (int q = 0; q < HC_WARPS; ++q) s = cadd(s, scratch[q]);
  return s;
}

__global__ void __cluster_dims__(HC_CS, 1, 1) __launch_bounds__(HC_THREADS, 1)
    hess_cluster_kernel(cplx* const* __restrict__ Hs, cplx* const* __restrict__ Zs, int n) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ cplx s_red[HC_WARPS];
  __shared__ cplx s_scale;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const HcLayout L = hc_layout(n);
  cplx* A = reinterpret_cast<cplx*>(smem_raw + L.a);  // local column jl is global column rank + HC_CS*jl
  cplx* vb = reinterpret_cast<cplx*>(smem_raw + L.vb);
  cplx* yp = reinterpret_cast<cplx*>(smem_raw + L.yp);
  cplx* taus = reinterpret_cast<cplx*>(smem_raw + L.tau);
  cplx* us = reinterpret_cast<cplx*>(smem_raw + L.u);  // u_j, then b_j
  cplx* ca = us + L.w;                                 // a_j

  // columns are dealt out cyclically, so every CTA keeps about the same
  // number of active columns as the reduction moves right
  const int nc = rank < n ? (n - rank + HC_CS - 1) / HC_CS : 0;
  auto first_local = [&](int j0) { return j0 > rank ? (j0 - rank + HC_CS - 1) / HC_CS : 0; };
  cplx* H = Hs[blockIdx.y];
  cplx* Z = Zs[blockIdx.y];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int i = tid;  // this thread's row
  const bool row = i < n;

  if (row)
    for (int jl = 0; jl < nc; ++jl) A[(size_t)jl * n + i] = H[(size_t)(rank + HC_CS * jl) * n + i];
  cluster.sync();  // every CTA of the cluster runs before shared memory is written remotely

#ifdef HC_TIMING
  long long tph[6] = {0, 0, 0, 0, 0, 0}, tl = clock64();
#define HC_T(q) { long long t_ = clock64(); tph[q] += t_ - tl; tl = t_; }
#else
#define HC_T(q)
#endif
  for (int k = 0; k + 2 < n; ++k) {
    const int j0 = k + 1;
    const int par = k & 1;
    cplx* v = vb + par * HC_THREADS;
    // --- the owner of column k forms the reflector and sends it everywhere
    if (k % HC_CS == rank) {
      cplx* col = A + (size_t)(k / HC_CS) * n;
      const cplx a = (row && i > j0) ? col[i] : mk(0.0, 0.0);
      const double xn = block_sum(mk(cabs2(a), 0.0), s_red).x;
      if (tid == 0) {
        double beta;
        cplx tau, scale;
        householder(col[j0], xn, &beta, &tau, &scale);
        col[j0] = mk(beta, 0.0);
        s_scale = scale;
        for (int r = 0; r < HC_CS; ++r) cluster.map_shared_rank(taus, r)[k] = tau;
      }
      __syncthreads();
      cplx vi = mk(0.0, 0.0);
      if (row && i == j0) vi = mk(1.0, 0.0);
      if (row && i > j0) {
        vi = cmul(a, s_scale);
        col[i] = vi;  // kept below the subdiagonal for Q
      }
      if (row && i >= j0)
        for (int r = 0; r < HC_CS; ++r) cluster.map_shared_rank(v, r)[i] = vi;
    }
    HC_T(0)
    cluster.sync();  // reflector k visible in every CTA
    HC_T(1)
    const cplx tau = taus[k];
    if (tau.x == 0.0 && tau.y == 0.0) continue;  // the same decision in every CTA
    const cplx vi = (row && i >= j0) ? v[i] : mk(0.0, 0.0);
    const int jl0 = first_local(j0);
    // --- partial y = A[:, J_own] v_own (thread per row) ...
    cplx ya = mk(0.0, 0.0), yb = mk(0.0, 0.0);
    if (row) {
      int jl = jl0;
      for (; jl + 1 < nc; jl += 2) {
        ya = cfma(A[(size_t)jl * n + i], v[rank + HC_CS * jl], ya);
        yb = cfma(A[(size_t)(jl + 1) * n + i], v[rank + HC_CS * (jl + 1)], yb);
      }
      if (jl < nc) ya = cfma(A[(size_t)jl * n + i], v[rank + HC_CS * jl], ya);
    }
    const cplx yi = cadd(ya, yb);
    if (row)
      for (int r = 0; r < HC_CS; ++r) cluster.map_shared_rank(yp, r)[(par * HC_CS + rank) * HC_THREADS + i] = yi;
    // ... and u_j = v^H A[J, j] (warp per column)
    for (int jl = jl0 + warp; jl < nc; jl += HC_WARPS) {
      const cplx* col = A + (size_t)jl * n;
      cplx pu = mk(0.0, 0.0);
      for (int r = j0 + lane; r < n; r += 32) pu = cadd(pu, cmulc(v[r], col[r]));
      pu = warp_sum_c(pu);
      if (lane == 0) us[jl] = pu;
    }
    HC_T(2)
    cluster.sync();  // all partial y delivered
    HC_T(3)
    cplx y = mk(0.0, 0.0);
    if (row) {
#pragma unroll
      for (int r = 0; r < HC_CS; ++r) y = cadd(y, yp[(par * HC_CS + r) * HC_THREADS + i]);
    }
    const cplx s = block_sum((row && i >= j0) ? cmulc(vi, y) : mk(0.0, 0.0), s_red);
    // per-column coefficients of the rank-2 update: a_j = tau conj(v_j),
    // b_j = conj(tau) z_j with z_j = u_j - tau s conj(v_j)
    const cplx ts = cmul(tau, s), tauc = cconj(tau);
    for (int jl = jl0 + tid; jl < nc; jl += HC_THREADS) {
      const cplx vjc = cconj(v[rank + HC_CS * jl]);
      ca[jl] = cmul(tau, vjc);
      us[jl] = cmul(tauc, csub(us[jl], cmul(ts, vjc)));
    }
    __syncthreads();
    // --- rank-2 update of this CTA's columns of J (thread per row)
    if (row) {
      const cplx vt = (i >= j0) ? vi : mk(0.0, 0.0);
#pragma unroll 4
      for (int jl = jl0; jl < nc; ++jl) {
        cplx* p = A + (size_t)jl * n + i;
        *p = csub(csub(*p, cmul(y, ca[jl])), cmul(vt, us[jl]));
      }
    }
    __syncthreads();
    HC_T(4)
  }
#ifdef HC_TIMING
  if (tid == 0 && blockIdx.y == 0)
    printf("hc rank %d: owner %lld sync1 %lld yu %lld sync2 %lld update %lld\n", rank, tph[0], tph[1], tph[2],
           tph[3], tph[4]);
#endif

  // --- write back (reflectors below the subdiagonal), then accumulate Q
  if (row)
    for (int jl = 0; jl < nc; ++jl) H[(size_t)(rank + HC_CS * jl) * n + i] = A[(size_t)jl * n + i];
  __threadfence();
  cluster.sync();  // every column of H, with its reflector, is in global memory
  if (row)
    for (int jl = 0; jl < nc; ++jl) A[(size_t)jl * n + i] = mk(i == rank + HC_CS * jl ? 1.0 : 0.0, 0.0);
  // v of column k, prefetched one step ahead into a register per row
  auto fetch = [&](int k) -> cplx {
    if (k < 0 || !row) return mk(0.0, 0.0);
    if (i == k + 1) return mk(1.0, 0.0);
    return i > k + 1 ? H[(size_t)k * n + i] : mk(0.0, 0.0);
  };
  cplx vnext = fetch(n - 3);
  for (int k = n - 3; k >= 0; --k) {
    const int j0 = k + 1;
    cplx* v = vb + (k & 1) * HC_THREADS;
    if (row) v[i] = vnext;
    vnext = fetch(k - 1);
    __syncthreads();
    const cplx tau = taus[k];
    if (tau.x == 0.0 && tau.y == 0.0) continue;
    // Z[J, j] -= tau v (v^H Z[J, j]) for own columns j in J (the others are
    // still identity columns there)
    for (int jl = first_local(j0) + warp; jl < nc; jl += HC_WARPS) {
      cplx* col = A + (size_t)jl * n;
      cplx wp = mk(0.0, 0.0);
      for (int r = j0 + lane; r < n; r += 32) wp = cadd(wp, cmulc(v[r], col[r]));
      wp = warp_sum_c(wp);
      const cplx tw = cmul(tau, wp);
      for (int r = j0 + lane; r < n; r += 32) col[r] = csub(col[r], cmul(v[r], tw));
    }
  }
  __syncthreads();
  if (row)
    for (int jl = 0; jl < nc; ++jl) Z[(size_t)(rank + HC_CS * jl) * n + i] = A[(size_t)jl * n + i];
  cluster.sync();  // no CTA still reads reflectors from H
  if (row)
    for (int jl = 0; jl < nc; ++jl) {
      const int c = rank + HC_CS * jl;
      if (i > c + 1) H[(size_t)c * n + i] = mk(0.0, 0.0);
    }
}

// The same cluster reduction for 256 < n <= 512 with the matrix left in
// global memory (L2 resident for the clusters in flight): there is not enough
// shared memory for it.  Each CTA works in place on its own columns of H
// (cyclic), each thread on rows tid and tid + 256; only the reflector, the
// partial products y and the tau are exchanged, as above.  Q is accumulated
// in place in the CTA's own columns of Z.
constexpr int HG_RPT = 2;                     // rows per thread
constexpr int HG_MAXN = HC_THREADS * HG_RPT;  // 512
constexpr int HG_MAXW = (HG_MAXN + HC_CS - 1) / HC_CS;
constexpr size_t HG_SMEM = (2 * (size_t)HG_MAXN + 2 * (size_t)HC_CS * HG_MAXN + HG_MAXN + 2 * HG_MAXW) * sizeof(cplx);

__global__ void __cluster_dims__(HC_CS, 1, 1) __launch_bounds__(HC_THREADS, 1)
    hess_cluster_global_kernel(cplx* const* __restrict__ Hs, cplx* const* __restrict__ Zs, int n) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ cplx s_red[HC_WARPS];
  __shared__ cplx s_scale;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  cplx* vb = reinterpret_cast<cplx*>(smem_raw);  // [2][HG_MAXN]
  cplx* yp = vb + 2 * HG_MAXN;                    // [2][HC_CS][HG_MAXN]
  cplx* taus = yp + 2 * HC_CS * HG_MAXN;          // [HG_MAXN]
  cplx* us = taus + HG_MAXN;                      // [HG_MAXW]
  cplx* ca = us + HG_MAXW;                        // [HG_MAXW]

  const int nc = rank < n ? (n - rank + HC_CS - 1) / HC_CS : 0;
  auto first_local = [&](int j0) { return j0 > rank ? (j0 - rank + HC_CS - 1) / HC_CS : 0; };
  cplx* H = Hs[blockIdx.y];
  cplx* Z = Zs[blockIdx.y];
  auto colp = [&](int jl) { return H + (size_t)(rank + HC_CS * jl) * n; };
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  cluster.sync();  // every CTA of the cluster runs before shared memory is written remotely

  for (int k = 0; k + 2 < n; ++k) {
    const int j0 = k + 1;
    const int par = k & 1;
    cplx* v = vb + par * HG_MAXN;
    if (k % HC_CS == rank) {
      cplx* col = colp(k / HC_CS);
      cplx a[HG_RPT];
      double part = 0.0;
#pragma unroll
      for (int q = 0; q < HG_RPT; ++q) {
        const int i = tid + HC_THREADS * q;
        a[q] = (i < n && i > j0) ? col[i] : mk(0.0, 0.0);
        part += cabs2(a[q]);
      }
      const double xn = block_sum(mk(part, 0.0), s_red).x;
      if (tid == 0) {
        double beta;
        cplx tau, scale;
        householder(col[j0], xn, &beta, &tau, &scale);
        col[j0] = mk(beta, 0.0);
        s_scale = scale;
        for (int r = 0; r < HC_CS; ++r) cluster.map_shared_rank(taus, r)[k] = tau;
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < HG_RPT; ++q) {
        const int i = tid + HC_THREADS * q;
        if (i >= n || i < j0) continue;
        cplx vi = mk(1.0, 0.0);
        if (i > j0) {
          vi = cmul(a[q], s_scale);
          col[i] = vi;  // kept below the subdiagonal for Q
        }
        for (int r = 0; r < HC_CS; ++r) cluster.map_shared_rank(v, r)[i] = vi;
      }
    }
    cluster.sync();  // reflector k visible in every CTA
    const cplx tau = taus[k];
    if (tau.x == 0.0 && tau.y == 0.0) continue;  // the same decision in every CTA
    const int jl0 = first_local(j0);
    cplx vi[HG_RPT];
#pragma unroll
    for (int q = 0; q < HG_RPT; ++q) {
      const int i = tid + HC_THREADS * q;
      vi[q] = (i < n && i >= j0) ? v[i] : mk(0.0, 0.0);
    }
    // partial y (thread per row) and u (warp per column)
#pragma unroll
    for (int q = 0; q < HG_RPT; ++q) {
      const int i = tid + HC_THREADS * q;
      if (i >= n) continue;
      cplx ya = mk(0.0, 0.0), yb = mk(0.0, 0.0);
      int jl = jl0;
      for (; jl + 1 < nc; jl += 2) {
        ya = cfma(colp(jl)[i], v[rank + HC_CS * jl], ya);
        yb = cfma(colp(jl + 1)[i], v[rank + HC_CS * (jl + 1)], yb);
      }
      if (jl < nc) ya = cfma(colp(jl)[i], v[rank + HC_CS * jl], ya);
      const cplx yi = cadd(ya, yb);
      for (int r = 0; r < HC_CS; ++r) cluster.map_shared_rank(yp, r)[(par * HC_CS + rank) * HG_MAXN + i] = yi;
    }
    for (int jl = jl0 + warp; jl < nc; jl += HC_WARPS) {
      const cplx* col = colp(jl);
      cplx p0 = mk(0.0, 0.0), p1 = mk(0.0, 0.0);
      int r = j0 + lane;
      for (; r + 32 < n; r += 64) {
        p0 = cadd(p0, cmulc(v[r], col[r]));
        p1 = cadd(p1, cmulc(v[r + 32], col[r + 32]));
      }
      if (r < n) p0 = cadd(p0, cmulc(v[r], col[r]));
      const cplx pu = warp_sum_c(cadd(p0, p1));
      if (lane == 0) us[jl] = pu;
    }
    cluster.sync();  // all partial y delivered
    cplx y[HG_RPT];
    cplx sl = mk(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < HG_RPT; ++q) {
      const int i = tid + HC_THREADS * q;
      y[q] = mk(0.0, 0.0);
      if (i < n) {
#pragma unroll
        for (int r = 0; r < HC_CS; ++r) y[q] = cadd(y[q], yp[(par * HC_CS + r) * HG_MAXN + i]);
        if (i >= j0) sl = cadd(sl, cmulc(vi[q], y[q]));
      }
    }
    const cplx s = block_sum(sl, s_red);
    const cplx ts = cmul(tau, s), tauc = cconj(tau);
    for (int jl = jl0 + tid; jl < nc; jl += HC_THREADS) {
      const cplx vjc = cconj(v[rank + HC_CS * jl]);
      ca[jl] = cmul(tau, vjc);
      us[jl] = cmul(tauc, csub(us[jl], cmul(ts, vjc)));
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < HG_RPT; ++q) {
      const int i = tid + HC_THREADS * q;
      if (i >= n) continue;
      const cplx vt = (i >= j0) ? vi[q] : mk(0.0, 0.0);
#pragma unroll 4
      for (int jl = jl0; jl < nc; ++jl) {
        cplx* p = colp(jl) + i;
        *p = csub(csub(*p, cmul(y[q], ca[jl])), cmul(vt, us[jl]));
      }
    }
    __syncthreads();
  }

  // --- accumulate Q in place in this CTA's columns of Z
  __threadfence();
  cluster.sync();  // every column of H, with its reflector, is in global memory
  for (int jl = 0; jl < nc; ++jl) {
    cplx* zc = Z + (size_t)(rank + HC_CS * jl) * n;
    for (int i = tid; i < n; i += HC_THREADS) zc[i] = mk(i == rank + HC_CS * jl ? 1.0 : 0.0, 0.0);
  }
  auto fetch = [&](int k, int i) -> cplx {
    if (k < 0 || i >= n) return mk(0.0, 0.0);
    if (i == k + 1) return mk(1.0, 0.0);
    return i > k + 1 ? H[(size_t)k * n + i] : mk(0.0, 0.0);
  };
  cplx vnext[HG_RPT];
#pragma unroll
  for (int q = 0; q < HG_RPT; ++q) vnext[q] = fetch(n - 3, tid + HC_THREADS * q);
  for (int k = n - 3; k >= 0; --k) {
    const int j0 = k + 1;
    cplx* v = vb + (k & 1) * HG_MAXN;
#pragma unroll
    for (int q = 0; q < HG_RPT; ++q) {
      const int i = tid + HC_THREADS * q;
      if (i < n) v[i] = vnext[q];
      vnext[q] = fetch(k - 1, i);
    }
    __syncthreads();
    const cplx tau = taus[k];
    if (tau.x == 0.0 && tau.y == 0.0) continue;
    for (int jl = first_local(j0) + warp; jl < nc; jl += HC_WARPS) {
      cplx* col = Z + (size_t)(rank + HC_CS * jl) * n;
      cplx wp = mk(0.0, 0.0);
      for (int r = j0 + lane; r < n; r += 32) wp = cadd(wp, cmulc(v[r], col[r]));
      wp = warp_sum_c(wp);
      const cplx tw = cmul(tau, wp);
      for (int r = j0 + lane; r < n; r += 32) col[r] = csub(col[r], cmul(v[r], tw));
    }
  }
  __syncthreads();
  cluster.sync();  // no CTA still reads reflectors from H
  for (int jl = 0; jl < nc; ++jl) {
    const int c = rank + HC_CS * jl;
    cplx* hc = H + (size_t)c * n;
    for (int i = c + 2 + tid; i < n; i += HC_THREADS) hc[i] = mk(0.0, 0.0);
  }
}

// ---------------------------------------------------------------------------
// Blocked reduction (the panel scheme of LAPACK's xGEHRD / xLAHR2, complex
// form): for a panel of nb columns starting at column k, a panel kernel (one
// CTA per matrix) forms the panel's reflectors v_i (tau_i), the triangular
// factor T of H_k ... H_(k+nb-1) = I - V T V^H, and Y = A0 V T (A0 = the
// matrix at the panel's start), finishing the panel's columns; the rest is
// DMMA GEMMs:
//   right update   A[:, k+nb:]   -= Y V[k+nb:, :]^H
//   left update    A[J, k+nb:]   -= V[J, :] (T^H (V[J, :]^H A[J, k+nb:]))   (J = k+1 .. n-1)
//   Q accumulation Q[:, J]       -= (Q[:, J] V[J, :]) T V[J, :]^H
// In the panel, column j = k + i is first brought up to date with the
// panel's previous reflectors -- from the right, c -= Y[:, :i] conj(V[j, :i]),
// and from the left, c[J] -= V[:, :i] T[:i, :i]^H V[:, :i]^H c[J] -- then
// reduced; Y[:, i] = tau_i (A0[:, j+1:] v_i - Y[:, :i] (V[:, :i]^H v_i)) and
// T[:i, i] = -tau_i T[:i, :i] V[:, :i]^H v_i, T[i, i] = tau_i.  The only
// pass over the trailing matrix per column is that product with A0, which
// reads columns j+1 .. n-1, not yet written in this panel.
constexpr int HB_NB = 32;
constexpr int HB_THREADS = 256;
constexpr int HB_WARPS = HB_THREADS / 32;

struct HbLayout {
  size_t V, Y, X, W, T, total;  // complex-element offsets in a matrix's scratch
};
__host__ __device__ inline HbLayout hb_layout(int n) {
  HbLayout L;
  size_t o = 0;
  L.V = o;
  o += (size_t)n * HB_NB;  // reflectors, column i = v_i (all n rows)
  L.Y = o;
  o += (size_t)n * HB_NB;
  L.X = o;
  o += (size_t)n * HB_NB;
  L.W = o;
  o += (size_t)HB_NB * n;  // V^H A, then T^H V^H A (leading dimension HB_NB)
  L.T = o;
  o += (size_t)HB_NB * HB_NB;
  L.total = (o + 15) / 16 * 16;
  return L;
}

template <int NT>
__global__ void __launch_bounds__(HB_THREADS)
    hb_panel_kernel(cplx* const* __restrict__ Hs, cplx* __restrict__ scratch, size_t stride, int n, int k, int nbp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* c = reinterpret_cast<cplx*>(smem_raw);  // [n] column being reduced
  cplx* v = c + n;                              // [n] its reflector
  __shared__ cplx s_w[HB_NB], s_w2[HB_NB], s_red[HB_WARPS];
  __shared__ cplx s_tau, s_scale;
  __shared__ double s_beta;
  const HbLayout L = hb_layout(n);
  cplx* H = Hs[blockIdx.x];
  cplx* base = scratch + (size_t)blockIdx.x * stride;
  cplx* V = base + L.V;
  cplx* Y = base + L.Y;
  cplx* T = base + L.T;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int J0 = k + 1;
  // w[l] = sum_{r >= J0} conj(V[r, l]) x[r] for l < i (warp per l)
  auto vh_dot = [&](const cplx* x, int i, cplx* w) {
    for (int l = warp; l < i; l += HB_WARPS) {
      const cplx* vl = V + (size_t)l * n;
      cplx sacc = mk(0.0, 0.0);
      for (int r = J0 + lane; r < n; r += 32) sacc = cadd(sacc, cmulc(vl[r], x[r]));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        sacc.x += __shfl_xor_sync(0xffffffffu, sacc.x, o);
        sacc.y += __shfl_xor_sync(0xffffffffu, sacc.y, o);
      }
      if (lane == 0) w[l] = sacc;
    }
  };
  for (int i = 0; i < nbp; ++i) {
    const int j = k + i;
    // 1-2. column j, updated from the right by the panel's previous reflectors
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int r = tid + HB_THREADS * t;
      if (r < n) {
        cplx a = H[(size_t)j * n + r];
        for (int l = 0; l < i; ++l) a = csub(a, cmul(Y[(size_t)l * n + r], cconj(V[(size_t)l * n + j])));
        c[r] = a;
      }
    }
    __syncthreads();
    // 3. and from the left: c[J] -= V T^H V^H c[J]
    if (i > 0) {
      vh_dot(c, i, s_w);
      __syncthreads();
      if (tid < i) {  // w2 = T^H w, T upper triangular (T(q, l) at T[l * HB_NB + q])
        cplx a = mk(0.0, 0.0);
        for (int q = 0; q <= tid; ++q) a = cadd(a, cmulc(T[(size_t)tid * HB_NB + q], s_w[q]));
        s_w2[tid] = a;
      }
      __syncthreads();
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        const int r = tid + HB_THREADS * t;
        if (r >= J0 && r < n) {
          cplx a = c[r];
          for (int l = 0; l < i; ++l) a = csub(a, cmul(V[(size_t)l * n + r], s_w2[l]));
          c[r] = a;
        }
      }
      __syncthreads();
    }
    // 4. reflector from c[j+1 ..]
    {
      double part = 0.0;
      for (int r = j + 2 + tid; r < n; r += HB_THREADS) part += cabs2(c[r]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
      if (lane == 0) s_red[warp] = mk(part, 0.0);
      __syncthreads();
      if (tid == 0) {
        double xn = 0.0;
        for (int w = 0; w < HB_WARPS; ++w) xn += s_red[w].x;
        double beta;
        cplx tau, scale;
        householder(c[j + 1], xn, &beta, &tau, &scale);
        s_beta = beta;
        s_tau = tau;
        s_scale = scale;
      }
      __syncthreads();
    }
    const cplx tau = s_tau;
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int r = tid + HB_THREADS * t;
      if (r < n) {
        cplx vr = mk(0.0, 0.0), hr = c[r];
        if (r == j + 1) {
          vr = mk(1.0, 0.0);
          hr = mk(s_beta, 0.0);
        } else if (r > j + 1) {
          vr = cmul(c[r], s_scale);
          hr = mk(0.0, 0.0);
        }
        v[r] = vr;
        V[(size_t)i * n + r] = vr;
        H[(size_t)j * n + r] = hr;  // column j is final
      }
    }
    __syncthreads();
    // 5. y = A0[:, j+1:] v (columns right of j are untouched in this panel);
    // four partial sums over interleaved columns keep four independent FMA
    // chains (and their loads) in flight, added in a fixed order
    cplx y[NT];
    {
      cplx ya[4][NT];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int t = 0; t < NT; ++t) ya[u][t] = mk(0.0, 0.0);
      if (!(tau.x == 0.0 && tau.y == 0.0)) {
        int col = j + 1;
        for (; col + 3 < n; col += 4) {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const cplx vc = v[col + u];
            const cplx* hc = H + (size_t)(col + u) * n;
#pragma unroll
            for (int t = 0; t < NT; ++t) {
              const int r = tid + HB_THREADS * t;
              if (r < n) ya[u][t] = cfma(hc[r], vc, ya[u][t]);
            }
          }
        }
        for (; col < n; ++col) {
          const cplx vc = v[col];
          const cplx* hc = H + (size_t)col * n;
#pragma unroll
          for (int t = 0; t < NT; ++t) {
            const int r = tid + HB_THREADS * t;
            if (r < n) ya[0][t] = cfma(hc[r], vc, ya[0][t]);
          }
        }
      }
#pragma unroll
      for (int t = 0; t < NT; ++t) y[t] = cadd(cadd(ya[0][t], ya[1][t]), cadd(ya[2][t], ya[3][t]));
    }
    // 6. Y[:, i] = tau (y - Y[:, :i] w'), w' = V[:, :i]^H v; T column i
    if (i > 0) vh_dot(v, i, s_w);
    __syncthreads();
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int r = tid + HB_THREADS * t;
      if (r < n) {
        cplx a = y[t];
        for (int l = 0; l < i; ++l) a = csub(a, cmul(Y[(size_t)l * n + r], s_w[l]));
        Y[(size_t)i * n + r] = cmul(tau, a);
      }
    }
    if (tid <= i) {
      cplx a = tau;
      if (tid < i) {  // T(q, i) = -tau sum_{p = q}^{i-1} T(q, p) w'[p]
        a = mk(0.0, 0.0);
        for (int p = tid; p < i; ++p) a = cadd(a, cmul(T[(size_t)p * HB_NB + tid], s_w[p]));
        a = cneg(cmul(tau, a));
      }
      T[(size_t)i * HB_NB + tid] = a;
    } else if (tid < HB_NB) {
      // the strictly lower part: the GEMM stages read T as a full block
      T[(size_t)i * HB_NB + tid] = mk(0.0, 0.0);
    }
    __syncthreads();
  }
}

// GEMM descriptors of one panel's seven products for every matrix (stage s
// at descs + s * batch): right update, V^H A, T^H (.), left update, Q V, (.) T,
// Q update.
__global__ void hb_desc_kernel(cplx* const* __restrict__ Hs, cplx* const* __restrict__ Zs, cplx* __restrict__ scratch,
                               size_t stride, int n, int k, int nbp, int batch, GemmDesc* __restrict__ descs) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  const HbLayout L = hb_layout(n);
  cplx* H = Hs[b];
  cplx* Z = Zs[b];
  cplx* base = scratch + (size_t)b * stride;
  cplx *V = base + L.V, *Y = base + L.Y, *X = base + L.X, *W = base + L.W, *T = base + L.T;
  const int J0 = k + 1, c0 = k + nbp;
  cplx* Hr = H + (size_t)c0 * n;  // columns right of the panel
  descs[0 * batch + b] = {Y, V + c0, Hr, Hr, nullptr, nullptr};            // Hr -= Y V[c0:]^H
  descs[1 * batch + b] = {V + J0, Hr + J0, W, nullptr, nullptr, nullptr};  // W = V[J]^H Hr[J]
  descs[2 * batch + b] = {T, W, X, nullptr, nullptr, nullptr};             // X = T^H W
  descs[3 * batch + b] = {V + J0, X, Hr + J0, Hr + J0, nullptr, nullptr};  // Hr[J] -= V[J] X
  descs[4 * batch + b] = {Z + (size_t)J0 * n, V + J0, X, nullptr, nullptr, nullptr};  // X = Z[:, J] V[J]
  descs[5 * batch + b] = {X, T, Y, nullptr, nullptr, nullptr};                      // Y = X T
  descs[6 * batch + b] = {Y, V + J0, Z + (size_t)J0 * n, Z + (size_t)J0 * n, nullptr, nullptr};  // Z[:, J] -= Y V[J]^H
}

template <int NT>
void launch_hb_panel(cplx* const* H, cplx* scratch, size_t stride, int batch, int n, int k, int nbp, cudaStream_t st) {
  const size_t smem = 2 * (size_t)n * sizeof(cplx);
  ensure_smem((const void*)hb_panel_kernel<NT>, smem);
  hb_panel_kernel<NT><<<batch, HB_THREADS, smem, st>>>(H, scratch, stride, n, k, nbp);
}

}  // namespace

size_t hessenberg_blocked_scratch(int n) { return hb_layout(n).total * sizeof(cplx); }
size_t hessenberg_blocked_descs(int batch) { return 7 * (size_t)batch * sizeof(GemmDesc); }

void hessenberg_blocked_batched(cplx* const* d_H, cplx* const* d_Z, int batch, int n, void* scratch,
                                size_t stride_bytes, void* descs, cudaStream_t st) {
  if (batch <= 0) return;
  if (n < 3 || n > 1024 || batch > 65535) throw StatusError(ST_EINVAL, "blocked Hessenberg: n in [3, 1024]");
  if (stride_bytes < hessenberg_blocked_scratch(n) || stride_bytes % sizeof(cplx))
    throw StatusError(ST_EINVAL, "blocked Hessenberg: scratch stride below its layout");
  const size_t stride = stride_bytes / sizeof(cplx);
  cplx* scr = static_cast<cplx*>(scratch);
  GemmDesc* dd = static_cast<GemmDesc*>(descs);
  set_identity_batched(d_Z, batch, n, 1.0, st);
  const cplx one = mk(1.0, 0.0), mone = mk(-1.0, 0.0), zero = mk(0.0, 0.0);
  for (int k = 0; k < n - 2; k += HB_NB) {
    const int nbp = std::min(HB_NB, n - 2 - k);
    const int J0 = k + 1, MJ = n - J0, c0 = k + nbp, N2 = n - c0;
    if (n <= 256) launch_hb_panel<1>(d_H, scr, stride, batch, n, k, nbp, st);
    else if (n <= 512) launch_hb_panel<2>(d_H, scr, stride, batch, n, k, nbp, st);
    else launch_hb_panel<4>(d_H, scr, stride, batch, n, k, nbp, st);
    VRC_CUDA_CHECK(cudaGetLastError());
    hb_desc_kernel<<<(batch + 127) / 128, 128, 0, st>>>(d_H, d_Z, scr, stride, n, k, nbp, batch, dd);
    VRC_CUDA_CHECK(cudaGetLastError());
    if (N2 > 0) {
      zgemm_rect_batched(dd + 0 * (size_t)batch, batch, n, N2, nbp, n, n, n, mone, one, st, 0, 1);
      zgemm_rect_batched(dd + 1 * (size_t)batch, batch, nbp, N2, MJ, n, n, HB_NB, one, zero, st, 1, 0);
      zgemm_rect_batched(dd + 2 * (size_t)batch, batch, nbp, N2, nbp, HB_NB, HB_NB, HB_NB, one, zero, st, 1, 0);
      zgemm_rect_batched(dd + 3 * (size_t)batch, batch, MJ, N2, nbp, n, HB_NB, n, mone, one, st, 0, 0);
    }
    zgemm_rect_batched(dd + 4 * (size_t)batch, batch, n, nbp, MJ, n, n, n, one, zero, st, 0, 0);
    zgemm_rect_batched(dd + 5 * (size_t)batch, batch, n, nbp, nbp, n, HB_NB, n, one, zero, st, 0, 0);
    zgemm_rect_batched(dd + 6 * (size_t)batch, batch, n, MJ, nbp, n, n, n, mone, one, st, 0, 1);
  }
}

bool hessenberg_cluster_fits(int n) { return n >= 3 && n <= HG_MAXN; }

void hessenberg_cluster_batched(cplx* const* d_H, cplx* const* d_Z, int batch, int n, cudaStream_t st) {
  if (batch <= 0) return;
  if (n > HC_THREADS || hc_layout(n).total > 227 * 1024) {
    ensure_smem((const void*)hess_cluster_global_kernel, HG_SMEM);
    for (int b0 = 0; b0 < batch; b0 += 65535) {
      const int nb = min(65535, batch - b0);
      hess_cluster_global_kernel<<<dim3(HC_CS, nb), HC_THREADS, HG_SMEM, st>>>(d_H + b0, d_Z + b0, n);
    }
    VRC_CUDA_CHECK(cudaGetLastError());
    return;
  }
  const size_t smem = hc_layout(n).total;
  ensure_smem((const void*)hess_cluster_kernel, smem);
  for (int b0 = 0; b0 < batch; b0 += 65535) {
    const int nb = min(65535, batch - b0);
    hess_cluster_kernel<<<dim3(HC_CS, nb), HC_THREADS, smem, st>>>(d_H + b0, d_Z + b0, n);
  }
  VRC_CUDA_CHECK(cudaGetLastError());
}

}  // namespace vrc
