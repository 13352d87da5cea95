// P,Q assembly per z-sample (Fourier-Toeplitz convolution matrices, Laurent
// rule for eps33, Li inverse rule for eps11/eps22) -- the device restatement
// of Layer::waveEqnCoeff (src/rcwa/Layer.cpp:36-171) over
// FourierSolver2D::solve (src/rcwa/FourierSolver2D.cpp:12-351).
//
// The closed-form Fourier coefficient of cell [x0,x1] of a period-d grid is
//   E[p][c] = exp(-i pi m (x0+x1)/d) sin(pi m w/d)/(pi m),  E = w/d at m = 0
// (src/rcwa/FourierSolver1D.cpp:23-39).  Every sum of the reference becomes a
// small batched contraction with these twiddle tables:
//   AX = Ex * (1/eps)^T     x-Fourier of 1/eps per y-strip      (fe11)
//   AY = Ey * (1/eps)       y-Fourier of 1/eps per x-cell       (fe22)
//   F2 = (Ex * eps^T) Ey^T  2D Fourier of eps                   (fe33)
//   G11 = vec(inv Toep(AX_r)) * Ey^T,  G22 = Exs * vec(inv Toep(AY_c))^T
// followed by the Toeplitz / block-Toeplitz gathers
// (src/rcwa/ToeplitzMatrixXcs.cpp:8-38, BlockToeplitzMatrixXcs.cpp:5-53).
#include "common.cuh"
#include "kernels.h"

#include <algorithm>

namespace vrc {
namespace {

constexpr double PI_D = 3.1415926535897932;  // src/rcwa/defns.h:25

// ---------------------------------------------------------------------------
// Pillar raster: eps[r][c] (row-major, rows = y strips) for each sample.
// ---------------------------------------------------------------------------
__global__ void pillar_raster_kernel(const double* __restrict__ radius, cplx* const* __restrict__ eps,
                                     int npx, int npy, double Lx, double Ly, cplx eps_in,
                                     cplx eps_out) {
  const int s = blockIdx.y;
  const double r = radius[s];
  const double r2 = r * r;
  cplx* e = eps[s];
  const int total = npx * npy;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    int row = idx / npx, col = idx - row * npx;
    double xc = (col + 0.5) * (Lx / npx) - 0.5 * Lx;
    double yc = (row + 0.5) * (Ly / npy) - 0.5 * Ly;
    e[idx] = (xc * xc + yc * yc <= r2) ? eps_in : eps_out;
  }
}

// ---------------------------------------------------------------------------
// Grid geometry on the device (the coordinate rules of
// VarLayerSampler::addXRule / addYRule, src/core/VarLayerSampler.cpp:42-69,
// tabulated once per structure): per sample the moving coordinates at z, the
// sorted copy of x and, where coordinates cross, the painter's-order refill
// of the permittivity columns (src/rcwa/FourierSolver1D.cpp:145-193).
// ---------------------------------------------------------------------------
// Rule value at z through knots zs with values vals: linear, or the natural
// cubic spline with second derivatives M (h = z_hi - z_lo, b = (z - z_lo) / h,
// a = 1 - b: a y_lo + b y_hi + ((a^3 - a) M_lo + (b^3 - b) M_hi) h^2 / 6);
// constant beyond the end knots.
__device__ double rule_eval(double z, const double* zs, const double* vals, const double* M, int K, int spline) {
  if (K <= 0) return 0.0;
  if (z <= zs[0]) return vals[0];
  if (z >= zs[K - 1]) return vals[K - 1];
  int lo = 0, hi = K - 1;  // zs[lo] <= z < zs[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (zs[mid] <= z) lo = mid;
    else hi = mid;
  }
  const double h = zs[hi] - zs[lo];
  const double b = (z - zs[lo]) / h, a = 1.0 - b;
  double x = a * vals[lo] + b * vals[hi];
  if (spline) x += ((a * a * a - a) * M[lo] + (b * b * b - b) * M[hi]) * h * h / 6.0;
  return x;
}

// One block per sample.  Table layout (GridGeomJob): gd = base x (ncx), base
// y (ncy), then each rule's knots, values and second derivatives at its
// offset; gi = per rule (axis, index, K, offset, spline).  Rules apply in
// order (a later rule on the same coordinate wins).  Output: coords = x
// (ncx), sorted x (ncx), y (ncy); eps_out[slot] = the structure's eps, or
// the refilled copy in refill where coordinates cross.
__global__ void grid_geometry_kernel(const GridGeomJob* __restrict__ jobs, int ncx, int ncy, int nr, int nc,
                                     const cplx** __restrict__ eps_out) {
  extern __shared__ __align__(16) unsigned char gsm[];
  double* x = reinterpret_cast<double*>(gsm);
  int* rindex = reinterpret_cast<int*>(x + ncx);
  const GridGeomJob jb = jobs[blockIdx.x];
  const int t = threadIdx.x;
  double* xo = jb.coords;
  double* xso = xo + ncx;
  double* yo = xso + ncx;
  for (int q = t; q < ncx; q += blockDim.x) x[q] = jb.gd[q];
  for (int q = t; q < ncy; q += blockDim.x) yo[q] = jb.gd[ncx + q];
  __syncthreads();
  if (t == 0) {
    for (int r = 0; r < jb.nrules; ++r) {
      const int* g = jb.gi + 5 * r;
      const double* base = jb.gd + ncx + ncy + g[3];
      const double v = rule_eval(jb.z, base, base + g[2], base + 2 * g[2], g[2], g[4]);
      if (g[0] == 0) x[g[1]] = v;
      else yo[g[1]] = v;
    }
  }
  __syncthreads();
  // stable rank of each x (ties keep their order): the sorted copy and the
  // painter's order of the cells
  int moved = 0;
  for (int q = t; q < ncx; q += blockDim.x) {
    const double v = x[q];
    int rank = 0;
    for (int j = 0; j < ncx; ++j) rank += (x[j] < v || (x[j] == v && j < q)) ? 1 : 0;
    rindex[q] = rank;
    xo[q] = v;
    xso[rank] = v;
    moved |= rank != q;
  }
  const int need = __syncthreads_or(moved);
  if (!need) {
    if (t == 0) eps_out[jb.slot] = jb.eps;
    return;
  }
  // a later cell overrides an earlier one on the columns its sorted span covers
  for (int e = t; e < nr * nc; e += blockDim.x) {
    const int row = e / nc, j = e - row * nc;
    cplx v = jb.eps[e];
    for (int i = 0; i < nc; ++i)
      if (x[i] < x[i + 1] && rindex[i] <= j && rindex[i + 1] >= j + 1) v = jb.eps[(size_t)row * nc + i];
    jb.refill[e] = v;
  }
  if (t == 0) eps_out[jb.slot] = jb.refill;
}

// ---------------------------------------------------------------------------
// Twiddle tables: T[p][c] column-major (P x ncell), P = 2*nh-1.
// ---------------------------------------------------------------------------
__global__ void twiddle_kernel(const double* const* __restrict__ coords, cplx* const* __restrict__ out,
                               int ncoord, int P) {
  const int s = blockIdx.y;
  const double* x = coords[s];
  cplx* T = out[s];
  const int ncell = ncoord - 1;
  const double d = x[ncoord - 1] - x[0];
  const int half = (P - 1) / 2;
  const int total = P * ncell;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    int c = idx / P, p = idx - c * P;
    int m = p - half;
    double x0 = x[c], x1 = x[c + 1];
    double w = x1 - x0;
    cplx v;
    if (m == 0) {
      v = mk(w / d, 0.0);
    } else {
      double sn, cs;
      sincos(-(m * PI_D * (x1 + x0) / d), &sn, &cs);
      double amp = sin(PI_D * m * w / d) / (PI_D * m);
      v = mk(amp * cs, amp * sn);
    }
    T[idx] = v;
  }
}

__global__ void reciprocal_kernel(cplx* const* __restrict__ in, cplx* const* __restrict__ out, int total) {
  const cplx* a = in[blockIdx.y];
  cplx* b = out[blockIdx.y];
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x)
    b[idx] = cinv(a[idx]);
}

// ---------------------------------------------------------------------------
// Small batched contraction C[M x N] = A[M x K] * op(B), column-major,
// one thread per output element (the operands are L1/L2 resident).
// transB = 0: B is K x N (ldb); transB = 1: B is N x K (ldb), use B^T.
// ---------------------------------------------------------------------------
__global__ void small_gemm_kernel(int M, int N, int K, const cplx* const* __restrict__ As, int lda,
                                  const cplx* const* __restrict__ Bs, int ldb, int transB,
                                  cplx* const* __restrict__ Cs, int ldc) {
  const int s = blockIdx.y;
  const cplx* A = As[s];
  const cplx* B = Bs[s];
  cplx* C = Cs[s];
  const int total = M * N;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    int j = idx / M, i = idx - j * M;
    cplx acc = mk(0.0, 0.0);
    if (!transB) {
      const cplx* b = B + (size_t)j * ldb;
      for (int k = 0; k < K; ++k) acc = cfma(A[(size_t)k * lda + i], b[k], acc);
    } else {
      for (int k = 0; k < K; ++k) acc = cfma(A[(size_t)k * lda + i], B[(size_t)k * ldb + j], acc);
    }
    C[(size_t)j * ldc + i] = acc;
  }
}

// ---------------------------------------------------------------------------
// Toeplitz inverses: for each column r of F (P x nmat, P = 2t-1), build
// T[i][k] = F[t-1+i-k][r] and write inv(T) column-major (t x t) at
// out + r*t*t.  One warp per matrix (t <= 64, lanes own columns j and
// j+32); Gauss-Jordan with partial pivoting, pivot search by warp shuffle.
// ---------------------------------------------------------------------------
constexpr int TI_WARPS = 8;
constexpr int TI_MAXT = 64;

__global__ void __launch_bounds__(TI_WARPS * 32)
    toeplitz_inv_kernel(const cplx* const* __restrict__ Fs, cplx* const* __restrict__ outs, int t,
                        int nmat, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  cplx* a = reinterpret_cast<cplx*>(smem_raw) + warp * (t * t + t);
  cplx* fcol = a + t * t;
  int* piv = reinterpret_cast<int*>(reinterpret_cast<cplx*>(smem_raw) + nw * (t * t + t)) + warp * TI_MAXT;
  const int s = blockIdx.y;
  const int r = blockIdx.x * nw + warp;
  if (r >= nmat) return;
  const int P = 2 * t - 1;
  const cplx* F = Fs[s] + (size_t)r * P;
  for (int idx = lane; idx < t * t; idx += 32) {
    int k = idx / t, i = idx - k * t;
    a[k * t + i] = F[t - 1 + i - k];
  }
  __syncwarp();
  bool bad = false;
  for (int k = 0; k < t; ++k) {
    // pivot search over rows k..t-1 of column k
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
    if (!(best > 0.0)) {
      bad = true;
      p = k;
    }
    if (lane == 0) piv[k] = p;
    // swap rows k, p
    if (p != k) {
      for (int j = lane; j < t; j += 32) {
        cplx tmp = a[j * t + k];
        a[j * t + k] = a[j * t + p];
        a[j * t + p] = tmp;
      }
    }
    __syncwarp();
    const cplx pv = a[k * t + k];
    const cplx ip = (best > 0.0) ? cinv(pv) : mk(1.0, 0.0);
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
  // undo pivoting: swap columns k <-> piv[k], k descending
  for (int k = t - 1; k >= 0; --k) {
    const int p = piv[k];
    if (p != k) {
      for (int i = lane; i < t; i += 32) {
        cplx tmp = a[k * t + i];
        a[k * t + i] = a[p * t + i];
        a[p * t + i] = tmp;
      }
    }
    __syncwarp();
  }
  cplx* out = outs[s] + (size_t)r * t * t;
  for (int idx = lane; idx < t * t; idx += 32) out[idx] = a[idx];
  if (bad && lane == 0 && status) status[s] = ST_ESINGULAR;
}

// ---------------------------------------------------------------------------
// Gathers into fe11 / fe22 / fe33 (m x m, m = nx*ny, index i*ny + j).
// ---------------------------------------------------------------------------
__global__ void gather_fe_kernel(const cplx* const* __restrict__ G11s, const cplx* const* __restrict__ G22s,
                                 const cplx* const* __restrict__ F2s, cplx* const* __restrict__ fe11s,
                                 cplx* const* __restrict__ fe22s, cplx* const* __restrict__ fe33s, int nx,
                                 int ny) {
  const int s = blockIdx.y;
  const int m = nx * ny;
  const int P = 2 * nx - 1, Q = 2 * ny - 1;
  const cplx* G11 = G11s[s];  // (nx*nx) x Q, column-major; row index i + k*nx
  const cplx* G22 = G22s[s];  // P x (ny*ny); column index j + l*ny
  const cplx* F2 = F2s[s];    // P x Q
  cplx* fe11 = fe11s[s];
  cplx* fe22 = fe22s[s];
  cplx* fe33 = fe33s[s];
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < m * m; idx += gridDim.x * blockDim.x) {
    int col = idx / m, row = idx - col * m;
    int i = row / ny, j = row - i * ny;
    int k = col / ny, l = col - k * ny;
    int dx = i - k + nx - 1, dy = j - l + ny - 1;
    fe11[idx] = G11[(size_t)dy * (nx * nx) + (i + k * nx)];
    fe22[idx] = G22[(size_t)(j + l * ny) * P + dx];
    fe33[idx] = F2[(size_t)dy * P + dx];
  }
  (void)Q;
}

// ---------------------------------------------------------------------------
// P, Q assembly for periodic boundaries (Kx = diag(alpha), Ky = diag(beta)).
// src/rcwa/Layer.cpp:91-100 and :134-138.
// ---------------------------------------------------------------------------
__global__ void assemble_periodic_kernel(const cplx* const* __restrict__ finvs,
                                         const cplx* const* __restrict__ fe11s,
                                         const cplx* const* __restrict__ fe22s, const double* __restrict__ ab,
                                         const double* __restrict__ k0sq, cplx* const* __restrict__ Ps,
                                         cplx* const* __restrict__ Qs, int m) {
  const int s = blockIdx.y;
  const double* alpha = ab + (size_t)s * 2 * m;  // per sample: alpha then beta
  const double* beta = alpha + m;
  const cplx* f = finvs[s];
  const cplx* f11 = fe11s[s];
  const cplx* f22 = fe22s[s];
  const double k02 = k0sq[s];
  cplx* P = Ps[s];
  cplx* Q = Qs[s];
  const int n = 2 * m;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < m * m; idx += gridDim.x * blockDim.x) {
    int b = idx / m, a = idx - b * m;
    const double aa = alpha[a], ab = alpha[b], ba = beta[a], bb = beta[b];
    const cplx fv = f[idx];
    const double dlt = (a == b) ? 1.0 : 0.0;
    // P blocks (row a, col b): [0,0] Kx F2h; [0,1] k0^2 I - Kx F1h;
    //                          [1,0] Ky F2h - k0^2 I; [1,1] -Ky F1h
    P[(size_t)b * n + a] = cscale(fv, aa * bb);
    P[(size_t)(b + m) * n + a] = mk(k02 * dlt - aa * ab * fv.x, -aa * ab * fv.y);
    P[(size_t)b * n + a + m] = mk(ba * bb * fv.x - k02 * dlt, ba * bb * fv.y);
    P[(size_t)(b + m) * n + a + m] = cscale(fv, -ba * ab);
    // Q blocks: [0,0] -Kx Ky; [0,1] Kx Kx - k0^2 fe22; [1,0] -Ky Ky + k0^2 fe11; [1,1] Ky Kx
    const cplx g22 = f22[idx], g11 = f11[idx];
    Q[(size_t)b * n + a] = mk(-aa * ba * dlt, 0.0);
    Q[(size_t)(b + m) * n + a] = mk(aa * aa * dlt - k02 * g22.x, -k02 * g22.y);
    Q[(size_t)b * n + a + m] = mk(-ba * ba * dlt + k02 * g11.x, k02 * g11.y);
    Q[(size_t)(b + m) * n + a + m] = mk(ba * aa * dlt, 0.0);
  }
}

// PML: the K products are dense m x m matrices computed by the GEMM engine;
// this kernel places them into the n x n blocks.
//   P = [[KxF2h, k0^2 I - KxF1h], [KyF2h - k0^2 I, -KyF1h]]
//   Q = [[-KxKy, KxKx - k0^2 fe22], [-KyKy + k0^2 fe11, KyKx]]
__global__ void assemble_dense_kernel(const cplx* const* __restrict__ KxF2h, const cplx* const* __restrict__ KxF1h,
                                      const cplx* const* __restrict__ KyF2h, const cplx* const* __restrict__ KyF1h,
                                      const cplx* const* __restrict__ fe11s, const cplx* const* __restrict__ fe22s,
                                      const cplx* const* __restrict__ KxKys, const cplx* const* __restrict__ KxKxs,
                                      const cplx* const* __restrict__ KyKys, const cplx* const* __restrict__ KyKxs,
                                      const double* __restrict__ k0sq, cplx* const* __restrict__ Ps,
                                      cplx* const* __restrict__ Qs, int m) {
  const int s = blockIdx.y;
  const double k02 = k0sq[s];
  const cplx *KxKy = KxKys[s], *KxKx = KxKxs[s], *KyKy = KyKys[s], *KyKx = KyKxs[s];
  const int n = 2 * m;
  cplx* P = Ps[s];
  cplx* Q = Qs[s];
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < m * m; idx += gridDim.x * blockDim.x) {
    int b = idx / m, a = idx - b * m;
    const double dlt = (a == b) ? 1.0 : 0.0;
    P[(size_t)b * n + a] = KxF2h[s][idx];
    cplx t = KxF1h[s][idx];
    P[(size_t)(b + m) * n + a] = mk(k02 * dlt - t.x, -t.y);
    t = KyF2h[s][idx];
    P[(size_t)b * n + a + m] = mk(t.x - k02 * dlt, t.y);
    P[(size_t)(b + m) * n + a + m] = cneg(KyF1h[s][idx]);
    Q[(size_t)b * n + a] = cneg(KxKy[idx]);
    cplx g22 = fe22s[s][idx], g11 = fe11s[s][idx];
    Q[(size_t)(b + m) * n + a] = csub(KxKx[idx], cscale(g22, k02));
    Q[(size_t)b * n + a + m] = cadd(cneg(KyKy[idx]), cscale(g11, k02));
    Q[(size_t)(b + m) * n + a + m] = KyKx[idx];
  }
}

inline dim3 grid_for(int total, int batch, int threads = 256) {
  int bx = (total + threads - 1) / threads;
  if (bx > 1024) bx = 1024;
  if (bx < 1) bx = 1;
  return dim3(bx, batch);
}

}  // namespace

void pillar_raster(const double* d_radius, cplx* const* d_eps, int batch, int npx, int npy, double Lx,
                   double Ly, cplx eps_in, cplx eps_out, cudaStream_t st) {
  if (batch <= 0) return;
  pillar_raster_kernel<<<grid_for(npx * npy, batch), 256, 0, st>>>(d_radius, d_eps, npx, npy, Lx, Ly, eps_in,
                                                                  eps_out);
  VRC_CUDA_CHECK(cudaGetLastError());
}

void grid_geometry(const GridGeomJob* d_jobs, int njobs, int ncx, int ncy, const cplx** d_eps_out, cudaStream_t st) {
  if (njobs <= 0) return;
  const size_t sm = (size_t)ncx * (sizeof(double) + sizeof(int));
  ensure_smem((const void*)grid_geometry_kernel, sm);
  grid_geometry_kernel<<<njobs, 128, sm, st>>>(d_jobs, ncx, ncy, ncy - 1, ncx - 1, d_eps_out);
  VRC_CUDA_CHECK(cudaGetLastError());
}

void twiddles(const double* const* d_coords, cplx* const* d_out, int batch, int ncoord, int P, cudaStream_t st) {
  if (batch <= 0) return;
  twiddle_kernel<<<grid_for(P * (ncoord - 1), batch), 256, 0, st>>>(d_coords, d_out, ncoord, P);
  VRC_CUDA_CHECK(cudaGetLastError());
}

void reciprocal(cplx* const* d_in, cplx* const* d_out, int batch, int total, cudaStream_t st) {
  if (batch <= 0) return;
  reciprocal_kernel<<<grid_for(total, batch), 256, 0, st>>>(d_in, d_out, total);
  VRC_CUDA_CHECK(cudaGetLastError());
}

void small_gemm(int M, int N, int K, const cplx* const* d_A, int lda, const cplx* const* d_B, int ldb, int transB,
                cplx* const* d_C, int ldc, int batch, cudaStream_t st) {
  if (batch <= 0) return;
  small_gemm_kernel<<<grid_for(M * N, batch), 256, 0, st>>>(M, N, K, d_A, lda, d_B, ldb, transB, d_C, ldc);
  VRC_CUDA_CHECK(cudaGetLastError());
}

void toeplitz_inverses(const cplx* const* d_F, cplx* const* d_out, int t, int nmat, int batch, int* d_status,
                       cudaStream_t st) {
  if (batch <= 0 || nmat <= 0) return;
  if (t > TI_MAXT) throw StatusError(ST_EINVAL, "harmonics per axis must be <= 64");
  const size_t per_warp = (size_t)(t * t + t) * 16 + TI_MAXT * sizeof(int);
  int nw = (int)std::min<size_t>(TI_WARPS, std::max<size_t>(1, (200u << 10) / per_warp));
  size_t smem = per_warp * nw;
  ensure_smem((const void*)toeplitz_inv_kernel, smem);
  dim3 grid((nmat + nw - 1) / nw, batch);
  toeplitz_inv_kernel<<<grid, nw * 32, smem, st>>>(d_F, d_out, t, nmat, d_status);
  VRC_CUDA_CHECK(cudaGetLastError());
}

void gather_fe(const cplx* const* d_G11, const cplx* const* d_G22, const cplx* const* d_F2, cplx* const* d_fe11,
               cplx* const* d_fe22, cplx* const* d_fe33, int nx, int ny, int batch, cudaStream_t st) {
  if (batch <= 0) return;
  int m = nx * ny;
  gather_fe_kernel<<<grid_for(m * m, batch), 256, 0, st>>>(d_G11, d_G22, d_F2, d_fe11, d_fe22, d_fe33, nx, ny);
  VRC_CUDA_CHECK(cudaGetLastError());
}

void assemble_periodic(const cplx* const* d_finv, const cplx* const* d_fe11, const cplx* const* d_fe22,
                       const double* d_ab, const double* d_k0sq, cplx* const* d_P, cplx* const* d_Q, int m, int batch,
                       cudaStream_t st) {
  if (batch <= 0) return;
  assemble_periodic_kernel<<<grid_for(m * m, batch), 256, 0, st>>>(d_finv, d_fe11, d_fe22, d_ab, d_k0sq, d_P, d_Q,
                                                                   m);
  VRC_CUDA_CHECK(cudaGetLastError());
}

void assemble_dense(const cplx* const* KxF2h, const cplx* const* KxF1h, const cplx* const* KyF2h,
                    const cplx* const* KyF1h, const cplx* const* fe11, const cplx* const* fe22,
                    const cplx* const* KxKy, const cplx* const* KxKx, const cplx* const* KyKy,
                    const cplx* const* KyKx, const double* d_k0sq, cplx* const* d_P, cplx* const* d_Q, int m,
                    int batch, cudaStream_t st) {
  if (batch <= 0) return;
  assemble_dense_kernel<<<grid_for(m * m, batch), 256, 0, st>>>(KxF2h, KxF1h, KyF2h, KyF1h, fe11, fe22, KxKy, KxKx,
                                                                KyKy, KyKx, d_k0sq, d_P, d_Q, m);
  VRC_CUDA_CHECK(cudaGetLastError());
}

}  // namespace vrc
