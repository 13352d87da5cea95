// Host-side launchers of the device kernels (internal interface of the
// engine; the public boundary is include/vrc.h).
#pragma once

#include "common.cuh"

namespace vrc {

// Raise a kernel's dynamic shared-memory limit to at least `bytes` (above the
// 48 KB default).  The limit only grows, under a lock, so launchers may run
// from several host threads (one engine per thread).
void ensure_smem(const void* kernel, size_t bytes);

// ---- GEMM: C = diag(rs) (alpha A B) diag(cs) + beta Cin + delta I -----------
struct GemmDesc {
  const cplx* A;
  const cplx* B;
  cplx* C;
  const cplx* Cin;  // may be null (beta ignored) or alias C
  const cplx* rs;   // optional row scale (n)
  const cplx* cs;   // optional column scale (n)
};
// opA / opB = 1 takes that operand as its conjugate transpose (kdim == n).
// tile: 64 (64 x 64 complex per CTA) or 32 (32 x 32); results are identical.
// throws ST_ETIMEOUT when a bulk-staged GEMM (VRC_GEMM_BULK) gave up waiting
// for a stage since the last check; call after a stream synchronisation
void gemm_bulk_check();
void zgemm_batched(const GemmDesc* d_descs, int batch, int n, cplx alpha, cplx beta, double delta,
                   cudaStream_t stream, int kdim = -1, int opA = 0, int opB = 0, int tile = 64);  // kdim < 0: n
// Rectangular form: C (M x N, leading dimension ldc) = alpha op(A) op(B)
// (+ beta Cin, same ldc) with op(A) M x K and op(B) K x N; A is stored M x K
// (lda) or, with opA, K x M; B is stored K x N (ldb) or, with opB, N x K.
// The descriptors' rs / cs scale rows (M) / columns (N).
void zgemm_rect_batched(const GemmDesc* d_descs, int batch, int M, int N, int K, int lda, int ldb, int ldc,
                        cplx alpha, cplx beta, cudaStream_t stream, int opA = 0, int opB = 0, int tile = 64);

// ---- inverse (in place) -------------------------------------------------------
int zinv_panel_width(int n);
void zinv_batched(cplx* const* d_mats, int batch, int n, int* d_status, cudaStream_t stream);
// Blocked inversion with the rank-w updates as tensor-core GEMMs.  scratch:
// zinv_blocked_scratch(n) bytes per matrix; d_descs[b] = {M_b, M_b + n W,
// mat_b, mat_b} with M_b = scratch + b * zinv_blocked_scratch(n) and
// W = zinv_blocked_width(n).
int zinv_blocked_width(int n);
size_t zinv_blocked_scratch(int n);
void zinv_blocked_batched(cplx* const* d_mats, int batch, int n, int* d_status, void* scratch,
                          const GemmDesc* d_descs, cudaStream_t stream);

// ---- eigensolver ---------------------------------------------------------------
void hessenberg_batched(cplx* const* d_H, cplx* const* d_Z, int batch, int n, cudaStream_t st);
// The same reduction by one cluster of CTAs per matrix with the matrix in
// distributed shared memory (hessenberg.cu); for n where it fits.
bool hessenberg_cluster_fits(int n);
void hessenberg_cluster_batched(cplx* const* d_H, cplx* const* d_Z, int batch, int n, cudaStream_t st);
// Blocked reduction (32-column panels, DMMA GEMM updates): scratch of
// hessenberg_blocked_scratch(n) bytes per matrix (matrix b's at scratch +
// b * stride_bytes) and a device buffer of hessenberg_blocked_descs(batch)
// bytes for the GEMM descriptors; batch <= 65535.
size_t hessenberg_blocked_scratch(int n);
size_t hessenberg_blocked_descs(int batch);
void hessenberg_blocked_batched(cplx* const* d_H, cplx* const* d_Z, int batch, int n, void* scratch,
                                size_t stride_bytes, void* descs, cudaStream_t st);
// Complex Schur form + Schur vectors.  d_logs: one rotation-log buffer of
// schur_log_bytes(n) bytes per matrix (device scratch, contents overwritten).
// parts: SCHUR_ITERATE (QR sweeps on the active windows, rotations logged),
// SCHUR_REPLAY (logged rotations applied to Z and to H outside the windows),
// or both, in that order.
size_t schur_log_bytes(int n);
constexpr int SCHUR_ITERATE = 1, SCHUR_REPLAY = 2;
void schur_batched(cplx* const* d_H, cplx* const* d_Z, cplx* const* d_W, void* const* d_logs, int batch, int n,
                   int* d_status, cudaStream_t st, int parts = SCHUR_ITERATE | SCHUR_REPLAY);
void trevc_batched(cplx* const* d_T, cplx* const* d_Y, int batch, int n, cudaStream_t st);
void vecnorm_batched(cplx* const* d_X, int batch, int n, cudaStream_t st);

// ---- assembly -------------------------------------------------------------------
void pillar_raster(const double* d_radius, cplx* const* d_eps, int batch, int npx, int npy, double Lx,
                   double Ly, cplx eps_in, cplx eps_out, cudaStream_t st);
// per-sample grid geometry from a structure's rule tables (one job each)
struct GridGeomJob {
  double z;
  const double* gd;  // base x, base y, rule knots / values / second derivatives
  const int* gi;     // per rule: axis, index, knot count, offset into gd after the bases, spline
  int nrules, slot;  // slot: entry of the eps pointer array this sample sets
  const cplx* eps;   // the structure's eps table (ncy-1) x (ncx-1)
  cplx* refill;      // room for a refilled copy
  double* coords;    // out: x, sorted x, y
};
void grid_geometry(const GridGeomJob* d_jobs, int njobs, int ncx, int ncy, const cplx** d_eps_out, cudaStream_t st);
void twiddles(const double* const* d_coords, cplx* const* d_out, int batch, int ncoord, int P, cudaStream_t st);
void reciprocal(cplx* const* d_in, cplx* const* d_out, int batch, int total, cudaStream_t st);
void small_gemm(int M, int N, int K, const cplx* const* d_A, int lda, const cplx* const* d_B, int ldb, int transB,
                cplx* const* d_C, int ldc, int batch, cudaStream_t st);
void toeplitz_inverses(const cplx* const* d_F, cplx* const* d_out, int t, int nmat, int batch, int* d_status,
                       cudaStream_t st);
void gather_fe(const cplx* const* d_G11, const cplx* const* d_G22, const cplx* const* d_F2, cplx* const* d_fe11,
               cplx* const* d_fe22, cplx* const* d_fe33, int nx, int ny, int batch, cudaStream_t st);
// d_ab: per sample alpha (m) then beta (m), 2 m doubles per sample
void assemble_periodic(const cplx* const* d_finv, const cplx* const* d_fe11, const cplx* const* d_fe22,
                       const double* d_ab, const double* d_k0sq, cplx* const* d_P, cplx* const* d_Q, int m, int batch,
                       cudaStream_t st);
// KxKy ... KyKx: per sample (each sample's cell constants)
void assemble_dense(const cplx* const* KxF2h, const cplx* const* KxF1h, const cplx* const* KyF2h,
                    const cplx* const* KyF1h, const cplx* const* fe11, const cplx* const* fe22,
                    const cplx* const* KxKy, const cplx* const* KxKx, const cplx* const* KyKy,
                    const cplx* const* KyKx, const double* d_k0sq, cplx* const* d_P, cplx* const* d_Q, int m,
                    int batch, cudaStream_t st);

// ---- segment / elementwise ------------------------------------------------------
struct SegDesc {
  const cplx* X0;
  const cplx* Y0;
  const cplx* X2;
  const cplx* Y2;
  const cplx* gam;
  cplx* tdd;
  cplx* tuu;
  cplx* rud;
  cplx* rdu;
  double* err;
  double z0, z1, k0;
};
struct PowerDesc {
  const cplx* r;  // reflected harmonics [rx; ry] (2m)
  const cplx* t;  // transmitted harmonics [tx; ty]
  const double* alpha;
  const double* beta;
  double* R;
  double* T;
  cplx eps_in, eps_out;
  double k0, tnorm;
};
struct MatVecDesc {
  const cplx* A;
  const cplx* x;
  cplx* y;
};
void gamma_batched(const cplx* const* lams, cplx* const* gams, cplx* const* invgams, int batch, int n,
                   cudaStream_t st);
void sub_batched(const cplx* const* A, const cplx* const* B, cplx* const* C, int batch, long long total,
                 cudaStream_t st);
void ab_batched(cplx* const* F, cplx* const* G, int batch, long long total, cudaStream_t st);
void simpson_batched(const SegDesc* d_segs, int batch, int n, cudaStream_t st);
void phase_rows_batched(const cplx* const* A, const cplx* const* gam, const double* t, cplx* const* out, int batch,
                        int n, cudaStream_t st);
void set_identity_batched(cplx* const* A, int batch, int n, double diag, cudaStream_t st);
void axpby_batched(const cplx* const* A, const cplx* const* B, cplx* const* C, cplx alpha, cplx beta, double delta,
                   int batch, int n, cudaStream_t st);
void order_power_batched(const PowerDesc* d, int batch, int m, cudaStream_t st);
void matvec_batched(const MatVecDesc* d, int batch, int n, cudaStream_t st);

// ---- layer-stack forward / adjoint (adjoint.cu) ------------------------------------
// out = diag(rs) A diag(cs); rs / cs (or an entry of them) may be null.
void scale_batched(const cplx* const* A, const cplx* const* rs, const cplx* const* cs, cplx* const* out, int batch,
                   int n, cudaStream_t st);
// out_i = exp(i gam_i t)
void phase_vec_batched(const cplx* const* gam, const double* t, cplx* const* out, int batch, int n, cudaStream_t st);
struct LayerAdjDesc {
  const cplx *gtdd, *gtuu, *grud, *grdu;  // own-basis block adjoints
  const cplx* gam;
  cplx *gS, *gD;  // gA + gB, gA - gB
  double d, k0;
};
void layer_adjoint_batched(const LayerAdjDesc* d, int batch, int n, cudaStream_t st);
struct PQAdjDesc {
  const cplx *gP, *gQ;
  const double *alpha, *beta;
  cplx *g11, *g22, *Z;  // m x m each
  double k0;
};
void pq_adjoint_batched(const PQAdjDesc* d, int batch, int m, cudaStream_t st);
struct PixAdjDesc {
  const cplx* eps;                 // npy x npx, row-major (rows = y strips)
  const cplx *g11, *g22, *g33;     // m x m
  double* grad;                    // npy x npx
  cplx* kscr;                      // pixel_adjoint_scratch(nx, ny) bytes of device scratch
  double Lx, Ly;
};
// dL/d(thickness) of a layer: Re sum_i conj(gtdd_ii + gtuu_ii) (i gam_i / k0) x_i
// with x = exp(i gam d / k0) (one CTA per layer).
struct ThickAdjDesc {
  const cplx *gtdd, *gtuu, *gam, *x;
  double* out;
  double k0;
};
void thick_adjoint_batched(const ThickAdjDesc* d, int batch, int n, cudaStream_t st);
// Interface fields: e = W (ap + am) (one CTA per interface), then Ex, Ey on an
// ngx x ngy grid over the period from the harmonics (index ny*i + j).
struct IfFieldDesc {
  const cplx *W, *ap, *am;
  cplx* e;  // n
  const double *alpha, *beta;
  cplx* img;  // 2 * ngy * ngx (Ex then Ey), may be null
  double Lx, Ly;
};
void interface_fields_batched(const IfFieldDesc* d, int batch, int n, int ngx, int ngy, cudaStream_t st);
// y = a + b * s (vectors of n)
void vec_axpy_batched(const cplx* const* a, const cplx* const* b, cplx s, cplx* const* y, int batch, int n,
                      cudaStream_t st);
bool pixel_adjoint_fits(int nx, int ny, int npx, int npy);
size_t pixel_adjoint_scratch(int nx, int ny);
void pixel_adjoint_batched(const PixAdjDesc* d, int batch, int nx, int ny, int npx, int npy, cudaStream_t st);
struct StackPowerDesc {
  const cplx *W0, *W0inv, *W1, *Tuu, *Rdu;
  const double *alpha, *beta;
  const double *wR, *wT;  // adjoint weights (m), used when adj
  double *REF, *TRN;      // m
  cplx *gRdu, *gTuu;      // n x n, written when adj
  cplx eps_in, eps_out;
  double k0, px, py;
  int nx, ny;
};
void stack_power_batched(const StackPowerDesc* d, int batch, int m, int adj, cudaStream_t st);

}  // namespace vrc
