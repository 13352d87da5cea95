/*
 * vrc.h -- C-ABI of the B200-native varRCWA hot path.
 *
 * Plain C types only (pointers, sizes, structs of scalars).  Every matrix is
 * complex128, column-major with leading dimension n (the layout of
 * Eigen::MatrixXcs and of the reference's cuDoubleComplex buffers), where
 * n = 2*nx*ny (src/core/LayerSampler.h:44).  All buffers passed to these
 * entry points are HOST memory unless stated otherwise.
 *
 * Each entry point returns a status code (vrc_status_code); on error
 * vrc_last_error() describes it.  A context is bound to one CUDA device and
 * is not thread-safe (the reference integrators are not either).
 *
 * The reference has no C-ABI; each function below lists the reference
 * interface it replaces.
 */
#ifndef VRC_H_
#define VRC_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double re, im;
} vrc_complex;

typedef struct vrc_context vrc_context;

enum vrc_status_code {
  VRC_OK = 0,
  VRC_EINVAL = 1,     /* invalid argument */
  VRC_ECUDA = 2,      /* CUDA runtime error */
  VRC_ENOMEM = 3,     /* device memory exhausted */
  VRC_ESINGULAR = 4,  /* singular pivot in an LU / inverse */
  VRC_ENOCONV = 5,    /* eigensolver did not converge within its iteration cap */
  VRC_ENONFINITE = 6, /* non-finite value in a segment error estimate */
  VRC_ETIMEOUT = 7,   /* reserved: bounded wait expired */
  VRC_EDEPTH = 8,     /* adaptive recursion hit max_depth before the tolerance */
  VRC_ENODEV = 9      /* no CUDA device / extension not usable */
};

enum vrc_geometry_kind {
  VRC_GEOM_GRID = 0,    /* tensor grid, fixed eps table, moving coordinates */
  VRC_GEOM_PILLAR = 1,  /* uniform raster of a circular pillar, linear radius */
  VRC_GEOM_PIXELS = 2,  /* fixed uniform pixel raster (z-invariant) */
  VRC_GEOM_PLANAR = 3,  /* planar device seen from above: layout polygons in (x, z) */
  VRC_GEOM_SAMPLER = 4  /* the caller's own sampler (callbacks below) */
};

/* The caller's own layer sampler: the two virtual functions of the
 * reference's LayerSampler that the integrators call
 * (src/core/LayerSampler.h:49-55).  Either fills P and Q (n x n,
 * column-major complex128, n = 2*nx*ny, the layout of Eigen::MatrixXcs) at
 * height z and returns 0, or returns nonzero on failure (the call then
 * fails with VRC_EINVAL).
 * vrc_sample_fn: replaces LayerSampler::sample; P and Q are host buffers
 *   (pinned staging inside the engine, copied to the device afterwards).
 * vrc_sample_device_fn: replaces LayerSampler::sampleOnGPU; P and Q are
 *   device buffers on the context's device, preallocated by the engine as
 *   the reference's integrators preallocate theirs
 *   (src/gpu/RedhefferIntegratorGPU.cpp:17-20); `stream` (a cudaStream_t)
 *   is the engine stream that reads them next: work queued on it needs no
 *   further synchronisation, work on other streams must be complete on
 *   return.
 * The engine calls a sampler from the thread that runs its cell: cells of
 * one call may be solved on concurrent host threads, so callbacks of
 * different cells that share state must tolerate concurrent calls. */
typedef int (*vrc_sample_fn)(void* user, double z, vrc_complex* P, vrc_complex* Q);
typedef int (*vrc_sample_device_fn)(void* user, double z, vrc_complex* P, vrc_complex* Q, void* stream);

/* Tabulated z-rule for one coordinate: x[index](z) through the knots
 * (zs[k], vals[k]), zs increasing, constant beyond the end knots;
 * piecewise-linear (interp 0) or the natural cubic spline (interp 1).
 * Replaces VarLayerSampler::addXRule/addYRule with a tabulated rule
 * (src/core/VarLayerSampler.cpp:42-50).  The knot values are the geometric
 * parameters of vrc_redheffer_backward. */
typedef struct {
  int index;
  int nknots;
  const double* zs;
  const double* vals;
  int interp;
} vrc_rule;

/* Optional host callback evaluating arbitrary coordinate rules: called with
 * the z of each sample and the coordinate arrays (already holding the base
 * coordinates and the tabulated rules) to modify in place.  This is how a
 * std::function rule of the reference reaches the engine. */
typedef void (*vrc_geometry_fn)(void* user, double z, double* x, double* y);

/* One structure.  Replaces VarLayerSampler(lambda, nx, ny, x, y, eps,
 * enablePML) (src/core/VarLayerSampler.h:20-28) plus the z-range given to
 * the integrators' constructors (src/core/RedhefferIntegrator.h:34-35). */
typedef struct {
  int kind;          /* vrc_geometry_kind */
  int nx, ny;        /* harmonics per axis, odd; n = 2*nx*ny <= 1024 */
  int pml;           /* 0: periodic, 1: PML on both lateral boundaries */
  double lambda;     /* wavelength (same length unit as the geometry) */
  double z0, z1;     /* integration range */
  /* VRC_GEOM_GRID / VRC_GEOM_PIXELS */
  int ncx, ncy;              /* number of x / y coordinates */
  const double* x;           /* ncx */
  const double* y;           /* ncy */
  const vrc_complex* eps;    /* (ncy-1)*(ncx-1), row-major: rows are y strips */
  int n_xrules;
  const vrc_rule* xrules;
  int n_yrules;
  const vrc_rule* yrules;
  vrc_geometry_fn geometry_fn; /* may be NULL */
  void* geometry_user;
  /* VRC_GEOM_PILLAR */
  double Lx, Ly;
  int npx, npy;
  vrc_complex eps_in, eps_out;
  double r0, r1; /* radius at z0 and at z1 */
  /* homogeneous half-spaces joined at z0 / z1 (else the structure's own
   * eigen-bases there, as the reference integrators do) */
  int has_end0, has_end1;
  vrc_complex eps_end0, eps_end1;
  /* VRC_GEOM_PLANAR: replaces GDSIISampler(lambda, nx, ny, filename, shift,
   * lPML, rPML, lspace, rspace, bPML, uPML, bspace, uspace, permBackground,
   * permDevice, thickness) (src/core/GDSIISampler.h:25-35).  Polygons lie in
   * the layout plane (x across, z along the propagation); at every z the
   * cross-section is the device layer (thickness along y) cut by the
   * polygons, between spacers and PML on all four sides (pml is ignored:
   * always on).  vrc_gds_read loads the polygons of a GDSII file. */
  int npoly;
  const int* poly_start;  /* npoly + 1 point offsets into poly_xz */
  const double* poly_xz;  /* (x, z) pairs */
  double shift[3];        /* x, y, z */
  double pml_w[4];        /* left, right, bottom, top PML widths */
  double space[4];        /* left, right, bottom, top spaces between PML and device */
  double thickness;
  vrc_complex eps_background, eps_device;
  /* VRC_GEOM_SAMPLER: a sampler object of the caller driving any integrator
   * entry point (vrc_redheffer, vrc_redheffer_segments, vrc_rcwa,
   * vrc_differential, vrc_order_powers, vrc_sample_pq), as a
   * std::shared_ptr<LayerSampler> drives the reference integrators
   * (src/core/RedhefferIntegrator.h:34-35).  Set sample or sample_device
   * (sample_device wins when both are set); nx * ny = nDim / 2 is all the
   * integrators need, lambda gives k0.  Half-space ends (has_end0/1) and
   * order powers also need the true odd nx, ny and the periods Lx, Ly
   * (periodic boundaries), from which the engine forms the half-space
   * bases itself. */
  vrc_sample_fn sample;
  vrc_sample_device_fn sample_device;
  void* sample_user;
} vrc_cell;

/* Outputs of one integration.  Matrix pointers may be NULL (not copied). */
typedef struct {
  vrc_complex *Tdd, *Tuu, *Rud, *Rdu; /* n*n each */
  vrc_complex *W0, *V0, *gam0;        /* basis at z0 (n*n, n*n, n) */
  vrc_complex *W1, *V1, *gam1;        /* basis at z1 */
  int status;                         /* per-cell vrc_status_code */
  int n;                              /* matrix dimension */
  int N;                              /* accepted segments / slices (N()) */
  int n_eig;                          /* eigen-decompositions (nEigVal()) */
  int n_samples;                      /* P,Q samples assembled */
  int n_nodes;                        /* segments evaluated (accepted + rejected) */
} vrc_result;

/* Timing of the last integrator call (CUDA events on the engine stream). */
typedef struct {
  double device_ms;   /* first kernel to last kernel of the call */
  long long launches; /* kernel launches issued by the call */
} vrc_timing;

/* ---- context ------------------------------------------------------------ */
int vrc_create(int device, vrc_context** ctx);
void vrc_destroy(vrc_context* ctx);
const char* vrc_last_error(const vrc_context* ctx);
const char* vrc_status_string(int status);
int vrc_get_timing(const vrc_context* ctx, vrc_timing* t);

/* ---- A1-A6: P,Q of the wave equation at given z (one structure) ---------
 * Replaces LayerSampler::sample / sampleOnGPU (src/core/LayerSampler.h:49-55,
 * src/core/VarLayerSampler.cpp:52-69, src/gpu/VarLayerSamplerGPU.cpp:130-214)
 * over Layer::waveEqnCoeff (src/rcwa/Layer.cpp:36-171).
 * P, Q: nz blocks of n*n. */
int vrc_sample_pq(vrc_context* ctx, const vrc_cell* cell, int nz, const double* z, vrc_complex* P,
                  vrc_complex* Q);

/* ---- A7: eigen step -------------------------------------------------------
 * Replaces WaveEquationSolver::solve (src/rcwa/WaveEquationSolver.cpp:24-37):
 * W = eigenvectors of P*Q (unit 2-norm, largest component real),
 * gam = sqrt(eig) on the reference branch, V = Q W diag(1/gam). */
int vrc_wave_solve(vrc_context* ctx, int batch, int n, const vrc_complex* P, const vrc_complex* Q,
                   vrc_complex* W, vrc_complex* V, vrc_complex* gam);
/* Plain eigen-decomposition of batch n*n matrices A (replaces
 * MKLEigenSolver::compute / LAPACKE_zgeev, src/rcwa/MKLEigenSolver.hpp:25-74). */
int vrc_eig(vrc_context* ctx, int batch, int n, const vrc_complex* A, vrc_complex* W, vrc_complex* lam);

/* ---- A8-A11: adaptive varRCWA ---------------------------------------------
 * Replaces RedhefferIntegrator(z0, z1, sampler).compute(p, maxN, pe)
 * (src/core/RedhefferIntegrator.h:34-50, RedhefferIntegrator.cpp:174-314)
 * and RedhefferIntegratorGPU::compute_recursive
 * (src/gpu/RedhefferIntegratorGPU.h:103).  `p` and `maxN` are unused by the
 * reference and omitted; max_depth bounds the trisection depth. */
int vrc_redheffer(vrc_context* ctx, int ncells, const vrc_cell* cells, double pe, int max_depth,
                  vrc_result* results);
/* varRCWA over explicit segment boundaries (cell c: ncuts[c] boundaries
 * cuts[c][0]=z0 < ... < z1), each segment referenced at its midpoint.
 * Replaces RedhefferIntegratorGPU::compute_direct(N) (uniform cuts,
 * src/gpu/RedhefferIntegratorGPU.cpp:361-412) and replays a recorded tree. */
int vrc_redheffer_segments(vrc_context* ctx, int ncells, const vrc_cell* cells, const int* ncuts,
                           const double* const* cuts, vrc_result* results);
/* Segmentation tree of cell `cell` of the last adaptive call: nodes in
 * evaluation order (breadth-first).  Returns the node count (may exceed
 * max_nodes; arrays hold the first max_nodes). */
int vrc_get_tree(vrc_context* ctx, int cell, int max_nodes, double* a, double* b, double* err, int* accepted);

/* ---- gradients of adaptive cells with respect to geometric parameters ------
 * No counterpart in the reference, which has no integrator gradients (its
 * building block is the forward-mode dP/dx of Layer::waveEqnCoeff,
 * src/rcwa/Layer.cpp:104-162); this pair is the C form of an autograd
 * function.  vrc_redheffer_forward is vrc_redheffer (same arguments and
 * results) and keeps the cells and their accepted segmentations for
 * vrc_redheffer_backward until the next forward on the context.
 *
 * vrc_redheffer_backward takes, per cell in call order, the cotangents of
 * the forward's outputs -- gS: 4 n*n (Tdd, Tuu, Rud, Rdu), gB: 4 n*n (W0,
 * V0, W1, V1; NULL: none) -- with the convention dL = Re sum conj(g) dX, and
 * returns grad: per cell, dL/d vals[k] of every knot of every x rule, then
 * every y rule (sum of nknots doubles per cell).  Cells must be
 * VRC_GEOM_GRID; a geometry callback must not overwrite ruled coordinates.
 * The gradient is that of the forward on its accepted segmentation (bases
 * frozen inside, end bases differentiated through their eigen step; exact
 * for objectives that do not depend on how the end modes are normalised,
 * e.g. Fourier-basis blocks and flux-normalised modal powers).  The reverse
 * pass recomputes the segment chain, keeping a checkpoint every
 * `checkpoint_every` segments (0: about the square root of the count), and
 * recomputes each block from its checkpoint. */
int vrc_redheffer_forward(vrc_context* ctx, int ncells, const vrc_cell* cells, double pe, int max_depth,
                          vrc_result* results);
int vrc_redheffer_backward(vrc_context* ctx, const vrc_complex* gS, const vrc_complex* gB, int checkpoint_every,
                           double* grad);

/* ---- A12: plain RCWA --------------------------------------------------------
 * Replaces RCWAIntegrator::compute(N) (src/core/RCWAIntegrator.cpp:20-87)
 * and RCWAIntegratorGPU::compute(N) (src/gpu/RCWAIntegratorGPU.h:59). */
int vrc_rcwa(vrc_context* ctx, int ncells, const vrc_cell* cells, int N, vrc_result* results);

/* ---- A13: differential method ------------------------------------------------
 * Replaces DifferentialIntegrator::compute(N)
 * (src/core/DifferentialIntegrator.cpp:21-134). */
int vrc_differential(vrc_context* ctx, int ncells, const vrc_cell* cells, int N, vrc_result* results);

/* ---- stacks of sections ---------------------------------------------------------
 * A stack of nsections cells, each on its own z-range, solved in order along
 * z: RCWASolver::solve(lambda, layerStack, thickness)
 * (src/rcwa/RCWASolver.cpp:104-113) for layers that may vary with z, so
 * adaptive varRCWA sections and z-uniform layers mix.  Every section is
 * integrated (method 0: adaptive varRCWA with pe, max_depth; 1: RCWA, 2:
 * the differential method, with nslices), all sections as one batch; then
 * the sections are joined in order, each section's entrance re-expressed in
 * the previous section's exit basis (matching the transverse fields W c,
 * V c of the two sides, as RCWASolver's interface matrices do, :460-580)
 * and star-multiplied (:343-458).  The first section's has_end0 and the
 * last's has_end1 set the outer media (the others' end flags are ignored);
 * all sections need the same nx, ny and periods.  result: the stack's
 * blocks, the entrance basis (W0, V0, gam0) and the exit basis (W1, V1,
 * gam1), with N, n_eig ... summed over the sections; vrc_get_tree(ctx, s)
 * gives section s's segmentation.  The stack stays on the device for
 * vrc_chain_order_powers and vrc_chain_fields until the next vrc_chain. */
int vrc_chain(vrc_context* ctx, int nsections, const vrc_cell* sections, int method, double pe, int max_depth,
              int nslices, vrc_result* result);
/* Per-order powers of the last stack (vrc_order_powers' side, flux_norm and
 * layout for one cell: R, T of 2 * nx*ny doubles); needs half-space ends and
 * periodic boundaries (RCWASolver::scatterPlaneWave, :1636-1733). */
int vrc_chain_order_powers(vrc_context* ctx, int side, int flux_norm, double* R, double* T);
/* Mode amplitudes at every interface of the last stack for incident
 * amplitudes c (n, in the entrance basis, going up): interface j = 0 ..
 * nsections is the entrance of section j (j = nsections: the exit); amps
 * holds per interface the up- then the down-going amplitudes in the basis of
 * the region below it (j = 0: incident and reflected; j = nsections:
 * transmitted and zero) -- (nsections + 1) * 2 * n -- the role of
 * RCWASolver::evaluateIntermediateField (:1373-1480).  With ngx, ngy > 0,
 * fields ((nsections + 1) * 2 * ngy * ngx: Ex then Ey, rows of constant y)
 * samples the transverse E field over the period there (fields may be NULL
 * otherwise).  Fields inside a section: split it into two sections there. */
int vrc_chain_fields(vrc_context* ctx, const vrc_complex* c, int ngx, int ngy, vrc_complex* amps,
                     vrc_complex* fields);

/* ---- A14: per-order power -----------------------------------------------------
 * Integrate (method 0: adaptive varRCWA with pe/max_depth, 1: RCWA with
 * N = nslices, 2: differential with N) and return per-order reflected /
 * transmitted power for unit plane waves at normal incidence, polarisation
 * (px,py) = (1,0) then (0,1): R and T hold ncells * 2 * (nx*ny) doubles.
 * side 0: incidence from the z0 medium (Rdu, Tuu); 1: from z1 (Rud, Tdd, the
 * reference's choice).  flux_norm 1 normalises T by the incident medium (so
 * R+T = 1 when lossless); 0 divides by sqrt(eps_out) as the reference does.
 * Replaces RCWASolver::scatterPlaneWave (src/rcwa/RCWASolver.cpp:1636-1733).
 * Requires has_end0 = has_end1 = 1 and periodic boundaries; cells of one
 * call may have different truncations (R/T offsets follow each cell's nx*ny
 * in order). */
int vrc_order_powers(vrc_context* ctx, int ncells, const vrc_cell* cells, int method, double pe, int max_depth,
                     int nslices, int side, int flux_norm, double* R, double* T, int* status);

/* ---- layer stacks: forward solve and adjoint (gradients) -------------------
 * No counterpart in the reference, which has no gradients; this pair is the C
 * form of an autograd function.  A stack is nlayers z-uniform layers, each an
 * npy x npx raster of real permittivity on a uniform (Lx, Ly) grid, between
 * eps_in (below z0, the incidence side) and eps_out; periodic boundaries.
 * vrc_stack_forward integrates each stack as the Redheffer chain of its
 * layers (RedhefferIntegrator.cpp:174-277 on a piecewise-constant structure;
 * equal to RCWAIntegrator with one slice per layer) and returns per-order
 * REF / TRN (nstacks * nx*ny each, flux-normalised, order index ny*i + j for
 * orders (i - (nx-1)/2, j - (ny-1)/2)) for a plane wave (px, py) at normal
 * incidence from eps_in.  Every stack of a call has the same nx, ny, npx, npy
 * and nlayers.  What the backward needs stays on the device until the next
 * vrc_stack_forward on the context.
 * vrc_stack_backward returns grad_eps (nstacks * nlayers * npy * npx) =
 * dL/d(eps pixel) for L = sum_k wR[k] REF[k] + wT[k] TRN[k] (wR, wT:
 * nstacks * nx*ny weights each) and, when grad_thick is not NULL,
 * dL/d(layer thickness) (nstacks * nlayers), a geometric parameter.  The adjoint covers the star-product chain,
 * the eigen step (exact first-order layer perturbation in fixed bases, valid
 * for degenerate eigenvalues) and the Fourier-Toeplitz assembly. */
typedef struct {
  double lam, Lx, Ly;
  int nx, ny;          /* harmonics per axis, odd */
  int npx, npy;        /* raster of every layer */
  int nlayers;
  const double* eps;   /* nlayers * npy * npx, row-major (rows = y), layer 0 at z0 */
  const double* thick; /* nlayers */
  vrc_complex eps_in, eps_out;
} vrc_stack;
int vrc_stack_forward(vrc_context* ctx, int nstacks, const vrc_stack* stacks, double px, double py, double* REF,
                      double* TRN, int* status);
int vrc_stack_backward(vrc_context* ctx, const double* wR, const double* wT, double* grad_eps, double* grad_thick);

/* Internal amplitudes and fields of the stacks of the last vrc_stack_forward
 * (the role of RCWASolver::evaluateIntermediateField and of its field images,
 * src/rcwa/RCWASolver.cpp:1373-1480; written to host buffers here).
 * Interface j = 0..nlayers is the top of region j-1 (region -1: eps_in,
 * region nlayers: eps_out); amps holds, per stack and interface, the up- then
 * the down-going mode amplitudes in that region's eigenbasis
 * (nstacks * (nlayers+1) * 2 * n; j = 0: incident and reflected, j = nlayers:
 * transmitted and zero).  fields (nstacks * (nlayers+1) * 2 * ngy * ngx, Ex
 * then Ey, rows of constant y) samples the transverse E field on an
 * ngx x ngy grid over the period; ngx = ngy = 0 skips it (fields may be NULL). */
int vrc_stack_fields(vrc_context* ctx, int ngx, int ngy, vrc_complex* amps, vrc_complex* fields);

/* ---- GDSII layouts ---------------------------------------------------------
 * BOUNDARY and BOX polygons of the first structure of a GDSII file (the
 * polygons gdstk::read_gds gives GDSIISampler, src/core/GDSIISampler.cpp:32),
 * coordinates in units of `unit` metres (1e-6: micrometres).  Sets npoly and
 * npoints; fills poly_start (npoly + 1 offsets) and poly_xz (2 * npoints)
 * when both are given and large enough (else VRC_EINVAL).  No context and
 * no GPU needed. */
int vrc_gds_read(const char* path, double unit, int* npoly, int* npoints, int* poly_start, double* poly_xz,
                 int max_poly, int max_points);
/* Cross-section of a VRC_GEOM_PLANAR cell at z (GDSIISampler::sampleLayout,
 * src/core/GDSIISampler.cpp:90-140): x (returned count, at most max_x), the
 * six y coordinates and the 5 x (count - 1) eps table (rows are y strips).
 * With NULL outputs only the count is returned; negative on error. */
int vrc_planar_section(const vrc_cell* cell, double z, int max_x, double* x, double* y, vrc_complex* eps);

/* ---- instrumentation (no counterpart in the reference) ---------------------
 * Per-kernel-family device time measured with CUDA events on the engine
 * streams, with the algorithmic FP64 flops and bytes of the timed launches.
 * ms sums the launches' durations; busy_ms is the length of the union of
 * their intervals (they overlap when a call's cells are solved on several
 * concurrent engines). */
typedef struct {
  char name[32];
  double ms;
  long long launches;
  double flops;
  double bytes;
  double busy_ms;
} vrc_kernel_stat;
int vrc_set_profiling(vrc_context* ctx, int enable); /* also resets the counters */
/* Returns the number of families (fills at most max entries of out). */
int vrc_get_kernel_stats(vrc_context* ctx, int max, vrc_kernel_stat* out);

/* ---- batched kernels (host buffers) --------------------------------------- */
/* C[b] = A[b] * B[b]  (batch n*n complex GEMMs on FP64 tensor cores). */
int vrc_zgemm(vrc_context* ctx, int batch, int n, const vrc_complex* A, const vrc_complex* B, vrc_complex* C);
/* In-place inverse of batch n*n matrices; status[b] = VRC_ESINGULAR on a zero pivot. */
int vrc_zinv(vrc_context* ctx, int batch, int n, vrc_complex* A, int* status);

/* ---- eigen-decomposition without device allocation ------------------------
 * No counterpart in the reference.  For callers that cannot let a library
 * call cudaMalloc (applications that own all device memory through their
 * own pool, pipelines where an allocation's implicit device synchronisation
 * is not acceptable).  Same kernels as vrc_eig for ONE n x n matrix:
 * A (input, not modified), W (eigenvectors, unit 2-norm, largest component
 * real) and lam (eigenvalues) are DEVICE pointers, column-major complex128,
 * on the calling thread's current device; work is queued on `stream`
 * (a cudaStream_t, NULL = legacy default stream) and the call blocks the
 * calling host thread until that stream has drained (it reads the
 * convergence flag back); other streams and devices are not waited for.  Scratch is a fixed area inside the library
 * (about 22 MiB per device, held until exit), so n must be in
 * [2, VRC_EIG_NOALLOC_MAX_N]; larger n returns VRC_EINVAL.  All calls share
 * that area: calls that overlap on the GPU race and must be serialised by
 * the caller.  The first call on a device looks the area up; make it before
 * any stream capture.  Returns VRC_ENOCONV if the QR iteration hit its cap. */
#define VRC_EIG_NOALLOC_MAX_N 256
int vrc_eig_noalloc(int n, const vrc_complex* A, vrc_complex* W, vrc_complex* lam, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VRC_H_ */
