// Host engine: memory pools, descriptor staging and the batched stages of
// the varRCWA hot path, driven from C++ (no host-side math on the path).
#pragma once

#include <array>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace vrc {

enum GeomKind { GEOM_GRID = 0, GEOM_PILLAR = 1, GEOM_PIXELS = 2, GEOM_PLANAR = 3, GEOM_SAMPLER = 4 };

// Coordinate rule x_index(z) through knots (zs, vals), constant beyond the
// end knots: piecewise-linear (interp 0) or the natural cubic spline
// (interp 1).  Both are linear in vals; weights(z) gives d x(z) / d vals[k].
struct PwlRule {
  int index;
  std::vector<double> zs, vals;
  int interp = 0;
  std::vector<double> D;  // spline: second derivatives = D vals (K x K, row-major)
  void prepare();         // forms D for a spline rule
  double eval(double z) const;
  void weights(double z, std::vector<double>& w) const;
};

// Geometry + optics of one structure (one "cell" of a batch).
struct CellSpec {
  int kind = GEOM_GRID;
  int nx = 1, ny = 1;
  bool pml = false;
  double lambda = 1.0;
  double z0 = 0.0, z1 = 1.0;
  // grid / pixels
  std::vector<double> x, y;
  std::vector<cplx> eps;  // (ncy-1) x (ncx-1), row-major (rows = y strips)
  std::vector<PwlRule> xrules, yrules;
  std::function<void(double, double*, double*)> geom_cb;  // optional host rule callback
  // pillar
  double Lx = 1.0, Ly = 1.0;
  int npx = 0, npy = 0;
  cplx eps_in{1.0, 0.0}, eps_out{1.0, 0.0};
  double r0 = 0.0, r1 = 0.0;
  // homogeneous end media (otherwise the structure's own bases at z0/z1)
  bool has_end0 = false, has_end1 = false;
  cplx eps_end0{1.0, 0.0}, eps_end1{1.0, 0.0};
  // planar device seen from above (a GDS layout: x across, z along the
  // propagation), a device layer of fixed thickness along y, PML all round
  std::vector<std::vector<double>> polys;  // per polygon x0, z0, x1, z1, ...
  double shift[3] = {0.0, 0.0, 0.0};       // x, y, z
  double pml_w[4] = {0.5, 0.5, 0.5, 0.5};  // left, right, bottom, top
  double space[4] = {1.5, 1.5, 1.08, 1.0};
  double thickness = 0.22;
  cplx eps_bg{1.0, 0.0}, eps_dev{1.0, 0.0};
  // x limits (l0, l1, r0, r1) and the six y coordinates of the planar cell
  void planar_region(double* xlim, double* y6) const;
  // cross-section at z: x (crossings between the PML / spacer coordinates),
  // y, and optionally the (5 x (nx-1)) eps table, rows = y strips
  void planar_section(double z, std::vector<double>& x, std::vector<double>& y, std::vector<cplx>* eps) const;

  // caller's sampler (the role of LayerSampler::sample / sampleOnGPU): P, Q
  // at z as n x n column-major matrices, into host memory (host_sample) or
  // into device buffers on the given stream (dev_sample); nonzero = failure
  std::function<int(double, cplx*, cplx*)> host_sample;
  std::function<int(double, cplx*, cplx*, cudaStream_t)> dev_sample;

  int ncx() const { return kind == GEOM_PILLAR ? npx + 1 : (int)x.size(); }
  int ncy() const { return kind == GEOM_PILLAR ? npy + 1 : (int)y.size(); }
  int m() const { return nx * ny; }
  int n() const { return 2 * nx * ny; }
  double k0() const { return 2.0 * 3.1415926535897932 / lambda; }
  void geometry(double z, std::vector<double>& xo, std::vector<double>& yo) const;
  double radius(double z) const;
};

// BOUNDARY and BOX polygons of a GDSII file's first structure, coordinates
// in `unit` metres (x0, y0, x1, y1, ...); db_unit_m receives the file's
// metres per database unit.
std::vector<std::vector<double>> gds_read_polygons(const std::string& path, double unit, double* db_unit_m);

struct NodeRecord {
  double a, b, err;
  int accepted;
};

struct CellResult {
  int status = ST_OK;
  int n = 0;
  int N = 0;          // accepted segments / slices
  int n_eig = 0;      // eigen-decompositions performed
  int n_samples = 0;  // P,Q samples assembled
  int n_nodes = 0;    // segments evaluated (accepted + rejected)
  // device-resident results (owned by the engine until released)
  cplx *Tdd = nullptr, *Tuu = nullptr, *Rud = nullptr, *Rdu = nullptr;
  cplx *W0 = nullptr, *V0 = nullptr, *gam0 = nullptr, *W0inv = nullptr;
  cplx *W1 = nullptr, *V1 = nullptr, *gam1 = nullptr, *W1inv = nullptr;
  std::vector<NodeRecord> nodes;
};

// Fixed-size device block pool.
class BlockPool {
 public:
  explicit BlockPool(size_t bytes) : bytes_(bytes) {}
  ~BlockPool();
  // a block (a new 64 MB chunk when none is free); nullptr when the device
  // has no room for a chunk
  void* get(cudaStream_t st);
  void put(void* p) { free_.push_back(p); }
  // frees the chunks none of whose blocks is handed out (cudaFree, which
  // waits for the device); returns the bytes released
  size_t release_free(cudaStream_t st);
  size_t bytes() const { return bytes_; }
  size_t blocks() const { return blocks_; }       // blocks created
  size_t free_blocks() const { return free_.size(); }

 private:
  size_t bytes_;
  size_t blocks_ = 0;
  std::vector<void*> free_;
  std::vector<std::pair<void*, size_t>> chunks_;  // base, blocks
};

class Engine {
 public:
  explicit Engine(int device);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  int device() const { return device_; }
  cudaStream_t stream() const { return stream_; }
  void set_stream(cudaStream_t s) { stream_ = s; }
  void sync();

  // memory
  void* take(size_t bytes);  // a block of a size class (frees idle chunks when the device is full)
  size_t trim_idle();        // frees every pool chunk with no block handed out
  cplx* mat(int n);
  cplx* vec(int n);
  void free_mat(cplx* p, int n);
  void free_vec(cplx* p, int n);
  void* bytes(size_t b);
  void free_bytes(void* p, size_t b);
  template <class T>
  T* upload(const T* data, size_t count);
  template <class T>
  T* upload(const std::vector<T>& v) {
    return upload(v.data(), v.size());
  }
  void* workspace(size_t bytes);
  // diagnostic: bytes held by the pools and the workspace, and the part of
  // the pools handed out (not returned), summed over the pools
  void pool_report(size_t* held, size_t* out, size_t* npools, size_t* ws) const;
  size_t batch_budget_bytes() const;

  // batched primitives
  // opA / opB = 1: that operand enters as its conjugate transpose.
  void gemm(std::vector<GemmDesc>& d, int n, cplx alpha, cplx beta, double delta, int opA = 0, int opB = 0);
  // GEMM tile for order n and operand modes: timed once per shape on scratch
  // operands (both tiles give identical results) and cached for the whole
  // process; VRC_GEMM_TILE forces one.  0 from gemm_tile_cached when the
  // shape was not tuned yet.
  int gemm_tile(int n, int opA, int opB, size_t batch);
  int gemm_tile_cached(int n, int opA, int opB) const;
  void inverse(const std::vector<cplx*>& mats, int n, std::vector<int>* status);
  void copy(const std::vector<cplx*>& src, const std::vector<cplx*>& dst, int n);
  void axpby(const std::vector<const cplx*>& A, const std::vector<const cplx*>& B, const std::vector<cplx*>& C,
             cplx alpha, cplx beta, double delta, int n);

  // ---- stages ----
  // Per-cell constant data (K matrices).
  struct CellDev {
    int nx, ny, m, n;
    double k0;
    bool pml;
    double* alpha = nullptr;  // device (m)
    double* beta = nullptr;
    std::vector<double> h_alpha, h_beta;
    cplx *Kx = nullptr, *Ky = nullptr, *KxKy = nullptr, *KxKx = nullptr, *KyKy = nullptr, *KyKx = nullptr;
    cplx* eps_dev = nullptr;  // fixed permittivity table (grid / pixels)
    size_t eps_count = 0;
    // grid cells whose moving coordinates follow tabulated rules: the rule
    // tables on the device (geometry per sample by grid_geometry)
    bool dev_geom = false;
    int nrules = 0;
    double* geo_d = nullptr;
    int* geo_i = nullptr;
    size_t geo_nd = 0, geo_ni = 0;
  };
  CellDev* prepare_cell(const CellSpec& c);
  void release_cell(CellDev* cd);

  struct SampleReq {
    const CellSpec* spec;
    CellDev* cd;
    double z;
    bool homogeneous;  // sample a homogeneous medium eps_h instead of the structure
    cplx eps_h;
    cplx* P;
    cplx* Q;
    cplx* keep_fe33inv = nullptr;  // optional copy of fe33^-1 (m x m; periodic cells)
  };
  void assemble(std::vector<SampleReq>& reqs, std::vector<int>* status);
  // samples of caller-sampler cells (GEOM_SAMPLER): the callbacks fill P, Q
  void sample_external(const std::vector<SampleReq*>& reqs);
  // Fourier-Toeplitz assembly of the geometry kinds the engine samples itself
  void assemble_grid(std::vector<SampleReq>& reqs, std::vector<int>* status);

  struct EigReq {
    const cplx* P;
    const cplx* Q;
    cplx *W, *V, *Winv, *Vinv, *gam;
    cplx* lam = nullptr;  // optional copy of the eigenvalues of P*Q
  };
  void eig(std::vector<EigReq>& reqs, int n, std::vector<int>* status);

  struct SegReq {
    const cplx *Pr, *Qr, *W, *V, *Winv, *Vinv, *gam;
    const cplx *Pa, *Qa, *Pb, *Qb;
    double z0, z1, k0;
    cplx *tdd, *tuu, *rud, *rdu;
    double* err;  // device
  };
  void segments(std::vector<SegReq>& reqs, int n);

  // Left-end re-expression of segment blocks from the basis (Winv,Vinv) of
  // the segment into (leftW, leftV).  Blocks updated in place.
  struct ProjReq {
    const cplx *Winv, *Vinv, *leftW, *leftV;
    cplx *tdd, *tuu, *rud, *rdu;
  };
  void project_left(std::vector<ProjReq>& reqs, int n, std::vector<int>* status);
  // Right-end re-expression: S's right end from basis (leftWinv,leftVinv) to (W1,V1).
  struct ProjRReq {
    const cplx *leftWinv, *leftVinv, *W1, *V1;
    cplx *Tdd, *Tuu, *Rud, *Rdu;
  };
  void project_right(std::vector<ProjRReq>& reqs, int n, std::vector<int>* status);
  // RCWA-style left-end projection: chain expressed in (W1,V1) on both ends,
  // left end moved to (W0,V0); W1inv, V1inv given.
  struct ProjLEReq {
    const cplx *W1inv, *V1inv, *W0, *V0;
    cplx *Tdd, *Tuu, *Rud, *Rdu;
  };
  void project_left_end(std::vector<ProjLEReq>& reqs, int n, std::vector<int>* status);

  // Star product: out = L * R (L on the z0 side).  Out buffers must not
  // alias the inputs.
  struct StarReq {
    const cplx *Tdd, *Tuu, *Rud, *Rdu;  // left (accumulated)
    const cplx *tdd, *tuu, *rud, *rdu;  // right (new)
    cplx *oTdd, *oTuu, *oRud, *oRdu;
  };
  void star(std::vector<StarReq>& reqs, int n, std::vector<int>* status);

  // Reduce per-cell ordered lists of S-matrices (4 blocks each) to one per
  // cell by pairwise star products.  Inputs are consumed (freed) except the
  // final survivor, returned in place of lists[c][0].
  struct SBlocks {
    cplx *tdd, *tuu, *rud, *rdu;
  };
  void star_reduce(std::vector<std::vector<SBlocks>>& lists, int n, std::vector<int>* cell_status);

  // RCWA slab S-matrix (tuu, rud) in the basis (W1, V1) for samples P,Q.
  struct SlabReq {
    const cplx *P, *Q, *W1, *V1;
    double k0, dz;
    cplx *tuu, *rud;
  };
  void rcwa_slabs(std::vector<SlabReq>& reqs, int n, std::vector<int>* status);

  // Differential-method slice from samples at (zl, zm, zr).
  struct DiffReq {
    const cplx *P0, *Q0, *P1, *Q1, *P2, *Q2;
    const cplx *W1, *V1, *W1inv, *V1inv;
    double k0, dz;
    cplx *tdd, *tuu, *rud, *rdu;
  };
  void diff_slices(std::vector<DiffReq>& reqs, int n, std::vector<int>* status);

  // ---- drivers ----
  struct RedhefferOpts {
    double pe = 1e-2;
    int max_depth = 40;
    const std::vector<std::vector<double>>* cuts = nullptr;  // explicit segments (replay)
    // cells of several truncations are solved one size class after another;
    // the class order starts at class `rotate` (mod the class count), so that
    // concurrent engines given the same mix work on different sizes at once
    int rotate = 0;
  };
  void redheffer(const std::vector<CellSpec>& cells, const RedhefferOpts& o, std::vector<CellResult>& out);
  // Gradient with respect to the rule knots of grid cells of one truncation,
  // on the accepted segmentation `cuts` of each: gS (4 n^2 per cell: the
  // cotangents of Tdd, Tuu, Rud, Rdu) and gB (4 n^2 or null: of W0, V0, W1,
  // V1), host column-major; ends (per cell W0, V0, gam0, W1, V1, gam1, host)
  // are the forward's end bases, which the cotangents refer to.  grad[c]:
  // dL/d vals of every x rule, then every y rule.  The chain is recomputed
  // with a checkpoint every `every` segments (0: about the square root of
  // the segment count).
  void cell_backward(const std::vector<CellSpec>& cells, const std::vector<std::vector<double>>& cuts,
                     const std::vector<const cplx*>& gS, const std::vector<const cplx*>& gB,
                     const std::vector<const cplx*>& ends, int every, std::vector<std::vector<double>>& grad);
  void rcwa(const std::vector<CellSpec>& cells, int N, std::vector<CellResult>& out);
  void differential(const std::vector<CellSpec>& cells, int N, std::vector<CellResult>& out);
  void release_result(CellResult& r);

  // Per-order powers for the two polarisations (px,py) = (1,0), (0,1).
  // side 0: incidence from z0 (Rdu, Tuu), 1: from z1 (Rud, Tdd).
  void order_powers(const std::vector<CellSpec>& cells, const std::vector<CellResult>& res, int side,
                    int flux_norm, std::vector<std::vector<double>>& R, std::vector<std::vector<double>>& T);

  // ---- layer stacks of z-uniform pixel rasters: forward and adjoint ----
  // Layer l (0 nearest z0) holds an npy x npx raster of real permittivity on a
  // uniform (Lx, Ly) grid and has thickness thick[l]; eps_in below z0 (the
  // incidence side), eps_out above.  Periodic boundaries.
  struct StackSpec {
    int nx = 1, ny = 1, npx = 1, npy = 1, L = 0;
    double lambda = 1.0, Lx = 1.0, Ly = 1.0;
    std::vector<double> eps;    // L * npy * npx, row-major per layer (rows = y)
    std::vector<double> thick;  // L
    cplx eps_in{1.0, 0.0}, eps_out{1.0, 0.0};
  };
  // Per-order (REF, TRN) of every stack (m each) for incidence (px, py) from
  // eps_in; keeps what stack_backward needs until the next stack_forward.
  void stack_forward(const std::vector<StackSpec>& stacks, double px, double py, double* REF, double* TRN,
                     int* status);
  // Gradient of L = sum_k wR[k] REF[k] + wT[k] TRN[k] (m weights each per
  // stack) with respect to every pixel of every layer (L * npy * npx per stack).
  // grad_thick (L per stack, may be null): dL/d(layer thickness).
  void stack_backward(const double* wR, const double* wT, double* grad, double* grad_thick = nullptr);
  void release_stack_tape();
  // Up- and down-going amplitudes at every interface j = 0..L of the stacks of
  // the last stack_forward (amps: per stack (L+1) x 2 x n, a+ then a-, in the
  // basis of the region below the interface) and Ex, Ey on an ngx x ngy grid
  // over the period (img: per stack (L+1) x 2 x ngy x ngx; may be null).
  void stack_fields(int ngx, int ngy, cplx* amps, cplx* img);

  // counters
  long long launches = 0;

  // Per-kernel-family timing with CUDA events on the engine stream
  // (enabled on demand; resolved at every sync()).
  struct FamStat {
    double ms = 0.0;
    long long launches = 0;
    double flops = 0.0;  // algorithmic real FP64 flops
    double bytes = 0.0;  // algorithmic bytes moved
    std::vector<std::pair<double, double>> iv;  // launch intervals (ms after the time origin)
  };
  void set_profiling(bool on);
  // Event that launch intervals are measured from (one event shared by the
  // engines of a context, so their intervals share one time line).
  void set_time_origin(cudaEvent_t e) { origin_ = e; }
  bool profiling() const { return profiling_; }
  std::map<std::string, FamStat>& fam_stats();
  void reset_fam_stats();
  struct Prof {
    Engine& e;
    const char* fam;
    double flops, bytes;
    int nl;
    cudaEvent_t a = nullptr;
    Prof(Engine& eng, const char* f, double fl = 0.0, double by = 0.0, int nlaunch = 1);
    ~Prof();
  };

 private:
  int device_;
  cudaStream_t stream_;
  bool own_stream_;
  std::map<size_t, std::unique_ptr<BlockPool>> pools_;
  char* h_stage_ = nullptr;
  char* d_stage_ = nullptr;
  size_t stage_cap_ = 0, stage_off_ = 0;
  int stage_half_ = 0;  // the half of the staging ring in use
  void* ws_ = nullptr;
  size_t ws_cap_ = 0;
  // pinned staging of host-sampler matrices and the event of its last copy
  char* ext_host_ = nullptr;
  size_t ext_cap_ = 0;
  cudaEvent_t ext_ev_ = nullptr;
  bool profiling_ = false;
  cudaEvent_t origin_ = nullptr;
  // host-bubble diagnostic (VRC_HOST_STATS): time from a sync's return to
  // the next profiled launch, when the GPU has nothing queued
 public:
  double bubble_ms_ = 0.0, sync_ms_ = 0.0;
  std::map<std::string, double> gap_;  // GPU gaps between consecutive profiled families
  cudaEvent_t last_b_ = nullptr;
  std::string last_fam_;
  long long nsync_ = 0;
  double t_sync_ret_ = -1.0;
 private:
  double alloc_ms0_ = 0.0;
  long long alloc_calls0_ = 0;
  struct PendingProf {
    const char* fam;
    cudaEvent_t a, b;
    double flops, bytes;
    int nl;
  };
  std::vector<PendingProf> pend_prof_;
  std::vector<cudaEvent_t> ev_pool_;
  std::map<std::string, FamStat> fam_;
  cudaEvent_t take_event();
  void resolve_prof();
  BlockPool& pool(size_t bytes);
  void* stage(const void* data, size_t bytes);
  struct EndBasis {
    cplx *W, *V, *Winv, *Vinv, *gam;
  };
 public:
  // Device state of the last stack_forward (one block per stack).
  struct StackLayer {
    cplx *P, *Q, *W, *V, *Winv, *Vinv, *gam, *A, *B, *Ainv, *x, *fe33inv, *eps;
    cplx* seg[4];  // projected layer blocks (tdd, tuu, rud, rdu)
    cplx* pre[4];  // chain before this layer's star product
  };
  struct StackCell {
    char* mem = nullptr;
    size_t bytes = 0;
    EndBasis e0, e1;
    std::vector<StackLayer> lay;
    cplx *Sc[4], *S[4], *Ar, *Br, *Mrinv;
    double *alpha, *beta;
  };
  struct StackTape {
    int C = 0, L = 0, n = 0, m = 0, nx = 0, ny = 0, npx = 0, npy = 0;
    double px = 1.0, py = 0.0;
    std::vector<StackSpec> specs;
    std::vector<StackCell> cells;
    std::vector<int> status;
  };
  const StackTape& stack_tape() const { return tape_; }

  // ---- stacks of sections (each a cell on its own z-range) ----
  struct ChainTape {
    int n = 0, m = 0;
    std::vector<CellResult> secs;               // every section's result
    std::vector<std::array<cplx*, 4>> proj;    // blocks, entrance in the previous exit basis
    std::vector<std::array<cplx*, 4>> prefix;  // chain of sections 0..s
    std::vector<cplx*> V0inv;                  // sections 1..
    double *alpha = nullptr, *beta = nullptr;  // harmonics (field images)
    double Lx = 1.0, Ly = 1.0;
    CellSpec spec;      // outer media of the stack (order powers)
    CellResult result;  // points into secs / prefix
  };
  // Solves the sections (method 0 adaptive varRCWA, 1 RCWA, 2 differential)
  // and joins them; out points into the kept stack (valid until the next
  // chain); trees: every section's segmentation.
  void chain(const std::vector<CellSpec>& sections, int method, double pe, int max_depth, int nslices,
             CellResult& out, std::vector<std::vector<NodeRecord>>& trees);
  void chain_order_powers(int side, int flux_norm, std::vector<double>& R, std::vector<double>& T);
  // amplitudes (a+, a-) at every interface for incident entrance amplitudes
  // c (host, n); amps: (S+1) x 2 x n, img: (S+1) x 2 x ngy x ngx or null
  void chain_fields(const cplx* c, int ngx, int ngy, cplx* amps, cplx* img);
  void release_chain();

 private:
  StackTape tape_;
  ChainTape chain_;
};

template <class T>
T* Engine::upload(const T* data, size_t count) {
  return reinterpret_cast<T*>(stage(data, count * sizeof(T)));
}

}  // namespace vrc
