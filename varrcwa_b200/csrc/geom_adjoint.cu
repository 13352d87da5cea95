// Gradients of adaptive varRCWA cells with respect to geometric parameters:
// the knot values of the coordinate rules of tensor-grid cells (the moving
// coordinates of VarLayerSampler::addXRule / addYRule,
// src/core/VarLayerSampler.cpp:42-59), on the segmentation the forward
// accepted.  The reference has no integrator gradients; its building block
// is the forward-mode dP/dx of Layer::waveEqnCoeff (src/rcwa/Layer.cpp:104-162).
//
// Frozen bases: every intermediate basis only re-expresses the same operator,
// so a parameter reaches the S-matrix through the samples P(z), Q(z) inside
// each segment (first order: the segment formula of
// src/core/RedhefferIntegrator.cpp:343-396 applied to dP, dQ at its three
// Simpson nodes) and through the two end bases the result is expressed in.
//
// Reverse pass, batched over the cells of a call:
//   1. the chain is recomputed left to right (star products as
//      RedhefferIntegrator.cpp:267-277, projections as :253-262), keeping the
//      chain state before every `every`-th segment (checkpoints);
//   2. the right-end projection (:211-223) is reversed with respect to the
//      chain and to the exit basis; the exit eigen step is reversed;
//   3. checkpoint blocks are recomputed from the last to the first, each kept
//      whole (prefix chain, own-basis and projected blocks, projection
//      matrices, bases) and reversed segment by segment: star product,
//      projection, then the segment formula with respect to its node samples
//      (node_adjoint_kernel and four GEMMs per node);
//   4. the entrance projection and eigen step are reversed;
//   5. at every node z, dL/dP, dL/dQ are contracted with dP/dx, dQ/dx of each
//      moving coordinate (central differences of the device assembly, +-h on
//      that coordinate alone) into dL/dx(z), which the host spreads over the
//      rule's knots (d x(z) / d value of knot k: hat or spline functions).
//
// The eigen step's adjoint (A = P Q = W diag(lam) W^-1, V = Q W diag(1/gam))
// keeps C_ij = (W^-1 dA W)_ij / (lam_j - lam_i) off the diagonal, broadened
// as conj(d) / (|d|^2 + eta^2) with eta = 1e-12 max|lam|; the column
// normalisation is left out, which is exact for objectives that do not depend
// on how the end modes are scaled (Fourier-basis blocks, flux-normalised
// modal powers).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>

#include "batch.h"
#include "engine.h"

namespace vrc {

namespace {

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
struct NodeAdjDesc {
  const cplx *gtdd, *gtuu, *grud, *grdu;  // own-basis block adjoints
  const cplx* gam;
  cplx* gx[3];  // per node (a, midpoint, b): cotangent of W^-1 dP V
  cplx* gy[3];  // and of V^-1 dQ W
  double dz, k0;
};

// Transpose of the segment formula: with pf = exp(i dz gam / k0),
// ph = exp(i dz gam / (2 k0)), c = i dz / (12 k0), the blocks are
//   tuu = c (pf_i dA0 + 4 ph_i dA1 ph_j + dA2 pf_j)
//   tdd = c (dA0 pf_j + 4 ph_i dA1 ph_j + pf_i dA2)
//   rud = -c (pf_i dB0 pf_j + 4 ph_i dB1 ph_j + dB2)
//   rdu = -c (dB0 + 4 ph_i dB1 ph_j + pf_i dB2 pf_j)
// with dA = x + y, dB = x - y per node; the cotangents of x, y follow.
__global__ void node_adjoint_kernel(const NodeAdjDesc* __restrict__ ds, int n) {
  const NodeAdjDesc d = ds[blockIdx.y];
  const size_t nn = (size_t)n * n;
  const double t = d.dz / d.k0;
  const cplx cc = mk(0.0, -d.dz / (12.0 * d.k0));  // conj(c)
  const cplx cc4 = cscale(cc, 4.0);
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < nn; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);  // column-major: row i, column j
    const cplx gi = d.gam[i], gj = d.gam[j];
    const cplx Fi = cconj(cexp_i(gi, t)), Fj = cconj(cexp_i(gj, t));
    const cplx P2 = cconj(cmul(cexp_i(gi, 0.5 * t), cexp_i(gj, 0.5 * t)));
    const cplx tdd = d.gtdd[idx], tuu = d.gtuu[idx], rud = d.grud[idx], rdu = d.grdu[idx];
    const cplx A0 = cmul(cc, cadd(cmul(Fi, tuu), cmul(tdd, Fj)));
    const cplx A1 = cmul(cc4, cmul(P2, cadd(tuu, tdd)));
    const cplx A2 = cmul(cc, cadd(cmul(tuu, Fj), cmul(Fi, tdd)));
    const cplx B0 = cneg(cmul(cc, cadd(cmul(cmul(Fi, rud), Fj), rdu)));
    const cplx B1 = cneg(cmul(cc4, cmul(P2, cadd(rud, rdu))));
    const cplx B2 = cneg(cmul(cc, cadd(rud, cmul(cmul(Fi, rdu), Fj))));
    d.gx[0][idx] = cadd(A0, B0);
    d.gy[0][idx] = csub(A0, B0);
    d.gx[1][idx] = cadd(A1, B1);
    d.gy[1][idx] = csub(A1, B1);
    d.gx[2][idx] = cadd(A2, B2);
    d.gy[2][idx] = csub(A2, B2);
  }
}

struct GamAdjDesc {
  const cplx *V, *gV, *gam;
  cplx* glam;   // out: cotangent of lam = gam^2 from V = Q W diag(1/gam)
  cplx* igc;    // out: conj(1 / gam)
  double* eta;  // out: 1e-12 max |lam|
};

// One block per matrix: ggam_j = -sum_r conj(V_rj) gV_rj conj(1/gam_j),
// glam_j = ggam_j conj(1 / (2 gam_j)) (gam = sqrt(lam), d gam = d lam / (2 gam)).
__global__ void __launch_bounds__(256) gamma_adjoint_kernel(const GamAdjDesc* __restrict__ ds, int n) {
  const GamAdjDesc d = ds[blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ double s_max[8];
  double mx = 0.0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const cplx g = d.gam[j];
    mx = fmax(mx, cabs2(g));  // |lam| = |gam|^2
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) s_max[warp] = mx;
  for (int j = warp; j < n; j += blockDim.x / 32) {
    const cplx* v = d.V + (size_t)j * n;
    const cplx* g = d.gV + (size_t)j * n;
    cplx s = mk(0.0, 0.0);
    for (int r = lane; r < n; r += 32) s = cadd(s, cmulc(v[r], g[r]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
      s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
    }
    if (lane == 0) {
      const cplx ig = cconj(cinv(d.gam[j]));
      const cplx ggam = cneg(cmul(s, ig));
      d.glam[j] = cmul(ggam, cscale(ig, 0.5));
      d.igc[j] = ig;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) m = fmax(m, s_max[w]);
    *d.eta = 1e-12 * m;
  }
}

struct EigFDesc {
  cplx* M;  // in: W^H gW; out: F
  const cplx *gam, *glam;
  const double* eta;
};

// F_ij = M_ij (lam_j - lam_i) / (|lam_j - lam_i|^2 + eta^2) off the diagonal,
// F_ii = glam_i.
__global__ void eig_f_kernel(const EigFDesc* __restrict__ ds, int n) {
  const EigFDesc d = ds[blockIdx.y];
  const size_t nn = (size_t)n * n;
  const double eta = *d.eta;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < nn; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    if (i == j) {
      d.M[idx] = d.glam[i];
      continue;
    }
    const cplx gi = d.gam[i], gj = d.gam[j];
    const cplx dl = csub(cmul(gj, gj), cmul(gi, gi));
    const double den = cabs2(dl) + eta * eta;
    d.M[idx] = den > 0.0 ? cscale(cmul(d.M[idx], dl), 1.0 / den) : mk(0.0, 0.0);
  }
}

struct DotDiffDesc {
  const cplx *g, *A, *B;
  double* out;
  double scale;
};

// out += scale Re sum conj(g) (A - B), one block column per descriptor.
__global__ void __launch_bounds__(256) dotdiff_kernel(const DotDiffDesc* __restrict__ ds, long long count) {
  const DotDiffDesc d = ds[blockIdx.y];
  double s = 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < count; k += (long long)gridDim.x * blockDim.x) {
    const cplx g = d.g[k], a = d.A[k], b = d.B[k];
    s += g.x * (a.x - b.x) + g.y * (a.y - b.y);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) t += red[w];
    atomicAdd(d.out, d.scale * t);
  }
}

int grid_for(size_t work, int threads) {
  return (int)std::min<size_t>((work + threads - 1) / threads, 148 * 8);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct Bas {
  cplx *W = nullptr, *V = nullptr, *Wi = nullptr, *Vi = nullptr, *gam = nullptr;
};

struct Ckpt {  // chain state before segment j0
  cplx* S[4];
  cplx *lW, *lV;  // left basis (previous segment's, or the entrance basis)
  cplx *Pa, *Qa;  // sample at the segment's left end
};

struct Node {  // one contraction: dL/dP, dL/dQ at z of a cell
  int cell;
  double z;
  cplx *gP, *gQ;
};

}  // namespace

void Engine::cell_backward(const std::vector<CellSpec>& cells, const std::vector<std::vector<double>>& cuts,
                           const std::vector<const cplx*>& gS_host, const std::vector<const cplx*>& gB_host,
                           const std::vector<const cplx*>& ends, int every, std::vector<std::vector<double>>& grad) {
  const int C = (int)cells.size();
  grad.assign(C, {});
  if (C == 0) return;
  const int n = cells[0].n();
  const size_t nn = (size_t)n * n;
  for (const auto& c : cells) {
    if (c.n() != n) throw StatusError(ST_EINVAL, "cell backward: one truncation per batch");
    if (c.kind != GEOM_GRID) throw StatusError(ST_EINVAL, "cell backward: parameters are the rule knots of grid cells");
  }
  std::vector<int> K(C);
  int Kmax = 0;
  for (int c = 0; c < C; ++c) {
    K[c] = (int)cuts[c].size() - 1;
    if (K[c] < 1) throw StatusError(ST_EINVAL, "cell backward: no segments");
    Kmax = std::max(Kmax, K[c]);
    size_t nk = 0;
    for (const auto& r : cells[c].xrules) nk += r.zs.size();
    for (const auto& r : cells[c].yrules) nk += r.zs.size();
    grad[c].assign(nk, 0.0);
  }
  if (every <= 0) every = std::max(1, (int)std::ceil(std::sqrt((double)Kmax)));
  std::vector<CellDev*> cds(C);
  for (int c = 0; c < C; ++c) cds[c] = prepare_cell(cells[c]);

  // perturbed copies of every cell for each moving coordinate (+h, -h)
  struct Coord {
    int axis, index, rule;  // rule: position in grad's knot list
    double h;
    CellSpec plus, minus;
  };
  std::vector<std::vector<Coord>> coords(C);
  for (int c = 0; c < C; ++c) {
    const CellSpec& s = cells[c];
    size_t off = 0;
    for (int axis = 0; axis < 2; ++axis) {
      const auto& rules = axis == 0 ? s.xrules : s.yrules;
      const auto& base = axis == 0 ? s.x : s.y;
      const double L = base.back() - base.front();
      for (const auto& r : rules) {
        Coord co{axis, r.index, (int)off, 1e-6 * std::fabs(L), s, s};
        for (int sg = 0; sg < 2; ++sg) {
          CellSpec& t = sg == 0 ? co.plus : co.minus;
          const double dlt = sg == 0 ? co.h : -co.h;
          auto prev = s.geom_cb;
          const int ax = axis, ix = r.index;
          t.geom_cb = [prev, ax, ix, dlt](double z, double* x, double* y) {
            if (prev) prev(z, x, y);
            (ax == 0 ? x : y)[ix] += dlt;
          };
        }
        coords[c].push_back(std::move(co));
        off += r.zs.size();
      }
    }
  }

  Batch all{*this, C};
  // Long-lived matrices (samples, bases, blocks, chain states) are reference
  // counted: every holder (a chain state, a checkpoint, a recomputed block,
  // the ends) takes one reference and drops it when done.
  std::map<cplx*, int> refs;
  auto own = [&]() {
    cplx* p = mat(n);
    refs[p] = 1;
    return p;
  };
  auto hold = [&](cplx* p) { ++refs.at(p); };
  auto drop = [&](cplx* p) {
    auto it = refs.find(p);
    if (it == refs.end()) throw StatusError(ST_EINVAL, "cell backward: released an unowned matrix");
    if (--it->second == 0) {
      free_mat(p, n);
      refs.erase(it);
    }
  };
  auto sample_into = [&](const std::vector<std::pair<int, double>>& req, const std::vector<const CellSpec*>* specs,
                         Vec& P, Vec& Q) {
    std::vector<SampleReq> sr;
    P.assign(req.size(), nullptr);
    Q.assign(req.size(), nullptr);
    for (size_t k = 0; k < req.size(); ++k) {
      P[k] = own();
      Q[k] = own();
      const CellSpec* sp = specs ? (*specs)[k] : &cells[req[k].first];
      sr.push_back({sp, cds[req[k].first], req[k].second, false, mk(1, 0), P[k], Q[k]});
    }
    std::vector<int> st;
    assemble(sr, &st);
    for (int v : st)
      if (v) throw StatusError(v, "cell backward: assembly failed");
  };
  auto decompose = [&](const Vec& P, const Vec& Q, std::vector<Bas>& out) {
    std::vector<EigReq> er;
    out.assign(P.size(), Bas());
    for (size_t k = 0; k < P.size(); ++k) {
      out[k] = {own(), own(), own(), own(), vec(n)};
      er.push_back({P[k], Q[k], out[k].W, out[k].V, out[k].Wi, out[k].Vi, out[k].gam});
    }
    std::vector<int> st;
    eig(er, n, &st);
    for (int v : st)
      if (v) throw StatusError(v, "cell backward: eigensolver failure");
  };
  auto drop_bas = [&](Bas& b) {
    for (cplx* p : {b.W, b.V, b.Wi, b.Vi})
      if (p) drop(p);
    if (b.gam) free_vec(b.gam, n);
    b = Bas();
  };
  auto sub = [](const Vec& v, const std::vector<int>& idx) {
    Vec o;
    for (int i : idx) o.push_back(v[i]);
    return o;
  };

  // ---- ends: structure samples at z0, z1 and the end bases ----
  Vec P0, Q0, P1, Q1;
  {
    std::vector<std::pair<int, double>> r0, r1;
    for (int c = 0; c < C; ++c) {
      r0.push_back({c, cuts[c].front()});
      r1.push_back({c, cuts[c].back()});
    }
    sample_into(r0, nullptr, P0, Q0);
    sample_into(r1, nullptr, P1, Q1);
  }
  // the forward's end bases (the cotangents refer to their modes); W^-1 here
  std::vector<Bas> e0(C), e1(C);
  std::vector<bool> own0(C), own1(C);
  {
    Vec Wi;
    for (int c = 0; c < C; ++c) {
      own0[c] = !cells[c].has_end0;  // else a half-space's basis: no parameter dependence
      own1[c] = !cells[c].has_end1;
      for (int end = 0; end < 2; ++end) {
        Bas& b = end == 0 ? e0[c] : e1[c];
        const cplx* src = ends[c] + end * (2 * nn + n);
        b = {own(), own(), own(), nullptr, vec(n)};
        VRC_CUDA_CHECK(cudaMemcpyAsync(b.W, src, nn * 16, cudaMemcpyHostToDevice, stream_));
        VRC_CUDA_CHECK(cudaMemcpyAsync(b.V, src + nn, nn * 16, cudaMemcpyHostToDevice, stream_));
        VRC_CUDA_CHECK(cudaMemcpyAsync(b.gam, src + 2 * nn, (size_t)n * 16, cudaMemcpyHostToDevice, stream_));
        Wi.push_back(b.Wi);
      }
    }
    Vec W;
    for (int c = 0; c < C; ++c) {
      W.push_back(e0[c].W);
      W.push_back(e1[c].W);
    }
    copy(W, Wi, n);
    std::vector<int> ist;
    inverse(Wi, n, &ist);
    for (int v : ist)
      if (v) throw StatusError(v, "cell backward: singular end basis");
  }

  // ---- blocks of segments ----
  struct St {
    cplx* S[4];
    cplx *lW, *lV, *Pa, *Qa;
  };
  std::vector<St> st(C);
  std::vector<Bas> last(C);  // inverses of each cell's last basis (exit projection)
  struct It {                // one segment of one cell inside a block
    int j, c;
    cplx *Pb, *Qb;  // sample at its right end
    Bas b;          // midpoint basis
    cplx *seg[4], *segp[4], *A, *B, *Minv, *pre[4];
  };
  // Segments [j0, j1) of the cells still running there, from their states.
  // Node samples, midpoint bases, own-basis blocks and left projections do
  // not depend on the chain, so they run batched over the whole block; then
  // the star products in order, batched over the cells.  With keep, the
  // items keep everything (the prefix chain included) for the reverse pass;
  // without, they are dropped.  States advance to the block's end.
  auto run_block = [&](int j0, int j1, bool keep, std::vector<It>& items) {
    items.clear();
    for (int j = j0; j < j1; ++j)
      for (int c = 0; c < C; ++c)
        if (j < K[c]) items.push_back(It{j, c});
    const int NB = (int)items.size();
    std::map<std::pair<int, int>, int> at;  // (cell, j) -> item
    for (int i = 0; i < NB; ++i) at[{items[i].c, items[i].j}] = i;
    std::vector<std::pair<int, double>> rm, rb;
    std::vector<int> need_b;
    for (int i = 0; i < NB; ++i) {
      const It& it = items[i];
      const double za = cuts[it.c][it.j], zb = cuts[it.c][it.j + 1];
      rm.push_back({it.c, 0.5 * (za + zb)});
      if (it.j + 1 < K[it.c]) {
        rb.push_back({it.c, zb});
        need_b.push_back(i);
      }
    }
    Vec Pm, Qm, Pbn, Qbn;
    sample_into(rm, nullptr, Pm, Qm);
    sample_into(rb, nullptr, Pbn, Qbn);
    for (int i = 0; i < NB; ++i) {  // the exit sample: one more holder
      items[i].Pb = P1[items[i].c];
      items[i].Qb = Q1[items[i].c];
    }
    for (size_t k = 0; k < need_b.size(); ++k) {
      items[need_b[k]].Pb = Pbn[k];
      items[need_b[k]].Qb = Qbn[k];
    }
    for (auto& it : items)
      if (it.Pb == P1[it.c]) {
        hold(it.Pb);
        hold(it.Qb);
      }
    std::vector<Bas> bm;
    decompose(Pm, Qm, bm);
    for (int i = 0; i < NB; ++i) items[i].b = bm[i];
    // left sample and basis of every item: the state's for the block's first
    // segment, the previous item's otherwise
    Vec Pa(NB), Qa(NB), lW(NB), lV(NB);
    for (int i = 0; i < NB; ++i) {
      const It& it = items[i];
      if (it.j == j0) {
        Pa[i] = st[it.c].Pa;
        Qa[i] = st[it.c].Qa;
        lW[i] = st[it.c].lW;
        lV[i] = st[it.c].lV;
      } else {
        const It& pv = items[at.at({it.c, it.j - 1})];
        Pa[i] = pv.Pb;
        Qa[i] = pv.Qb;
        lW[i] = pv.b.W;
        lV[i] = pv.b.V;
      }
    }
    Batch bt{*this, NB};
    Vec seg[4], segp[4];
    for (int k = 0; k < 4; ++k) {
      seg[k].resize(NB);
      segp[k].resize(NB);
      for (int i = 0; i < NB; ++i) {
        items[i].seg[k] = seg[k][i] = own();
        items[i].segp[k] = segp[k][i] = own();
      }
    }
    {
      double* derr = (double*)bytes((size_t)NB * sizeof(double));
      std::vector<SegReq> sr;
      for (int i = 0; i < NB; ++i) {
        const It& it = items[i];
        sr.push_back({Pm[i], Qm[i], it.b.W, it.b.V, it.b.Wi, it.b.Vi, it.b.gam, Pa[i], Qa[i], it.Pb, it.Qb,
                      cuts[it.c][it.j], cuts[it.c][it.j + 1], cells[it.c].k0(), seg[0][i], seg[1][i], seg[2][i],
                      seg[3][i], derr + i});
      }
      segments(sr, n);
      free_bytes(derr, (size_t)NB * sizeof(double));
    }
    for (int i = 0; i < NB; ++i) {
      drop(Pm[i]);
      drop(Qm[i]);
    }
    // left projections with their matrices kept: A, B = (Wm^-1 lW +- Vm^-1 lV) / 2
    Vec A(NB), Bm(NB), Mi(NB), Wi(NB), Vi(NB), T1 = bt.alloc(n), T2 = bt.alloc(n);
    for (int i = 0; i < NB; ++i) {
      items[i].A = A[i] = own();
      items[i].B = Bm[i] = own();
      items[i].Minv = Mi[i] = own();
      Wi[i] = items[i].b.Wi;
      Vi[i] = items[i].b.Vi;
    }
    bt.mm(T1, Wi, lW, C_ONE, 0, 0, nullptr, C_ZERO, n);
    bt.mm(T2, Vi, lV, C_ONE, 0, 0, nullptr, C_ZERO, n);
    {
      std::vector<const cplx*> t1(T1.begin(), T1.end()), t2(T2.begin(), T2.end());
      axpby(t1, t2, A, C_HALF, C_HALF, 0.0, n);
      axpby(t1, t2, Bm, C_HALF, C_MHALF, 0.0, n);
    }
    bt.mm(Mi, seg[3], Bm, C_MONE, 0, 0, &A, C_ONE, n);  // M = A - rdu B
    std::vector<int> ist;
    inverse(Mi, n, &ist);
    for (int v : ist)
      if (v) throw StatusError(v, "cell backward: singular left projection");
    bt.mm(T1, seg[3], A, C_ONE, 0, 0, &Bm, C_MONE, n);  // rdu A - B
    bt.mm(segp[3], Mi, T1, C_ONE, 0, 0, nullptr, C_ZERO, n);
    bt.mm(segp[0], Mi, seg[0], C_ONE, 0, 0, nullptr, C_ZERO, n);
    bt.mm(T2, seg[1], Bm, C_ONE, 0, 0, nullptr, C_ZERO, n);  // tuu B
    bt.mm(segp[2], T2, segp[0], C_ONE, 0, 0, &seg[2], C_ONE, n);
    bt.mm(T1, seg[1], A, C_ONE, 0, 0, nullptr, C_ZERO, n);
    bt.mm(segp[1], T2, segp[3], C_ONE, 0, 0, &T1, C_ONE, n);
    bt.release(T1, n);
    bt.release(T2, n);
    // the chain, segment by segment (batched over the cells)
    for (int j = j0; j < j1; ++j) {
      std::vector<StarReq> sq;
      std::vector<int> idx;
      for (int c = 0; c < C; ++c)
        if (j < K[c]) idx.push_back(at.at({c, j}));
      std::vector<std::array<cplx*, 4>> Sn(idx.size());
      for (size_t q = 0; q < idx.size(); ++q) {
        It& it = items[idx[q]];
        St& s = st[it.c];
        for (int k = 0; k < 4; ++k) Sn[q][k] = own();
        sq.push_back({s.S[0], s.S[1], s.S[2], s.S[3], it.segp[0], it.segp[1], it.segp[2], it.segp[3], Sn[q][0],
                      Sn[q][1], Sn[q][2], Sn[q][3]});
      }
      std::vector<int> sst;
      star(sq, n, &sst);
      for (int v : sst)
        if (v) throw StatusError(v, "cell backward: singular star product");
      for (size_t q = 0; q < idx.size(); ++q) {
        It& it = items[idx[q]];
        St& s = st[it.c];
        for (int k = 0; k < 4; ++k) {
          it.pre[k] = s.S[k];  // the item takes the state's reference
          s.S[k] = Sn[q][k];
        }
      }
    }
    // states to the block's end: left basis and sample of each cell's last item
    for (int c = 0; c < C; ++c) {
      if (j0 >= K[c]) continue;
      const It& lt = items[at.at({c, std::min(j1, K[c]) - 1})];
      St& s = st[c];
      for (cplx* p : {s.lW, s.lV, s.Pa, s.Qa}) drop(p);
      s.lW = lt.b.W;
      s.lV = lt.b.V;
      s.Pa = lt.Pb;
      s.Qa = lt.Qb;
      for (cplx* p : {s.lW, s.lV, s.Pa, s.Qa}) hold(p);
      if (!keep && lt.j + 1 == K[c]) {  // exit projection (first pass): the last basis's inverses
        last[c].Wi = lt.b.Wi;
        last[c].Vi = lt.b.Vi;
        hold(last[c].Wi);
        hold(last[c].Vi);
      }
    }
    if (!keep) {
      for (It& it : items) {
        for (int k = 0; k < 4; ++k) {
          drop(it.seg[k]);
          drop(it.segp[k]);
          drop(it.pre[k]);
        }
        for (cplx* p : {it.A, it.B, it.Minv, it.b.W, it.b.V, it.b.Wi, it.b.Vi, it.Pb, it.Qb}) drop(p);
        free_vec(it.b.gam, n);
      }
      items.clear();
    }
  };
  auto release_items = [&](std::vector<It>& items) {
    for (It& it : items) {
      for (int k = 0; k < 4; ++k) {
        drop(it.seg[k]);
        drop(it.segp[k]);
        drop(it.pre[k]);
      }
      for (cplx* p : {it.A, it.B, it.Minv, it.b.W, it.b.V, it.b.Wi, it.b.Vi, it.Pb, it.Qb}) drop(p);
      free_vec(it.b.gam, n);
    }
    items.clear();
  };

  // ---- 1. forward with checkpoints ----
  std::vector<std::map<int, Ckpt>> ck(C);
  for (int c = 0; c < C; ++c) {
    St& s = st[c];
    for (int k = 0; k < 4; ++k) s.S[k] = own();
    s.lW = e0[c].W;
    s.lV = e0[c].V;
    s.Pa = P0[c];
    s.Qa = Q0[c];
    for (cplx* p : {s.lW, s.lV, s.Pa, s.Qa}) hold(p);
  }
  {
    Vec I1(C), I2(C), Z1(C), Z2(C);
    for (int c = 0; c < C; ++c) {
      I1[c] = st[c].S[0];
      I2[c] = st[c].S[1];
      Z1[c] = st[c].S[2];
      Z2[c] = st[c].S[3];
    }
    std::vector<const cplx*> none(C, nullptr);
    axpby(none, none, I1, C_ZERO, C_ZERO, 1.0, n);
    axpby(none, none, I2, C_ZERO, C_ZERO, 1.0, n);
    axpby(none, none, Z1, C_ZERO, C_ZERO, 0.0, n);
    axpby(none, none, Z2, C_ZERO, C_ZERO, 0.0, n);
  }
  std::vector<It> items;
  for (int j0 = 0; j0 < Kmax; j0 += every) {
    for (int c = 0; c < C; ++c)
      if (j0 < K[c]) {  // the checkpoint holds the state's pieces
        const St& s = st[c];
        ck[c][j0] = Ckpt{{s.S[0], s.S[1], s.S[2], s.S[3]}, s.lW, s.lV, s.Pa, s.Qa};
        for (cplx* p : {s.S[0], s.S[1], s.S[2], s.S[3], s.lW, s.lV, s.Pa, s.Qa}) hold(p);
      }
    run_block(j0, std::min(Kmax, j0 + every), false, items);
  }

  // ---- 2. exit: projection onto the exit basis, reversed ----
  Vec G[4];
  for (auto& g : G) g = all.alloc(n);
  Vec gW0 = all.alloc(n), gV0 = all.alloc(n), gW1 = all.alloc(n), gV1 = all.alloc(n);
  {
    // cotangents from the caller
    for (int c = 0; c < C; ++c) {
      for (int k = 0; k < 4; ++k)
        VRC_CUDA_CHECK(cudaMemcpyAsync(G[k][c], gS_host[c] + k * nn, nn * 16, cudaMemcpyHostToDevice, stream_));
      Vec* gb[4] = {&gW0, &gV0, &gW1, &gV1};
      for (int k = 0; k < 4; ++k) {
        if (gB_host[c])
          VRC_CUDA_CHECK(
              cudaMemcpyAsync((*gb[k])[c], gB_host[c] + k * nn, nn * 16, cudaMemcpyHostToDevice, stream_));
        else
          VRC_CUDA_CHECK(cudaMemsetAsync((*gb[k])[c], 0, nn * 16, stream_));
      }
    }
    sync();  // host cotangents may go away
  }
  {
    Vec Sc[4], Sn[4];
    for (int k = 0; k < 4; ++k) {
      Sc[k].resize(C);
      for (int c = 0; c < C; ++c) Sc[k][c] = st[c].S[k];
      Sn[k] = all.alloc(n);
    }
    Vec Lwi(C), Lvi(C), W1(C), V1(C);
    for (int c = 0; c < C; ++c) {
      Lwi[c] = last[c].Wi;
      Lvi[c] = last[c].Vi;
      W1[c] = e1[c].W;
      V1[c] = e1[c].V;
    }
    Vec A = all.alloc(n), Bm = all.alloc(n), Mi = all.alloc(n), T1 = all.alloc(n), T2 = all.alloc(n),
        T3 = all.alloc(n);
    all.mm(T1, Lwi, W1, C_ONE, 0, 0, nullptr, C_ZERO, n);
    all.mm(T2, Lvi, V1, C_ONE, 0, 0, nullptr, C_ZERO, n);
    {
      std::vector<const cplx*> t1(T1.begin(), T1.end()), t2(T2.begin(), T2.end());
      axpby(t1, t2, A, C_HALF, C_HALF, 0.0, n);
      axpby(t1, t2, Bm, C_HALF, C_MHALF, 0.0, n);
    }
    all.mm(Mi, Sc[2], Bm, C_MONE, 0, 0, &A, C_ONE, n);  // M = A - Rud B
    inverse(Mi, n, nullptr);
    // forward of the projection (outputs Sn)
    all.mm(Sn[1], Mi, Sc[1], C_ONE, 0, 0, nullptr, C_ZERO, n);        // Tuu' = M^-1 Tuu
    all.mm(T1, Sc[2], A, C_ONE, 0, 0, &Bm, C_MONE, n);                // Rud A - B
    all.mm(Sn[2], Mi, T1, C_ONE, 0, 0, nullptr, C_ZERO, n);           // Rud' = M^-1 (Rud A - B)
    all.mm(T2, Sc[0], Bm, C_ONE, 0, 0, nullptr, C_ZERO, n);           // TB = Tdd B
    all.mm(Sn[3], T2, Sn[1], C_ONE, 0, 0, &Sc[3], C_ONE, n);          // Rdu' = Rdu + TB Tuu'
    all.mm(T1, Bm, Sn[2], C_ONE, 0, 0, &A, C_ONE, n);                 // B Rud' + A
    all.mm(Sn[0], Sc[0], T1, C_ONE, 0, 0, nullptr, C_ZERO, n);        // Tdd' = Tdd (B Rud' + A)
    // reverse (blocks): G holds the adjoints of Sn
    Vec gT[4];
    for (auto& g : gT) g = all.alloc(n);
    copy(G[3], gT[3], n);                                             // gRdu = gRdu'
    all.mm(T3, Bm, Sn[1], C_ONE, 0, 0, nullptr, C_ZERO, n);           // B Tuu'
    all.mm(gT[0], G[3], T3, C_ONE, 0, 1, nullptr, C_ZERO, n);
    all.mm(gT[0], G[0], T1, C_ONE, 0, 1, &gT[0], C_ONE, n);           // gTdd = gRdu' (B Tuu')^H + gTdd' (B Rud' + A)^H
    Vec gTuu2 = all.alloc(n), gRud2 = all.alloc(n), gY = all.alloc(n), gM = all.alloc(n);
    all.mm(gTuu2, T2, G[3], C_ONE, 1, 0, &G[1], C_ONE, n);            // gTuu' + TB^H gRdu'
    all.mm(gRud2, T2, G[0], C_ONE, 1, 0, &G[2], C_ONE, n);            // gRud' + TB^H gTdd'
    all.mm(gT[1], Mi, gTuu2, C_ONE, 1, 0, nullptr, C_ZERO, n);        // gTuu = M^-H (...)
    all.mm(gY, Mi, gRud2, C_ONE, 1, 0, nullptr, C_ZERO, n);           // gY = M^-H (...)
    all.mm(gM, gT[1], Sn[1], C_MONE, 0, 1, nullptr, C_ZERO, n);
    all.mm(gM, gY, Sn[2], C_MONE, 0, 1, &gM, C_ONE, n);               // gM = -gTuu Tuu'^H - gY Rud'^H
    all.mm(gT[2], gY, A, C_ONE, 0, 1, nullptr, C_ZERO, n);
    all.mm(gT[2], gM, Bm, C_MONE, 0, 1, &gT[2], C_ONE, n);            // gRud = gY A^H - gM B^H
    // reverse (projection matrices) -> exit basis
    Vec gA = all.alloc(n), gB = all.alloc(n);
    all.mm(gA, Sc[0], G[0], C_ONE, 1, 0, nullptr, C_ZERO, n);         // Tdd^H gTdd'
    all.mm(T3, Sc[0], G[3], C_ONE, 1, 0, nullptr, C_ZERO, n);
    all.mm(gB, T3, Sn[1], C_ONE, 0, 1, nullptr, C_ZERO, n);           // Tdd^H gRdu' Tuu'^H
    all.mm(gB, gA, Sn[2], C_ONE, 0, 1, &gB, C_ONE, n);                // + Tdd^H gTdd' Rud'^H
    all.mm(gA, Sc[2], gY, C_ONE, 1, 0, &gA, C_ONE, n);                // + Rud^H gY
    {
      std::vector<const cplx*> a(gA.begin(), gA.end()), m(gM.begin(), gM.end()), b(gB.begin(), gB.end()),
          y(gY.begin(), gY.end());
      axpby(a, m, gA, C_ONE, C_ONE, 0.0, n);                          // + gM
      axpby(b, y, gB, C_ONE, C_MONE, 0.0, n);                         // gB - gY
    }
    all.mm(gB, Sc[2], gM, C_MONE, 1, 0, &gB, C_ONE, n);               // - Rud^H gM
    {
      std::vector<const cplx*> a(gA.begin(), gA.end()), b(gB.begin(), gB.end());
      axpby(a, b, T1, C_ONE, C_ONE, 0.0, n);
      axpby(a, b, T2, C_ONE, C_MONE, 0.0, n);
    }
    all.mm(gW1, Lwi, T1, C_HALF, 1, 0, &gW1, C_ONE, n);               // gW1 += Lw^-H (gA + gB) / 2
    all.mm(gV1, Lvi, T2, C_HALF, 1, 0, &gV1, C_ONE, n);               // gV1 += Lv^-H (gA - gB) / 2
    for (int k = 0; k < 4; ++k) std::swap(G[k], gT[k]);
    for (Vec* v : {&gT[0], &gT[1], &gT[2], &gT[3], &A, &Bm, &Mi, &T1, &T2, &T3, &gTuu2, &gRud2, &gY, &gM, &gA, &gB,
                   &Sn[0], &Sn[1], &Sn[2], &Sn[3]})
      all.release(*v, n);
  }

  // the first pass's final states are done with (chain, last basis, exit sample)
  for (int c = 0; c < C; ++c) {
    St& s = st[c];
    for (cplx* p : {s.S[0], s.S[1], s.S[2], s.S[3], s.lW, s.lV, s.Pa, s.Qa}) drop(p);
  }

  // eigen-step adjoint of the end bases (cells whose end is the structure's own)
  auto eig_adjoint = [&](const std::vector<int>& idx, const Vec& P, const Vec& Q, const std::vector<Bas>& bs,
                         const Vec& gW, const Vec& gV, Vec& gP, Vec& gQ) {
    const int B = (int)idx.size();
    if (B == 0) return;
    Batch bt{*this, B};
    Vec W(B), Vv(B), Wi(B), gam(B), gWs(B), gVs(B), Ps(B), Qs(B);
    for (int q = 0; q < B; ++q) {
      const int c = idx[q];
      W[q] = bs[c].W;
      Vv[q] = bs[c].V;
      Wi[q] = bs[c].Wi;
      gam[q] = bs[c].gam;
      gWs[q] = gW[c];
      gVs[q] = gV[c];
      Ps[q] = P[c];
      Qs[q] = Q[c];
    }
    Vec glam(B), igc(B), T = bt.alloc(n), Wt = bt.alloc(n), M = bt.alloc(n);
    for (int q = 0; q < B; ++q) {
      glam[q] = vec(n);
      igc[q] = vec(n);
    }
    double* eta = (double*)bytes((size_t)B * sizeof(double));
    {
      std::vector<GamAdjDesc> gd(B);
      for (int q = 0; q < B; ++q) gd[q] = {Vv[q], gVs[q], gam[q], glam[q], igc[q], eta + q};
      Prof pr(*this, "adjoint", 0.0, 32.0 * n * (double)n * B);
      gamma_adjoint_kernel<<<B, 256, 0, stream_>>>(upload(gd), n);
      VRC_CUDA_CHECK(cudaGetLastError());
    }
    bt.scale(gVs, nullptr, &igc, T, n);                          // T = gV conj(G^-1)
    gP = bt.alloc(n);
    gQ = bt.alloc(n);
    bt.mm(gQ, T, W, C_ONE, 0, 1, nullptr, C_ZERO, n);            // gQ = gV G^-H W^H
    bt.mm(Wt, Qs, T, C_ONE, 1, 0, &gWs, C_ONE, n);               // gW + Q^H gV G^-H
    bt.mm(M, W, Wt, C_ONE, 1, 0, nullptr, C_ZERO, n);            // M = W^H gW
    {
      std::vector<EigFDesc> fd(B);
      for (int q = 0; q < B; ++q) fd[q] = {M[q], gam[q], glam[q], eta + q};
      Prof pr(*this, "adjoint", 0.0, 32.0 * n * (double)n * B);
      eig_f_kernel<<<dim3(grid_for(nn, 256), B), 256, 0, stream_>>>(upload(fd), n);
      VRC_CUDA_CHECK(cudaGetLastError());
    }
    bt.mm(T, Wi, M, C_ONE, 1, 0, nullptr, C_ZERO, n);            // W^-H F
    bt.mm(Wt, T, W, C_ONE, 0, 1, nullptr, C_ZERO, n);            // gA = W^-H F W^H
    bt.mm(gP, Wt, Qs, C_ONE, 0, 1, nullptr, C_ZERO, n);          // gP = gA Q^H
    bt.mm(gQ, Ps, Wt, C_ONE, 1, 0, &gQ, C_ONE, n);               // gQ += P^H gA
    for (int q = 0; q < B; ++q) {
      free_vec(glam[q], n);
      free_vec(igc[q], n);
    }
    free_bytes(eta, (size_t)B * sizeof(double));
    bt.release(T, n);
    bt.release(Wt, n);
    bt.release(M, n);
  };

  // ---- contraction of node adjoints with central differences of the assembly ----
  std::vector<Node> nodes;  // (cell, z, gP, gQ) collected, contracted in groups
  std::vector<std::pair<int, int>> slot_of;  // per contraction result: (node, coordinate)
  std::vector<double> dLdx_host;
  double* dLdx = nullptr;
  size_t dLdx_cap = 0;
  auto contract = [&](std::vector<Node>& ns) {
    if (ns.empty()) return;
    std::vector<std::pair<int, double>> rq;
    std::vector<const CellSpec*> specs;
    std::vector<std::pair<int, int>> who;  // (node, coordinate)
    for (size_t k = 0; k < ns.size(); ++k)
      for (size_t q = 0; q < coords[ns[k].cell].size(); ++q) {
        const Coord& co = coords[ns[k].cell][q];
        rq.push_back({ns[k].cell, ns[k].z});
        specs.push_back(&co.plus);
        rq.push_back({ns[k].cell, ns[k].z});
        specs.push_back(&co.minus);
        who.push_back({(int)k, (int)q});
      }
    if (who.empty()) return;
    Vec Pp, Qp;
    sample_into(rq, &specs, Pp, Qp);
    const size_t base = slot_of.size();
    if (base + who.size() > dLdx_cap) {
      const size_t cap = std::max<size_t>(2 * dLdx_cap, base + who.size() + 1024);
      double* nd = (double*)bytes(cap * sizeof(double));
      VRC_CUDA_CHECK(cudaMemsetAsync(nd, 0, cap * sizeof(double), stream_));
      if (dLdx) {
        VRC_CUDA_CHECK(cudaMemcpyAsync(nd, dLdx, base * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
        free_bytes(dLdx, dLdx_cap * sizeof(double));
      }
      dLdx = nd;
      dLdx_cap = cap;
    }
    std::vector<DotDiffDesc> dd;
    for (size_t w = 0; w < who.size(); ++w) {
      const Node& nd = ns[who[w].first];
      const double sc = 1.0 / (2.0 * coords[nd.cell][who[w].second].h);
      double* out = dLdx + base + w;
      dd.push_back({nd.gP, Pp[2 * w], Pp[2 * w + 1], out, sc});
      dd.push_back({nd.gQ, Qp[2 * w], Qp[2 * w + 1], out, sc});
    }
    {
      Prof pr(*this, "adjoint", 0.0, 48.0 * (double)nn * dd.size());
      dotdiff_kernel<<<dim3(std::min<int>(grid_for(nn, 256), 64), (unsigned)dd.size()), 256, 0, stream_>>>(
          upload(dd), (long long)nn);
      VRC_CUDA_CHECK(cudaGetLastError());
    }
    for (size_t w = 0; w < who.size(); ++w) {
      slot_of.push_back({(int)nodes.size() + who[w].first, who[w].second});
    }
    for (auto& nd : ns) {
      nodes.push_back(nd);
      free_mat(nd.gP, n);
      free_mat(nd.gQ, n);
      nodes.back().gP = nodes.back().gQ = nullptr;
    }
    for (auto* p : Pp) drop(p);
    for (auto* p : Qp) drop(p);
    ns.clear();
  };

  // pending cotangent at each cell's shared node (right end of the segment
  // being reversed); starts with the exit eigen step's (dL/dP, dL/dQ) at z1
  Vec penP(C, nullptr), penQ(C, nullptr);
  {
    std::vector<int> idx;
    for (int c = 0; c < C; ++c)
      if (own1[c]) idx.push_back(c);
    Vec gP, gQ;
    eig_adjoint(idx, P1, Q1, e1, gW1, gV1, gP, gQ);
    for (size_t q = 0; q < idx.size(); ++q) {
      penP[idx[q]] = gP[q];
      penQ[idx[q]] = gQ[q];
    }
  }

  // ---- 3. reverse, block by block from the last checkpoint ----
  for (int j0 = ((Kmax - 1) / every) * every; j0 >= 0; j0 -= every) {
    const int j1 = std::min(Kmax, j0 + every);
    for (int c = 0; c < C; ++c)
      if (j0 < K[c]) {  // the states take over the checkpoint's references
        const Ckpt& k = ck[c].at(j0);
        St& s = st[c];
        for (int q = 0; q < 4; ++q) s.S[q] = k.S[q];
        s.lW = k.lW;
        s.lV = k.lV;
        s.Pa = k.Pa;
        s.Qa = k.Qa;
      }
    run_block(j0, j1, true, items);
    const int NB = (int)items.size();
    std::map<std::pair<int, int>, int> at;
    for (int i = 0; i < NB; ++i) at[{items[i].c, items[i].j}] = i;
    std::vector<std::array<cplx*, 4>> gown(NB);  // own-basis block adjoints of every item
    for (int j = j1 - 1; j >= j0; --j) {
      std::vector<int> idx;
      for (int c = 0; c < C; ++c)
        if (j < K[c]) idx.push_back(at.at({c, j}));
      const int B = (int)idx.size();
      if (B == 0) continue;
      Batch bt{*this, B};
      auto col = [&](auto fn) {
        Vec v(B);
        for (int q = 0; q < B; ++q) v[q] = fn(items[idx[q]]);
        return v;
      };
      Vec Gs[4], pre[4], sgp[4], sg[4];
      for (int k = 0; k < 4; ++k) {
        Gs[k] = col([&](It& t) { return G[k][t.c]; });
        pre[k] = col([&](It& t) { return t.pre[k]; });
        sgp[k] = col([&](It& t) { return t.segp[k]; });
        sg[k] = col([&](It& t) { return t.seg[k]; });
      }
      // ---- star product reversed (both operands) ----
      Vec GP[4], gs[4];
      for (int k = 0; k < 4; ++k) {
        GP[k] = bt.alloc(n);
        gs[k] = bt.alloc(n);
      }
      {
        const Vec &Tdd = pre[0], &Tuu = pre[1], &Rud = pre[2];
        const Vec &tdd = sgp[0], &tuu = sgp[1], &rdu = sgp[3];
        Vec C1 = bt.alloc(n), C1r = bt.alloc(n), C2 = bt.alloc(n), X1 = bt.alloc(n), X2 = bt.alloc(n),
            Y = bt.alloc(n), Zm = bt.alloc(n), RC1 = bt.alloc(n), U = bt.alloc(n), gC1 = bt.alloc(n),
            gC2 = bt.alloc(n), T1 = bt.alloc(n), T2 = bt.alloc(n), T3 = bt.alloc(n), T4 = bt.alloc(n);
        bt.mm(C1, rdu, Rud, C_MONE, 0, 0, nullptr, C_ZERO, n, nullptr, 1.0);  // I - rdu Rud
        inverse(C1, n, nullptr);
        bt.mm(C1r, C1, rdu, C_ONE, 0, 0, nullptr, C_ZERO, n);
        bt.mm(C2, Rud, C1r, C_ONE, 0, 0, nullptr, C_ZERO, n, nullptr, 1.0);   // I + Rud C1 rdu
        bt.mm(X1, Tdd, rdu, C_ONE, 0, 0, nullptr, C_ZERO, n);
        bt.mm(X2, C2, Tuu, C_ONE, 0, 0, nullptr, C_ZERO, n);
        bt.mm(Y, C1, tdd, C_ONE, 0, 0, nullptr, C_ZERO, n);
        bt.mm(Zm, Rud, Y, C_ONE, 0, 0, nullptr, C_ZERO, n);
        bt.mm(RC1, Rud, C1, C_ONE, 0, 0, nullptr, C_ZERO, n);
        copy(Gs[3], GP[3], n);                                                 // gRdu
        bt.mm(T1, Gs[3], X2, C_ONE, 0, 1, nullptr, C_ZERO, n);                 // gX1
        bt.mm(GP[0], T1, rdu, C_ONE, 0, 1, nullptr, C_ZERO, n);                // gTdd = gX1 rdu^H
        bt.mm(gs[3], Tdd, T1, C_ONE, 1, 0, nullptr, C_ZERO, n);                // grdu = Tdd^H gX1
        bt.mm(U, X1, Gs[3], C_ONE, 1, 0, nullptr, C_ZERO, n);
        bt.mm(U, tuu, Gs[1], C_ONE, 1, 0, &U, C_ONE, n);                       // U = X1^H gRdu' + tuu^H gTuu'
        bt.mm(gC2, U, Tuu, C_ONE, 0, 1, nullptr, C_ZERO, n);                   // gC2 = U Tuu^H
        bt.mm(GP[1], C2, U, C_ONE, 1, 0, nullptr, C_ZERO, n);                  // gTuu = C2^H U
        bt.mm(gs[1], Gs[1], X2, C_ONE, 0, 1, nullptr, C_ZERO, n);
        bt.mm(gs[1], Gs[2], Zm, C_ONE, 0, 1, &gs[1], C_ONE, n);                // gtuu
        copy(Gs[2], gs[2], n);                                                 // grud
        bt.mm(GP[0], Gs[0], Y, C_ONE, 0, 1, &GP[0], C_ONE, n);                 // gTdd += gTdd' Y^H
        bt.mm(T2, tuu, Gs[2], C_ONE, 1, 0, nullptr, C_ZERO, n);                // gZ = tuu^H gRud'
        bt.mm(GP[2], T2, Y, C_ONE, 0, 1, nullptr, C_ZERO, n);                  // gRud = gZ Y^H
        bt.mm(T3, Tdd, Gs[0], C_ONE, 1, 0, nullptr, C_ZERO, n);
        bt.mm(T3, Rud, T2, C_ONE, 1, 0, &T3, C_ONE, n);                        // gY = Tdd^H gTdd' + Rud^H gZ
        bt.mm(gC1, T3, tdd, C_ONE, 0, 1, nullptr, C_ZERO, n);                  // gC1 = gY tdd^H
        bt.mm(gs[0], C1, T3, C_ONE, 1, 0, nullptr, C_ZERO, n);                 // gtdd = C1^H gY
        bt.mm(GP[2], gC2, C1r, C_ONE, 0, 1, &GP[2], C_ONE, n);                 // gRud += gC2 (C1 rdu)^H
        bt.mm(T1, Rud, gC2, C_ONE, 1, 0, nullptr, C_ZERO, n);
        bt.mm(gC1, T1, rdu, C_ONE, 0, 1, &gC1, C_ONE, n);                      // gC1 += Rud^H gC2 rdu^H
        bt.mm(gs[3], RC1, gC2, C_ONE, 1, 0, &gs[3], C_ONE, n);                 // grdu += (Rud C1)^H gC2
        bt.mm(T1, gC1, C1, C_ONE, 0, 1, nullptr, C_ZERO, n);
        bt.mm(T4, C1, T1, C_MONE, 1, 0, nullptr, C_ZERO, n);                   // gN = -C1^H gC1 C1^H
        bt.mm(gs[3], T4, Rud, C_MONE, 0, 1, &gs[3], C_ONE, n);                 // grdu -= gN Rud^H
        bt.mm(GP[2], rdu, T4, C_MONE, 1, 0, &GP[2], C_ONE, n);                 // gRud -= rdu^H gN
        for (Vec* v : {&C1, &C1r, &C2, &X1, &X2, &Y, &Zm, &RC1, &U, &gC1, &gC2, &T1, &T2, &T3, &T4})
          bt.release(*v, n);
      }
      // ---- left projection reversed (blocks; and its matrices for j = 0) ----
      Vec go[4];
      for (auto& g : go) g = bt.alloc(n);
      {
        Vec A = col([](It& t) { return t.A; }), Bm = col([](It& t) { return t.B; }),
            Mi = col([](It& t) { return t.Minv; });
        Vec T1 = bt.alloc(n), T2 = bt.alloc(n), tB = bt.alloc(n), gt2 = bt.alloc(n), gY = bt.alloc(n),
            gM = bt.alloc(n);
        const Vec &gtdd_n = gs[0], &gtuu_n = gs[1], &grud_n = gs[2], &grdu_n = gs[3];
        bt.mm(T1, Bm, sgp[3], C_ONE, 0, 0, &A, C_ONE, n);                      // A + B rdu'
        bt.mm(go[1], gtuu_n, T1, C_ONE, 0, 1, nullptr, C_ZERO, n);
        bt.mm(T2, Bm, sgp[0], C_ONE, 0, 0, nullptr, C_ZERO, n);                // B tdd'
        bt.mm(go[1], grud_n, T2, C_ONE, 0, 1, &go[1], C_ONE, n);               // gtuu
        bt.mm(tB, sg[1], Bm, C_ONE, 0, 0, nullptr, C_ZERO, n);                 // tuu B
        bt.mm(T1, tB, gtuu_n, C_ONE, 1, 0, &grdu_n, C_ONE, n);                 // grdu' + tB^H gtuu'
        bt.mm(gt2, tB, grud_n, C_ONE, 1, 0, &gtdd_n, C_ONE, n);                // gtdd' + tB^H grud'
        copy(grud_n, go[2], n);                                                // grud
        bt.mm(go[0], Mi, gt2, C_ONE, 1, 0, nullptr, C_ZERO, n);                // gtdd = M^-H (...)
        bt.mm(gY, Mi, T1, C_ONE, 1, 0, nullptr, C_ZERO, n);                    // gY = M^-H (...)
        bt.mm(gM, go[0], sgp[0], C_MONE, 0, 1, nullptr, C_ZERO, n);
        bt.mm(gM, gY, sgp[3], C_MONE, 0, 1, &gM, C_ONE, n);                    // gM = -gtdd tdd'^H - gY rdu'^H
        bt.mm(go[3], gY, A, C_ONE, 0, 1, nullptr, C_ZERO, n);
        bt.mm(go[3], gM, Bm, C_MONE, 0, 1, &go[3], C_ONE, n);                  // grdu = gY A^H - gM B^H
        if (j == 0) {
          // entrance basis: A, B = (Wm^-1 W0 +- Vm^-1 V0) / 2
          std::vector<int> o0;
          for (int q = 0; q < B; ++q)
            if (own0[items[idx[q]].c]) o0.push_back(q);
          if (!o0.empty()) {
            Batch b0{*this, (int)o0.size()};
            Vec gA = b0.alloc(n), gB = b0.alloc(n), S1 = b0.alloc(n), S2 = b0.alloc(n);
            Vec tuu = sub(sg[1], o0), rdu = sub(sg[3], o0), gtuu = sub(gs[1], o0), grud = sub(gs[2], o0),
                rdun = sub(sgp[3], o0), tddn = sub(sgp[0], o0), gYs = sub(gY, o0), gMs = sub(gM, o0),
                Wi = sub(col([](It& t) { return t.b.Wi; }), o0), Vi = sub(col([](It& t) { return t.b.Vi; }), o0);
            Vec gW(o0.size()), gV(o0.size());
            for (size_t q = 0; q < o0.size(); ++q) {
              gW[q] = gW0[items[idx[o0[q]]].c];
              gV[q] = gV0[items[idx[o0[q]]].c];
            }
            b0.mm(gA, tuu, gtuu, C_ONE, 1, 0, nullptr, C_ZERO, n);              // tuu^H gtuu'
            b0.mm(S1, gA, rdun, C_ONE, 0, 1, nullptr, C_ZERO, n);               // tuu^H gtuu' rdu'^H
            b0.mm(S2, tuu, grud, C_ONE, 1, 0, nullptr, C_ZERO, n);
            b0.mm(gB, S2, tddn, C_ONE, 0, 1, &S1, C_ONE, n);                    // + tuu^H grud' tdd'^H
            b0.mm(gA, rdu, gYs, C_ONE, 1, 0, &gA, C_ONE, n);                    // + rdu^H gY
            {
              std::vector<const cplx*> a(gA.begin(), gA.end()), m(gMs.begin(), gMs.end()),
                  b(gB.begin(), gB.end()), y(gYs.begin(), gYs.end());
              axpby(a, m, gA, C_ONE, C_ONE, 0.0, n);                            // + gM
              axpby(b, y, gB, C_ONE, C_MONE, 0.0, n);                           // - gY
            }
            b0.mm(gB, rdu, gMs, C_MONE, 1, 0, &gB, C_ONE, n);                   // - rdu^H gM
            {
              std::vector<const cplx*> a(gA.begin(), gA.end()), b(gB.begin(), gB.end());
              axpby(a, b, S1, C_ONE, C_ONE, 0.0, n);
              axpby(a, b, S2, C_ONE, C_MONE, 0.0, n);
            }
            b0.mm(gW, Wi, S1, C_HALF, 1, 0, &gW, C_ONE, n);                     // gW0 += Wm^-H (gA + gB) / 2
            b0.mm(gV, Vi, S2, C_HALF, 1, 0, &gV, C_ONE, n);                     // gV0 += Vm^-H (gA - gB) / 2
            for (Vec* v : {&gA, &gB, &S1, &S2}) b0.release(*v, n);
          }
        }
        for (Vec* v : {&T1, &T2, &tB, &gt2, &gY, &gM}) bt.release(*v, n);
      }
      for (int q = 0; q < B; ++q) {
        const int c = items[idx[q]].c;
        for (int k = 0; k < 4; ++k) {
          gown[idx[q]][k] = go[k][q];
          std::swap(G[k][c], GP[k][q]);  // G <- adjoint of the prefix
        }
      }
      for (int k = 0; k < 4; ++k) {
        bt.release(GP[k], n);
        bt.release(gs[k], n);
      }
    }
    // ---- segment formula reversed for the whole block: node cotangents ----
    Batch ball{*this, NB};
    Vec gx[3], gy[3], gP[3], gQ[3];
    for (int k = 0; k < 3; ++k) {
      gx[k] = ball.alloc(n);
      gy[k] = ball.alloc(n);
    }
    {
      std::vector<NodeAdjDesc> nd(NB);
      for (int i = 0; i < NB; ++i) {
        const It& it = items[i];
        nd[i] = {gown[i][0], gown[i][1], gown[i][2], gown[i][3], it.b.gam, {gx[0][i], gx[1][i], gx[2][i]},
                 {gy[0][i], gy[1][i], gy[2][i]}, cuts[it.c][it.j + 1] - cuts[it.c][it.j], cells[it.c].k0()};
      }
      Prof pr(*this, "adjoint", 0.0, 160.0 * (double)nn * NB);
      node_adjoint_kernel<<<dim3(grid_for(nn, 256), NB), 256, 0, stream_>>>(upload(nd), n);
      VRC_CUDA_CHECK(cudaGetLastError());
    }
    for (int i = 0; i < NB; ++i)
      for (int k = 0; k < 4; ++k) free_mat(gown[i][k], n);
    {
      Vec Wm(NB), Vm(NB), Wmi(NB), Vmi(NB), T1 = ball.alloc(n);
      for (int i = 0; i < NB; ++i) {
        Wm[i] = items[i].b.W;
        Vm[i] = items[i].b.V;
        Wmi[i] = items[i].b.Wi;
        Vmi[i] = items[i].b.Vi;
      }
      for (int k = 0; k < 3; ++k) {
        gP[k] = ball.alloc(n);
        gQ[k] = ball.alloc(n);
        ball.mm(T1, Wmi, gx[k], C_ONE, 1, 0, nullptr, C_ZERO, n);
        ball.mm(gP[k], T1, Vm, C_ONE, 0, 1, nullptr, C_ZERO, n);               // dL/dP = Wm^-H gx Vm^H
        ball.mm(T1, Vmi, gy[k], C_ONE, 1, 0, nullptr, C_ZERO, n);
        ball.mm(gQ[k], T1, Wm, C_ONE, 0, 1, nullptr, C_ZERO, n);               // dL/dQ = Vm^-H gy Wm^H
        ball.release(gx[k], n);
        ball.release(gy[k], n);
      }
      ball.release(T1, n);
    }
    // shared nodes: the right node of segment j meets the left node of j + 1
    // (inside the block) or the pending cotangent left by the next block (or
    // by the exit basis); the left node of each cell's first segment here
    // becomes the pending one
    {
      std::vector<const cplx*> a, b2;
      Vec outv;
      for (int i = 0; i < NB; ++i) {
        const It& it = items[i];
        const cplx *addP = nullptr, *addQ = nullptr;
        auto nx = at.find({it.c, it.j + 1});
        if (nx != at.end()) {
          addP = gP[0][nx->second];
          addQ = gQ[0][nx->second];
        } else if (penP[it.c]) {
          addP = penP[it.c];
          addQ = penQ[it.c];
        }
        if (addP) {
          a.push_back(gP[2][i]);
          b2.push_back(addP);
          outv.push_back(gP[2][i]);
          a.push_back(gQ[2][i]);
          b2.push_back(addQ);
          outv.push_back(gQ[2][i]);
        }
      }
      axpby(a, b2, outv, C_ONE, C_ONE, 0.0, n);
    }
    std::vector<Node> ns;
    for (int i = 0; i < NB; ++i) {
      const It& it = items[i];
      const double za = cuts[it.c][it.j], zb = cuts[it.c][it.j + 1];
      ns.push_back({it.c, 0.5 * (za + zb), gP[1][i], gQ[1][i]});
      ns.push_back({it.c, zb, gP[2][i], gQ[2][i]});
    }
    for (int c = 0; c < C; ++c)
      if (j0 < K[c] && penP[c]) {
        free_mat(penP[c], n);
        free_mat(penQ[c], n);
        penP[c] = penQ[c] = nullptr;
      }
    for (int i = 0; i < NB; ++i) {
      const It& it = items[i];
      if (it.j == j0) {
        penP[it.c] = gP[0][i];
        penQ[it.c] = gQ[0][i];
      } else {
        free_mat(gP[0][i], n);
        free_mat(gQ[0][i], n);
      }
    }
    contract(ns);
    release_items(items);
    for (int c = 0; c < C; ++c)
      if (j0 < K[c]) {
        St& s = st[c];
        for (cplx* p : {s.S[0], s.S[1], s.S[2], s.S[3], s.lW, s.lV, s.Pa, s.Qa}) drop(p);
      }
  }

  // ---- 4. entrance eigen step, merged with the first node ----
  {
    std::vector<int> idx;
    for (int c = 0; c < C; ++c)
      if (own0[c]) idx.push_back(c);
    Vec gP, gQ;
    eig_adjoint(idx, P0, Q0, e0, gW0, gV0, gP, gQ);
    std::vector<const cplx*> a, b;
    Vec o;
    for (size_t q = 0; q < idx.size(); ++q) {
      const int c = idx[q];
      a.push_back(penP[c]);
      b.push_back(gP[q]);
      o.push_back(penP[c]);
      a.push_back(penQ[c]);
      b.push_back(gQ[q]);
      o.push_back(penQ[c]);
    }
    axpby(a, b, o, C_ONE, C_ONE, 0.0, n);
    for (size_t q = 0; q < idx.size(); ++q) {
      free_mat(gP[q], n);
      free_mat(gQ[q], n);
    }
    std::vector<Node> ns;
    for (int c = 0; c < C; ++c) ns.push_back({c, cuts[c].front(), penP[c], penQ[c]});
    contract(ns);
  }

  // ---- 5. dL/dx(z) spread over the knots ----
  dLdx_host.resize(slot_of.size());
  if (!slot_of.empty())
    VRC_CUDA_CHECK(cudaMemcpyAsync(dLdx_host.data(), dLdx, slot_of.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                   stream_));
  sync();
  for (size_t s = 0; s < slot_of.size(); ++s) {
    const Node& nd = nodes[slot_of[s].first];
    const Coord& co = coords[nd.cell][slot_of[s].second];
    const auto& rules = co.axis == 0 ? cells[nd.cell].xrules : cells[nd.cell].yrules;
    for (const auto& r : rules)
      if (r.index == co.index) {
        std::vector<double> w;
        r.weights(nd.z, w);
        for (size_t k = 0; k < w.size(); ++k) grad[nd.cell][co.rule + k] += dLdx_host[s] * w[k];
      }
  }

  // ---- release ----
  if (dLdx) free_bytes(dLdx, dLdx_cap * sizeof(double));
  for (int c = 0; c < C; ++c) {
    for (cplx* p : {P0[c], Q0[c], P1[c], Q1[c], last[c].Wi, last[c].Vi}) drop(p);
    drop_bas(e0[c]);
    drop_bas(e1[c]);
    release_cell(cds[c]);
  }
  for (auto& g : G) all.release(g, n);
  for (Vec* v : {&gW0, &gV0, &gW1, &gV1}) all.release(*v, n);
  if (!refs.empty()) throw StatusError(ST_EINVAL, "cell backward: matrices left held");
}

}  // namespace vrc
