// Integrator drivers.
//
// Adaptive varRCWA (RedhefferIntegrator::compute + recursive_solve,
// src/core/RedhefferIntegrator.cpp:174-314, trisecting branch): every node
// [a,b] of the segmentation tree uses the eigen-basis of its own midpoint
// sample as reference, and its accept test depends on that node alone.  The
// tree is therefore explored level by level for all cells of a batch at
// once: each level evaluates every open node (one batched launch per GEMM /
// inverse / elementwise stage), the host reads back one error per node, and
// rejected nodes are replaced by their three children (two new eigen
// samples; the middle third keeps the parent's reference, as the reference
// does).  Accepted leaves are projected onto their in-order predecessor's
// basis and combined by a pairwise (tree-shaped) Redheffer star-product
// reduction, then the right end is projected onto the z1 basis.
#include "engine.h"

#include <algorithm>
#include <cmath>
#include <list>
#include <map>

namespace vrc {

namespace {
struct SampleB {
  int cell;
  double z;
  bool homog;
  cplx eps_h;
  cplx *P, *Q;
  int refc;
};
struct RefB {
  int sample;
  cplx *W, *V, *Winv, *Vinv, *gam;
  int refc;
};
struct NodeB {
  int cell;
  double a, b;
  int ref, sa, sm, sb, depth;
  cplx *tdd, *tuu, *rud, *rdu;
  double err;
  bool leaf;
};

struct Book {
  Engine& E;
  int n;
  const std::vector<CellSpec>& cells;
  std::vector<Engine::CellDev*>& cds;
  std::vector<SampleB> S;
  std::vector<RefB> R;
  std::vector<int> pend_samples, pend_refs;
  std::vector<int> cell_status;
  std::vector<CellResult>* out;

  Book(Engine& e, int n_, const std::vector<CellSpec>& c, std::vector<Engine::CellDev*>& cd)
      : E(e), n(n_), cells(c), cds(cd) {}

  int sample(int cell, double z, bool homog = false, cplx eps_h = mk(1, 0)) {
    S.push_back({cell, z, homog, eps_h, E.mat(n), E.mat(n), 0});
    pend_samples.push_back((int)S.size() - 1);
    return (int)S.size() - 1;
  }
  int ref(int s) {
    R.push_back({s, E.mat(n), E.mat(n), E.mat(n), E.mat(n), E.vec(n), 0});
    S[s].refc++;  // the eigen step reads P,Q of its sample
    pend_refs.push_back((int)R.size() - 1);
    return (int)R.size() - 1;
  }
  void release_sample(int s) {
    if (--S[s].refc == 0) {
      E.free_mat(S[s].P, n);
      E.free_mat(S[s].Q, n);
      S[s].P = S[s].Q = nullptr;
    }
  }
  void release_ref(int r) {
    if (--R[r].refc == 0) {
      E.free_mat(R[r].W, n);
      E.free_mat(R[r].V, n);
      E.free_mat(R[r].Winv, n);
      E.free_mat(R[r].Vinv, n);
      E.free_vec(R[r].gam, n);
      R[r].W = R[r].V = R[r].Winv = R[r].Vinv = R[r].gam = nullptr;
    }
  }
  // Assemble all pending samples and decompose all pending references.
  void flush() {
    std::vector<Engine::SampleReq> sr;
    for (int s : pend_samples) {
      const SampleB& b = S[s];
      sr.push_back({&cells[b.cell], cds[b.cell], b.z, b.homog, b.eps_h, b.P, b.Q});
      (*out)[b.cell].n_samples++;
    }
    std::vector<int> st;
    E.assemble(sr, &st);
    for (size_t i = 0; i < st.size(); ++i)
      if (st[i]) cell_status[S[pend_samples[i]].cell] = st[i];
    std::vector<Engine::EigReq> er;
    for (int r : pend_refs) {
      const RefB& b = R[r];
      er.push_back({S[b.sample].P, S[b.sample].Q, b.W, b.V, b.Winv, b.Vinv, b.gam});
      (*out)[S[b.sample].cell].n_eig++;
    }
    st.clear();
    E.eig(er, n, &st);
    for (size_t i = 0; i < st.size(); ++i)
      if (st[i]) cell_status[S[R[pend_refs[i]].sample].cell] = st[i];
    for (int r : pend_refs) release_sample(R[r].sample);
    pend_samples.clear();
    pend_refs.clear();
  }
  int end_basis(int cell, int own_sample, bool has, cplx eps) {
    int s = own_sample;
    if (has) s = sample(cell, cells[cell].z0, true, eps);
    int r = ref(s);
    R[r].refc++;  // held by the cell until the end
    return r;
  }
  void export_basis(int r, cplx*& W, cplx*& V, cplx*& gam, cplx*& Winv) {
    W = R[r].W;
    V = R[r].V;
    gam = R[r].gam;
    Winv = R[r].Winv;
    E.free_mat(R[r].Vinv, n);
    R[r].W = R[r].V = R[r].gam = R[r].Winv = R[r].Vinv = nullptr;
  }
};

void start_results(const std::vector<CellSpec>& cells, std::vector<CellResult>& out) {
  out.assign(cells.size(), CellResult());
  for (size_t c = 0; c < cells.size(); ++c) out[c].n = cells[c].n();
}

void validate(const CellSpec& c) {
  if (c.kind == GEOM_SAMPLER) {
    // only n = 2 nx ny matters to the integrators (a LayerSampler exposes nDim)
    if (c.nx < 1 || c.ny < 1 || c.n() > 1024) throw StatusError(ST_EINVAL, "sampler cell: need 2 <= n <= 1024");
    if (!c.host_sample && !c.dev_sample) throw StatusError(ST_EINVAL, "sampler cell without a sampler callback");
    if (!(c.lambda > 0.0)) throw StatusError(ST_EINVAL, "wavelength must be positive");
    if ((c.has_end0 || c.has_end1) && ((c.nx % 2) == 0 || (c.ny % 2) == 0 || c.nx > 64 || c.ny > 64))
      throw StatusError(ST_EINVAL, "half-space ends need the odd harmonic counts nx, ny of the sampler");
    return;
  }
  if (c.nx < 1 || c.ny < 1 || (c.nx % 2) == 0 || (c.ny % 2) == 0)
    throw StatusError(ST_EINVAL, "harmonic counts must be odd and positive");
  if (c.nx > 64 || c.ny > 64 || c.n() > 1024)
    throw StatusError(ST_EINVAL, "truncation too large (nx, ny <= 64 and n <= 1024)");
  if (!(c.lambda > 0.0)) throw StatusError(ST_EINVAL, "wavelength must be positive");
  if (c.kind == GEOM_PILLAR) {
    if (c.npx < 1 || c.npy < 1) throw StatusError(ST_EINVAL, "pillar raster must be non-empty");
  } else if (c.kind == GEOM_PLANAR) {
    if (c.polys.empty()) throw StatusError(ST_EINVAL, "planar cell needs polygons");
    for (const auto& p : c.polys)
      if (p.size() < 6 || p.size() % 2) throw StatusError(ST_EINVAL, "planar polygons need >= 3 points");
    if (!(c.thickness > 0.0)) throw StatusError(ST_EINVAL, "planar device thickness must be positive");
    for (int q = 0; q < 4; ++q)
      if (!(c.pml_w[q] > 0.0) || !(c.space[q] >= 0.0)) throw StatusError(ST_EINVAL, "planar PML / spaces invalid");
  } else {
    if (c.x.size() < 2 || c.y.size() < 2) throw StatusError(ST_EINVAL, "grid needs at least 2 coordinates per axis");
    if (c.eps.size() != (c.x.size() - 1) * (c.y.size() - 1))
      throw StatusError(ST_EINVAL, "eps table does not match the coordinates");
    if (c.pml && (c.x.size() < 4 || c.y.size() < 4))
      throw StatusError(ST_EINVAL, "PML needs at least 4 coordinates per axis");
    for (const auto& r : c.xrules)
      if (r.index < 0 || r.index >= (int)c.x.size() || r.zs.size() != r.vals.size() || r.zs.empty())
        throw StatusError(ST_EINVAL, "invalid x rule");
    for (const auto& r : c.yrules)
      if (r.index < 0 || r.index >= (int)c.y.size() || r.zs.size() != r.vals.size() || r.zs.empty())
        throw StatusError(ST_EINVAL, "invalid y rule");
  }
}
}  // namespace

void Engine::release_result(CellResult& r) {
  const int n = r.n;
  free_mat(r.Tdd, n); free_mat(r.Tuu, n); free_mat(r.Rud, n); free_mat(r.Rdu, n);
  free_mat(r.W0, n); free_mat(r.V0, n); free_vec(r.gam0, n); free_mat(r.W0inv, n);
  free_mat(r.W1, n); free_mat(r.V1, n); free_vec(r.gam1, n); free_mat(r.W1inv, n);
  r.Tdd = r.Tuu = r.Rud = r.Rdu = r.W0 = r.V0 = r.gam0 = r.W0inv = r.W1 = r.V1 = r.gam1 = r.W1inv = nullptr;
}

// ---------------------------------------------------------------------------
// Adaptive varRCWA
// ---------------------------------------------------------------------------
void Engine::redheffer(const std::vector<CellSpec>& cells, const RedhefferOpts& o, std::vector<CellResult>& out) {
  for (const auto& c : cells) validate(c);
  start_results(cells, out);
  std::map<int, std::vector<int>> by_n;
  for (size_t c = 0; c < cells.size(); ++c) by_n[cells[c].n()].push_back((int)c);
  std::vector<std::pair<int, std::vector<int>>> classes(by_n.begin(), by_n.end());
  if (!classes.empty())
    std::rotate(classes.begin(), classes.begin() + (size_t)std::max(0, o.rotate) % classes.size(), classes.end());
  for (auto& kv : classes) {
    const int n = kv.first;
    const std::vector<int>& ids = kv.second;
    std::vector<CellSpec> sub;
    for (int c : ids) sub.push_back(cells[c]);
    std::vector<CellDev*> cds;
    for (auto& c : sub) cds.push_back(prepare_cell(c));
    std::vector<CellResult> res(sub.size());
    for (size_t c = 0; c < sub.size(); ++c) res[c].n = n;
    Book bk(*this, n, sub, cds);
    bk.out = &res;
    bk.cell_status.assign(sub.size(), ST_OK);
    const int C = (int)sub.size();
    std::vector<NodeB> N;
    std::vector<std::list<int>> order(C);
    std::vector<int> e0(C), e1(C);
    std::vector<int> active;
    for (int c = 0; c < C; ++c) {
      const CellSpec& s = sub[c];
      const double z0 = s.z0, z1 = s.z1;
      const int s0 = bk.sample(c, z0), s1 = bk.sample(c, z1);
      e0[c] = bk.end_basis(c, s0, s.has_end0, s.eps_end0);
      e1[c] = bk.end_basis(c, s1, s.has_end1, s.eps_end1);
      if (o.cuts && !(*o.cuts)[ids[c]].empty()) {
        // explicit segments: each with its own midpoint reference
        const std::vector<double>& cut = (*o.cuts)[ids[c]];
        int sa = s0;
        for (size_t k = 0; k + 1 < cut.size(); ++k) {
          double a = cut[k], b = cut[k + 1];
          int sm = bk.sample(c, 0.5 * (a + b));
          int sb = (k + 2 == cut.size()) ? s1 : bk.sample(c, b);
          int r = bk.ref(sm);
          NodeB nd{c, a, b, r, sa, sm, sb, 0, nullptr, nullptr, nullptr, nullptr, 0.0, false};
          bk.R[r].refc++;
          bk.S[sa].refc++;
          bk.S[sm].refc++;
          bk.S[sb].refc++;
          N.push_back(nd);
          order[c].push_back((int)N.size() - 1);
          active.push_back((int)N.size() - 1);
          sa = sb;
        }
      } else {
        const double zm = 0.5 * (z0 + z1);
        const int sm = bk.sample(c, zm);
        const int r = bk.ref(sm);
        NodeB nd{c, z0, z1, r, s0, sm, s1, 0, nullptr, nullptr, nullptr, nullptr, 0.0, false};
        bk.R[r].refc++;
        bk.S[s0].refc++;
        bk.S[sm].refc++;
        bk.S[s1].refc++;
        N.push_back(nd);
        order[c].push_back(0 + (int)N.size() - 1);
        active.push_back((int)N.size() - 1);
      }
    }
    bk.flush();
    const bool replay = (o.cuts != nullptr);
    while (!active.empty()) {
      // Evaluate every open node of this level.
      double* derr = (double*)bytes(active.size() * sizeof(double));
      VRC_CUDA_CHECK(cudaMemsetAsync(derr, 0, active.size() * sizeof(double), stream_));
      std::vector<SegReq> sr;
      for (size_t i = 0; i < active.size(); ++i) {
        NodeB& nd = N[active[i]];
        nd.tdd = mat(n); nd.tuu = mat(n); nd.rud = mat(n); nd.rdu = mat(n);
        const RefB& r = bk.R[nd.ref];
        const SampleB& sm = bk.S[nd.sm];
        sr.push_back({sm.P, sm.Q, r.W, r.V, r.Winv, r.Vinv, r.gam, bk.S[nd.sa].P, bk.S[nd.sa].Q, bk.S[nd.sb].P,
                      bk.S[nd.sb].Q, nd.a, nd.b, sub[nd.cell].k0(), nd.tdd, nd.tuu, nd.rud, nd.rdu, derr + i});
      }
      segments(sr, n);
      std::vector<double> herr(active.size());
      VRC_CUDA_CHECK(cudaMemcpyAsync(herr.data(), derr, herr.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_));
      sync();
      free_bytes(derr, active.size() * sizeof(double));
      std::vector<int> next;
      for (size_t i = 0; i < active.size(); ++i) {
        const int id = active[i];
        NodeB nd = N[id];
        nd.err = herr[i];
        const bool accept = replay || nd.err <= o.pe || nd.depth >= o.max_depth;
        res[nd.cell].nodes.push_back({nd.a, nd.b, nd.err, accept ? 1 : 0});
        res[nd.cell].n_nodes++;
        if (!std::isfinite(nd.err)) bk.cell_status[nd.cell] = ST_ENONFINITE;
        if (accept) {
          nd.leaf = true;
          if (nd.depth >= o.max_depth && nd.err > o.pe && !replay) bk.cell_status[nd.cell] = ST_EDEPTH;
          res[nd.cell].N++;
          N[id] = nd;
          bk.release_sample(nd.sa);
          bk.release_sample(nd.sm);
          bk.release_sample(nd.sb);
          continue;
        }
        free_mat(nd.tdd, n); free_mat(nd.tuu, n); free_mat(nd.rud, n); free_mat(nd.rdu, n);
        nd.tdd = nd.tuu = nd.rud = nd.rdu = nullptr;
        const int c = nd.cell;
        const double a = nd.a, b = nd.b;
        const double zm0 = 2. / 3. * a + 1. / 3. * b;
        const double zm1 = 1. / 3. * a + 2. / 3. * b;
        const int st = bk.sample(c, 0.5 * (a + zm0));
        const int sk = bk.sample(c, zm0);
        const int st2 = bk.sample(c, zm1);
        const int sk2 = bk.sample(c, 0.5 * (zm1 + b));
        const int rl = bk.ref(st), rr = bk.ref(sk2);
        NodeB L{c, a, zm0, rl, nd.sa, st, sk, nd.depth + 1, nullptr, nullptr, nullptr, nullptr, 0.0, false};
        NodeB M{c, zm0, zm1, nd.ref, sk, nd.sm, st2, nd.depth + 1, nullptr, nullptr, nullptr, nullptr, 0.0, false};
        NodeB Rn{c, zm1, b, rr, st2, sk2, nd.sb, nd.depth + 1, nullptr, nullptr, nullptr, nullptr, 0.0, false};
        for (const NodeB* ch : {&L, &M, &Rn}) {
          bk.R[ch->ref].refc++;
          bk.S[ch->sa].refc++;
          bk.S[ch->sm].refc++;
          bk.S[ch->sb].refc++;
        }
        N.push_back(L);
        const int il = (int)N.size() - 1;
        N.push_back(M);
        const int im = (int)N.size() - 1;
        N.push_back(Rn);
        const int ir = (int)N.size() - 1;
        auto it = std::find(order[c].begin(), order[c].end(), id);
        it = order[c].erase(it);
        order[c].insert(it, {il, im, ir});
        next.push_back(il);
        next.push_back(im);
        next.push_back(ir);
        bk.release_ref(nd.ref);
        bk.release_sample(nd.sa);
        bk.release_sample(nd.sm);
        bk.release_sample(nd.sb);
        N[id] = nd;
      }
      bk.flush();
      active.swap(next);
    }
    // Left-end projections of all leaves onto their predecessors' bases.
    std::vector<ProjReq> pr;
    std::vector<int> pr_cell;
    for (int c = 0; c < C; ++c) {
      int prev = e0[c];
      for (int id : order[c]) {
        const NodeB& nd = N[id];
        const RefB& r = bk.R[nd.ref];
        pr.push_back({r.Winv, r.Vinv, bk.R[prev].W, bk.R[prev].V, nd.tdd, nd.tuu, nd.rud, nd.rdu});
        pr_cell.push_back(c);
        prev = nd.ref;
      }
    }
    std::vector<int> pst;
    project_left(pr, n, &pst);
    for (size_t i = 0; i < pst.size(); ++i)
      if (pst[i]) bk.cell_status[pr_cell[i]] = pst[i];
    std::vector<std::vector<SBlocks>> lists(C);
    std::vector<int> last(C);
    for (int c = 0; c < C; ++c) {
      for (int id : order[c]) lists[c].push_back({N[id].tdd, N[id].tuu, N[id].rud, N[id].rdu});
      last[c] = N[order[c].back()].ref;
      for (int id : order[c])
        if (N[id].ref != last[c]) bk.release_ref(N[id].ref);
    }
    star_reduce(lists, n, &bk.cell_status);
    std::vector<ProjRReq> rr;
    for (int c = 0; c < C; ++c) {
      const SBlocks& s = lists[c][0];
      rr.push_back({bk.R[last[c]].Winv, bk.R[last[c]].Vinv, bk.R[e1[c]].W, bk.R[e1[c]].V, s.tdd, s.tuu, s.rud, s.rdu});
    }
    std::vector<int> rst;
    project_right(rr, n, &rst);
    sync();
    for (int c = 0; c < C; ++c) {
      if (rst.size() > (size_t)c && rst[c]) bk.cell_status[c] = rst[c];
      // release the remaining holds of the last leaf's reference
      for (int id : order[c])
        if (N[id].ref == last[c]) bk.release_ref(last[c]);
      CellResult& r = res[c];
      r.Tdd = lists[c][0].tdd;
      r.Tuu = lists[c][0].tuu;
      r.Rud = lists[c][0].rud;
      r.Rdu = lists[c][0].rdu;
      bk.export_basis(e0[c], r.W0, r.V0, r.gam0, r.W0inv);
      bk.export_basis(e1[c], r.W1, r.V1, r.gam1, r.W1inv);
      r.status = bk.cell_status[c];
    }
    // samples still referenced by end bases
    for (size_t s = 0; s < bk.S.size(); ++s)
      if (bk.S[s].P) {
        free_mat(bk.S[s].P, n);
        free_mat(bk.S[s].Q, n);
      }
    for (auto* cd : cds) release_cell(cd);
    for (size_t c = 0; c < ids.size(); ++c) out[ids[c]] = res[c];
  }
}

// ---------------------------------------------------------------------------
// Plain RCWA: N midpoint slices (RCWAIntegrator::compute,
// src/core/RCWAIntegrator.cpp:20-87).
// ---------------------------------------------------------------------------
void Engine::rcwa(const std::vector<CellSpec>& cells, int Nsl, std::vector<CellResult>& out) {
  if (Nsl < 1) throw StatusError(ST_EINVAL, "N must be >= 1");
  for (const auto& c : cells) validate(c);
  start_results(cells, out);
  std::map<int, std::vector<int>> by_n;
  for (size_t c = 0; c < cells.size(); ++c) by_n[cells[c].n()].push_back((int)c);
  for (auto& kv : by_n) {
    const int n = kv.first;
    const std::vector<int>& ids = kv.second;
    std::vector<CellSpec> sub;
    for (int c : ids) sub.push_back(cells[c]);
    std::vector<CellDev*> cds;
    for (auto& c : sub) cds.push_back(prepare_cell(c));
    std::vector<CellResult> res(sub.size());
    for (auto& r : res) r.n = n;
    Book bk(*this, n, sub, cds);
    bk.out = &res;
    const int C = (int)sub.size();
    bk.cell_status.assign(C, ST_OK);
    std::vector<int> e0(C), e1(C);
    std::vector<std::vector<int>> slices(C);
    for (int c = 0; c < C; ++c) {
      const CellSpec& s = sub[c];
      const int s1 = bk.sample(c, s.z1);
      e1[c] = bk.end_basis(c, s1, s.has_end1, s.eps_end1);
      const double dz = (s.z1 - s.z0) / (double)Nsl;
      for (int i = 0; i < Nsl; ++i) {
        int si = bk.sample(c, s.z0 + (i + 0.5) * dz);
        bk.S[si].refc++;
        slices[c].push_back(si);
      }
      const int s0 = bk.sample(c, s.z0);
      e0[c] = bk.end_basis(c, s0, s.has_end0, s.eps_end0);
    }
    bk.flush();
    std::vector<SlabReq> sl;
    std::vector<std::vector<SBlocks>> lists(C);
    std::vector<int> sl_cell;
    for (int c = 0; c < C; ++c) {
      const CellSpec& s = sub[c];
      const double dz = (s.z1 - s.z0) / (double)Nsl;
      for (int si : slices[c]) {
        SBlocks b{mat(n), mat(n), mat(n), mat(n)};
        sl.push_back({bk.S[si].P, bk.S[si].Q, bk.R[e1[c]].W, bk.R[e1[c]].V, s.k0(), dz, b.tuu, b.rud});
        sl_cell.push_back(c);
        lists[c].push_back(b);
      }
      res[c].n_eig += Nsl;
      res[c].N = Nsl;
    }
    std::vector<int> sst;
    rcwa_slabs(sl, n, &sst);
    for (size_t i = 0; i < sst.size(); ++i)
      if (sst[i]) bk.cell_status[sl_cell[i]] = sst[i];
    // symmetric slab: tdd = tuu, rdu = rud (RCWAScatterMatrix.h:44-47)
    std::vector<cplx*> src, dst;
    for (auto& L : lists)
      for (auto& b : L) {
        src.push_back(b.tuu); dst.push_back(b.tdd);
        src.push_back(b.rud); dst.push_back(b.rdu);
      }
    copy(src, dst, n);
    for (int c = 0; c < C; ++c)
      for (int si : slices[c]) bk.release_sample(si);
    star_reduce(lists, n, &bk.cell_status);
    std::vector<ProjLEReq> pl;
    for (int c = 0; c < C; ++c) {
      const SBlocks& s = lists[c][0];
      pl.push_back({bk.R[e1[c]].Winv, bk.R[e1[c]].Vinv, bk.R[e0[c]].W, bk.R[e0[c]].V, s.tdd, s.tuu, s.rud, s.rdu});
    }
    std::vector<int> pst;
    project_left_end(pl, n, &pst);
    sync();
    for (int c = 0; c < C; ++c) {
      if (pst.size() > (size_t)c && pst[c]) bk.cell_status[c] = pst[c];
      CellResult& r = res[c];
      r.Tdd = lists[c][0].tdd; r.Tuu = lists[c][0].tuu; r.Rud = lists[c][0].rud; r.Rdu = lists[c][0].rdu;
      bk.export_basis(e0[c], r.W0, r.V0, r.gam0, r.W0inv);
      bk.export_basis(e1[c], r.W1, r.V1, r.gam1, r.W1inv);
      r.status = bk.cell_status[c];
    }
    for (size_t s = 0; s < bk.S.size(); ++s)
      if (bk.S[s].P) { free_mat(bk.S[s].P, n); free_mat(bk.S[s].Q, n); }
    for (auto* cd : cds) release_cell(cd);
    for (size_t c = 0; c < ids.size(); ++c) out[ids[c]] = res[c];
  }
}

// ---------------------------------------------------------------------------
// Differential method (DifferentialIntegrator::compute,
// src/core/DifferentialIntegrator.cpp:21-134).
// ---------------------------------------------------------------------------
void Engine::differential(const std::vector<CellSpec>& cells, int Nsl, std::vector<CellResult>& out) {
  if (Nsl < 1) throw StatusError(ST_EINVAL, "N must be >= 1");
  for (const auto& c : cells) validate(c);
  start_results(cells, out);
  std::map<int, std::vector<int>> by_n;
  for (size_t c = 0; c < cells.size(); ++c) by_n[cells[c].n()].push_back((int)c);
  for (auto& kv : by_n) {
    const int n = kv.first;
    const std::vector<int>& ids = kv.second;
    std::vector<CellSpec> sub;
    for (int c : ids) sub.push_back(cells[c]);
    std::vector<CellDev*> cds;
    for (auto& c : sub) cds.push_back(prepare_cell(c));
    std::vector<CellResult> res(sub.size());
    for (auto& r : res) r.n = n;
    Book bk(*this, n, sub, cds);
    bk.out = &res;
    const int C = (int)sub.size();
    bk.cell_status.assign(C, ST_OK);
    std::vector<int> e0(C), e1(C);
    std::vector<std::vector<int>> pts(C);  // samples at z0, zm_0, zr_0, zm_1, zr_1, ...
    for (int c = 0; c < C; ++c) {
      const CellSpec& s = sub[c];
      const int s1 = bk.sample(c, s.z1);
      e1[c] = bk.end_basis(c, s1, s.has_end1, s.eps_end1);
      const double dz = (s.z1 - s.z0) / (double)Nsl;
      int p0 = bk.sample(c, s.z0);
      bk.S[p0].refc++;
      pts[c].push_back(p0);
      for (int i = 0; i < Nsl; ++i) {
        const double zl = s.z0 + i * dz, zr = s.z0 + (i + 1) * dz, zm = 0.5 * (zl + zr);
        int pm = bk.sample(c, zm), pr = bk.sample(c, zr);
        bk.S[pm].refc++;
        bk.S[pr].refc++;
        pts[c].push_back(pm);
        pts[c].push_back(pr);
      }
      const int s0 = bk.sample(c, s.z0);
      e0[c] = bk.end_basis(c, s0, s.has_end0, s.eps_end0);
      res[c].N = Nsl;
    }
    bk.flush();
    std::vector<DiffReq> dr;
    std::vector<std::vector<SBlocks>> lists(C);
    std::vector<int> dr_cell;
    for (int c = 0; c < C; ++c) {
      const CellSpec& s = sub[c];
      const double dz = (s.z1 - s.z0) / (double)Nsl;
      const RefB& b1 = bk.R[e1[c]];
      for (int i = 0; i < Nsl; ++i) {
        const SampleB &A0 = bk.S[pts[c][2 * i]], &A1 = bk.S[pts[c][2 * i + 1]], &A2 = bk.S[pts[c][2 * i + 2]];
        SBlocks b{mat(n), mat(n), mat(n), mat(n)};
        dr.push_back({A0.P, A0.Q, A1.P, A1.Q, A2.P, A2.Q, b1.W, b1.V, b1.Winv, b1.Vinv, s.k0(), dz, b.tdd, b.tuu, b.rud,
                      b.rdu});
        dr_cell.push_back(c);
        lists[c].push_back(b);
      }
    }
    std::vector<int> dst;
    diff_slices(dr, n, &dst);
    for (size_t i = 0; i < dst.size(); ++i)
      if (dst[i]) bk.cell_status[dr_cell[i]] = dst[i];
    for (int c = 0; c < C; ++c)
      for (int p : pts[c]) bk.release_sample(p);
    star_reduce(lists, n, &bk.cell_status);
    std::vector<ProjLEReq> pl;
    for (int c = 0; c < C; ++c) {
      const SBlocks& s = lists[c][0];
      pl.push_back({bk.R[e1[c]].Winv, bk.R[e1[c]].Vinv, bk.R[e0[c]].W, bk.R[e0[c]].V, s.tdd, s.tuu, s.rud, s.rdu});
    }
    std::vector<int> pst;
    project_left_end(pl, n, &pst);
    sync();
    for (int c = 0; c < C; ++c) {
      if (pst.size() > (size_t)c && pst[c]) bk.cell_status[c] = pst[c];
      CellResult& r = res[c];
      r.Tdd = lists[c][0].tdd; r.Tuu = lists[c][0].tuu; r.Rud = lists[c][0].rud; r.Rdu = lists[c][0].rdu;
      bk.export_basis(e0[c], r.W0, r.V0, r.gam0, r.W0inv);
      bk.export_basis(e1[c], r.W1, r.V1, r.gam1, r.W1inv);
      r.status = bk.cell_status[c];
    }
    for (size_t s = 0; s < bk.S.size(); ++s)
      if (bk.S[s].P) { free_mat(bk.S[s].P, n); free_mat(bk.S[s].Q, n); }
    for (auto* cd : cds) release_cell(cd);
    for (size_t c = 0; c < ids.size(); ++c) out[ids[c]] = res[c];
  }
}

// ---------------------------------------------------------------------------
// Per-order powers (RCWASolver::scatterPlaneWave, src/rcwa/RCWASolver.cpp:1636-1733)
// ---------------------------------------------------------------------------
void Engine::order_powers(const std::vector<CellSpec>& cells, const std::vector<CellResult>& res, int side,
                          int flux_norm, std::vector<std::vector<double>>& Rout,
                          std::vector<std::vector<double>>& Tout) {
  const size_t C = cells.size();
  Rout.assign(C, {});
  Tout.assign(C, {});
  std::map<int, std::vector<int>> by_n;
  for (size_t c = 0; c < C; ++c) {
    if (!cells[c].has_end0 || !cells[c].has_end1)
      throw StatusError(ST_EINVAL, "order powers need homogeneous end media");
    if (cells[c].pml) throw StatusError(ST_EINVAL, "order powers need periodic boundaries");
    by_n[cells[c].n()].push_back((int)c);
  }
  for (auto& kv : by_n) {
    const int n = kv.first, m = n / 2;
    const std::vector<int>& ids = kv.second;
    const size_t B = ids.size();
    // two polarisations per cell
    std::vector<cplx*> cvec(2 * B), rc(2 * B), rf(2 * B), tc(2 * B), tf(2 * B);
    std::vector<MatVecDesc> mv1, mv2;
    std::vector<double*> Rd(2 * B), Td(2 * B);
    std::vector<double*> ab(B);
    for (size_t b = 0; b < B; ++b) {
      const CellSpec& s = cells[ids[b]];
      const CellResult& r = res[ids[b]];
      const int nx = s.nx, ny = s.ny;
      const int c0 = (ny * (nx - 1)) / 2 + (ny - 1) / 2;
      const cplx* Win = side == 0 ? r.W0 : r.W1;
      const cplx* Wininv = side == 0 ? r.W0inv : r.W1inv;
      const cplx* Wout = side == 0 ? r.W1 : r.W0;
      const cplx* Rm = side == 0 ? r.Rdu : r.Rud;
      const cplx* Tm = side == 0 ? r.Tuu : r.Tdd;
      for (int p = 0; p < 2; ++p) {
        const size_t k = 2 * b + p;
        // c = Win^-1 s with s the unit vector of the zero order (px or py)
        cvec[k] = const_cast<cplx*>(Wininv) + (size_t)(p == 0 ? c0 : m + c0) * n;
        rc[k] = vec(n); rf[k] = vec(n); tc[k] = vec(n); tf[k] = vec(n);
        mv1.push_back({Rm, cvec[k], rc[k]});
        mv1.push_back({Tm, cvec[k], tc[k]});
        mv2.push_back({Win, rc[k], rf[k]});
        mv2.push_back({Wout, tc[k], tf[k]});
        Rd[k] = (double*)bytes(m * sizeof(double));
        Td[k] = (double*)bytes(m * sizeof(double));
      }
      ab[b] = (double*)bytes(2 * m * sizeof(double));
    }
    {
      Prof pr(*this, "powers", 16.0 * n * (double)n * (mv1.size() + mv2.size()), 16.0 * n * (double)n * (mv1.size() + mv2.size()), 2);
      matvec_batched(upload(mv1), (int)mv1.size(), n, stream_);
      matvec_batched(upload(mv2), (int)mv2.size(), n, stream_);
    }
    std::vector<PowerDesc> pd;
    std::vector<std::vector<double>> hab(B);
    for (size_t b = 0; b < B; ++b) {
      const CellSpec& s = cells[ids[b]];
      // alpha/beta: src/core/LayerSampler.cpp:9-32
      std::vector<double> x, y;
      s.geometry(s.z0, x, y);
      const double Lx = x.back() - x.front(), Ly = y.back() - y.front();
      hab[b].resize(2 * m);
      const int Nx = (s.nx - 1) / 2, Ny = (s.ny - 1) / 2;
      for (int i = 0; i < s.nx; ++i)
        for (int j = 0; j < s.ny; ++j) {
          hab[b][s.ny * i + j] = (2 * 3.1415926535897932 / Lx) * (double)(i - Nx);
          hab[b][m + s.ny * i + j] = (2 * 3.1415926535897932 / Ly) * (double)(j - Ny);
        }
      VRC_CUDA_CHECK(cudaMemcpyAsync(ab[b], hab[b].data(), 2 * m * sizeof(double), cudaMemcpyHostToDevice, stream_));
      const cplx ein = side == 0 ? s.eps_end0 : s.eps_end1;
      const cplx eout = side == 0 ? s.eps_end1 : s.eps_end0;
      const double tn = flux_norm ? std::sqrt(ein.x) : std::sqrt(eout.x);
      for (int p = 0; p < 2; ++p) {
        const size_t k = 2 * b + p;
        pd.push_back({rf[k], tf[k], ab[b], ab[b] + m, Rd[k], Td[k], ein, eout, s.k0(), tn});
      }
    }
    {
      Prof pr(*this, "powers", 0.0, 64.0 * m * (double)pd.size());
      order_power_batched(upload(pd), (int)pd.size(), m, stream_);
    }
    for (size_t b = 0; b < B; ++b) {
      Rout[ids[b]].resize(2 * m);
      Tout[ids[b]].resize(2 * m);
      for (int p = 0; p < 2; ++p) {
        const size_t k = 2 * b + p;
        VRC_CUDA_CHECK(cudaMemcpyAsync(Rout[ids[b]].data() + p * m, Rd[k], m * sizeof(double), cudaMemcpyDeviceToHost,
                                       stream_));
        VRC_CUDA_CHECK(cudaMemcpyAsync(Tout[ids[b]].data() + p * m, Td[k], m * sizeof(double), cudaMemcpyDeviceToHost,
                                       stream_));
      }
    }
    sync();
    for (size_t k = 0; k < 2 * B; ++k) {
      free_vec(rc[k], n); free_vec(rf[k], n); free_vec(tc[k], n); free_vec(tf[k], n);
      free_bytes(Rd[k], m * sizeof(double));
      free_bytes(Td[k], m * sizeof(double));
    }
    for (size_t b = 0; b < B; ++b) free_bytes(ab[b], 2 * m * sizeof(double));
  }
}

}  // namespace vrc
