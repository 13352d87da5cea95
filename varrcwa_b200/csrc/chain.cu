// Stacks of sections: the role of RCWASolver::solve(lambda, layerStack,
// thickness) (src/rcwa/RCWASolver.cpp:104-113: solveLayers,
// solveInterfaces :460-580, solveScatterMatrix :343-458) for layers that may
// vary with z.  Every section is a cell on its own z-range, integrated as one
// batch by adaptive varRCWA, RCWA or the differential method; the sections
// are then joined in order: section s's entrance, in its own basis W0_s,
// is re-expressed in section s-1's exit basis W1_(s-1) (the projection of
// RedhefferIntegrator.cpp:253-262, which matches the transverse fields W c,
// V c of the two sides, as RCWASolver's interface matrices do) and the
// chain is star-multiplied (:267-277).  The prefix chains are kept, so the
// internal amplitudes at every interface follow from the suffix chains
// (RCWASolver::evaluateIntermediateField, :1373-1480).
#include <cstring>

#include "batch.h"
#include "engine.h"

namespace vrc {

void Engine::release_chain() {
  const int n = chain_.n;
  for (auto& r : chain_.secs) release_result(r);
  for (auto& p : chain_.proj)
    for (auto* m : p) free_mat(m, n);
  for (auto& p : chain_.prefix)
    for (auto* m : p) free_mat(m, n);
  for (auto* m : chain_.V0inv) free_mat(m, n);
  if (chain_.alpha) free_bytes(chain_.alpha, (size_t)chain_.m * sizeof(double));
  if (chain_.beta) free_bytes(chain_.beta, (size_t)chain_.m * sizeof(double));
  chain_ = ChainTape();
}

void Engine::chain(const std::vector<CellSpec>& sections, int method, double pe, int max_depth, int nslices,
                   CellResult& out, std::vector<std::vector<NodeRecord>>& trees) {
  release_chain();
  const int S = (int)sections.size();
  if (S < 1) throw StatusError(ST_EINVAL, "chain: no sections");
  for (const auto& s : sections)
    if (s.nx != sections[0].nx || s.ny != sections[0].ny)
      throw StatusError(ST_EINVAL, "chain: all sections need the same harmonics");
  std::vector<CellSpec> sp(sections);
  for (int s = 0; s < S; ++s) {  // outer media only at the stack's two ends
    sp[s].has_end0 = s == 0 && sections[0].has_end0;
    sp[s].has_end1 = s == S - 1 && sections[S - 1].has_end1;
  }
  ChainTape& t = chain_;
  t.n = sp[0].n();
  t.m = sp[0].m();
  const int n = t.n;
  if (method == 0) {
    RedhefferOpts o;
    o.pe = pe;
    o.max_depth = max_depth;
    redheffer(sp, o, t.secs);
  } else if (method == 1) {
    rcwa(sp, nslices, t.secs);
  } else if (method == 2) {
    differential(sp, nslices, t.secs);
  } else {
    throw StatusError(ST_EINVAL, "chain: unknown method");
  }
  trees.clear();
  for (auto& r : t.secs) trees.push_back(r.nodes);
  // V0^-1 of every section after the first (the projections need W0^-1, V0^-1)
  std::vector<cplx*> vi;
  for (int s = 1; s < S; ++s) {
    cplx* p = mat(n);
    t.V0inv.push_back(p);
    vi.push_back(p);
  }
  {
    std::vector<cplx*> src;
    for (int s = 1; s < S; ++s) src.push_back(t.secs[s].V0);
    copy(src, vi, n);
    std::vector<int> st;
    inverse(vi, n, &st);
    for (int v : st)
      if (v) throw StatusError(v, "chain: singular section basis");
  }
  // projected blocks of every section (section 0 as it is)
  t.proj.resize(S);
  std::vector<ProjReq> pr;
  std::vector<cplx*> src, dst;
  for (int s = 0; s < S; ++s) {
    const CellResult& r = t.secs[s];
    t.proj[s] = {mat(n), mat(n), mat(n), mat(n)};
    const cplx* blk[4] = {r.Tdd, r.Tuu, r.Rud, r.Rdu};
    for (int k = 0; k < 4; ++k) {
      src.push_back(const_cast<cplx*>(blk[k]));
      dst.push_back(t.proj[s][k]);
    }
    if (s > 0)
      pr.push_back({r.W0inv, t.V0inv[s - 1], t.secs[s - 1].W1, t.secs[s - 1].V1, t.proj[s][0], t.proj[s][1],
                    t.proj[s][2], t.proj[s][3]});
  }
  copy(src, dst, n);
  std::vector<int> st;
  project_left(pr, n, &st);
  for (int v : st)
    if (v) throw StatusError(v, "chain: singular interface projection");
  // prefix chains
  t.prefix.resize(S);
  t.prefix[0] = {mat(n), mat(n), mat(n), mat(n)};
  {
    std::vector<cplx*> a(t.proj[0].begin(), t.proj[0].end()), b(t.prefix[0].begin(), t.prefix[0].end());
    copy(a, b, n);
  }
  for (int s = 1; s < S; ++s) {
    t.prefix[s] = {mat(n), mat(n), mat(n), mat(n)};
    std::vector<StarReq> sq = {{t.prefix[s - 1][0], t.prefix[s - 1][1], t.prefix[s - 1][2], t.prefix[s - 1][3],
                                t.proj[s][0], t.proj[s][1], t.proj[s][2], t.proj[s][3], t.prefix[s][0],
                                t.prefix[s][1], t.prefix[s][2], t.prefix[s][3]}};
    std::vector<int> sst;
    star(sq, n, &sst);
    for (int v : sst)
      if (v) throw StatusError(v, "chain: singular star product");
  }
  // periods and harmonics for field images
  {
    std::vector<double> x, y;
    sp[0].geometry(sp[0].z0, x, y);
    t.Lx = x.back() - x.front();
    t.Ly = y.back() - y.front();
    const int nx = sp[0].nx, ny = sp[0].ny, m = t.m;
    std::vector<double> ha(m), hb(m);
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j) {
        ha[ny * i + j] = (2 * 3.1415926535897932 / t.Lx) * (double)(i - (nx - 1) / 2);
        hb[ny * i + j] = (2 * 3.1415926535897932 / t.Ly) * (double)(j - (ny - 1) / 2);
      }
    t.alpha = (double*)bytes((size_t)m * sizeof(double));
    t.beta = (double*)bytes((size_t)m * sizeof(double));
    VRC_CUDA_CHECK(cudaMemcpyAsync(t.alpha, ha.data(), m * sizeof(double), cudaMemcpyHostToDevice, stream_));
    VRC_CUDA_CHECK(cudaMemcpyAsync(t.beta, hb.data(), m * sizeof(double), cudaMemcpyHostToDevice, stream_));
    sync();
  }
  // the stack's result: the last prefix, the entrance and exit bases
  out = CellResult();
  out.n = n;
  for (auto& r : t.secs) {
    out.N += r.N;
    out.n_eig += r.n_eig;
    out.n_samples += r.n_samples;
    out.n_nodes += r.n_nodes;
    if (r.status && !out.status) out.status = r.status;
  }
  out.Tdd = t.prefix[S - 1][0];
  out.Tuu = t.prefix[S - 1][1];
  out.Rud = t.prefix[S - 1][2];
  out.Rdu = t.prefix[S - 1][3];
  const CellResult &f = t.secs[0], &l = t.secs[S - 1];
  out.W0 = f.W0;
  out.V0 = f.V0;
  out.gam0 = f.gam0;
  out.W0inv = f.W0inv;
  out.W1 = l.W1;
  out.V1 = l.V1;
  out.gam1 = l.gam1;
  out.W1inv = l.W1inv;
  t.spec = sp[0];
  t.spec.has_end1 = sp[S - 1].has_end1;
  t.spec.eps_end1 = sp[S - 1].eps_end1;
  t.result = out;
}

void Engine::chain_order_powers(int side, int flux_norm, std::vector<double>& R, std::vector<double>& T) {
  if (chain_.secs.empty()) throw StatusError(ST_EINVAL, "chain powers: no stack solved");
  std::vector<std::vector<double>> Rv, Tv;
  order_powers({chain_.spec}, {chain_.result}, side, flux_norm, Rv, Tv);
  R = Rv[0];
  T = Tv[0];
}

void Engine::chain_fields(const cplx* c_host, int ngx, int ngy, cplx* amps, cplx* img) {
  ChainTape& t = chain_;
  const int S = (int)t.secs.size();
  if (S == 0) throw StatusError(ST_EINVAL, "chain fields: no stack solved");
  if (ngx < 0 || ngy < 0) throw StatusError(ST_EINVAL, "chain fields: negative grid");
  const int n = t.n;
  const size_t nv = n, npix = (size_t)ngx * ngy;
  // device vectors: c, a scratch, and (S+1) x (a+, a-, e)
  cplx* dv = (cplx*)bytes((2 + (size_t)(S + 1) * 3) * nv * 16);
  cplx* cvec = dv;
  cplx* tvec = dv + nv;
  auto ap = [&](int j) { return dv + 2 * nv + (size_t)j * 3 * nv; };
  auto am = [&](int j) { return ap(j) + nv; };
  auto ev = [&](int j) { return ap(j) + 2 * nv; };
  VRC_CUDA_CHECK(cudaMemsetAsync(dv, 0, (2 + (size_t)(S + 1) * 3) * nv * 16, stream_));
  VRC_CUDA_CHECK(cudaMemcpyAsync(cvec, c_host, nv * 16, cudaMemcpyHostToDevice, stream_));
  cplx* dimg = npix ? (cplx*)bytes((size_t)(S + 1) * 2 * npix * 16) : nullptr;
  auto matvec = [&](const std::vector<MatVecDesc>& d) {
    Prof pr(*this, "fields", 8.0 * nv * nv * d.size(), 16.0 * nv * nv * d.size());
    matvec_batched(upload(d), (int)d.size(), n, stream_);
  };
  const auto& F = t.prefix[S - 1];
  {
    // entrance: incident c and reflected Rdu c; exit: transmitted Tuu c
    VRC_CUDA_CHECK(cudaMemcpyAsync(ap(0), cvec, nv * 16, cudaMemcpyDeviceToDevice, stream_));
    matvec({{F[3], cvec, am(0)}, {F[1], cvec, ap(S)}});
  }
  if (S > 1) {
    // suffix chains R_j = proj_j * ... * proj_(S-1) (left end in W1_(j-1)),
    // then at interface j: a+ = (I - Rud_L Rdu_R)^-1 Tuu_L c, a- = Rdu_R a+
    std::vector<std::array<cplx*, 4>> suf(S);
    suf[S - 1] = t.proj[S - 1];
    std::vector<cplx*> made;
    for (int j = S - 2; j >= 1; --j) {
      suf[j] = {mat(n), mat(n), mat(n), mat(n)};
      for (auto* p : suf[j]) made.push_back(p);
      std::vector<StarReq> sq = {{t.proj[j][0], t.proj[j][1], t.proj[j][2], t.proj[j][3], suf[j + 1][0],
                                  suf[j + 1][1], suf[j + 1][2], suf[j + 1][3], suf[j][0], suf[j][1], suf[j][2],
                                  suf[j][3]}};
      star(sq, n, nullptr);
    }
    Batch bt{*this, 1};
    Vec M = bt.alloc(n);
    for (int j = 1; j < S; ++j) {
      const auto& L = t.prefix[j - 1];
      bt.mm(M, {L[2]}, {suf[j][3]}, C_MONE, 0, 0, nullptr, C_ZERO, n, nullptr, 1.0);  // I - Rud_L Rdu_R
      std::vector<int> ist;
      inverse(M, n, &ist);
      for (int v : ist)
        if (v) throw StatusError(v, "chain fields: singular interface system");
      matvec({{L[1], cvec, tvec}});
      matvec({{M[0], tvec, ap(j)}});
      matvec({{suf[j][3], ap(j), am(j)}});
    }
    bt.release(M, n);
    for (auto* p : made) free_mat(p, n);
  }
  {
    std::vector<IfFieldDesc> fd;
    for (int j = 0; j <= S; ++j) {
      const cplx* W = j == 0 ? t.secs[0].W0 : t.secs[j - 1].W1;
      fd.push_back({W, ap(j), am(j), ev(j), t.alpha, t.beta, dimg ? dimg + (size_t)j * 2 * npix : nullptr, t.Lx,
                    t.Ly});
    }
    Prof pr(*this, "fields", 8.0 * nv * nv * fd.size(), 16.0 * (nv * nv + 2.0 * npix) * fd.size());
    interface_fields_batched(upload(fd), (int)fd.size(), n, ngx, ngy, stream_);
  }
  std::vector<cplx> ha((2 + (size_t)(S + 1) * 3) * nv);
  VRC_CUDA_CHECK(cudaMemcpyAsync(ha.data(), dv, ha.size() * 16, cudaMemcpyDeviceToHost, stream_));
  std::vector<cplx> hi(dimg ? (size_t)(S + 1) * 2 * npix : 0);
  if (dimg) VRC_CUDA_CHECK(cudaMemcpyAsync(hi.data(), dimg, hi.size() * 16, cudaMemcpyDeviceToHost, stream_));
  sync();
  for (int j = 0; j <= S; ++j) {
    const cplx* src = ha.data() + 2 * nv + (size_t)j * 3 * nv;
    std::memcpy(amps + (size_t)j * 2 * nv, src, 2 * nv * 16);
  }
  if (img && dimg) std::memcpy(img, hi.data(), hi.size() * 16);
  free_bytes(dv, (2 + (size_t)(S + 1) * 3) * nv * 16);
  if (dimg) free_bytes(dimg, (size_t)(S + 1) * 2 * npix * 16);
}

}  // namespace vrc
