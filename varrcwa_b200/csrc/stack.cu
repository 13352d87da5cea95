// Layer stacks of z-uniform pixel rasters: batched forward solve and adjoint.
//
// Forward (the Redheffer chain of src/core/RedhefferIntegrator.cpp:174-277 on
// a piecewise-constant structure): a z-uniform layer's perturbative segment
// (RedhefferIntegrator.cpp:317-399) has zero perturbation, so its S-matrix in
// its own eigenbasis is (tdd, tuu, rud, rdu) = (X, X, 0, 0) with
// X = diag(exp(i gamma d / k0)).  Each layer's left end is re-expressed in the
// previous layer's basis (RedhefferIntegrator.cpp:253-262; with rdu = 0 the
// projection matrix M is A itself), the chain is star-multiplied
// (:267-277) and its right end finally moved to the exit medium (:211-223).
// Per-order powers follow RCWASolver::scatterPlaneWave
// (src/rcwa/RCWASolver.cpp:1636-1733), incidence from eps_in.
//
// Adjoint: every basis is held fixed, so a pixel perturbation reaches the
// S-matrix only through the perturbed layer's own-basis blocks (adjoint.cu has
// the exact first-order kernel).  The reverse pass runs the star products and
// projections backwards with respect to their block operands, then the
// Toeplitz assembly (FourierSolver2D, Layer::waveEqnCoeff) back to pixels.
// Each stage is batched over all stacks of the call.
#include <cstring>

#include "batch.h"
#include "engine.h"

namespace vrc {

namespace {

const cplx ONE = C_ONE, ZERO = C_ZERO, MONE = C_MONE, HALF = C_HALF, MHALF = C_MHALF;

struct Carve {
  char* base;
  size_t off = 0;
  cplx* take(size_t count) {
    cplx* p = base ? reinterpret_cast<cplx*>(base + off) : nullptr;
    off += (count * 16 + 255) / 256 * 256;
    return p;
  }
};

}  // namespace

void Engine::release_stack_tape() {
  for (auto& c : tape_.cells)
    if (c.mem) free_bytes(c.mem, c.bytes);
  tape_ = StackTape();
}

void Engine::stack_forward(const std::vector<StackSpec>& stacks, double px, double py, double* REF, double* TRN,
                           int* status) {
  release_stack_tape();
  if (stacks.empty()) return;
  const StackSpec& s0 = stacks[0];
  for (const auto& s : stacks) {
    if (s.nx < 1 || s.ny < 1 || (s.nx % 2) == 0 || (s.ny % 2) == 0 || s.npx < 1 || s.npy < 1 || s.L < 1)
      throw StatusError(ST_EINVAL, "stack: harmonics must be odd and positive, rasters and layers non-empty");
    if (s.nx != s0.nx || s.ny != s0.ny || s.npx != s0.npx || s.npy != s0.npy || s.L != s0.L)
      throw StatusError(ST_EINVAL, "stack: every stack of a call needs the same harmonics, raster and layer count");
    if ((int)s.eps.size() != s.L * s.npx * s.npy || (int)s.thick.size() != s.L)
      throw StatusError(ST_EINVAL, "stack: eps / thickness arrays do not match the layer count");
    if (!(s.lambda > 0.0) || !(s.Lx > 0.0) || !(s.Ly > 0.0))
      throw StatusError(ST_EINVAL, "stack: wavelength and period must be positive");
    for (double t : s.thick)
      if (!(t > 0.0)) throw StatusError(ST_EINVAL, "stack: layer thickness must be positive");
    for (double v : s.eps)
      if (!(v != 0.0) || v != v) throw StatusError(ST_EINVAL, "stack: permittivity must be finite and non-zero");
  }
  if (!pixel_adjoint_fits(s0.nx, s0.ny, s0.npx, s0.npy))
    throw StatusError(ST_EINVAL, "stack: raster and harmonics exceed the adjoint's shared-memory tile");
  StackTape& tp = tape_;
  const int C = (int)stacks.size(), L = s0.L, nx = s0.nx, ny = s0.ny, npx = s0.npx, npy = s0.npy;
  const int m = nx * ny, n = 2 * m;
  tp.C = C; tp.L = L; tp.n = n; tp.m = m; tp.nx = nx; tp.ny = ny; tp.npx = npx; tp.npy = npy;
  tp.px = px; tp.py = py;
  tp.specs = stacks;
  tp.status.assign(C, ST_OK);
  tp.cells.resize(C);
  const size_t nn = (size_t)n * n;
  auto carve = [&](StackCell& sc, char* base) {
    Carve cv{base};
    auto basis = [&](EndBasis& b) {
      b.W = cv.take(nn); b.V = cv.take(nn); b.Winv = cv.take(nn); b.Vinv = cv.take(nn); b.gam = cv.take(n);
    };
    basis(sc.e0);
    basis(sc.e1);
    sc.lay.resize(L);
    for (auto& l : sc.lay) {
      l.P = cv.take(nn); l.Q = cv.take(nn); l.W = cv.take(nn); l.V = cv.take(nn); l.Winv = cv.take(nn);
      l.Vinv = cv.take(nn); l.gam = cv.take(n); l.A = cv.take(nn); l.B = cv.take(nn); l.Ainv = cv.take(nn);
      l.x = cv.take(n); l.fe33inv = cv.take((size_t)m * m); l.eps = cv.take((size_t)npx * npy);
      for (int k = 0; k < 4; ++k) l.seg[k] = cv.take(nn);
      for (int k = 0; k < 4; ++k) l.pre[k] = cv.take(nn);
    }
    for (int k = 0; k < 4; ++k) sc.Sc[k] = cv.take(nn);
    for (int k = 0; k < 4; ++k) sc.S[k] = cv.take(nn);
    sc.Ar = cv.take(nn); sc.Br = cv.take(nn); sc.Mrinv = cv.take(nn);
    sc.alpha = reinterpret_cast<double*>(cv.take((m + 1) / 2));
    sc.beta = reinterpret_cast<double*>(cv.take((m + 1) / 2));
    return cv.off;
  };
  for (auto& sc : tp.cells) {
    sc.bytes = carve(sc, nullptr);
    sc.mem = (char*)bytes(sc.bytes);
    carve(sc, sc.mem);
  }

  // ---- P, Q of every layer and of the two end media ----
  std::vector<CellSpec> lspec((size_t)C * L);
  std::vector<CellDev*> cds((size_t)C * L);
  std::vector<SampleReq> reqs;
  std::vector<cplx*> endP, endQ;
  for (int c = 0; c < C; ++c) {
    const StackSpec& s = stacks[c];
    for (int l = 0; l < L; ++l) {
      CellSpec& cs = lspec[(size_t)c * L + l];
      cs.kind = GEOM_PIXELS;
      cs.nx = nx; cs.ny = ny; cs.pml = false; cs.lambda = s.lambda;
      cs.z0 = 0.0; cs.z1 = s.thick[l];
      cs.x.resize(npx + 1);
      cs.y.resize(npy + 1);
      for (int i = 0; i <= npx; ++i) cs.x[i] = s.Lx * i / npx;
      for (int j = 0; j <= npy; ++j) cs.y[j] = s.Ly * j / npy;
      cs.eps.resize((size_t)npx * npy);
      const double* e = s.eps.data() + (size_t)l * npx * npy;
      for (size_t k = 0; k < cs.eps.size(); ++k) cs.eps[k] = mk(e[k], 0.0);
      cds[(size_t)c * L + l] = prepare_cell(cs);
      StackLayer& ly = tp.cells[c].lay[l];
      VRC_CUDA_CHECK(cudaMemcpyAsync(ly.eps, cds[(size_t)c * L + l]->eps_dev, cs.eps.size() * 16,
                                     cudaMemcpyDeviceToDevice, stream_));
      SampleReq r{&cs, cds[(size_t)c * L + l], 0.5 * s.thick[l], false, ZERO, ly.P, ly.Q};
      r.keep_fe33inv = ly.fe33inv;
      reqs.push_back(r);
    }
    const CellDev* cd0 = cds[(size_t)c * L];
    StackCell& sc = tp.cells[c];
    VRC_CUDA_CHECK(cudaMemcpyAsync(sc.alpha, cd0->h_alpha.data(), m * sizeof(double), cudaMemcpyHostToDevice, stream_));
    VRC_CUDA_CHECK(cudaMemcpyAsync(sc.beta, cd0->h_beta.data(), m * sizeof(double), cudaMemcpyHostToDevice, stream_));
    for (int side = 0; side < 2; ++side) {
      cplx* P = mat(n);
      cplx* Q = mat(n);
      endP.push_back(P);
      endQ.push_back(Q);
      reqs.push_back({&lspec[(size_t)c * L], cds[(size_t)c * L], 0.0, true, side ? s.eps_out : s.eps_in, P, Q});
    }
  }
  std::vector<int> ast;
  assemble(reqs, &ast);
  std::vector<EigReq> er;
  std::vector<int> er_cell;
  for (int c = 0; c < C; ++c) {
    StackCell& sc = tp.cells[c];
    for (auto& l : sc.lay) {
      er.push_back({l.P, l.Q, l.W, l.V, l.Winv, l.Vinv, l.gam});
      er_cell.push_back(c);
    }
    er.push_back({endP[2 * c], endQ[2 * c], sc.e0.W, sc.e0.V, sc.e0.Winv, sc.e0.Vinv, sc.e0.gam});
    er.push_back({endP[2 * c + 1], endQ[2 * c + 1], sc.e1.W, sc.e1.V, sc.e1.Winv, sc.e1.Vinv, sc.e1.gam});
    er_cell.push_back(c);
    er_cell.push_back(c);
  }
  std::vector<int> est;
  eig(er, n, &est);
  for (size_t i = 0; i < est.size(); ++i)
    if (est[i]) tp.status[er_cell[i]] = est[i];
  for (auto* p : endP) free_mat(p, n);
  for (auto* p : endQ) free_mat(p, n);

  // ---- the chain ----
  Batch bt{*this, C};
  auto gather = [&](auto fn) {
    Vec v(C);
    for (int c = 0; c < C; ++c) v[c] = fn(tp.cells[c]);
    return v;
  };
  {
    Vec id0 = gather([](StackCell& s) { return s.lay[0].pre[0]; });
    Vec id1 = gather([](StackCell& s) { return s.lay[0].pre[1]; });
    Vec z2 = gather([](StackCell& s) { return s.lay[0].pre[2]; });
    Vec z3 = gather([](StackCell& s) { return s.lay[0].pre[3]; });
    Vec one(id0), zero(z2);
    one.insert(one.end(), id1.begin(), id1.end());
    zero.insert(zero.end(), z3.begin(), z3.end());
    set_identity_batched(upload(one), (int)one.size(), n, 1.0, stream_);
    set_identity_batched(upload(zero), (int)zero.size(), n, 0.0, stream_);
  }
  Vec T1 = bt.alloc(n), T2 = bt.alloc(n);
  for (int l = 0; l < L; ++l) {
    Vec lW = gather([&](StackCell& s) { return l ? s.lay[l - 1].W : s.e0.W; });
    Vec lV = gather([&](StackCell& s) { return l ? s.lay[l - 1].V : s.e0.V; });
    Vec Wi = gather([&](StackCell& s) { return s.lay[l].Winv; });
    Vec Vi = gather([&](StackCell& s) { return s.lay[l].Vinv; });
    Vec A = gather([&](StackCell& s) { return s.lay[l].A; });
    Vec B = gather([&](StackCell& s) { return s.lay[l].B; });
    Vec Ai = gather([&](StackCell& s) { return s.lay[l].Ainv; });
    Vec x = gather([&](StackCell& s) { return s.lay[l].x; });
    Vec g = gather([&](StackCell& s) { return s.lay[l].gam; });
    Vec sg[4], pr[4];
    for (int k = 0; k < 4; ++k) {
      sg[k] = gather([&](StackCell& s) { return s.lay[l].seg[k]; });
      pr[k] = gather([&](StackCell& s) { return s.lay[l].pre[k]; });
    }
    bt.mm(T1, Wi, lW, HALF, 0, 0, nullptr, ZERO, n);            // T1 = Winv leftW / 2
    bt.mm(A, Vi, lV, HALF, 0, 0, &T1, ONE, n);                  // A = T1 + Vinv leftV / 2
    bt.mm(B, Vi, lV, MHALF, 0, 0, &T1, ONE, n);                 // B = T1 - Vinv leftV / 2
    copy(A, Ai, n);
    std::vector<int> ist;
    inverse(Ai, n, &ist);
    for (int c = 0; c < C; ++c)
      if (ist.size() > (size_t)c && ist[c]) tp.status[c] = ist[c];
    std::vector<double> ts(C);
    for (int c = 0; c < C; ++c) ts[c] = stacks[c].thick[l] / (2.0 * 3.1415926535897932 / stacks[c].lambda);
    {
      std::vector<const cplx*> gc(g.begin(), g.end());
      phase_vec_batched(upload(gc), upload(ts), upload(x), C, n, stream_);
    }
    bt.mm(sg[3], Ai, B, MONE, 0, 0, nullptr, ZERO, n);          // rdu' = -A^-1 B
    bt.scale(Ai, nullptr, &x, sg[0], n);                        // tdd' = A^-1 X
    bt.mm(sg[2], B, sg[0], ONE, 0, 0, nullptr, ZERO, n, &x);    // rud' = X B tdd'
    bt.mm(T2, B, sg[3], ONE, 0, 0, &A, ONE, n);                 // A + B rdu'
    bt.scale(T2, &x, nullptr, sg[1], n);                        // tuu' = X (A + B rdu')
    Vec out[4];
    for (int k = 0; k < 4; ++k)
      out[k] = gather([&](StackCell& s) { return l + 1 < L ? s.lay[l + 1].pre[k] : s.Sc[k]; });
    std::vector<StarReq> sr(C);
    for (int c = 0; c < C; ++c)
      sr[c] = {pr[0][c], pr[1][c], pr[2][c], pr[3][c], sg[0][c], sg[1][c], sg[2][c], sg[3][c],
               out[0][c], out[1][c], out[2][c], out[3][c]};
    std::vector<int> sst;
    star(sr, n, &sst);
    for (int c = 0; c < C; ++c)
      if (sst.size() > (size_t)c && sst[c]) tp.status[c] = sst[c];
  }
  // ---- right end to the exit medium ----
  {
    Vec Wi = gather([&](StackCell& s) { return s.lay[L - 1].Winv; });
    Vec Vi = gather([&](StackCell& s) { return s.lay[L - 1].Vinv; });
    Vec W1 = gather([](StackCell& s) { return s.e1.W; });
    Vec V1 = gather([](StackCell& s) { return s.e1.V; });
    Vec Ar = gather([](StackCell& s) { return s.Ar; });
    Vec Br = gather([](StackCell& s) { return s.Br; });
    Vec Mi = gather([](StackCell& s) { return s.Mrinv; });
    Vec Sc[4], S[4];
    for (int k = 0; k < 4; ++k) {
      Sc[k] = gather([&](StackCell& s) { return s.Sc[k]; });
      S[k] = gather([&](StackCell& s) { return s.S[k]; });
    }
    bt.mm(T1, Wi, W1, HALF, 0, 0, nullptr, ZERO, n);
    bt.mm(Ar, Vi, V1, HALF, 0, 0, &T1, ONE, n);
    bt.mm(Br, Vi, V1, MHALF, 0, 0, &T1, ONE, n);
    bt.mm(Mi, Sc[2], Br, MONE, 0, 0, &Ar, ONE, n);              // M = A - Rud B
    std::vector<int> ist;
    inverse(Mi, n, &ist);
    for (int c = 0; c < C; ++c)
      if (ist.size() > (size_t)c && ist[c]) tp.status[c] = ist[c];
    bt.mm(S[1], Mi, Sc[1], ONE, 0, 0, nullptr, ZERO, n);        // Tuu = M^-1 Tuu
    bt.mm(T1, Sc[2], Ar, ONE, 0, 0, &Br, MONE, n);              // Rud A - B
    bt.mm(S[2], Mi, T1, ONE, 0, 0, nullptr, ZERO, n);           // Rud = M^-1 (Rud A - B)
    bt.mm(T1, Br, S[1], ONE, 0, 0, nullptr, ZERO, n);           // B Tuu'
    bt.mm(S[3], Sc[0], T1, ONE, 0, 0, &Sc[3], ONE, n);          // Rdu = Rdu + Tdd B Tuu'
    bt.mm(T2, Br, S[2], ONE, 0, 0, &Ar, ONE, n);                // B Rud' + A
    bt.mm(S[0], Sc[0], T2, ONE, 0, 0, nullptr, ZERO, n);        // Tdd = Tdd (B Rud' + A)
  }
  bt.release(T1, n);
  bt.release(T2, n);
  for (auto* cd : cds) release_cell(cd);

  // ---- per-order powers ----
  double* dR = (double*)bytes((size_t)C * m * 8);
  double* dT = (double*)bytes((size_t)C * m * 8);
  std::vector<StackPowerDesc> pd(C);
  for (int c = 0; c < C; ++c) {
    StackCell& sc = tp.cells[c];
    const StackSpec& s = stacks[c];
    pd[c] = {sc.e0.W, sc.e0.Winv, sc.e1.W, sc.S[1], sc.S[3], sc.alpha, sc.beta, nullptr, nullptr,
             dR + (size_t)c * m, dT + (size_t)c * m, nullptr, nullptr, s.eps_in, s.eps_out,
             2.0 * 3.1415926535897932 / s.lambda, px, py, nx, ny};
  }
  {
    Prof pr(*this, "powers", 0.0, 0.0);
    stack_power_batched(upload(pd), C, m, 0, stream_);
  }
  std::vector<double> hR((size_t)C * m), hT((size_t)C * m);
  VRC_CUDA_CHECK(cudaMemcpyAsync(hR.data(), dR, hR.size() * 8, cudaMemcpyDeviceToHost, stream_));
  VRC_CUDA_CHECK(cudaMemcpyAsync(hT.data(), dT, hT.size() * 8, cudaMemcpyDeviceToHost, stream_));
  sync();
  free_bytes(dR, (size_t)C * m * 8);
  free_bytes(dT, (size_t)C * m * 8);
  for (size_t i = 0; i < ast.size() && i < reqs.size(); ++i)
    if (ast[i]) tp.status[i / (L + 2)] = ast[i];  // L layers + 2 end media per stack
  if (REF) std::memcpy(REF, hR.data(), hR.size() * 8);
  if (TRN) std::memcpy(TRN, hT.data(), hT.size() * 8);
  if (status) std::memcpy(status, tp.status.data(), C * sizeof(int));
}

void Engine::stack_backward(const double* wR, const double* wT, double* grad, double* grad_thick) {
  StackTape& tp = tape_;
  if (tp.C == 0) throw StatusError(ST_EINVAL, "stack backward: no forward solve to differentiate");
  const int C = tp.C, L = tp.L, n = tp.n, m = tp.m, npx = tp.npx, npy = tp.npy;
  Batch bt{*this, C};
  auto gather = [&](auto fn) {
    Vec v(C);
    for (int c = 0; c < C; ++c) v[c] = fn(tp.cells[c]);
    return v;
  };
  // ---- order powers -> dL/dTuu, dL/dRdu of the final blocks ----
  double* dw = (double*)bytes((size_t)2 * C * m * 8);
  VRC_CUDA_CHECK(cudaMemcpyAsync(dw, wR, (size_t)C * m * 8, cudaMemcpyHostToDevice, stream_));
  VRC_CUDA_CHECK(cudaMemcpyAsync(dw + (size_t)C * m, wT, (size_t)C * m * 8, cudaMemcpyHostToDevice, stream_));
  double* dR = (double*)bytes((size_t)2 * C * m * 8);
  Vec gTuu_n = bt.alloc(n), gRdu_n = bt.alloc(n);
  {
    std::vector<StackPowerDesc> pd(C);
    for (int c = 0; c < C; ++c) {
      StackCell& sc = tp.cells[c];
      const StackSpec& s = tp.specs[c];
      pd[c] = {sc.e0.W, sc.e0.Winv, sc.e1.W, sc.S[1], sc.S[3], sc.alpha, sc.beta, dw + (size_t)c * m,
               dw + (size_t)(C + c) * m, dR + (size_t)c * m, dR + (size_t)(C + c) * m, gRdu_n[c], gTuu_n[c],
               s.eps_in, s.eps_out, 2.0 * 3.1415926535897932 / s.lambda, tp.px, tp.py, tp.nx, tp.ny};
    }
    Prof pr(*this, "powers", 0.0, 32.0 * n * (double)n * C);
    stack_power_batched(upload(pd), C, m, 1, stream_);
  }
  // ---- reverse of the right-end projection (top adjoints: Tuu and Rdu only) ----
  Vec G[4];
  for (auto& g : G) g = bt.alloc(n);
  Vec T1 = bt.alloc(n), T2 = bt.alloc(n), T3 = bt.alloc(n);
  {
    Vec Ar = gather([](StackCell& s) { return s.Ar; });
    Vec Br = gather([](StackCell& s) { return s.Br; });
    Vec Mi = gather([](StackCell& s) { return s.Mrinv; });
    Vec S1 = gather([](StackCell& s) { return s.S[1]; });
    Vec Sc0 = gather([](StackCell& s) { return s.Sc[0]; });
    (void)Ar;
    copy(gRdu_n, G[3], n);                                       // gRdu = gRdu'
    bt.mm(T1, Br, S1, ONE, 0, 0, nullptr, ZERO, n);              // B Tuu'
    bt.mm(G[0], gRdu_n, T1, ONE, 0, 1, nullptr, ZERO, n);        // gTdd = gRdu' (B Tuu')^H
    bt.mm(T2, Sc0, Br, ONE, 0, 0, nullptr, ZERO, n);             // Tdd B
    bt.mm(T3, T2, gRdu_n, ONE, 1, 0, &gTuu_n, ONE, n);           // gTuu' + (Tdd B)^H gRdu'
    bt.mm(G[1], Mi, T3, ONE, 1, 0, nullptr, ZERO, n);            // gTuu = M^-H (...)
    bt.mm(T1, G[1], S1, MONE, 0, 1, nullptr, ZERO, n);           // gM = -gTuu Tuu'^H
    bt.mm(G[2], T1, Br, MONE, 0, 1, nullptr, ZERO, n);           // gRud = -gM B^H
  }
  bt.release(gTuu_n, n);
  bt.release(gRdu_n, n);
  double* dgrad = (double*)bytes((size_t)C * L * npx * npy * 8);
  double* dthick = (double*)bytes((size_t)C * L * 8);
  const size_t kper = pixel_adjoint_scratch(tp.nx, tp.ny);
  char* kscr = (char*)bytes((size_t)C * kper);
  Vec GP[4];
  for (auto& g : GP) g = bt.alloc(n);
  Vec gs[4];
  for (auto& g : gs) g = bt.alloc(n);
  Vec C1 = bt.alloc(n), C1r = bt.alloc(n), C2 = bt.alloc(n), X1 = bt.alloc(n), X2 = bt.alloc(n), Y = bt.alloc(n),
      Zm = bt.alloc(n), RC1 = bt.alloc(n), U = bt.alloc(n), gC1 = bt.alloc(n), gC2 = bt.alloc(n), T4 = bt.alloc(n);
  Vec g11 = bt.alloc(m), g22 = bt.alloc(m), Zq = bt.alloc(m), g33 = bt.alloc(m), Tm = bt.alloc(m);
  for (int l = L - 1; l >= 0; --l) {
    Vec pr[4], sg[4];
    for (int k = 0; k < 4; ++k) {
      pr[k] = gather([&](StackCell& s) { return s.lay[l].pre[k]; });
      sg[k] = gather([&](StackCell& s) { return s.lay[l].seg[k]; });
    }
    const Vec &Tdd = pr[0], &Tuu = pr[1], &Rud = pr[2];
    const Vec &tdd = sg[0], &tuu = sg[1], &rdu = sg[3];
    // ---- reverse of the star product (both operands) ----
    bt.mm(C1, rdu, Rud, MONE, 0, 0, nullptr, ZERO, n, nullptr, 1.0);  // I - rdu Rud
    inverse(C1, n, nullptr);
    bt.mm(C1r, C1, rdu, ONE, 0, 0, nullptr, ZERO, n);
    bt.mm(C2, Rud, C1r, ONE, 0, 0, nullptr, ZERO, n, nullptr, 1.0);   // I + Rud C1 rdu
    bt.mm(X1, Tdd, rdu, ONE, 0, 0, nullptr, ZERO, n);
    bt.mm(X2, C2, Tuu, ONE, 0, 0, nullptr, ZERO, n);
    bt.mm(Y, C1, tdd, ONE, 0, 0, nullptr, ZERO, n);
    bt.mm(Zm, Rud, Y, ONE, 0, 0, nullptr, ZERO, n);
    bt.mm(RC1, Rud, C1, ONE, 0, 0, nullptr, ZERO, n);
    const Vec &gTdd_n = G[0], &gTuu_n2 = G[1], &gRud_n2 = G[2], &gRdu_n2 = G[3];
    copy(gRdu_n2, GP[3], n);                                           // gRdu
    bt.mm(T1, gRdu_n2, X2, ONE, 0, 1, nullptr, ZERO, n);               // gX1
    bt.mm(GP[0], T1, rdu, ONE, 0, 1, nullptr, ZERO, n);                // gTdd = gX1 rdu^H
    bt.mm(gs[3], Tdd, T1, ONE, 1, 0, nullptr, ZERO, n);                // grdu = Tdd^H gX1
    bt.mm(U, X1, gRdu_n2, ONE, 1, 0, nullptr, ZERO, n);
    bt.mm(U, tuu, gTuu_n2, ONE, 1, 0, &U, ONE, n);                     // U = X1^H gRdu' + tuu^H gTuu'
    bt.mm(gC2, U, Tuu, ONE, 0, 1, nullptr, ZERO, n);                   // gC2 = U Tuu^H
    bt.mm(GP[1], C2, U, ONE, 1, 0, nullptr, ZERO, n);                  // gTuu = C2^H U
    bt.mm(gs[1], gTuu_n2, X2, ONE, 0, 1, nullptr, ZERO, n);
    bt.mm(gs[1], gRud_n2, Zm, ONE, 0, 1, &gs[1], ONE, n);              // gtuu
    copy(gRud_n2, gs[2], n);                                           // grud
    bt.mm(GP[0], gTdd_n, Y, ONE, 0, 1, &GP[0], ONE, n);                // gTdd += gTdd' Y^H
    bt.mm(T2, tuu, gRud_n2, ONE, 1, 0, nullptr, ZERO, n);              // gZ = tuu^H gRud'
    bt.mm(GP[2], T2, Y, ONE, 0, 1, nullptr, ZERO, n);                  // gRud = gZ Y^H
    bt.mm(T3, Tdd, gTdd_n, ONE, 1, 0, nullptr, ZERO, n);
    bt.mm(T3, Rud, T2, ONE, 1, 0, &T3, ONE, n);                        // gY = Tdd^H gTdd' + Rud^H gZ
    bt.mm(gC1, T3, tdd, ONE, 0, 1, nullptr, ZERO, n);                  // gC1 = gY tdd^H
    bt.mm(gs[0], C1, T3, ONE, 1, 0, nullptr, ZERO, n);                 // gtdd = C1^H gY
    bt.mm(GP[2], gC2, C1r, ONE, 0, 1, &GP[2], ONE, n);                 // gRud += gC2 (C1 rdu)^H
    bt.mm(T1, Rud, gC2, ONE, 1, 0, nullptr, ZERO, n);
    bt.mm(gC1, T1, rdu, ONE, 0, 1, &gC1, ONE, n);                      // gC1 += Rud^H gC2 rdu^H
    bt.mm(gs[3], RC1, gC2, ONE, 1, 0, &gs[3], ONE, n);                 // grdu += (Rud C1)^H gC2
    bt.mm(T1, gC1, C1, ONE, 0, 1, nullptr, ZERO, n);
    bt.mm(T4, C1, T1, MONE, 1, 0, nullptr, ZERO, n);                   // gN = -C1^H gC1 C1^H
    bt.mm(gs[3], T4, Rud, MONE, 0, 1, &gs[3], ONE, n);                 // grdu -= gN Rud^H
    bt.mm(GP[2], rdu, T4, MONE, 1, 0, &GP[2], ONE, n);                 // gRud -= rdu^H gN
    // ---- reverse of the left projection of (X, X, 0, 0) ----
    Vec A = gather([&](StackCell& s) { return s.lay[l].A; });
    Vec B = gather([&](StackCell& s) { return s.lay[l].B; });
    Vec Ai = gather([&](StackCell& s) { return s.lay[l].Ainv; });
    Vec x = gather([&](StackCell& s) { return s.lay[l].x; });
    const Vec &gtdd_n = gs[0], &gtuu_n = gs[1], &grud_n = gs[2], &grdu_n = gs[3];
    Vec& o_tdd = C1r;  // reuse as outputs of this step
    Vec& o_tuu = C2;
    Vec& o_rdu = X1;
    bt.mm(T1, B, sg[3], ONE, 0, 0, &A, ONE, n);                        // A + B rdu'
    bt.mm(o_tuu, gtuu_n, T1, ONE, 0, 1, nullptr, ZERO, n);
    bt.mm(T2, B, sg[0], ONE, 0, 0, nullptr, ZERO, n);                  // B tdd'
    bt.mm(o_tuu, grud_n, T2, ONE, 0, 1, &o_tuu, ONE, n);               // gtuu
    bt.scale(B, &x, nullptr, T3, n);                                   // X B
    bt.mm(T1, T3, gtuu_n, ONE, 1, 0, &grdu_n, ONE, n);                 // grdu' + (X B)^H gtuu'
    bt.mm(T2, T3, grud_n, ONE, 1, 0, &gtdd_n, ONE, n);                 // gtdd' + (X B)^H grud'
    bt.mm(o_tdd, Ai, T2, ONE, 1, 0, nullptr, ZERO, n);                 // gtdd = A^-H (...)
    bt.mm(Y, Ai, T1, ONE, 1, 0, nullptr, ZERO, n);                     // gY = A^-H (...)
    bt.mm(T4, o_tdd, sg[0], MONE, 0, 1, nullptr, ZERO, n);
    bt.mm(T4, Y, sg[3], MONE, 0, 1, &T4, ONE, n);                      // gM
    bt.mm(o_rdu, Y, A, ONE, 0, 1, nullptr, ZERO, n);
    bt.mm(o_rdu, T4, B, MONE, 0, 1, &o_rdu, ONE, n);                   // grdu = gY A^H - gM B^H
    // grud of the own-basis blocks is grud' itself (gs[2])
    {
      std::vector<ThickAdjDesc> td(C);
      for (int c = 0; c < C; ++c)
        td[c] = {o_tdd[c], o_tuu[c], tp.cells[c].lay[l].gam, tp.cells[c].lay[l].x, dthick + (size_t)c * L + l,
                 2.0 * 3.1415926535897932 / tp.specs[c].lambda};
      Prof pr(*this, "adjoint", 0.0, 32.0 * n * (double)C);
      thick_adjoint_batched(upload(td), C, n, stream_);
    }
    // ---- exact first-order layer kernel -> dL/dP, dL/dQ ----
    {
      std::vector<LayerAdjDesc> ld(C);
      for (int c = 0; c < C; ++c) {
        const StackSpec& s = tp.specs[c];
        ld[c] = {o_tdd[c], o_tuu[c], gs[2][c], o_rdu[c], tp.cells[c].lay[l].gam, Zm[c], RC1[c], s.thick[l],
                 2.0 * 3.1415926535897932 / s.lambda};
      }
      Prof pr(*this, "adjoint", 0.0, 96.0 * n * (double)n * C);
      layer_adjoint_batched(upload(ld), C, n, stream_);
    }
    Vec Wi = gather([&](StackCell& s) { return s.lay[l].Winv; });
    Vec Vi = gather([&](StackCell& s) { return s.lay[l].Vinv; });
    Vec W = gather([&](StackCell& s) { return s.lay[l].W; });
    Vec V = gather([&](StackCell& s) { return s.lay[l].V; });
    bt.mm(T1, Wi, Zm, ONE, 1, 0, nullptr, ZERO, n);
    bt.mm(T2, T1, V, ONE, 0, 1, nullptr, ZERO, n);                     // gP = W^-H gS V^H
    bt.mm(T1, Vi, RC1, ONE, 1, 0, nullptr, ZERO, n);
    bt.mm(T3, T1, W, ONE, 0, 1, nullptr, ZERO, n);                     // gQ = V^-H gD W^H
    // ---- Toeplitz assembly adjoint -> pixels ----
    {
      std::vector<PQAdjDesc> qd(C);
      for (int c = 0; c < C; ++c)
        qd[c] = {T2[c], T3[c], tp.cells[c].alpha, tp.cells[c].beta, g11[c], g22[c], Zq[c],
                 2.0 * 3.1415926535897932 / tp.specs[c].lambda};
      Prof pr(*this, "adjoint", 0.0, 16.0 * (2.0 * n * n + 3.0 * m * m) * C);
      pq_adjoint_batched(upload(qd), C, m, stream_);
    }
    Vec fi = gather([&](StackCell& s) { return s.lay[l].fe33inv; });
    bt.mm(Tm, Zq, fi, ONE, 0, 1, nullptr, ZERO, m);                    // Z fe33^-H
    bt.mm(g33, fi, Tm, MONE, 1, 0, nullptr, ZERO, m);                  // g33 = -fe33^-H Z fe33^-H
    {
      std::vector<PixAdjDesc> xd(C);
      for (int c = 0; c < C; ++c)
        xd[c] = {tp.cells[c].lay[l].eps, g11[c], g22[c], g33[c], dgrad + ((size_t)c * L + l) * npx * npy,
                 reinterpret_cast<cplx*>(kscr + (size_t)c * kper), tp.specs[c].Lx, tp.specs[c].Ly};
      Prof pr(*this, "adjoint", 0.0, 16.0 * (3.0 * m * m + (double)npx * npy) * C);
      pixel_adjoint_batched(upload(xd), C, tp.nx, tp.ny, npx, npy, stream_);
    }
    for (int k = 0; k < 4; ++k) std::swap(G[k], GP[k]);
  }
  std::vector<double> hg((size_t)C * L * npx * npy), ht((size_t)C * L);
  VRC_CUDA_CHECK(cudaMemcpyAsync(hg.data(), dgrad, hg.size() * 8, cudaMemcpyDeviceToHost, stream_));
  VRC_CUDA_CHECK(cudaMemcpyAsync(ht.data(), dthick, ht.size() * 8, cudaMemcpyDeviceToHost, stream_));
  sync();
  std::memcpy(grad, hg.data(), hg.size() * 8);
  if (grad_thick) std::memcpy(grad_thick, ht.data(), ht.size() * 8);
  free_bytes(dgrad, (size_t)C * L * npx * npy * 8);
  free_bytes(dthick, (size_t)C * L * 8);
  free_bytes(kscr, (size_t)C * kper);
  free_bytes(dw, (size_t)2 * C * m * 8);
  free_bytes(dR, (size_t)2 * C * m * 8);
  for (Vec* v : {&T1, &T2, &T3, &T4, &C1, &C1r, &C2, &X1, &X2, &Y, &Zm, &RC1, &U, &gC1, &gC2}) bt.release(*v, n);
  for (int k = 0; k < 4; ++k) {
    bt.release(G[k], n);
    bt.release(GP[k], n);
    bt.release(gs[k], n);
  }
  for (Vec* v : {&g11, &g22, &Zq, &g33, &Tm}) bt.release(*v, m);
}

}  // namespace vrc

namespace vrc {

// Internal amplitudes (the role of RCWASolver::evaluateIntermediateField,
// src/rcwa/RCWASolver.cpp:1373-1480) from the forward's prefix chains and
// suffix chains formed here: at interface j (0 < j < L) between the chain S_L
// of layers 0..j-1 and the rest S_R (layers j..L-1 and the exit, left end in
// the basis of layer j-1),  a+ = (I - Rud_L Rdu_R)^-1 Tuu_L c,  a- = Rdu_R a+.
void Engine::stack_fields(int ngx, int ngy, cplx* amps, cplx* img) {
  StackTape& tp = tape_;
  if (tp.C == 0) throw StatusError(ST_EINVAL, "stack fields: no forward solve");
  if (ngx < 0 || ngy < 0) throw StatusError(ST_EINVAL, "stack fields: negative grid");
  const int C = tp.C, L = tp.L, n = tp.n, m = tp.m;
  Batch bt{*this, C};
  auto gather = [&](auto fn) {
    Vec v(C);
    for (int c = 0; c < C; ++c) v[c] = fn(tp.cells[c]);
    return v;
  };
  const size_t nv = (size_t)n;
  // device vectors: per stack c, s, v, and (L+1) x (a+, a-, e)
  const size_t per = 3 * nv + (size_t)(L + 1) * 3 * nv;
  cplx* dv = (cplx*)bytes((size_t)C * per * 16);
  auto cvec = [&](int c) { return dv + c * per; };
  auto svec = [&](int c) { return dv + c * per + nv; };
  auto tvec = [&](int c) { return dv + c * per + 2 * nv; };
  auto ap = [&](int c, int j) { return dv + c * per + 3 * nv + (size_t)j * 3 * nv; };
  auto am = [&](int c, int j) { return ap(c, j) + nv; };
  auto ev = [&](int c, int j) { return ap(c, j) + 2 * nv; };
  VRC_CUDA_CHECK(cudaMemsetAsync(dv, 0, (size_t)C * per * 16, stream_));
  const size_t npix = (size_t)ngx * ngy;
  cplx* dimg = npix ? (cplx*)bytes((size_t)C * (L + 1) * 2 * npix * 16) : nullptr;
  auto matvec = [&](const std::vector<MatVecDesc>& d) {
    Prof pr(*this, "fields", 8.0 * nv * nv * d.size(), 16.0 * nv * nv * d.size());
    matvec_batched(upload(d), (int)d.size(), n, stream_);
  };
  // incidence c = W0^-1 s, s the (px, py) plane wave of the forward
  {
    const int ctr = (tp.ny * (tp.nx - 1)) / 2 + (tp.ny - 1) / 2;
    std::vector<cplx> hs((size_t)C * nv, mk(0.0, 0.0));
    for (int c = 0; c < C; ++c) {
      hs[(size_t)c * nv + ctr] = mk(tp.px, 0.0);
      hs[(size_t)c * nv + m + ctr] = mk(tp.py, 0.0);
    }
    cplx* ds = upload(hs);
    std::vector<MatVecDesc> d(C);
    for (int c = 0; c < C; ++c) {
      VRC_CUDA_CHECK(cudaMemcpyAsync(svec(c), ds + (size_t)c * nv, nv * 16, cudaMemcpyDeviceToDevice, stream_));
      d[c] = {tp.cells[c].e0.Winv, svec(c), cvec(c)};
    }
    matvec(d);
  }
  // entrance (incident, reflected) and exit (transmitted, nothing incoming)
  {
    std::vector<const cplx*> a, b;
    std::vector<cplx*> y;
    std::vector<MatVecDesc> d;
    for (int c = 0; c < C; ++c) {
      a.push_back(cvec(c));
      b.push_back(cvec(c));
      y.push_back(ap(c, 0));
      d.push_back({tp.cells[c].S[3], cvec(c), am(c, 0)});
      d.push_back({tp.cells[c].S[1], cvec(c), ap(c, L)});
    }
    vec_axpy_batched(upload(a), upload(b), mk(0.0, 0.0), upload(y), C, n, stream_);
    matvec(d);
  }
  if (L > 1) {
    // exit interface (zero thickness, left end in the last layer's basis):
    // Tuu = Ar^-1, Rud = -Ar^-1 Br, Rdu = Br Ar^-1, Tdd = Ar - Br Ar^-1 Br
    Vec Ar = gather([](StackCell& s) { return s.Ar; });
    Vec Br = gather([](StackCell& s) { return s.Br; });
    std::vector<Vec> SR(L + 1);
    for (int j = 1; j <= L; ++j) {
      SR[j].resize(4 * C);
      for (auto& p : SR[j]) p = mat(n);
    }
    auto blk = [&](int j, int k) {
      Vec v(C);
      for (int c = 0; c < C; ++c) v[c] = SR[j][4 * c + k];
      return v;
    };
    Vec Ai = blk(L, 1);
    copy(Ar, Ai, n);
    inverse(Ai, n, nullptr);
    bt.mm(blk(L, 2), Ai, Br, MONE, 0, 0, nullptr, ZERO, n);   // Rud
    bt.mm(blk(L, 3), Br, Ai, ONE, 0, 0, nullptr, ZERO, n);    // Rdu
    bt.mm(blk(L, 0), Br, blk(L, 2), ONE, 0, 0, &Ar, ONE, n);  // Tdd = Ar + Br Rud
    for (int j = L - 1; j >= 1; --j) {
      std::vector<StarReq> sr(C);
      for (int c = 0; c < C; ++c) {
        const StackLayer& ly = tp.cells[c].lay[j];
        sr[c] = {ly.seg[0], ly.seg[1], ly.seg[2], ly.seg[3], SR[j + 1][4 * c], SR[j + 1][4 * c + 1],
                 SR[j + 1][4 * c + 2], SR[j + 1][4 * c + 3], SR[j][4 * c], SR[j][4 * c + 1], SR[j][4 * c + 2],
                 SR[j][4 * c + 3]};
      }
      star(sr, n, nullptr);
    }
    Vec M = bt.alloc(n);
    for (int j = 1; j < L; ++j) {
      Vec RudL = gather([&](StackCell& s) { return s.lay[j].pre[2]; });
      Vec RduR = blk(j, 3);
      bt.mm(M, RudL, RduR, MONE, 0, 0, nullptr, ZERO, n, nullptr, 1.0);  // I - Rud_L Rdu_R
      inverse(M, n, nullptr);
      std::vector<MatVecDesc> d1(C), d2(C), d3(C);
      for (int c = 0; c < C; ++c) d1[c] = {tp.cells[c].lay[j].pre[1], cvec(c), tvec(c)};  // Tuu_L c
      matvec(d1);
      for (int c = 0; c < C; ++c) d2[c] = {M[c], tvec(c), ap(c, j)};
      matvec(d2);
      for (int c = 0; c < C; ++c) d3[c] = {RduR[c], ap(c, j), am(c, j)};
      matvec(d3);
    }
    bt.release(M, n);
    for (int j = 1; j <= L; ++j)
      for (auto* p : SR[j]) free_mat(p, n);
  }
  // transverse E harmonics and images at every interface
  {
    std::vector<IfFieldDesc> fd;
    for (int c = 0; c < C; ++c)
      for (int j = 0; j <= L; ++j) {
        const StackCell& sc = tp.cells[c];
        const cplx* W = j == 0 ? sc.e0.W : (j == L ? sc.e1.W : sc.lay[j - 1].W);
        fd.push_back({W, ap(c, j), am(c, j), ev(c, j), sc.alpha, sc.beta,
                      dimg ? dimg + ((size_t)c * (L + 1) + j) * 2 * npix : nullptr, tp.specs[c].Lx, tp.specs[c].Ly});
      }
    Prof pr(*this, "fields", 8.0 * nv * nv * fd.size(), 16.0 * (nv * nv + 2.0 * npix) * fd.size());
    interface_fields_batched(upload(fd), (int)fd.size(), n, ngx, ngy, stream_);
  }
  // copy out: amplitudes (a+, a-) per interface, then the images
  std::vector<cplx> ha((size_t)C * per);
  VRC_CUDA_CHECK(cudaMemcpyAsync(ha.data(), dv, ha.size() * 16, cudaMemcpyDeviceToHost, stream_));
  std::vector<cplx> hi(dimg ? (size_t)C * (L + 1) * 2 * npix : 0);
  if (dimg) VRC_CUDA_CHECK(cudaMemcpyAsync(hi.data(), dimg, hi.size() * 16, cudaMemcpyDeviceToHost, stream_));
  sync();
  if (amps)
    for (int c = 0; c < C; ++c)
      for (int j = 0; j <= L; ++j) {
        const cplx* src = ha.data() + c * per + 3 * nv + (size_t)j * 3 * nv;
        std::memcpy(amps + ((size_t)c * (L + 1) + j) * 2 * nv, src, 2 * nv * 16);
      }
  if (img && dimg) std::memcpy(img, hi.data(), hi.size() * 16);
  free_bytes(dv, (size_t)C * per * 16);
  if (dimg) free_bytes(dimg, (size_t)C * (L + 1) * 2 * npix * 16);
}

}  // namespace vrc
