// Batched-GEMM helper shared by the adjoint drivers (layer stacks and
// adaptive cells): one entry per solve of a call, C = alpha op(A) op(B)
// (+ beta Cin) on the tensor-core GEMM, plus pool allocation of per-solve
// matrices and diagonal scalings.
#pragma once

#include <vector>

#include "engine.h"

namespace vrc {

using Vec = std::vector<cplx*>;

constexpr cplx C_ONE{1.0, 0.0}, C_ZERO{0.0, 0.0}, C_MONE{-1.0, 0.0}, C_HALF{0.5, 0.0}, C_MHALF{-0.5, 0.0};

struct Batch {
  Engine& e;
  int C;
  void mm(const Vec& Cm, const Vec& A, const Vec& B, cplx alpha = C_ONE, int oa = 0, int ob = 0,
          const Vec* Cin = nullptr, cplx beta = C_ZERO, int n = 0, const Vec* rs = nullptr, double delta = 0.0) {
    if (n <= 0) throw StatusError(ST_EINVAL, "batched GEMM without an order");
    std::vector<GemmDesc> d(C);
    for (int c = 0; c < C; ++c)
      d[c] = {A[c], B[c], Cm[c], Cin ? (*Cin)[c] : nullptr, rs ? (*rs)[c] : nullptr, nullptr};
    e.gemm(d, n, alpha, beta, delta, oa, ob);
  }
  Vec alloc(int n) {
    Vec v(C);
    for (auto& p : v) p = e.mat(n);
    return v;
  }
  void release(Vec& v, int n) {
    for (auto& p : v) e.free_mat(p, n);
    v.clear();
  }
  void scale(const Vec& A, const Vec* rs, const Vec* cs, const Vec& out, int n) {
    std::vector<const cplx*> a(A.begin(), A.end()), r(C, nullptr), s(C, nullptr);
    if (rs) r.assign(rs->begin(), rs->end());
    if (cs) s.assign(cs->begin(), cs->end());
    Engine::Prof pr(e, "adjoint", 0.0, 32.0 * n * (double)n * C);
    scale_batched(e.upload(a), rs ? e.upload(r) : nullptr, cs ? e.upload(s) : nullptr, e.upload(out), C, n,
                  e.stream());
  }
};

}  // namespace vrc
