// A C++ caller of the library through the reference-shaped integrator
// classes of include/vrc_integrators.hpp (no Eigen: a minimal column-major
// matrix type stands in for Eigen::MatrixXcs).
//
// The structure is a caller-defined sampler, as a LayerSampler subclass of
// the reference would be: P(z) = P0 + (z - za) / (zb - za) * (P1 - P0) and
// likewise Q, from four n x n matrices read from the input file.  Usage:
//   shim_check <input> <output> host|device <pe> <N_rcwa> <N_diff>
// Input (little-endian): int32 n, float64 lambda, za, zb, z0, z1, then P0,
// P1, Q0, Q1 (n*n complex128 each, column-major).  Output: for the
// RedhefferIntegrator (with N(), nEigVal() and its tree's cuts), the
// RCWAIntegrator and the DifferentialIntegrator in turn: Tdd, Tuu, Rud, Rdu,
// W0, W1 (n*n complex128 each).
#include <algorithm>
#include <complex>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "vrc_integrators.hpp"

using cd = std::complex<double>;

struct Mat {
  int r = 0, c = 0;
  std::vector<cd> v;
  void resize(int rows, int cols) {
    r = rows;
    c = cols;
    v.assign((size_t)rows * cols, cd(0.0, 0.0));
  }
  void resize(int n) { resize(n, 1); }
  cd* data() { return v.data(); }
  const cd* data() const { return v.data(); }
};

struct LinearSampler {
  int n = 0;
  double lam = 1.0, za = 0.0, zb = 1.0;
  std::vector<cd> P0, P1, Q0, Q1;
  int nDim() const { return n; }
  double lambda() const { return lam; }
  void fill(double z, cd* P, cd* Q) const {
    const double t = (z - za) / (zb - za);
    for (size_t i = 0; i < P0.size(); ++i) {
      P[i] = P0[i] + t * (P1[i] - P0[i]);
      Q[i] = Q0[i] + t * (Q1[i] - Q0[i]);
    }
  }
  void sample(double z, Mat& P, Mat& Q) {
    P.resize(n, n);
    Q.resize(n, n);
    fill(z, P.data(), Q.data());
  }
  // the reference's sampleOnGPU: device buffers preallocated by the caller
  void sampleOnGPU(double z, double2* P, double2* Q) {
    std::vector<cd> hp((size_t)n * n), hq((size_t)n * n);
    fill(z, hp.data(), hq.data());
    if (cudaMemcpy(P, hp.data(), hp.size() * sizeof(cd), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(Q, hq.data(), hq.size() * sizeof(cd), cudaMemcpyHostToDevice) != cudaSuccess)
      throw std::runtime_error("sampleOnGPU copy failed");
  }
};

template <class I>
void dump(std::ofstream& out, const I& it) {
  for (const Mat* m : {&it.Tdd(), &it.Tuu(), &it.Rud(), &it.Rdu(), &it.W0(), &it.W1()})
    out.write(reinterpret_cast<const char*>(m->data()), m->v.size() * sizeof(cd));
}

int main(int argc, char** argv) {
  if (argc != 7) {
    std::cerr << "usage: shim_check <input> <output> host|device <pe> <N_rcwa> <N_diff>\n";
    return 2;
  }
  auto s = std::make_shared<LinearSampler>();
  std::ifstream in(argv[1], std::ios::binary);
  int32_t n = 0;
  double hdr[5];
  in.read(reinterpret_cast<char*>(&n), 4);
  in.read(reinterpret_cast<char*>(hdr), sizeof(hdr));
  s->n = n;
  s->lam = hdr[0];
  s->za = hdr[1];
  s->zb = hdr[2];
  const double z0 = hdr[3], z1 = hdr[4];
  for (auto* m : {&s->P0, &s->P1, &s->Q0, &s->Q1}) {
    m->resize((size_t)n * n);
    in.read(reinterpret_cast<char*>(m->data()), m->size() * sizeof(cd));
  }
  if (!in) {
    std::cerr << "short input\n";
    return 2;
  }
  const auto on = std::string(argv[3]) == "device" ? vrc_cxx::SampleOn::Device : vrc_cxx::SampleOn::Host;
  const double pe = std::stod(argv[4]);
  const int nr = std::stoi(argv[5]), nd = std::stoi(argv[6]);
  try {
    std::ofstream out(argv[2], std::ios::binary);
    vrc_cxx::RedhefferIntegrator<LinearSampler, Mat, Mat> red(z0, z1, s, on);
    red.compute(0, 1000000, pe);  // p and maxN as the reference's drivers pass them
    const int32_t counts[2] = {red.N(), red.nEigVal()};
    out.write(reinterpret_cast<const char*>(counts), sizeof(counts));
    const int nodes = vrc_get_tree(red.context(), 0, 0, nullptr, nullptr, nullptr, nullptr);
    std::vector<double> a(nodes), b(nodes), err(nodes);
    std::vector<int> acc(nodes);
    vrc_get_tree(red.context(), 0, nodes, a.data(), b.data(), err.data(), acc.data());
    std::vector<std::pair<double, double>> leaves;
    for (int k = 0; k < nodes; ++k)
      if (acc[k]) leaves.push_back({a[k], b[k]});
    std::sort(leaves.begin(), leaves.end());
    std::vector<double> cuts = {leaves.front().first};
    for (auto& l : leaves) cuts.push_back(l.second);
    const int32_t ncut = (int32_t)cuts.size();
    out.write(reinterpret_cast<const char*>(&ncut), 4);
    out.write(reinterpret_cast<const char*>(cuts.data()), cuts.size() * sizeof(double));
    dump(out, red);
    vrc_cxx::RCWAIntegrator<LinearSampler, Mat, Mat> rc(z0, z1, s, on);
    rc.compute(nr);
    dump(out, rc);
    vrc_cxx::DifferentialIntegrator<LinearSampler, Mat, Mat> df(z0, z1, s, on);
    df.compute(nd);
    dump(out, df);
  } catch (const vrc_cxx::Error& e) {
    std::cerr << "vrc error " << e.status() << ": " << e.what() << "\n";
    return 1;
  }
  std::printf("ok\n");
  return 0;
}
