/*
 * vrc_integrators.hpp -- the reference's integrator classes over the C ABI
 * of vrc.h, header-only C++17.
 *
 * Drop-in counterparts, with the reference's constructors, compute() and
 * accessors, of
 *   RedhefferIntegrator(z0, z1, std::shared_ptr<LayerSampler>)
 *       ::compute(int p, int maxN = 10, scalar pe = 1e-2), N(), nEigVal()
 *       (src/core/RedhefferIntegrator.h:34-50),
 *   RCWAIntegrator(z0, z1, sampler)::compute(int N)
 *       (src/core/RCWAIntegrator.h:25-38),
 *   DifferentialIntegrator(z0, z1, sampler)::compute(int N)
 *       (src/core/DifferentialIntegrator.h:25-38),
 * each with Tdd() Tuu() Rud() Rdu() W0() V0() gam0() W1() V1() gam1().
 *
 * They are templates over the sampler and matrix types so that they need no
 * particular linear-algebra library:
 *   Sampler  int nDim() const; double lambda() const;
 *            void sample(double z, Matrix& P, Matrix& Q);          (host)
 *            void sampleOnGPU(double z, T* P, T* Q);  (SampleOn::Device only;
 *            T any 16-byte complex type, e.g. cuDoubleComplex)
 *   Matrix   resize(rows, cols); data() -> std::complex<double>*, column-major
 *   Vector   resize(n); data() -> std::complex<double>*
 * The reference's LayerSampler with Eigen::MatrixXcs / Eigen::VectorXcs
 * satisfies these, so in the reference's code base
 *   using RedhefferIntegrator =
 *       vrc_cxx::RedhefferIntegrator<LayerSampler, Eigen::MatrixXcs, Eigen::VectorXcs>;
 * replaces the CPU and GPU integrators without touching their callers.
 *
 * The engine calls the sampler for every z it needs: sample() fills host
 * matrices that the engine copies to the device; sampleOnGPU() writes the
 * engine's device buffers, after which the shim waits for the device (the
 * reference's sampleOnGPU names no stream).  Errors (a status other than
 * VRC_OK) throw vrc_cxx::Error; the reference printed them and continued.
 */
#ifndef VRC_INTEGRATORS_HPP_
#define VRC_INTEGRATORS_HPP_

#include <cuda_runtime.h>

#include <complex>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>

#include "vrc.h"

namespace vrc_cxx {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& what) : std::runtime_error(what), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

inline void check(const vrc_context* ctx, int st) {
  if (st != VRC_OK)
    throw Error(st, std::string(vrc_status_string(st)) + ": " + (ctx ? vrc_last_error(ctx) : ""));
}

/* One context per device, created on first use and shared by every
 * integrator of the process (a context holds the engine's streams and
 * memory pools).  It lives until the process exits. */
inline vrc_context* default_context(int device = 0) {
  static std::mutex mu;
  static std::map<int, vrc_context*> ctxs;
  std::lock_guard<std::mutex> lock(mu);
  vrc_context*& c = ctxs[device];
  if (!c) check(nullptr, vrc_create(device, &c));
  return c;
}

enum class SampleOn { Host, Device };

namespace detail {
template <class C, class R, class T, class S>
void call_gpu(S& s, double z, void* P, void* Q, R (C::*f)(double, T*, T*)) {
  (s.*f)(z, static_cast<T*>(P), static_cast<T*>(Q));
}
}  // namespace detail

template <class Sampler, class Matrix, class Vector>
class IntegratorBase {
 public:
  const Matrix& Tdd() const { return Tdd_; }
  const Matrix& Tuu() const { return Tuu_; }
  const Matrix& Rud() const { return Rud_; }
  const Matrix& Rdu() const { return Rdu_; }
  const Matrix& W0() const { return W0_; }
  const Matrix& V0() const { return V0_; }
  const Vector& gam0() const { return gam0_; }
  const Matrix& W1() const { return W1_; }
  const Matrix& V1() const { return V1_; }
  const Vector& gam1() const { return gam1_; }
  vrc_context* context() const { return ctx_; }

 protected:
  IntegratorBase(double z0, double z1, std::shared_ptr<Sampler> sampler, SampleOn on, vrc_context* ctx)
      : z0_(z0), z1_(z1), sampler_(std::move(sampler)), on_(on), ctx_(ctx ? ctx : default_context()) {
    if (!sampler_) throw Error(VRC_EINVAL, "null sampler");
  }

  // The structure as a caller-sampler cell: only nDim and lambda matter.
  vrc_cell cell() const {
    vrc_cell c;
    std::memset(&c, 0, sizeof(c));
    c.kind = VRC_GEOM_SAMPLER;
    c.nx = sampler_->nDim() / 2;
    c.ny = 1;
    c.lambda = sampler_->lambda();
    c.z0 = z0_;
    c.z1 = z1_;
    if (on_ == SampleOn::Device) c.sample_device = &device_cb;
    else c.sample = &host_cb;
    c.sample_user = sampler_.get();
    return c;
  }

  // Result struct pointing into the accessors' storage (resized to n).
  vrc_result outputs() {
    const int n = sampler_->nDim();
    for (Matrix* m : {&Tdd_, &Tuu_, &Rud_, &Rdu_, &W0_, &V0_, &W1_, &V1_}) m->resize(n, n);
    gam0_.resize(n);
    gam1_.resize(n);
    vrc_result r;
    std::memset(&r, 0, sizeof(r));
    auto p = [](auto& m) { return reinterpret_cast<vrc_complex*>(m.data()); };
    r.Tdd = p(Tdd_);
    r.Tuu = p(Tuu_);
    r.Rud = p(Rud_);
    r.Rdu = p(Rdu_);
    r.W0 = p(W0_);
    r.V0 = p(V0_);
    r.gam0 = p(gam0_);
    r.W1 = p(W1_);
    r.V1 = p(V1_);
    r.gam1 = p(gam1_);
    return r;
  }

  static int host_cb(void* user, double z, vrc_complex* P, vrc_complex* Q) {
    try {
      Sampler& s = *static_cast<Sampler*>(user);
      const int n = s.nDim();
      Matrix Pm, Qm;
      s.sample(z, Pm, Qm);
      std::memcpy(P, Pm.data(), sizeof(vrc_complex) * n * n);
      std::memcpy(Q, Qm.data(), sizeof(vrc_complex) * n * n);
      return 0;
    } catch (...) {
      return 1;
    }
  }

  static int device_cb(void* user, double z, vrc_complex* P, vrc_complex* Q, void*) {
    try {
      Sampler& s = *static_cast<Sampler*>(user);
      detail::call_gpu(s, z, P, Q, &Sampler::sampleOnGPU);
      return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
    } catch (...) {
      return 1;
    }
  }

  double z0_, z1_;
  std::shared_ptr<Sampler> sampler_;
  SampleOn on_;
  vrc_context* ctx_;
  Matrix Tdd_, Tuu_, Rud_, Rdu_, W0_, V0_, W1_, V1_;
  Vector gam0_, gam1_;
};

/* RedhefferIntegrator(z0, z1, sampler).compute(p, maxN, pe): adaptive
 * varRCWA (trisection, accept when the perturbation's max-norm <= pe).  As
 * in the reference, p and maxN are accepted and unused. */
template <class Sampler, class Matrix, class Vector>
class RedhefferIntegrator : public IntegratorBase<Sampler, Matrix, Vector> {
  using Base = IntegratorBase<Sampler, Matrix, Vector>;

 public:
  RedhefferIntegrator(double z0, double z1, std::shared_ptr<Sampler> sampler, SampleOn on = SampleOn::Host,
                      vrc_context* ctx = nullptr)
      : Base(z0, z1, std::move(sampler), on, ctx) {}

  void compute(int /*p*/, int /*maxN*/ = 10, double pe = 1e-2) {
    vrc_cell c = this->cell();
    vrc_result r = this->outputs();
    check(this->ctx_, vrc_redheffer(this->ctx_, 1, &c, pe, 40, &r));
    check(this->ctx_, r.status);
    N_ = r.N;
    nEigVal_ = r.n_eig;
  }
  int N() const { return N_; }
  int nEigVal() const { return nEigVal_; }

 private:
  int N_ = 0, nEigVal_ = 0;
};

/* RCWAIntegrator(z0, z1, sampler).compute(N): N midpoint slabs. */
template <class Sampler, class Matrix, class Vector>
class RCWAIntegrator : public IntegratorBase<Sampler, Matrix, Vector> {
  using Base = IntegratorBase<Sampler, Matrix, Vector>;

 public:
  RCWAIntegrator(double z0, double z1, std::shared_ptr<Sampler> sampler, SampleOn on = SampleOn::Host,
                 vrc_context* ctx = nullptr)
      : Base(z0, z1, std::move(sampler), on, ctx) {}

  void compute(int N = 10) {
    vrc_cell c = this->cell();
    vrc_result r = this->outputs();
    check(this->ctx_, vrc_rcwa(this->ctx_, 1, &c, N, &r));
    check(this->ctx_, r.status);
  }
};

/* DifferentialIntegrator(z0, z1, sampler).compute(N): N second-order
 * differential-method slices. */
template <class Sampler, class Matrix, class Vector>
class DifferentialIntegrator : public IntegratorBase<Sampler, Matrix, Vector> {
  using Base = IntegratorBase<Sampler, Matrix, Vector>;

 public:
  DifferentialIntegrator(double z0, double z1, std::shared_ptr<Sampler> sampler, SampleOn on = SampleOn::Host,
                         vrc_context* ctx = nullptr)
      : Base(z0, z1, std::move(sampler), on, ctx) {}

  void compute(int N = 10) {
    vrc_cell c = this->cell();
    vrc_result r = this->outputs();
    check(this->ctx_, vrc_differential(this->ctx_, 1, &c, N, &r));
    check(this->ctx_, r.status);
  }
};

}  // namespace vrc_cxx

#endif  // VRC_INTEGRATORS_HPP_
