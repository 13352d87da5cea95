// extern "C" boundary (include/vrc.h) over the engine.
#include <cstdlib>
#include "../../include/vrc.h"
#include "engine.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <string>
#include <thread>

struct vrc_context {
  std::unique_ptr<vrc::Engine> eng;
  // further engines ("lanes") that solve groups of a call's cells
  // concurrently, each with its own stream, memory pools and host thread
  std::vector<std::unique_ptr<vrc::Engine>> lanes;
  cudaEvent_t origin = nullptr;  // time origin of the profiled launch intervals
  int stack_lanes = 1;           // lanes of the last vrc_stack_forward (its tape lives there)
  std::string err;
  vrc_timing timing{0.0, 0};
  std::vector<std::vector<vrc::NodeRecord>> trees;
  // cells and accepted segmentations of the last vrc_redheffer_forward
  std::vector<vrc::CellSpec> grad_cells;
  std::vector<std::vector<double>> grad_cuts;
  std::vector<std::vector<vrc::cplx>> grad_ends;  // per cell W0, V0, gam0, W1, V1, gam1 (host)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {
using vrc::cplx;

template <class F>
int guarded(vrc_context* ctx, F&& f) {
  if (!ctx) return VRC_EINVAL;
  ctx->err.clear();
  try {
    cudaSetDevice(ctx->eng->device());
    f();
    return VRC_OK;
  } catch (const vrc::StatusError& e) {
    ctx->err = e.what;
    return e.status;
  } catch (const vrc::CudaError& e) {
    ctx->err = std::string("CUDA error: ") + cudaGetErrorString(e.err);
    return VRC_ECUDA;
  } catch (const std::bad_alloc&) {
    ctx->err = "host memory exhausted";
    return VRC_ENOMEM;
  } catch (const std::exception& e) {
    ctx->err = e.what();
    return VRC_EINVAL;
  }
}

long long all_launches(const vrc_context* ctx) {
  long long l = ctx->eng->launches;
  for (auto& e : ctx->lanes) l += e->launches;
  return l;
}

struct Timed {
  vrc_context* ctx;
  long long l0;
  explicit Timed(vrc_context* c) : ctx(c), l0(all_launches(c)) {
    VRC_CUDA_CHECK(cudaEventRecord(ctx->ev0, ctx->eng->stream()));
    c->eng->bubble_ms_ = c->eng->sync_ms_ = 0.0;
    c->eng->nsync_ = 0;
    c->eng->gap_.clear();
    c->eng->t_sync_ret_ = std::chrono::duration<double, std::milli>(
                              std::chrono::steady_clock::now().time_since_epoch()).count();
  }
  void done() {
    if (std::getenv("VRC_HOST_STATS"))
    {
      ctx->eng->sync();
      fprintf(stderr, "[vrc host] syncs %lld, blocked %.1f ms, host gaps before the next launch %.1f ms\n",
              ctx->eng->nsync_, ctx->eng->sync_ms_, ctx->eng->bubble_ms_);
      std::vector<std::pair<double, std::string>> g;
      double tot = 0.0;
      for (auto& kv : ctx->eng->gap_) {
        g.push_back({kv.second, kv.first});
        tot += kv.second;
      }
      std::sort(g.rbegin(), g.rend());
      fprintf(stderr, "[vrc host] GPU gaps between profiled families: %.1f ms total\n", tot);
      for (size_t q = 0; q < g.size() && q < 12; ++q) fprintf(stderr, "  %8.1f ms  %s\n", g[q].first, g[q].second.c_str());
      auto rep = [](const char* who, const vrc::Engine& e) {
        size_t held, out, np, ws;
        e.pool_report(&held, &out, &np, &ws);
        fprintf(stderr, "[vrc host] %s: pools %zu, held %.2f GB, handed out %.2f GB, workspace %.2f GB\n", who, np,
                held / 1e9, out / 1e9, ws / 1e9);
      };
      rep("engine", *ctx->eng);
      for (size_t q = 0; q < ctx->lanes.size(); ++q) rep("lane", *ctx->lanes[q]);
    }
    VRC_CUDA_CHECK(cudaEventRecord(ctx->ev1, ctx->eng->stream()));
    VRC_CUDA_CHECK(cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    VRC_CUDA_CHECK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->timing.device_ms = ms;
    ctx->timing.launches = all_launches(ctx) - l0;
  }
};

vrc::CellSpec to_spec(const vrc_cell& c) {
  vrc::CellSpec s;
  s.kind = c.kind;
  s.nx = c.nx;
  s.ny = c.ny;
  s.pml = c.pml != 0;
  s.lambda = c.lambda;
  s.z0 = c.z0;
  s.z1 = c.z1;
  if (c.kind == VRC_GEOM_PILLAR) {
    s.Lx = c.Lx;
    s.Ly = c.Ly;
    s.npx = c.npx;
    s.npy = c.npy;
    s.eps_in = vrc::mk(c.eps_in.re, c.eps_in.im);
    s.eps_out = vrc::mk(c.eps_out.re, c.eps_out.im);
    s.r0 = c.r0;
    s.r1 = c.r1;
    if (c.npx < 1 || c.npy < 1 || !(c.Lx > 0) || !(c.Ly > 0))
      throw vrc::StatusError(VRC_EINVAL, "invalid pillar raster");
  } else if (c.kind == VRC_GEOM_GRID || c.kind == VRC_GEOM_PIXELS) {
    if (c.ncx < 2 || c.ncy < 2 || !c.eps) throw vrc::StatusError(VRC_EINVAL, "grid needs ncx, ncy >= 2 and eps");
    if (c.x) s.x.assign(c.x, c.x + c.ncx);
    else {
      if (!(c.Lx > 0)) throw vrc::StatusError(VRC_EINVAL, "missing x coordinates");
      for (int i = 0; i < c.ncx; ++i) s.x.push_back(c.Lx * i / (c.ncx - 1));
    }
    if (c.y) s.y.assign(c.y, c.y + c.ncy);
    else {
      if (!(c.Ly > 0)) throw vrc::StatusError(VRC_EINVAL, "missing y coordinates");
      for (int j = 0; j < c.ncy; ++j) s.y.push_back(c.Ly * j / (c.ncy - 1));
    }
    size_t ne = (size_t)(c.ncx - 1) * (c.ncy - 1);
    s.eps.resize(ne);
    for (size_t i = 0; i < ne; ++i) s.eps[i] = vrc::mk(c.eps[i].re, c.eps[i].im);
    for (int axis = 0; axis < 2; ++axis) {
      const int nr = axis == 0 ? c.n_xrules : c.n_yrules;
      const vrc_rule* rs = axis == 0 ? c.xrules : c.yrules;
      for (int i = 0; i < nr; ++i) {
        const vrc_rule& r = rs[i];
        if (r.nknots < 1 || !r.zs || !r.vals || r.interp < 0 || r.interp > 1)
          throw vrc::StatusError(VRC_EINVAL, "invalid coordinate rule");
        if (r.index < 0 || r.index >= (axis == 0 ? c.ncx : c.ncy))
          throw vrc::StatusError(VRC_EINVAL, "coordinate rule index out of range");
        for (int k = 0; k + 1 < r.nknots; ++k)
          if (!(r.zs[k + 1] > r.zs[k])) throw vrc::StatusError(VRC_EINVAL, "rule knots must increase");
        vrc::PwlRule pr;
        pr.index = r.index;
        pr.zs.assign(r.zs, r.zs + r.nknots);
        pr.vals.assign(r.vals, r.vals + r.nknots);
        pr.interp = r.interp;
        pr.prepare();
        (axis == 0 ? s.xrules : s.yrules).push_back(std::move(pr));
      }
    }
    if (c.geometry_fn) {
      vrc_geometry_fn fn = c.geometry_fn;
      void* user = c.geometry_user;
      s.geom_cb = [fn, user](double z, double* x, double* y) { fn(user, z, x, y); };
    }
  } else if (c.kind == VRC_GEOM_PLANAR) {
    if (c.npoly < 1 || !c.poly_start || !c.poly_xz) throw vrc::StatusError(VRC_EINVAL, "planar cell needs polygons");
    s.pml = true;  // GDSIISampler always encloses the device in PML
    for (int p = 0; p < c.npoly; ++p) {
      const int a = c.poly_start[p], b = c.poly_start[p + 1];
      if (a < 0 || b - a < 3) throw vrc::StatusError(VRC_EINVAL, "planar polygons need >= 3 points");
      s.polys.emplace_back(c.poly_xz + 2 * (size_t)a, c.poly_xz + 2 * (size_t)b);
    }
    for (int q = 0; q < 3; ++q) s.shift[q] = c.shift[q];
    for (int q = 0; q < 4; ++q) {
      s.pml_w[q] = c.pml_w[q];
      s.space[q] = c.space[q];
    }
    s.thickness = c.thickness;
    s.eps_bg = vrc::mk(c.eps_background.re, c.eps_background.im);
    s.eps_dev = vrc::mk(c.eps_device.re, c.eps_device.im);
  } else if (c.kind == VRC_GEOM_SAMPLER) {
    if (!c.sample && !c.sample_device) throw vrc::StatusError(VRC_EINVAL, "sampler cell needs a sampler callback");
    void* user = c.sample_user;
    if (c.sample_device) {
      vrc_sample_device_fn fn = c.sample_device;
      s.dev_sample = [fn, user](double z, cplx* P, cplx* Q, cudaStream_t st) {
        return fn(user, z, reinterpret_cast<vrc_complex*>(P), reinterpret_cast<vrc_complex*>(Q),
                  static_cast<void*>(st));
      };
    } else {
      vrc_sample_fn fn = c.sample;
      s.host_sample = [fn, user](double z, cplx* P, cplx* Q) {
        return fn(user, z, reinterpret_cast<vrc_complex*>(P), reinterpret_cast<vrc_complex*>(Q));
      };
    }
    // the period (periodic half-space ends and order powers); 1 otherwise
    const double Lx = c.Lx > 0 ? c.Lx : 1.0, Ly = c.Ly > 0 ? c.Ly : 1.0;
    if ((c.has_end0 || c.has_end1) && !(c.Lx > 0 && c.Ly > 0))
      throw vrc::StatusError(VRC_EINVAL, "sampler cell with half-space ends needs the periods Lx, Ly");
    s.pml = false;
    s.x = {0.0, Lx};
    s.y = {0.0, Ly};
    s.eps = {vrc::mk(1.0, 0.0)};
  } else {
    throw vrc::StatusError(VRC_EINVAL, "unknown geometry kind");
  }
  s.has_end0 = c.has_end0 != 0;
  s.has_end1 = c.has_end1 != 0;
  s.eps_end0 = vrc::mk(c.eps_end0.re, c.eps_end0.im);
  s.eps_end1 = vrc::mk(c.eps_end1.re, c.eps_end1.im);
  return s;
}

std::vector<vrc::CellSpec> to_specs(int ncells, const vrc_cell* cells) {
  if (ncells < 0 || (ncells > 0 && !cells)) throw vrc::StatusError(VRC_EINVAL, "invalid cell array");
  std::vector<vrc::CellSpec> v;
  v.reserve(ncells);
  for (int i = 0; i < ncells; ++i) v.push_back(to_spec(cells[i]));
  return v;
}

void d2h(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (dst && src) VRC_CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
}

vrc::Engine& lane(vrc_context* ctx, int g) { return g == 0 ? *ctx->eng : *ctx->lanes[g - 1]; }

// Lanes for a call on ncells cells: three when every lane gets at least two
// cells (measured: 128 config-2 cells solve 10% faster on three lanes than
// on one, as one lane's partly filled kernel waves overlap another's work),
// else one; VRC_LANES (1..8) overrides.
int lane_count(int ncells) {
  int g = ncells >= 6 ? 3 : 1;
  if (const char* e = std::getenv("VRC_LANES")) g = std::atoi(e);
  return std::max(1, std::min({g, 8, std::max(ncells, 1)}));
}

void ensure_lanes(vrc_context* ctx, int G) {
  while ((int)ctx->lanes.size() < G - 1) {
    auto e = std::make_unique<vrc::Engine>(ctx->eng->device());
    e->set_profiling(ctx->eng->profiling());
    e->set_time_origin(ctx->origin);
    ctx->lanes.push_back(std::move(e));
  }
}

// Runs fn(g, engine of lane g) for g = 0..G-1, lanes 1.. in their own host
// threads after the call's first event on the context's stream; the
// context's stream then waits for every lane, so the call's device time spans
// all of them.  The first exception is rethrown after every lane finished
// (cleanup(g) runs on every lane first).
template <class F, class Cleanup>
void for_lanes(vrc_context* ctx, int G, F&& fn, Cleanup&& cleanup) {
  ensure_lanes(ctx, G);
  for (int g = 1; g < G; ++g) VRC_CUDA_CHECK(cudaStreamWaitEvent(lane(ctx, g).stream(), ctx->ev0, 0));
  std::vector<std::exception_ptr> err(G);
  std::vector<std::thread> th;
  const int dev = ctx->eng->device();
  for (int g = 1; g < G; ++g)
    th.emplace_back([&, g] {
      try {
        VRC_CUDA_CHECK(cudaSetDevice(dev));
        fn(g, lane(ctx, g));
      } catch (...) {
        err[g] = std::current_exception();
      }
    });
  try {
    fn(0, *ctx->eng);
  } catch (...) {
    err[0] = std::current_exception();
  }
  for (auto& t : th) t.join();
  for (int g = 0; g < G; ++g)
    if (err[g]) {
      for (int h = 0; h < G; ++h) {
        lane(ctx, h).sync();
        cleanup(h);
      }
      std::rethrow_exception(err[g]);
    }
  for (int g = 1; g < G; ++g) {
    cudaEvent_t ev;
    VRC_CUDA_CHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    VRC_CUDA_CHECK(cudaEventRecord(ev, lane(ctx, g).stream()));
    VRC_CUDA_CHECK(cudaStreamWaitEvent(ctx->eng->stream(), ev, 0));
    VRC_CUDA_CHECK(cudaEventDestroy(ev));
  }
}

// Lane of every cell of a call on G lanes.  Cells of one truncation are
// dealt round-robin.  A call mixing truncations is dealt by cost (n^3 per
// cell, longest first onto the least loaded lane), so that every lane carries
// about the same arithmetic; together with each lane starting its size
// classes at a different class (RedhefferOpts::rotate), the lanes then work
// on different truncations at the same time instead of all on the smallest.
std::vector<int> deal_lanes(const std::vector<vrc::CellSpec>& specs, int G) {
  const int C = (int)specs.size();
  std::vector<int> lane_of(C, 0);
  bool mixed = false;
  for (int k = 1; k < C; ++k) mixed |= specs[k].n() != specs[0].n();
  if (!mixed) {
    for (int k = 0; k < C; ++k) lane_of[k] = k % G;
    return lane_of;
  }
  auto cost = [&](int k) {
    const double n = specs[k].n();
    return n * n * n;
  };
  std::vector<int> order(C);
  for (int k = 0; k < C; ++k) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
  std::vector<double> load(G, 0.0);
  for (int k : order) {
    const int g = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    lane_of[k] = g;
    load[g] += cost(k);
  }
  return lane_of;
}

// Deals the cells over the lanes (deal_lanes) and runs
// solve(lane index, engine, cells, their indices in the call, results) on
// every lane.  Results come back in call order with the lane that owns each
// one (its device blocks live in that engine).
template <class F>
void run_lanes(vrc_context* ctx, const std::vector<vrc::CellSpec>& specs, std::vector<vrc::CellResult>& res,
               std::vector<int>& owner, F&& solve) {
  const int C = (int)specs.size();
  const int G = lane_count(C);
  std::vector<std::vector<vrc::CellSpec>> gs(G);
  std::vector<std::vector<int>> ids(G);
  const std::vector<int> lane_of = deal_lanes(specs, G);
  for (int c = 0; c < C; ++c) ids[lane_of[c]].push_back(c);
  for (int g = 0; g < G; ++g) {
    std::sort(ids[g].begin(), ids[g].end());  // call order inside a lane
    for (int c : ids[g]) gs[g].push_back(specs[c]);
  }
  std::vector<std::vector<vrc::CellResult>> out(G);
  for_lanes(
      ctx, G, [&](int g, vrc::Engine& E) { solve(g, E, gs[g], ids[g], out[g]); },
      [&](int g) {
        for (auto& r : out[g]) lane(ctx, g).release_result(r);
      });
  res.assign(C, vrc::CellResult());
  owner.assign(C, 0);
  for (int g = 0; g < G; ++g)
    for (size_t k = 0; k < ids[g].size(); ++k) {
      res[ids[g][k]] = out[g][k];
      owner[ids[g][k]] = g;
    }
}

// Copies the results to the caller's buffers; with ends, also every cell's
// end bases (W0, V0, gam0, W1, V1, gam1) into host vectors.
void export_results(vrc_context* ctx, std::vector<vrc::CellResult>& res, const std::vector<int>& owner,
                    vrc_result* out, std::vector<std::vector<cplx>>* ends = nullptr) {
  ctx->trees.clear();
  if (ends) ends->assign(res.size(), {});
  for (size_t c = 0; c < res.size(); ++c) {
    vrc::CellResult& r = res[c];
    vrc::Engine& E = lane(ctx, owner[c]);
    const size_t nn = (size_t)r.n * r.n * 16, nv = (size_t)r.n * 16;
    if (ends) {
      const size_t n2 = (size_t)r.n * r.n, n1 = r.n;
      std::vector<cplx>& e = (*ends)[c];
      e.resize(4 * n2 + 2 * n1);
      d2h(e.data(), r.W0, nn, E.stream());
      d2h(e.data() + n2, r.V0, nn, E.stream());
      d2h(e.data() + 2 * n2, r.gam0, nv, E.stream());
      d2h(e.data() + 2 * n2 + n1, r.W1, nn, E.stream());
      d2h(e.data() + 3 * n2 + n1, r.V1, nn, E.stream());
      d2h(e.data() + 4 * n2 + n1, r.gam1, nv, E.stream());
    }
    if (out) {
      vrc_result& o = out[c];
      d2h(o.Tdd, r.Tdd, nn, E.stream());
      d2h(o.Tuu, r.Tuu, nn, E.stream());
      d2h(o.Rud, r.Rud, nn, E.stream());
      d2h(o.Rdu, r.Rdu, nn, E.stream());
      d2h(o.W0, r.W0, nn, E.stream());
      d2h(o.V0, r.V0, nn, E.stream());
      d2h(o.gam0, r.gam0, nv, E.stream());
      d2h(o.W1, r.W1, nn, E.stream());
      d2h(o.V1, r.V1, nn, E.stream());
      d2h(o.gam1, r.gam1, nv, E.stream());
      o.status = r.status;
      o.n = r.n;
      o.N = r.N;
      o.n_eig = r.n_eig;
      o.n_samples = r.n_samples;
      o.n_nodes = r.n_nodes;
    }
    ctx->trees.push_back(r.nodes);
  }
  ctx->eng->sync();
  for (auto& e : ctx->lanes) e->sync();
  for (size_t c = 0; c < res.size(); ++c) lane(ctx, owner[c]).release_result(res[c]);
}
}  // namespace

extern "C" {

int vrc_create(int device, vrc_context** ctx) {
  if (!ctx) return VRC_EINVAL;
  *ctx = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    (void)cudaGetLastError();
    return VRC_ENODEV;
  }
  if (device < 0 || device >= ndev) return VRC_EINVAL;
  auto* c = new vrc_context();
  try {
    c->eng = std::make_unique<vrc::Engine>(device);
    VRC_CUDA_CHECK(cudaEventCreate(&c->ev0));
    VRC_CUDA_CHECK(cudaEventCreate(&c->ev1));
  } catch (...) {
    delete c;
    return VRC_ECUDA;
  }
  *ctx = c;
  return VRC_OK;
}

void vrc_destroy(vrc_context* ctx) {
  if (!ctx) return;
  if (ctx->eng) cudaSetDevice(ctx->eng->device());
  ctx->lanes.clear();
  if (ctx->origin) cudaEventDestroy(ctx->origin);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  ctx->eng.reset();
  delete ctx;
}

const char* vrc_last_error(const vrc_context* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

const char* vrc_status_string(int s) {
  switch (s) {
    case VRC_OK: return "ok";
    case VRC_EINVAL: return "invalid argument";
    case VRC_ECUDA: return "CUDA error";
    case VRC_ENOMEM: return "out of device memory";
    case VRC_ESINGULAR: return "singular matrix";
    case VRC_ENOCONV: return "eigensolver did not converge";
    case VRC_ENONFINITE: return "non-finite value";
    case VRC_ETIMEOUT: return "timeout";
    case VRC_EDEPTH: return "maximum recursion depth reached";
    case VRC_ENODEV: return "no CUDA device";
    default: return "unknown status";
  }
}

int vrc_get_timing(const vrc_context* ctx, vrc_timing* t) {
  if (!ctx || !t) return VRC_EINVAL;
  *t = ctx->timing;
  return VRC_OK;
}

int vrc_sample_pq(vrc_context* ctx, const vrc_cell* cell, int nz, const double* z, vrc_complex* P, vrc_complex* Q) {
  return guarded(ctx, [&] {
    if (!cell || nz < 0 || (nz > 0 && (!z || !P || !Q))) throw vrc::StatusError(VRC_EINVAL, "invalid arguments");
    vrc::Engine& E = *ctx->eng;
    vrc::CellSpec s = to_spec(*cell);
    const int n = s.n();
    vrc::Engine::CellDev* cd = E.prepare_cell(s);
    std::vector<cplx*> Pd(nz), Qd(nz);
    std::vector<vrc::Engine::SampleReq> req;
    for (int i = 0; i < nz; ++i) {
      Pd[i] = E.mat(n);
      Qd[i] = E.mat(n);
      req.push_back({&s, cd, z[i], false, vrc::mk(1, 0), Pd[i], Qd[i]});
    }
    Timed tm(ctx);
    std::vector<int> st;
    E.assemble(req, &st);
    tm.done();
    for (int i = 0; i < nz; ++i) {
      d2h(P + (size_t)i * n * n, Pd[i], (size_t)n * n * 16, E.stream());
      d2h(Q + (size_t)i * n * n, Qd[i], (size_t)n * n * 16, E.stream());
    }
    E.sync();
    for (int i = 0; i < nz; ++i) {
      E.free_mat(Pd[i], n);
      E.free_mat(Qd[i], n);
    }
    E.release_cell(cd);
    for (int v : st)
      if (v) throw vrc::StatusError(v, "assembly reported a singular Toeplitz / eps33 system");
  });
}

static int eig_common(vrc_context* ctx, int batch, int n, const vrc_complex* P, const vrc_complex* Q, vrc_complex* W,
                      vrc_complex* V, vrc_complex* gam, vrc_complex* lam) {
  return guarded(ctx, [&] {
    if (batch < 0 || n < 2 || n > 1024 || (batch > 0 && (!P || !W))) throw vrc::StatusError(VRC_EINVAL, "invalid arguments");
    vrc::Engine& E = *ctx->eng;
    const size_t nn = (size_t)n * n;
    std::vector<cplx*> Pd(batch), Qd(batch), Wd(batch), Vd(batch), gd(batch), ld(batch);
    std::vector<vrc::Engine::EigReq> req;
    for (int b = 0; b < batch; ++b) {
      Pd[b] = E.mat(n); Qd[b] = E.mat(n); Wd[b] = E.mat(n); Vd[b] = E.mat(n); gd[b] = E.vec(n); ld[b] = E.vec(n);
      VRC_CUDA_CHECK(cudaMemcpyAsync(Pd[b], P + (size_t)b * nn, nn * 16, cudaMemcpyHostToDevice, E.stream()));
      if (Q)
        VRC_CUDA_CHECK(cudaMemcpyAsync(Qd[b], Q + (size_t)b * nn, nn * 16, cudaMemcpyHostToDevice, E.stream()));
      // without Q the eigenpairs of P itself (no product, so no rounding)
      vrc::Engine::EigReq r{Pd[b], Q ? Qd[b] : nullptr, Wd[b], Vd[b], nullptr, nullptr, gd[b]};
      r.lam = ld[b];
      req.push_back(r);
    }
    Timed tm(ctx);
    std::vector<int> st;
    E.eig(req, n, &st);
    tm.done();
    for (int b = 0; b < batch; ++b) {
      d2h(W + (size_t)b * nn, Wd[b], nn * 16, E.stream());
      if (V) d2h(V + (size_t)b * nn, Vd[b], nn * 16, E.stream());
      if (gam) d2h(gam + (size_t)b * n, gd[b], (size_t)n * 16, E.stream());
      if (lam) d2h(lam + (size_t)b * n, ld[b], (size_t)n * 16, E.stream());
    }
    E.sync();
    for (int b = 0; b < batch; ++b) {
      E.free_mat(Pd[b], n); E.free_mat(Qd[b], n); E.free_mat(Wd[b], n); E.free_mat(Vd[b], n);
      E.free_vec(gd[b], n); E.free_vec(ld[b], n);
    }
    for (int v : st)
      if (v) throw vrc::StatusError(v, "eigensolver failure");
  });
}

int vrc_wave_solve(vrc_context* ctx, int batch, int n, const vrc_complex* P, const vrc_complex* Q, vrc_complex* W,
                   vrc_complex* V, vrc_complex* gam) {
  if (!Q) return VRC_EINVAL;
  return eig_common(ctx, batch, n, P, Q, W, V, gam, nullptr);
}

int vrc_eig(vrc_context* ctx, int batch, int n, const vrc_complex* A, vrc_complex* W, vrc_complex* lam) {
  return eig_common(ctx, batch, n, A, nullptr, W, nullptr, nullptr, lam);
}

int vrc_redheffer(vrc_context* ctx, int ncells, const vrc_cell* cells, double pe, int max_depth, vrc_result* results) {
  return guarded(ctx, [&] {
    if (!(pe > 0.0) || max_depth < 0) throw vrc::StatusError(VRC_EINVAL, "pe must be > 0 and max_depth >= 0");
    auto specs = to_specs(ncells, cells);
    vrc::Engine::RedhefferOpts o;
    o.pe = pe;
    o.max_depth = max_depth;
    std::vector<vrc::CellResult> res;
    std::vector<int> owner;
    Timed tm(ctx);
    run_lanes(ctx, specs, res, owner,
              [&](int g, vrc::Engine& E, const std::vector<vrc::CellSpec>& sp, const std::vector<int>&,
                  std::vector<vrc::CellResult>& r) {
                vrc::Engine::RedhefferOpts lo = o;
                lo.rotate = g;
                E.redheffer(sp, lo, r);
              });
    tm.done();
    export_results(ctx, res, owner, results);
  });
}

int vrc_redheffer_segments(vrc_context* ctx, int ncells, const vrc_cell* cells, const int* ncuts,
                           const double* const* cuts, vrc_result* results) {
  return guarded(ctx, [&] {
    auto specs = to_specs(ncells, cells);
    if (ncells > 0 && (!ncuts || !cuts)) throw vrc::StatusError(VRC_EINVAL, "missing cuts");
    std::vector<std::vector<double>> cv(ncells);
    for (int c = 0; c < ncells; ++c) {
      if (ncuts[c] < 2 || !cuts[c]) throw vrc::StatusError(VRC_EINVAL, "each cell needs >= 2 cut points");
      cv[c].assign(cuts[c], cuts[c] + ncuts[c]);
      for (int k = 0; k + 1 < ncuts[c]; ++k)
        if (!(cv[c][k + 1] > cv[c][k])) throw vrc::StatusError(VRC_EINVAL, "cut points must increase");
      specs[c].z0 = cv[c].front();
      specs[c].z1 = cv[c].back();
    }
    std::vector<vrc::CellResult> res;
    std::vector<int> owner;
    Timed tm(ctx);
    run_lanes(ctx, specs, res, owner,
              [&](int g, vrc::Engine& E, const std::vector<vrc::CellSpec>& sp, const std::vector<int>& ids,
                  std::vector<vrc::CellResult>& r) {
                std::vector<std::vector<double>> lc;
                for (int c : ids) lc.push_back(cv[c]);
                vrc::Engine::RedhefferOpts o;
                o.cuts = &lc;
                o.rotate = g;
                E.redheffer(sp, o, r);
              });
    tm.done();
    export_results(ctx, res, owner, results);
  });
}

int vrc_redheffer_forward(vrc_context* ctx, int ncells, const vrc_cell* cells, double pe, int max_depth,
                          vrc_result* results) {
  if (!ctx) return VRC_EINVAL;
  ctx->grad_cells.clear();
  ctx->grad_cuts.clear();
  ctx->grad_ends.clear();
  return guarded(ctx, [&] {
    if (!(pe > 0.0) || max_depth < 0) throw vrc::StatusError(VRC_EINVAL, "pe must be > 0 and max_depth >= 0");
    auto specs = to_specs(ncells, cells);
    vrc::Engine::RedhefferOpts o;
    o.pe = pe;
    o.max_depth = max_depth;
    std::vector<vrc::CellResult> res;
    std::vector<int> owner;
    Timed tm(ctx);
    run_lanes(ctx, specs, res, owner,
              [&](int g, vrc::Engine& E, const std::vector<vrc::CellSpec>& sp, const std::vector<int>&,
                  std::vector<vrc::CellResult>& r) {
                vrc::Engine::RedhefferOpts lo = o;
                lo.rotate = g;
                E.redheffer(sp, lo, r);
              });
    tm.done();
    export_results(ctx, res, owner, results, &ctx->grad_ends);
    ctx->grad_cells = std::move(specs);
    for (int c = 0; c < ncells; ++c) {
      std::vector<std::pair<double, double>> leaves;
      for (const auto& nd : ctx->trees[c])
        if (nd.accepted) leaves.push_back({nd.a, nd.b});
      std::sort(leaves.begin(), leaves.end());
      std::vector<double> cuts = {leaves.front().first};
      for (auto& l : leaves) cuts.push_back(l.second);
      ctx->grad_cuts.push_back(std::move(cuts));
    }
  });
}

int vrc_redheffer_backward(vrc_context* ctx, const vrc_complex* gS, const vrc_complex* gB, int checkpoint_every,
                           double* grad) {
  return guarded(ctx, [&] {
    if (!gS || !grad || checkpoint_every < 0) throw vrc::StatusError(VRC_EINVAL, "invalid arguments");
    const auto& cells = ctx->grad_cells;
    const int C = (int)cells.size();
    if (C == 0) throw vrc::StatusError(VRC_EINVAL, "redheffer backward: no forward solve to differentiate");
    std::vector<size_t> goff(C + 1, 0), soff(C + 1, 0);
    for (int c = 0; c < C; ++c) {
      size_t nk = 0;
      for (const auto& r : cells[c].xrules) nk += r.zs.size();
      for (const auto& r : cells[c].yrules) nk += r.zs.size();
      goff[c + 1] = goff[c] + nk;
      soff[c + 1] = soff[c] + 4 * (size_t)cells[c].n() * cells[c].n();
    }
    Timed tm(ctx);
    const int G = lane_count(C);
    const std::vector<int> lane_of = deal_lanes(cells, G);
    std::vector<std::vector<double>> out(C);
    for_lanes(
        ctx, G,
        [&](int g, vrc::Engine& E) {
          std::map<int, std::vector<int>> by_n;  // one truncation per reverse pass
          for (int c = 0; c < C; ++c)
            if (lane_of[c] == g) by_n[cells[c].n()].push_back(c);
          for (auto& kv : by_n) {
            std::vector<vrc::CellSpec> sp;
            std::vector<std::vector<double>> cu;
            std::vector<const cplx*> gs, gb, ends;
            for (int c : kv.second) {
              sp.push_back(cells[c]);
              cu.push_back(ctx->grad_cuts[c]);
              gs.push_back(reinterpret_cast<const cplx*>(gS) + soff[c]);
              gb.push_back(gB ? reinterpret_cast<const cplx*>(gB) + soff[c] : nullptr);
              ends.push_back(ctx->grad_ends[c].data());
            }
            std::vector<std::vector<double>> gr;
            E.cell_backward(sp, cu, gs, gb, ends, checkpoint_every, gr);
            for (size_t k = 0; k < kv.second.size(); ++k) out[kv.second[k]] = std::move(gr[k]);
          }
        },
        [](int) {});
    for (int c = 0; c < C; ++c) std::memcpy(grad + goff[c], out[c].data(), out[c].size() * sizeof(double));
    tm.done();
  });
}

int vrc_chain(vrc_context* ctx, int nsections, const vrc_cell* sections, int method, double pe, int max_depth,
              int nslices, vrc_result* result) {
  return guarded(ctx, [&] {
    if (nsections < 1 || !result) throw vrc::StatusError(VRC_EINVAL, "invalid arguments");
    if (method == 0 && (!(pe > 0.0) || max_depth < 0))
      throw vrc::StatusError(VRC_EINVAL, "pe must be > 0 and max_depth >= 0");
    if (method != 0 && nslices < 1) throw vrc::StatusError(VRC_EINVAL, "nslices must be >= 1");
    auto specs = to_specs(nsections, sections);
    vrc::Engine& E = *ctx->eng;
    vrc::CellResult r;
    Timed tm(ctx);
    E.chain(specs, method, pe, max_depth, nslices, r, ctx->trees);
    tm.done();
    const size_t nn = (size_t)r.n * r.n * 16, nv = (size_t)r.n * 16;
    vrc_result& o = *result;
    d2h(o.Tdd, r.Tdd, nn, E.stream());
    d2h(o.Tuu, r.Tuu, nn, E.stream());
    d2h(o.Rud, r.Rud, nn, E.stream());
    d2h(o.Rdu, r.Rdu, nn, E.stream());
    d2h(o.W0, r.W0, nn, E.stream());
    d2h(o.V0, r.V0, nn, E.stream());
    d2h(o.gam0, r.gam0, nv, E.stream());
    d2h(o.W1, r.W1, nn, E.stream());
    d2h(o.V1, r.V1, nn, E.stream());
    d2h(o.gam1, r.gam1, nv, E.stream());
    E.sync();
    o.status = r.status;
    o.n = r.n;
    o.N = r.N;
    o.n_eig = r.n_eig;
    o.n_samples = r.n_samples;
    o.n_nodes = r.n_nodes;
  });
}

int vrc_chain_order_powers(vrc_context* ctx, int side, int flux_norm, double* R, double* T) {
  return guarded(ctx, [&] {
    if (!R || !T || (side != 0 && side != 1)) throw vrc::StatusError(VRC_EINVAL, "invalid arguments");
    std::vector<double> r, t;
    ctx->eng->chain_order_powers(side, flux_norm, r, t);
    std::memcpy(R, r.data(), r.size() * sizeof(double));
    std::memcpy(T, t.data(), t.size() * sizeof(double));
  });
}

int vrc_chain_fields(vrc_context* ctx, const vrc_complex* c, int ngx, int ngy, vrc_complex* amps,
                     vrc_complex* fields) {
  return guarded(ctx, [&] {
    if (!c || !amps || ngx < 0 || ngy < 0 || ((ngx > 0) != (ngy > 0)) || (ngx > 0 && !fields))
      throw vrc::StatusError(VRC_EINVAL, "invalid arguments");
    Timed tm(ctx);
    ctx->eng->chain_fields(reinterpret_cast<const cplx*>(c), ngx, ngy, reinterpret_cast<cplx*>(amps),
                           ngx > 0 ? reinterpret_cast<cplx*>(fields) : nullptr);
    tm.done();
  });
}

int vrc_get_tree(vrc_context* ctx, int cell, int max_nodes, double* a, double* b, double* err, int* accepted) {
  if (!ctx || cell < 0 || cell >= (int)ctx->trees.size()) return -VRC_EINVAL;
  const auto& t = ctx->trees[cell];
  for (int i = 0; i < (int)t.size() && i < max_nodes; ++i) {
    if (a) a[i] = t[i].a;
    if (b) b[i] = t[i].b;
    if (err) err[i] = t[i].err;
    if (accepted) accepted[i] = t[i].accepted;
  }
  return (int)t.size();
}

int vrc_rcwa(vrc_context* ctx, int ncells, const vrc_cell* cells, int N, vrc_result* results) {
  return guarded(ctx, [&] {
    auto specs = to_specs(ncells, cells);
    std::vector<vrc::CellResult> res;
    std::vector<int> owner;
    Timed tm(ctx);
    run_lanes(ctx, specs, res, owner,
              [&](int, vrc::Engine& E, const std::vector<vrc::CellSpec>& sp, const std::vector<int>&,
                  std::vector<vrc::CellResult>& r) { E.rcwa(sp, N, r); });
    tm.done();
    export_results(ctx, res, owner, results);
  });
}

int vrc_differential(vrc_context* ctx, int ncells, const vrc_cell* cells, int N, vrc_result* results) {
  return guarded(ctx, [&] {
    auto specs = to_specs(ncells, cells);
    std::vector<vrc::CellResult> res;
    std::vector<int> owner;
    Timed tm(ctx);
    run_lanes(ctx, specs, res, owner,
              [&](int, vrc::Engine& E, const std::vector<vrc::CellSpec>& sp, const std::vector<int>&,
                  std::vector<vrc::CellResult>& r) { E.differential(sp, N, r); });
    tm.done();
    export_results(ctx, res, owner, results);
  });
}

int vrc_order_powers(vrc_context* ctx, int ncells, const vrc_cell* cells, int method, double pe, int max_depth,
                     int nslices, int side, int flux_norm, double* R, double* T, int* status) {
  return guarded(ctx, [&] {
    if (!R || !T || (side != 0 && side != 1)) throw vrc::StatusError(VRC_EINVAL, "invalid arguments");
    auto specs = to_specs(ncells, cells);
    if (method < 0 || method > 2) throw vrc::StatusError(VRC_EINVAL, "unknown method");
    if (method == 0 && !(pe > 0.0)) throw vrc::StatusError(VRC_EINVAL, "pe must be > 0");
    std::vector<vrc::CellResult> res;
    std::vector<int> owner;
    std::vector<std::vector<double>> Rv(ncells), Tv(ncells);
    Timed tm(ctx);
    run_lanes(ctx, specs, res, owner,
              [&](int g, vrc::Engine& E, const std::vector<vrc::CellSpec>& sp, const std::vector<int>& ids,
                  std::vector<vrc::CellResult>& r) {
                if (method == 0) {
                  vrc::Engine::RedhefferOpts o;
                  o.pe = pe;
                  o.max_depth = max_depth;
                  o.rotate = g;
                  E.redheffer(sp, o, r);
                } else if (method == 1) {
                  E.rcwa(sp, nslices, r);
                } else {
                  E.differential(sp, nslices, r);
                }
                std::vector<std::vector<double>> lr, lt;
                E.order_powers(sp, r, side, flux_norm, lr, lt);
                for (size_t k = 0; k < ids.size(); ++k) {
                  Rv[ids[k]] = std::move(lr[k]);
                  Tv[ids[k]] = std::move(lt[k]);
                }
              });
    tm.done();
    size_t off = 0;
    for (int c = 0; c < ncells; ++c) {
      std::memcpy(R + off, Rv[c].data(), Rv[c].size() * sizeof(double));
      std::memcpy(T + off, Tv[c].data(), Tv[c].size() * sizeof(double));
      off += Rv[c].size();
      if (status) status[c] = res[c].status;
    }
    ctx->trees.clear();
    for (int c = 0; c < ncells; ++c) {
      ctx->trees.push_back(res[c].nodes);
      lane(ctx, owner[c]).release_result(res[c]);
    }
  });
}

int vrc_stack_forward(vrc_context* ctx, int nstacks, const vrc_stack* stacks, double px, double py, double* REF,
                      double* TRN, int* status) {
  return guarded(ctx, [&] {
    if (nstacks < 1 || !stacks || !REF || !TRN) throw vrc::StatusError(VRC_EINVAL, "invalid arguments");
    std::vector<vrc::Engine::StackSpec> specs(nstacks);
    for (int c = 0; c < nstacks; ++c) {
      const vrc_stack& s = stacks[c];
      if (s.nlayers < 1 || s.npx < 1 || s.npy < 1 || !s.eps || !s.thick)
        throw vrc::StatusError(VRC_EINVAL, "stack: empty layer list or raster");
      auto& o = specs[c];
      o.nx = s.nx; o.ny = s.ny; o.npx = s.npx; o.npy = s.npy; o.L = s.nlayers;
      o.lambda = s.lam; o.Lx = s.Lx; o.Ly = s.Ly;
      o.eps.assign(s.eps, s.eps + (size_t)s.nlayers * s.npx * s.npy);
      o.thick.assign(s.thick, s.thick + s.nlayers);
      o.eps_in = vrc::mk(s.eps_in.re, s.eps_in.im);
      o.eps_out = vrc::mk(s.eps_out.re, s.eps_out.im);
    }
    Timed tm(ctx);
    // stacks dealt round-robin over the lanes; each lane keeps the tape of
    // its own stacks for vrc_stack_backward
    const int G = lane_count(nstacks);
    const int m = specs[0].nx * specs[0].ny;
    std::vector<std::vector<vrc::Engine::StackSpec>> gs(G);
    for (int c = 0; c < nstacks; ++c) gs[c % G].push_back(specs[c]);
    std::vector<std::vector<double>> lr(G), lt(G);
    std::vector<std::vector<int>> ls(G);
    ctx->stack_lanes = 1;
    for (int g = 0; g < (int)ctx->lanes.size() + 1; ++g) lane(ctx, g).release_stack_tape();
    for_lanes(
        ctx, G,
        [&](int g, vrc::Engine& E) {
          const size_t k = gs[g].size();
          lr[g].resize(k * m);
          lt[g].resize(k * m);
          ls[g].resize(k);
          E.stack_forward(gs[g], px, py, lr[g].data(), lt[g].data(), ls[g].data());
        },
        [&](int g) { lane(ctx, g).release_stack_tape(); });
    ctx->stack_lanes = G;
    for (int c = 0; c < nstacks; ++c) {
      const int g = c % G, k = c / G;
      std::memcpy(REF + (size_t)c * m, lr[g].data() + (size_t)k * m, m * sizeof(double));
      std::memcpy(TRN + (size_t)c * m, lt[g].data() + (size_t)k * m, m * sizeof(double));
      if (status) status[c] = ls[g][k];
    }
    tm.done();
  });
}

int vrc_stack_backward(vrc_context* ctx, const double* wR, const double* wT, double* grad_eps, double* grad_thick) {
  return guarded(ctx, [&] {
    if (!wR || !wT || !grad_eps) throw vrc::StatusError(VRC_EINVAL, "invalid arguments");
    const int G = ctx->stack_lanes;
    const vrc::Engine::StackTape& t0 = ctx->eng->stack_tape();
    if (t0.C == 0) throw vrc::StatusError(VRC_EINVAL, "stack backward: no forward solve to differentiate");
    const int m = t0.m;
    const size_t per = (size_t)t0.L * t0.npx * t0.npy;
    int nst = 0;
    for (int g = 0; g < G; ++g) nst += lane(ctx, g).stack_tape().C;
    Timed tm(ctx);
    std::vector<std::vector<double>> wr(G), wt(G), gr(G), gth(G);
    for (int c = 0; c < nst; ++c) {
      const int g = c % G;
      wr[g].insert(wr[g].end(), wR + (size_t)c * m, wR + (size_t)(c + 1) * m);
      wt[g].insert(wt[g].end(), wT + (size_t)c * m, wT + (size_t)(c + 1) * m);
    }
    for_lanes(
        ctx, G,
        [&](int g, vrc::Engine& E) {
          gr[g].resize((size_t)E.stack_tape().C * per);
          gth[g].resize((size_t)E.stack_tape().C * t0.L);
          E.stack_backward(wr[g].data(), wt[g].data(), gr[g].data(), gth[g].data());
        },
        [](int) {});
    for (int c = 0; c < nst; ++c) {
      std::memcpy(grad_eps + (size_t)c * per, gr[c % G].data() + (size_t)(c / G) * per, per * sizeof(double));
      if (grad_thick)
        std::memcpy(grad_thick + (size_t)c * t0.L, gth[c % G].data() + (size_t)(c / G) * t0.L,
                    t0.L * sizeof(double));
    }
    tm.done();
  });
}

int vrc_stack_fields(vrc_context* ctx, int ngx, int ngy, vrc_complex* amps, vrc_complex* fields) {
  return guarded(ctx, [&] {
    if (!amps || ngx < 0 || ngy < 0 || ((ngx > 0) != (ngy > 0)) || (ngx > 0 && !fields))
      throw vrc::StatusError(VRC_EINVAL, "invalid arguments");
    const int G = ctx->stack_lanes;
    const vrc::Engine::StackTape& t0 = ctx->eng->stack_tape();
    if (t0.C == 0) throw vrc::StatusError(VRC_EINVAL, "stack fields: no forward solve");
    const size_t pa = (size_t)(t0.L + 1) * 2 * t0.n, pi = (size_t)(t0.L + 1) * 2 * ngx * ngy;
    int nst = 0;
    for (int g = 0; g < G; ++g) nst += lane(ctx, g).stack_tape().C;
    Timed tm(ctx);
    std::vector<std::vector<cplx>> la(G), li(G);
    for_lanes(
        ctx, G,
        [&](int g, vrc::Engine& E) {
          la[g].resize((size_t)E.stack_tape().C * pa);
          li[g].resize((size_t)E.stack_tape().C * pi);
          E.stack_fields(ngx, ngy, la[g].data(), pi ? li[g].data() : nullptr);
        },
        [](int) {});
    for (int c = 0; c < nst; ++c) {
      std::memcpy(amps + (size_t)c * pa, la[c % G].data() + (size_t)(c / G) * pa, pa * 16);
      if (pi) std::memcpy(fields + (size_t)c * pi, li[c % G].data() + (size_t)(c / G) * pi, pi * 16);
    }
    tm.done();
  });
}

int vrc_gds_read(const char* path, double unit, int* npoly, int* npoints, int* poly_start, double* poly_xz,
                 int max_poly, int max_points) {
  if (!path || !npoly || !npoints || !(unit > 0.0)) return VRC_EINVAL;
  try {
    double dbu = 0.0;
    auto polys = vrc::gds_read_polygons(path, unit, &dbu);
    int tot = 0;
    for (auto& p : polys) tot += (int)(p.size() / 2);
    *npoly = (int)polys.size();
    *npoints = tot;
    if (!poly_start && !poly_xz) return VRC_OK;
    if (!poly_start || !poly_xz || max_poly < *npoly || max_points < tot) return VRC_EINVAL;
    int off = 0;
    for (size_t p = 0; p < polys.size(); ++p) {
      poly_start[p] = off;
      std::memcpy(poly_xz + 2 * (size_t)off, polys[p].data(), polys[p].size() * sizeof(double));
      off += (int)(polys[p].size() / 2);
    }
    poly_start[polys.size()] = off;
    return VRC_OK;
  } catch (const vrc::StatusError& e) {
    return e.status;
  } catch (...) {
    return VRC_EINVAL;
  }
}

int vrc_planar_section(const vrc_cell* cell, double z, int max_x, double* x, double* y, vrc_complex* eps) {
  if (!cell || cell->kind != VRC_GEOM_PLANAR) return -VRC_EINVAL;
  try {
    vrc::CellSpec s = to_spec(*cell);
    std::vector<double> xs, ys;
    std::vector<cplx> es;
    s.planar_section(z, xs, ys, &es);
    const int nxs = (int)xs.size();
    if (x && y && eps) {
      if (max_x < nxs) return -VRC_EINVAL;
      std::memcpy(x, xs.data(), nxs * sizeof(double));
      std::memcpy(y, ys.data(), ys.size() * sizeof(double));
      for (size_t i = 0; i < es.size(); ++i) eps[i] = {es[i].x, es[i].y};
    }
    return nxs;
  } catch (const vrc::StatusError& e) {
    return -e.status;
  } catch (...) {
    return -VRC_EINVAL;
  }
}

int vrc_set_profiling(vrc_context* ctx, int enable) {
  return guarded(ctx, [&] {
    ctx->eng->set_profiling(enable != 0);
    ctx->eng->reset_fam_stats();
    for (auto& e : ctx->lanes) {
      e->set_profiling(enable != 0);
      e->reset_fam_stats();
    }
    if (!ctx->origin) VRC_CUDA_CHECK(cudaEventCreate(&ctx->origin));
    VRC_CUDA_CHECK(cudaEventRecord(ctx->origin, ctx->eng->stream()));
    ctx->eng->set_time_origin(ctx->origin);
    for (auto& e : ctx->lanes) {
      VRC_CUDA_CHECK(cudaStreamWaitEvent(e->stream(), ctx->origin, 0));
      e->set_time_origin(ctx->origin);
    }
  });
}

int vrc_get_kernel_stats(vrc_context* ctx, int max, vrc_kernel_stat* out) {
  if (!ctx) return -VRC_EINVAL;
  int count = 0;
  int st = guarded(ctx, [&] {
    // summed over the lanes: with concurrent lanes a family's time is the
    // sum of its launches' durations, each measured on its own stream
    std::map<std::string, vrc::Engine::FamStat> f = ctx->eng->fam_stats();
    // "~busy ...": the union of every family's launch intervals, on all
    // engines and on each one (GPU time with at least one kernel running)
    auto& all = f["~busy all"];
    for (auto& kv : f)
      if (kv.first[0] != '~') all.iv.insert(all.iv.end(), kv.second.iv.begin(), kv.second.iv.end());
    for (size_t q = 0; q < ctx->lanes.size(); ++q) {
      auto& mine = f["~busy lane " + std::to_string(q)];
      for (auto& kv : ctx->lanes[q]->fam_stats()) {
        auto& d = f[kv.first];
        d.ms += kv.second.ms;
        d.launches += kv.second.launches;
        d.flops += kv.second.flops;
        d.bytes += kv.second.bytes;
        d.iv.insert(d.iv.end(), kv.second.iv.begin(), kv.second.iv.end());
        all.iv.insert(all.iv.end(), kv.second.iv.begin(), kv.second.iv.end());
        mine.iv.insert(mine.iv.end(), kv.second.iv.begin(), kv.second.iv.end());
      }
    }
    for (auto& kv : f) {
      if (out && count < max) {
        vrc_kernel_stat& o = out[count];
        std::memset(o.name, 0, sizeof(o.name));
        std::strncpy(o.name, kv.first.c_str(), sizeof(o.name) - 1);
        o.ms = kv.second.ms;
        o.launches = kv.second.launches;
        o.flops = kv.second.flops;
        o.bytes = kv.second.bytes;
        auto iv = kv.second.iv;  // union of the launch intervals
        std::sort(iv.begin(), iv.end());
        double busy = 0.0, s0 = 0.0, s1 = -1.0;
        for (auto& p : iv) {
          if (p.first > s1) {
            if (s1 > s0) busy += s1 - s0;
            s0 = p.first;
            s1 = p.second;
          } else if (p.second > s1) {
            s1 = p.second;
          }
        }
        if (s1 > s0) busy += s1 - s0;
        o.busy_ms = iv.empty() ? kv.second.ms : busy;
      }
      ++count;
    }
  });
  return st == VRC_OK ? count : -st;
}

int vrc_zgemm(vrc_context* ctx, int batch, int n, const vrc_complex* A, const vrc_complex* B, vrc_complex* C) {
  return guarded(ctx, [&] {
    if (batch < 0 || n < 1 || (batch > 0 && (!A || !B || !C))) throw vrc::StatusError(VRC_EINVAL, "invalid arguments");
    vrc::Engine& E = *ctx->eng;
    const size_t nn = (size_t)n * n;
    std::vector<vrc::GemmDesc> g;
    std::vector<cplx*> bufs;
    for (int b = 0; b < batch; ++b) {
      cplx *a = E.mat(n), *bb = E.mat(n), *c = E.mat(n);
      bufs.insert(bufs.end(), {a, bb, c});
      VRC_CUDA_CHECK(cudaMemcpyAsync(a, A + b * nn, nn * 16, cudaMemcpyHostToDevice, E.stream()));
      VRC_CUDA_CHECK(cudaMemcpyAsync(bb, B + b * nn, nn * 16, cudaMemcpyHostToDevice, E.stream()));
      g.push_back({a, bb, c, nullptr, nullptr, nullptr});
    }
    Timed tm(ctx);
    E.gemm(g, n, vrc::mk(1, 0), vrc::mk(0, 0), 0.0);
    tm.done();
    for (int b = 0; b < batch; ++b) d2h(C + b * nn, g[b].C, nn * 16, E.stream());
    E.sync();
    for (auto* p : bufs) E.free_mat(p, n);
  });
}

int vrc_zinv(vrc_context* ctx, int batch, int n, vrc_complex* A, int* status) {
  return guarded(ctx, [&] {
    if (batch < 0 || n < 1 || (batch > 0 && !A)) throw vrc::StatusError(VRC_EINVAL, "invalid arguments");
    vrc::Engine& E = *ctx->eng;
    const size_t nn = (size_t)n * n;
    std::vector<cplx*> m(batch);
    for (int b = 0; b < batch; ++b) {
      m[b] = E.mat(n);
      VRC_CUDA_CHECK(cudaMemcpyAsync(m[b], A + b * nn, nn * 16, cudaMemcpyHostToDevice, E.stream()));
    }
    std::vector<int> st;
    Timed tm(ctx);
    E.inverse(m, n, &st);
    tm.done();
    for (int b = 0; b < batch; ++b) d2h(A + b * nn, m[b], nn * 16, E.stream());
    E.sync();
    for (int b = 0; b < batch; ++b) {
      E.free_mat(m[b], n);
      if (status) status[b] = b < (int)st.size() ? st[b] : 0;
    }
  });
}

}  // extern "C"
