// Eigen-decomposition entry point that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: applications that own
// every byte of device memory through their own pool (a library allocation
// would bypass their accounting and limits), and pipelines that must not
// stall, since cudaMalloc/cudaFree synchronise the device.  For them
// vrc_eig_noalloc runs the same eigensolver kernels as vrc_eig on one
// n x n matrix (n <= VRC_EIG_NOALLOC_MAX_N) with the caller's device buffers
// and a fixed scratch area that is part of the library image: a file-scope
// __device__ array holding three 256 x 256 complex128 work matrices and the
// QR rotation log (about 22 MiB on every GPU that loads the library, held
// until exit).
//
// The scratch is shared by every call in the process on that device and
// keeps the last call's contents; the entry point overwrites or clears all
// of it that a call reads.  Calls that overlap on the GPU (other streams or
// threads on the same device) race on the scratch and must be serialised by
// the caller.  The first call on a device looks up the scratch address
// (cudaGetSymbolAddress); make that first call before any stream capture.
// Every call blocks the calling host thread until `stream` has drained (it
// reads the convergence flag back); other streams keep running.
#include "../../include/vrc.h"
#include "common.cuh"
#include "kernels.h"

#include <cstdio>
#include <exception>
#include <new>
#include <map>
#include <mutex>

namespace {
using vrc::cplx;

constexpr int kMaxN = VRC_EIG_NOALLOC_MAX_N;
constexpr size_t kMat = (size_t)kMaxN * kMaxN * sizeof(cplx);
// scratch layout (byte offsets)
constexpr size_t kOffH = 0;
constexpr size_t kOffZ = kOffH + kMat;
constexpr size_t kOffY = kOffZ + kMat;
constexpr size_t kOffPtr = kOffY + kMat;          // 8 pointers
constexpr size_t kOffDesc = kOffPtr + 8 * sizeof(void*);
constexpr size_t kOffStatus = kOffDesc + 256;     // one int
constexpr size_t kOffLog = kOffStatus + 256;      // QR rotation log
// log capacity for n = kMaxN: 64-byte header, sweep records of 32 bytes
// (bounded here by half the rotation capacity + 256, more than the iteration
// cap allows) and 6n^2+64 rotations of 32 bytes (checked against
// schur_log_bytes at run time)
constexpr size_t kRotCap = (size_t)6 * kMaxN * kMaxN + 64;
constexpr size_t kLogBytes = (64 + (kRotCap / 2 + 256) * 32 + kRotCap * 32 + 255) / 256 * 256;
constexpr size_t kScratchBytes = kOffLog + kLogBytes;

static __device__ __align__(256) unsigned char g_eig_scratch[kScratchBytes];

// Writes the pointer arrays and the GEMM descriptor the batched launchers
// read (a batch of one), so no host-to-device copy of descriptors is needed.
__global__ void noalloc_setup_kernel(cplx* W, cplx* lam) {
  unsigned char* base = g_eig_scratch;
  cplx** p = reinterpret_cast<cplx**>(base + kOffPtr);
  p[0] = reinterpret_cast<cplx*>(base + kOffH);
  p[1] = reinterpret_cast<cplx*>(base + kOffZ);
  p[2] = reinterpret_cast<cplx*>(base + kOffY);
  p[3] = lam;
  p[4] = W;
  p[5] = reinterpret_cast<cplx*>(base + kOffLog);
  vrc::GemmDesc* d = reinterpret_cast<vrc::GemmDesc*>(base + kOffDesc);
  d->A = p[1];
  d->B = p[2];
  d->C = W;
  d->Cin = nullptr;
  d->rs = nullptr;
  d->cs = nullptr;
}

std::mutex g_mu;
std::map<int, unsigned char*> g_base;  // device ordinal -> scratch address

unsigned char* scratch_address(int dev) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_base.find(dev);
  if (it != g_base.end()) return it->second;
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_eig_scratch) != cudaSuccess || p == nullptr) {
    (void)cudaGetLastError();
    return nullptr;
  }
  g_base[dev] = static_cast<unsigned char*>(p);
  return g_base[dev];
}
}  // namespace

extern "C" int vrc_eig_noalloc(int n, const vrc_complex* A, vrc_complex* W, vrc_complex* lam, void* stream) {
  if (n < 2 || n > kMaxN) {
    fprintf(stderr, "vrc_eig_noalloc: n = %d is outside [2, %d]\n", n, kMaxN);
    return VRC_EINVAL;
  }
  if (!A || !W || !lam) {
    fprintf(stderr, "vrc_eig_noalloc: A, W and lam must be device pointers\n");
    return VRC_EINVAL;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return VRC_ENODEV;
  }
  unsigned char* base = nullptr;
  try {
    base = scratch_address(dev);  // host map insert and mutex: may throw
  } catch (const std::bad_alloc&) {
    return VRC_ENOMEM;
  } catch (const std::exception&) {
    return VRC_EINVAL;
  }
  if (!base) return VRC_ECUDA;
  if (vrc::schur_log_bytes(kMaxN) > kLogBytes) {
    fprintf(stderr, "vrc_eig_noalloc: rotation-log scratch too small\n");
    return VRC_EINVAL;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  try {
    cplx* H = reinterpret_cast<cplx*>(base + kOffH);
    cplx* const* pH = reinterpret_cast<cplx* const*>(base + kOffPtr);
    cplx* const* pZ = pH + 1;
    cplx* const* pY = pH + 2;
    cplx* const* pLam = pH + 3;
    cplx* const* pW = pH + 4;
    const vrc::GemmDesc* desc = reinterpret_cast<const vrc::GemmDesc*>(base + kOffDesc);
    int* status = reinterpret_cast<int*>(base + kOffStatus);
    VRC_CUDA_CHECK(cudaMemcpyAsync(H, A, (size_t)n * n * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
    VRC_CUDA_CHECK(cudaMemsetAsync(status, 0, sizeof(int), st));
    noalloc_setup_kernel<<<1, 1, 0, st>>>(reinterpret_cast<cplx*>(W), reinterpret_cast<cplx*>(lam));
    VRC_CUDA_CHECK(cudaGetLastError());
    vrc::hessenberg_batched(pH, pZ, 1, n, st);
    void* const* pLog = reinterpret_cast<void* const*>(pH + 5);
    vrc::schur_batched(pH, pZ, pLam, pLog, 1, n, status, st);
    vrc::trevc_batched(pH, pY, 1, n, st);
    vrc::zgemm_batched(desc, 1, n, vrc::mk(1, 0), vrc::mk(0, 0), 0.0, st);  // W = Z Y
    vrc::vecnorm_batched(pW, 1, n, st);
    int h = 0;
    VRC_CUDA_CHECK(cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, st));
    VRC_CUDA_CHECK(cudaStreamSynchronize(st));
    return h ? VRC_ENOCONV : VRC_OK;
  } catch (const vrc::CudaError&) {
    return VRC_ECUDA;
  } catch (const vrc::StatusError& e) {
    return e.status;
  } catch (const std::bad_alloc&) {
    return VRC_ENOMEM;
  } catch (const std::exception&) {
    return VRC_EINVAL;
  }
}
