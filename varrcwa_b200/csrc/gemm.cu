// Batched complex128 GEMM on FP64 tensor cores (DMMA, mma.sync m16n8k4 f64).
//
//   C = diag(rs) * (alpha * A * B) * diag(cs) + beta * Cin + delta * I
//
// for column-major n x n operands (every contraction of the hot path is
// square: projections, star products, perturbation terms, P*Q), or with an
// inner dimension kdim != n (A is n x kdim, B is kdim x n) for the rank-kdim
// updates of the blocked inversion, or of general shape M x N x K with
// leading dimensions (zgemm_rect_batched: the panel updates of the blocked
// Hessenberg reduction).  Either operand may be taken as its conjugate
// transpose (used by the adjoint and the Hessenberg reflectors).  One CTA
// computes a 64 x 64 complex tile (eight warps of 32 x 16), or a 32 x 32
// tile (four warps of 16 x 16) for small orders, where 64-wide tiles would
// mostly compute padding (n = 82: 41% of a 128 x 128 cover is useful, 73% of
// 96 x 96).  Every output element accumulates over k in the same order with
// either tile, so the choice does not change results; the engine times both
// once per shape and keeps the faster.  Operands are staged through shared
// memory by 16-byte cp.async copies in a 3-stage pipeline or, for the 64-wide
// tile with VRC_GEMM_BULK set, by the TMA unit's bulk copies in a 4-stage
// pipeline (zgemm_bulk_kernel).  The complex product
// uses three real products (P1 = Ar Br, P2 = Ai Bi, P3 = (Ar+Ai)(Br+Bi);
// Cr = P1 - P2, Ci = P3 - P1 - P2), as cuBLAS Zgemm3m on the reference GPU
// path (src/gpu/types.cuh:33): a quarter fewer tensor-core products than the
// four-product form, with the normwise-stable error bound of the 3M method.
#include <cstdlib>

#include "common.cuh"
#include "kernels.h"

namespace vrc {

namespace {

constexpr int BK = 8, STAGES = 3;

// Tile shape: WM x WN warps, each MT m16 tiles by NT n8 tiles.
template <int WM_, int WN_, int MT_, int NT_>
struct Tile {
  static constexpr int WM = WM_, WN = WN_, MT = MT_, NT = NT_;
  static constexpr int BM = WM * MT * 16, BN = WN * NT * 8;
  static constexpr int THREADS = WM * WN * 32;
  static constexpr int LDA = BM + 2;  // complex elements per k-row of the A tile
  static constexpr int LDB = BN + 2;
  static constexpr int SMEM = STAGES * BK * (LDA + LDB) * 16;
  static constexpr int LOADS_A = BM * BK / THREADS, LOADS_B = BN * BK / THREADS;
  static_assert(BM * BK % THREADS == 0 && BN * BK % THREADS == 0, "tile loads");
};
using T64 = Tile<2, 4, 2, 2>;  // 64 x 64, 256 threads
using T32 = Tile<2, 2, 1, 2>;  // 32 x 32, 128 threads

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

// Shape of a batched product: C (M x N, ldc) = op(A) (M x K) op(B) (K x N);
// A stored M x K (lda) or, transposed, K x M; B stored K x N (ldb) or N x K.
struct GemmShape {
  int M, N, K, lda, ldb, ldc;
};

// C tile store: C = diag(rs) (alpha A B) diag(cs) + beta Cin + delta I, from
// the three real products of the 3M form, entries outside M x N dropped.
template <class TL>
__device__ __forceinline__ void store_tile(const GemmDesc& d, const GemmShape& sh, int m0, int n0, int wm, int wn,
                                           int g, int tig, const double (&acc1)[TL::MT][TL::NT][4],
                                           const double (&acc2)[TL::MT][TL::NT][4],
                                           const double (&acc3)[TL::MT][TL::NT][4], cplx alpha, cplx beta,
                                           double delta) {
  constexpr int MT = TL::MT, NT = TL::NT;
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        int row = m0 + wm * (MT * 16) + mt * 16 + g + ((c >> 1) << 3);
        int col = n0 + wn * (NT * 8) + nt * 8 + tig * 2 + (c & 1);
        if (row < sh.M && col < sh.N) {
          const double p1 = acc1[mt][nt][c], p2 = acc2[mt][nt][c];
          cplx v = mk(p1 - p2, acc3[mt][nt][c] - p1 - p2);
          v = cmul(alpha, v);
          if (d.rs) v = cmul(d.rs[row], v);
          if (d.cs) v = cmul(v, d.cs[col]);
          size_t off = (size_t)col * sh.ldc + row;
          if (d.Cin) v = cfma(beta, d.Cin[off], v);
          if (row == col) v.x += delta;
          d.C[off] = v;
        }
      }
}

// OPA / OPB: 0 = the operand as stored, 1 = its conjugate transpose.  A
// transposed operand is staged with consecutive threads along its stored
// columns (coalesced) and conjugated when fragments are read.

template <class TL, int OPA, int OPB>
__global__ void __launch_bounds__(TL::THREADS, 512 / TL::THREADS)
    zgemm_kernel(const GemmDesc* __restrict__ descs, GemmShape sh, cplx alpha, cplx beta, double delta) {
  constexpr int BM = TL::BM, BN = TL::BN, LDA = TL::LDA, LDB = TL::LDB, MT = TL::MT, NT = TL::NT;
  constexpr int NTHREADS = TL::THREADS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* As = reinterpret_cast<cplx*>(smem_raw);        // [STAGES][BK][LDA]
  cplx* Bs = As + STAGES * BK * LDA;                    // [STAGES][BK][LDB]

  const GemmDesc d = descs[blockIdx.y];
  const int kdim = sh.K;
  const int tiles_m = (sh.M + BM - 1) / BM;
  const int m0 = (blockIdx.x % tiles_m) * BM;
  const int n0 = (blockIdx.x / tiles_m) * BN;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, tig = lane & 3;
  const int wm = warp % TL::WM, wn = warp / TL::WM;  // warp tile: MT*16 x NT*8 complex

  const cplx* __restrict__ A = d.A;
  const cplx* __restrict__ B = d.B;
  const int KT = (kdim + BK - 1) / BK;

  auto load_tile = [&](int stage, int kt) {
    const int k0 = kt * BK;
    cplx* as = As + stage * BK * LDA;
    cplx* bs = Bs + stage * BK * LDB;
#pragma unroll
    for (int i = 0; i < TL::LOADS_A; ++i) {
      int idx = tid + i * NTHREADS;
      if (OPA == 0) {
        // A tile: BM rows x 8 cols, consecutive threads -> consecutive rows.
        int r = idx % BM, k = idx / BM;
        int gr = m0 + r, gk = k0 + k;
        bool va = (gr < sh.M) && (gk < kdim);
        cp_async16(as + k * LDA + r, va ? (const void*)(A + (size_t)gk * sh.lda + gr) : (const void*)A, va);
      } else {
        // op(A)(r, k) = conj(A(k, r)), stored at A[r * lda + k]: threads along k.
        int k = idx & 7, r = idx >> 3;
        int gr = m0 + r, gk = k0 + k;
        bool va = (gr < sh.M) && (gk < kdim);
        cp_async16(as + k * LDA + r, va ? (const void*)(A + (size_t)gr * sh.lda + gk) : (const void*)A, va);
      }
    }
#pragma unroll
    for (int i = 0; i < TL::LOADS_B; ++i) {
      int idx = tid + i * NTHREADS;
      if (OPB == 0) {
        // B tile: 8 rows x BN cols, consecutive threads -> consecutive k.
        int kb = idx & 7, c = idx >> 3;
        int gkb = k0 + kb, gc = n0 + c;
        bool vb = (gkb < kdim) && (gc < sh.N);
        cp_async16(bs + kb * LDB + c, vb ? (const void*)(B + (size_t)gc * sh.ldb + gkb) : (const void*)B, vb);
      } else {
        // op(B)(k, c) = conj(B(c, k)), stored at B[k * ldb + c]: threads along c.
        int c = idx % BN, kb = idx / BN;
        int gkb = k0 + kb, gc = n0 + c;
        bool vb = (gkb < kdim) && (gc < sh.N);
        cp_async16(bs + kb * LDB + c, vb ? (const void*)(B + (size_t)gkb * sh.ldb + gc) : (const void*)B, vb);
      }
    }
  };

  double acc1[MT][NT][4], acc2[MT][NT][4], acc3[MT][NT][4];
#pragma unroll
  for (int a = 0; a < MT; ++a)
#pragma unroll
    for (int b = 0; b < NT; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc1[a][b][c] = acc2[a][b][c] = acc3[a][b][c] = 0.0;

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < KT) load_tile(s, s);
    cp_async_commit();
  }

  for (int kt = 0; kt < KT; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    int nk = kt + STAGES - 1;
    if (nk < KT) load_tile(nk % STAGES, nk);
    cp_async_commit();

    const cplx* as = As + (kt % STAGES) * BK * LDA;
    const cplx* bs = Bs + (kt % STAGES) * BK * LDB;
#pragma unroll
    for (int ks = 0; ks < BK; ks += 4) {
      cplx af[MT][2], bf[NT];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        int row = wm * (MT * 16) + mt * 16 + g;
        af[mt][0] = as[(ks + tig) * LDA + row];
        af[mt][1] = as[(ks + tig) * LDA + row + 8];
        if (OPA) {
          af[mt][0].y = -af[mt][0].y;
          af[mt][1].y = -af[mt][1].y;
        }
      }
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        bf[nt] = bs[(ks + tig) * LDB + wn * (NT * 8) + nt * 8 + g];
        if (OPB) bf[nt].y = -bf[nt].y;
      }
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          dmma(acc1[mt][nt], af[mt][0].x, af[mt][1].x, bf[nt].x);
          dmma(acc2[mt][nt], af[mt][0].y, af[mt][1].y, bf[nt].y);
          dmma(acc3[mt][nt], af[mt][0].x + af[mt][0].y, af[mt][1].x + af[mt][1].y, bf[nt].x + bf[nt].y);
        }
    }
  }
  cp_async_wait<0>();

  store_tile<TL>(d, sh, m0, n0, wm, wn, g, tig, acc1, acc2, acc3, alpha, beta, delta);
}

// ---------------------------------------------------------------------------
// Bulk-copy (TMA) staging: the same 64 x 64 DMMA tile, its operand tiles
// brought into shared memory by the tensor memory accelerator's
// non-tensor bulk copies (cp.async.bulk, one elected warp per CTA issues a
// stage: one copy per stored column of the tile) completing on a per-stage
// mbarrier, instead of 16-byte cp.async by every thread.  A stored column
// of the tile is contiguous in global memory (column-major operands), so
// no tensor map is needed and per-matrix pointers stay plain.  Edges: rows
// or columns beyond M, N are not copied (their stale contents only reach
// output entries that are not stored); the k range beyond K is masked to
// zero at fragment load.  Every output element accumulates over k in the
// same order as zgemm_kernel, so results are bit-identical.
constexpr int BULK_STAGES = 4;
constexpr int BULK_LDK = BK + 4;  // [col][k] stages: 12 complex per stored column (bank-conflict free fragments)
constexpr int BULK_WAIT_LIMIT = 1 << 20;

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
// bounded wait for the phase of the given parity; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
  for (int it = 0; it < BULK_WAIT_LIMIT; ++it) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

template <int OPA, int OPB, int MINB>
__global__ void __launch_bounds__(T64::THREADS, MINB)
    zgemm_bulk_kernel(const GemmDesc* __restrict__ descs, GemmShape sh, cplx alpha, cplx beta, double delta,
                      int* __restrict__ timeouts) {
  using TL = T64;
  constexpr int BM = TL::BM, BN = TL::BN, MT = TL::MT, NT = TL::NT;
  constexpr int LDA = TL::LDA, LDB = TL::LDB;
  // per stage: A then B, each the larger of its two layouts
  constexpr int SA = (BK * LDA > BM * BULK_LDK) ? BK * LDA : BM * BULK_LDK;
  constexpr int SB = (BK * LDB > BN * BULK_LDK) ? BK * LDB : BN * BULK_LDK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* stg = reinterpret_cast<cplx*>(smem_raw);  // [BULK_STAGES][SA + SB]
  __shared__ __align__(8) unsigned long long s_full[BULK_STAGES];
  __shared__ int s_issued;

  const GemmDesc d = descs[blockIdx.y];
  const int K = sh.K;
  const int tiles_m = (sh.M + BM - 1) / BM;
  const int m0 = (blockIdx.x % tiles_m) * BM;
  const int n0 = (blockIdx.x / tiles_m) * BN;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, tig = lane & 3;
  const int wm = warp % TL::WM, wn = warp / TL::WM;
  const int KT = (K + BK - 1) / BK;
  const cplx* __restrict__ A = d.A;
  const cplx* __restrict__ B = d.B;

  if (tid == 0) {
    for (int s = 0; s < BULK_STAGES; ++s) mbar_init(smem_addr(&s_full[s]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_issued = 0;
  }
  __syncthreads();

  // warp 0 issues the copies of k-tile kt into stage kt % BULK_STAGES; in
  // a partial last k-tile it also zeroes the k range beyond K
  auto issue = [&](int kt) {
    const int s = kt % BULK_STAGES, k0 = kt * BK, kv = min(BK, K - k0);
    const int rows = min(BM, sh.M - m0), cols = min(BN, sh.N - n0);
    cplx* as = stg + (size_t)s * (SA + SB);
    cplx* bs = as + SA;
    const unsigned bar = smem_addr(&s_full[s]);
    if (lane == 0) mbar_expect_tx(bar, (unsigned)(kv * (rows + cols)) * 16u);
    __syncwarp();
    if (OPA == 0) {
      if (lane < kv) bulk_g2s(smem_addr(as + lane * LDA), A + (size_t)(k0 + lane) * sh.lda + m0, rows * 16u, bar);
    } else {
      for (int r = lane; r < rows; r += 32)
        bulk_g2s(smem_addr(as + r * BULK_LDK), A + (size_t)(m0 + r) * sh.lda + k0, kv * 16u, bar);
    }
    if (OPB == 0) {
      for (int c = lane; c < cols; c += 32)
        bulk_g2s(smem_addr(bs + c * BULK_LDK), B + (size_t)(n0 + c) * sh.ldb + k0, kv * 16u, bar);
    } else {
      if (lane < kv) bulk_g2s(smem_addr(bs + lane * LDB), B + (size_t)(k0 + lane) * sh.ldb + n0, cols * 16u, bar);
    }
    if (kv < BK) {
      for (int e = lane; e < (BK - kv) * BM; e += 32) {
        const int k = kv + e / BM, r = e % BM;
        as[OPA == 0 ? k * LDA + r : r * BULK_LDK + k] = mk(0.0, 0.0);
      }
      for (int e = lane; e < (BK - kv) * BN; e += 32) {
        const int k = kv + e / BN, c = e % BN;
        bs[OPB == 0 ? c * BULK_LDK + k : k * LDB + c] = mk(0.0, 0.0);
      }
    }
    if (lane == 0) s_issued = kt + 1;
  };

  double acc1[MT][NT][4], acc2[MT][NT][4], acc3[MT][NT][4];
#pragma unroll
  for (int a = 0; a < MT; ++a)
#pragma unroll
    for (int b = 0; b < NT; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc1[a][b][c] = acc2[a][b][c] = acc3[a][b][c] = 0.0;

  if (warp == 0)
    for (int s = 0; s < BULK_STAGES - 1 && s < KT; ++s) issue(s);

  bool ok = true;
  for (int kt = 0; kt < KT; ++kt) {
    const int s = kt % BULK_STAGES;
    const bool landed = mbar_wait(smem_addr(&s_full[s]), (unsigned)((kt / BULK_STAGES) & 1));
    // every thread is past the previous stage's reads; all leave together
    // if any gave up waiting
    if (__syncthreads_or(!landed)) {
      ok = false;
      break;
    }
    if (warp == 0 && kt + BULK_STAGES - 1 < KT) issue(kt + BULK_STAGES - 1);
    const cplx* as = stg + (size_t)s * (SA + SB);
    const cplx* bs = as + SA;
#pragma unroll
    for (int ks = 0; ks < BK; ks += 4) {
      cplx af[MT][2], bf[NT];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        const int row = wm * (MT * 16) + mt * 16 + g;
        if (OPA == 0) {
          af[mt][0] = as[(ks + tig) * LDA + row];
          af[mt][1] = as[(ks + tig) * LDA + row + 8];
        } else {
          af[mt][0] = as[row * BULK_LDK + ks + tig];
          af[mt][1] = as[(row + 8) * BULK_LDK + ks + tig];
          af[mt][0].y = -af[mt][0].y;
          af[mt][1].y = -af[mt][1].y;
        }
      }
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const int col = wn * (NT * 8) + nt * 8 + g;
        if (OPB == 0) {
          bf[nt] = bs[col * BULK_LDK + ks + tig];
        } else {
          bf[nt] = bs[(ks + tig) * LDB + col];
          bf[nt].y = -bf[nt].y;
        }
      }
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          dmma(acc1[mt][nt], af[mt][0].x, af[mt][1].x, bf[nt].x);
          dmma(acc2[mt][nt], af[mt][0].y, af[mt][1].y, bf[nt].y);
          dmma(acc3[mt][nt], af[mt][0].x + af[mt][0].y, af[mt][1].x + af[mt][1].y, bf[nt].x + bf[nt].y);
        }
    }
  }
  if (!ok) {
    // a stage never completed: record it, let the copies in flight land
    // (bounded), and store nothing
    if (tid == 0) {
      atomicAdd(timeouts, 1);
      for (int q = max(0, s_issued - BULK_STAGES); q < s_issued; ++q)
        mbar_wait(smem_addr(&s_full[q % BULK_STAGES]), (unsigned)((q / BULK_STAGES) & 1));
    }
    __syncthreads();
    return;
  }
  store_tile<TL>(d, sh, m0, n0, wm, wn, g, tig, acc1, acc2, acc3, alpha, beta, delta);
}

template <class TL>
void launch_tile(const GemmDesc* d_descs, int batch, const GemmShape& sh, cplx alpha, cplx beta, double delta,
                 cudaStream_t stream, int opA, int opB) {
  auto kern = opA ? (opB ? zgemm_kernel<TL, 1, 1> : zgemm_kernel<TL, 1, 0>)
                  : (opB ? zgemm_kernel<TL, 0, 1> : zgemm_kernel<TL, 0, 0>);
  ensure_smem((const void*)kern, TL::SMEM);
  const int tiles = ((sh.M + TL::BM - 1) / TL::BM) * ((sh.N + TL::BN - 1) / TL::BN);
  for (int b0 = 0; b0 < batch; b0 += 65535) {
    int nb = batch - b0 < 65535 ? batch - b0 : 65535;
    dim3 grid(tiles, nb);
    kern<<<grid, TL::THREADS, TL::SMEM, stream>>>(d_descs + b0, sh, alpha, beta, delta);
  }
}

// Wait-timeout counter of the bulk-staged kernels: mapped pinned host memory
// (written by a kernel only when a stage never completes), read by the host
// after a stream synchronisation without a copy.
int* bulk_timeouts() {
  static int* p = [] {
    int* h = nullptr;
    VRC_CUDA_CHECK(cudaHostAlloc(&h, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable));
    *h = 0;
    return h;
  }();
  return p;
}

// Operand staging of the 64 x 64 tile: VRC_GEMM_BULK unset or 0: 16-byte
// cp.async by every thread; 2: bulk copies, registers sized for two CTAs per
// SM; 1: bulk copies, one CTA per SM.  Results are the same bit for bit.
int bulk_mode() {
  const char* e = std::getenv("VRC_GEMM_BULK");
  if (!e) return 0;
  const int v = std::atoi(e);
  return (v == 1 || v == 2) ? v : 0;
}

template <int MINB>
void launch_bulk(const GemmDesc* d_descs, int batch, const GemmShape& sh, cplx alpha, cplx beta, double delta,
                 cudaStream_t stream, int opA, int opB) {
  constexpr int SA = (BK * T64::LDA > T64::BM * BULK_LDK) ? BK * T64::LDA : T64::BM * BULK_LDK;
  constexpr int SB = (BK * T64::LDB > T64::BN * BULK_LDK) ? BK * T64::LDB : T64::BN * BULK_LDK;
  constexpr int smem = BULK_STAGES * (SA + SB) * 16;
  auto kern = opA ? (opB ? zgemm_bulk_kernel<1, 1, MINB> : zgemm_bulk_kernel<1, 0, MINB>)
                  : (opB ? zgemm_bulk_kernel<0, 1, MINB> : zgemm_bulk_kernel<0, 0, MINB>);
  ensure_smem((const void*)kern, smem);
  int* flag = bulk_timeouts();
  const int tiles = ((sh.M + T64::BM - 1) / T64::BM) * ((sh.N + T64::BN - 1) / T64::BN);
  for (int b0 = 0; b0 < batch; b0 += 65535) {
    int nb = batch - b0 < 65535 ? batch - b0 : 65535;
    kern<<<dim3(tiles, nb), T64::THREADS, smem, stream>>>(d_descs + b0, sh, alpha, beta, delta, flag);
  }
}

void launch(const GemmDesc* d_descs, int batch, const GemmShape& sh, cplx alpha, cplx beta, double delta,
            cudaStream_t stream, int opA, int opB, int tile) {
  if (tile != 32 && tile != 64) throw StatusError(ST_EINVAL, "GEMM tile must be 32 or 64");
  if (batch <= 0 || sh.M <= 0 || sh.N <= 0) return;
  if (tile == 64 && bulk_mode() != 0) {
    if (bulk_mode() == 2)
      launch_bulk<2>(d_descs, batch, sh, alpha, beta, delta, stream, opA, opB);
    else
      launch_bulk<1>(d_descs, batch, sh, alpha, beta, delta, stream, opA, opB);
    VRC_CUDA_CHECK(cudaGetLastError());
    return;
  }
  if (tile == 32)
    launch_tile<T32>(d_descs, batch, sh, alpha, beta, delta, stream, opA, opB);
  else
    launch_tile<T64>(d_descs, batch, sh, alpha, beta, delta, stream, opA, opB);
  VRC_CUDA_CHECK(cudaGetLastError());
}

}  // namespace

void gemm_bulk_check() {
  volatile int* flag = bulk_timeouts();
  if (*flag != 0) {
    *flag = 0;
    throw StatusError(ST_ETIMEOUT, "GEMM bulk-copy stage wait timed out");
  }
}

void zgemm_batched(const GemmDesc* d_descs, int batch, int n, cplx alpha, cplx beta, double delta,
                   cudaStream_t stream, int kdim, int opA, int opB, int tile) {
  if (kdim < 0) kdim = n;
  if ((opA || opB) && kdim != n) throw StatusError(ST_EINVAL, "transposed GEMM operands must be square");
  launch(d_descs, batch, GemmShape{n, n, kdim, n, kdim, n}, alpha, beta, delta, stream, opA, opB, tile);
}

void zgemm_rect_batched(const GemmDesc* d_descs, int batch, int M, int N, int K, int lda, int ldb, int ldc,
                        cplx alpha, cplx beta, cudaStream_t stream, int opA, int opB, int tile) {
  if (K < 1 || lda < 1 || ldb < 1 || ldc < M) throw StatusError(ST_EINVAL, "invalid GEMM shape");
  if ((opA ? lda < K : lda < M) || (opB ? ldb < N : ldb < K))
    throw StatusError(ST_EINVAL, "GEMM leading dimension below the operand's rows");
  launch(d_descs, batch, GemmShape{M, N, K, lda, ldb, ldc}, alpha, beta, 0.0, stream, opA, opB, tile);
}

}  // namespace vrc
