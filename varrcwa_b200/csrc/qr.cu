// Complex Schur form by implicitly shifted QR with several bulges per sweep
// (FP64, one CTA per matrix), plus the replay of the logged rotations onto
// the Schur vectors and the parts of T outside the active window.
//
// Sweep on the active window [m, i] with nb shifts (the eigenvalues of the
// trailing nb x nb block; one Wilkinson or exceptional shift when nb = 1):
// bulge a (warp a) is introduced at round 3a and moves one position per
// round, so in round r it performs step k = m + r - 3a.  Bulges three apart
// use reflectors on disjoint index pairs.  In a round every entry receives at
// most one row transform (L) and one column transform (R), and L (X R) =
// (L X) R, so the warps need not wait for one another inside a round: the
// only entries two warps share are the 2 x 2 blocks where a bulge's rows
// cross a leading bulge's columns, and the row-transforming warp applies both
// there (L first, then R, as a row phase followed by a column phase would),
// while the leading bulge's column transform skips those rows.  Each warp
// then forms its bulge's next reflector, and one CTA barrier ends the round.
// Rounds run in chunks of QB inside a diagonal
// window D held in shared memory; after a chunk the rest of the active
// window is updated by one thread per row or column, which carries a value
// down each bulge's chain of the chunk (carry_chain).  Rows above the
// window, columns right of it and all of Z are not touched here: every
// sweep's rotations are logged round-major and replayed afterwards, whole
// rounds at a time from a sliding register ring (qr_replay_rows_kernel /
// qr_replay_cols_kernel).  For
// any entry, eager in-window updates precede deferred column transforms,
// which precede deferred row transforms (the window's bottom only moves up
// and windows never straddle a zero subdiagonal), so the replay reproduces
// the full transformation.
//
// Deflation: small subdiagonals (Ahues-Tisseur test) split the window;
// exceptional shifts at iterations 10 and 20; at most 30*max(10,n)
// iterations per eigenvalue and 30n+300 in total, else ST_ENOCONV.
#include <cstdlib>

#include "common.cuh"
#include "householder.cuh"
#include "kernels.h"

namespace vrc {
namespace {

constexpr int QR_THREADS = 256;
constexpr int NBMAX = QR_THREADS / 32;           // bulges per sweep (one warp each)
constexpr int QB = 32;                           // rounds per chunk
constexpr int QD = QB + 3 * (NBMAX - 1) + 3;     // diagonal window size (56)
// leading dimension of the window: odd in 16-byte units, so that the lanes
// of a row access (stride QLD) fall in distinct shared-memory banks
constexpr int QLD = QD + 1;
constexpr size_t QR_SMEM = (size_t)(QD * QLD + 2 * NBMAX * QB) * sizeof(cplx);

struct QrLogHeader {
  int nsweeps, nrot;
  int nrounds, pad0;                           // statistics
  long long t_defl, t_shift, t_rounds, t_far;  // statistics: SM clock cycles per phase
  long long pad[2];
};
constexpr int QR_HDR = sizeof(QrLogHeader);  // 64
// A sweep on the active window [m, i] with nb bulges and R rounds; its
// rotations are stored round-major from rotation index start: round u,
// bulge b at start + u*nb + b, acting on the pair (k, k+1), k = m + u - 3b,
// when m <= k <= i - 1 (other slots are padding and never read).
struct QrSweep {
  int m, i, nb, R;
  int start, pad0, pad1, pad2;
};

}  // namespace

long long schur_rot_cap(int n) { return 6LL * n * n + 64; }
int schur_sweep_cap(int n) { return 30 * n + 301; }  // the total iteration cap + 1
size_t schur_log_bytes(int n) {
  size_t b = QR_HDR + (size_t)schur_sweep_cap(n) * sizeof(QrSweep) + (size_t)schur_rot_cap(n) * 2 * sizeof(cplx);
  return (b + 255) / 256 * 256;
}

namespace {

__device__ __forceinline__ QrSweep* log_sweeps(char* logb) { return reinterpret_cast<QrSweep*>(logb + QR_HDR); }
__device__ __forceinline__ cplx* log_rot(char* logb, int sweep_cap) {
  return reinterpret_cast<cplx*>(logb + QR_HDR + (size_t)sweep_cap * sizeof(QrSweep));
}

// Eigenvalues of a small upper Hessenberg matrix A (nb x nb, column-major,
// nb <= NBMAX, shared memory) by single-shift QR, used only to pick shifts
// (on failure to converge the remaining diagonal entries are used).  One
// warp (all lanes call it): the reflectors are formed redundantly by every
// lane from the same shared-memory entries (identical results), and lanes own
// the columns of each row transform and the rows of each column transform.
__device__ void small_eigvals_warp(cplx* A, int nb, cplx* out, int lane) {
  auto a = [&](int r, int c) -> cplx& { return A[c * nb + r]; };
  int hi = nb - 1, it = 0;
  while (hi >= 0) {
    __syncwarp();
    if (hi == 0) {
      if (lane == 0) out[0] = a(0, 0);
      break;
    }
    int lo = hi;
    while (lo > 0 && cabs1(a(lo, lo - 1)) > EIG_ULP * (cabs1(a(lo - 1, lo - 1)) + cabs1(a(lo, lo)))) --lo;
    if (lo == hi) {
      if (lane == 0) out[hi] = a(hi, hi);
      --hi;
      it = 0;
      continue;
    }
    if (++it > 40) {
      if (lane == 0)
        for (int k = 0; k <= hi; ++k) out[k] = a(k, k);
      break;
    }
    const cplx p = a(hi - 1, hi - 1), q = a(hi - 1, hi), r = a(hi, hi - 1), d = a(hi, hi);
    const cplx half = cscale(csub(p, d), 0.5);
    const cplx disc = csqrt(cadd(cmul(half, half), cmul(q, r)));
    const cplx e1 = cadd(cadd(d, half), disc), e2 = csub(cadd(d, half), disc);
    cplx sh = (cabs2(csub(e1, d)) < cabs2(csub(e2, d))) ? e1 : e2;
    if (it % 10 == 0) sh = cadd(d, mk(0.75 * fabs(a(hi, hi - 1).x), 0.0));
    for (int k = lo; k < hi; ++k) {
      cplx x, y, beta, tau, v2;
      if (k == lo) {
        x = csub(a(lo, lo), sh);
        y = a(lo + 1, lo);
      } else {
        x = a(k, k - 1);
        y = a(k + 1, k - 1);
      }
      refl2(x, y, &beta, &tau, &v2);
      __syncwarp();  // every lane has read x, y
      if (k > lo && lane == 0) {
        a(k, k - 1) = beta;
        a(k + 1, k - 1) = mk(0.0, 0.0);
      }
      const cplx tauc = cconj(tau), v2c = cconj(v2);
      const int j = k + lane;
      if (j <= hi) {
        cplx u = a(k, j), w = a(k + 1, j);
        cplx s = cmul(tauc, cadd(u, cmul(v2c, w)));
        a(k, j) = csub(u, s);
        a(k + 1, j) = csub(w, cmul(s, v2));
      }
      __syncwarp();
      const int re = min(k + 2, hi), rr = lo + lane;
      if (rr <= re) {
        cplx u = a(rr, k), w = a(rr, k + 1);
        cplx s = cmul(tau, cadd(u, cmul(v2, w)));
        a(rr, k) = csub(u, s);
        a(rr, k + 1) = csub(w, cmul(s, v2c));
      }
      __syncwarp();
    }
  }
}

// Single shift for window [l, i]: exceptional at iterations 10 and 20, else
// Wilkinson's (the eigenvalue of the trailing 2x2 block closer to H[i][i],
// computed in scaled form).
__device__ cplx single_shift(const cplx* H, int n, int l, int i, int its) {
  auto h = [&](int r, int c) { return H[(size_t)c * n + r]; };
  if (its == 10) return cadd(mk(0.75 * fabs(h(l + 1, l).x), 0.0), h(l, l));
  if (its == 20) return cadd(mk(0.75 * fabs(h(i, i - 1).x), 0.0), h(i, i));
  cplx t = h(i, i);
  cplx uu = cmul(csqrt(h(i - 1, i)), csqrt(h(i, i - 1)));
  double s = cabs1(uu);
  if (s != 0.0) {
    cplx x = cscale(csub(h(i - 1, i - 1), t), 0.5);
    double sx = cabs1(x);
    s = fmax(s, sx);
    cplx xs = cscale(x, 1.0 / s), us = cscale(uu, 1.0 / s);
    cplx yv = cscale(csqrt(cadd(cmul(xs, xs), cmul(us, us))), s);
    if (sx > 0.0) {
      cplx xn = cscale(x, 1.0 / sx);
      if (xn.x * yv.x + xn.y * yv.y < 0.0) yv = cneg(yv);
    }
    t = csub(t, cmul(uu, cdiv(uu, cadd(x, yv))));
  }
  return t;
}

// One reflector I - tau v v^H, v = (1, v2), on the pair (a, b): from the
// left (ROWOP, conj(tau)) or from the right.
template <bool ROWOP>
__device__ __forceinline__ void rotate2(cplx& a, cplx& b, cplx tau, cplx v2) {
  if (ROWOP) {
    const cplx s = cmul(cconj(tau), cadd(a, cmul(cconj(v2), b)));
    a = csub(a, s);
    b = csub(b, cmul(s, v2));
  } else {
    const cplx s = cmul(tau, cadd(a, cmul(v2, b)));
    a = csub(a, s);
    b = csub(b, cmul(s, cconj(v2)));
  }
}

// Carries one value down a chain of cnt rotations on consecutive index
// pairs (k0, k0+1), (k0+1, k0+2), ...: row transforms on a column (rowop,
// entries p0[t], stride 1) or column transforms on a row (stride n).  The
// entries are fetched in groups of CG, double buffered: the loads of the
// next group are issued before the current group's rotations, so their
// latency overlaps the arithmetic.  Every entry a rotation writes lies below
// the next group's (the chain moves forward), so the early loads read
// values no rotation of this chain changes.
template <int CG>
__device__ __forceinline__ void carry_chain(cplx* p0, size_t stride, int cnt, const cplx* taus, const cplx* v2s,
                                            bool rowop) {
  cplx c = p0[0];
  cplx q[CG], qn[CG];
#pragma unroll
  for (int u = 0; u < CG; ++u)
    if (u < cnt) q[u] = p0[(size_t)(u + 1) * stride];
  for (int t0 = 0; t0 < cnt; t0 += CG) {
#pragma unroll
    for (int u = 0; u < CG; ++u)
      if (t0 + CG + u < cnt) qn[u] = p0[(size_t)(t0 + CG + u + 1) * stride];
#pragma unroll
    for (int u = 0; u < CG; ++u) {
      if (t0 + u < cnt) {
        cplx b = q[u];
        if (rowop)
          rotate2<true>(c, b, taus[t0 + u], v2s[t0 + u]);
        else
          rotate2<false>(c, b, taus[t0 + u], v2s[t0 + u]);
        p0[(size_t)(t0 + u) * stride] = c;
        c = b;
      }
    }
#pragma unroll
    for (int u = 0; u < CG; ++u) q[u] = qn[u];
  }
  p0[(size_t)cnt * stride] = c;
}

// MINB: resident CTAs per SM the registers are sized for; with three the
// carry chains prefetch two entries instead of four (no spills either way).
template <int MINB>
__global__ void __launch_bounds__(QR_THREADS, MINB)
    hqr_kernel(cplx* const* __restrict__ Hs, void* const* __restrict__ logs, cplx* const* __restrict__ Ws, int n,
               int sweep_cap, long long rot_cap, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* D = reinterpret_cast<cplx*>(smem_raw);  // [QD][QLD] column-major window
  cplx* s_tau = D + QD * QLD;                   // [NBMAX][QB]
  cplx* s_v2 = s_tau + NBMAX * QB;              // [NBMAX][QB]
  __shared__ cplx s_shift[NBMAX];
  __shared__ cplx s_small[NBMAX * NBMAX];
  __shared__ int s_red[QR_THREADS / 32];
  __shared__ int s_l, s_nb, s_nsw, s_nrot, s_over, s_nround, s_cur;
  __shared__ long long s_clk[5];  // statistics: phase timers (defl, shift, rounds, far) and the last stamp

  cplx* H = Hs[blockIdx.x];
  char* logb = static_cast<char*>(logs[blockIdx.x]);
  QrSweep* sweeps = log_sweeps(logb);
  cplx* rot = log_rot(logb, sweep_cap);
  cplx* W = Ws[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double smlnum = EIG_SAFMIN * ((double)n / EIG_ULP);
  const int itmax = 30 * max(10, n);       // per eigenvalue
  const long long totmax = 30LL * n + 300;  // whole matrix
  long long tot = 0;
  auto h = [&](int r, int c) -> cplx& { return H[(size_t)c * n + r]; };
  if (tid == 0) {
    s_nsw = 0;
    s_nrot = 0;
    s_over = 0;
    s_nround = 0;
    for (int q = 0; q < 5; ++q) s_clk[q] = 0;
  }
  __syncthreads();
  // tid 0 only: charge the time since the last stamp to phase q
  auto stamp = [&](int q) {
    const long long t = clock64();
    if (q >= 0) s_clk[q] += t - s_clk[4];
    s_clk[4] = t;
  };
  int i = n - 1;
  int failed = 0;
  while (i >= 0) {
    int l = 0;
    int its;
    for (its = 0; its <= itmax && tot <= totmax; ++its, ++tot) {
      if (tid == 0) stamp(-1);
      // Deflation search: largest k in (l, i] with a negligible H[k][k-1].
      int best = l;
      for (int k = l + 1 + tid; k <= i; k += QR_THREADS) {
        const cplx sub = h(k, k - 1);
        bool small = false;
        const double cs = cabs1(sub);
        if (cs <= smlnum) {
          small = true;
        } else {
          const cplx dkm = h(k - 1, k - 1), dk = h(k, k);
          double tst = cabs1(dkm) + cabs1(dk);
          if (tst == 0.0) {
            if (k - 2 >= 0) tst += fabs(h(k - 1, k - 2).x);
            if (k + 1 <= n - 1) tst += fabs(h(k + 1, k).x);
          }
          if (cs <= EIG_ULP * tst) {
            const double a1 = cs, a2 = cabs1(h(k - 1, k));
            const double ab = fmax(a1, a2), ba = fmin(a1, a2);
            const double b1 = cabs1(dk), b2 = cabs1(csub(dkm, dk));
            const double aa = fmax(b1, b2), bb = fmin(b1, b2);
            const double s = aa + ab;
            if (ba * (ab / s) <= fmax(smlnum, EIG_ULP * (bb * (aa / s)))) small = true;
          }
        }
        if (small && k > best) best = k;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
      if (lane == 0) s_red[warp] = best;
      __syncthreads();
      if (tid == 0) {
        int b = l;
        for (int w = 0; w < QR_THREADS / 32; ++w) b = max(b, s_red[w]);
        s_l = b;
        if (b > l) h(b, b - 1) = mk(0.0, 0.0);
      }
      __syncthreads();
      l = s_l;
      if (tid == 0) stamp(0);
      if (l >= i) break;  // H[i][i] isolated
      // Number of bulges and their shifts.
      if (warp == 0) {
        const int w = i - l + 1;
        const int nb = (its == 10 || its == 20) ? 1 : min(NBMAX, max(1, (w - 4) / 6));
        if (nb == 1) {
          if (lane == 0) s_shift[0] = single_shift(H, n, l, i, its);
        } else {
          const int b0 = i - nb + 1;
          for (int idx = lane; idx < nb * nb; idx += 32) {
            const int c = idx / nb, r = idx - c * nb;
            s_small[c * nb + r] = (r <= c + 1) ? h(b0 + r, b0 + c) : mk(0.0, 0.0);
          }
          small_eigvals_warp(s_small, nb, s_shift, lane);
        }
        if (lane == 0) {
          s_nb = nb;
          stamp(1);
        }
      }
      __syncthreads();
      const int nb = s_nb, m = l;
      const int R = (i - m) + 3 * (nb - 1);  // rounds of this sweep
      if (tid == 0) {
        if (s_nsw + 1 > sweep_cap || (long long)s_nrot + (long long)R * nb > rot_cap) {
          s_over = 1;
        } else {
          sweeps[s_nsw] = QrSweep{m, i, nb, R, s_nrot, 0, 0, 0};
          s_cur = s_nrot;
          s_nsw += 1;
          s_nrot += R * nb;
          s_nround += R;
        }
      }
      const int a = warp;                      // this warp's bulge
      const bool mine = a < nb;
      for (int r0 = 0; r0 < R; r0 += QB) {
        const int r1 = min(r0 + QB, R);
        const int kmin = max(m, m + r0 - 3 * (nb - 1));
        const int kmax = min(i - 1, m + r1 - 1);
        const int ds = (kmin > m) ? kmin - 1 : m;
        const int de = min(kmax + 2, i);
        const int dn = de - ds + 1;
        for (int idx = tid; idx < dn * dn; idx += QR_THREADS) {
          const int c = idx / dn, r = idx - c * dn;
          D[c * QLD + r] = h(ds + r, ds + c);
        }
        __syncthreads();
        if (s_over) break;
        auto dd = [&](int r, int c) -> cplx& { return D[(c - ds) * QLD + (r - ds)]; };
        auto reflect = [&](int r) {
          const int k = m + r - 3 * a;
          if (lane == 0 && mine && k >= m && k <= i - 1) {
            cplx x, y, beta, tau, v2;
            if (k == m) {
              x = csub(dd(m, m), s_shift[a]);
              y = dd(m + 1, m);
            } else {
              x = dd(k, k - 1);
              y = dd(k + 1, k - 1);
            }
            refl2(x, y, &beta, &tau, &v2);
            if (k > m) {
              dd(k, k - 1) = beta;
              dd(k + 1, k - 1) = mk(0.0, 0.0);
            }
            s_tau[a * QB + (r - r0)] = tau;
            s_v2[a * QB + (r - r0)] = v2;
          }
        };
        reflect(r0);
        __syncthreads();
        for (int r = r0; r < r1; ++r) {
          const int k = m + r - 3 * a;
          const bool act = mine && k >= m && k <= i - 1;
          if (act) {
            const cplx tau = s_tau[a * QB + (r - r0)], v2 = s_v2[a * QB + (r - r0)];
            // row transform of rows k, k+1 over columns k..de
            {
              const cplx tauc = cconj(tau), v2c = cconj(v2);
              for (int j = k + lane; j <= de; j += 32) {
                const cplx x = dd(k, j), y = dd(k + 1, j);
                const cplx s = cmul(tauc, cadd(x, cmul(v2c, y)));
                dd(k, j) = csub(x, s);
                dd(k + 1, j) = csub(y, cmul(s, v2));
              }
            }
            __syncwarp();
            // the leading bulges' column transforms on rows k, k+1: bulge
            // b = a - 1 - lane acts on columns kb, kb + 1, kb = k + 3 (a - b)
            {
              const int b = a - 1 - lane, kb = k + 3 * (lane + 1);
              if (b >= 0 && kb <= i - 1) {
                const cplx tb = s_tau[b * QB + (r - r0)], vb = s_v2[b * QB + (r - r0)], vbc = cconj(vb);
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                  const cplx p = dd(k + q, kb), w = dd(k + q, kb + 1);
                  const cplx s = cmul(tb, cadd(p, cmul(vb, w)));
                  dd(k + q, kb) = csub(p, s);
                  dd(k + q, kb + 1) = csub(w, cmul(s, vbc));
                }
              }
            }
            // column transform of columns k, k+1 over rows ds..min(k+2, i),
            // except the rows of the trailing bulges (bulge a + q on rows
            // k - 3q, k - 3q + 1), which their own warps transform
            {
              const cplx v2c = cconj(v2);
              const int re = min(k + 2, i);
              for (int rr = ds + lane; rr <= re; rr += 32) {
                const int dk = k - rr, q = (dk + 1) / 3;
                if (dk >= 2 && dk % 3 != 1 && a + q < nb && k - 3 * q >= m) continue;
                const cplx p = dd(rr, k), w = dd(rr, k + 1);
                const cplx s = cmul(tau, cadd(p, cmul(v2, w)));
                dd(rr, k) = csub(p, s);
                dd(rr, k + 1) = csub(w, cmul(s, v2c));
              }
            }
          }
          __syncwarp();
          if (r + 1 < r1) reflect(r + 1);
          __syncthreads();
        }
        if (tid == 0) stamp(2);
        // Write the window back and log this chunk's rotations (round-major).
        for (int idx = tid; idx < dn * dn; idx += QR_THREADS) {
          const int c = idx / dn, r = idx - c * dn;
          h(ds + r, ds + c) = D[c * QLD + r];
        }
        const int nr = r1 - r0;
        for (int idx = tid; idx < nb * nr; idx += QR_THREADS) {
          const int u = idx / nb, b = idx - u * nb;
          const size_t ri = (size_t)s_cur + (size_t)(r0 + u) * nb + b;
          const int kk = m + r0 + u - 3 * b;  // slots of bulges outside the window hold the identity
          const bool on = kk >= m && kk <= i - 1;
          rot[2 * ri] = on ? s_tau[b * QB + u] : mk(0.0, 0.0);
          rot[2 * ri + 1] = on ? s_v2[b * QB + u] : mk(0.0, 0.0);
        }
        // Rest of the active window: columns de+1..i (row transforms) and rows
        // m..ds-1 (column transforms), one bulge chain at a time, leading
        // bulge first (the order of every pair of conflicting rotations).
        const int nright = i - de, nabove = ds - m;
        for (int task = tid; task < nright + nabove; task += QR_THREADS) {
          const bool rowop = task < nright;
          for (int b = 0; b < nb; ++b) {
            const int ra0 = max(r0, 3 * b), ra1 = min(r1, 3 * b + (i - m));
            if (ra1 <= ra0) continue;
            const int k0 = m + ra0 - 3 * b;
            cplx* p0 = rowop ? H + (size_t)(de + 1 + task) * n + k0 : H + (size_t)k0 * n + (m + task - nright);
            carry_chain<(MINB >= 3 ? 2 : 4)>(p0, rowop ? 1 : (size_t)n, ra1 - ra0, s_tau + b * QB + (ra0 - r0), s_v2 + b * QB + (ra0 - r0),
                        rowop);
          }
        }
        __syncthreads();
        if (tid == 0) stamp(3);
      }
      if (s_over) {
        failed = 1;
        break;
      }
    }
    if (failed || its > itmax || tot > totmax) {
      failed = 1;
      break;
    }
    i = l - 1;
  }
  __syncthreads();
  for (int k = tid; k < n; k += QR_THREADS) W[k] = h(k, k);
  if (tid == 0) {
    QrLogHeader* hdr = reinterpret_cast<QrLogHeader*>(logb);
    hdr->nsweeps = s_nsw;
    hdr->nrot = s_nrot;
    hdr->nrounds = s_nround;
    hdr->t_defl = s_clk[0];
    hdr->t_shift = s_clk[1];
    hdr->t_rounds = s_clk[2];
    hdr->t_far = s_clk[3];
    if (failed && status) status[blockIdx.x] = ST_ENOCONV;
  }
}

// Replay kernels: one thread per row (column transforms: rows of Z for
// every sweep, rows of H above the sweep's window) or per column (row
// transforms: columns of H right of the window).  All threads of a block
// belong to one matrix, so each sweep's rotations are staged through shared
// memory in slabs of RS rounds and read as broadcasts.  A thread's entries
// arrive PFD rounds ahead through 16-byte cp.async copies into its own
// shared-memory slots (the rounds are short, so register prefetch cannot
// cover the memory latency), then move into a ring of registers indexed by
// compile-time slots (round loops are unrolled by the ring size): each round
// takes in the entry the leading bulge reaches and retires the one the
// trailing bulge has passed; the group's rotations within a round touch
// disjoint pairs and run independently.
constexpr int RP_THREADS = 128;
constexpr int RP_NBG = 4;  // bulges per register ring
constexpr int RP_PFD = 7;  // prefetch depth in rounds (ring of PFD + 1 = 8 slots)

__device__ __forceinline__ void cpa16(cplx* smem, const cplx* g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int NBG, int PFD, bool ROWOP>
struct ReplayRing {
  static constexpr int L = 3 * (NBG - 1);  // retire lag
  static constexpr int P = L + 3;          // register ring: entries t-L .. t+1
  static constexpr int S = PFD + 1;        // shared-memory slots per thread
  cplx w[P];
  cplx* x;
  cplx* pf;  // this thread's slot 0; slot q at pf[q * RP_THREADS]
  size_t stride;
  int kb, lo, hi, rmin, cnt;

  __device__ __forceinline__ void begin(cplx* x_, size_t stride_, int kb_, int lo_, int hi_, int ng, int cnt_,
                                        cplx* pf_) {
    x = x_;
    pf = pf_;
    stride = stride_;
    kb = kb_;
    lo = lo_;
    hi = hi_;
    rmin = -3 * (ng - 1);
    cnt = cnt_;
    if (cnt <= 0) return;
#pragma unroll
    for (int q = -L; q <= 0; ++q) {
      const int c = kb + q;
      w[(q + P) % P] = (q >= rmin && c >= lo && c <= hi) ? x[(size_t)c * stride] : mk(0.0, 0.0);
    }
#pragma unroll
    for (int d = 1; d <= PFD; ++d) {  // one commit group per entry
      const int c = kb + d;
      if (c >= lo && c <= hi) cpa16(pf + (d % S) * RP_THREADS, x + (size_t)c * stride);
      cpa_commit();
    }
  }

  // srot: this group's rotations of rounds [t0, t1), NBG (tau, v2) pairs per
  // round, identity where a bulge is outside the window or beyond the group
  __device__ __forceinline__ void run(int t0, int t1, const cplx* __restrict__ srot) {
    t1 = min(t1, cnt);
    for (int tb = t0; tb < t1; tb += P) {
#pragma unroll
      for (int tt = 0; tt < P; ++tt) {
        const int t = tb + tt;
        if (t < t1) {
          const int cb = kb + t;
          cpa_wait<PFD - 1>();  // the group of entry t+1 has landed
          w[(tt + 1) % P] = (cb + 1 >= lo && cb + 1 <= hi) ? pf[((t + 1) % S) * RP_THREADS] : mk(0.0, 0.0);
          {
            const int c = cb + 1 + PFD;  // into the slot of entry t, consumed last round
            if (c >= lo && c <= hi) cpa16(pf + ((t + 1 + PFD) % S) * RP_THREADS, x + (size_t)c * stride);
            cpa_commit();
          }
          const cplx* rr = srot + 2 * NBG * (t - t0);
#pragma unroll
          for (int g = 0; g < NBG; ++g)  // straight-line: inactive pairs carry the identity
            rotate2<ROWOP>(w[(tt - 3 * g + 2 * P) % P], w[(tt - 3 * g + 1 + 2 * P) % P], rr[2 * g], rr[2 * g + 1]);
          {
            const int q = t - L, c = cb - L;
            if (q >= rmin && c >= lo && c <= hi) x[(size_t)c * stride] = w[(tt - L + 2 * P) % P];
          }
          if (t == cnt - 1) {
#pragma unroll
            for (int d = 1; d <= L + 1; ++d) {  // entries t-L+1 .. t+1 still held
              const int q = t - L + d, c = cb - L + d;
              if (q >= rmin && c >= lo && c <= hi) x[(size_t)c * stride] = w[(tt - L + d + 2 * P) % P];
            }
            cpa_wait<0>();  // no copy may land in the slots after this vector is done
          }
        }
      }
    }
  }
};

constexpr int RS = 4 * ReplayRing<RP_NBG, RP_PFD, false>::P;  // rounds per slab (a multiple of the ring size)
constexpr size_t RP_SMEM =
    (size_t)RS * NBMAX * 2 * sizeof(cplx) + (size_t)(RP_PFD + 1) * RP_THREADS * sizeof(cplx);

template <bool ROWOP>
__device__ __forceinline__ void replay_sweeps(cplx* x, size_t stride, int sel, int idx, const QrSweep* sw,
                                              int nsweeps, const cplx* rot, cplx* s_rot, cplx* s_pf) {
  // sel: 0 = every sweep, 1 = sweeps with idx < m (rows of H above the
  // window), 2 = sweeps with idx > i (columns of H right of the window);
  // idx < 0 marks a thread without a vector (it still joins the barriers).
  // Bulges are applied RP_NBG at a time, leading group first, each group
  // over the whole sweep.
  for (int s = 0; s < nsweeps; ++s) {
    const QrSweep q = sw[s];
    const int nb = q.nb;
    const bool active = idx >= 0 && (sel == 0 || (sel == 1 && idx < q.m) || (sel == 2 && idx > q.i));
    const cplx* src = rot + 2 * (size_t)q.start;
    for (int b0 = 0; b0 < nb; b0 += RP_NBG) {
      const int ng = min(RP_NBG, nb - b0);
      ReplayRing<RP_NBG, RP_PFD, ROWOP> ring;
      if (active) ring.begin(x, stride, q.m - 3 * b0, q.m, q.i, ng, q.R, s_pf + threadIdx.x);
      for (int t0 = 0; t0 < q.R; t0 += RS) {
        const int nr = min(RS, q.R - t0);
        __syncthreads();  // the previous slab is consumed
        for (int e = threadIdx.x; e < nr * RP_NBG; e += blockDim.x) {
          const int u = e / RP_NBG, b = b0 + (e % RP_NBG);
          const bool on = b < nb;
          const cplx* q2 = src + 2 * ((size_t)(t0 + u) * nb + b);
          s_rot[2 * e] = on ? ld(q2) : mk(0.0, 0.0);
          s_rot[2 * e + 1] = on ? ld(q2 + 1) : mk(0.0, 0.0);
        }
        __syncthreads();
        if (active) ring.run(t0, t0 + nr, s_rot);
      }
    }
  }
}

__global__ void __launch_bounds__(RP_THREADS, 4)
    qr_replay_rows_kernel(cplx* const* __restrict__ Hs, cplx* const* __restrict__ Zs,
                          void* const* __restrict__ logs, int n, int sweep_cap, int row_blocks) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* s_rot = reinterpret_cast<cplx*>(smem_raw);
  cplx* s_pf = s_rot + RS * NBMAX * 2;
  const int mat = blockIdx.y;
  const bool isZ = blockIdx.x >= row_blocks;
  const int r = (isZ ? blockIdx.x - row_blocks : blockIdx.x) * blockDim.x + threadIdx.x;
  cplx* X = isZ ? Zs[mat] : Hs[mat];
  char* logb = static_cast<char*>(logs[mat]);
  const QrLogHeader hdr = *reinterpret_cast<const QrLogHeader*>(logb);
  replay_sweeps<false>(X + min(r, n - 1), (size_t)n, isZ ? 0 : 1, r < n ? r : -1, log_sweeps(logb), hdr.nsweeps,
                       log_rot(logb, sweep_cap), s_rot, s_pf);
}

// Runs after qr_replay_rows_kernel: for any entry all column transforms
// precede all row transforms.
__global__ void __launch_bounds__(RP_THREADS, 4)
    qr_replay_cols_kernel(cplx* const* __restrict__ Hs, void* const* __restrict__ logs, int n, int sweep_cap) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* s_rot = reinterpret_cast<cplx*>(smem_raw);
  cplx* s_pf = s_rot + RS * NBMAX * 2;
  const int mat = blockIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  cplx* H = Hs[mat];
  char* logb = static_cast<char*>(logs[mat]);
  const QrLogHeader hdr = *reinterpret_cast<const QrLogHeader*>(logb);
  replay_sweeps<true>(H + (size_t)min(j, n - 1) * n, 1, 2, j < n ? j : -1, log_sweeps(logb), hdr.nsweeps,
                      log_rot(logb, sweep_cap), s_rot, s_pf);
}

}  // namespace

void schur_batched(cplx* const* d_H, cplx* const* d_Z, cplx* const* d_W, void* const* d_logs, int batch, int n,
                   int* d_status, cudaStream_t st, int parts) {
  if (batch <= 0) return;
  // resident Schur CTAs per SM: 2 (default) or 3 (VRC_QR_CTAS=3); the
  // arithmetic is the same, only the registers and the prefetch depth differ
  static const int minb = [] {
    const char* e = std::getenv("VRC_QR_CTAS");
    return (e && std::atoi(e) == 3) ? 3 : 2;
  }();
  auto hqr = minb == 3 ? hqr_kernel<3> : hqr_kernel<2>;
  ensure_smem((const void*)hqr, QR_SMEM);
  ensure_smem((const void*)qr_replay_rows_kernel, RP_SMEM);
  ensure_smem((const void*)qr_replay_cols_kernel, RP_SMEM);
  const int cc = schur_sweep_cap(n);
  const long long rc = schur_rot_cap(n);
  const int row_blocks = (n + RP_THREADS - 1) / RP_THREADS;
  const size_t rp_smem = RP_SMEM;
  for (int b0 = 0; b0 < batch; b0 += 65535) {
    const int nb = min(65535, batch - b0);
    if (parts & SCHUR_ITERATE)
      hqr<<<nb, QR_THREADS, QR_SMEM, st>>>(d_H + b0, d_logs + b0, d_W + b0, n, cc, rc,
                                                  d_status ? d_status + b0 : nullptr);
    if (parts & SCHUR_REPLAY) {
      qr_replay_rows_kernel<<<dim3(2 * row_blocks, nb), RP_THREADS, rp_smem, st>>>(d_H + b0, d_Z + b0, d_logs + b0,
                                                                                  n, cc, row_blocks);
      qr_replay_cols_kernel<<<dim3(row_blocks, nb), RP_THREADS, rp_smem, st>>>(d_H + b0, d_logs + b0, n, cc);
    }
  }
  VRC_CUDA_CHECK(cudaGetLastError());
}

}  // namespace vrc
