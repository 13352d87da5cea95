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
// iterations per eigenvalue and 30n+300 in total, else ST_ENOCONV.  Before
// a sweep, aggressive early deflation examines the trailing jw x jw block of
// the window (aed_* below): its converged eigenvalues deflate at once, and
// its unconverged ones are the sweep's shifts.  Its similarity transform U is
// applied eagerly inside the active window and logged as a dense block for
// the replay, in sequence with the sweeps' rotations.
#include <algorithm>
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
  int nrounds, naed;                           // statistics (naed: deflation-window blocks)
  long long t_defl, t_shift, t_rounds, t_far;  // statistics: SM clock cycles per phase
  long long t_wschur, t_wdefl;                 // statistics: window Schur form, window deflation
};
constexpr int QR_HDR = sizeof(QrLogHeader);  // 64
// A sweep on the active window [m, i] with nb bulges and R rounds; its
// rotations are stored round-major from rotation index start: round u,
// bulge b at start + u*nb + b, acting on the pair (k, k+1), k = m + u - 3b,
// when m <= k <= i - 1 (other slots are padding and never read).  A
// deflation-window block on the active window [m, i] has nb = -1: the
// unitary U of order R (columns and rows pad0..i) is stored column-major
// (leading dimension R) from rotation index start.
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

// cp.async copies of 16 bytes into shared memory, one commit group each.
__device__ __forceinline__ void cpa16(cplx* smem, const cplx* g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// A group of NBG bulges' rotations applied round by round to one vector x
// (entries x[c * stride]): in round t bulge g acts on the pair
// (kb + t - 3g, kb + t - 3g + 1).  Entries arrive PFD rounds ahead through
// 16-byte cp.async copies into this thread's shared-memory slots (THREADS
// apart), then move into a ring of registers indexed by compile-time slots
// (round loops are unrolled by the ring size): each round takes in the entry
// the leading bulge reaches and retires the one the trailing bulge has
// passed; the group's rotations within a round touch disjoint pairs and run
// independently.  Entries outside [lo, hi] are neither read nor written.
template <int NBG, int PFD, bool ROWOP, int THREADS>
struct RotRing {
  static constexpr int L = 3 * (NBG - 1);  // retire lag
  static constexpr int P = L + 3;          // register ring: entries t-L .. t+1
  static constexpr int S = PFD + 1;        // shared-memory slots per thread
  cplx w[P];
  cplx* x;
  cplx* pf;  // this thread's slot 0; slot q at pf[q * THREADS]
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
      if (c >= lo && c <= hi) cpa16(pf + (d % S) * THREADS, x + (size_t)c * stride);
      cpa_commit();
    }
  }

  // Rounds [t0, t1) (t0 a multiple of P); rot(t, g, tau, v2) gives bulge g's
  // rotation of round t, the identity where it is outside the window
  template <class ROT>
  __device__ __forceinline__ void run(int t0, int t1, ROT rot) {
    t1 = min(t1, cnt);
    for (int tb = t0; tb < t1; tb += P) {
#pragma unroll
      for (int tt = 0; tt < P; ++tt) {
        const int t = tb + tt;
        if (t < t1) {
          const int cb = kb + t;
          cpa_wait<PFD - 1>();  // the group of entry t+1 has landed
          w[(tt + 1) % P] = (cb + 1 >= lo && cb + 1 <= hi) ? pf[((t + 1) % S) * THREADS] : mk(0.0, 0.0);
          {
            const int c = cb + 1 + PFD;  // into the slot of entry t, consumed last round
            if (c >= lo && c <= hi) cpa16(pf + ((t + 1 + PFD) % S) * THREADS, x + (size_t)c * stride);
            cpa_commit();
          }
#pragma unroll
          for (int g = 0; g < NBG; ++g) {  // straight-line: inactive pairs carry the identity
            cplx tau, v2;
            rot(t, g, tau, v2);
            rotate2<ROWOP>(w[(tt - 3 * g + 2 * P) % P], w[(tt - 3 * g + 1 + 2 * P) % P], tau, v2);
          }
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

// ---------------------------------------------------------------------------
// Aggressive early deflation (Braman, Byers & Mathias, "The multishift QR
// algorithm. Part II: aggressive early deflation", SIAM J. Matrix Anal.
// Appl. 23 (2002); LAPACK xLAQR3).  The trailing jw x jw block of the active
// window (jw <= AW, one lane per row or column) is brought to Schur form
// T = U^H H_w U by one warp in shared memory.  The subdiagonal entry s0 that
// couples the block to the rest becomes the spike s0 * conj(U[0, :]); an
// eigenvalue whose spike entry is negligible deflates, the others are moved
// to the top of T by swaps of adjacent diagonal entries.  If any deflated,
// the undeflated top block with its spike is returned to Hessenberg form
// (one reflector, then a Householder reduction) and U is applied to the rows
// of the active window above the block; the rest of H and Z receive U through
// the log (a dense entry, replayed like the sweeps).  The undeflated
// eigenvalues become the next sweep's shifts.
constexpr int AW = 32;       // largest deflation window
constexpr int ALD = AW + 1;  // its leading dimension in shared memory (odd in 16-byte units)

// Givens rotation [cs sn; -conj(sn) cs] (cs real) with cs f + sn g = r and
// -conj(sn) f + cs g = 0.
__device__ __forceinline__ void givens(cplx f, cplx g, double* cs, cplx* sn) {
  const double ag = hypot(g.x, g.y);
  if (ag == 0.0) {
    *cs = 1.0;
    *sn = mk(0.0, 0.0);
    return;
  }
  const double af = hypot(f.x, f.y);
  if (af == 0.0) {
    *cs = 0.0;
    *sn = cscale(cconj(g), 1.0 / ag);
    return;
  }
  const double d = hypot(af, ag);
  *cs = af / d;
  *sn = cscale(cmul(cscale(f, 1.0 / af), cconj(g)), 1.0 / d);
}

// Negligible subdiagonal entry T[k][k-1] of a small window (the test of the
// main iteration: Ahues-Tisseur, LAPACK xLAHQR).
__device__ __forceinline__ bool small_negligible(const cplx* T, int nw, int k, double smlnum) {
  auto t = [&](int r, int c) { return T[c * ALD + r]; };
  const double cs = cabs1(t(k, k - 1));
  if (cs <= smlnum) return true;
  const cplx dkm = t(k - 1, k - 1), dk = t(k, k);
  double tst = cabs1(dkm) + cabs1(dk);
  if (tst == 0.0) {
    if (k - 2 >= 0) tst += fabs(t(k - 1, k - 2).x);
    if (k + 1 <= nw - 1) tst += fabs(t(k + 1, k).x);
  }
  if (cs > EIG_ULP * tst) return false;
  const double a1 = cs, a2 = cabs1(t(k - 1, k));
  const double ab = fmax(a1, a2), ba = fmin(a1, a2);
  const double b1 = cabs1(dk), b2 = cabs1(csub(dkm, dk));
  const double aa = fmax(b1, b2), bb = fmin(b1, b2);
  const double s = aa + ab;
  return ba * (ab / s) <= fmax(smlnum, EIG_ULP * (bb * (aa / s)));
}

// Schur form of the nw x nw upper Hessenberg T (shared memory, leading
// dimension ALD) by single-shift QR with Wilkinson shifts (exceptional at
// iterations 10 and 20), accumulating the rotations into U.  One warp; lanes
// own the columns of a row transform and the rows of a column transform.
// Returns false if an eigenvalue needs more than 30 * max(10, nw) iterations.
__device__ bool small_schur_warp(cplx* T, cplx* U, int nw, int lane, double smlnum) {
  auto t = [&](int r, int c) -> cplx& { return T[c * ALD + r]; };
  auto u = [&](int r, int c) -> cplx& { return U[c * ALD + r]; };
  const int itmax = 30 * max(10, nw);
  int hi = nw - 1, its = 0;
  while (hi > 0) {
    __syncwarp();
    // largest k <= hi with a negligible T[k][k-1] (lane k-1 tests k), else 0
    const bool negl = lane + 1 <= hi && small_negligible(T, nw, lane + 1, smlnum);
    const unsigned bal = __ballot_sync(0xffffffffu, negl);
    const int lo = bal ? 32 - __clz(bal) : 0;
    if (lo > 0 && lane == 0) t(lo, lo - 1) = mk(0.0, 0.0);
    __syncwarp();
    if (lo == hi) {
      --hi;
      its = 0;
      continue;
    }
    if (++its > itmax) return false;
    const cplx sh = single_shift(T, ALD, lo, hi, its);
    for (int k = lo; k < hi; ++k) {
      cplx x, y, beta, tau, v2;
      __syncwarp();
      if (k == lo) {
        x = csub(t(lo, lo), sh);
        y = t(lo + 1, lo);
      } else {
        x = t(k, k - 1);
        y = t(k + 1, k - 1);
      }
      refl2(x, y, &beta, &tau, &v2);
      __syncwarp();  // every lane has read x, y
      if (k > lo && lane == 0) {
        t(k, k - 1) = beta;
        t(k + 1, k - 1) = mk(0.0, 0.0);
      }
      const int j = k + lane;  // row transform over columns k..nw-1 (nw - k <= 32)
      if (j < nw) rotate2<true>(t(k, j), t(k + 1, j), tau, v2);
      __syncwarp();
      if (lane <= min(k + 2, hi)) rotate2<false>(t(lane, k), t(lane, k + 1), tau, v2);
      if (lane < nw) rotate2<false>(u(lane, k), u(lane, k + 1), tau, v2);
    }
  }
  __syncwarp();
  return true;
}

// Swaps the adjacent diagonal entries k, k+1 of the upper triangular T and
// updates U (LAPACK xTREXC's step: T <- G T G^H, U <- U G^H).  One warp.
__device__ void schur_swap_warp(cplx* T, cplx* U, int nw, int k, int lane) {
  auto t = [&](int r, int c) -> cplx& { return T[c * ALD + r]; };
  auto u = [&](int r, int c) -> cplx& { return U[c * ALD + r]; };
  const cplx t11 = t(k, k), t22 = t(k + 1, k + 1);
  double cs;
  cplx sn;
  givens(t(k, k + 1), csub(t22, t11), &cs, &sn);
  const cplx snc = cconj(sn);
  __syncwarp();
  const int j = k + 2 + lane;
  if (j < nw) {  // rows k, k+1 over columns k+2..nw-1
    const cplx x = t(k, j), y = t(k + 1, j);
    t(k, j) = cadd(cscale(x, cs), cmul(sn, y));
    t(k + 1, j) = csub(cscale(y, cs), cmul(snc, x));
  }
  if (lane < k) {  // columns k, k+1 over rows 0..k-1
    const cplx x = t(lane, k), y = t(lane, k + 1);
    t(lane, k) = cadd(cscale(x, cs), cmul(snc, y));
    t(lane, k + 1) = csub(cscale(y, cs), cmul(sn, x));
  }
  if (lane < nw) {
    const cplx x = u(lane, k), y = u(lane, k + 1);
    u(lane, k) = cadd(cscale(x, cs), cmul(snc, y));
    u(lane, k + 1) = csub(cscale(y, cs), cmul(sn, x));
  }
  __syncwarp();
  if (lane == 0) {
    t(k, k) = t22;
    t(k + 1, k + 1) = t11;
  }
  __syncwarp();
}

// Reflector I - tau v v^H (v in shared memory, v[0] = 1) from the left,
// conjugated, on rows r0..r0+len-1 of T over columns c0..nc-1, and from the
// right on columns c0'..c0'+len-1 of a matrix over rows 0..nr-1.
__device__ __forceinline__ void refl_left_warp(cplx* T, const cplx* v, int r0, int len, cplx tau, int c0, int nc,
                                               int lane) {
  const int c = c0 + lane;
  if (c < nc) {
    cplx w = mk(0.0, 0.0);
    for (int q = 0; q < len; ++q) w = cadd(w, cmulc(v[q], T[c * ALD + r0 + q]));
    w = cmul(cconj(tau), w);
    for (int q = 0; q < len; ++q) T[c * ALD + r0 + q] = csub(T[c * ALD + r0 + q], cmul(v[q], w));
  }
}
__device__ __forceinline__ void refl_right_warp(cplx* M, const cplx* v, int c0, int len, cplx tau, int nr,
                                                int lane) {
  if (lane < nr) {
    cplx w = mk(0.0, 0.0);
    for (int q = 0; q < len; ++q) w = cadd(w, cmul(M[(c0 + q) * ALD + lane], v[q]));
    w = cmul(tau, w);
    for (int q = 0; q < len; ++q) M[(c0 + q) * ALD + lane] = csub(M[(c0 + q) * ALD + lane], cmul(w, cconj(v[q])));
  }
}

// Warp sum of a real value.
__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// The deflation window's analysis by one warp (after small_schur_warp):
// deflation of the eigenvalues with negligible spike entries, reordering of
// the others to the top, their values into ev[0..ns-1], and, if anything
// deflated, the return of the top ns x ns block to Hessenberg form.
// Returns ns, the number of undeflated eigenvalues.
__device__ int aed_deflate_warp(cplx* T, cplx* U, cplx* v, cplx* ev, int nw, cplx s0, int lane, double smlnum) {
  auto t = [&](int r, int c) -> cplx& { return T[c * ALD + r]; };
  auto u = [&](int r, int c) -> cplx& { return U[c * ALD + r]; };
  int ns = nw, ilst = 0;
  const double as0 = cabs1(s0);
  for (int knt = 0; knt < nw; ++knt) {
    double foo = cabs1(t(ns - 1, ns - 1));
    if (foo == 0.0) foo = as0;
    if (as0 * cabs1(u(0, ns - 1)) <= fmax(smlnum, EIG_ULP * foo)) {
      --ns;  // converged: stays below the undeflated block
    } else {
      for (int k = ns - 2; k >= ilst; --k) schur_swap_warp(T, U, nw, k, lane);  // move it to position ilst
      ++ilst;
    }
  }
  if (lane < ns) ev[lane] = t(lane, lane);
  __syncwarp();
  if (ns == nw || ns <= 1 || (s0.x == 0.0 && s0.y == 0.0)) return ns;
  // reflector taking the spike's top ns entries to a multiple of e_0
  {
    const cplx sp = lane < ns ? cmul(s0, cconj(u(0, lane))) : mk(0.0, 0.0);
    const double xn2 = warp_sum(lane >= 1 ? cabs2(sp) : 0.0);
    const cplx alpha = mk(__shfl_sync(0xffffffffu, sp.x, 0), __shfl_sync(0xffffffffu, sp.y, 0));
    double beta;
    cplx tau, scale;
    householder(alpha, xn2, &beta, &tau, &scale);
    if (lane < ns) v[lane] = lane == 0 ? mk(1.0, 0.0) : cmul(sp, scale);
    __syncwarp();
    refl_left_warp(T, v, 0, ns, tau, 0, nw, lane);
    __syncwarp();
    refl_right_warp(T, v, 0, ns, tau, ns, lane);
    refl_right_warp(U, v, 0, ns, tau, nw, lane);
    __syncwarp();
  }
  // Householder reduction of the top ns x ns block to Hessenberg form
  for (int j = 0; j + 2 < ns; ++j) {
    const int len = ns - 1 - j;  // rows j+1..ns-1
    const cplx xr = (lane >= 1 && lane < len) ? t(j + 1 + lane, j) : mk(0.0, 0.0);
    const double xn2 = warp_sum(cabs2(xr));
    const cplx alpha = t(j + 1, j);
    double beta;
    cplx tau, scale;
    householder(alpha, xn2, &beta, &tau, &scale);
    __syncwarp();  // every lane has read column j
    if (lane < len) v[lane] = lane == 0 ? mk(1.0, 0.0) : cmul(xr, scale);
    if (lane == 0) t(j + 1, j) = mk(beta, 0.0);
    if (lane >= 1 && lane < len) t(j + 1 + lane, j) = mk(0.0, 0.0);
    __syncwarp();
    refl_left_warp(T, v, j + 1, len, tau, j + 1, nw, lane);
    __syncwarp();
    refl_right_warp(T, v, j + 1, len, tau, ns, lane);
    refl_right_warp(U, v, j + 1, len, tau, nw, lane);
    __syncwarp();
  }
  return ns;
}

// MINB: resident CTAs per SM the registers are sized for; with three the
// carry chains prefetch two entries instead of four (no spills either way).
template <int MINB>
__global__ void __launch_bounds__(QR_THREADS, MINB)
    hqr_kernel(cplx* const* __restrict__ Hs, void* const* __restrict__ logs, cplx* const* __restrict__ Ws, int n,
               int sweep_cap, long long rot_cap, int* __restrict__ status, int aed_min, int aed_w) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* D = reinterpret_cast<cplx*>(smem_raw);  // [QD][QLD] column-major window
  cplx* s_tau = D + QD * QLD;                   // [NBMAX][QB]
  cplx* s_v2 = s_tau + NBMAX * QB;              // [NBMAX][QB]
  __shared__ cplx s_shift[NBMAX];
  __shared__ cplx s_small[NBMAX * NBMAX];
  __shared__ int s_red[QR_THREADS / 32];
  __shared__ int s_l, s_nb, s_nsw, s_nrot, s_over, s_nround, s_cur;
  // deflation window: reflector vector, undeflated eigenvalues, outcome
  // (undeflated count, or -1 when skipped), shifts it left for the next sweep
  __shared__ cplx s_aedv[AW], s_aedev[AW];
  __shared__ int s_aed_ns, s_pend, s_naed;
  __shared__ long long s_clk[7];  // statistics: phase timers (defl, shift, rounds, far), the last stamp,
                                  // window Schur form and window deflation

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
    s_pend = 0;
    s_naed = 0;
    s_nrot = 0;
    s_over = 0;
    s_nround = 0;
    for (int q = 0; q < 7; ++q) s_clk[q] = 0;
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
      // Aggressive early deflation on the trailing block of the window
      // (skipped at the exceptional-shift iterations and while shifts from
      // the previous one are pending).
      const bool exceptional = its == 10 || its == 20;
      if (aed_min > 0 && !exceptional && s_pend == 0 && i - l + 1 >= aed_min) {
        const int jw = min(aed_w, i - l + 1), kw = i - jw + 1;
        const cplx s0 = kw > l ? h(kw, kw - 1) : mk(0.0, 0.0);
        cplx* T = D;               // [AW][ALD]
        cplx* U = D + AW * ALD;    // [AW][ALD]
        for (int idx = tid; idx < jw * jw; idx += QR_THREADS) {
          const int c = idx / jw, r = idx - c * jw;
          T[c * ALD + r] = (r <= c + 1) ? h(kw + r, kw + c) : mk(0.0, 0.0);
          U[c * ALD + r] = mk(r == c ? 1.0 : 0.0, 0.0);
        }
        __syncthreads();
        if (warp == 0) {
          int ns = -1;
          const long long c0 = clock64();
          const bool conv = small_schur_warp(T, U, jw, lane, smlnum);
          const long long c1 = clock64();
          if (conv) ns = aed_deflate_warp(T, U, s_aedv, s_aedev, jw, s0, lane, smlnum);
          if (lane == 0) {
            s_clk[5] += c1 - c0;
            s_clk[6] += clock64() - c1;
            // a deflation is logged as a dense jw x jw block; without room, skip it
            if (ns >= 0 && ns < jw &&
                (s_nsw + 1 > sweep_cap || (long long)s_nrot + (jw * jw + 1) / 2 > rot_cap))
              ns = -1;
            s_aed_ns = ns;
          }
        }
        __syncthreads();
        const int ns = s_aed_ns;
        if (ns >= 0 && ns < jw) {
          // write the block back, the spike's first entry left of it
          for (int idx = tid; idx < jw * jw; idx += QR_THREADS) {
            const int c = idx / jw, r = idx - c * jw;
            h(kw + r, kw + c) = T[c * ALD + r];
          }
          if (tid == 0 && kw > l) h(kw, kw - 1) = ns > 0 ? cmul(s0, cconj(U[0])) : mk(0.0, 0.0);
          // rows l..kw-1 of the window: H[r, kw:i] <- H[r, kw:i] U (a warp per row)
          for (int r = l + warp; r < kw; r += QR_THREADS / 32) {
            const cplx hv = lane < jw ? h(r, kw + lane) : mk(0.0, 0.0);
            cplx acc = mk(0.0, 0.0);
            for (int k = 0; k < jw; ++k) {
              const cplx x = mk(__shfl_sync(0xffffffffu, hv.x, k), __shfl_sync(0xffffffffu, hv.y, k));
              if (lane < jw) acc = cfma(x, U[lane * ALD + k], acc);
            }
            if (lane < jw) h(r, kw + lane) = acc;
          }
          // the dense log entry: U column-major (leading dimension jw)
          const int start = s_nrot;
          for (int idx = tid; idx < jw * jw; idx += QR_THREADS) {
            const int c = idx / jw, r = idx - c * jw;
            rot[2 * (size_t)start + idx] = U[c * ALD + r];
          }
          __syncthreads();
          if (tid == 0) {
            sweeps[s_nsw] = QrSweep{l, i, -1, jw, start, kw, 0, 0};
            s_nsw += 1;
            s_nrot += (jw * jw + 1) / 2;
            s_naed += 1;
          }
        }
        if (ns >= 0) {
          // shifts: up to NBMAX undeflated eigenvalues of the block, the
          // smallest in magnitude (LAPACK xLAQR0's choice); ranks by a warp
          const int ie = i - (jw - ns);
          const int want = min(NBMAX, max(1, (ie - l + 1 - 4) / 6));
          if (warp == 0 && ns >= 1) {
            const int nsh = min(want, ns);
            if (lane < ns) {
              const double me = cabs1(s_aedev[lane]);
              int rank = 0;
              for (int q = 0; q < ns; ++q) {
                const double o = cabs1(s_aedev[q]);
                rank += (o < me || (o == me && q < lane)) ? 1 : 0;
              }
              if (rank < nsh) s_shift[rank] = s_aedev[lane];
            }
            if (lane == 0) s_pend = nsh;
          }
          __syncthreads();
          // many deflations: skip the sweep and look again (LAPACK's 14%)
          if (ns < jw && 100 * (jw - ns) > 14 * jw) {
            if (tid == 0) s_pend = 0;
            __syncthreads();
          }
          // a deflation: isolate the deflated eigenvalues first (the shifts wait)
          if (ns < jw) {
            if (tid == 0) stamp(1);
            continue;
          }
        }
      }
      // Number of bulges and their shifts.
      if (warp == 0) {
        const int w = i - l + 1;
        const int pend = exceptional ? 0 : s_pend;  // shifts left by the deflation window
        const int nb0 = exceptional ? 1 : min(NBMAX, max(1, (w - 4) / 6));
        const int nb = pend > 0 ? min(nb0, pend) : nb0;
        if (pend > 0) {
        } else if (nb == 1) {
          if (lane == 0) s_shift[0] = single_shift(H, n, l, i, its);
        } else {
          const int b0 = i - nb + 1;
          for (int idx = lane; idx < nb * nb; idx += 32) {
            const int c = idx / nb, r = idx - c * nb;
            s_small[c * nb + r] = (r <= c + 1) ? h(b0 + r, b0 + c) : mk(0.0, 0.0);
          }
          small_eigvals_warp(s_small, nb, s_shift, lane);
        }
        __syncwarp();  // every lane has read s_pend
        if (lane == 0) {
          s_nb = nb;
          s_pend = 0;
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
          if (lane == 0 && mine && !(k >= m && k <= i - 1)) {  // outside the window: the identity
            s_tau[a * QB + (r - r0)] = mk(0.0, 0.0);
            s_v2[a * QB + (r - r0)] = mk(0.0, 0.0);
          }
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
    hdr->naed = s_naed;
    hdr->t_defl = s_clk[0];
    hdr->t_shift = s_clk[1];
    hdr->t_rounds = s_clk[2];
    hdr->t_far = s_clk[3];
    hdr->t_wschur = s_clk[5];
    hdr->t_wdefl = s_clk[6];
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

constexpr int RS = 4 * RotRing<RP_NBG, RP_PFD, false, RP_THREADS>::P;  // rounds per slab (a multiple of the ring size)
// staged rotations of a slab, or one deflation-window block (AW x AW)
constexpr int RP_ROT = RS * NBMAX * 2 > AW * AW ? RS * NBMAX * 2 : AW * AW;
constexpr size_t RP_SMEM = (size_t)RP_ROT * sizeof(cplx) + (size_t)(RP_PFD + 1) * RP_THREADS * sizeof(cplx);

// A deflation-window block on one vector: x[kw..kw+jw-1] <- U^H x (row
// transforms, ROWOP) or x U (column transforms); U in shared memory, AW x AW
// column-major, zero outside jw x jw.
template <bool ROWOP>
__device__ __noinline__ void replay_block(cplx* x, size_t stride, int kw, int jw, const cplx* U) {
  cplx v[AW];
#pragma unroll
  for (int k = 0; k < AW; ++k) v[k] = k < jw ? x[(size_t)(kw + k) * stride] : mk(0.0, 0.0);
  for (int j = 0; j < jw; ++j) {
    cplx acc = mk(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < AW; ++k) {
      const cplx u = U[j * AW + k];
      acc = ROWOP ? cadd(acc, cmulc(u, v[k])) : cfma(v[k], u, acc);
    }
    x[(size_t)(kw + j) * stride] = acc;
  }
}

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
    if (nb < 0) {  // deflation-window block
      const int jw = q.R;
      __syncthreads();  // the previous slab is consumed
      for (int e = threadIdx.x; e < AW * AW; e += blockDim.x) {
        const int c = e / AW, r = e - c * AW;
        s_rot[e] = (r < jw && c < jw) ? ld(src + (size_t)c * jw + r) : mk(0.0, 0.0);
      }
      __syncthreads();
      if (active) replay_block<ROWOP>(x, stride, q.pad0, jw, s_rot);
      continue;
    }
    for (int b0 = 0; b0 < nb; b0 += RP_NBG) {
      const int ng = min(RP_NBG, nb - b0);
      RotRing<RP_NBG, RP_PFD, ROWOP, RP_THREADS> ring;
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
        if (active)
          ring.run(t0, t0 + nr, [&](int t, int g, cplx& tau, cplx& v2) {
            const cplx* rr = s_rot + 2 * RP_NBG * (t - t0);
            tau = rr[2 * g];
            v2 = rr[2 * g + 1];
          });
      }
    }
  }
}

__global__ void __launch_bounds__(RP_THREADS, 4)
    qr_replay_rows_kernel(cplx* const* __restrict__ Hs, cplx* const* __restrict__ Zs,
                          void* const* __restrict__ logs, int n, int sweep_cap, int row_blocks) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* s_rot = reinterpret_cast<cplx*>(smem_raw);
  cplx* s_pf = s_rot + RP_ROT;
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
  cplx* s_pf = s_rot + RP_ROT;
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
  // order of the deflation window (VRC_QR_AEDW, 4..32): measured on B200,
  // 12 balances the window's cost (one warp) against the sweeps it saves
  static const int aed_w_env = [] {
    const char* e = std::getenv("VRC_QR_AEDW");
    return e ? std::min(AW, std::max(4, std::atoi(e))) : 0;
  }();
  const int aed_w = aed_w_env ? aed_w_env : 12;
  // aggressive early deflation on active windows of at least this order
  // (VRC_QR_AED; 0 turns it off; by default the window's order for n > 128,
  // off below, where the sweeps it saves cost less than the windows)
  static const int aed_env = [] {
    const char* e = std::getenv("VRC_QR_AED");
    return e ? std::max(0, std::atoi(e)) : -1;
  }();
  const int aed_min = aed_env >= 0 ? aed_env : (n <= 128 ? 0 : aed_w);
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
                                                  d_status ? d_status + b0 : nullptr, aed_min, aed_w);
    if (parts & SCHUR_REPLAY) {
      qr_replay_rows_kernel<<<dim3(2 * row_blocks, nb), RP_THREADS, rp_smem, st>>>(d_H + b0, d_Z + b0, d_logs + b0,
                                                                                  n, cc, row_blocks);
      qr_replay_cols_kernel<<<dim3(row_blocks, nb), RP_THREADS, rp_smem, st>>>(d_H + b0, d_logs + b0, n, cc);
    }
  }
  VRC_CUDA_CHECK(cudaGetLastError());
}

}  // namespace vrc
