// The generic J/K path (declarations and scope in jk_generic.cuh): shell quartets with an f
// shell, or with any shell layout the generated class kernels do not cover, by
// McMurchie-Davidson with run-time angular momenta.
//
// Per quartet (PQ|IJ) and primitive quartet (ij|kl), as the class kernels do it but with loops:
//   (ab|cd) = sum_tuv E^ab_tuv sum_tau,nu,phi (-1)^(tau+nu+phi) E^cd_tau,nu,phi R_{t+tau,u+nu,v+phi}
// with E the products of 1-D Hermite coefficients (times contraction weights and
// exp(-ab|AB|^2/p)/p), R^(0) from the Hermite recursion seeded by
// 2 pi^(5/2) / sqrt(p+q) (-2 alpha)^n F_n(alpha |PQ|^2).  The ket side is summed over the ket
// primitives first, G[tuv][cd], and transformed by the bra E once per bra primitive.  The
// screens (Schwarz outer/fixed cutoffs, density screen below dscreen_rmax, the 1e-15 primitive
// prefactor cut) and the digestion into J, KA, KB with the 8-fold degeneracy factors are those
// of the class kernels (GTO_JK_Matrix_Quartet_Parallel and storeQuartetEE, reference
// src/matrix.c:3773-3986, 2934-3396), so the two paths add into the same accumulators.
//
// Layout: the 1-D Hermite tables and contraction weights of every primitive pair and the
// component descriptors of every function pair are computed on the host and read through L1;
// one warp per quartet, two warps per CTA, each warp with a shared-memory region holding the
// Boys-scaled seeds, two buffers of the R recursion (tetrahedral order t+u+v <= 12), and G and
// the contracted block O for a chunk of ket function pairs (chunks when a (ff|ff)-sized block
// does not fit).
#include "jk_generic.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "jk_common.cuh"
#include "../../include/sqb200.h"

namespace sqb {
int set_error(int code, const std::string& msg);
std::vector<double> boys_table(int ncol);
}  // namespace sqb

namespace {

using sqb::GenItem;
using sqb::GenPairRec;
using sqb::kGenPrimStride;

using sqb::kGenBoysCols;
constexpr int kGenR = 455;                             // tetrahedral entries with t+u+v <= 12
constexpr int kGenWarps = 2;                           // warps per CTA
constexpr int kGenKets = 16;                           // kets per work item
constexpr int kGenGO = 1024;                           // doubles for G and O of one chunk
constexpr int kGenWarpDoubles = 16 + 2 * kGenR + kGenGO;
constexpr size_t kGenSmem = (size_t)kGenWarps * kGenWarpDoubles * sizeof(double);   // 31,200 B

static_assert(sqb::kGenMmax == 12 && (sqb::kGenMmax + 1) * (sqb::kGenMmax + 2) * (sqb::kGenMmax + 3) / 6 == kGenR,
              "R table size");
static_assert(sizeof(GenPairRec) == 56, "pair record layout");
static_assert(kGenSmem <= 48 * 1024, "the generic kernels launch without a shared-memory opt-in");

// (t, u, v) of tetrahedral index k: order n = t+u+v, then m = u+v, then v ascending
struct TuvTable {
  unsigned int v[kGenR];
  constexpr TuvTable() : v() {
    int k = 0;
    for (int n = 0; n <= sqb::kGenMmax; ++n)
      for (int m = 0; m <= n; ++m)
        for (int w = 0; w <= m; ++w) v[k++] = (unsigned)(n - m) | ((unsigned)(m - w) << 8) | ((unsigned)w << 16);
  }
};
__device__ const TuvTable g_tuv = TuvTable();

__device__ __forceinline__ int gtet(int t, int u, int v) {
  const int n = t + u + v, m = u + v;
  return n * (n + 1) * (n + 2) / 6 + m * (m + 1) / 2 + v;
}

struct GenArgs {
  const GenPairRec* __restrict__ pairs;
  const double* __restrict__ prims;
  const double* __restrict__ coef;      // per primitive pair: 1-D Hermite tables, then weights
  const int* __restrict__ desc;         // per pair: component descriptor of each function pair
  const double* __restrict__ boys;
  sqb::GenBuild b;
  unsigned long long* counters;
};

// A primitive pair's tables in `coef`: axis d, E^{ij}_t at e + d*sz + (i*lq1 + j)*lt + t
// (i <= lP, j <= lQ, t <= i+j; lq1 = lQ+1, lt = lP+lQ+1, sz = (lP+1) lq1 lt); then the weights
// c_a c_b exp(-ab|AB|^2/p)/p of its function pairs at e + 3*sz.
struct EView {
  const double* e;
  int lq1, lt, sz;
  __device__ EView(const double* coef, const double* rec, const GenPairRec& P)
      : e(coef + (long long)rec[11]), lq1(P.lQ + 1), lt(P.lP + P.lQ + 1), sz((P.lP + 1) * (P.lQ + 1) * (P.lP + P.lQ + 1)) {}
  __device__ __forceinline__ const double* ax(int d, int i, int j) const { return e + d * sz + (i * lq1 + j) * lt; }
  __device__ __forceinline__ double w(int ab) const { return __ldg(e + 3 * sz + ab); }
};

// component exponents of a function pair: a_x, b_x, a_y, b_y, a_z, b_z in 2 bits each
__device__ __forceinline__ int dsc(unsigned d, int k) { return (d >> (2 * k)) & 3; }

// F_n(T) for one order n <= 12: below BOYS_TMAX the 9-term Taylor expansion about the nearest
// grid point, F_n(T0+d) = sum_k F_{n+k}(T0) (-d)^k / k!, from the table's own column n; above,
// F_0 = sqrt(pi/T)/2 and the upward recursion F_{m+1} = ((2m+1) F_m - e^-T)/(2T).
__device__ double gen_boys(int n, double T, const double* __restrict__ tab) {
  if (T < BOYS_TMAX) {
    const int g = __double2int_rn(T * BOYS_INV_H);
    const double d = T - g * BOYS_H;
    const double* row = tab + g * kGenBoysCols + n;
    double s = __ldg(row + BOYS_NTAY - 1);
    for (int k = BOYS_NTAY - 2; k >= 0; --k) s = fma(s, -d * (1.0 / (double)(k + 1)), __ldg(row + k));
    return s;
  }
  const double it = 1.0 / T;
  double F = 0.88622692545275801365 * sqrt(it);   // sqrt(pi)/2 / sqrt(T)
  if (n > 0) {
    const double e = exp(-T), h = 0.5 * it;
    for (int m = 0; m < n; ++m) F = ((2 * m + 1) * F - e) * h;
  }
  return F;
}

// Seeds base[n] = 2 pi^(5/2)/sqrt(p+q) (-2 alpha)^n F_n(T), n <= L, one lane per order.
__device__ __forceinline__ void gen_seeds(int L, double alpha, double rs, double T, const double* tab, double* base,
                                          int lane) {
  if (lane <= L) {
    const double m2a = -2.0 * alpha;
    double w = TWO_PI_2_5 * rs;
    for (int k = 0; k < lane; ++k) w *= m2a;
    base[lane] = w * gen_boys(lane, T, tab);
  }
}

// R^(0)_{tuv}, t+u+v <= L, from the seeds by the Hermite recursion
//   R^(n)_{t+1,u,v} = t R^(n+1)_{t-1,u,v} + X R^(n+1)_{t,u,v}   (likewise in u, v),
// level by level from n = L down to 0, the lanes sharing each level; returns the buffer that
// holds level 0.  The seeds must be visible to the warp (synchronised) before the call.
__device__ const double* gen_rtab(int L, double X, double Y, double Z, const double* base, double* b0, double* b1,
                                  int lane) {
  double* cur = b0;
  double* nxt = b1;
  if (lane == 0) cur[0] = base[L];
  __syncwarp();
  for (int n = L - 1; n >= 0; --n) {
    const int top = L - n;
    const int cnt = (top + 1) * (top + 2) * (top + 3) / 6;
    for (int idx = lane; idx < cnt; idx += 32) {
      const unsigned e = g_tuv.v[idx];
      const int t = e & 255, u = (e >> 8) & 255, v = e >> 16;
      double r;
      if (idx == 0) r = base[n];
      else if (t > 0) r = X * cur[gtet(t - 1, u, v)] + (t > 1 ? (t - 1) * cur[gtet(t - 2, u, v)] : 0.0);
      else if (u > 0) r = Y * cur[gtet(t, u - 1, v)] + (u > 1 ? (u - 1) * cur[gtet(t, u - 2, v)] : 0.0);
      else r = Z * cur[gtet(t, u, v - 1)] + (v > 1 ? (v - 1) * cur[gtet(t, u, v - 2)] : 0.0);
      nxt[idx] = r;
    }
    __syncwarp();
    double* tmp = cur;
    cur = nxt;
    nxt = tmp;
  }
  return cur;
}

// sum_{tau,nu,phi} (-1)^(tau+nu+phi) E_x[tau] E_y[nu] E_z[phi] R_{t+tau,u+nu,v+phi}; the
// tetrahedral index of R steps along phi by increments (n = t+u+v and m = u+v both rise by one)
__device__ __forceinline__ double ket_sum(const double* __restrict__ ex, const double* __restrict__ ey,
                                          const double* __restrict__ ez, int nx, int ny, int nz, int t, int u, int v,
                                          const double* R) {
  double s = 0.0;
  for (int tau = 0; tau <= nx; ++tau) {
    const double et = __ldg(ex + tau);
    for (int nu = 0; nu <= ny; ++nu) {
      const int U = u + nu;
      int n = t + tau + U + v, m = U + v;
      int idx = n * (n + 1) * (n + 2) / 6 + m * (m + 1) / 2 + v;
      int dn = (n + 1) * (n + 2) / 2;                // tet(n+1) - tet(n)
      double sz = 0.0;
      for (int ph = 0; ph <= nz; ++ph) {
        const double e = __ldg(ez + ph);
        sz = fma((ph & 1) ? -e : e, R[idx], sz);
        idx += dn + m + 2;
        dn += n + 2;
        ++n;
        ++m;
      }
      const double en = __ldg(ey + nu);
      s = fma(((tau + nu) & 1) ? -et * en : et * en, sz, s);
    }
  }
  return s;
}

// J, KA (and KB) contributions of one contracted chunk O[ab][cc] (bra function pairs ab, ket
// function pairs cd = c0 + cc), in the class kernels' convention:
//   J[pq] += 2 deg sum O PT[ij],  J[ij] += 2 deg sum O PT[pq],
//   K[p][i] += deg O D[q][j],  K[q][i] += deg O D[p][j],  K[p][j] += deg O D[q][i],
//   K[q][j] += deg O D[p][i]   (D = PA into KA; PB into KB when unrestricted).
__device__ void gen_digest(const GenArgs& a, const GenPairRec& A, const GenPairRec& B, double deg, const double* O,
                           int c0, int nc, int lane) {
  const int N = a.b.nbf;
  const int nfP = A.nfP, nfQ = A.nfQ, nfJ = B.nfQ;
  const int fP = A.fP, fQ = A.fQ, fI = B.fP, fJ = B.fQ;
  const int nA = nfP * nfQ;
  const double* __restrict__ PT = a.b.PT;
  const double s2 = 2.0 * deg;
  for (int cc = lane; cc < nc; cc += 32) {
    const int cd = c0 + cc, ic = cd / nfJ, jd = cd - ic * nfJ;
    double s = 0.0;
    for (int ab = 0; ab < nA; ++ab) {
      const int p = ab / nfQ, q = ab - p * nfQ;
      s = fma(O[ab * nc + cc], PT[(size_t)(fP + p) * N + fQ + q], s);
    }
    atomicAdd(a.b.J + (size_t)(fI + ic) * N + fJ + jd, s2 * s);
  }
  for (int ab = lane; ab < nA; ab += 32) {
    const int p = ab / nfQ, q = ab - p * nfQ;
    double s = 0.0;
    for (int cc = 0; cc < nc; ++cc) {
      const int cd = c0 + cc, ic = cd / nfJ, jd = cd - ic * nfJ;
      s = fma(O[ab * nc + cc], PT[(size_t)(fI + ic) * N + fJ + jd], s);
    }
    atomicAdd(a.b.J + (size_t)(fP + p) * N + fQ + q, s2 * s);
  }
  const int i0 = c0 / nfJ, i1 = (c0 + nc - 1) / nfJ, ni = i1 - i0 + 1;   // ket rows in the chunk
  for (int ks = 0; ks < (a.b.uhf ? 2 : 1); ++ks) {
    const double* __restrict__ D = ks ? a.b.PB : a.b.PA;
    double* K = ks ? a.b.KB : a.b.KA;
    // K[p][i] (x = p, y = q) and K[q][i] (x = q, y = p): sums over y and the chunk's j
    for (int e = lane; e < (nfP + nfQ) * ni; e += 32) {
      const bool onP = e < nfP * ni;
      const int e2 = onP ? e : e - nfP * ni;
      const int x = e2 / ni, ic = i0 + (e2 - (e2 / ni) * ni);
      const int jlo = max(0, c0 - ic * nfJ), jhi = min(nfJ, c0 + nc - ic * nfJ);
      const int ny = onP ? nfQ : nfP;
      double s = 0.0;
      for (int y = 0; y < ny; ++y) {
        const int ab = onP ? x * nfQ + y : y * nfQ + x;
        const int fy = onP ? fQ + y : fP + y;
        for (int jd = jlo; jd < jhi; ++jd) s = fma(O[ab * nc + ic * nfJ + jd - c0], D[(size_t)fy * N + fJ + jd], s);
      }
      atomicAdd(K + (size_t)((onP ? fP : fQ) + x) * N + fI + ic, deg * s);
    }
    // K[p][j] and K[q][j]: sums over y and the chunk's i
    for (int e = lane; e < (nfP + nfQ) * nfJ; e += 32) {
      const bool onP = e < nfP * nfJ;
      const int e2 = onP ? e : e - nfP * nfJ;
      const int x = e2 / nfJ, jd = e2 - x * nfJ;
      const int ny = onP ? nfQ : nfP;
      double s = 0.0;
      for (int y = 0; y < ny; ++y) {
        const int ab = onP ? x * nfQ + y : y * nfQ + x;
        const int fy = onP ? fQ + y : fP + y;
        for (int ic = i0; ic <= i1; ++ic) {
          const int cd = ic * nfJ + jd;
          if (cd < c0 || cd >= c0 + nc) continue;
          s = fma(O[ab * nc + cd - c0], D[(size_t)fy * N + fI + ic], s);
        }
      }
      atomicAdd(K + (size_t)((onP ? fP : fQ) + x) * N + fJ + jd, deg * s);
    }
  }
}

// Largest |O - monopole value| over a chunk (multipole-mode error measurement).
__device__ double gen_mpole_err(const GenArgs& a, const GenPairRec& A, const GenPairRec& B, const double* O, int c0,
                                int nc, int lane) {
  const int nfQ = A.nfQ, nfJ = B.nfQ, nA = A.nfP * nfQ;
  double e = 0.0;
  for (int x = lane; x < nA * nc; x += 32) {
    const int ab = x / nc, cc = x - ab * nc, cd = c0 + cc;
    const int pp = ab / nfQ, ic = cd / nfJ;
    const double m = sqb::mpole_value(a.b.mpole, a.b.nbf, A.fP + pp, A.fQ + ab - pp * nfQ, B.fP + ic, B.fQ + cd - ic * nfJ);
    e = fmax(e, fabs(O[x] - m));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
  return e;
}

// One shell quartet (A|B) by one warp; W is the warp's shared-memory region.  npq counts the
// primitive quartets that pass the prefactor cut (first chunk only).  Multipole mode: mpq
// substitutes the monopole values for the integrals (no primitive work), erx >= 0 records the
// largest monopole error of the exact block in the bank's scratch.
__device__ void gen_quartet(const GenArgs& a, const GenPairRec& A, const GenPairRec& B, double deg, double* W, int lane,
                            unsigned long long& npq, bool mpq, int erx, unsigned long long& nfl) {
  double* base = W;
  double* R0 = base + 16;
  double* R1 = R0 + kGenR;
  double* G = R1 + kGenR;
  const int nfQ = A.nfQ, nfJ = B.nfQ;
  const int nA = A.nfP * nfQ, nB = B.nfP * nfJ;
  const int LA = A.lP + A.lQ, LB = B.lP + B.lQ, L = LA + LB;
  const int nHA = (LA + 1) * (LA + 2) * (LA + 3) / 6;
  const int ncm = min(nB, kGenGO / (nA + nHA));
  double* O = G + nHA * ncm;
  for (int c0 = 0; c0 < nB; c0 += ncm) {
    const int nc = min(ncm, nB - c0);
    if (mpq) {
      for (int e = lane; e < nA * nc; e += 32) {
        const int ab = e / nc, cd = c0 + e - (e / nc) * nc;
        const int pp = ab / nfQ, ic = cd / nfJ;
        O[e] = sqb::mpole_value(a.b.mpole, a.b.nbf, A.fP + pp, A.fQ + ab - pp * nfQ, B.fP + ic, B.fQ + cd - ic * nfJ);
      }
      __syncwarp();
      gen_digest(a, A, B, deg, O, c0, nc, lane);
      __syncwarp();
      continue;
    }
    // lane steps through the entries of a block: 32 = dq*nc + dr (O, column fastest) and
    // 32 = dc*nHA + dh (G, Hermite index fastest)
    const int dq = 32 / nc, dr = 32 - dq * nc;
    const int dc = 32 / nHA, dh = 32 - dc * nHA;
    for (int e = lane; e < nA * nc; e += 32) O[e] = 0.0;
    for (int i = 0; i < A.nprim; ++i) {
      const double* pa = a.prims + (size_t)(A.poff + i) * kGenPrimStride;
      const double p = pa[0], Px = pa[1], Py = pa[2], Pz = pa[3], kpa = pa[4];
      const EView Ei(a.coef, pa, A);
      __syncwarp();                                  // the previous O step is done with G
      for (int e = lane; e < nHA * nc; e += 32) G[e] = 0.0;
      bool any = false;
      for (int j = 0; j < B.nprim; ++j) {
        const double* pb = a.prims + (size_t)(B.poff + j) * kGenPrimStride;
        const double q = pb[0], kpb = pb[4];
        const double pq = p + q, rs = rsqrt(pq);
        if (TWO_PI_2_5 * kpa * kpb * rs < PRIM_CUTOFF) continue;
        any = true;
        if (c0 == 0) ++npq;
        const double alpha = p * q * (rs * rs);
        const double X = Px - pb[1], Y = Py - pb[2], Z = Pz - pb[3];
        const double T = alpha * fma(X, X, fma(Y, Y, Z * Z));
        __syncwarp();                                // the previous G step is done with R
        gen_seeds(L, alpha, rs, T, a.boys, base, lane);
        __syncwarp();
        const double* R = gen_rtab(L, X, Y, Z, base, R0, R1, lane);
        // operations of the Boys seeds (about 20 per order) and of the R recursion (3 per entry)
        if (lane == 0) {
          unsigned long long r = 20ull * (L + 1);
          for (int top = 1; top <= L; ++top) r += 3ull * (top + 1) * (top + 2) * (top + 3) / 6;
          nfl += r;
        }
        const EView Ej(a.coef, pb, B);
        // Hermite index fastest across the lanes: neighbouring lanes share a ket function pair,
        // so the loop bounds of ket_sum agree across them
        int cc = lane / nHA, h = lane - (lane / nHA) * nHA;
        for (int e = lane; e < nHA * nc; e += 32) {
          const unsigned tv = g_tuv.v[h];
          const int t = tv & 255, u = (tv >> 8) & 255, v = tv >> 16;
          const int cd = c0 + cc;
          const unsigned d = __ldg(a.desc + B.doff + cd);
          const int cx = dsc(d, 0), dx = dsc(d, 1), cy = dsc(d, 2), dy = dsc(d, 3), cz = dsc(d, 4), dz = dsc(d, 5);
          const double s = ket_sum(Ej.ax(0, cx, dx), Ej.ax(1, cy, dy), Ej.ax(2, cz, dz), cx + dx, cy + dy, cz + dz,
                                   t, u, v, R);
          G[h * nc + cc] = fma(Ej.w(cd), s, G[h * nc + cc]);
          nfl += 2ull * ((cx + dx + 1) * (cy + dy + 1) * (cz + dz + 2) + 1);
          h += dh;
          cc += dc;
          if (h >= nHA) { h -= nHA; ++cc; }
        }
      }
      __syncwarp();
      if (!any) continue;
      int ab = lane / nc, cc = lane - (lane / nc) * nc;
      for (int e = lane; e < nA * nc; e += 32) {
        const unsigned d = __ldg(a.desc + A.doff + ab);
        const int ax = dsc(d, 0), bx = dsc(d, 1), ay = dsc(d, 2), by = dsc(d, 3), az = dsc(d, 4), bz = dsc(d, 5);
        const double* ex = Ei.ax(0, ax, bx);
        const double* ey = Ei.ax(1, ay, by);
        const double* ez = Ei.ax(2, az, bz);
        double s = 0.0;
        for (int t = 0; t <= ax + bx; ++t)
          for (int u = 0; u <= ay + by; ++u) {
            // G row gtet(t, u, v) for v = 0, 1, ...: n = t+u+v and m = u+v rise together
            int n = t + u, m = u;
            int row = n * (n + 1) * (n + 2) / 6 + m * (m + 1) / 2;
            int dn = (n + 1) * (n + 2) / 2;
            double sz = 0.0;
            for (int v = 0; v <= az + bz; ++v) {
              sz = fma(__ldg(ez + v), G[row * nc + cc], sz);
              row += dn + m + 2;
              dn += n + 2;
              ++n;
              ++m;
            }
            s = fma(__ldg(ex + t) * __ldg(ey + u), sz, s);
          }
        O[e] = fma(Ei.w(ab), s, O[e]);
        nfl += 2ull * ((ax + bx + 1) * (ay + by + 1) * (az + bz + 2) + 1);
        ab += dq;
        cc += dr;
        if (cc >= nc) { cc -= nc; ++ab; }
      }
    }
    __syncwarp();
    if (erx >= 0) {
      const double e = gen_mpole_err(a, A, B, O, c0, nc, lane);
      if (lane == 0) atomicMax(a.b.erscr + erx, (unsigned long long)__double_as_longlong(e) | (1ull << 63));
    }
    gen_digest(a, A, B, deg, O, c0, nc, lane);
    // digestion: two J and four K products per integral and spin
    if (lane == 0) nfl += 2ull * nA * nc * (2 + 4 * (a.b.uhf ? 2 : 1));
    __syncwarp();
  }
}

__global__ void __launch_bounds__(32 * kGenWarps) k_jk_gen(const GenArgs a, const GenItem* __restrict__ items) {
  extern __shared__ double gsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* W = gsm + warp * kGenWarpDoubles;
  const GenItem it = items[blockIdx.x];
  const GenPairRec A = a.pairs[it.bra];
  unsigned long long nq = 0, npq = 0, nfl = 0;
  for (int kk = warp; kk < it.cnt; kk += kGenWarps) {
    const int kb = it.k0 + kk;
    const GenPairRec B = a.pairs[kb];
    if (B.gen && kb < it.bra) continue;              // two generic pairs: taken once, from the later one
    const double r = A.schwarz * B.schwarz;
    bool ok = !(r < a.b.cut_outer) && !(r < a.b.cut_fixed);
    // multipole mode: the quartet's bank slot and stored exponent; a known exponent below the
    // cache bound makes it a substitution candidate (the class kernels' rule)
    int erx = -1, erexp = sqb::ERR_UNKNOWN;
    if (ok && a.b.erbank && it.er >= 0) { erx = it.er + kb; erexp = a.b.erbank[erx]; }
    const bool mpc = erexp != sqb::ERR_UNKNOWN && r < a.b.mp_rmax;
    bool mpq = false;
    if (ok && (r < a.b.dscreen_rmax || mpc)) {
      // density screen in the reference's orientation, pair(P,Q) >= pair(I,J)
      const bool bf = (A.P > B.P) || (A.P == B.P && A.Q >= B.Q);
      const int P = bf ? A.P : B.P, Q = bf ? A.Q : B.Q, I = bf ? B.P : A.P, J = bf ? B.Q : A.Q;
      const double* PM = a.b.PM;
      const int ns = a.b.ns;
      const double mp = PM[P * ns + Q] + PM[I * ns + J] + PM[P * ns + I] + PM[P * ns + J] + PM[Q * ns + I] + PM[Q * ns + J];
      if (r < a.b.dscreen_rmax) ok = !(r * mp < a.b.cut_fixed);
      if (ok && mpc) mpq = a.b.pow15[erexp - sqb::ERR_MIN] * mp < a.b.cut_fixed;
    }
    if (!ok) continue;
    const double deg = (A.P == A.Q ? 0.5 : 1.0) * (B.P == B.Q ? 0.5 : 1.0) * (kb == it.bra ? 0.5 : 1.0);
    ++nq;
    gen_quartet(a, A, B, deg, W, lane, npq, mpq, erexp == sqb::ERR_UNKNOWN ? erx : -1, nfl);
  }
  if (lane == 0) {
    if (nq) atomicAdd(a.counters, nq);
    if (npq) atomicAdd(a.counters + 1, npq);
  }
  // operations: every lane counted its own share
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nfl += __shfl_xor_sync(0xffffffffu, nfl, o);
  if (lane == 0) {
    if (nfl) atomicAdd(a.counters + 2, nfl);
  }
}

// sqrt|(ab|ab)| for every function pair of the generic pairs: one warp per pair, lanes over
// its function pairs, every primitive quartet of (A|A) (no prefactor cut, as create_Schwarz,
// reference src/matrix.c:389-440, evaluates the full contracted integral).
__global__ void __launch_bounds__(32 * kGenWarps) k_gen_schwarz(const GenArgs a, const int* __restrict__ gidx, int ngen,
                                                               int nbf, double* __restrict__ S) {
  extern __shared__ double gsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * kGenWarps + warp;
  if (w >= ngen) return;                             // whole warps leave together
  double* base = gsm + warp * kGenWarpDoubles;
  double* R0 = base + 16;
  double* R1 = R0 + kGenR;
  double* acc = R1 + kGenR;
  const GenPairRec A = a.pairs[gidx[w]];
  const int nfQ = A.nfQ, nA = A.nfP * nfQ, L = 2 * (A.lP + A.lQ);
  for (int e = lane; e < nA; e += 32) acc[e] = 0.0;
  for (int i = 0; i < A.nprim; ++i) {
    const double* pi = a.prims + (size_t)(A.poff + i) * kGenPrimStride;
    const double p = pi[0];
    const EView Ei(a.coef, pi, A);
    for (int j = 0; j < A.nprim; ++j) {
      const double* pj = a.prims + (size_t)(A.poff + j) * kGenPrimStride;
      const double q = pj[0];
      const double pq = p + q, rs = rsqrt(pq), alpha = p * q * (rs * rs);
      const double X = pi[1] - pj[1], Y = pi[2] - pj[2], Z = pi[3] - pj[3];
      const double T = alpha * (X * X + Y * Y + Z * Z);
      const EView Ej(a.coef, pj, A);
      __syncwarp();
      gen_seeds(L, alpha, rs, T, a.boys, base, lane);
      __syncwarp();
      const double* R = gen_rtab(L, X, Y, Z, base, R0, R1, lane);
      for (int e = lane; e < nA; e += 32) {
        const unsigned d = __ldg(a.desc + A.doff + e);
        const int ax = dsc(d, 0), bx = dsc(d, 1), ay = dsc(d, 2), by = dsc(d, 3), az = dsc(d, 4), bz = dsc(d, 5);
        const int nx = ax + bx, ny = ay + by, nz = az + bz;
        const double* ex = Ei.ax(0, ax, bx);
        const double* ey = Ei.ax(1, ay, by);
        const double* ez = Ei.ax(2, az, bz);
        double s = 0.0;
        for (int t = 0; t <= nx; ++t)
          for (int u = 0; u <= ny; ++u)
            for (int v = 0; v <= nz; ++v)
              s = fma(__ldg(ex + t) * __ldg(ey + u) * __ldg(ez + v),
                      ket_sum(Ej.ax(0, ax, bx), Ej.ax(1, ay, by), Ej.ax(2, az, bz), nx, ny, nz, t, u, v, R), s);
        acc[e] = fma(Ei.w(e) * Ej.w(e), s, acc[e]);
      }
    }
  }
  __syncwarp();
  for (int e = lane; e < nA; e += 32) {
    const int pp = e / nfQ, qq = e - pp * nfQ;
    const double v = sqrt(fabs(acc[e]));
    S[(size_t)(A.fP + pp) * nbf + A.fQ + qq] = v;
    S[(size_t)(A.fQ + qq) * nbf + A.fP + pp] = v;
  }
}

GenArgs make_args(const sqb::GenPath& g) {
  GenArgs a;
  memset(&a, 0, sizeof(a));
  a.pairs = g.d_pairs;
  a.prims = g.d_prims;
  a.coef = g.d_coef;
  a.desc = g.d_desc;
  a.boys = g.d_boys;
  a.counters = g.d_counters;
  return a;
}

}  // namespace

namespace sqb {

// 1-D Hermite coefficients E^{ij}_t (i, j <= 3, t <= i+j) of a primitive pair along one axis:
// E^{00}_0 = 1, E^{i+1,j}_t = E^{ij}_{t-1}/(2p) + X_PA E^{ij}_t + (t+1) E^{ij}_{t+1}, likewise in
// j with X_PB.
static void hermite_1d(double p, double xpa, double xpb, double E[4][4][7]) {
  memset(E, 0, sizeof(double) * 4 * 4 * 7);
  const double h = 0.5 / p;
  E[0][0][0] = 1.0;
  for (int i = 0; i <= 3; ++i)
    for (int j = 0; j <= 3; ++j) {
      if (i == 0 && j == 0) continue;
      const bool up = i > 0;
      const int si = up ? i - 1 : i, sj = up ? j : j - 1;
      const double X = up ? xpa : xpb;
      for (int t = 0; t <= i + j; ++t) {
        double v = X * E[si][sj][t];
        if (t > 0) v += h * E[si][sj][t - 1];
        if (t + 1 <= si + sj) v += (t + 1) * E[si][sj][t + 1];
        E[i][j][t] = v;
      }
    }
}

void gen_build_pairs(GenPath& g, const std::vector<GenShell>& sh, const double* schwarz, int nbf) {
  g.pairs.clear();
  g.prims.clear();
  g.coef.clear();
  g.desc.clear();
  g.gen_idx.clear();
  const int ns = (int)sh.size();
  struct Tmp { double s; int P, Q; };
  std::vector<Tmp> all;
  all.reserve((size_t)ns * (ns + 1) / 2);
  for (int P = 0; P < ns; ++P)
    for (int Q = 0; Q <= P; ++Q) {
      double r = 0.0;
      for (int p = 0; p < sh[P].nfunc; ++p)
        for (int q = 0; q < sh[Q].nfunc; ++q) r = std::max(r, schwarz[(size_t)(sh[P].first + p) * nbf + sh[Q].first + q]);
      all.push_back({r, P, Q});
    }
  std::stable_sort(all.begin(), all.end(), [](const Tmp& x, const Tmp& y) { return x.s > y.s; });
  for (const Tmp& t : all) {
    const GenShell& A = sh[t.P];
    const GenShell& B = sh[t.Q];
    GenPairRec rec;
    rec.P = t.P; rec.Q = t.Q; rec.fP = A.first; rec.fQ = B.first;
    rec.nfP = A.nfunc; rec.nfQ = B.nfunc; rec.lP = A.lmax; rec.lQ = B.lmax;
    rec.nprim = A.nprim * B.nprim;
    rec.poff = (int)(g.prims.size() / kGenPrimStride);
    rec.gen = (A.gen || B.gen) ? 1 : 0;
    rec.doff = (int)g.desc.size();
    rec.schwarz = t.s;
    for (int fa = 0; fa < A.nfunc; ++fa)
      for (int fb = 0; fb < B.nfunc; ++fb) {
        const int* la = A.lmn + 3 * fa;
        const int* lb = B.lmn + 3 * fb;
        g.desc.push_back(la[0] | lb[0] << 2 | la[1] << 4 | lb[1] << 6 | la[2] << 8 | lb[2] << 10);
      }
    const int lq1 = B.lmax + 1, lt = A.lmax + B.lmax + 1;
    // primitive data as the class kernels' pair records compute it (same expressions, so the
    // prefactor cut decides alike)
    const double ab2 = (A.x - B.x) * (A.x - B.x) + (A.y - B.y) * (A.y - B.y) + (A.z - B.z) * (A.z - B.z);
    for (int i = 0; i < A.nprim; ++i)
      for (int j = 0; j < B.nprim; ++j) {
        const double a = A.exps[i], b = B.exps[j], p = a + b;
        const double Px = (a * A.x + b * B.x) / p, Py = (a * A.y + b * B.y) / p, Pz = (a * A.z + b * B.z) / p;
        const double kp = std::exp(-a * b * ab2 / p) / p;
        const double f[kGenPrimStride] = {p, Px, Py, Pz, kp, Px - A.x, Py - A.y, Pz - A.z, Px - B.x, Py - B.y,
                                          Pz - B.z, (double)g.coef.size(), 0.0, 0.0, (double)i, (double)j};
        g.prims.insert(g.prims.end(), f, f + kGenPrimStride);
        // its 1-D Hermite tables, axis-major, [i][j][t] for i <= lP, j <= lQ; then the weights
        const double PA3[3] = {Px - A.x, Py - A.y, Pz - A.z}, PB3[3] = {Px - B.x, Py - B.y, Pz - B.z};
        for (int d = 0; d < 3; ++d) {
          double E[4][4][7];
          hermite_1d(p, PA3[d], PB3[d], E);
          for (int ii = 0; ii <= A.lmax; ++ii)
            for (int jj = 0; jj < lq1; ++jj)
              for (int tt = 0; tt < lt; ++tt) g.coef.push_back(E[ii][jj][tt]);
        }
        for (int fa = 0; fa < A.nfunc; ++fa)
          for (int fb = 0; fb < B.nfunc; ++fb) g.coef.push_back(A.coef[i * 16 + fa] * B.coef[j * 16 + fb] * kp);
      }
    if (rec.gen) g.gen_idx.push_back((int)g.pairs.size());
    g.pairs.push_back(rec);
  }
}

int gen_upload(GenPath& g, cudaStream_t st) {
  const std::vector<double> tab = boys_table(kGenBoysCols);
  struct Slot { void** dst; size_t bytes; const void* src; };
  const Slot slots[] = {
      {(void**)&g.d_pairs, g.pairs.size() * sizeof(GenPairRec), g.pairs.data()},
      {(void**)&g.d_prims, g.prims.size() * sizeof(double), g.prims.data()},
      {(void**)&g.d_coef, g.coef.size() * sizeof(double), g.coef.data()},
      {(void**)&g.d_desc, g.desc.size() * sizeof(int), g.desc.data()},
      {(void**)&g.d_gen_idx, g.gen_idx.size() * sizeof(int), g.gen_idx.data()},
      {(void**)&g.d_boys, tab.size() * sizeof(double), tab.data()},
      {(void**)&g.d_counters, 3 * sizeof(unsigned long long), nullptr},
  };
  auto rnd = [](size_t b) { return (std::max<size_t>(b, 1) + 255) / 256 * 256; };
  size_t bytes = 0;
  for (const Slot& s : slots) bytes += rnd(s.bytes);
  if (g.d_base && g.bytes != bytes) gen_free(g);
  if (!g.d_base) {
    const cudaError_t e = cudaMalloc(&g.d_base, bytes);
    if (e != cudaSuccess) {
      g.d_base = nullptr;
      return set_error(SQB200_ENOMEM, std::string("cudaMalloc (generic path): ") + cudaGetErrorString(e));
    }
    g.bytes = bytes;
  }
  std::vector<char> img(bytes, 0);
  size_t o = 0;
  for (const Slot& s : slots) {
    *s.dst = (char*)g.d_base + o;
    if (s.src && s.bytes) memcpy(img.data() + o, s.src, s.bytes);
    o += rnd(s.bytes);
  }
  cudaError_t e = cudaMemcpyAsync(g.d_base, img.data(), bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_error(SQB200_ECUDA, std::string("generic path upload: ") + cudaGetErrorString(e));
  return SQB200_OK;
}

int gen_schwarz(const GenPath& g, int nbf, double* S, cudaStream_t st) {
  if (g.gen_idx.empty()) return SQB200_OK;
  const int ngen = (int)g.gen_idx.size();
  k_gen_schwarz<<<(ngen + kGenWarps - 1) / kGenWarps, 32 * kGenWarps, kGenSmem, st>>>(make_args(g), g.d_gen_idx, ngen,
                                                                                     nbf, S);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(SQB200_ECUDA, std::string("k_gen_schwarz: ") + cudaGetErrorString(e));
  return SQB200_OK;
}

void gen_items(const GenPath& g, double outer, double fixed, std::vector<GenItem>& items, double& cost,
               long long* er_run) {
  const double cut = std::max(outer, fixed);
  const int np = (int)g.pairs.size();
  // kets with schwarz >= c / S(A) (less a relative 1e-12 that the kernel's exact test takes
  // back): a prefix of the sorted list
  auto prefix = [&](double c, double sa) {
    const double thr = c / sa * (1.0 - 1e-12);
    int lo = 0, hi = np;
    while (lo < hi) {
      const int mid = (lo + hi) / 2;
      if (g.pairs[mid].schwarz >= thr) lo = mid + 1; else hi = mid;
    }
    return lo;
  };
  for (int a : g.gen_idx) {
    const GenPairRec& A = g.pairs[a];
    if (!(A.schwarz > 0.0)) continue;
    const int lo = prefix(cut, A.schwarz);
    int er = -1;
    if (er_run) {   // slots for the outer cutoff's survivors, so the layout does not depend on `fixed`
      er = (int)*er_run;
      *er_run += prefix(outer, A.schwarz);
    }
    for (int k0 = 0; k0 < lo; k0 += kGenKets) items.push_back({a, k0, std::min(kGenKets, lo - k0), er});
    cost += (double)lo * A.nprim * A.nfP * A.nfQ * 200.0;
  }
}

int gen_launch(const GenPath& g, const GenItem* d_items, int nitems, const GenBuild& b, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(g.d_counters, 0, 3 * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return set_error(SQB200_ECUDA, std::string("generic counters: ") + cudaGetErrorString(e));
  if (nitems <= 0) return SQB200_OK;
  GenArgs a = make_args(g);
  a.b = b;
  k_jk_gen<<<nitems, 32 * kGenWarps, kGenSmem, st>>>(a, d_items);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(SQB200_ECUDA, std::string("k_jk_gen: ") + cudaGetErrorString(e));
  return SQB200_OK;
}

void gen_free(GenPath& g) {
  if (g.d_base) cudaFree(g.d_base);
  g.d_base = nullptr;
  g.bytes = 0;
  g.d_pairs = nullptr;
  g.d_prims = nullptr;
  g.d_coef = nullptr;
  g.d_desc = nullptr;
  g.d_gen_idx = nullptr;
  g.d_boys = nullptr;
  g.d_counters = nullptr;
}

}  // namespace sqb
