// Host runtime of the B200 J/K engine and its C ABI (include/sqb200.h).
//
// Set-up per basis (sqb200_jk_create):
//   * shells exactly as the reference partitions and orders them: consecutive functions with
//     the same centre and exponent list form a shell (genGTOShell, reference
//     src/matrix.c:2457-2541), stably sorted by type S < L < P < D (sortGTOShell, :2415);
//   * every shell pair P >= Q, grouped into 10 pair classes (SS LS LL PS PL PP DS DL DP DD),
//     each pair with its primitive-pair records [p, Px, Py, Pz, exp(-mu R^2)/p, E-table]
//     where the E-table holds the McMurchie-Davidson Hermite coefficients times the
//     contraction weights (norm*coef, as the reference's shell coef[][]);
//   * within a class, pairs sorted by decreasing Schwarz bound, so for a bra pair the ket
//     pairs that survive the Schwarz screen form one prefix (plus, inside one class, the
//     suffix starting at the bra itself: each unordered pair of pairs is visited once).
// Per build: PT = PA + PB and the shell-block density maxima PM on the device, one
// generated kernel launch per quartet class, and a finalize kernel that forms
// JT = J + J^T, KA = -(K + K^T) (KB likewise, or KB = KA when restricted).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "jk_common.cuh"
#include "jk_registry.h"
#include "../../include/sqb200.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CUDA_OK(call)                                                              \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return fail(SQB200_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// ---------------------------------------------------------------- Boys table (host)

// F_m(T0) for the grid T0 = g*BOYS_H, m = 0..BOYS_NCOL-1, in long double:
// the top order by its convergent series e^-T sum_i (2T)^i / ((2m+1)(2m+3)...(2m+2i+1)),
// the rest by downward recursion F_m = (2T F_{m+1} + e^-T)/(2m+1).
std::vector<double> make_boys_table() {
  std::vector<double> tab(BOYS_NGRID * BOYS_NCOL);
  const int top = BOYS_NCOL - 1;
  for (int g = 0; g < BOYS_NGRID; ++g) {
    const long double T = (long double)g * (long double)BOYS_H;
    long double term = 1.0L / (2 * top + 1), sum = 0.0L;
    for (int i = 1; i < 2000; ++i) {
      sum += term;
      term *= (2.0L * T) / (2 * top + 2 * i + 1);
      if (term < sum * 1e-22L) break;
    }
    const long double e = expl(-T);
    long double F = e * sum;
    std::vector<long double> col(BOYS_NCOL);
    col[top] = F;
    for (int m = top - 1; m >= 0; --m) col[m] = (2.0L * T * col[m + 1] + e) / (2 * m + 1);
    for (int m = 0; m < BOYS_NCOL; ++m) tab[g * BOYS_NCOL + m] = (double)col[m];
  }
  return tab;
}

// ---------------------------------------------------------------- shells

struct Shell {
  int first, nfunc, type, nprim;
  double x, y, z;
  double exps[32];
  double coef[32][16];
  int lmn[16][3];
};

const int kComp[4][6][3] = {
    {{0, 0, 0}},
    {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}},
    {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}},
    {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}}};
const int kNComp[4] = {1, 4, 3, 6};

int build_shells(int nbf, const int* nprim, const int* lmn, const double* xyz,
                 const double* exps, const double* ncoefs, std::vector<Shell>& sh) {
  std::vector<long> off(nbf + 1, 0);
  for (int i = 0; i < nbf; ++i) {
    if (nprim[i] < 1 || nprim[i] > 32) return fail(SQB200_EUNSUPPORTED, "contraction length outside 1..32");
    off[i + 1] = off[i] + nprim[i];
  }
  auto same = [&](int i, int j) {
    if (xyz[3 * i] != xyz[3 * j] || xyz[3 * i + 1] != xyz[3 * j + 1] || xyz[3 * i + 2] != xyz[3 * j + 2]) return false;
    if (nprim[i] != nprim[j]) return false;
    for (int k = 0; k < nprim[i]; ++k)
      if (exps[off[i] + k] != exps[off[j] + k]) return false;
    return true;
  };
  sh.clear();
  for (int p = 0; p < nbf;) {
    Shell s;
    memset(&s, 0, sizeof(s));
    s.first = p;
    s.x = xyz[3 * p]; s.y = xyz[3 * p + 1]; s.z = xyz[3 * p + 2];
    s.nprim = nprim[p];
    for (int k = 0; k < s.nprim; ++k) s.exps[k] = exps[off[p] + k];
    int q = p;
    while (q < nbf && same(p, q) && s.nfunc < 16) {
      for (int d = 0; d < 3; ++d) s.lmn[s.nfunc][d] = lmn[3 * q + d];
      for (int k = 0; k < s.nprim; ++k) s.coef[k][s.nfunc] = ncoefs[off[q] + k];
      ++s.nfunc;
      ++q;
    }
    switch (s.nfunc) {
      case 1: s.type = 0; break;
      case 4: s.type = 1; break;
      case 3: s.type = 2; break;
      case 6: s.type = 3; break;
      default: return fail(SQB200_EUNSUPPORTED, "shell with " + std::to_string(s.nfunc) + " functions (only s, sp, p, d supported)");
    }
    for (int f = 0; f < s.nfunc; ++f)
      for (int d = 0; d < 3; ++d)
        if (s.lmn[f][d] != kComp[s.type][f][d])
          return fail(SQB200_EUNSUPPORTED, "shell components not in the canonical Cartesian order");
    sh.push_back(s);
    p = q;
  }
  std::stable_sort(sh.begin(), sh.end(), [](const Shell& a, const Shell& b) { return a.type < b.type; });
  return SQB200_OK;
}

// 1-D Hermite expansion coefficients E^{ij}_t (i <= 2, j <= 2, t <= i+j) of a Gaussian pair
// product relative to the product centre: E^{00}_0 = 1,
// E^{i+1,j}_t = E^{ij}_{t-1}/(2p) + XPA E^{ij}_t + (t+1) E^{ij}_{t+1}, likewise for j.
void hermite_e(double p, double xpa, double xpb, double E[3][3][5]) {
  memset(E, 0, sizeof(double) * 45);
  const double h = 0.5 / p;
  E[0][0][0] = 1.0;
  for (int i = 0; i <= 2; ++i)
    for (int j = 0; j <= 2; ++j) {
      if (i == 0 && j == 0) continue;
      const bool up_i = i > 0;
      const int si = up_i ? i - 1 : i, sj = up_i ? j : j - 1;
      const double X = up_i ? xpa : xpb;
      for (int t = 0; t <= i + j; ++t) {
        double v = X * E[si][sj][t];
        if (t > 0) v += h * E[si][sj][t - 1];
        if (t + 1 <= si + sj) v += (t + 1) * E[si][sj][t + 1];
        E[i][j][t] = v;
      }
    }
}

int pair_class_of(int ta, int tb) {
  // generator order: SS LS LL PS PL PP DS DL DP DD  (ta >= tb)
  static const int idx[4][4] = {{0, -1, -1, -1}, {1, 2, -1, -1}, {3, 4, 5, -1}, {6, 7, 8, 9}};
  return idx[ta][tb];
}

int etable_size(int ta, int tb) {
  int n = 0;
  for (int a = 0; a < kNComp[ta]; ++a)
    for (int b = 0; b < kNComp[tb]; ++b)
      n += (kComp[ta][a][0] + kComp[tb][b][0] + 1) * (kComp[ta][a][1] + kComp[tb][b][1] + 1) *
           (kComp[ta][a][2] + kComp[tb][b][2] + 1);
  return n;
}

struct PairClass {
  int ta = -1, tb = -1, ne = 0, stride = 0, max_nprim = 0;
  // sorted by primitive-pair count, then by decreasing Schwarz bound; sub[] holds the start
  // of every run of equal primitive count (plus the end)
  std::vector<sqb::PairRec> pairs;
  std::vector<int> sub;
  std::vector<double> prims;
  sqb::PairRec* d_pairs = nullptr;
  double* d_prims = nullptr;
  float* d_primsf = nullptr;     // FP32 copy for the mixed-precision kernels
};

}  // namespace

struct sqb200_jk {
  int device = 0;
  int nbf = 0, ns = 0;
  std::vector<Shell> shells;
  std::vector<double> schwarz;   // basis level, nbf*nbf
  PairClass cls[sqb::kNumPairClasses];
  cudaStream_t stream = nullptr;
  double* d_boys = nullptr;
  int* d_shfirst = nullptr;   // per shell first function
  int* d_shn = nullptr;       // per shell function count
  double *d_PA = nullptr, *d_PB = nullptr, *d_PT = nullptr, *d_PM = nullptr;
  double *d_J = nullptr, *d_KA = nullptr, *d_KB = nullptr;
  double *d_JT = nullptr, *d_KAo = nullptr, *d_KBo = nullptr;   // outputs for host builds
  unsigned long long* d_counters = nullptr;  // 3 per class kernel
  // work lists cached per (outer, fixed) cutoff
  // a segment's kernel index v < K is the FP64 form of class v, v >= K the FP32 form of
  // class v - K (K = kNumClassKernels); counters and timings use the same index
  struct Work {
    std::vector<int> kernel;      // kernel index per segment
    std::vector<int> first, count;
    sqb::WorkItem* d_items = nullptr;
    int total = 0;
  };
  std::map<std::tuple<double, double, double>, Work> work;
  double fp32_below = 0.0;      // quartets with Schwarz product below this use the FP32 form
  bool use_ws = true;           // warp-specialised form where a class has one (SQB200_WS=0 disables)
  std::vector<char> ran_ws;     // per class kernel: which form the last build launched
  std::vector<long long> last_counts;
  long long last_flops = 0;
  int last_launches = 0;        // kernels enqueued by the last build
  // per-class event timing (sqb200_jk_profile)
  bool profile = false;
  struct Ev { int kernel; cudaEvent_t a, b; };
  std::vector<Ev> events;
  std::vector<double> prof_ms;
  std::vector<long long> prof_launches;
};

namespace {

// ---------------------------------------------------------------- device helpers

__global__ void k_prep(const double* __restrict__ PA, const double* __restrict__ PB, double* __restrict__ PT,
                       double* __restrict__ J, double* __restrict__ KA, double* __restrict__ KB, int nn, int uhf) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    PT[i] = PA[i] + PB[i];
    J[i] = 0.0;
    KA[i] = 0.0;
    if (uhf) KB[i] = 0.0;
  }
}

// PM[P][Q] = max over the block of |PT|, |PA|, |PB| (reference src/matrix.c:3894-3904)
__global__ void k_pmax(const double* __restrict__ PA, const double* __restrict__ PB, const double* __restrict__ PT,
                       const int* __restrict__ first, const int* __restrict__ nf, int ns, int nbf,
                       double* __restrict__ PM) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ns * ns) return;
  const int P = idx / ns, Q = idx % ns;
  double r = 0.0;
  for (int p = 0; p < nf[P]; ++p)
    for (int q = 0; q < nf[Q]; ++q) {
      const int o = (first[P] + p) * nbf + first[Q] + q;
      r = fmax(r, fabs(PT[o]));
      r = fmax(r, fabs(PA[o]));
      r = fmax(r, fabs(PB[o]));
    }
  PM[idx] = r;
}

// JT = J + J^T, KA = -(K + K^T), KB likewise or = KA
__global__ void k_finalize(const double* __restrict__ J, const double* __restrict__ KA, const double* __restrict__ KB,
                           double* __restrict__ JT, double* __restrict__ KAo, double* __restrict__ KBo, int n, int uhf) {
  const int nn = n * n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    const int r = i / n, c = i % n, t = c * n + r;
    JT[i] = J[i] + J[t];
    const double ka = -(KA[i] + KA[t]);
    KAo[i] = ka;
    if (KBo) KBo[i] = uhf ? -(KB[i] + KB[t]) : ka;
  }
}

// ---------------------------------------------------------------- Schwarz on the device
//
// sqrt|(ab|ab)| for every function pair of every shell pair (create_Schwarz, reference
// src/matrix.c:389-440; contracted with no primitive cut, as its contr_eri), by the same
// McMurchie-Davidson expansion: (ab|ab) = sum_{i,j} sum_{tuv,tau nu phi} E_i[tuv] E_j[tau nu phi]
// (-1)^(tau+nu+phi) R_ij[t+tau, u+nu, v+phi].  One thread per (pair, a, b); runtime loops,
// Hermite integrals in a per-thread tetrahedral table.

struct SchwarzFn {
  int nfn;
  int sx[36], sy[36], sz[36], eoff[36];
};

__device__ __forceinline__ int tetra(int t, int u, int v) {
  const int n = t + u + v, m = u + v;
  return n * (n + 1) * (n + 2) / 6 + m * (m + 1) / 2 + v;
}

__global__ void k_schwarz(const sqb::PairRec* __restrict__ pairs, const double* __restrict__ prims, int npairs,
                          int stride, int nfb, SchwarzFn fd, const double* __restrict__ tab, int nbf,
                          double* __restrict__ S) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= npairs * fd.nfn) return;
  const int pr = idx / fd.nfn, f = idx % fd.nfn;
  const sqb::PairRec rec = pairs[pr];
  const int sx = fd.sx[f], sy = fd.sy[f], sz = fd.sz[f], eo = fd.eoff[f];
  const int L = 2 * (sx + sy + sz);
  double acc = 0.0;
  double Ra[165], Rb[165], F[9];
  for (int i = 0; i < rec.nprim; ++i) {
    const double* pi = prims + rec.poff + i * stride;
    for (int j = 0; j < rec.nprim; ++j) {
      const double* pj = prims + rec.poff + j * stride;
      const double p = pi[0], q = pj[0], pq = p + q, rs = rsqrt(pq), alpha = p * q * (rs * rs);
      const double X = pi[1] - pj[1], Y = pi[2] - pj[2], Z = pi[3] - pj[3];
      const double T = alpha * (X * X + Y * Y + Z * Z);
      sqb::boys<8>(T, tab, F);
      // R^{(n)} from n = L down to 0
      double* cur = Ra;
      double* nxt = Rb;
      const double s0 = TWO_PI_2_5 * rs;
      double w = s0;
      double base[9];
      for (int n = 0; n <= L; ++n) { base[n] = w * F[n]; w *= -2.0 * alpha; }
      cur[0] = base[L];
      for (int n = L - 1; n >= 0; --n) {
        const int top = L - n;
        for (int N = 0; N <= top; ++N)
          for (int t = N; t >= 0; --t)
            for (int u = N - t; u >= 0; --u) {
              const int v = N - t - u;
              double r;
              if (N == 0) r = base[n];
              else if (t > 0) r = X * cur[tetra(t - 1, u, v)] + (t > 1 ? (t - 1) * cur[tetra(t - 2, u, v)] : 0.0);
              else if (u > 0) r = Y * cur[tetra(t, u - 1, v)] + (u > 1 ? (u - 1) * cur[tetra(t, u - 2, v)] : 0.0);
              else r = Z * cur[tetra(t, u, v - 1)] + (v > 1 ? (v - 1) * cur[tetra(t, u, v - 2)] : 0.0);
              nxt[tetra(t, u, v)] = r;
            }
        double* tmp = cur; cur = nxt; nxt = tmp;
      }
      // contract with both E tables (same function pair)
      int ka = 0;
      for (int t = 0; t <= sx; ++t)
        for (int u = 0; u <= sy; ++u)
          for (int v = 0; v <= sz; ++v, ++ka) {
            const double ea = pi[5 + eo + ka];
            int kb = 0;
            double s = 0.0;
            for (int tt = 0; tt <= sx; ++tt)
              for (int uu = 0; uu <= sy; ++uu)
                for (int vv = 0; vv <= sz; ++vv, ++kb) {
                  const double e = pj[5 + eo + kb];
                  s += (((tt + uu + vv) & 1) ? -e : e) * cur[tetra(t + tt, u + uu, v + vv)];
                }
            acc += ea * s;
          }
    }
  }
  const int a = f / nfb, b = f % nfb;
  const double v = sqrt(fabs(acc));
  S[(size_t)(rec.fP + a) * nbf + rec.fQ + b] = v;
  S[(size_t)(rec.fQ + b) * nbf + rec.fP + a] = v;
}


// ---------------------------------------------------------------- one-electron integrals
//
// Overlap S, kinetic T and nuclear attraction V over contracted Cartesian functions (the
// reference builds them with overlap/kinetic/nai, src/int.c, for uhf(), src/uhf.c:1307-1334).
// One thread per function pair (p, q), McMurchie-Davidson per primitive pair:
//   S = c K (pi/p)^{3/2} Ex0 Ey0 Ez0,  with E^{ij}_0 the 1-D Hermite coefficients
//   T = -1/2 sum_axes [ j(j-1) S(i,j-2) - 2b(2j+1) S(i,j) + 4b^2 S(i,j+2) ] x (other axes' S)
//   V = -sum_C Z_C 2pi/p c K sum_tuv E_t E_u E_v R_tuv(p, P - C)

__device__ void oe_hermite(double p, double xpa, double xpb, int la, int lb, double E[3][5][7]) {
  const double h = 0.5 / p;
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j)
      for (int t = 0; t <= i + j; ++t) {
        double v;
        if (i == 0 && j == 0) v = (t == 0) ? 1.0 : 0.0;
        else if (i > 0) {
          v = xpa * E[i - 1][j][t];
          if (t > 0) v += h * E[i - 1][j][t - 1];
          if (t + 1 <= i - 1 + j) v += (t + 1) * E[i - 1][j][t + 1];
        } else {
          v = xpb * E[i][j - 1][t];
          if (t > 0) v += h * E[i][j - 1][t - 1];
          if (t + 1 <= i + j - 1) v += (t + 1) * E[i][j - 1][t + 1];
        }
        E[i][j][t] = v;
      }
}

__global__ void k_oneint(int nbf, const int* __restrict__ nprim, const int* __restrict__ off,
                         const int* __restrict__ lmn, const double* __restrict__ xyz,
                         const double* __restrict__ exps, const double* __restrict__ nc, int natom,
                         const double* __restrict__ Z, const double* __restrict__ axyz,
                         const double* __restrict__ tab, double* __restrict__ S, double* __restrict__ T,
                         double* __restrict__ V) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nbf * nbf) return;
  const int pa = idx / nbf, pb = idx % nbf;
  const int* la = lmn + 3 * pa;
  const int* lb = lmn + 3 * pb;
  const double* A = xyz + 3 * pa;
  const double* B = xyz + 3 * pb;
  double s = 0.0, t = 0.0, v = 0.0;
  double Ex[3][5][7], Ey[3][5][7], Ez[3][5][7];
  double Rc[165], Rn[165], F[9];
  const double ab2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]);
  for (int i = 0; i < nprim[pa]; ++i)
    for (int j = 0; j < nprim[pb]; ++j) {
      const double a = exps[off[pa] + i], b = exps[off[pb] + j], p = a + b;
      const double c = nc[off[pa] + i] * nc[off[pb] + j] * exp(-a * b * ab2 / p);
      const double P[3] = {(a * A[0] + b * B[0]) / p, (a * A[1] + b * B[1]) / p, (a * A[2] + b * B[2]) / p};
      oe_hermite(p, P[0] - A[0], P[0] - B[0], la[0], lb[0] + 2, Ex);
      oe_hermite(p, P[1] - A[1], P[1] - B[1], la[1], lb[1] + 2, Ey);
      oe_hermite(p, P[2] - A[2], P[2] - B[2], la[2], lb[2] + 2, Ez);
      const double sq = sqrt(M_PI / p);
      // 1-D overlaps S_d(i, j) = E^{ij}_0 sqrt(pi/p)
      double sd[3], td[3];
      double (*E[3])[5][7] = {Ex, Ey, Ez};
      for (int d = 0; d < 3; ++d) {
        const int ii = la[d], jj = lb[d];
        sd[d] = E[d][ii][jj][0] * sq;
        double k = -2.0 * b * (2 * jj + 1) * E[d][ii][jj][0] + 4.0 * b * b * E[d][ii][jj + 2][0];
        if (jj >= 2) k += jj * (jj - 1) * E[d][ii][jj - 2][0];
        td[d] = -0.5 * k * sq;
      }
      s += c * sd[0] * sd[1] * sd[2];
      t += c * (td[0] * sd[1] * sd[2] + sd[0] * td[1] * sd[2] + sd[0] * sd[1] * td[2]);
      // nuclear attraction
      const int L = la[0] + lb[0] + la[1] + lb[1] + la[2] + lb[2];
      for (int at = 0; at < natom; ++at) {
        const double X = P[0] - axyz[3 * at], Y = P[1] - axyz[3 * at + 1], Zc = P[2] - axyz[3 * at + 2];
        sqb::boys<8>(p * (X * X + Y * Y + Zc * Zc), tab, F);
        double base[9], w = 1.0;
        for (int n = 0; n <= L; ++n) { base[n] = w * F[n]; w *= -2.0 * p; }
        double* cur = Rc;
        double* nxt = Rn;
        cur[0] = base[L];
        for (int n = L - 1; n >= 0; --n) {
          for (int N = 0; N <= L - n; ++N)
            for (int tt = N; tt >= 0; --tt)
              for (int uu = N - tt; uu >= 0; --uu) {
                const int vv = N - tt - uu;
                double r;
                if (N == 0) r = base[n];
                else if (tt > 0) r = X * cur[tetra(tt - 1, uu, vv)] + (tt > 1 ? (tt - 1) * cur[tetra(tt - 2, uu, vv)] : 0.0);
                else if (uu > 0) r = Y * cur[tetra(tt, uu - 1, vv)] + (uu > 1 ? (uu - 1) * cur[tetra(tt, uu - 2, vv)] : 0.0);
                else r = Zc * cur[tetra(tt, uu, vv - 1)] + (vv > 1 ? (vv - 1) * cur[tetra(tt, uu, vv - 2)] : 0.0);
                nxt[tetra(tt, uu, vv)] = r;
              }
          double* tmp = cur; cur = nxt; nxt = tmp;
        }
        double sum = 0.0;
        for (int tt = 0; tt <= la[0] + lb[0]; ++tt)
          for (int uu = 0; uu <= la[1] + lb[1]; ++uu)
            for (int vv = 0; vv <= la[2] + lb[2]; ++vv)
              sum += Ex[la[0]][lb[0]][tt] * Ey[la[1]][lb[1]][uu] * Ez[la[2]][lb[2]][vv] * cur[tetra(tt, uu, vv)];
        v -= Z[at] * (2.0 * M_PI / p) * c * sum;
      }
    }
  S[idx] = s;
  T[idx] = t;
  V[idx] = v;
}

int grid_for(long n, int block) {
  long g = (n + block - 1) / block;
  return (int)std::min<long>(std::max<long>(g, 1), 148L * 16);
}

// ---------------------------------------------------------------- pair data

void build_pairs(sqb200_jk* c) {
  const std::vector<Shell>& sh = c->shells;
  const int ns = (int)sh.size();
  for (int k = 0; k < sqb::kNumPairClasses; ++k) {
    c->cls[k] = PairClass();
  }
  // Schwarz block max in the reference orientation (first shell index >= second)
  auto sch = [&](int P, int Q) {
    double r = 0.0;
    for (int p = 0; p < sh[P].nfunc; ++p)
      for (int q = 0; q < sh[Q].nfunc; ++q) r = std::max(r, c->schwarz[(size_t)(sh[P].first + p) * c->nbf + sh[Q].first + q]);
    return r;
  };
  struct Tmp { double s; int P, Q, np; };
  std::vector<Tmp> lists[sqb::kNumPairClasses];
  for (int P = 0; P < ns; ++P)
    for (int Q = 0; Q <= P; ++Q) {
      const int k = pair_class_of(sh[P].type, sh[Q].type);
      lists[k].push_back({sch(P, Q), P, Q, sh[P].nprim * sh[Q].nprim});
    }
  for (int k = 0; k < sqb::kNumPairClasses; ++k) {
    PairClass& pc = c->cls[k];
    std::stable_sort(lists[k].begin(), lists[k].end(),
                     [](const Tmp& a, const Tmp& b) { return a.np != b.np ? a.np < b.np : a.s > b.s; });
    if (lists[k].empty()) continue;
    for (size_t i = 0; i < lists[k].size(); ++i)
      if (i == 0 || lists[k][i].np != lists[k][i - 1].np) pc.sub.push_back((int)i);
    pc.sub.push_back((int)lists[k].size());
    const Shell& s0 = sh[lists[k][0].P];
    const Shell& s1 = sh[lists[k][0].Q];
    pc.ta = s0.type;
    pc.tb = s1.type;
    pc.ne = etable_size(pc.ta, pc.tb);
    pc.stride = 5 + pc.ne;
    for (const Tmp& t : lists[k]) {
      const Shell& A = sh[t.P];
      const Shell& B = sh[t.Q];
      sqb::PairRec rec;
      rec.P = t.P; rec.Q = t.Q; rec.fP = A.first; rec.fQ = B.first;
      rec.nprim = A.nprim * B.nprim;
      rec.poff = (int)pc.prims.size();
      rec.schwarz = t.s;
      pc.max_nprim = std::max(pc.max_nprim, rec.nprim);
      const double ab2 = (A.x - B.x) * (A.x - B.x) + (A.y - B.y) * (A.y - B.y) + (A.z - B.z) * (A.z - B.z);
      for (int i = 0; i < A.nprim; ++i)
        for (int j = 0; j < B.nprim; ++j) {
          const double a = A.exps[i], b = B.exps[j], p = a + b;
          const double Px = (a * A.x + b * B.x) / p, Py = (a * A.y + b * B.y) / p, Pz = (a * A.z + b * B.z) / p;
          const double kp = std::exp(-a * b * ab2 / p) / p;
          double Ex[3][3][5], Ey[3][3][5], Ez[3][3][5];
          hermite_e(p, Px - A.x, Px - B.x, Ex);
          hermite_e(p, Py - A.y, Py - B.y, Ey);
          hermite_e(p, Pz - A.z, Pz - B.z, Ez);
          pc.prims.push_back(p);
          pc.prims.push_back(Px);
          pc.prims.push_back(Py);
          pc.prims.push_back(Pz);
          pc.prims.push_back(kp);
          for (int fa = 0; fa < A.nfunc; ++fa)
            for (int fb = 0; fb < B.nfunc; ++fb) {
              const int* la = kComp[A.type][fa];
              const int* lb = kComp[B.type][fb];
              const double w = A.coef[i][fa] * B.coef[j][fb] * kp;
              for (int tt = 0; tt <= la[0] + lb[0]; ++tt)
                for (int uu = 0; uu <= la[1] + lb[1]; ++uu)
                  for (int vv = 0; vv <= la[2] + lb[2]; ++vv)
                    pc.prims.push_back(w * Ex[la[0]][lb[0]][tt] * Ey[la[1]][lb[1]][uu] * Ez[la[2]][lb[2]][vv]);
            }
        }
      pc.pairs.push_back(rec);
    }
  }
}

int compute_schwarz_device(sqb200_jk* c, double* S_host) {
  const size_t nn = (size_t)c->nbf * c->nbf;
  double* dS = nullptr;
  CUDA_OK(cudaMalloc(&dS, nn * sizeof(double)));
  CUDA_OK(cudaMemset(dS, 0, nn * sizeof(double)));
  for (int k = 0; k < sqb::kNumPairClasses; ++k) {
    const PairClass& pc = c->cls[k];
    if (pc.pairs.empty()) continue;
    SchwarzFn fd;
    memset(&fd, 0, sizeof(fd));
    int off = 0;
    for (int a = 0; a < kNComp[pc.ta]; ++a)
      for (int b = 0; b < kNComp[pc.tb]; ++b) {
        const int f = fd.nfn++;
        fd.sx[f] = kComp[pc.ta][a][0] + kComp[pc.tb][b][0];
        fd.sy[f] = kComp[pc.ta][a][1] + kComp[pc.tb][b][1];
        fd.sz[f] = kComp[pc.ta][a][2] + kComp[pc.tb][b][2];
        fd.eoff[f] = off;
        off += (fd.sx[f] + 1) * (fd.sy[f] + 1) * (fd.sz[f] + 1);
      }
    const long nthr = (long)pc.pairs.size() * fd.nfn;
    k_schwarz<<<(int)((nthr + 127) / 128), 128, 0, c->stream>>>(pc.d_pairs, pc.d_prims, (int)pc.pairs.size(), pc.stride,
                                                               kNComp[pc.tb], fd, c->d_boys, c->nbf, dS);
    CUDA_OK(cudaGetLastError());
  }
  CUDA_OK(cudaMemcpyAsync(S_host, dS, nn * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_OK(cudaStreamSynchronize(c->stream));
  CUDA_OK(cudaFree(dS));
  return SQB200_OK;
}

void free_pairs(sqb200_jk* c) {
  for (int k = 0; k < sqb::kNumPairClasses; ++k) {
    cudaFree(c->cls[k].d_primsf);
    c->cls[k].d_primsf = nullptr;
  }
  for (int k = 0; k < sqb::kNumPairClasses; ++k) {
    cudaFree(c->cls[k].d_pairs);
    cudaFree(c->cls[k].d_prims);
    c->cls[k].d_pairs = nullptr;
    c->cls[k].d_prims = nullptr;
  }
}

int upload_pairs(sqb200_jk* c) {
  for (int k = 0; k < sqb::kNumPairClasses; ++k) {
    PairClass& pc = c->cls[k];
    if (pc.pairs.empty()) continue;
    CUDA_OK(cudaMalloc(&pc.d_pairs, pc.pairs.size() * sizeof(sqb::PairRec)));
    CUDA_OK(cudaMalloc(&pc.d_prims, pc.prims.size() * sizeof(double)));
    CUDA_OK(cudaMemcpy(pc.d_pairs, pc.pairs.data(), pc.pairs.size() * sizeof(sqb::PairRec), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(pc.d_prims, pc.prims.data(), pc.prims.size() * sizeof(double), cudaMemcpyHostToDevice));
    std::vector<float> pf(pc.prims.begin(), pc.prims.end());
    CUDA_OK(cudaMalloc(&pc.d_primsf, pf.size() * sizeof(float)));
    CUDA_OK(cudaMemcpy(pc.d_primsf, pf.data(), pf.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  return SQB200_OK;
}

// Work list: per class kernel, one item per (bra pair, <=128 ket pairs).
int build_work(sqb200_jk* c, double outer, double fixed, sqb200_jk::Work** out) {
  auto key = std::make_tuple(outer, fixed, c->fp32_below);
  auto it = c->work.find(key);
  if (it != c->work.end()) {
    *out = &it->second;
    return SQB200_OK;
  }
  sqb200_jk::Work w;
  std::vector<sqb::WorkItem> items, items32;
  const double cut = std::max(outer, fixed);
  for (int ki = 0; ki < sqb::kNumClassKernels; ++ki) {
    const sqb::ClassKernel& K = sqb::kClassKernels[ki];
    const PairClass& B = c->cls[K.bra_cls];
    const PairClass& T = c->cls[K.ket_cls];
    if (B.pairs.empty() || T.pairs.empty()) continue;
    const int first = (int)items.size();
    const bool same = K.bra_cls == K.ket_cls;
    const bool mixed = c->fp32_below > 0.0 && K.fn_r32 != nullptr;
    items32.clear();
    // every (bra sub-list, ket sub-list) combination; inside one class each unordered pair of
    // sub-lists once, and inside one sub-list each unordered pair of pairs once (k >= b)
    for (size_t sx = 0; sx + 1 < B.sub.size(); ++sx)
      for (size_t sy = 0; sy + 1 < T.sub.size(); ++sy) {
        if (same && sx > sy) continue;
        const int b0 = B.sub[sx], b1 = B.sub[sx + 1], k0s = T.sub[sy], k1s = T.sub[sy + 1];
        const int nbp = B.pairs[b0].nprim, nkp = T.pairs[k0s].nprim;
        // split the bra primitives over up to 32 threads when a quartet has many primitives
        // (the warp-specialised form takes 32 kets per CTA, one lane each)
        const bool ws = c->use_ws && K.ws_r != nullptr;
        int isplit = 1;
        while (!ws && isplit * 2 <= nbp && isplit * 2 <= 32 && (long)nbp * nkp / (isplit * 2) >= 32) isplit *= 2;
        const int kper = ws ? 32 : 128 / isplit;
        for (int b = b0; b < b1; ++b) {
          const double sb = B.pairs[b].schwarz;
          if (!(sb > 0.0)) break;   // sorted: the rest are zero
          const double thr = cut / sb * (1.0 - 1e-12);
          // ket pairs of the sub-list with schwarz >= thr form a prefix of it
          int lo = k0s, hi = k1s;
          while (lo < hi) {
            const int mid = (lo + hi) / 2;
            if (T.pairs[mid].schwarz >= thr) lo = mid + 1; else hi = mid;
          }
          const int end = lo;
          const int start = (same && sx == sy) ? b : k0s;
          // kets with Sch(bra)*Sch(ket) >= fp32_below (a prefix) stay FP64, the rest go FP32
          int mid = end;
          if (mixed) {
            const double t32 = c->fp32_below / sb;
            int l2 = start, h2 = end;
            while (l2 < h2) {
              const int m2 = (l2 + h2) / 2;
              if (T.pairs[m2].schwarz >= t32) l2 = m2 + 1; else h2 = m2;
            }
            mid = l2;
          }
          for (int k0 = start; k0 < mid; k0 += kper) items.push_back({b, k0, std::min(kper, mid - k0), isplit});
          for (int k0 = std::max(start, mid); k0 < end; k0 += kper)
            items32.push_back({b, k0, std::min(kper, end - k0), isplit});
        }
      }
    const int cnt = (int)items.size() - first;
    if (cnt > 0) {
      w.kernel.push_back(ki);
      w.first.push_back(first);
      w.count.push_back(cnt);
    }
    if (!items32.empty()) {
      w.kernel.push_back(ki + sqb::kNumClassKernels);
      w.first.push_back((int)items.size());
      w.count.push_back((int)items32.size());
      items.insert(items.end(), items32.begin(), items32.end());
    }
  }
  w.total = (int)items.size();
  if (w.total > 0) {
    CUDA_OK(cudaMalloc(&w.d_items, items.size() * sizeof(sqb::WorkItem)));
    CUDA_OK(cudaMemcpy(w.d_items, items.data(), items.size() * sizeof(sqb::WorkItem), cudaMemcpyHostToDevice));
  }
  auto ins = c->work.emplace(key, w);
  *out = &ins.first->second;
  return SQB200_OK;
}

int launch_build(sqb200_jk* c, const double* dPA, const double* dPB, int restricted, double outer,
                 double fixed, double dscreen, double* dJT, double* dKA, double* dKB, cudaStream_t st) {
  const int n = c->nbf, nn = n * n;
  const int uhf = restricted ? 0 : 1;
  if (!restricted && dPB == nullptr) return fail(SQB200_EINVAL, "unrestricted build needs PB");
  if (dPB == nullptr) dPB = dPA;
  sqb200_jk::Work* w = nullptr;
  int rc = build_work(c, outer, fixed, &w);
  if (rc) return rc;
  k_prep<<<grid_for(nn, 256), 256, 0, st>>>(dPA, dPB, c->d_PT, c->d_J, c->d_KA, c->d_KB, nn, uhf);
  k_pmax<<<(c->ns * c->ns + 127) / 128, 128, 0, st>>>(dPA, dPB, c->d_PT, c->d_shfirst, c->d_shn, c->ns, n, c->d_PM);
  CUDA_OK(cudaMemsetAsync(c->d_counters, 0, sizeof(unsigned long long) * 8 * sqb::kNumClassKernels, st));
  c->last_launches = 3 + (int)w->kernel.size();
  for (size_t s = 0; s < w->kernel.size(); ++s) {
    const int v = w->kernel[s];
    const bool f32 = v >= sqb::kNumClassKernels;
    const int kidx = f32 ? v - sqb::kNumClassKernels : v;
    const sqb::ClassKernel& K = sqb::kClassKernels[kidx];
    const PairClass& B = c->cls[K.bra_cls];
    const PairClass& T = c->cls[K.ket_cls];
    sqb::JKArgs a;
    memset(&a, 0, sizeof(a));
    a.bra_pairs = B.d_pairs; a.bra_prims = B.d_prims;
    a.ket_pairs = T.d_pairs; a.ket_prims = T.d_prims;
    a.PA = dPA; a.PB = dPB; a.PT = c->d_PT; a.PM = c->d_PM;
    a.Jacc = c->d_J; a.KAacc = c->d_KA; a.KBacc = c->d_KB;
    a.boys_tab = c->d_boys;
    a.counters = c->d_counters + 4 * v;
    a.bra_prims_f = B.d_primsf; a.ket_prims_f = T.d_primsf;
    a.nbf = n; a.ns = c->ns;
    a.same_class = K.bra_cls == K.ket_cls;
    a.cut_outer = outer; a.cut_fixed = fixed; a.dscreen_rmax = dscreen;
    const sqb::WorkItem* items = w->d_items + w->first[s];
    void* args[] = {&a, &items};
    const bool ws = !f32 && c->use_ws && K.ws_r != nullptr;
    if (!f32) c->ran_ws[kidx] = ws;
    const size_t smem = (size_t)B.max_nprim * B.stride * (f32 ? sizeof(float) : sizeof(double)) +
                        (ws ? (size_t)K.ws_warps * K.ws_nr * 32 * sizeof(double) : 0);
    const void* fn = f32 ? (uhf ? K.fn_u32 : K.fn_r32) : ws ? (uhf ? K.ws_u : K.ws_r) : (uhf ? K.fn_u : K.fn_r);
    const dim3 grid(w->count[s], ws ? 1 : (f32 ? K.passes32 : K.passes)), block(ws ? 32 * K.ws_warps : 128);
    if (smem > 48 * 1024) CUDA_OK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    sqb200_jk::Ev ev{v, nullptr, nullptr};
    if (c->profile) {
      CUDA_OK(cudaEventCreate(&ev.a));
      CUDA_OK(cudaEventCreate(&ev.b));
      CUDA_OK(cudaEventRecord(ev.a, st));
    }
    CUDA_OK(cudaLaunchKernel(fn, grid, block, args, smem, st));
    if (c->profile) {
      CUDA_OK(cudaEventRecord(ev.b, st));
      c->events.push_back(ev);
    }
  }
  k_finalize<<<grid_for(nn, 256), 256, 0, st>>>(c->d_J, c->d_KA, c->d_KB, dJT, dKA, dKB, n, uhf);
  CUDA_OK(cudaGetLastError());
  return SQB200_OK;
}

// Algorithmic FP64/FP32 operations of kernel index v (FP64 form v < K, FP32 form v - K)
// from its four counters [quartets, primitive quartets, bra flushes, digestions].
double kernel_flops(const sqb200_jk* c, int v, const unsigned long long* h) {
  const int K_ = sqb::kNumClassKernels;
  const bool f32 = v >= K_;
  const sqb::ClassKernel& K = sqb::kClassKernels[f32 ? v - K_ : v];
  const bool ws = !f32 && v < (int)c->ran_ws.size() && c->ran_ws[v];
  const double fp = f32 ? K.f32_flops_prim : ws ? K.ws_flops_prim : K.flops_prim;
  const double ff = f32 ? K.f32_flops_flush : ws ? K.ws_flops_flush : K.flops_flush;
  const double fq = f32 ? K.f32_flops_quartet : ws ? K.ws_flops_quartet : K.flops_quartet;
  return (double)h[1] * fp + (double)h[2] * ff + (double)h[3] * fq;
}

}  // namespace

// ---------------------------------------------------------------- C ABI

extern "C" {

const char* sqb200_last_error(void) { return g_err.c_str(); }

int sqb200_jk_create(sqb200_jk** out, int nbf, const int* nprim, const int* lmn, const double* xyz,
                     const double* exps, const double* ncoefs, const double* schwarz, int device) {
  if (!out || nbf <= 0 || !nprim || !lmn || !xyz || !exps || !ncoefs) return fail(SQB200_EINVAL, "null argument or nbf <= 0");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SQB200_ENODEV, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(SQB200_EINVAL, "bad device index");
  CUDA_OK(cudaSetDevice(device));
  sqb200_jk* c = new sqb200_jk();
  c->device = device;
  const char* ws_env = getenv("SQB200_WS");
  c->use_ws = !(ws_env && ws_env[0] == '0');
  c->ran_ws.assign(sqb::kNumClassKernels, 0);
  c->nbf = nbf;
  int rc = build_shells(nbf, nprim, lmn, xyz, exps, ncoefs, c->shells);
  if (rc) { delete c; return rc; }
  c->ns = (int)c->shells.size();
  if (schwarz) c->schwarz.assign(schwarz, schwarz + (size_t)nbf * nbf);
  else c->schwarz.assign((size_t)nbf * nbf, 1.0);   // placeholder until the device pass below
  build_pairs(c);
  rc = upload_pairs(c);
  if (rc) { sqb200_jk_destroy(c); return rc; }
  const size_t nn = (size_t)nbf * nbf;
  std::vector<double> tab = make_boys_table();
  std::vector<int> fst(c->ns), nf(c->ns);
  for (int s = 0; s < c->ns; ++s) { fst[s] = c->shells[s].first; nf[s] = c->shells[s].nfunc; }
#define ALLOC(p, bytes) do { cudaError_t e_ = cudaMalloc(&(p), (bytes)); if (e_ != cudaSuccess) { sqb200_jk_destroy(c); return fail(SQB200_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e_)); } } while (0)
  ALLOC(c->d_boys, tab.size() * sizeof(double));
  ALLOC(c->d_shfirst, c->ns * sizeof(int));
  ALLOC(c->d_shn, c->ns * sizeof(int));
  ALLOC(c->d_PA, nn * sizeof(double));
  ALLOC(c->d_PB, nn * sizeof(double));
  ALLOC(c->d_PT, nn * sizeof(double));
  ALLOC(c->d_PM, (size_t)c->ns * c->ns * sizeof(double));
  ALLOC(c->d_J, nn * sizeof(double));
  ALLOC(c->d_KA, nn * sizeof(double));
  ALLOC(c->d_KB, nn * sizeof(double));
  ALLOC(c->d_JT, nn * sizeof(double));
  ALLOC(c->d_KAo, nn * sizeof(double));
  ALLOC(c->d_KBo, nn * sizeof(double));
  ALLOC(c->d_counters, 8 * sqb::kNumClassKernels * sizeof(unsigned long long));
#undef ALLOC
  cudaError_t e = cudaMemcpy(c->d_boys, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(c->d_shfirst, fst.data(), c->ns * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(c->d_shn, nf.data(), c->ns * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { sqb200_jk_destroy(c); return fail(SQB200_ECUDA, cudaGetErrorString(e)); }
  if (!schwarz) {
    // Schwarz bounds from the device, then the pair lists in their final (sorted) order
    rc = compute_schwarz_device(c, c->schwarz.data());
    if (rc) { sqb200_jk_destroy(c); return rc; }
    free_pairs(c);
    build_pairs(c);
    rc = upload_pairs(c);
    if (rc) { sqb200_jk_destroy(c); return rc; }
  }
  *out = c;
  return SQB200_OK;
}

int sqb200_jk_destroy(sqb200_jk* c) {
  if (!c) return SQB200_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& kv : c->work) cudaFree(kv.second.d_items);
  for (auto& e : c->events) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
  free_pairs(c);
  void* ptrs[] = {c->d_boys, c->d_shfirst, c->d_shn, c->d_PA, c->d_PB, c->d_PT, c->d_PM, c->d_J, c->d_KA,
                  c->d_KB, c->d_JT, c->d_KAo, c->d_KBo, c->d_counters};
  for (void* p : ptrs) cudaFree(p);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return SQB200_OK;
}

int sqb200_jk_build_device(sqb200_jk* c, const double* dPA, const double* dPB, int restricted, double outer,
                           double fixed, double dscreen, double* dJT, double* dKA, double* dKB, void* stream) {
  if (!c || !dPA || !dJT || !dKA) return fail(SQB200_EINVAL, "null argument");
  CUDA_OK(cudaSetDevice(c->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  return launch_build(c, dPA, dPB, restricted, outer, fixed, dscreen, dJT, dKA, dKB, st);
}

int sqb200_jk_build(sqb200_jk* c, const double* PA, const double* PB, int restricted, double outer, double fixed,
                    double dscreen, double* JT, double* KA, double* KB) {
  if (!c || !PA || !JT || !KA || !KB) return fail(SQB200_EINVAL, "null argument");
  CUDA_OK(cudaSetDevice(c->device));
  const size_t bytes = (size_t)c->nbf * c->nbf * sizeof(double);
  CUDA_OK(cudaMemcpyAsync(c->d_PA, PA, bytes, cudaMemcpyHostToDevice, c->stream));
  const double* dPB = c->d_PA;
  if (PB && PB != PA) {
    CUDA_OK(cudaMemcpyAsync(c->d_PB, PB, bytes, cudaMemcpyHostToDevice, c->stream));
    dPB = c->d_PB;
  }
  int rc = launch_build(c, c->d_PA, dPB, restricted, outer, fixed, dscreen, c->d_JT, c->d_KAo, c->d_KBo, c->stream);
  if (rc) return rc;
  CUDA_OK(cudaMemcpyAsync(JT, c->d_JT, bytes, cudaMemcpyDeviceToHost, c->stream));
  CUDA_OK(cudaMemcpyAsync(KA, c->d_KAo, bytes, cudaMemcpyDeviceToHost, c->stream));
  CUDA_OK(cudaMemcpyAsync(KB, c->d_KBo, bytes, cudaMemcpyDeviceToHost, c->stream));
  CUDA_OK(cudaStreamSynchronize(c->stream));
  return SQB200_OK;
}

int sqb200_jk_stats(sqb200_jk* c, long long* out, int n) {
  if (!c || !out) return fail(SQB200_EINVAL, "null argument");
  CUDA_OK(cudaSetDevice(c->device));
  CUDA_OK(cudaStreamSynchronize(c->stream));
  std::vector<unsigned long long> h(8 * sqb::kNumClassKernels);
  CUDA_OK(cudaMemcpy(h.data(), c->d_counters, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  long long q = 0, pq = 0, fl = 0;
  for (int v = 0; v < 2 * sqb::kNumClassKernels; ++v) {
    q += (long long)h[4 * v];
    pq += (long long)h[4 * v + 1];
    fl += (long long)kernel_flops(c, v, &h[4 * v]);
  }
  long long v[6] = {q, pq, fl, (long long)c->ns, 0, (long long)c->last_launches};
  for (int k = 0; k < sqb::kNumPairClasses; ++k) v[4] += (long long)c->cls[k].pairs.size();
  for (int i = 0; i < n && i < 6; ++i) out[i] = v[i];
  return SQB200_OK;
}

int sqb200_jk_schwarz(sqb200_jk* c, double* S) {
  if (!c || !S) return fail(SQB200_EINVAL, "null argument");
  CUDA_OK(cudaSetDevice(c->device));
  return compute_schwarz_device(c, S);
}

int sqb200_jk_profile(sqb200_jk* c, int enable) {
  if (!c) return fail(SQB200_EINVAL, "null argument");
  CUDA_OK(cudaSetDevice(c->device));
  CUDA_OK(cudaStreamSynchronize(c->stream));
  for (auto& e : c->events) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
  c->events.clear();
  c->prof_ms.assign(2 * sqb::kNumClassKernels, 0.0);
  c->prof_launches.assign(2 * sqb::kNumClassKernels, 0);
  c->profile = enable != 0;
  return SQB200_OK;
}

int sqb200_jk_profile_read(sqb200_jk* c, double* rows, int max_rows, int* nrows) {
  if (!c || !rows || !nrows) return fail(SQB200_EINVAL, "null argument");
  CUDA_OK(cudaSetDevice(c->device));
  for (auto& e : c->events) {
    CUDA_OK(cudaEventSynchronize(e.b));
    float ms = 0.f;
    CUDA_OK(cudaEventElapsedTime(&ms, e.a, e.b));
    if (c->prof_ms.size() != (size_t)(2 * sqb::kNumClassKernels)) {
      c->prof_ms.assign(2 * sqb::kNumClassKernels, 0.0);
      c->prof_launches.assign(2 * sqb::kNumClassKernels, 0);
    }
    c->prof_ms[e.kernel] += ms;
    c->prof_launches[e.kernel] += 1;
    cudaEventDestroy(e.a);
    cudaEventDestroy(e.b);
  }
  c->events.clear();
  std::vector<unsigned long long> h(8 * sqb::kNumClassKernels);
  CUDA_OK(cudaMemcpy(h.data(), c->d_counters, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  int r = 0;
  for (int v = 0; v < 2 * sqb::kNumClassKernels && r < max_rows; ++v) {
    if (c->prof_launches.empty() || c->prof_launches[v] == 0) continue;
    double* row = rows + 6 * r;
    row[0] = v;
    row[1] = (double)c->prof_launches[v];
    row[2] = c->prof_ms[v];
    row[3] = kernel_flops(c, v, &h[4 * v]);
    row[4] = (double)h[4 * v + 1];
    row[5] = (double)h[4 * v];
    ++r;
  }
  *nrows = r;
  return SQB200_OK;
}

const char* sqb200_jk_class_name(int k) {
  if (k < 0 || k >= 2 * sqb::kNumClassKernels) return "";
  static std::vector<std::string> names;
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  if (names.empty())
    for (int i = 0; i < 2 * sqb::kNumClassKernels; ++i) {
      const sqb::ClassKernel& K = sqb::kClassKernels[i % sqb::kNumClassKernels];
      names.push_back(std::string(sqb::kPairClassNames[K.bra_cls]) + "|" + sqb::kPairClassNames[K.ket_cls] +
                      (i >= sqb::kNumClassKernels ? " f32" : ""));
    }
  return names[k].c_str();
}

int sqb200_jk_set_precision(sqb200_jk* c, double fp32_below) {
  if (!c || !(fp32_below >= 0.0)) return fail(SQB200_EINVAL, "null context or negative threshold");
  c->fp32_below = fp32_below;
  return SQB200_OK;
}

int sqb200_jk_mem_cutoff(sqb200_jk* c, double fixed, int max_mem_mb, double* out) {
  // getMemCutoff_Parallel (reference src/matrix.c:3703-3760), nCPU = 1
  if (!c || !out) return fail(SQB200_EINVAL, "null argument");
  const std::vector<Shell>& sh = c->shells;
  const int ns = c->ns;
  std::vector<double> S((size_t)ns * ns);
  for (int P = 0; P < ns; ++P)
    for (int Q = 0; Q < ns; ++Q) {
      double r = 0.0;
      for (int p = 0; p < sh[P].nfunc; ++p)
        for (int q = 0; q < sh[Q].nfunc; ++q) r = std::max(r, c->schwarz[(size_t)(sh[P].first + p) * c->nbf + sh[Q].first + q]);
      S[(size_t)P * ns + Q] = r;
    }
  const unsigned long long maxEE = (unsigned long long)max_mem_mb * 1000000ULL / sizeof(double);
  double cut = fixed;
  bool coarse = true;
  for (;;) {
    unsigned long long cnt = 0;
    bool over = false;
    for (int P = 0; P < ns && !over; ++P)
      for (int Q = 0; Q <= P && !over; ++Q)
        for (int I = 0; I <= P && !over; ++I) {
          const int N = (I == P) ? Q : I;
          for (int J = 0; J <= N; ++J) {
            if (S[(size_t)P * ns + Q] * S[(size_t)I * ns + J] < cut) continue;
            cnt += (unsigned long long)sh[P].nfunc * sh[Q].nfunc * sh[I].nfunc * sh[J].nfunc;
            if (cnt > maxEE) { over = true; break; }
          }
        }
    if (over) { cut *= coarse ? 2.00 : 1.05; continue; }
    if (coarse && cnt < maxEE) { coarse = false; cut /= 2.0; continue; }
    break;
  }
  *out = std::max(cut, fixed);
  return SQB200_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- build without allocation
//
// sqb200_jk_build_noalloc: the J/K build of sqb200_jk_build_device with every piece of scratch
// (PT, PM, the J/K accumulators, the class counters and the work list) placed in one
// file-scope device array instead of buffers the library allocates.  The array is sized for
// at most kNoAllocMaxNbf basis functions and kNoAllocMaxItems work items; every device that
// loads the library holds it until the process exits.

namespace {

constexpr int kNoAllocMaxNbf = 256;
constexpr int kNoAllocMaxItems = 65536;
constexpr int kNoAllocMaxKernels = 64;
constexpr size_t kNoAllocMat = (size_t)kNoAllocMaxNbf * kNoAllocMaxNbf;          // doubles per matrix
constexpr size_t kNoAllocCountersOff = 5 * kNoAllocMat * sizeof(double);            // PT PM J KA KB
constexpr size_t kNoAllocItemsOff = kNoAllocCountersOff + 4 * kNoAllocMaxKernels * sizeof(unsigned long long);
constexpr size_t kNoAllocBytes = kNoAllocItemsOff + (size_t)kNoAllocMaxItems * sizeof(sqb::WorkItem);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {nullptr};

// Device address of the scratch array on the current device (looked up once per device; the
// host-side symbol itself is not a device address).
int noalloc_scratch(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (device < 0 || device >= 64) return fail(SQB200_EINVAL, "device index beyond 63");
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return fail(SQB200_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_noalloc_addr[device] = p;
  }
  *out = (unsigned char*)g_noalloc_addr[device];
  return SQB200_OK;
}

// The work list of the standard kernel form on the host (no device copy kept).
void noalloc_items(const sqb200_jk* c, double outer, double fixed, std::vector<sqb::WorkItem>& items,
                   std::vector<int>& kernel, std::vector<int>& first, std::vector<int>& count) {
  items.clear(); kernel.clear(); first.clear(); count.clear();
  const double cut = std::max(outer, fixed);
  for (int ki = 0; ki < sqb::kNumClassKernels; ++ki) {
    const sqb::ClassKernel& K = sqb::kClassKernels[ki];
    const PairClass& B = c->cls[K.bra_cls];
    const PairClass& T = c->cls[K.ket_cls];
    if (B.pairs.empty() || T.pairs.empty()) continue;
    const int f0 = (int)items.size();
    const bool same = K.bra_cls == K.ket_cls;
    for (size_t sx = 0; sx + 1 < B.sub.size(); ++sx)
      for (size_t sy = 0; sy + 1 < T.sub.size(); ++sy) {
        if (same && sx > sy) continue;
        const int b0 = B.sub[sx], b1 = B.sub[sx + 1], k0s = T.sub[sy], k1s = T.sub[sy + 1];
        const int nbp = B.pairs[b0].nprim, nkp = T.pairs[k0s].nprim;
        int isplit = 1;
        while (isplit * 2 <= nbp && isplit * 2 <= 32 && (long)nbp * nkp / (isplit * 2) >= 32) isplit *= 2;
        const int kper = 128 / isplit;
        for (int b = b0; b < b1; ++b) {
          const double sb = B.pairs[b].schwarz;
          if (!(sb > 0.0)) break;
          const double thr = cut / sb * (1.0 - 1e-12);
          int lo = k0s, hi = k1s;
          while (lo < hi) {
            const int mid = (lo + hi) / 2;
            if (T.pairs[mid].schwarz >= thr) lo = mid + 1; else hi = mid;
          }
          const int start = (same && sx == sy) ? b : k0s;
          for (int k0 = start; k0 < lo; k0 += kper) items.push_back({b, k0, std::min(kper, lo - k0), isplit});
        }
      }
    if ((int)items.size() > f0) {
      kernel.push_back(ki);
      first.push_back(f0);
      count.push_back((int)items.size() - f0);
    }
  }
}

}  // namespace

extern "C" int sqb200_jk_build_noalloc(sqb200_jk* c, const double* dPA, const double* dPB, int restricted,
                                       double outer, double fixed, double dscreen, double* dJT, double* dKA,
                                       double* dKB, void* stream) {
  if (!c || !dPA || !dJT || !dKA) return fail(SQB200_EINVAL, "null argument");
  if (!restricted && (dPB == nullptr || dKB == nullptr)) return fail(SQB200_EINVAL, "unrestricted build needs PB and KB");
  if (c->nbf > kNoAllocMaxNbf)
    return fail(SQB200_EINVAL, "sqb200_jk_build_noalloc: " + std::to_string(c->nbf) + " basis functions exceed its limit of " +
                                   std::to_string(kNoAllocMaxNbf));
  if (sqb::kNumClassKernels > kNoAllocMaxKernels) return fail(SQB200_EINVAL, "class table larger than the scratch counters");
  CUDA_OK(cudaSetDevice(c->device));
  unsigned char* base = nullptr;
  int rc = noalloc_scratch(c->device, &base);
  if (rc) return rc;
  thread_local std::vector<sqb::WorkItem> items;
  thread_local std::vector<int> kernel, first, count;
  noalloc_items(c, outer, fixed, items, kernel, first, count);
  if ((int)items.size() > kNoAllocMaxItems)
    return fail(SQB200_EINVAL, "sqb200_jk_build_noalloc: " + std::to_string(items.size()) +
                                   " work items exceed its limit of " + std::to_string(kNoAllocMaxItems));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  const int n = c->nbf, nn = n * n, uhf = restricted ? 0 : 1;
  if (dPB == nullptr) dPB = dPA;
  double* PT = (double*)base;
  double* PM = PT + kNoAllocMat;
  double* J = PM + kNoAllocMat;
  double* KA = J + kNoAllocMat;
  double* KB = KA + kNoAllocMat;
  unsigned long long* counters = (unsigned long long*)(base + kNoAllocCountersOff);
  sqb::WorkItem* d_items = (sqb::WorkItem*)(base + kNoAllocItemsOff);
  if (!items.empty())
    CUDA_OK(cudaMemcpyAsync(d_items, items.data(), items.size() * sizeof(sqb::WorkItem), cudaMemcpyHostToDevice, st));
  // k_prep zeroes J, KA (and KB when unrestricted); the counters are cleared here
  k_prep<<<grid_for(nn, 256), 256, 0, st>>>(dPA, dPB, PT, J, KA, KB, nn, uhf);
  k_pmax<<<(c->ns * c->ns + 127) / 128, 128, 0, st>>>(dPA, dPB, PT, c->d_shfirst, c->d_shn, c->ns, n, PM);
  CUDA_OK(cudaMemsetAsync(counters, 0, sizeof(unsigned long long) * 4 * sqb::kNumClassKernels, st));
  for (size_t s = 0; s < kernel.size(); ++s) {
    const sqb::ClassKernel& K = sqb::kClassKernels[kernel[s]];
    const PairClass& B = c->cls[K.bra_cls];
    const PairClass& T = c->cls[K.ket_cls];
    sqb::JKArgs a;
    memset(&a, 0, sizeof(a));
    a.bra_pairs = B.d_pairs; a.bra_prims = B.d_prims;
    a.ket_pairs = T.d_pairs; a.ket_prims = T.d_prims;
    a.PA = dPA; a.PB = dPB; a.PT = PT; a.PM = PM;
    a.Jacc = J; a.KAacc = KA; a.KBacc = KB;
    a.boys_tab = c->d_boys;
    a.counters = counters + 4 * kernel[s];
    a.nbf = n; a.ns = c->ns;
    a.same_class = K.bra_cls == K.ket_cls;
    a.cut_outer = outer; a.cut_fixed = fixed; a.dscreen_rmax = dscreen;
    const sqb::WorkItem* it = d_items + first[s];
    void* args[] = {&a, &it};
    const size_t smem = (size_t)B.max_nprim * B.stride * sizeof(double);
    const void* fn = uhf ? K.fn_u : K.fn_r;
    if (smem > 48 * 1024) CUDA_OK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CUDA_OK(cudaLaunchKernel(fn, dim3(count[s], K.passes), dim3(128), args, smem, st));
  }
  k_finalize<<<grid_for(nn, 256), 256, 0, st>>>(J, KA, KB, dJT, dKA, dKB, n, uhf);
  CUDA_OK(cudaGetLastError());
  return SQB200_OK;
}


extern "C" int sqb200_oneint(sqb200_jk* c, int natom, const double* Z, const double* axyz, double* S, double* T,
                             double* V) {
  if (!c || natom < 0 || (natom > 0 && (!Z || !axyz)) || !S || !T || !V) return fail(SQB200_EINVAL, "null argument");
  CUDA_OK(cudaSetDevice(c->device));
  const int n = c->nbf;
  std::vector<int> np(n), off(n), lmn(3 * n);
  std::vector<double> xyz(3 * n), ex, nc;
  for (const Shell& sh : c->shells)
    for (int f = 0; f < sh.nfunc; ++f) {
      const int q = sh.first + f;
      np[q] = sh.nprim;
      for (int d = 0; d < 3; ++d) lmn[3 * q + d] = sh.lmn[f][d];
      xyz[3 * q] = sh.x; xyz[3 * q + 1] = sh.y; xyz[3 * q + 2] = sh.z;
    }
  for (int q = 0; q < n; ++q) off[q] = (int)ex.size(), ex.resize(ex.size() + np[q]), nc.resize(nc.size() + np[q]);
  for (const Shell& sh : c->shells)
    for (int f = 0; f < sh.nfunc; ++f)
      for (int k = 0; k < sh.nprim; ++k) {
        ex[off[sh.first + f] + k] = sh.exps[k];
        nc[off[sh.first + f] + k] = sh.coef[k][f];
      }
  const size_t nn = (size_t)n * n;
  int *d_np = nullptr, *d_off = nullptr, *d_lmn = nullptr;
  double *d_xyz = nullptr, *d_ex = nullptr, *d_nc = nullptr, *d_Z = nullptr, *d_A = nullptr, *d_out = nullptr;
  cudaError_t e = cudaMalloc(&d_np, n * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&d_off, n * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&d_lmn, 3 * n * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&d_xyz, 3 * n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_ex, ex.size() * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_nc, nc.size() * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_Z, (natom + 1) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_A, (3 * natom + 3) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_out, 3 * nn * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(d_np, np.data(), n * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_off, off.data(), n * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_lmn, lmn.data(), 3 * n * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_xyz, xyz.data(), 3 * n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_ex, ex.data(), ex.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_nc, nc.data(), nc.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && natom > 0) e = cudaMemcpy(d_Z, Z, natom * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && natom > 0) e = cudaMemcpy(d_A, axyz, 3 * natom * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_oneint<<<(int)((nn + 127) / 128), 128, 0, c->stream>>>(n, d_np, d_off, d_lmn, d_xyz, d_ex, d_nc, natom, d_Z, d_A,
                                                              c->d_boys, d_out, d_out + nn, d_out + 2 * nn);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) e = cudaMemcpy(S, d_out, nn * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(T, d_out + nn, nn * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(V, d_out + 2 * nn, nn * sizeof(double), cudaMemcpyDeviceToHost);
  void* ptrs[] = {d_np, d_off, d_lmn, d_xyz, d_ex, d_nc, d_Z, d_A, d_out};
  for (void* q : ptrs) cudaFree(q);
  if (e != cudaSuccess) return fail(SQB200_ECUDA, std::string("sqb200_oneint: ") + cudaGetErrorString(e));
  return SQB200_OK;
}
