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
#include <cusolverDn.h>

#include <algorithm>
#include <climits>
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
#include "jk_generic.cuh"
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

// Host-to-device copy that has landed when it returns.  A plain cudaMemcpy from pageable host
// memory may return once the data are staged, before the last DMA has reached the device, and
// the non-blocking streams the kernels run on are not ordered after the legacy stream that
// copy uses; so every upload goes through the stream it is named for and waits for it.
inline cudaError_t h2d(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e;
}

// Device buffers laid out in one allocation, each start 256-byte aligned.  One cudaMalloc and
// one cudaFree instead of one per buffer: each call changes the GPU's mappings (hundreds of
// microseconds on a large GPU), and cudaFree synchronises the whole device, stalling every
// other job that runs on it.
struct Carve {
  std::vector<std::pair<void**, size_t>> slots;
  template <class T>
  void add(T** dst, size_t bytes) { slots.push_back({(void**)dst, bytes}); }
  static size_t round(size_t b) { return (std::max<size_t>(b, 1) + 255) / 256 * 256; }
  size_t bytes() const {
    size_t tot = 0;
    for (auto& sl : slots) tot += round(sl.second);
    return tot;
  }
  void place(void* base) {
    size_t o = 0;
    for (auto& sl : slots) { *sl.first = (char*)base + o; o += round(sl.second); }
  }
  cudaError_t alloc(void** base) {
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, std::max<size_t>(bytes(), 256));
    *base = e == cudaSuccess ? p : nullptr;
    if (e == cudaSuccess) place(p);
    return e;
  }
};

// A Carve whose buffers are (partly) filled from host arrays: one allocation and one staged
// host-to-device copy for all of them.
struct Staged : Carve {
  std::vector<const void*> src;   // per buffer: its host data, or nullptr (left unset)
  template <class T>
  void put(T** dst, size_t bytes, const void* host) { add(dst, bytes); src.push_back(host); }
  cudaError_t upload(void** base, cudaStream_t st) {
    src.resize(slots.size(), nullptr);
    cudaError_t e = alloc(base);
    if (e != cudaSuccess) return e;
    size_t o = 0, end = 0;
    std::vector<size_t> at;
    for (size_t i = 0; i < slots.size(); ++i) {
      at.push_back(o);
      if (src[i] && slots[i].second) end = o + slots[i].second;
      o += round(slots[i].second);
    }
    if (end == 0) return cudaSuccess;
    std::vector<char> img(end, 0);
    for (size_t i = 0; i < slots.size(); ++i)
      if (src[i] && slots[i].second) memcpy(img.data() + at[i], src[i], slots[i].second);
    return h2d(*base, img.data(), end, st);
  }
};

// ---------------------------------------------------------------- Boys table (host)

}  // namespace

namespace sqb {
// F_m(T0) for the grid T0 = g*BOYS_H, m = 0..ncol-1, in long double:
// the top order by its convergent series e^-T sum_i (2T)^i / ((2m+1)(2m+3)...(2m+2i+1)),
// the rest by downward recursion F_m = (2T F_{m+1} + e^-T)/(2m+1).
std::vector<double> boys_table(int ncol) {
  std::vector<double> tab(BOYS_NGRID * ncol);
  const int top = ncol - 1;
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
    std::vector<long double> col(ncol);
    col[top] = F;
    for (int m = top - 1; m >= 0; --m) col[m] = (2.0L * T * col[m + 1] + e) / (2 * m + 1);
    for (int m = 0; m < ncol; ++m) tab[g * ncol + m] = (double)col[m];
  }
  return tab;
}
}  // namespace sqb

namespace {

// the class kernels' table: BOYS_NGRID rows of BOYS_NCOL orders, then e^-T0 per grid point
std::vector<double> make_boys_table() {
  std::vector<double> t = sqb::boys_table(BOYS_NCOL);
  for (int g = 0; g < BOYS_NGRID; ++g) t.push_back((double)expl(-(long double)g * (long double)BOYS_H));
  return t;
}

// ---------------------------------------------------------------- shells

struct Shell {
  int first, nfunc, type, nprim;
  int gen;                 // 1: its pairs take the generic path (jk_generic.cu)
  int lmax;                // highest l+m+n of its functions
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
    // the reference's type by function count (genGTOShell, src/matrix.c:2527-2535: S, P, L, D,
    // F = 4 for ten functions, X = 6 otherwise); it fixes the shell order (sortGTOShell)
    switch (s.nfunc) {
      case 1: s.type = 0; break;
      case 4: s.type = 1; break;
      case 3: s.type = 2; break;
      case 6: s.type = 3; break;
      case 10: s.type = 4; break;
      default: s.type = 6; break;
    }
    // s, sp, p and d shells in the canonical component order run in the generated class kernels;
    // every other shell (f, or another layout) on the generic path
    s.gen = s.type > 3 ? 1 : 0;
    for (int f = 0; f < s.nfunc; ++f) {
      int l = 0;
      for (int d = 0; d < 3; ++d) {
        if (s.lmn[f][d] < 0) return fail(SQB200_EINVAL, "negative angular index");
        l += s.lmn[f][d];
        if (!s.gen && s.lmn[f][d] != kComp[s.type][f][d]) s.gen = 1;
      }
      if (l > sqb::kGenLmax)
        return fail(SQB200_EUNSUPPORTED, "function with l+m+n = " + std::to_string(l) + " (f, 3, is the highest supported)");
      s.lmax = std::max(s.lmax, l);
    }
    sh.push_back(s);
    p = q;
  }
  std::stable_sort(sh.begin(), sh.end(), [](const Shell& a, const Shell& b) { return a.type < b.type; });
  return SQB200_OK;
}

// 1-D Hermite expansion coefficients E^{ij}_t (i <= 3, j <= 3, t <= i+j: up to f) of a
// Gaussian pair product relative to the product centre: E^{00}_0 = 1,
// E^{i+1,j}_t = E^{ij}_{t-1}/(2p) + XPA E^{ij}_t + (t+1) E^{ij}_{t+1}, likewise for j.
void hermite_e(double p, double xpa, double xpb, double E[4][4][7]) {
  memset(E, 0, sizeof(double) * 4 * 4 * 7);
  const double h = 0.5 / p;
  E[0][0][0] = 1.0;
  for (int i = 0; i <= 3; ++i)
    for (int j = 0; j <= 3; ++j) {
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

namespace sqb {
// The library's error text for the other translation units (sqb200_last_error).
int set_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace sqb

struct sqb200_jk {
  int device = 0;
  int nbf = 0, ns = 0;
  std::vector<Shell> shells;
  std::vector<double> schwarz;   // basis level, nbf*nbf
  PairClass cls[sqb::kNumPairClasses];
  cudaStream_t stream = nullptr;
  void* d_base = nullptr;       // one allocation holding every buffer below
  void* d_pairbase = nullptr;   // one allocation holding the pair classes' device arrays
  size_t pairbase_bytes = 0;
  double* d_boys = nullptr;
  float* d_boysf = nullptr;   // the Boys table in FP32 (mixed-precision forms)
  int* d_shfirst = nullptr;   // per shell first function
  int* d_shn = nullptr;       // per shell function count
  double *d_PA = nullptr, *d_PB = nullptr, *d_PT = nullptr, *d_PM = nullptr;
  double *d_J = nullptr, *d_KA = nullptr, *d_KB = nullptr;
  double *d_JT = nullptr, *d_KAo = nullptr, *d_KBo = nullptr;   // outputs for host builds
  unsigned long long* d_counters = nullptr;  // 4 per class kernel form
  unsigned long long* d_queue = nullptr;     // persistent launches: work-unit counter per kernel form
  bool persistent = false;                   // class kernels as persistent work-queue launches
  sqb::MolRec* d_mol = nullptr;              // the build's molecule record (written by k_prep)
  // work lists cached per (outer, fixed) cutoff
  // a segment's kernel index v < K is the FP64 form of class v, v >= K the FP32 form of
  // class v - K (K = kNumClassKernels); counters and timings use the same index
  struct Work {
    std::vector<int> kernel;      // kernel index per segment
    std::vector<int> first, count;
    std::vector<double> cost;     // estimated FP operations per segment (launch order, stream choice)
    sqb::WorkItem* d_items = nullptr;
    int* d_er = nullptr;          // multipole mode: per item, the error-bank slot of its first ket
    int total = 0;
    sqb::GenItem* d_gitems = nullptr;   // the generic path's items (shells outside the classes)
    int gtotal = 0;
  };
  // key: outer cutoff, fixed cutoff, FP32 threshold, multipole mode
  std::map<std::tuple<double, double, double, int>, Work> work;
  double fp32_below = 0.0;      // quartets with Schwarz product below this use the FP32 form
  bool use_ws = true;           // warp-specialised form where a class has one (SQB200_WS=0 disables)
  std::vector<char> ran_ws;     // per class kernel: which form the last build launched
  std::vector<char> form;       // per class kernel: FP64 form to run, 0 narrow / 1 wide / 2 swapped (autotuner)
  std::vector<char> ran_form;   // per class kernel: the FP64 form the last build launched
  std::vector<long long> last_counts;
  long long last_flops = 0;
  int last_launches = 0;        // kernels enqueued by the last build
  // side streams for concurrent class launches: the build forks them off its stream after the
  // prologue and joins them before k_finalize (SQB200_STREAMS, default 4; 0 = one stream)
  int nside = -1;
  std::vector<cudaStream_t> side;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
  // per-class event timing (sqb200_jk_profile)
  bool profile = false;
  struct Ev { int kernel; cudaEvent_t a, b; };
  std::vector<Ev> events;
  std::vector<double> prof_ms;
  std::vector<long long> prof_launches;
  // device address of the static scratch array of sqb200_jk_build_noalloc on this context's
  // device, looked up when the context is created (nullptr + the lookup's error otherwise)
  unsigned char* noalloc_base = nullptr;
  cudaError_t noalloc_err = cudaSuccess;
  // reference-parity multipole mode (sqb200_jk_set_multipole): monopole table, powers of 1.5,
  // and the error bank, one slot per quartet that survives the outer Schwarz cutoff, laid out
  // in work-list order for that cutoff (er_outer) and kept from build to build
  bool mp_on = false;
  double mp_rmax = 0.0;
  void* d_mpbase = nullptr;             // one allocation: d_mpole, d_pow15
  double* d_mpole = nullptr;
  double* d_pow15 = nullptr;
  void* d_erbase = nullptr;             // one allocation: d_erscr, d_erbank
  unsigned long long* d_erscr = nullptr;
  signed char* d_erbank = nullptr;
  long long er_total = -1;
  double er_outer = -1.0;
  // quartets with a shell outside the generated classes (f shells and other layouts)
  sqb::GenPath gen;
};

namespace {

// Device address of the static scratch array of sqb200_jk_build_noalloc (defined with it below)
// on the current device.
cudaError_t noalloc_lookup(unsigned char** out);

// ---------------------------------------------------------------- device helpers

// PT = PA + PB and zeroed accumulators; the first thread also writes the build's molecule
// record (offsets 0, sizes and this build's cutoffs), which the class kernels read
__global__ void k_prep(const double* __restrict__ PA, const double* __restrict__ PB, double* __restrict__ PT,
                       double* __restrict__ J, double* __restrict__ KA, double* __restrict__ KB, int nn, int uhf,
                       sqb::MolRec* __restrict__ mol, sqb::MolRec mv) {
  if (mol && blockIdx.x == 0 && threadIdx.x == 0) *mol = mv;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    PT[i] = PA[i] + PB[i];
    J[i] = 0.0;
    KA[i] = 0.0;
    if (uhf) KB[i] = 0.0;
  }
}

// PM[P][Q] = max over the block of |PT|, |PA|, |PB| (reference src/matrix.c:3894-3904).  One
// warp per shell pair: the lanes share the block's (at most 36) elements, then a warp max (the
// maximum does not depend on the order, so every launch shape gives the same PM).
constexpr int kPmaxWarps = 4;
__global__ void __launch_bounds__(32 * kPmaxWarps) k_pmax(const double* __restrict__ PA, const double* __restrict__ PB,
                                                         const double* __restrict__ PT, const int* __restrict__ first,
                                                         const int* __restrict__ nf, int ns, int nbf,
                                                         double* __restrict__ PM) {
  const int idx = blockIdx.x * kPmaxWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (idx >= ns * ns) return;                     // whole warps leave together
  const int P = idx / ns, Q = idx % ns;
  const int np = nf[P], nq = nf[Q], fp = first[P], fq = first[Q];
  double r = 0.0;
  for (int e = lane; e < np * nq; e += 32) {
    const int p = e / nq, q = e - p * nq;
    const int o = (fp + p) * nbf + fq + q;
    r = fmax(r, fmax(fabs(PT[o]), fmax(fabs(PA[o]), fabs(PB[o]))));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
  if (lane == 0) PM[idx] = r;
}

void launch_pmax(const double* PA, const double* PB, const double* PT, const int* first, const int* nf, int ns,
                 int nbf, double* PM, cudaStream_t st) {
  k_pmax<<<(ns * ns + kPmaxWarps - 1) / kPmaxWarps, 32 * kPmaxWarps, 0, st>>>(PA, PB, PT, first, nf, ns, nbf, PM);
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

// Multipole mode: every bank slot still unknown that this build measured (scratch bit 63) takes
// the reference's exponent of the largest error, (signed char) clamp(log(maxErr) * LNBASEI)
// with ERROR_MIN for an exact zero (getErrExpQuartetMPole, src/matrix.c:2594-2599); the
// scratch is cleared for the next build.
__global__ void k_erbank(signed char* __restrict__ bank, unsigned long long* __restrict__ scr, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long v = scr[i];
    if (!v) continue;
    scr[i] = 0ull;
    if (bank[i] != sqb::ERR_UNKNOWN) continue;
    const double e = __longlong_as_double((long long)(v & ~(1ull << 63)));
    double x = e == 0.0 ? (double)sqb::ERR_MIN : log(e) * 2.4663034624;   // LNBASEI, 1/ln(1.5)
    if (x < sqb::ERR_MIN) x = sqb::ERR_MIN;
    if (x > sqb::ERR_MAX) x = sqb::ERR_MAX;
    bank[i] = (signed char)x;
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
    const int ks = rec.kstride;
    const double* pi = prims + rec.poff + (long long)i * stride * ks;
    for (int j = 0; j < rec.nprim; ++j) {
      const double* pj = prims + rec.poff + (long long)j * stride * ks;
      const double p = pi[0], q = pj[0], pq = p + q, rs = rsqrt(pq), alpha = p * q * (rs * rs);
      const double X = pi[ks] - pj[ks], Y = pi[2 * ks] - pj[2 * ks], Z = pi[3 * ks] - pj[3 * ks];
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
            const double ea = pi[(5 + eo + ka) * ks];
            int kb = 0;
            double s = 0.0;
            for (int tt = 0; tt <= sx; ++tt)
              for (int uu = 0; uu <= sy; ++uu)
                for (int vv = 0; vv <= sz; ++vv, ++kb) {
                  const double e = pj[(5 + eo + kb) * ks];
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

// E[i][j][t] for i <= la <= 3, j <= lb <= 5 (f functions, plus 2 for the kinetic term), t <= i+j
__device__ void oe_hermite(double p, double xpa, double xpb, int la, int lb, double E[4][6][9]) {
  const double h = 0.5 / p;
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j)
      for (int t = 0; t <= i + j; ++t) {
        double v;
        if (i == 0 && j == 0) v = (t == 0) ? 1.0 : 0.0;
        else if (i > 0) {
          // E^{i-1,j}_t vanishes for t > i-1+j: that entry was never written, read it as 0
          v = (t <= i - 1 + j) ? xpa * E[i - 1][j][t] : 0.0;
          if (t > 0) v += h * E[i - 1][j][t - 1];
          if (t + 1 <= i - 1 + j) v += (t + 1) * E[i - 1][j][t + 1];
        } else {
          v = (t <= i + j - 1) ? xpb * E[i][j - 1][t] : 0.0;
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
  double Ex[4][6][9], Ey[4][6][9], Ez[4][6][9];
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
      double (*E[3])[6][9] = {Ex, Ey, Ez};
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
      if (sh[P].gen || sh[Q].gen) continue;   // the generic path's
      const int k = pair_class_of(sh[P].type, sh[Q].type);
      lists[k].push_back({sch(P, Q), P, Q, sh[P].nprim * sh[Q].nprim});
    }
  // Layout of a class's primitive records: inside each run of pairs with one primitive count
  // (a sub-list, S pairs), field f of record j of the run's pair l is element
  // run_base + (j * stride + f) * S + l -- consecutive pairs side by side, so the lanes of a
  // warp, which hold consecutive ket pairs of one sub-list, read one field of their records in
  // coalesced loads (PairRec::poff = run_base + l, kstride = S).  SQB200_AOS=1 keeps each
  // record's fields contiguous instead (kstride 1), for comparison.
  const char* aos_env = getenv("SQB200_AOS");
  const bool aos = aos_env && aos_env[0] == '1';
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
      rec.kstride = 1;
      rec.pad_ = 0;
      rec.schwarz = t.s;
      pc.max_nprim = std::max(pc.max_nprim, rec.nprim);
      const double ab2 = (A.x - B.x) * (A.x - B.x) + (A.y - B.y) * (A.y - B.y) + (A.z - B.z) * (A.z - B.z);
      for (int i = 0; i < A.nprim; ++i)
        for (int j = 0; j < B.nprim; ++j) {
          const double a = A.exps[i], b = B.exps[j], p = a + b;
          const double Px = (a * A.x + b * B.x) / p, Py = (a * A.y + b * B.y) / p, Pz = (a * A.z + b * B.z) / p;
          const double kp = std::exp(-a * b * ab2 / p) / p;
          double Ex[4][4][7], Ey[4][4][7], Ez[4][4][7];
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
    if (!aos) {
      // records were appended contiguously (pair-major); transpose every sub-list run
      std::vector<double> soa(pc.prims.size());
      for (size_t r = 0; r + 1 < pc.sub.size(); ++r) {
        const int l0 = pc.sub[r], l1 = pc.sub[r + 1], S = l1 - l0;
        const size_t base = (size_t)pc.pairs[l0].poff;
        const size_t per = (size_t)pc.pairs[l0].nprim * pc.stride;   // elements per pair
        for (int l = 0; l < S; ++l) {
          const double* src = pc.prims.data() + base + (size_t)l * per;
          for (size_t e = 0; e < per; ++e) soa[base + e * S + l] = src[e];
          pc.pairs[l0 + l].poff = (int)(base + l);
          pc.pairs[l0 + l].kstride = S;
        }
      }
      pc.prims.swap(soa);
    }
  }
}

// The generic path's pair data (every shell pair, sorted by the current Schwarz bounds) when
// the basis has a shell outside the generated classes.
int setup_generic(sqb200_jk* c) {
  bool any = false;
  for (const Shell& s : c->shells) any = any || s.gen;
  c->gen.on = any;
  if (!any) return SQB200_OK;
  std::vector<sqb::GenShell> gs;
  for (const Shell& s : c->shells)
    gs.push_back({s.first, s.nfunc, s.nprim, s.lmax, s.gen, s.x, s.y, s.z, s.exps, &s.coef[0][0], &s.lmn[0][0]});
  sqb::gen_build_pairs(c->gen, gs, c->schwarz.data(), c->nbf);
  return sqb::gen_upload(c->gen, c->stream);
}

int compute_schwarz_device(sqb200_jk* c, double* S_host) {
  const size_t nn = (size_t)c->nbf * c->nbf;
  double* dS = c->d_JT;         // scratch: the host-build output buffer, rewritten by every build
  CUDA_OK(cudaMemsetAsync(dS, 0, nn * sizeof(double), c->stream));
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
  if (c->gen.on) {
    const int rc = sqb::gen_schwarz(c->gen, c->nbf, dS, c->stream);
    if (rc) return rc;
  }
  CUDA_OK(cudaMemcpyAsync(S_host, dS, nn * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_OK(cudaStreamSynchronize(c->stream));
  return SQB200_OK;
}

void free_pairs(sqb200_jk* c) {
  cudaFree(c->d_pairbase);
  c->d_pairbase = nullptr;
  c->pairbase_bytes = 0;
  for (int k = 0; k < sqb::kNumPairClasses; ++k) {
    c->cls[k].d_pairs = nullptr;
    c->cls[k].d_prims = nullptr;
    c->cls[k].d_primsf = nullptr;
  }
}

int upload_pairs(sqb200_jk* c) {
  Carve cv;
  for (int k = 0; k < sqb::kNumPairClasses; ++k) {
    PairClass& pc = c->cls[k];
    if (pc.pairs.empty()) continue;
    cv.add(&pc.d_pairs, pc.pairs.size() * sizeof(sqb::PairRec));
    cv.add(&pc.d_prims, pc.prims.size() * sizeof(double));
    cv.add(&pc.d_primsf, pc.prims.size() * sizeof(float));
  }
  if (cv.slots.empty()) return SQB200_OK;
  // the same layout again (the pair lists re-sorted by new Schwarz bounds) reuses the allocation
  const size_t tot = cv.bytes();
  if (c->d_pairbase && c->pairbase_bytes != tot) free_pairs(c);
  if (c->d_pairbase) {
    cv.place(c->d_pairbase);
  } else {
    const cudaError_t e = cv.alloc(&c->d_pairbase);
    if (e != cudaSuccess) return fail(SQB200_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    c->pairbase_bytes = tot;
  }
  // one staged host image of every class's arrays, one copy
  std::vector<char> img(tot, 0);
  const char* base = (const char*)c->d_pairbase;
  for (int k = 0; k < sqb::kNumPairClasses; ++k) {
    const PairClass& pc = c->cls[k];
    if (pc.pairs.empty()) continue;
    memcpy(img.data() + ((const char*)pc.d_pairs - base), pc.pairs.data(), pc.pairs.size() * sizeof(sqb::PairRec));
    memcpy(img.data() + ((const char*)pc.d_prims - base), pc.prims.data(), pc.prims.size() * sizeof(double));
    float* pf = (float*)(img.data() + ((const char*)pc.d_primsf - base));
    for (size_t i = 0; i < pc.prims.size(); ++i) pf[i] = (float)pc.prims[i];
  }
  CUDA_OK(h2d(c->d_pairbase, img.data(), tot, c->stream));
  return SQB200_OK;
}

// Threads per CTA of the class kernels (SQB200_CTA: 32, 64 or 128; default 64).  A work item
// holds one bra pair and up to (threads / isplit) ket pairs, so narrower CTAs give a small
// molecule's short ket lists CTAs that are not mostly empty: the registers of a CTA are
// allocated for all its threads, and an idle warp holds them as long as its CTA lives.
// Measured on B200: benzene/6-31G* 1080 / 1368 / 1340 builds/s at 128 / 64 / 32 threads;
// C60/6-31G 73.7 / 73.5 / 74.7 ms per build.
int cta_threads() {
  static const int n = [] {
    int v = 64;
    if (const char* e = getenv("SQB200_CTA")) v = atoi(e);
    return (v == 32 || v == 128) ? v : 64;
  }();
  return n;
}

int ensure_side_streams(sqb200_jk* c) {
  if (c->nside >= 0) return SQB200_OK;
  int n = 4;
  if (const char* e = getenv("SQB200_STREAMS")) n = std::max(0, std::min(16, atoi(e)));
  CUDA_OK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
  for (int i = 0; i < n; ++i) {
    cudaStream_t s;
    cudaEvent_t e;
    CUDA_OK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    CUDA_OK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    c->side.push_back(s);
    c->ev_join.push_back(e);
  }
  c->nside = n;
  return SQB200_OK;
}

// Work items of class kernel ki for one molecule (context c): every surviving (bra pair, <=kper
// ket pairs) unit, with pair indices shifted by bra_base/ket_base (the molecule's first pair in
// a merged class array; 0 for a single-molecule build).  Kets whose Schwarz product is below the
// context's fp32_below go to items32 (the FP32 form).  cost64/cost32 accumulate the emitted
// operations, the launch-order and stream-balancing estimate.
void class_items(const sqb200_jk* c, int ki, double outer, double fixed, int bra_base, int ket_base, int mol,
                 std::vector<sqb::WorkItem>& items, std::vector<sqb::WorkItem>& items32, double& cost64,
                 double& cost32, std::vector<int>* ers = nullptr, long long* er_run = nullptr,
                 bool allow_f32 = true) {
  const sqb::ClassKernel& K = sqb::kClassKernels[ki];
  const PairClass& B = c->cls[K.bra_cls];
  const PairClass& T = c->cls[K.ket_cls];
  if (B.pairs.empty() || T.pairs.empty()) return;
  const double cut = std::max(outer, fixed);
  const bool same = K.bra_cls == K.ket_cls;
  // multipole mode (er_run != nullptr): FP64 narrow form with one thread per quartet, and every
  // item records the error-bank slot of its first ket; the slots of each (bra, ket sub-list)
  // run are the outer-cutoff survivors in order, so the layout does not depend on `fixed`
  const bool mpm = er_run != nullptr;
  const bool mixed = allow_f32 && !mpm && c->fp32_below > 0.0 && K.fn_r32 != nullptr;
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
      while (!ws && !mpm && isplit * 2 <= nbp && isplit * 2 <= 32 && (long)nbp * nkp / (isplit * 2) >= 32) isplit *= 2;
      const int kper = ws ? 32 : cta_threads() / isplit;
      const double pq = (double)nbp * nkp;
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
        long long er0 = 0;
        if (mpm) {
          // outer-cutoff survivors of this run: the bank slots er0 .. er0 + count - 1
          const double tho = outer / sb * (1.0 - 1e-12);
          int lo2 = k0s, hi2 = k1s;
          while (lo2 < hi2) {
            const int m2 = (lo2 + hi2) / 2;
            if (T.pairs[m2].schwarz >= tho) lo2 = m2 + 1; else hi2 = m2;
          }
          er0 = *er_run;
          *er_run += std::max(0, lo2 - start);
        }
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
        for (int k0 = start; k0 < mid; k0 += kper) {
          items.push_back({bra_base + b, ket_base + k0, std::min(kper, mid - k0), isplit, mol});
          if (mpm) ers->push_back((int)(er0 + (k0 - start)));
        }
        for (int k0 = std::max(start, mid); k0 < end; k0 += kper)
          items32.push_back({bra_base + b, ket_base + k0, std::min(kper, end - k0), isplit, mol});
        cost64 += std::max(0, mid - start) * (pq * K.flops_prim + K.flops_quartet);
        cost32 += std::max(0, end - std::max(start, mid)) * (pq * K.f32_flops_prim + K.f32_flops_quartet);
      }
    }
}

// Launch order inside one class kernel: the CTAs with the longest primitive loop first (a
// thread runs ceil(bra primitives / isplit) x ket primitives iterations; more kets per item next),
// so that a launch does not end on a few long CTAs while the rest of the GPU idles.
// nprims(item) gives the item's (bra, ket) primitive counts.
template <class F>
void sort_heavy_first(std::vector<sqb::WorkItem>& v, size_t first, F nprims) {
  const size_t n = v.size() - first;
  std::vector<std::pair<long long, size_t>> key(n);
  for (size_t i = 0; i < n; ++i) {
    const sqb::WorkItem& it = v[first + i];
    const std::pair<int, int> np = nprims(it);
    const long long loop = (long long)((np.first + it.isplit - 1) / it.isplit) * np.second;
    key[i] = {-(loop * 4096 + it.cnt), i};
  }
  std::stable_sort(key.begin(), key.end());
  std::vector<sqb::WorkItem> tmp(n);
  for (size_t i = 0; i < n; ++i) tmp[i] = v[first + key[i].second];
  std::copy(tmp.begin(), tmp.end(), v.begin() + first);
}

// A class whose FP32 work items would number fewer than this runs all its quartets in FP64: a
// second launch of a few hundred CTAs costs more than its FP32 arithmetic saves, and splitting
// the ket ranges at the FP32 threshold leaves the FP64 items shorter (SQB200_F32_MIN_ITEMS,
// default 2400, read whenever a work list is made; measured on B200: benzene/6-31G* at tau 1e-5
// 0.729 ms with 600, 0.725 with 1200, 0.716 with 2400, against 0.713-0.720 in FP64; C60/6-31G
// 50.5 ms with each, against 63.1 in FP64).
size_t f32_min_items() {
  const char* e = getenv("SQB200_F32_MIN_ITEMS");
  return e ? (size_t)std::max(0L, atol(e)) : (size_t)2400;
}

// True when a class's FP32 items are too few to launch: the class then runs all its quartets
// in FP64, with the work items of a build without the FP32 split.
bool too_few_f32(const std::vector<sqb::WorkItem>& items32) {
  return !items32.empty() && items32.size() < f32_min_items();
}

int build_work(sqb200_jk* c, double outer, double fixed, sqb200_jk::Work** out) {
  const int mpm = c->mp_on ? 1 : 0;
  auto key = std::make_tuple(outer, fixed, mpm ? 0.0 : c->fp32_below, mpm);
  auto it = c->work.find(key);
  if (it != c->work.end()) {
    *out = &it->second;
    return SQB200_OK;
  }
  sqb200_jk::Work w;
  std::vector<sqb::WorkItem> items, items32;
  std::vector<int> ers;
  long long er_run = 0;
  for (int ki = 0; ki < sqb::kNumClassKernels; ++ki) {
    const int first = (int)items.size();
    items32.clear();
    double cost64 = 0.0, cost32 = 0.0;
    class_items(c, ki, outer, fixed, 0, 0, 0, items, items32, cost64, cost32, mpm ? &ers : nullptr,
                mpm ? &er_run : nullptr);
    if (too_few_f32(items32)) {
      items.resize(first);
      items32.clear();
      cost64 = cost32 = 0.0;
      class_items(c, ki, outer, fixed, 0, 0, 0, items, items32, cost64, cost32, nullptr, nullptr, false);
    }
    if (!mpm) {   // (multipole mode keeps the items with their bank slots in generation order)
      const PairClass& B = c->cls[sqb::kClassKernels[ki].bra_cls];
      const PairClass& T = c->cls[sqb::kClassKernels[ki].ket_cls];
      auto np = [&](const sqb::WorkItem& it) { return std::make_pair(B.pairs[it.bra].nprim, T.pairs[it.k0].nprim); };
      sort_heavy_first(items, first, np);
      sort_heavy_first(items32, 0, np);
    }
    const int cnt = (int)items.size() - first;
    if (cnt > 0) {
      w.kernel.push_back(ki);
      w.first.push_back(first);
      w.count.push_back(cnt);
      w.cost.push_back(cost64);
    }
    if (!items32.empty()) {
      w.kernel.push_back(ki + sqb::kNumClassKernels);
      w.first.push_back((int)items.size());
      w.count.push_back((int)items32.size());
      w.cost.push_back(cost32);
      items.insert(items.end(), items32.begin(), items32.end());
    }
  }
  w.total = (int)items.size();
  if (w.total > 0) {
    CUDA_OK(cudaMalloc(&w.d_items, items.size() * sizeof(sqb::WorkItem)));
    CUDA_OK(h2d(w.d_items, items.data(), items.size() * sizeof(sqb::WorkItem), c->stream));
  }
  if (c->gen.on) {
    std::vector<sqb::GenItem> gi;
    double gcost = 0.0;
    sqb::gen_items(c->gen, outer, fixed, gi, gcost, mpm ? &er_run : nullptr);
    if (gi.size() > (size_t)INT_MAX) return fail(SQB200_EINVAL, "generic path: more than 2^31 work items");
    w.gtotal = (int)gi.size();
    if (!gi.empty()) {
      CUDA_OK(cudaMalloc(&w.d_gitems, gi.size() * sizeof(sqb::GenItem)));
      CUDA_OK(h2d(w.d_gitems, gi.data(), gi.size() * sizeof(sqb::GenItem), c->stream));
    }
  }
  if (mpm) {
    if (er_run > INT_MAX) return fail(SQB200_EINVAL, "multipole mode: more than 2^31 quartets survive the outer cutoff");
    if (!ers.empty()) {
      CUDA_OK(cudaMalloc(&w.d_er, ers.size() * sizeof(int)));
      CUDA_OK(h2d(w.d_er, ers.data(), ers.size() * sizeof(int), c->stream));
    }
    // the bank: laid out for this outer cutoff; a new outer cutoff starts a new bank
    if (c->er_outer != outer || c->er_total != er_run) {
      if (c->d_erbase) { cudaFree(c->d_erbase); c->d_erbase = nullptr; }
      const size_t ns = (size_t)std::max<long long>(1, er_run);
      Carve cv;
      cv.add(&c->d_erscr, ns * sizeof(unsigned long long));
      cv.add(&c->d_erbank, ns);
      cudaError_t e = cv.alloc(&c->d_erbase);
      if (e != cudaSuccess) return fail(SQB200_ENOMEM, std::string("cudaMalloc (error bank): ") + cudaGetErrorString(e));
      CUDA_OK(cudaMemsetAsync(c->d_erscr, 0, ns * sizeof(unsigned long long), c->stream));
      CUDA_OK(cudaMemsetAsync(c->d_erbank, sqb::ERR_UNKNOWN, ns, c->stream));
      CUDA_OK(cudaStreamSynchronize(c->stream));
      c->er_outer = outer;
      c->er_total = er_run;
    }
  }
  auto ins = c->work.emplace(key, w);
  *out = &ins.first->second;
  return SQB200_OK;
}

// Profile and class-name index of the generic path's kernel (after the FP64 and FP32 forms).
const int kGenericKernel = 2 * sqb::kNumClassKernels;

// One class-kernel launch of a work segment, ready to enqueue.
struct SegLaunch {
  const void* fn = nullptr;
  dim3 grid, block;
  size_t smem = 0;
  sqb::JKArgs a;
  const sqb::WorkItem* items = nullptr;
};

// FP64 forms of a class: 0 narrow tile, 1 wide tile, 2 swapped loop roles.
bool has_form(const sqb::ClassKernel& K, int form) {
  return form == 0 || (form == 1 && K.fn_rw) || (form == 2 && K.fn_rs);
}

// The kernel of class K (FP32 form when f32) for spin uhf in FP64 form `form` (falls back to the
// narrow tile where the class lacks it).  Returns the FP64 form picked (0 for the FP32 form).
int pick_form(const sqb::ClassKernel& K, bool f32, int uhf, int form, const void** fn, int* passes) {
  if (f32) { *fn = uhf ? K.fn_u32 : K.fn_r32; *passes = K.passes32; return 0; }
  if (form == 1 && K.fn_rw) { *fn = uhf ? K.fn_uw : K.fn_rw; *passes = K.passes_w; return 1; }
  if (form == 2 && K.fn_rs) { *fn = uhf ? K.fn_us : K.fn_rs; *passes = K.passes_s; return 2; }
  *fn = uhf ? K.fn_u : K.fn_r;
  *passes = K.passes;
  return 0;
}

// Shared-memory accumulators of the wide form: the region follows the staged bra primitives.
// The kernels index it thread-fastest with a stride of 128 threads, whatever the CTA width.
void add_acc_region(const sqb::ClassKernel& K, int form_used, SegLaunch& L) {
  const int dbl = form_used == 1 ? K.w_o_dbl : form_used == 2 ? K.s_o_dbl : 0;
  if (dbl <= 0) return;
  const size_t off = (L.smem + 15) / 16 * 16;
  L.a.so_off = (int)(off / sizeof(double));
  L.smem = off + (size_t)dbl * 128 * sizeof(double);
}

// Raise a kernel's dynamic shared-memory limit once per (device, kernel, size class), so that a
// build captured into a CUDA graph after a first uncaptured build issues only stream work.
int ensure_smem(const void* fn, size_t smem) {
  if (smem <= 48 * 1024) return SQB200_OK;
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> done;
  int dev = 0;
  CUDA_OK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  size_t& have = done[{dev, fn}];
  if (have >= smem) return SQB200_OK;
  CUDA_OK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  have = smem;
  return SQB200_OK;
}

int enqueue(const SegLaunch& L, cudaStream_t st) {
  sqb::JKArgs a = L.a;
  const sqb::WorkItem* items = L.items;
  void* args[] = {&a, &items};
  const int rc = ensure_smem(L.fn, L.smem);
  if (rc) return rc;
  CUDA_OK(cudaLaunchKernel(L.fn, L.grid, L.block, args, L.smem, st));
  return SQB200_OK;
}

// Resident CTAs of kernel fn per SM at this block size and dynamic shared memory (cached).
int resident_ctas(const void* fn, int block, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<int, const void*, int, size_t>, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  std::lock_guard<std::mutex> lock(mu);
  auto key = std::make_tuple(dev, fn, block, smem);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int n = 0, sms = 0;
  if (ensure_smem(fn, smem) != SQB200_OK ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, block, smem) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    (void)cudaGetLastError();
    n = 1; sms = 148;
  }
  const int r = std::max(1, n) * std::max(1, sms);
  cache[key] = r;
  return r;
}

// A persistent work-queue launch of segment launch L: a grid of at most one CTA per resident
// slot of the GPU takes L's (item, pass) units from the zeroed device counter q, in work-list
// order (heaviest first), instead of one CTA per unit.
void make_persistent(SegLaunch& L, unsigned long long* q) {
  const long long units = (long long)L.grid.x * L.grid.y;
  if (units <= 0 || units > INT_MAX) return;
  L.a.queue = q;
  L.a.nqueue = (int)units;
  L.a.npass = (int)L.grid.y;
  const int slots = resident_ctas(L.fn, (int)L.block.x, L.smem);
  L.grid = dim3((unsigned)std::min<long long>(units, slots), 1);
  static const bool trace = getenv("SQB200_TRACE_PERSISTENT") != nullptr;
  if (trace) fprintf(stderr, "persistent launch %p: %lld units, %d resident CTAs, grid %u x %u threads\n", L.fn, units,
                     slots, L.grid.x, L.block.x);
}

// Segment s of a single-context work list; form < 0 takes the context's choice.
SegLaunch seg_single(sqb200_jk* c, const sqb200_jk::Work* w, size_t s, const double* dPA, const double* dPB,
                     int uhf, int form) {
  SegLaunch L;
  const int v = w->kernel[s];
  const bool f32 = v >= sqb::kNumClassKernels;
  const int kidx = f32 ? v - sqb::kNumClassKernels : v;
  const sqb::ClassKernel& K = sqb::kClassKernels[kidx];
  const PairClass& B = c->cls[K.bra_cls];
  const PairClass& T = c->cls[K.ket_cls];
  sqb::JKArgs& a = L.a;
  memset(&a, 0, sizeof(a));
  a.bra_pairs = B.d_pairs; a.bra_prims = B.d_prims;
  a.ket_pairs = T.d_pairs; a.ket_prims = T.d_prims;
  a.PA = dPA; a.PB = dPB; a.PT = c->d_PT; a.PM = c->d_PM;
  a.Jacc = c->d_J; a.KAacc = c->d_KA; a.KBacc = c->d_KB;
  a.boys_tab = c->d_boys;
  a.boys_tab_f = c->d_boysf;
  a.counters = c->d_counters + 4 * v;
  a.bra_prims_f = B.d_primsf; a.ket_prims_f = T.d_primsf;
  a.mols = c->d_mol;
  a.same_class = K.bra_cls == K.ket_cls;
  L.items = w->d_items + w->first[s];
  if (c->mp_on && w->d_er) {
    a.erbank = c->d_erbank;
    a.erscr = c->d_erscr;
    a.er_items = w->d_er + w->first[s];
    a.mpole = c->d_mpole;
    a.pow15 = c->d_pow15;
    a.mp_rmax = c->mp_rmax;
    form = 0;                              // the narrow form carries the multipole mode
  }
  const bool ws = !f32 && !c->mp_on && c->use_ws && K.ws_r != nullptr;
  if (!f32) c->ran_ws[kidx] = ws;
  L.smem = (size_t)B.max_nprim * B.stride * (f32 ? sizeof(float) : sizeof(double)) +
           (ws ? (size_t)K.ws_warps * K.ws_nr * 32 * sizeof(double) : 0);
  int passes = 1;
  if (ws) {
    L.fn = uhf ? K.ws_u : K.ws_r;
  } else {
    const int fu = pick_form(K, f32, uhf, form < 0 ? c->form[kidx] : form, &L.fn, &passes);
    if (!f32) c->ran_form[kidx] = (char)fu;
    add_acc_region(K, fu, L);
  }
  L.grid = dim3(w->count[s], passes);
  L.block = dim3(ws ? 32 * K.ws_warps : cta_threads());
  if (c->persistent && !ws) make_persistent(L, c->d_queue + v);
  return L;
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
  const sqb::MolRec mv{0, 0, n, c->ns, outer, fixed, dscreen, 0, uhf};
  k_prep<<<grid_for(nn, 256), 256, 0, st>>>(dPA, dPB, c->d_PT, c->d_J, c->d_KA, c->d_KB, nn, uhf, c->d_mol, mv);
  launch_pmax(dPA, dPB, c->d_PT, c->d_shfirst, c->d_shn, c->ns, n, c->d_PM, st);
  CUDA_OK(cudaMemsetAsync(c->d_counters, 0, sizeof(unsigned long long) * 8 * sqb::kNumClassKernels, st));
  if (c->persistent) CUDA_OK(cudaMemsetAsync(c->d_queue, 0, sizeof(unsigned long long) * 2 * sqb::kNumClassKernels, st));
  c->last_launches = 3 + (int)w->kernel.size() + (w->gtotal > 0 ? 1 : 0);
  // segments largest first, each on the least-loaded lane (lane 0 = st, the others are side
  // streams forked off st); per-class profiling keeps every launch on st so that each event
  // pair times one kernel alone
  rc = ensure_side_streams(c);
  if (rc) return rc;
  const int nlanes = c->profile ? 1 : 1 + c->nside;
  std::vector<size_t> order(w->kernel.size());
  for (size_t s = 0; s < order.size(); ++s) order[s] = s;
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return w->cost[x] > w->cost[y]; });
  std::vector<double> load(nlanes, 0.0);
  std::vector<char> used(nlanes, 0);
  if (nlanes > 1) {
    CUDA_OK(cudaEventRecord(c->ev_fork, st));
    for (int l = 1; l < nlanes; ++l) CUDA_OK(cudaStreamWaitEvent(c->side[l - 1], c->ev_fork, 0));
  }
  if (c->gen.on) {
    // the generic path's quartets (f shells), on lane 0 ahead of the class kernels
    sqb::GenBuild gb{dPA, dPB, c->d_PT, c->d_PM, c->d_J, c->d_KA, c->d_KB, n, c->ns, uhf, outer, fixed, dscreen,
                     nullptr, nullptr, nullptr, nullptr, 0.0};
    if (c->mp_on && c->d_erbank) {
      gb.erbank = c->d_erbank;
      gb.erscr = c->d_erscr;
      gb.mpole = c->d_mpole;
      gb.pow15 = c->d_pow15;
      gb.mp_rmax = c->mp_rmax;
    }
    sqb200_jk::Ev ev{kGenericKernel, nullptr, nullptr};
    if (c->profile && w->gtotal > 0) {
      CUDA_OK(cudaEventCreate(&ev.a));
      CUDA_OK(cudaEventCreate(&ev.b));
      CUDA_OK(cudaEventRecord(ev.a, st));
    }
    rc = sqb::gen_launch(c->gen, w->d_gitems, w->gtotal, gb, st);
    if (rc) return rc;
    if (ev.a) {
      CUDA_OK(cudaEventRecord(ev.b, st));
      c->events.push_back(ev);
    }
    used[0] = 1;
  }
  for (size_t s : order) {
    const int lane = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    load[lane] += w->cost[s];
    used[lane] = 1;
    const cudaStream_t ls = lane == 0 ? st : c->side[lane - 1];
    const int v = w->kernel[s];
    const SegLaunch L = seg_single(c, w, s, dPA, dPB, uhf, -1);
    sqb200_jk::Ev ev{v, nullptr, nullptr};
    if (c->profile) {
      CUDA_OK(cudaEventCreate(&ev.a));
      CUDA_OK(cudaEventCreate(&ev.b));
      CUDA_OK(cudaEventRecord(ev.a, st));
    }
    rc = enqueue(L, ls);
    if (rc) return rc;
    if (c->profile) {
      CUDA_OK(cudaEventRecord(ev.b, st));
      c->events.push_back(ev);
    }
  }
  for (int l = 1; l < nlanes; ++l) {   // join (every forked lane, used or not, so st waits on all)
    CUDA_OK(cudaEventRecord(c->ev_join[l - 1], c->side[l - 1]));
    CUDA_OK(cudaStreamWaitEvent(st, c->ev_join[l - 1], 0));
  }
  if (c->mp_on && c->er_total > 0)
    k_erbank<<<grid_for(c->er_total, 256), 256, 0, st>>>(c->d_erbank, c->d_erscr, c->er_total);
  k_finalize<<<grid_for(nn, 256), 256, 0, st>>>(c->d_J, c->d_KA, c->d_KB, dJT, dKA, dKB, n, uhf);
  CUDA_OK(cudaGetLastError());
  return SQB200_OK;
}

// Algorithmic FP64/FP32 operations of kernel index v (FP64 form v < K, FP32 form v - K)
// from its four counters [quartets, primitive quartets, bra flushes, digestions]: per
// primitive quartet the pass-free count (Boys function and R once), per flush and digestion
// the operations of the form that ran (those are not repeated across passes).
double kernel_flops_form(int v, int form, const unsigned long long* h) {
  const int K_ = sqb::kNumClassKernels;
  const bool f32 = v >= K_;
  const sqb::ClassKernel& K = sqb::kClassKernels[f32 ? v - K_ : v];
  const double fp = K.alg_flops_prim;
  const double ff = f32 ? K.f32_flops_flush : form == 1 ? K.w_flops_flush : form == 2 ? K.s_flops_flush : K.flops_flush;
  const double fq = f32 ? K.f32_flops_quartet : form == 1 ? K.w_flops_quartet : form == 2 ? K.s_flops_quartet : K.flops_quartet;
  return (double)h[1] * fp + (double)h[2] * ff + (double)h[3] * fq;
}

double kernel_flops(const sqb200_jk* c, int v, const unsigned long long* h) {
  const bool f32 = v >= sqb::kNumClassKernels;
  return kernel_flops_form(v, f32 || v >= (int)c->ran_form.size() ? 0 : c->ran_form[v], h);
}

// The autotuner times every form of a class in up to kTuneRounds interleaved rounds (narrow,
// wide, swapped, narrow, ...) and keeps each form's fastest round, so that clocks still ramping
// up at start-up or a stray slow launch do not favour the forms timed later.  Launches longer
// than kTuneLongMs get one round: the ramp is over long before, and more rounds of a large
// batch would only lengthen the set-up.
constexpr int kTuneRounds = 3;
constexpr double kTuneLongMs = 2.0;

// The form to run from the forms' times t[0..2]: the narrow tile unless another form is at
// least 3% faster than every form before it (near-ties keep the earlier form, so that the
// choice does not flip between runs).
int pick_tuned(const sqb::ClassKernel& K, const double* t) {
  int bf = 0;
  for (int f = 1; f < 3; ++f)
    if (has_form(K, f) && t[f] < 0.97 * t[bf]) bf = f;
  return bf;
}

// Mean device time (ms) of `reps` launches of L on st after one untimed launch.
int time_seg(const SegLaunch& L, cudaStream_t st, int reps, double* ms) {
  cudaEvent_t a, b;
  CUDA_OK(cudaEventCreate(&a));
  CUDA_OK(cudaEventCreate(&b));
  int rc = enqueue(L, st);
  if (!rc) rc = cudaEventRecord(a, st) == cudaSuccess ? SQB200_OK : fail(SQB200_ECUDA, "cudaEventRecord");
  for (int r = 0; r < reps && !rc; ++r) rc = enqueue(L, st);
  if (!rc) rc = cudaEventRecord(b, st) == cudaSuccess ? SQB200_OK : fail(SQB200_ECUDA, "cudaEventRecord");
  float t = 0.f;
  if (!rc) rc = cudaEventSynchronize(b) == cudaSuccess ? SQB200_OK : fail(SQB200_ECUDA, "cudaEventSynchronize");
  if (!rc) rc = cudaEventElapsedTime(&t, a, b) == cudaSuccess ? SQB200_OK : fail(SQB200_ECUDA, "cudaEventElapsedTime");
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = t / reps;
  return rc;
}

}  // namespace

// ---------------------------------------------------------------- Boys function check

// F_0..F_M(T[i]) by the class kernels' own device routine sqb::boys<M>.
template <int M>
__global__ void k_boys_eval(const double* __restrict__ T, int n, const double* __restrict__ tab,
                            double* __restrict__ F) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double f[M + 1];
  sqb::boys<M>(T[i], tab, f);
  for (int m = 0; m <= M; ++m) F[(size_t)i * (M + 1) + m] = f[m];
}

template <int M>
void launch_boys(const double* T, int n, const double* tab, double* F) {
  k_boys_eval<M><<<(n + 127) / 128, 128>>>(T, n, tab, F);
}

// ---------------------------------------------------------------- multipole table (host)
//
// genMultipole (reference src/multipole.c:33-86) for every function pair (p, q): the charge
// q = <p|q> (contracted overlap, set to 0 below 1e-18 in magnitude) and the charge centre, the
// midpoint of the two function centres moved by dipole/q (the dipole <p|r - mid|q> taken about
// that midpoint), stored as [q, x, y, z] at 4 (p nbf + q).  Primitive integrals by
// McMurchie-Davidson: <a|b> = e^{-mu R^2} (pi/p)^{3/2} Ex_0 Ey_0 Ez_0 and
// <a|x - xc|b> = e^{-mu R^2} (pi/p)^{3/2} (Ex_1 + (Px - xc) Ex_0) Ey_0 Ez_0, summed over the
// primitives of p (outer) and q (inner) as the reference's GTO_overlap / GTO_moment do.
void multipole_table(const sqb200_jk* c, std::vector<double>& tab) {
  const int n = c->nbf;
  tab.assign((size_t)4 * n * n, 0.0);
  for (const Shell& A : c->shells)
    for (const Shell& B : c->shells)
      for (int f = 0; f < A.nfunc; ++f)
        for (int g = 0; g < B.nfunc; ++g) {
          const int la = A.lmn[f][0], ma = A.lmn[f][1], na = A.lmn[f][2];
          const int lb = B.lmn[g][0], mb = B.lmn[g][1], nb = B.lmn[g][2];
          const double mx = 0.5 * (A.x + B.x), my = 0.5 * (A.y + B.y), mz = 0.5 * (A.z + B.z);
          double q = 0.0, dx = 0.0, dy = 0.0, dz = 0.0;
          for (int k = 0; k < A.nprim; ++k)
            for (int l = 0; l < B.nprim; ++l) {
              const double a = A.exps[k], b = B.exps[l], p = a + b, mu = a * b / p;
              const double Px = (a * A.x + b * B.x) / p, Py = (a * A.y + b * B.y) / p, Pz = (a * A.z + b * B.z) / p;
              const double R2 = (A.x - B.x) * (A.x - B.x) + (A.y - B.y) * (A.y - B.y) + (A.z - B.z) * (A.z - B.z);
              double Ex[4][4][7], Ey[4][4][7], Ez[4][4][7];
              hermite_e(p, Px - A.x, Px - B.x, Ex);
              hermite_e(p, Py - A.y, Py - B.y, Ey);
              hermite_e(p, Pz - A.z, Pz - B.z, Ez);
              const double w = A.coef[k][f] * B.coef[l][g] * exp(-mu * R2) * pow(M_PI / p, 1.5);
              const double sx = Ex[la][lb][0], sy = Ey[ma][mb][0], sz = Ez[na][nb][0];
              q += w * sx * sy * sz;
              dx += w * (Ex[la][lb][1] + (Px - mx) * sx) * sy * sz;
              dy += w * sx * (Ey[ma][mb][1] + (Py - my) * sy) * sz;
              dz += w * sx * sy * (Ez[na][nb][1] + (Pz - mz) * sz);
            }
          if (fabs(q) < 1e-18) q = 0.0;                  // MULTIPOLE_CHARGE_CUTOFF
          double x = mx, y = my, z = mz;
          if (q != 0.0) { x += dx / q; y += dy / q; z += dz / q; }
          double* o = tab.data() + 4 * ((size_t)(A.first + f) * n + B.first + g);
          o[0] = q; o[1] = x; o[2] = y; o[3] = z;
        }
}

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
  const char* pe = getenv("SQB200_PERSISTENT");
  c->persistent = pe && pe[0] == '1';
  c->ran_ws.assign(sqb::kNumClassKernels, 0);
  c->form.assign(sqb::kNumClassKernels, 0);
  c->ran_form.assign(sqb::kNumClassKernels, 0);
  c->nbf = nbf;
  int rc = build_shells(nbf, nprim, lmn, xyz, exps, ncoefs, c->shells);
  if (rc) { delete c; return rc; }
  c->ns = (int)c->shells.size();
  if (schwarz) c->schwarz.assign(schwarz, schwarz + (size_t)nbf * nbf);
  else c->schwarz.assign((size_t)nbf * nbf, 1.0);   // placeholder until the device pass below
  build_pairs(c);
  rc = upload_pairs(c);
  if (!rc) rc = setup_generic(c);
  if (rc) { sqb200_jk_destroy(c); return rc; }
  const size_t nn = (size_t)nbf * nbf;
  std::vector<double> tab = make_boys_table();
  std::vector<int> fst(c->ns), nf(c->ns);
  for (int s = 0; s < c->ns; ++s) { fst[s] = c->shells[s].first; nf[s] = c->shells[s].nfunc; }
  Carve cv;
  cv.add(&c->d_boys, tab.size() * sizeof(double));
  cv.add(&c->d_boysf, tab.size() * sizeof(float));
  cv.add(&c->d_shfirst, c->ns * sizeof(int));
  cv.add(&c->d_shn, c->ns * sizeof(int));
  for (double** m : {&c->d_PA, &c->d_PB, &c->d_PT, &c->d_J, &c->d_KA, &c->d_KB, &c->d_JT, &c->d_KAo, &c->d_KBo})
    cv.add(m, nn * sizeof(double));
  cv.add(&c->d_PM, (size_t)c->ns * c->ns * sizeof(double));
  cv.add(&c->d_counters, 8 * sqb::kNumClassKernels * sizeof(unsigned long long));
  cv.add(&c->d_queue, 2 * sqb::kNumClassKernels * sizeof(unsigned long long));
  cv.add(&c->d_mol, sizeof(sqb::MolRec));
  cudaError_t e = cv.alloc(&c->d_base);
  if (e != cudaSuccess) {
    sqb200_jk_destroy(c);
    return fail(SQB200_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = h2d(c->d_boys, tab.data(), tab.size() * sizeof(double), c->stream);
  std::vector<float> tabf(tab.begin(), tab.end());
  if (e == cudaSuccess) e = h2d(c->d_boysf, tabf.data(), tabf.size() * sizeof(float), c->stream);
  if (e == cudaSuccess) e = h2d(c->d_shfirst, fst.data(), c->ns * sizeof(int), c->stream);
  if (e == cudaSuccess) e = h2d(c->d_shn, nf.data(), c->ns * sizeof(int), c->stream);
  if (e != cudaSuccess) { sqb200_jk_destroy(c); return fail(SQB200_ECUDA, cudaGetErrorString(e)); }
  if (!schwarz) {
    // Schwarz bounds from the device, then the pair lists in their final (sorted) order
    rc = compute_schwarz_device(c, c->schwarz.data());
    if (rc) { sqb200_jk_destroy(c); return rc; }
    build_pairs(c);
    rc = upload_pairs(c);
    if (!rc) rc = setup_generic(c);
    if (rc) { sqb200_jk_destroy(c); return rc; }
  }
  // the scratch array of sqb200_jk_build_noalloc: its device address on this device, looked up
  // here so that the no-allocation entry point itself does no set-up (a failed lookup only
  // disables that entry point, which then reports this error)
  c->noalloc_err = noalloc_lookup(&c->noalloc_base);
  if (c->noalloc_err != cudaSuccess) (void)cudaGetLastError();
  *out = c;
  return SQB200_OK;
}

int sqb200_jk_destroy(sqb200_jk* c) {
  if (!c) return SQB200_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (size_t i = 0; i < c->side.size(); ++i) {
    cudaStreamSynchronize(c->side[i]);
    cudaStreamDestroy(c->side[i]);
    cudaEventDestroy(c->ev_join[i]);
  }
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  for (auto& kv : c->work) { cudaFree(kv.second.d_items); cudaFree(kv.second.d_er); cudaFree(kv.second.d_gitems); }
  sqb::gen_free(c->gen);
  if (c->d_mpbase) cudaFree(c->d_mpbase);
  if (c->d_erbase) cudaFree(c->d_erbase);
  for (auto& e : c->events) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
  free_pairs(c);
  cudaFree(c->d_base);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return SQB200_OK;
}

int sqb200_jk_autotune(sqb200_jk* c, const double* dPA, const double* dPB, int restricted, double outer,
                       double fixed, double dscreen, void* stream) {
  if (!c || !dPA) return fail(SQB200_EINVAL, "null argument");
  CUDA_OK(cudaSetDevice(c->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  const int uhf = restricted ? 0 : 1;
  if (dPB == nullptr) dPB = dPA;
  sqb200_jk::Work* w = nullptr;
  int rc = build_work(c, outer, fixed, &w);
  if (rc) return rc;
  // the class kernels read PT, PM and the molecule record: set them up as a build does
  const int n = c->nbf, nn = n * n;
  const sqb::MolRec mv{0, 0, n, c->ns, outer, fixed, dscreen, 0, uhf};
  k_prep<<<grid_for(nn, 256), 256, 0, st>>>(dPA, dPB, c->d_PT, c->d_J, c->d_KA, c->d_KB, nn, uhf, c->d_mol, mv);
  launch_pmax(dPA, dPB, c->d_PT, c->d_shfirst, c->d_shn, c->ns, n, c->d_PM, st);
  for (size_t s = 0; s < w->kernel.size(); ++s) {
    const int v = w->kernel[s];
    if (v >= sqb::kNumClassKernels) continue;
    double tf[3] = {0.0, 0.0, 0.0};
    for (int round = 0; round < kTuneRounds; ++round) {
      for (int f = 0; f < 3; ++f) {
        if (!has_form(sqb::kClassKernels[v], f)) continue;
        double t = 0.0;
        rc = time_seg(seg_single(c, w, s, dPA, dPB, uhf, f), st, 2, &t);
        if (rc) return rc;
        tf[f] = round == 0 ? t : std::min(tf[f], t);
      }
      if (tf[0] > kTuneLongMs) break;
    }
    c->form[v] = (char)pick_tuned(sqb::kClassKernels[v], tf);
  }
  CUDA_OK(cudaStreamSynchronize(st));
  return SQB200_OK;
}

int sqb200_jk_tiles(sqb200_jk* c, int* form, int n) {
  if (!c || !form) return fail(SQB200_EINVAL, "null argument");
  for (int k = 0; k < n && k < sqb::kNumClassKernels; ++k) {
    const sqb::ClassKernel& K = sqb::kClassKernels[k];
    form[k] = (K.fn_rw || K.fn_rs) ? c->form[k] : -1;
  }
  return std::min(n, sqb::kNumClassKernels);
}

int sqb200_jk_set_tiles(sqb200_jk* c, const int* form, int n) {
  if (!c || !form) return fail(SQB200_EINVAL, "null argument");
  for (int k = 0; k < n && k < sqb::kNumClassKernels; ++k)
    c->form[k] = (char)(has_form(sqb::kClassKernels[k], form[k]) ? form[k] : 0);
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
  if (c->gen.on) {
    unsigned long long g2[3];
    CUDA_OK(cudaMemcpy(g2, c->gen.d_counters, sizeof(g2), cudaMemcpyDeviceToHost));
    q += (long long)g2[0];
    pq += (long long)g2[1];
    fl += (long long)g2[2];
  }
  long long v[6] = {q, pq, fl, (long long)c->ns, 0, (long long)c->last_launches};
  for (int k = 0; k < sqb::kNumPairClasses; ++k) v[4] += (long long)c->cls[k].pairs.size();
  v[4] += (long long)c->gen.gen_idx.size();
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
  c->prof_ms.assign(kGenericKernel + 1, 0.0);
  c->prof_launches.assign(kGenericKernel + 1, 0);
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
    if (c->prof_ms.size() != (size_t)(kGenericKernel + 1)) {
      c->prof_ms.assign(kGenericKernel + 1, 0.0);
      c->prof_launches.assign(kGenericKernel + 1, 0);
    }
    c->prof_ms[e.kernel] += ms;
    c->prof_launches[e.kernel] += 1;
    cudaEventDestroy(e.a);
    cudaEventDestroy(e.b);
  }
  c->events.clear();
  std::vector<unsigned long long> h(8 * sqb::kNumClassKernels);
  CUDA_OK(cudaMemcpy(h.data(), c->d_counters, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  unsigned long long g2[3] = {0, 0, 0};
  if (c->gen.on) CUDA_OK(cudaMemcpy(g2, c->gen.d_counters, sizeof(g2), cudaMemcpyDeviceToHost));
  int r = 0;
  for (int v = 0; v <= kGenericKernel && r < max_rows; ++v) {
    if ((int)c->prof_launches.size() <= v || c->prof_launches[v] == 0) continue;
    double* row = rows + 6 * r;
    row[0] = v;
    row[1] = (double)c->prof_launches[v];
    row[2] = c->prof_ms[v];
    // (the generic path counts the operations it executes: Boys seeds, R recursion, the ket and
    // bra Hermite sums and the digestion)
    row[3] = v == kGenericKernel ? (double)g2[2] : kernel_flops(c, v, &h[4 * v]);
    row[4] = v == kGenericKernel ? (double)g2[1] : (double)h[4 * v + 1];
    row[5] = v == kGenericKernel ? (double)g2[0] : (double)h[4 * v];
    ++r;
  }
  *nrows = r;
  return SQB200_OK;
}

const char* sqb200_jk_class_name(int k) {
  if (k == kGenericKernel) return "generic (f shells)";
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

int sqb200_boys_eval(int device, int mmax, int n, const double* T, double* F) {
  if (!T || !F || n <= 0 || mmax < 0 || mmax > BOYS_MMAX)
    return fail(SQB200_EINVAL, "sqb200_boys_eval: null array, n <= 0 or mmax outside 0..8");
  for (int i = 0; i < n; ++i)
    if (!(T[i] >= 0.0)) return fail(SQB200_EINVAL, "sqb200_boys_eval: T must be >= 0");
  CUDA_OK(cudaSetDevice(device));
  const std::vector<double> tab = make_boys_table();
  double *dT = nullptr, *dF = nullptr, *dtab = nullptr;
  const size_t nf = (size_t)n * (mmax + 1);
  cudaError_t e = cudaMalloc(&dT, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&dF, nf * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&dtab, tab.size() * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(dT, T, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dtab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    switch (mmax) {
      case 0: launch_boys<0>(dT, n, dtab, dF); break;
      case 1: launch_boys<1>(dT, n, dtab, dF); break;
      case 2: launch_boys<2>(dT, n, dtab, dF); break;
      case 3: launch_boys<3>(dT, n, dtab, dF); break;
      case 4: launch_boys<4>(dT, n, dtab, dF); break;
      case 5: launch_boys<5>(dT, n, dtab, dF); break;
      case 6: launch_boys<6>(dT, n, dtab, dF); break;
      case 7: launch_boys<7>(dT, n, dtab, dF); break;
      default: launch_boys<8>(dT, n, dtab, dF); break;
    }
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(F, dF, nf * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(dT); cudaFree(dF); cudaFree(dtab);
  if (e != cudaSuccess) return fail(SQB200_ECUDA, std::string("sqb200_boys_eval: ") + cudaGetErrorString(e));
  return SQB200_OK;
}

int sqb200_jk_set_persistent(sqb200_jk* c, int enable) {
  if (!c) return fail(SQB200_EINVAL, "null context");
  c->persistent = enable != 0;
  return SQB200_OK;
}

int sqb200_jk_set_multipole(sqb200_jk* c, int enable, double cache_rmax) {
  if (!c || (enable && !(cache_rmax >= 0.0))) return fail(SQB200_EINVAL, "null context or negative memory cutoff");
  CUDA_OK(cudaSetDevice(c->device));
  if (!enable) {
    c->mp_on = false;
    return SQB200_OK;
  }
  if (!c->d_mpbase) {
    std::vector<double> tab, pw(sqb::ERR_MAX - sqb::ERR_MIN + 1);
    multipole_table(c, tab);
    for (int e = sqb::ERR_MIN; e <= sqb::ERR_MAX; ++e) pw[e - sqb::ERR_MIN] = pow(1.5, (double)e);
    Staged sg;
    sg.put(&c->d_mpole, tab.size() * sizeof(double), tab.data());
    sg.put(&c->d_pow15, pw.size() * sizeof(double), pw.data());
    cudaError_t e = sg.upload(&c->d_mpbase, c->stream);
    if (e != cudaSuccess) return fail(SQB200_ENOMEM, std::string("multipole table: ") + cudaGetErrorString(e));
  }
  c->mp_on = true;
  c->mp_rmax = cache_rmax;
  return SQB200_OK;
}

int sqb200_jk_mem_cutoff(sqb200_jk* c, double fixed, int max_mem_mb, double* out) {
  // getMemCutoff_Parallel (reference src/matrix.c:3703-3760), nCPU = 1: starting from `fixed`,
  // double the cutoff until the shell quartets whose Schwarz product reaches it hold at most
  // max_mem_mb MB of doubles, step back by half and rise by 5% until they fit again.  The
  // quartets are the canonical ones, pair(I,J) <= pair(P,Q) in lower-triangle order, and the
  // reference skips one when S_PQ * S_IJ < cut.  Each count here is exact in
  // O(pairs log pairs) instead of a pass over all quartets: the pairs sorted by their bound, a
  // Fenwick tree over that order filled in pair order, and for pair PQ a binary search for the
  // first sorted bound b with S_PQ * b >= cut (a rounded product is monotonic in b, so the
  // search selects exactly the quartets the reference keeps).
  if (!c || !out) return fail(SQB200_EINVAL, "null argument");
  const std::vector<Shell>& sh = c->shells;
  const int ns = c->ns;
  const size_t np = (size_t)ns * (ns + 1) / 2;
  std::vector<double> sv(np);                    // Schwarz block max per pair, pair order
  std::vector<unsigned long long> wv(np);        // functions per pair
  for (int P = 0, k = 0; P < ns; ++P)
    for (int Q = 0; Q <= P; ++Q, ++k) {
      double r = 0.0;
      for (int p = 0; p < sh[P].nfunc; ++p)
        for (int q = 0; q < sh[Q].nfunc; ++q) r = std::max(r, c->schwarz[(size_t)(sh[P].first + p) * c->nbf + sh[Q].first + q]);
      sv[k] = r;
      wv[k] = (unsigned long long)sh[P].nfunc * sh[Q].nfunc;
    }
  std::vector<int> order(np), rank(np);
  for (size_t k = 0; k < np; ++k) order[k] = (int)k;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return sv[a] < sv[b]; });
  std::vector<double> vs(np);
  for (size_t k = 0; k < np; ++k) { rank[order[k]] = (int)k; vs[k] = sv[order[k]]; }
  std::vector<unsigned long long> fen(np + 1);
  const unsigned long long maxEE = (unsigned long long)max_mem_mb * 1000000ULL / sizeof(double);
  // true when the quartets kept at `cut` exceed maxEE; *cnt = their function count otherwise
  auto over = [&](double cut, unsigned long long* cnt) {
    std::fill(fen.begin(), fen.end(), 0ULL);
    unsigned long long tot = 0, ins = 0;
    for (size_t pq = 0; pq < np; ++pq) {
      for (size_t i = rank[pq] + 1; i <= np; i += i & (~i + 1)) fen[i] += wv[pq];
      ins += wv[pq];
      const double s = sv[pq];
      size_t lo = 0, hi = np;                      // first k with s * vs[k] >= cut
      while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if (s * vs[mid] < cut) lo = mid + 1; else hi = mid;
      }
      unsigned long long below = 0;                // inserted weight at ranks < lo
      for (size_t i = lo; i > 0; i -= i & (~i + 1)) below += fen[i];
      tot += wv[pq] * (ins - below);
      if (tot > maxEE) return true;
    }
    *cnt = tot;
    return false;
  };
  double cut = fixed;
  bool coarse = true;
  for (;;) {
    unsigned long long cnt = 0;
    if (over(cut, &cnt)) { cut *= coarse ? 2.00 : 1.05; continue; }
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
constexpr size_t kNoAllocMolOff = (kNoAllocItemsOff + (size_t)kNoAllocMaxItems * sizeof(sqb::WorkItem) + 255) / 256 * 256;
constexpr size_t kNoAllocBytes = kNoAllocMolOff + 256;   // one molecule record

static_assert(sizeof(sqb::MolRec) <= 256, "the molecule record must fit the 256 bytes reserved for it");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// The host-side symbol g_noalloc_scratch is only a stand-in: its device address on the current
// device comes from the runtime (called by sqb200_jk_create with the context's device current).
cudaError_t noalloc_lookup(unsigned char** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e == cudaSuccess && p == nullptr) e = cudaErrorInvalidSymbol;
  *out = e == cudaSuccess ? (unsigned char*)p : nullptr;
  return e;
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
          for (int k0 = start; k0 < lo; k0 += kper) items.push_back({b, k0, std::min(kper, lo - k0), isplit, 0});
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
  if (c->gen.on) return fail(SQB200_EUNSUPPORTED, "sqb200_jk_build_noalloc: shells outside s, sp, p, d (f shells)");
  CUDA_OK(cudaSetDevice(c->device));
  unsigned char* base = c->noalloc_base;
  if (!base)
    return fail(SQB200_ECUDA, std::string("sqb200_jk_build_noalloc: no device address for its scratch array: ") +
                                  cudaGetErrorString(c->noalloc_err));
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
  sqb::MolRec* d_mol = (sqb::MolRec*)(base + kNoAllocMolOff);
  const sqb::MolRec mv{0, 0, n, c->ns, outer, fixed, dscreen, 0, uhf};
  k_prep<<<grid_for(nn, 256), 256, 0, st>>>(dPA, dPB, PT, J, KA, KB, nn, uhf, d_mol, mv);
  launch_pmax(dPA, dPB, PT, c->d_shfirst, c->d_shn, c->ns, n, PM, st);
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
    a.mols = d_mol;
    a.same_class = K.bra_cls == K.ket_cls;
    const sqb::WorkItem* it = d_items + first[s];
    void* args[] = {&a, &it};
    const size_t smem = (size_t)B.max_nprim * B.stride * sizeof(double);
    const void* fn = uhf ? K.fn_u : K.fn_r;
    const int rs = ensure_smem(fn, smem);
    if (rs) return rs;
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
  Staged up;
  up.put(&d_np, n * sizeof(int), np.data());
  up.put(&d_off, n * sizeof(int), off.data());
  up.put(&d_lmn, 3 * n * sizeof(int), lmn.data());
  up.put(&d_xyz, 3 * n * sizeof(double), xyz.data());
  up.put(&d_ex, ex.size() * sizeof(double), ex.data());
  up.put(&d_nc, nc.size() * sizeof(double), nc.data());
  up.put(&d_Z, natom * sizeof(double), natom > 0 ? Z : nullptr);
  up.put(&d_A, 3 * natom * sizeof(double), natom > 0 ? axyz : nullptr);
  up.put(&d_out, 3 * nn * sizeof(double), nullptr);
  void* base = nullptr;
  cudaError_t e = up.upload(&base, c->stream);
  if (e == cudaSuccess) {
    k_oneint<<<(int)((nn + 127) / 128), 128, 0, c->stream>>>(n, d_np, d_off, d_lmn, d_xyz, d_ex, d_nc, natom, d_Z, d_A,
                                                              c->d_boys, d_out, d_out + nn, d_out + 2 * nn);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(S, d_out, nn * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(T, d_out + nn, nn * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(V, d_out + 2 * nn, nn * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(base);
  if (e != cudaSuccess) return fail(SQB200_ECUDA, std::string("sqb200_oneint: ") + cudaGetErrorString(e));
  return SQB200_OK;
}

// ---------------------------------------------------------------- batched builds
//
// A batch joins the contexts of many molecules (each created by sqb200_jk_create) into one set
// of merged class arrays, so that one launch per class kernel carries the work items of every
// molecule.  Densities and outputs are packed: molecule m's nbf_m x nbf_m block starts at
// offset off[m] of every array.  Pair records keep molecule-local shell and function indices;
// each work item names its molecule, whose MolRec gives the matrix offsets and cutoffs.

struct sqb200_batch {
  int device = 0, nmol = 0;
  std::vector<sqb200_jk*> mols;
  std::vector<long long> moff, pmoff;   // nmol + 1 entries
  std::vector<int> shoff;               // nmol + 1 entries
  int max_ns = 0, max_nbf = 0;
  struct Cls {
    std::vector<int> pair_base;         // per molecule: its first pair in the merged array
    int max_nprim = 0, stride = 0;
    sqb::PairRec* d_pairs = nullptr;
    double* d_prims = nullptr;
    float* d_primsf = nullptr;
  } cls[sqb::kNumPairClasses];
  std::vector<sqb::MolRec> rec;
  sqb::MolRec* d_mols = nullptr;
  int *d_shfirst = nullptr, *d_shn = nullptr;
  double *d_PT = nullptr, *d_PM = nullptr, *d_J = nullptr, *d_KA = nullptr, *d_KB = nullptr;
  unsigned long long* d_counters = nullptr;   // 4 per kernel form and spin: [spin][2K][4]
  unsigned long long* d_queue = nullptr;      // persistent launches: per kernel form and spin [spin][2K]
  bool persistent = false;
  // work list of the current step: segments per (class kernel form, spin)
  std::vector<int> kernel, spin, first, count;
  std::vector<double> cost;
  sqb::WorkItem* d_items = nullptr;
  size_t items_cap = 0;
  bool have_step = false;
  std::vector<unsigned long long> last_counts;
  std::vector<char> form;               // per class kernel: FP64 form (sqb200_batch_autotune)
  int last_launches = 0;
  int nside = -1;
  std::vector<cudaStream_t> side;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
  cudaStream_t stream = nullptr;
};

namespace {

// PM blocks of every molecule of a batch: grid.y = molecule
__global__ void k_pmax_batch(const double* __restrict__ PA, const double* __restrict__ PB,
                             const double* __restrict__ PT, const int* __restrict__ first,
                             const int* __restrict__ nf, const sqb::MolRec* __restrict__ mols,
                             double* __restrict__ PM) {
  const sqb::MolRec mr = mols[blockIdx.y];
  const int ns = mr.ns, n = mr.nbf;
  const int* f = first + mr.shoff;
  const int* c = nf + mr.shoff;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ns * ns; idx += gridDim.x * blockDim.x) {
    const int P = idx / ns, Q = idx % ns;
    double r = 0.0;
    for (int p = 0; p < c[P]; ++p)
      for (int q = 0; q < c[Q]; ++q) {
        const long long o = mr.moff + (long long)(f[P] + p) * n + f[Q] + q;
        r = fmax(r, fabs(PT[o]));
        r = fmax(r, fabs(PA[o]));
        r = fmax(r, fabs(PB[o]));
      }
    PM[mr.pmoff + idx] = r;
  }
}

// per-molecule symmetrisation of a batch: JT = J + J^T, KA = -(K + K^T), KB likewise or = KA
__global__ void k_finalize_batch(const double* __restrict__ J, const double* __restrict__ KA,
                                 const double* __restrict__ KB, double* __restrict__ JT,
                                 double* __restrict__ KAo, double* __restrict__ KBo,
                                 const sqb::MolRec* __restrict__ mols) {
  const sqb::MolRec mr = mols[blockIdx.y];
  const int n = mr.nbf;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * n; i += gridDim.x * blockDim.x) {
    const int r = i / n, c = i % n;
    const long long a = mr.moff + i, t = mr.moff + (long long)c * n + r;
    JT[a] = J[a] + J[t];
    const double ka = -(KA[a] + KA[t]);
    KAo[a] = ka;
    KBo[a] = mr.uhf ? -(KB[a] + KB[t]) : ka;
  }
}

void free_batch(sqb200_batch* b) {
  for (size_t i = 0; i < b->side.size(); ++i) {
    cudaStreamSynchronize(b->side[i]);
    cudaStreamDestroy(b->side[i]);
    cudaEventDestroy(b->ev_join[i]);
  }
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->stream) { cudaStreamSynchronize(b->stream); cudaStreamDestroy(b->stream); }
  for (auto& k : b->cls) { cudaFree(k.d_pairs); cudaFree(k.d_prims); cudaFree(k.d_primsf); }
  void* ptrs[] = {b->d_mols, b->d_shfirst, b->d_shn, b->d_PT, b->d_PM, b->d_J, b->d_KA, b->d_KB,
                  b->d_counters, b->d_queue, b->d_items};
  for (void* p : ptrs) cudaFree(p);
  delete b;
}

}  // namespace

extern "C" int sqb200_batch_create(sqb200_batch** out, int nmol, sqb200_jk* const* mols) {
  if (!out || nmol <= 0 || !mols) return fail(SQB200_EINVAL, "sqb200_batch_create: null argument or nmol <= 0");
  if (nmol > 65535) return fail(SQB200_EINVAL, "sqb200_batch_create: at most 65535 molecules per batch");
  *out = nullptr;
  for (int m = 0; m < nmol; ++m) {
    if (!mols[m]) return fail(SQB200_EINVAL, "sqb200_batch_create: null context");
    if (mols[m]->device != mols[0]->device) return fail(SQB200_EINVAL, "sqb200_batch_create: contexts on different devices");
    if (mols[m]->gen.on) return fail(SQB200_EUNSUPPORTED, "sqb200_batch_create: shells outside s, sp, p, d (f shells)");
  }
  sqb200_batch* b = new sqb200_batch();
  b->device = mols[0]->device;
  b->nmol = nmol;
  b->mols.assign(mols, mols + nmol);
  b->moff.assign(nmol + 1, 0);
  b->pmoff.assign(nmol + 1, 0);
  b->shoff.assign(nmol + 1, 0);
  for (int m = 0; m < nmol; ++m) {
    const sqb200_jk* c = mols[m];
    b->moff[m + 1] = b->moff[m] + (long long)c->nbf * c->nbf;
    b->pmoff[m + 1] = b->pmoff[m] + (long long)c->ns * c->ns;
    b->shoff[m + 1] = b->shoff[m] + c->ns;
    b->max_ns = std::max(b->max_ns, c->ns);
    b->max_nbf = std::max(b->max_nbf, c->nbf);
  }
  cudaError_t e = cudaSetDevice(b->device);
  auto bail = [&](int code, const std::string& msg) { free_batch(b); return fail(code, "sqb200_batch_create: " + msg); };
  if (e != cudaSuccess) return bail(SQB200_ECUDA, cudaGetErrorString(e));
  // merged class arrays
  for (int k = 0; k < sqb::kNumPairClasses; ++k) {
    auto& bc = b->cls[k];
    std::vector<sqb::PairRec> pairs;
    std::vector<double> prims;
    bc.pair_base.assign(nmol, 0);
    for (int m = 0; m < nmol; ++m) {
      const PairClass& pc = mols[m]->cls[k];
      bc.pair_base[m] = (int)pairs.size();
      if (pc.pairs.empty()) continue;
      const int pbase = (int)prims.size();
      for (sqb::PairRec r : pc.pairs) { r.poff += pbase; pairs.push_back(r); }
      prims.insert(prims.end(), pc.prims.begin(), pc.prims.end());
      bc.max_nprim = std::max(bc.max_nprim, pc.max_nprim);
      bc.stride = pc.stride;
    }
    if (pairs.empty()) continue;
    if (prims.size() >= (size_t)INT_MAX) return bail(SQB200_EINVAL, "merged primitive array exceeds 2^31 entries");
    std::vector<float> pf(prims.begin(), prims.end());
    e = cudaMalloc(&bc.d_pairs, pairs.size() * sizeof(sqb::PairRec));
    if (e == cudaSuccess) e = cudaMalloc(&bc.d_prims, prims.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&bc.d_primsf, pf.size() * sizeof(float));
    if (e != cudaSuccess) return bail(SQB200_ENOMEM, cudaGetErrorString(e));
    e = h2d(bc.d_pairs, pairs.data(), pairs.size() * sizeof(sqb::PairRec), b->stream);
    if (e == cudaSuccess) e = h2d(bc.d_prims, prims.data(), prims.size() * sizeof(double), b->stream);
    if (e == cudaSuccess) e = h2d(bc.d_primsf, pf.data(), pf.size() * sizeof(float), b->stream);
    if (e != cudaSuccess) return bail(SQB200_ECUDA, cudaGetErrorString(e));
  }
  // packed shell tables and per-molecule buffers
  std::vector<int> fst, nf;
  for (int m = 0; m < nmol; ++m)
    for (const Shell& sh : mols[m]->shells) { fst.push_back(sh.first); nf.push_back(sh.nfunc); }
  const size_t ntot = (size_t)b->moff[nmol], pmtot = (size_t)b->pmoff[nmol];
  e = cudaMalloc(&b->d_mols, nmol * sizeof(sqb::MolRec));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_shfirst, fst.size() * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_shn, nf.size() * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_PT, ntot * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_PM, pmtot * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_J, ntot * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_KA, ntot * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_KB, ntot * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_counters, 2 * 8 * sqb::kNumClassKernels * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_queue, 2 * 2 * sqb::kNumClassKernels * sizeof(unsigned long long));
  if (e != cudaSuccess) return bail(SQB200_ENOMEM, cudaGetErrorString(e));
  e = h2d(b->d_shfirst, fst.data(), fst.size() * sizeof(int), b->stream);
  if (e == cudaSuccess) e = h2d(b->d_shn, nf.data(), nf.size() * sizeof(int), b->stream);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(SQB200_ECUDA, cudaGetErrorString(e));
  b->form.assign(sqb::kNumClassKernels, 0);
  b->persistent = mols[0]->persistent;
  b->rec.resize(nmol);
  for (int m = 0; m < nmol; ++m)
    b->rec[m] = sqb::MolRec{b->moff[m], b->pmoff[m], mols[m]->nbf, mols[m]->ns, 0.0, 0.0, 0.0, b->shoff[m], 0};
  *out = b;
  return SQB200_OK;
}

extern "C" int sqb200_batch_destroy(sqb200_batch* b) {
  if (!b) return SQB200_OK;
  cudaSetDevice(b->device);
  free_batch(b);
  return SQB200_OK;
}

extern "C" int sqb200_batch_offsets(sqb200_batch* b, long long* off) {
  if (!b || !off) return fail(SQB200_EINVAL, "null argument");
  for (int m = 0; m <= b->nmol; ++m) off[m] = b->moff[m];
  return SQB200_OK;
}

extern "C" int sqb200_batch_set_step(sqb200_batch* b, const int* restricted, const double* scf_cutoff,
                                     const double* fixed_cutoff, const double* dscreen_rmax) {
  if (!b || !restricted || !scf_cutoff || !fixed_cutoff || !dscreen_rmax) return fail(SQB200_EINVAL, "null argument");
  CUDA_OK(cudaSetDevice(b->device));
  // the work list depends on the spins and the two Schwarz cutoffs (and each context's FP32
  // threshold); the density-screen bound only reaches the kernels through the records
  bool same = b->have_step;
  for (int m = 0; m < b->nmol && same; ++m)
    same = b->rec[m].uhf == (restricted[m] ? 0 : 1) && b->rec[m].cut_outer == scf_cutoff[m] &&
           b->rec[m].cut_fixed == fixed_cutoff[m];
  for (int m = 0; m < b->nmol; ++m) {
    b->rec[m].uhf = restricted[m] ? 0 : 1;
    b->rec[m].cut_outer = scf_cutoff[m];
    b->rec[m].cut_fixed = fixed_cutoff[m];
    b->rec[m].dscreen_rmax = dscreen_rmax[m];
  }
  CUDA_OK(cudaStreamSynchronize(b->stream));
  for (cudaStream_t s : b->side) CUDA_OK(cudaStreamSynchronize(s));
  CUDA_OK(h2d(b->d_mols, b->rec.data(), b->nmol * sizeof(sqb::MolRec), b->stream));
  if (same) return SQB200_OK;
  b->kernel.clear(); b->spin.clear(); b->first.clear(); b->count.clear(); b->cost.clear();
  std::vector<sqb::WorkItem> items, items32;
  const int K_ = sqb::kNumClassKernels;
  for (int sp = 0; sp < 2; ++sp)
    for (int ki = 0; ki < K_; ++ki) {
      const sqb::ClassKernel& K = sqb::kClassKernels[ki];
      const int f64 = (int)items.size();
      items32.clear();
      double c64 = 0.0, c32 = 0.0;
      // heaviest first inside each molecule's run of items: sorting across molecules would
      // interleave their pair data and J/K blocks in L2 (measured 4% slower on 256 molecules)
      auto np = [&](const sqb::WorkItem& it) {
        const sqb200_jk* mc = b->mols[it.mol];
        return std::make_pair(mc->cls[K.bra_cls].pairs[it.bra - b->cls[K.bra_cls].pair_base[it.mol]].nprim,
                              mc->cls[K.ket_cls].pairs[it.k0 - b->cls[K.ket_cls].pair_base[it.mol]].nprim);
      };
      for (int m = 0; m < b->nmol; ++m) {
        if (b->rec[m].uhf != sp) continue;
        const size_t a64 = items.size(), a32 = items32.size();
        class_items(b->mols[m], ki, scf_cutoff[m], fixed_cutoff[m], b->cls[K.bra_cls].pair_base[m],
                    b->cls[K.ket_cls].pair_base[m], m, items, items32, c64, c32);
        sort_heavy_first(items, a64, np);
        sort_heavy_first(items32, a32, np);
      }
      if (too_few_f32(items32)) {
        items.resize(f64);
        items32.clear();
        c64 = c32 = 0.0;
        for (int m = 0; m < b->nmol; ++m) {
          if (b->rec[m].uhf != sp) continue;
          const size_t a64 = items.size();
          class_items(b->mols[m], ki, scf_cutoff[m], fixed_cutoff[m], b->cls[K.bra_cls].pair_base[m],
                      b->cls[K.ket_cls].pair_base[m], m, items, items32, c64, c32, nullptr, nullptr, false);
          sort_heavy_first(items, a64, np);
        }
      }
      if ((int)items.size() > f64) {
        b->kernel.push_back(ki); b->spin.push_back(sp); b->first.push_back(f64);
        b->count.push_back((int)items.size() - f64); b->cost.push_back(c64);
      }
      if (!items32.empty()) {
        b->kernel.push_back(ki + K_); b->spin.push_back(sp); b->first.push_back((int)items.size());
        b->count.push_back((int)items32.size()); b->cost.push_back(c32);
        items.insert(items.end(), items32.begin(), items32.end());
      }
    }
  for (int c : b->count)
    if (c > 2147483647 / 2) return fail(SQB200_EINVAL, "sqb200_batch_set_step: too many work items in one class");
  if (items.size() > b->items_cap) {
    cudaFree(b->d_items);
    b->d_items = nullptr;
    b->items_cap = 0;
    CUDA_OK(cudaMalloc(&b->d_items, items.size() * sizeof(sqb::WorkItem)));
    b->items_cap = items.size();
  }
  if (!items.empty())
    CUDA_OK(h2d(b->d_items, items.data(), items.size() * sizeof(sqb::WorkItem), b->stream));
  b->have_step = true;
  return SQB200_OK;
}

// Segment s of a batch's work list; form < 0 takes the batch's choice.
SegLaunch seg_batch(sqb200_batch* b, size_t s, const double* dPA, const double* dPB, int form) {
  SegLaunch L;
  const int K_ = sqb::kNumClassKernels;
  const int v = b->kernel[s], uhf = b->spin[s];
  const bool f32 = v >= K_;
  const int kidx = f32 ? v - K_ : v;
  const sqb::ClassKernel& K = sqb::kClassKernels[kidx];
  const auto& B = b->cls[K.bra_cls];
  const auto& T = b->cls[K.ket_cls];
  sqb::JKArgs& a = L.a;
  memset(&a, 0, sizeof(a));
  a.bra_pairs = B.d_pairs; a.bra_prims = B.d_prims;
  a.ket_pairs = T.d_pairs; a.ket_prims = T.d_prims;
  a.bra_prims_f = B.d_primsf; a.ket_prims_f = T.d_primsf;
  a.PA = dPA; a.PB = dPB; a.PT = b->d_PT; a.PM = b->d_PM;
  a.Jacc = b->d_J; a.KAacc = b->d_KA; a.KBacc = b->d_KB;
  a.boys_tab = b->mols[0]->d_boys;
  a.boys_tab_f = b->mols[0]->d_boysf;
  a.counters = b->d_counters + 4 * (uhf * 2 * K_ + v);
  a.mols = b->d_mols;
  a.same_class = K.bra_cls == K.ket_cls;
  L.items = b->d_items + b->first[s];
  L.smem = (size_t)B.max_nprim * B.stride * (f32 ? sizeof(float) : sizeof(double));
  int passes = 1;
  const int fu = pick_form(K, f32, uhf, form < 0 ? b->form[kidx] : form, &L.fn, &passes);
  L.grid = dim3(b->count[s], passes);
  L.block = dim3(cta_threads());
  add_acc_region(K, fu, L);
  if (b->persistent) make_persistent(L, b->d_queue + uhf * 2 * K_ + v);
  return L;
}

void batch_prologue(sqb200_batch* b, const double* dPA, const double* dPB, cudaStream_t st) {
  const long long ntot = b->moff[b->nmol];
  k_prep<<<grid_for(ntot, 256), 256, 0, st>>>(dPA, dPB, b->d_PT, b->d_J, b->d_KA, b->d_KB, (int)ntot, 1,
                                              nullptr, sqb::MolRec{});
  k_pmax_batch<<<dim3((b->max_ns * b->max_ns + 127) / 128, b->nmol), 128, 0, st>>>(
      dPA, dPB, b->d_PT, b->d_shfirst, b->d_shn, b->d_mols, b->d_PM);
}

extern "C" int sqb200_batch_set_persistent(sqb200_batch* b, int enable) {
  if (!b) return fail(SQB200_EINVAL, "null batch");
  b->persistent = enable != 0;
  return SQB200_OK;
}

extern "C" int sqb200_batch_autotune(sqb200_batch* b, const double* dPA, const double* dPB, void* stream) {
  if (!b || !dPA || !dPB) return fail(SQB200_EINVAL, "null argument");
  if (!b->have_step) return fail(SQB200_EINVAL, "sqb200_batch_autotune: call sqb200_batch_set_step first");
  CUDA_OK(cudaSetDevice(b->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
  batch_prologue(b, dPA, dPB, st);
  // a class with restricted and unrestricted segments keeps one choice: the summed time decides
  std::vector<double> tf(3 * sqb::kNumClassKernels, 0.0);
  for (size_t s = 0; s < b->kernel.size(); ++s) {
    const int v = b->kernel[s];
    if (v >= sqb::kNumClassKernels) continue;
    double ts[3] = {0.0, 0.0, 0.0};
    for (int round = 0; round < kTuneRounds; ++round) {
      for (int f = 0; f < 3; ++f) {
        if (!has_form(sqb::kClassKernels[v], f)) continue;
        double t = 0.0;
        const int rc = time_seg(seg_batch(b, s, dPA, dPB, f), st, 2, &t);
        if (rc) return rc;
        ts[f] = round == 0 ? t : std::min(ts[f], t);
      }
      if (ts[0] > kTuneLongMs) break;
    }
    for (int f = 0; f < 3; ++f) tf[3 * v + f] += ts[f];
  }
  for (int k = 0; k < sqb::kNumClassKernels; ++k) b->form[k] = (char)pick_tuned(sqb::kClassKernels[k], &tf[3 * k]);
  CUDA_OK(cudaStreamSynchronize(st));
  return SQB200_OK;
}

extern "C" int sqb200_batch_build_device(sqb200_batch* b, const double* dPA, const double* dPB, double* dJT,
                                         double* dKA, double* dKB, void* stream) {
  if (!b || !dPA || !dPB || !dJT || !dKA || !dKB) return fail(SQB200_EINVAL, "null argument");
  if (!b->have_step) return fail(SQB200_EINVAL, "sqb200_batch_build_device: call sqb200_batch_set_step first");
  CUDA_OK(cudaSetDevice(b->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
  const int K_ = sqb::kNumClassKernels;
  batch_prologue(b, dPA, dPB, st);
  CUDA_OK(cudaMemsetAsync(b->d_counters, 0, 2 * 8 * K_ * sizeof(unsigned long long), st));
  if (b->persistent) CUDA_OK(cudaMemsetAsync(b->d_queue, 0, 2 * 2 * K_ * sizeof(unsigned long long), st));
  if (b->nside < 0) {
    int n = 4;
    if (const char* e = getenv("SQB200_STREAMS")) n = std::max(0, std::min(16, atoi(e)));
    CUDA_OK(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
    for (int i = 0; i < n; ++i) {
      cudaStream_t s;
      cudaEvent_t e;
      CUDA_OK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      CUDA_OK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      b->side.push_back(s);
      b->ev_join.push_back(e);
    }
    b->nside = n;
  }
  const int nlanes = 1 + b->nside;
  std::vector<size_t> order(b->kernel.size());
  for (size_t s = 0; s < order.size(); ++s) order[s] = s;
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return b->cost[x] > b->cost[y]; });
  std::vector<double> load(nlanes, 0.0);
  if (nlanes > 1) {
    CUDA_OK(cudaEventRecord(b->ev_fork, st));
    for (int l = 1; l < nlanes; ++l) CUDA_OK(cudaStreamWaitEvent(b->side[l - 1], b->ev_fork, 0));
  }
  for (size_t s : order) {
    const int lane = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    load[lane] += b->cost[s];
    const cudaStream_t ls = lane == 0 ? st : b->side[lane - 1];
    const int rc = enqueue(seg_batch(b, s, dPA, dPB, -1), ls);
    if (rc) return rc;
  }
  for (int l = 1; l < nlanes; ++l) {
    CUDA_OK(cudaEventRecord(b->ev_join[l - 1], b->side[l - 1]));
    CUDA_OK(cudaStreamWaitEvent(st, b->ev_join[l - 1], 0));
  }
  k_finalize_batch<<<dim3((b->max_nbf * b->max_nbf + 255) / 256, b->nmol), 256, 0, st>>>(
      b->d_J, b->d_KA, b->d_KB, dJT, dKA, dKB, b->d_mols);
  CUDA_OK(cudaGetLastError());
  b->last_launches = 3 + (int)b->kernel.size();
  return SQB200_OK;
}

extern "C" int sqb200_batch_stats(sqb200_batch* b, long long* out, int n) {
  if (!b || !out) return fail(SQB200_EINVAL, "null argument");
  CUDA_OK(cudaSetDevice(b->device));
  CUDA_OK(cudaDeviceSynchronize());      // the build ran on the caller's stream
  const int K_ = sqb::kNumClassKernels;
  std::vector<unsigned long long> h(2 * 8 * K_);
  CUDA_OK(cudaMemcpy(h.data(), b->d_counters, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  long long q = 0, pq = 0;
  double fl = 0.0;
  for (int sp = 0; sp < 2; ++sp)
    for (int v = 0; v < 2 * K_; ++v) {
      const unsigned long long* c = &h[4 * (sp * 2 * K_ + v)];
      q += (long long)c[0];
      pq += (long long)c[1];
      fl += kernel_flops_form(v, v < K_ ? b->form[v] : 0, c);
    }
  long long pairs = 0, shells = 0;
  for (const sqb200_jk* c : b->mols) {
    shells += c->ns;
    for (int k = 0; k < sqb::kNumPairClasses; ++k) pairs += (long long)c->cls[k].pairs.size();
  }
  long long v[6] = {q, pq, (long long)fl, shells, pairs, (long long)b->last_launches};
  for (int i = 0; i < n && i < 6; ++i) out[i] = v[i];
  return SQB200_OK;
}

// ---------------------------------------------------------------- batched eigensolver
//
// The SCF tail's generalised eigenproblems, already reduced to standard form, for many
// molecules of one padded size at once: cusolverDnXsyevBatched (one call per stack).

namespace {
struct SyevCtx {
  cusolverDnHandle_t h = nullptr;
  cusolverDnParams_t p = nullptr;
  void* dwork = nullptr;
  size_t dbytes = 0;
  std::vector<char> hwork;
  int* dinfo = nullptr;
  long long ninfo = 0;
};
// one handle and workspace per (device, stream): calls on different streams may run on the
// GPU at the same time and must not share a workspace
std::mutex g_syev_mu;
std::map<std::pair<int, void*>, SyevCtx> g_syev;
}  // namespace

extern "C" int sqb200_syev_batched(int device, int n, int batch, double* A, double* W, void* stream) {
  if (n <= 0 || batch <= 0 || !A || !W) return fail(SQB200_EINVAL, "sqb200_syev_batched: bad argument");
  std::lock_guard<std::mutex> lock(g_syev_mu);
  CUDA_OK(cudaSetDevice(device));
  SyevCtx& c = g_syev[{device, stream}];
  if (!c.h) {
    if (cusolverDnCreate(&c.h) != CUSOLVER_STATUS_SUCCESS) return fail(SQB200_ECUDA, "cusolverDnCreate failed");
    if (cusolverDnCreateParams(&c.p) != CUSOLVER_STATUS_SUCCESS) return fail(SQB200_ECUDA, "cusolverDnCreateParams failed");
  }
  if (cusolverDnSetStream(c.h, (cudaStream_t)stream) != CUSOLVER_STATUS_SUCCESS)
    return fail(SQB200_ECUDA, "cusolverDnSetStream failed");
  size_t db = 0, hb = 0;
  if (cusolverDnXsyevBatched_bufferSize(c.h, c.p, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, CUDA_R_64F, A,
                                        n, CUDA_R_64F, W, CUDA_R_64F, &db, &hb, batch) != CUSOLVER_STATUS_SUCCESS)
    return fail(SQB200_ECUDA, "cusolverDnXsyevBatched_bufferSize failed");
  if (db > c.dbytes || batch > c.ninfo) {
    // the previous call on this stream may still run: wait before freeing its workspace
    CUDA_OK(cudaStreamSynchronize((cudaStream_t)stream));
    if (db > c.dbytes) {
      cudaFree(c.dwork);
      c.dwork = nullptr;
      c.dbytes = 0;
      CUDA_OK(cudaMalloc(&c.dwork, db));
      c.dbytes = db;
    }
    if (batch > c.ninfo) {
      cudaFree(c.dinfo);
      c.dinfo = nullptr;
      c.ninfo = 0;
      CUDA_OK(cudaMalloc(&c.dinfo, sizeof(int) * (size_t)batch));
      c.ninfo = batch;
    }
  }
  if (hb > c.hwork.size()) c.hwork.resize(hb);
  if (cusolverDnXsyevBatched(c.h, c.p, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, CUDA_R_64F, A, n,
                             CUDA_R_64F, W, CUDA_R_64F, c.dwork, c.dbytes, hb ? c.hwork.data() : nullptr, hb,
                             c.dinfo, batch) != CUSOLVER_STATUS_SUCCESS)
    return fail(SQB200_ECUDA, "cusolverDnXsyevBatched failed");
  CUDA_OK(cudaGetLastError());
  return SQB200_OK;
}

// ---------------------------------------------------------------- nuclear gradient
//
// Gradient of the SCF energy with respect to the nuclear positions, as uhf_force computes it
// (src/grad.c:2155-2420; the forces are its negative): nuclear repulsion, -sum W dS (W the
// energy-weighted density), sum PT d(T + V) including the Hellmann-Feynman term of each
// nucleus, and the two-electron term of GradEri_ShellSet_Parallel (src/grad.c:1734):
// sum over unique shell quartets of Gamma_abcd d(ab|cd), with
// Gamma = deg * [4 PT_ab PT_cd - (PT_ac PT_bd + PT_ad PT_bc + PS_ac PS_bd + PS_ad PS_bc)]
// (the reference's 0.5 PT PT - 0.25 (PT PT + PS PS) summed over the eight index permutations),
// shell quartets skipped when Sch(PQ) Sch(IJ) maxPT(PQ) maxPT(IJ) < 1e-10, primitive quartets
// below the 1e-15 prefactor cut, and, as the reference does, a function quartet of a primitive
// quartet whose density factor times prefactor and weights is below 1e-10 (both 1e-10 screens
// follow SQB200_GRAD_SCREEN when it is set).  Derivatives of a primitive by its centre raise and lower
// its angular momentum, d/dA_x g_a = 2 alpha g_{a+1x} - a_x g_{a-1x}; the fourth centre follows
// from translational invariance.  The integrals are McMurchie-Davidson with runtime loops (one
// thread per shell quartet or function pair): a correctness-first form, not tuned.

namespace {

constexpr int GR_NF = 10;   // functions of one shell the gradient kernels take (an f shell)

struct GShell {
  int first, nfunc, nprim, poff;   // poff: first primitive in the exps / wts arrays
  int lmax, atom;
  double x, y, z;
  int lmn[GR_NF][3];
};

// Array bounds of the gradient kernels for functions up to l = LG (2: d, 3: f): the highest
// Hermite order of a quartet with one index raised ((dd|dd) + 1 = 9, (ff|ff) + 1 = 13), its
// tetrahedral R table, the 1-D Hermite tables E^{ij}_t with i, j <= LG + 1 (the raised index)
// and t <= 2 LG + 2 (the one-electron tables raise j by two more for the kinetic term), and the
// bra-side intermediates V (t+u+v <= 2 LG + 1).
template <int LG>
struct GDim {
  static constexpr int MAXL = 4 * LG + 1;
  static constexpr int NT = (MAXL + 1) * (MAXL + 2) * (MAXL + 3) / 6;
  static constexpr int NI = LG + 2;
  static constexpr int NJ1 = LG + 3;
  static constexpr int NTT = 2 * LG + 4;
  static constexpr int NV = (2 * LG + 2) * (2 * LG + 3) * (2 * LG + 4) / 6;
  static constexpr int NE = 3 * NI * NI * NTT;   // doubles of one pair's three tables
};

// F_0..F_M (M <= 13, runtime) from a Boys table of ncol columns: the top order by the Taylor
// expansion with as many terms as the table's columns allow, then downward recursion.
__device__ void boys_rt(int M, double T, const double* __restrict__ tab, int ncol, double* F) {
  if (T < BOYS_TMAX) {
    const int g = __double2int_rn(T * BOYS_INV_H);
    const double d = T - g * BOYS_H;
    const double* row = tab + g * ncol + M;
    const int nt = min(BOYS_NTAY, ncol - M);
    double s = row[nt - 1];
    for (int k = nt - 2; k >= 0; --k) s = fma(s, -d * (1.0 / (double)(k + 1)), row[k]);
    F[M] = s;
    if (M > 0) {
      const double e = exp(-T);
      for (int m = M - 1; m >= 0; --m) F[m] = (2.0 * T * F[m + 1] + e) / (2 * m + 1);
    }
  } else {
    F[0] = 0.5 * sqrt(M_PI / T);
    const double e = exp(-T);
    for (int m = 0; m < M; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) / (2.0 * T);
  }
}

// 1-D Hermite expansion coefficients E^{ij}_t, i <= imax, j <= jmax (prefactor excluded)
template <int NI, int NJ, int NT>
__device__ void herm1d(double p, double xpa, double xpb, int imax, int jmax, double E[NI][NJ][NT]) {
  const double h = 0.5 / p;
  for (int i = 0; i <= imax; ++i)
    for (int j = 0; j <= jmax; ++j)
      for (int t = 0; t <= i + j; ++t) {
        double v;
        if (i == 0 && j == 0) v = (t == 0) ? 1.0 : 0.0;
        else if (i > 0) {
          // E^{i-1,j}_t vanishes for t > i-1+j: that entry was never written, read it as 0
          v = (t <= i - 1 + j) ? xpa * E[i - 1][j][t] : 0.0;
          if (t > 0) v += h * E[i - 1][j][t - 1];
          if (t + 1 <= i - 1 + j) v += (t + 1) * E[i - 1][j][t + 1];
        } else {
          v = (t <= i + j - 1) ? xpb * E[i][j - 1][t] : 0.0;
          if (t > 0) v += h * E[i][j - 1][t - 1];
          if (t + 1 <= i + j - 1) v += (t + 1) * E[i][j - 1][t + 1];
        }
        E[i][j][t] = v;
      }
}

// R_tuv (order 0) for t+u+v <= L into R (tetra index), from base[n] = (-2 a)^n F_n
template <int LG>
__device__ void herm_R(int L, double a, double X, double Y, double Z, const double* F, double* R, double* tmp) {
  double base[GDim<LG>::MAXL + 1];
  double w = 1.0;
  for (int n = 0; n <= L; ++n) { base[n] = w * F[n]; w *= -2.0 * a; }
  double* cur = (L % 2 == 0) ? R : tmp;
  double* nxt = (L % 2 == 0) ? tmp : R;
  cur[0] = base[L];
  for (int n = L - 1; n >= 0; --n) {
    for (int N = 0; N <= L - n; ++N)
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
    double* s = cur; cur = nxt; nxt = s;
  }
}

// d/dA of a 1-D factor: 2 alpha f(i+1) - i f(i-1)
__device__ __forceinline__ double draise(double two_alpha, int i, double up, double down) {
  return two_alpha * up - (i > 0 ? i * down : 0.0);
}

template <int LG>
__device__ __noinline__ void grad_quartet(int pq, int ij, int ka, int kb, const double* __restrict__ sEb,
                                          const int2* __restrict__ pairs, const GShell* __restrict__ shells,
                                          const double* __restrict__ exps, const double* __restrict__ wts,
                                          const double* __restrict__ PT, const double* __restrict__ PS, int nbf,
                                          const double* __restrict__ tab, int ncol, double screen, double* gq);

// Two-electron part of the gradient: one block per (bra pair, 128 ket pairs), one thread per
// unique shell quartet (ket pair index <= bra pair index).
template <int LG>
__global__ void k_grad_eri(int npairs, const int2* __restrict__ pairs, const double* __restrict__ psch,
                           const double* __restrict__ ppm, const GShell* __restrict__ shells,
                           const double* __restrict__ exps, const double* __restrict__ wts,
                           const double* __restrict__ PT, const double* __restrict__ PS, int nbf,
                           const double* __restrict__ tab, int ncol, double screen, int natom,
                           double* __restrict__ grad) {
  using GD = GDim<LG>;
  // the block's contributions are summed per atom in shared memory first, then added to grad
  // with one atomic per touched component (grad has only 3 natom entries: atomics of every
  // thread straight into it collide)
  // The bra pair is the block's: the 1-D Hermite tables of its current primitive pair (with one
  // order more for the derivative) are built once per block in shared memory, by three threads
  // (one per axis), and read by every thread (the same entries across a warp: broadcasts).
  extern __shared__ double sgrad[];
  double* sEb = sgrad + 3 * natom;                 // [3][NI][NI][NTT]
  const int pq = blockIdx.y;
  if (pq >= npairs || (int)(blockIdx.x * blockDim.x) > pq) return;      // whole block: no quartet
  for (int x = threadIdx.x; x < 3 * natom; x += blockDim.x) sgrad[x] = 0.0;
  const int ij = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = ij <= pq && !(psch[pq] * psch[ij] * ppm[pq] * ppm[ij] < screen);
  const int2 PQ = pairs[pq];
  const GShell A = shells[PQ.x], B = shells[PQ.y];
  double gq[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};      // d/dA, d/dB, d/dC (x, y, z each)
  const bool any = __syncthreads_or(live);
  for (int ka = 0; any && ka < A.nprim; ++ka)
    for (int kb = 0; kb < B.nprim; ++kb) {
      __syncthreads();                             // the previous primitive pair's readers are done
      if (threadIdx.x < 3) {
        const int d = threadIdx.x;
        const double ea = exps[A.poff + ka], eb = exps[B.poff + kb], p = ea + eb;
        const double Ad = d == 0 ? A.x : d == 1 ? A.y : A.z, Bd = d == 0 ? B.x : d == 1 ? B.y : B.z;
        const double Pd = (ea * Ad + eb * Bd) / p;
        herm1d<GD::NI, GD::NI, GD::NTT>(p, Pd - Ad, Pd - Bd, A.lmax + 1, B.lmax + 1,
                                     reinterpret_cast<double (*)[GD::NI][GD::NTT]>(sEb + GD::NE / 3 * d));
      }
      __syncthreads();
      if (live) grad_quartet<LG>(pq, ij, ka, kb, sEb, pairs, shells, exps, wts, PT, PS, nbf, tab, ncol, screen, gq);
    }
  if (live) {
    const int2 IJ = pairs[ij];
    const int ac = shells[IJ.x].atom, ad = shells[IJ.y].atom;
    for (int x = 0; x < 3; ++x) {
      atomicAdd(sgrad + 3 * A.atom + x, gq[x]);
      atomicAdd(sgrad + 3 * B.atom + x, gq[3 + x]);
      atomicAdd(sgrad + 3 * ac + x, gq[6 + x]);
      atomicAdd(sgrad + 3 * ad + x, -(gq[x] + gq[3 + x] + gq[6 + x]));
    }
  }
  if (__syncthreads_or(live))
    for (int x = threadIdx.x; x < 3 * natom; x += blockDim.x) {
      const double v = sgrad[x];
      if (v != 0.0) atomicAdd(grad + x, v);
    }
}

// Bra primitive pair (ka, kb) of one shell quartet (pairs[pq] | pairs[ij]) of k_grad_eri, its
// contributions added to gq (d/dA, d/dB, d/dC); sEb holds the bra pair's Hermite tables.
template <int LG>
__device__ __noinline__ void grad_quartet(int pq, int ij, int ka, int kb, const double* __restrict__ sEb,
                                          const int2* __restrict__ pairs, const GShell* __restrict__ shells,
                                          const double* __restrict__ exps, const double* __restrict__ wts,
                                          const double* __restrict__ PT, const double* __restrict__ PS, int nbf,
                                          const double* __restrict__ tab, int ncol, double screen, double* gq) {
  using GD = GDim<LG>;
  const int2 PQ = pairs[pq], IJ = pairs[ij];
  const GShell A = shells[PQ.x], B = shells[PQ.y], C = shells[IJ.x], D = shells[IJ.y];
  const double deg = (PQ.x == PQ.y ? 0.5 : 1.0) * (IJ.x == IJ.y ? 0.5 : 1.0) * (pq == ij ? 0.5 : 1.0);
  const int Lb = A.lmax + B.lmax + 1, L = A.lmax + B.lmax + C.lmax + D.lmax + 1;
  double g[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  const double (*Eb)[GD::NI][GD::NI][GD::NTT] = reinterpret_cast<const double (*)[GD::NI][GD::NI][GD::NTT]>(sEb);
  double Ek[3][GD::NI][GD::NI][GD::NTT];
  double F[GD::MAXL + 1], R[GD::NT], tmp[GD::NT], V[4][GD::NV];
  const double ab2 = (A.x - B.x) * (A.x - B.x) + (A.y - B.y) * (A.y - B.y) + (A.z - B.z) * (A.z - B.z);
  const double cd2 = (C.x - D.x) * (C.x - D.x) + (C.y - D.y) * (C.y - D.y) + (C.z - D.z) * (C.z - D.z);
  {
      const double ea = exps[A.poff + ka], eb = exps[B.poff + kb], p = ea + eb;
      const double Px = (ea * A.x + eb * B.x) / p, Py = (ea * A.y + eb * B.y) / p, Pz = (ea * A.z + eb * B.z) / p;
      const double Kab = exp(-ea * eb / p * ab2);
      for (int kc = 0; kc < C.nprim; ++kc)
        for (int kd = 0; kd < D.nprim; ++kd) {
          const double ec = exps[C.poff + kc], ed = exps[D.poff + kd], q = ec + ed;
          const double Kcd = exp(-ec * ed / q * cd2);
          const double pre = TWO_PI_2_5 * Kab * Kcd / (p * q * sqrt(p + q));
          if (pre < PRIM_CUTOFF) continue;
          const double Qx = (ec * C.x + ed * D.x) / q, Qy = (ec * C.y + ed * D.y) / q, Qz = (ec * C.z + ed * D.z) / q;
          herm1d<GD::NI, GD::NI, GD::NTT>(q, Qx - C.x, Qx - D.x, C.lmax + 1, D.lmax, Ek[0]);
          herm1d<GD::NI, GD::NI, GD::NTT>(q, Qy - C.y, Qy - D.y, C.lmax + 1, D.lmax, Ek[1]);
          herm1d<GD::NI, GD::NI, GD::NTT>(q, Qz - C.z, Qz - D.z, C.lmax + 1, D.lmax, Ek[2]);
          const double al = p * q / (p + q);
          const double X = Px - Qx, Y = Py - Qy, Z = Pz - Qz;
          boys_rt(L, al * (X * X + Y * Y + Z * Z), tab, ncol, F);
          herm_R<LG>(L, al, X, Y, Z, F, R, tmp);
          for (int c = 0; c < C.nfunc; ++c)
            for (int d = 0; d < D.nfunc; ++d) {
              const int* lc = C.lmn[c];
              const int* ld = D.lmn[d];
              const double wcd = wts[(C.poff + kc) * GR_NF + c] * wts[(D.poff + kd) * GR_NF + d];
              if (wcd == 0.0) continue;
              // V0 = sum_k (-1)^k E^cd_k R_{h+k}; V1..3 the same with d/dC_{x,y,z} E^cd
              for (int N = 0; N <= Lb; ++N)
                for (int t = N; t >= 0; --t)
                  for (int u = N - t; u >= 0; --u) {
                    const int v = N - t - u, hi = tetra(t, u, v);
                    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
                    for (int tt = 0; tt <= lc[0] + 1 + ld[0]; ++tt)
                      for (int uu = 0; uu <= lc[1] + 1 + ld[1]; ++uu)
                        for (int vv = 0; vv <= lc[2] + 1 + ld[2]; ++vv) {
                          // R is computed up to order L; the terms beyond it pair a raised bra
                          // index with a raised ket index, which no derivative uses
                          if (N + tt + uu + vv > L) continue;
                          const double r = ((tt + uu + vv) & 1 ? -1.0 : 1.0) * R[tetra(t + tt, u + uu, v + vv)];
                          const bool bx = tt <= lc[0] + ld[0], by = uu <= lc[1] + ld[1], bz = vv <= lc[2] + ld[2];
                          const double ex = bx ? Ek[0][lc[0]][ld[0]][tt] : 0.0;
                          const double ey = by ? Ek[1][lc[1]][ld[1]][uu] : 0.0;
                          const double ez = bz ? Ek[2][lc[2]][ld[2]][vv] : 0.0;
                          const double dx = draise(2 * ec, lc[0], Ek[0][lc[0] + 1][ld[0]][tt],
                                                   lc[0] > 0 && tt <= lc[0] - 1 + ld[0] ? Ek[0][lc[0] - 1][ld[0]][tt] : 0.0);
                          const double dy = draise(2 * ec, lc[1], Ek[1][lc[1] + 1][ld[1]][uu],
                                                   lc[1] > 0 && uu <= lc[1] - 1 + ld[1] ? Ek[1][lc[1] - 1][ld[1]][uu] : 0.0);
                          const double dz = draise(2 * ec, lc[2], Ek[2][lc[2] + 1][ld[2]][vv],
                                                   lc[2] > 0 && vv <= lc[2] - 1 + ld[2] ? Ek[2][lc[2] - 1][ld[2]][vv] : 0.0);
                          s0 += ex * ey * ez * r;
                          s1 += dx * ey * ez * r;
                          s2 += ex * dy * ez * r;
                          s3 += ex * ey * dz * r;
                        }
                    V[0][hi] = s0; V[1][hi] = s1; V[2][hi] = s2; V[3][hi] = s3;
                  }
              const int fc = C.first + c, fd = D.first + d;
              for (int a = 0; a < A.nfunc; ++a)
                for (int b = 0; b < B.nfunc; ++b) {
                  const int fa = A.first + a, fb = B.first + b;
                  const double gam = 4.0 * PT[fa * nbf + fb] * PT[fc * nbf + fd] -
                                     (PT[fa * nbf + fc] * PT[fb * nbf + fd] + PT[fa * nbf + fd] * PT[fb * nbf + fc] +
                                      PS[fa * nbf + fc] * PS[fb * nbf + fd] + PS[fa * nbf + fd] * PS[fb * nbf + fc]);
                  const double wab = wts[(A.poff + ka) * GR_NF + a] * wts[(B.poff + kb) * GR_NF + b];
                  // the reference's per-primitive screen of one function quartet
                  // (src/grad.c:1982-1988): |coef r| < 1e-10, coef its density factor with the
                  // function-level degeneracy, r the primitive prefactor times the four weights
                  const double dfn = (fa == fb ? 0.5 : 1.0) * (fc == fd ? 0.5 : 1.0) *
                                     ((fa == fc && fb == fd) || (fa == fd && fb == fc) ? 0.5 : 1.0);
                  if (fabs(gam * dfn * pre * wab * wcd) < screen) continue;
                  const double G = deg * pre * wcd * wab * gam;
                  if (G == 0.0) continue;
                  const int* la = A.lmn[a];
                  const int* lb = B.lmn[b];
                  double dA[3] = {0, 0, 0}, dB[3] = {0, 0, 0}, dC[3] = {0, 0, 0};
                  for (int t = 0; t <= la[0] + lb[0] + 1; ++t)
                    for (int u = 0; u <= la[1] + lb[1] + 1; ++u)
                      for (int v = 0; v <= la[2] + lb[2] + 1; ++v) {
                        if (t + u + v > Lb) continue;
                        const int hi = tetra(t, u, v);
                        const bool bx = t <= la[0] + lb[0], by = u <= la[1] + lb[1], bz = v <= la[2] + lb[2];
                        const double ex = bx ? Eb[0][la[0]][lb[0]][t] : 0.0;
                        const double ey = by ? Eb[1][la[1]][lb[1]][u] : 0.0;
                        const double ez = bz ? Eb[2][la[2]][lb[2]][v] : 0.0;
                        const double ax = draise(2 * ea, la[0], Eb[0][la[0] + 1][lb[0]][t],
                                                 la[0] > 0 && t <= la[0] - 1 + lb[0] ? Eb[0][la[0] - 1][lb[0]][t] : 0.0);
                        const double ay = draise(2 * ea, la[1], Eb[1][la[1] + 1][lb[1]][u],
                                                 la[1] > 0 && u <= la[1] - 1 + lb[1] ? Eb[1][la[1] - 1][lb[1]][u] : 0.0);
                        const double az = draise(2 * ea, la[2], Eb[2][la[2] + 1][lb[2]][v],
                                                 la[2] > 0 && v <= la[2] - 1 + lb[2] ? Eb[2][la[2] - 1][lb[2]][v] : 0.0);
                        const double bxd = draise(2 * eb, lb[0], Eb[0][la[0]][lb[0] + 1][t],
                                                  lb[0] > 0 && t <= la[0] + lb[0] - 1 ? Eb[0][la[0]][lb[0] - 1][t] : 0.0);
                        const double byd = draise(2 * eb, lb[1], Eb[1][la[1]][lb[1] + 1][u],
                                                  lb[1] > 0 && u <= la[1] + lb[1] - 1 ? Eb[1][la[1]][lb[1] - 1][u] : 0.0);
                        const double bzd = draise(2 * eb, lb[2], Eb[2][la[2]][lb[2] + 1][v],
                                                  lb[2] > 0 && v <= la[2] + lb[2] - 1 ? Eb[2][la[2]][lb[2] - 1][v] : 0.0);
                        const double v0 = V[0][hi];
                        dA[0] += ax * ey * ez * v0;
                        dA[1] += ex * ay * ez * v0;
                        dA[2] += ex * ey * az * v0;
                        dB[0] += bxd * ey * ez * v0;
                        dB[1] += ex * byd * ez * v0;
                        dB[2] += ex * ey * bzd * v0;
                        const double e3 = ex * ey * ez;
                        dC[0] += e3 * V[1][hi];
                        dC[1] += e3 * V[2][hi];
                        dC[2] += e3 * V[3][hi];
                      }
                  for (int x = 0; x < 3; ++x) {
                    g[0][x] += G * dA[x];
                    g[1][x] += G * dB[x];
                    g[2][x] += G * dC[x];
                  }
                }
            }
        }
    }
  for (int x = 0; x < 3; ++x) {
    gq[x] += g[0][x];
    gq[3 + x] += g[1][x];
    gq[6 + x] += g[2][x];
  }
}

}  // namespace

namespace {

// One-electron part of the gradient, one thread per ordered function pair (a, b):
// -W_ab dS_ab, PT_ab d(T_ab + V_ab) on the atoms of a and b, and the Hellmann-Feynman term
// PT_ab dV^C_ab / dC = -PT_ab (dV^C/dA + dV^C/dB) on every nucleus C.
template <int LG>
__global__ void k_grad_1e(int nbf, const int* __restrict__ nprim, const int* __restrict__ off,
                          const int* __restrict__ lmn, const double* __restrict__ xyz,
                          const double* __restrict__ exps, const double* __restrict__ nc,
                          const int* __restrict__ fatom, int natom, const double* __restrict__ Z,
                          const double* __restrict__ axyz, const double* __restrict__ tab, int ncol,
                          const double* __restrict__ PT, const double* __restrict__ W, double* __restrict__ grad,
                          int terms) {
  using GD = GDim<LG>;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nbf * nbf) return;
  const int ia = idx / nbf, ib = idx % nbf;
  const double pt = (terms & SQB200_GRAD_HCORE) ? PT[idx] : 0.0;
  const double w = (terms & SQB200_GRAD_OVERLAP) ? W[idx] : 0.0;
  if (pt == 0.0 && w == 0.0) return;
  const int* la = lmn + 3 * ia;
  const int* lb = lmn + 3 * ib;
  const double* A = xyz + 3 * ia;
  const double* B = xyz + 3 * ib;
  double E[3][GD::NI][GD::NJ1][GD::NTT];
  double F[GD::MAXL + 1], R[GD::NT], tmp[GD::NT];
  double gA[3] = {0, 0, 0};      // d/dA of PT (T + V) - W S (the B side is added by translational invariance)
  double gB[3] = {0, 0, 0};      // d/dB of PT V (kinetic and overlap: -d/dA)
  const double ab2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]);
  const int L = la[0] + la[1] + la[2] + lb[0] + lb[1] + lb[2] + 1;
  for (int i = 0; i < nprim[ia]; ++i)
    for (int j = 0; j < nprim[ib]; ++j) {
      const double a = exps[off[ia] + i], b = exps[off[ib] + j], p = a + b;
      const double c = nc[off[ia] + i] * nc[off[ib] + j] * exp(-a * b * ab2 / p);
      const double P[3] = {(a * A[0] + b * B[0]) / p, (a * A[1] + b * B[1]) / p, (a * A[2] + b * B[2]) / p};
      for (int d = 0; d < 3; ++d) herm1d<GD::NI, GD::NJ1, GD::NTT>(p, P[d] - A[d], P[d] - B[d], la[d] + 1, lb[d] + 2, E[d]);
      const double sq = sqrt(M_PI / p);
      // 1-D overlap S(i,j) and kinetic T(i,j) factors and their d/dA
      double S0[3], T0[3], dS[3], dT[3];
      for (int d = 0; d < 3; ++d) {
        const int ii = la[d], jj = lb[d];
        auto Sf = [&](int i2, int j2) { return (i2 < 0 || j2 < 0) ? 0.0 : E[d][i2][j2][0] * sq; };
        auto Tf = [&](int i2, int j2) {
          if (i2 < 0) return 0.0;
          double k = -2.0 * b * (2 * j2 + 1) * Sf(i2, j2) + 4.0 * b * b * Sf(i2, j2 + 2);
          if (j2 >= 2) k += j2 * (j2 - 1) * Sf(i2, j2 - 2);
          return -0.5 * k;
        };
        S0[d] = Sf(ii, jj);
        T0[d] = Tf(ii, jj);
        dS[d] = draise(2 * a, ii, Sf(ii + 1, jj), Sf(ii - 1, jj));
        dT[d] = draise(2 * a, ii, Tf(ii + 1, jj), Tf(ii - 1, jj));
      }
      for (int x = 0; x < 3; ++x) {
        const int y = (x + 1) % 3, z = (x + 2) % 3;
        const double dSab = dS[x] * S0[y] * S0[z];
        const double dTab = dT[x] * S0[y] * S0[z] + dS[x] * (T0[y] * S0[z] + S0[y] * T0[z]);
        gA[x] += c * (pt * dTab - w * dSab);
        gB[x] -= c * (pt * dTab - w * dSab);
      }
      // nuclear attraction: V^C = -Z_C (2 pi / p) sum_tuv E^ab_tuv R_tuv(p, P - C)
      for (int at = 0; at < natom; ++at) {
        const double X = P[0] - axyz[3 * at], Y = P[1] - axyz[3 * at + 1], Zc = P[2] - axyz[3 * at + 2];
        boys_rt(L, p * (X * X + Y * Y + Zc * Zc), tab, ncol, F);
        herm_R<LG>(L, p, X, Y, Zc, F, R, tmp);
        const double f = -Z[at] * (2.0 * M_PI / p) * c * pt;
        double vA[3] = {0, 0, 0}, vB[3] = {0, 0, 0};
        for (int t = 0; t <= la[0] + lb[0] + 1; ++t)
          for (int u = 0; u <= la[1] + lb[1] + 1; ++u)
            for (int v = 0; v <= la[2] + lb[2] + 1; ++v) {
              if (t + u + v > L) continue;
              const double r = R[tetra(t, u, v)];
              const double ex = t <= la[0] + lb[0] ? E[0][la[0]][lb[0]][t] : 0.0;
              const double ey = u <= la[1] + lb[1] ? E[1][la[1]][lb[1]][u] : 0.0;
              const double ez = v <= la[2] + lb[2] ? E[2][la[2]][lb[2]][v] : 0.0;
              const double ax = draise(2 * a, la[0], E[0][la[0] + 1][lb[0]][t], la[0] > 0 && t <= la[0] - 1 + lb[0] ? E[0][la[0] - 1][lb[0]][t] : 0.0);
              const double ay = draise(2 * a, la[1], E[1][la[1] + 1][lb[1]][u], la[1] > 0 && u <= la[1] - 1 + lb[1] ? E[1][la[1] - 1][lb[1]][u] : 0.0);
              const double az = draise(2 * a, la[2], E[2][la[2] + 1][lb[2]][v], la[2] > 0 && v <= la[2] - 1 + lb[2] ? E[2][la[2] - 1][lb[2]][v] : 0.0);
              const double bx = draise(2 * b, lb[0], E[0][la[0]][lb[0] + 1][t], lb[0] > 0 && t <= la[0] + lb[0] - 1 ? E[0][la[0]][lb[0] - 1][t] : 0.0);
              const double by = draise(2 * b, lb[1], E[1][la[1]][lb[1] + 1][u], lb[1] > 0 && u <= la[1] + lb[1] - 1 ? E[1][la[1]][lb[1] - 1][u] : 0.0);
              const double bz = draise(2 * b, lb[2], E[2][la[2]][lb[2] + 1][v], lb[2] > 0 && v <= la[2] + lb[2] - 1 ? E[2][la[2]][lb[2] - 1][v] : 0.0);
              vA[0] += ax * ey * ez * r; vA[1] += ex * ay * ez * r; vA[2] += ex * ey * az * r;
              vB[0] += bx * ey * ez * r; vB[1] += ex * by * ez * r; vB[2] += ex * ey * bz * r;
            }
        for (int x = 0; x < 3; ++x) {
          gA[x] += f * vA[x];
          gB[x] += f * vB[x];
          atomicAdd(grad + 3 * at + x, -f * (vA[x] + vB[x]));
        }
      }
    }
  for (int x = 0; x < 3; ++x) {
    atomicAdd(grad + 3 * fatom[ia] + x, gA[x]);
    atomicAdd(grad + 3 * fatom[ib] + x, gB[x]);
  }
}

}  // namespace

extern "C" int sqb200_gradient_terms(sqb200_jk* c, int natom, const double* Z, const double* axyz,
                                     const double* PA, const double* PB, const double* W, int terms, double* grad) {
  if (!c || natom <= 0 || !Z || !axyz || !PA || !PB || !W || !grad) return fail(SQB200_EINVAL, "null argument");
  CUDA_OK(cudaSetDevice(c->device));
  const int n = c->nbf;
  const size_t nn = (size_t)n * n;
  // functions: primitive data, atom (the centre the basis function sits on)
  std::vector<int> np(n), off(n), lmn(3 * n), fat(n, -1);
  std::vector<double> xyz(3 * n), ex, nc;
  for (const Shell& sh : c->shells)
    for (int f = 0; f < sh.nfunc; ++f) {
      const int q = sh.first + f;
      np[q] = sh.nprim;
      off[q] = (int)ex.size();
      for (int d = 0; d < 3; ++d) lmn[3 * q + d] = sh.lmn[f][d];
      xyz[3 * q] = sh.x; xyz[3 * q + 1] = sh.y; xyz[3 * q + 2] = sh.z;
      for (int k = 0; k < sh.nprim; ++k) { ex.push_back(sh.exps[k]); nc.push_back(sh.coef[k][f]); }
    }
  auto atom_of = [&](double x, double y, double z) {
    for (int a = 0; a < natom; ++a)
      if (fabs(axyz[3 * a] - x) < 1e-8 && fabs(axyz[3 * a + 1] - y) < 1e-8 && fabs(axyz[3 * a + 2] - z) < 1e-8) return a;
    return -1;
  };
  for (int q = 0; q < n; ++q) {
    fat[q] = atom_of(xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2]);
    if (fat[q] < 0) return fail(SQB200_EINVAL, "sqb200_gradient: a basis function is not centred on an atom");
  }
  // shells, shell-major primitive weights (6 functions per primitive row)
  const int ns = (int)c->shells.size();
  std::vector<GShell> gs(ns);
  std::vector<double> sex, swt;
  int lmax_all = 0;
  for (int s = 0; s < ns; ++s) {
    const Shell& sh = c->shells[s];
    GShell& g = gs[s];
    g.first = sh.first; g.nfunc = sh.nfunc; g.nprim = sh.nprim; g.poff = (int)sex.size();
    g.lmax = 0;
    if (sh.nfunc > GR_NF)
      return fail(SQB200_EUNSUPPORTED, "sqb200_gradient: a shell of more than " + std::to_string(GR_NF) + " functions");
    for (int f = 0; f < sh.nfunc; ++f) {
      for (int d = 0; d < 3; ++d) g.lmn[f][d] = sh.lmn[f][d];
      g.lmax = std::max(g.lmax, sh.lmn[f][0] + sh.lmn[f][1] + sh.lmn[f][2]);
    }
    lmax_all = std::max(lmax_all, g.lmax);
    g.atom = fat[sh.first]; g.x = sh.x; g.y = sh.y; g.z = sh.z;
    for (int k = 0; k < sh.nprim; ++k) {
      sex.push_back(sh.exps[k]);
      for (int f = 0; f < GR_NF; ++f) swt.push_back(f < sh.nfunc ? sh.coef[k][f] : 0.0);
    }
  }
  // shell pairs P >= Q with their Schwarz and |PT| block maxima
  std::vector<int2> pairs;
  std::vector<double> psch, ppm;
  for (int P = 0; P < ns; ++P)
    for (int Q = 0; Q <= P; ++Q) {
      double sm = 0.0, pm = 0.0;
      for (int p = 0; p < c->shells[P].nfunc; ++p)
        for (int q = 0; q < c->shells[Q].nfunc; ++q) {
          const size_t e = (size_t)(c->shells[P].first + p) * n + c->shells[Q].first + q;
          sm = std::max(sm, c->schwarz[e]);
          pm = std::max(pm, fabs(PA[e] + PB[e]));
        }
      // the larger shell first ((ab|cd) = (ba|cd); the kernel's result does not depend on it)
      const Shell &SP = c->shells[P], &SQ = c->shells[Q];
      const bool swap = std::make_pair(SQ.nfunc, SQ.nprim) > std::make_pair(SP.nfunc, SP.nprim);
      pairs.push_back(swap ? make_int2(Q, P) : make_int2(P, Q));
      psch.push_back(sm);
      ppm.push_back(pm);
    }
  // Pairs grouped by shell types and contraction lengths: a thread takes one (bra pair, ket
  // pair <= bra pair) combination, so neighbouring lanes then run the same loops; inside a group
  // the largest Schwarz x density bound first, so that the quartets that pass the screen sit
  // together and whole warps leave together.  Any order of the list gives every unique quartet
  // once.
  {
    std::vector<int> ord(pairs.size());
    for (size_t k = 0; k < ord.size(); ++k) ord[k] = (int)k;
    auto key = [&](int k) {
      const Shell &X = c->shells[pairs[k].x], &Y = c->shells[pairs[k].y];
      return std::make_tuple(X.nfunc, Y.nfunc, X.nprim, Y.nprim, -(psch[k] * ppm[k]));
    };
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return key(a) < key(b); });
    std::vector<int2> p2(pairs.size());
    std::vector<double> s2(pairs.size()), m2(pairs.size());
    for (size_t k = 0; k < ord.size(); ++k) { p2[k] = pairs[ord[k]]; s2[k] = psch[ord[k]]; m2[k] = ppm[ord[k]]; }
    pairs.swap(p2); psch.swap(s2); ppm.swap(m2);
  }
  const int npairs = (int)pairs.size();
  if (npairs > 65535) return fail(SQB200_EINVAL, "sqb200_gradient: more than 65535 shell pairs");
  // kernels sized for d (LG = 2) or f (LG = 3) functions; the f forms read the generic path's
  // Boys table, whose 22 columns give orders to 13 their full Taylor expansion
  if (lmax_all > 3) return fail(SQB200_EUNSUPPORTED, "sqb200_gradient: functions above f");
  const bool fgrad = lmax_all > 2;
  if (fgrad && !c->gen.d_boys) return fail(SQB200_EINVAL, "sqb200_gradient: no Boys table for f functions");
  const double* btab = fgrad ? c->gen.d_boys : c->d_boys;
  const int bcol = fgrad ? sqb::kGenBoysCols : BOYS_NCOL;
  const size_t smem_eri = (3 * (size_t)natom + (fgrad ? GDim<3>::NE : GDim<2>::NE)) * sizeof(double);
  // the two-electron screens (shell quartet, function quartet of a primitive quartet): the
  // reference's 1e-10 unless SQB200_GRAD_SCREEN sets another (0 keeps every quartet)
  double screen = 1e-10;
  if (const char* ev = getenv("SQB200_GRAD_SCREEN")) screen = atof(ev);
  if (smem_eri > 48 * 1024)   // k_grad_eri: atom sums + the bra pair's tables
    return fail(SQB200_EINVAL, "sqb200_gradient: too many atoms (" + std::to_string(natom) + ") for the per-block sums");
  std::vector<double> PT(nn), PS(nn);
  for (size_t i = 0; i < nn; ++i) { PT[i] = PA[i] + PB[i]; PS[i] = PA[i] - PB[i]; }
  void* d[16] = {nullptr};
  void *dp = nullptr, *dsch = nullptr, *dpm = nullptr, *dg = nullptr;
  Staged up;
  up.put(&d[0], n * sizeof(int), np.data());
  up.put(&d[1], n * sizeof(int), off.data());
  up.put(&d[2], 3 * n * sizeof(int), lmn.data());
  up.put(&d[3], 3 * n * sizeof(double), xyz.data());
  up.put(&d[4], ex.size() * sizeof(double), ex.data());
  up.put(&d[5], nc.size() * sizeof(double), nc.data());
  up.put(&d[6], n * sizeof(int), fat.data());
  up.put(&d[7], natom * sizeof(double), Z);
  up.put(&d[8], 3 * natom * sizeof(double), axyz);
  up.put(&d[9], nn * sizeof(double), PT.data());
  up.put(&d[10], nn * sizeof(double), PS.data());
  up.put(&d[11], nn * sizeof(double), W);
  up.put(&d[12], ns * sizeof(GShell), gs.data());
  up.put(&d[13], sex.size() * sizeof(double), sex.data());
  up.put(&d[14], swt.size() * sizeof(double), swt.data());
  up.put(&dp, npairs * sizeof(int2), pairs.data());
  up.put(&dsch, npairs * sizeof(double), psch.data());
  up.put(&dpm, npairs * sizeof(double), ppm.data());
  up.put(&dg, 3 * natom * sizeof(double), nullptr);
  void* base = nullptr;
  cudaError_t e = up.upload(&base, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(dg, 0, 3 * natom * sizeof(double), c->stream);
  if (e == cudaSuccess) {
    const dim3 geri((npairs + 127) / 128, npairs);
    if ((terms & SQB200_GRAD_ERI) && fgrad)
      k_grad_eri<3><<<geri, 128, smem_eri, c->stream>>>(
          npairs, (const int2*)dp, (const double*)dsch, (const double*)dpm, (const GShell*)d[12], (const double*)d[13],
          (const double*)d[14], (const double*)d[9], (const double*)d[10], n, btab, bcol, screen, natom, (double*)dg);
    else if (terms & SQB200_GRAD_ERI)
      k_grad_eri<2><<<geri, 128, smem_eri, c->stream>>>(
          npairs, (const int2*)dp, (const double*)dsch, (const double*)dpm, (const GShell*)d[12], (const double*)d[13],
          (const double*)d[14], (const double*)d[9], (const double*)d[10], n, btab, bcol, screen, natom, (double*)dg);
    const int g1 = (int)((nn + 127) / 128);
    if ((terms & (SQB200_GRAD_HCORE | SQB200_GRAD_OVERLAP)) && fgrad)
      k_grad_1e<3><<<g1, 128, 0, c->stream>>>(
          n, (const int*)d[0], (const int*)d[1], (const int*)d[2], (const double*)d[3], (const double*)d[4],
          (const double*)d[5], (const int*)d[6], natom, (const double*)d[7], (const double*)d[8], btab, bcol,
          (const double*)d[9], (const double*)d[11], (double*)dg, terms);
    else if (terms & (SQB200_GRAD_HCORE | SQB200_GRAD_OVERLAP))
      k_grad_1e<2><<<g1, 128, 0, c->stream>>>(
          n, (const int*)d[0], (const int*)d[1], (const int*)d[2], (const double*)d[3], (const double*)d[4],
          (const double*)d[5], (const int*)d[6], natom, (const double*)d[7], (const double*)d[8], btab, bcol,
          (const double*)d[9], (const double*)d[11], (double*)dg, terms);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(grad, dg, 3 * natom * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(base);
  if (e != cudaSuccess) return fail(SQB200_ECUDA, std::string("sqb200_gradient: ") + cudaGetErrorString(e));
  // nuclear repulsion (GradVnn, src/grad.c:43)
  if (terms & SQB200_GRAD_NUCLEAR)
  for (int i = 0; i < natom; ++i)
    for (int j = 0; j < natom; ++j) {
      if (i == j) continue;
      const double dx = axyz[3 * i] - axyz[3 * j], dy = axyz[3 * i + 1] - axyz[3 * j + 1], dz = axyz[3 * i + 2] - axyz[3 * j + 2];
      const double r = sqrt(dx * dx + dy * dy + dz * dz), f = -Z[i] * Z[j] / (r * r * r);
      grad[3 * i] += f * dx; grad[3 * i + 1] += f * dy; grad[3 * i + 2] += f * dz;
    }
  return SQB200_OK;
}

extern "C" int sqb200_gradient(sqb200_jk* c, int natom, const double* Z, const double* axyz, const double* PA,
                               const double* PB, const double* W, double* grad) {
  return sqb200_gradient_terms(c, natom, Z, axyz, PA, PB, W, SQB200_GRAD_ALL, grad);
}
