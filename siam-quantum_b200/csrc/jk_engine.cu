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
  std::vector<sqb::PairRec> pairs;   // sorted by decreasing Schwarz bound
  std::vector<double> prims;
  sqb::PairRec* d_pairs = nullptr;
  double* d_prims = nullptr;
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
  struct Work {
    std::vector<int> kernel;      // class-kernel index per segment
    std::vector<int> first, count;
    sqb::WorkItem* d_items = nullptr;
    int total = 0;
  };
  std::map<std::pair<double, double>, Work> work;
  std::vector<long long> last_counts;
  long long last_flops = 0;
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
  struct Tmp { double s; int P, Q; };
  std::vector<Tmp> lists[sqb::kNumPairClasses];
  for (int P = 0; P < ns; ++P)
    for (int Q = 0; Q <= P; ++Q) {
      const int k = pair_class_of(sh[P].type, sh[Q].type);
      lists[k].push_back({sch(P, Q), P, Q});
    }
  for (int k = 0; k < sqb::kNumPairClasses; ++k) {
    PairClass& pc = c->cls[k];
    std::stable_sort(lists[k].begin(), lists[k].end(), [](const Tmp& a, const Tmp& b) { return a.s > b.s; });
    if (lists[k].empty()) continue;
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

int upload_pairs(sqb200_jk* c) {
  for (int k = 0; k < sqb::kNumPairClasses; ++k) {
    PairClass& pc = c->cls[k];
    if (pc.pairs.empty()) continue;
    CUDA_OK(cudaMalloc(&pc.d_pairs, pc.pairs.size() * sizeof(sqb::PairRec)));
    CUDA_OK(cudaMalloc(&pc.d_prims, pc.prims.size() * sizeof(double)));
    CUDA_OK(cudaMemcpy(pc.d_pairs, pc.pairs.data(), pc.pairs.size() * sizeof(sqb::PairRec), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(pc.d_prims, pc.prims.data(), pc.prims.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  return SQB200_OK;
}

// Work list: per class kernel, one item per (bra pair, <=128 ket pairs).
int build_work(sqb200_jk* c, double outer, double fixed, sqb200_jk::Work** out) {
  auto key = std::make_pair(outer, fixed);
  auto it = c->work.find(key);
  if (it != c->work.end()) {
    *out = &it->second;
    return SQB200_OK;
  }
  sqb200_jk::Work w;
  std::vector<sqb::WorkItem> items;
  const double cut = std::max(outer, fixed);
  for (int ki = 0; ki < sqb::kNumClassKernels; ++ki) {
    const sqb::ClassKernel& K = sqb::kClassKernels[ki];
    const PairClass& B = c->cls[K.bra_cls];
    const PairClass& T = c->cls[K.ket_cls];
    if (B.pairs.empty() || T.pairs.empty()) continue;
    const int first = (int)items.size();
    const bool same = K.bra_cls == K.ket_cls;
    for (int b = 0; b < (int)B.pairs.size(); ++b) {
      const double sb = B.pairs[b].schwarz;
      if (!(sb > 0.0)) break;   // sorted: the rest are zero
      const double thr = cut / sb * (1.0 - 1e-12);
      // ket pairs with schwarz >= thr form a prefix of the sorted class
      int lo = 0, hi = (int)T.pairs.size();
      while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (T.pairs[mid].schwarz >= thr) lo = mid + 1; else hi = mid;
      }
      const int end = lo;
      const int start = same ? b : 0;
      for (int k0 = start; k0 < end; k0 += 128) items.push_back({b, k0, std::min(128, end - k0), 0});
    }
    const int cnt = (int)items.size() - first;
    if (cnt > 0) {
      w.kernel.push_back(ki);
      w.first.push_back(first);
      w.count.push_back(cnt);
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
  CUDA_OK(cudaMemsetAsync(c->d_counters, 0, sizeof(unsigned long long) * 3 * sqb::kNumClassKernels, st));
  for (size_t s = 0; s < w->kernel.size(); ++s) {
    const sqb::ClassKernel& K = sqb::kClassKernels[w->kernel[s]];
    const PairClass& B = c->cls[K.bra_cls];
    const PairClass& T = c->cls[K.ket_cls];
    sqb::JKArgs a;
    memset(&a, 0, sizeof(a));
    a.bra_pairs = B.d_pairs; a.bra_prims = B.d_prims;
    a.ket_pairs = T.d_pairs; a.ket_prims = T.d_prims;
    a.PA = dPA; a.PB = dPB; a.PT = c->d_PT; a.PM = c->d_PM;
    a.Jacc = c->d_J; a.KAacc = c->d_KA; a.KBacc = c->d_KB;
    a.boys_tab = c->d_boys;
    a.counters = c->d_counters + 3 * w->kernel[s];
    a.nbf = n; a.ns = c->ns;
    a.same_class = K.bra_cls == K.ket_cls;
    a.cut_outer = outer; a.cut_fixed = fixed; a.dscreen_rmax = dscreen;
    const sqb::WorkItem* items = w->d_items + w->first[s];
    void* args[] = {&a, &items};
    const size_t smem = (size_t)B.max_nprim * B.stride * sizeof(double);
    const void* fn = uhf ? K.fn_u : K.fn_r;
    if (smem > 48 * 1024) CUDA_OK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CUDA_OK(cudaLaunchKernel(fn, dim3(w->count[s]), dim3(128), args, smem, st));
  }
  k_finalize<<<grid_for(nn, 256), 256, 0, st>>>(c->d_J, c->d_KA, c->d_KB, dJT, dKA, dKB, n, uhf);
  CUDA_OK(cudaGetLastError());
  return SQB200_OK;
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
  c->nbf = nbf;
  int rc = build_shells(nbf, nprim, lmn, xyz, exps, ncoefs, c->shells);
  if (rc) { delete c; return rc; }
  c->ns = (int)c->shells.size();
  if (schwarz) {
    c->schwarz.assign(schwarz, schwarz + (size_t)nbf * nbf);
  } else {
    delete c;
    return fail(SQB200_EINVAL, "device Schwarz not yet available: pass the Schwarz matrix");
  }
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
  ALLOC(c->d_counters, 3 * sqb::kNumClassKernels * sizeof(unsigned long long));
#undef ALLOC
  cudaError_t e = cudaMemcpy(c->d_boys, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(c->d_shfirst, fst.data(), c->ns * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(c->d_shn, nf.data(), c->ns * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { sqb200_jk_destroy(c); return fail(SQB200_ECUDA, cudaGetErrorString(e)); }
  *out = c;
  return SQB200_OK;
}

int sqb200_jk_destroy(sqb200_jk* c) {
  if (!c) return SQB200_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& kv : c->work) cudaFree(kv.second.d_items);
  for (int k = 0; k < sqb::kNumPairClasses; ++k) { cudaFree(c->cls[k].d_pairs); cudaFree(c->cls[k].d_prims); }
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
  std::vector<unsigned long long> h(3 * sqb::kNumClassKernels);
  CUDA_OK(cudaMemcpy(h.data(), c->d_counters, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  long long q = 0, pq = 0, fl = 0;
  for (int k = 0; k < sqb::kNumClassKernels; ++k) {
    const sqb::ClassKernel& K = sqb::kClassKernels[k];
    q += (long long)h[3 * k];
    pq += (long long)h[3 * k + 1];
    fl += (long long)h[3 * k + 1] * K.flops_prim + (long long)h[3 * k + 2] * K.flops_flush +
          (long long)h[3 * k] * K.flops_quartet;
  }
  long long v[5] = {q, pq, fl, (long long)c->ns, 0};
  for (int k = 0; k < sqb::kNumPairClasses; ++k) v[4] += (long long)c->cls[k].pairs.size();
  for (int i = 0; i < n && i < 5; ++i) out[i] = v[i];
  return SQB200_OK;
}

int sqb200_jk_schwarz(sqb200_jk* c, double* S) {
  if (!c || !S) return fail(SQB200_EINVAL, "null argument");
  return fail(SQB200_EINVAL, "device Schwarz not yet available");
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
